"""The oracle's pressure solver pinned on the CPU against plain-Python
restatements that follow the reference statement by statement, in the same
loop orders and the same operation order (IEEE doubles):

* applyCompressedMatrix (FluidSim/src/cpu/project-solver.cc:16-39);
* ModifiedIncompleteCholesky3D::precond (project-solver.cc:230-306): the pivot
  pass with its divide-by-E^2 tau terms, the Adiag != 0 guards and the sigma
  fallback, then the forward and the reversed backward sweep;
* CgSolver3D::solve (project-solver.cc:308-346) with dotProduct, saxpy,
  scaleAndAdd and LinfNorm (util.cc:380-410, util.h:56-63): zero start,
  absolute L-inf stop, `iter` from 1, the first preconditioner applied to rhs;
* FvmSolver3D::buildSystem (project-solver.cc:59-228) with fractionInside
  (util.cc:319-378) and SDF<3>::eval (sdf.h:35-60, whose node weights are the
  mirror of trilinear): face weights, theta clamps, ghost-fluid diagonals,
  the right-hand side, and the `j < width - 1` bound of the up face;
* FvmSolver3D::project (project-solver.cc:348-435): fluid-fluid faces, the
  ghost-fluid faces on either side, walls.

The reference ships no test or fixture for these functions and cannot be built
here, so this second, independent restatement is what catches a transcription
error in the C oracle.  Systems: the buildSystem sphere-pool system, a random
symmetric system with zero diagonals on some active cells, and a large dt/h
where the sigma fallback fires on most cells."""
import math

import numpy as np
import pytest

from helpers import poisson_system

LEFT, RIGHT, UP, DOWN, FRONT, BACK = range(6)  # Directions (project-solver.cc:7-14)


def literal_apply(adiag, an, x, active):
    W, H, D = adiag.shape
    b = np.zeros_like(adiag)
    for i in range(W):
        for j in range(H):
            for k in range(D):
                if not active[i, j, k]:
                    continue
                t = adiag[i, j, k] * x[i, j, k]
                if i > 0 and active[i - 1, j, k]:
                    t += an[LEFT][i, j, k] * x[i - 1, j, k]
                if j > 0 and active[i, j - 1, k]:
                    t += an[DOWN][i, j, k] * x[i, j - 1, k]
                if k > 0 and active[i, j, k - 1]:
                    t += an[BACK][i, j, k] * x[i, j, k - 1]
                if i < W - 1 and active[i + 1, j, k]:
                    t += an[RIGHT][i, j, k] * x[i + 1, j, k]
                if j < H - 1 and active[i, j + 1, k]:
                    t += an[UP][i, j, k] * x[i, j + 1, k]
                if k < D - 1 and active[i, j, k + 1]:
                    t += an[FRONT][i, j, k] * x[i, j, k + 1]
                b[i, j, k] = t
    return b


def literal_precond(adiag, an, r, active, tau, sigma, z=None):
    W, H, D = adiag.shape
    A, L, Dn, Bk = adiag.tolist(), an[LEFT].tolist(), an[DOWN].tolist(), an[BACK].tolist()
    act = active.tolist()
    E = [[[0.0] * D for _ in range(H)] for _ in range(W)]
    for i in range(W):
        for j in range(H):
            for k in range(D):
                if not act[i][j][k]:
                    continue
                e = A[i][j][k]
                if e == 0.0:
                    continue
                if i > 0 and act[i - 1][j][k] and A[i - 1][j][k] != 0.0:
                    e -= (L[i][j][k] * E[i - 1][j][k]) * (L[i][j][k] * E[i - 1][j][k])
                    if j < H - 1 and act[i - 1][j + 1][k]:
                        e -= tau * L[i][j][k] * L[i - 1][j + 1][k] / (E[i - 1][j][k] * E[i - 1][j][k])
                    if k < D - 1 and act[i - 1][j][k + 1]:
                        e -= tau * L[i][j][k] * L[i - 1][j][k + 1] / (E[i - 1][j][k] * E[i - 1][j][k])
                if j > 0 and act[i][j - 1][k] and A[i][j - 1][k] != 0.0:
                    e -= (Dn[i][j][k] * E[i][j - 1][k]) * (Dn[i][j][k] * E[i][j - 1][k])
                    if i < W - 1 and act[i + 1][j - 1][k]:
                        e -= tau * Dn[i][j][k] * Dn[i + 1][j - 1][k] / (E[i][j - 1][k] * E[i][j - 1][k])
                    if k < D - 1 and act[i][j - 1][k + 1]:
                        e -= tau * Dn[i][j][k] * Dn[i][j - 1][k + 1] / (E[i][j - 1][k] * E[i][j - 1][k])
                if k > 0 and act[i][j][k - 1] and A[i][j][k - 1] != 0.0:
                    e -= (Bk[i][j][k] * E[i][j][k - 1]) * (Bk[i][j][k] * E[i][j][k - 1])
                    if i < W - 1 and act[i + 1][j][k - 1]:
                        e -= tau * Bk[i][j][k] * Bk[i + 1][j][k - 1] / (E[i][j][k - 1] * E[i][j][k - 1])
                    if j < H - 1 and act[i][j + 1][k - 1]:
                        e -= tau * Bk[i][j][k] * Bk[i][j + 1][k - 1] / (E[i][j][k - 1] * E[i][j][k - 1])
                if e < sigma * A[i][j][k]:
                    e = A[i][j][k]
                E[i][j][k] = 1.0 / math.sqrt(e)
    R = r.tolist()
    q = [[[0.0] * D for _ in range(H)] for _ in range(W)]
    for i in range(W):
        for j in range(H):
            for k in range(D):
                if not act[i][j][k]:
                    continue
                t = R[i][j][k]
                if i > 0 and act[i - 1][j][k]:
                    t -= L[i][j][k] * E[i - 1][j][k] * q[i - 1][j][k]
                if j > 0 and act[i][j - 1][k]:
                    t -= Dn[i][j][k] * E[i][j - 1][k] * q[i][j - 1][k]
                if k > 0 and act[i][j][k - 1]:
                    t -= Bk[i][j][k] * E[i][j][k - 1] * q[i][j][k - 1]
                q[i][j][k] = t * E[i][j][k]
    zz = z.tolist() if z is not None else [[[0.0] * D for _ in range(H)] for _ in range(W)]
    for i in range(W - 1, -1, -1):
        for j in range(H - 1, -1, -1):
            for k in range(D - 1, -1, -1):
                if not act[i][j][k]:
                    continue
                t = q[i][j][k]
                if i < W - 1 and act[i + 1][j][k]:
                    t -= L[i + 1][j][k] * E[i][j][k] * zz[i + 1][j][k]
                if j < H - 1 and act[i][j + 1][k]:
                    t -= Dn[i][j + 1][k] * E[i][j][k] * zz[i][j + 1][k]
                if k < D - 1 and act[i][j][k + 1]:
                    t -= Bk[i][j][k + 1] * E[i][j][k] * zz[i][j][k + 1]
                zz[i][j][k] = t * E[i][j][k]
    return np.array(zz), np.array(E), np.array(q)


def literal_pcg(adiag, an, rhs, active, tol, max_iter, tau, sigma):
    act = active.astype(bool)
    flat = act.ravel()  # the loops below run in the arrays' x, y, z order, as forEach

    def dot(a, b):
        s = 0.0
        for x, y in zip(a.ravel()[flat].tolist(), b.ravel()[flat].tolist()):
            s += x * y
        return s

    def linf(a):
        m = 0.0
        for v in a.ravel()[flat].tolist():
            m = max(m, abs(v))
        return m

    pg = np.zeros_like(adiag)
    r = rhs.copy()
    residual = linf(r)
    if residual < tol:
        return pg, residual, 0
    z, _, _ = literal_precond(adiag, an, rhs, active, tau, sigma)
    s = z.copy()
    sig = dot(z, r)
    it = 1
    while it < max_iter:
        z = np.where(act, literal_apply(adiag, an, s, active), z)
        sdotz = dot(s, z)
        alpha = sig / sdotz
        pg = np.where(act, pg + alpha * s, pg)  # saxpy: a += x b
        r = np.where(act, r + (-alpha) * z, r)
        residual = linf(r)
        if residual < tol:
            break
        z, _, _ = literal_precond(adiag, an, r, active, tau, sigma, z)
        sig_new = dot(z, r)
        beta = sig_new / sig
        s = np.where(act, z + beta * s, s)  # scaleAndAdd: c = a + x c
        sig = sig_new
        it += 1
    return pg, residual, it


def random_symmetric(dims, seed):
    rng = np.random.default_rng(seed)
    active = (rng.random(dims) < 0.8).astype(np.uint8)
    an = [np.zeros(dims) for _ in range(6)]
    cx = -rng.uniform(0.1, 1.0, (dims[0] - 1, dims[1], dims[2]))
    cy = -rng.uniform(0.1, 1.0, (dims[0], dims[1] - 1, dims[2]))
    cz = -rng.uniform(0.1, 1.0, (dims[0], dims[1], dims[2] - 1))
    an[RIGHT][:-1], an[LEFT][1:] = cx, cx
    an[UP][:, :-1], an[DOWN][:, 1:] = cy, cy
    an[FRONT][:, :, :-1], an[BACK][:, :, 1:] = cz, cz
    adiag = 6.0 + rng.uniform(0.0, 1.0, dims)
    zero = (rng.random(dims) < 0.05) & (active > 0)
    adiag[zero] = 0.0
    rhs = rng.uniform(-1, 1, dims)
    return dict(adiag=adiag, an=an, rhs=rhs, active=active)


def systems(oracle):
    yield "sphere_pool", poisson_system(oracle, 9, seed=4, dims=(9, 7, 8))
    yield "random_zero_diag", random_symmetric((7, 6, 8), 9)
    yield "large_dt", poisson_system(oracle, 8, seed=5, dims=(8, 8, 7), dt_over_h=2.0)


@pytest.mark.parametrize("name", ["sphere_pool", "random_zero_diag", "large_dt"])
def test_apply_and_precond_equal_literal(oracle, name):
    S = dict(systems(oracle))[name]
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, S["adiag"].shape)
    b = oracle.apply_matrix(S["adiag"], S["an"], x, S["active"])
    assert np.array_equal(b, literal_apply(S["adiag"], S["an"], x, S["active"]))
    z, E, q = oracle.mic_precond(S["adiag"], S["an"], x, S["active"], return_scratch=True)
    lz, lE, lq = literal_precond(S["adiag"], S["an"], x, S["active"], 0.97, 0.25)
    act = S["active"] > 0
    assert np.array_equal(E[act], lE[act]) and np.array_equal(q[act], lq[act]) and np.array_equal(z[act], lz[act])
    if name == "random_zero_diag":
        assert (lE[act & (S["adiag"] == 0)] == 0).all() and (act & (S["adiag"] == 0)).any()


def test_sigma_fallback_fires_at_large_dt(oracle):
    """At dt/h = 2 the modified pivot falls below sigma Adiag on most active
    cells and the reference falls back to Adiag there."""
    S = dict(systems(oracle))["large_dt"]
    _, E, _ = literal_precond(S["adiag"], S["an"], np.zeros_like(S["adiag"]), S["active"], 0.97, 0.25)
    act = (S["active"] > 0) & (S["adiag"] != 0)
    fell_back = np.isclose(E[act], 1.0 / np.sqrt(S["adiag"][act]), rtol=0, atol=0)
    assert fell_back.mean() > 0.5


@pytest.mark.parametrize("name", ["sphere_pool", "large_dt"])
def test_pcg_equals_literal(oracle, name):
    S = dict(systems(oracle))[name]
    pg, res, it = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-6, max_iter=300)
    lpg, lres, lit = literal_pcg(S["adiag"], S["an"], S["rhs"], S["active"], 1e-6, 300, 0.97, 0.25)
    act = S["active"] > 0
    assert it == lit and res == lres and it > 1
    assert np.array_equal(pg[act], lpg[act])


# --- buildSystem (project-solver.cc:59-228), SDF::eval (sdf.h:35-60),
# --- fractionInside (util.cc:319-378)

def literal_eval(grid, h, p):
    """SDF<3>::eval on a cell-centred grid with origin 0: node (x, y, z) takes
    the weight tx ty tz (the mirror of trilinear), as the reference."""
    W, H, D = grid.shape
    ix, iy, iz = (int(c / h - 0.5) for c in p)  # Vec3i(...) truncates toward zero

    def clamp(a, lo, hi):
        return lo if a < lo else (hi if a > hi else a)

    x, y, z = clamp(ix, 0, W - 1), clamp(iy, 0, H - 1), clamp(iz, 0, D - 1)
    xn, yn, zn = clamp(ix + 1, 0, W - 1), clamp(iy + 1, 0, H - 1), clamp(iz + 1, 0, D - 1)
    pos = ((x + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h)
    tx = clamp((p[0] - pos[0]) / h, 0.0, 1.0)
    ty = clamp((p[1] - pos[1]) / h, 0.0, 1.0)
    tz = clamp((p[2] - pos[2]) / h, 0.0, 1.0)
    g = grid
    return (tx * ty * tz * g[x, y, z] + tx * ty * (1 - tz) * g[x, y, zn] + tx * (1 - ty) * tz * g[x, yn, z] +
            tx * (1 - ty) * (1 - tz) * g[x, yn, zn] + (1 - tx) * ty * tz * g[xn, y, z] +
            (1 - tx) * ty * (1 - tz) * g[xn, y, zn] + (1 - tx) * (1 - ty) * tz * g[xn, yn, z] +
            (1 - tx) * (1 - ty) * (1 - tz) * g[xn, yn, zn])


def literal_fraction_inside(lu, ru, rd, ld):
    n = int(lu <= 0.0) + int(ru <= 0.0) + int(rd <= 0.0) + int(ld <= 0.0)  # numpy bools would OR
    if n == 0:
        return 0.0
    if n == 4:
        return 1.0
    while lu > 0.0:
        lu, ru, rd, ld = ld, lu, ru, rd  # cycle
    if n == 1:
        fracu = ru / (ru - lu)
        fracl = ld / (ld - lu)
        return fracu * fracl * 0.5
    if n == 2:
        if ru <= 0.0:
            return 0.5 * (ld / (ld - lu) + rd / (rd - ru))
        if ld <= 0.0:
            return 0.5 * (ru / (ru - lu) + rd / (rd - ld))
        if rd <= 0.0:
            fracu = ru / (ru - lu)
            fracd = ld / (ld - rd)
            fracl = ld / (ld - lu)
            fracr = ru / (ru - rd)
            if lu + ru + rd + ld <= 0.0:
                return 1.0 - 0.5 * ((1.0 - fracu) * (1.0 - fracl) + (1.0 - fracd) * (1.0 - fracr))
            return 0.5 * (fracu * fracl + fracd * fracr)
    while lu <= 0.0:
        lu, ru, rd, ld = ld, lu, ru, rd
    fracu = ru / (ru - lu)
    fracl = ld / (ld - lu)
    return 1.0 - 0.5 * fracu * fracl


def literal_build_system(dims, h, dt, u, v, w, F, C):
    nx, ny, nz = dims
    uw, vw, ww = np.zeros((nx + 1, ny, nz)), np.zeros((nx, ny + 1, nz)), np.zeros((nx, ny, nz + 1))
    hh = 0.5 * h
    for i in range(nx + 1):
        for j in range(ny):
            for k in range(nz):
                if i == 0 or i == nx or (F[i - 1, j, k] > 0.0 and F[i, j, k] > 0.0):
                    continue
                p = (i * h, (j + 0.5) * h, (k + 0.5) * h)
                bu = literal_eval(C, h, (p[0] + 0.0, p[1] + hh, p[2] - hh))
                bd = literal_eval(C, h, (p[0] + 0.0, p[1] - hh, p[2] - hh))
                fd = literal_eval(C, h, (p[0] + 0.0, p[1] - hh, p[2] + hh))
                fu = literal_eval(C, h, (p[0] + 0.0, p[1] + hh, p[2] + hh))
                uw[i, j, k] = 1.0 - literal_fraction_inside(bu, bd, fd, fu)
    for i in range(nx):
        for j in range(ny + 1):
            for k in range(nz):
                if j == 0 or j == ny or (F[i, j - 1, k] > 0.0 and F[i, j, k] > 0.0):
                    continue
                p = ((i + 0.5) * h, j * h, (k + 0.5) * h)
                lb = literal_eval(C, h, (p[0] - hh, p[1] + 0.0, p[2] - hh))
                rb = literal_eval(C, h, (p[0] + hh, p[1] + 0.0, p[2] - hh))
                rf = literal_eval(C, h, (p[0] + hh, p[1] + 0.0, p[2] + hh))
                lf = literal_eval(C, h, (p[0] - hh, p[1] + 0.0, p[2] + hh))
                vw[i, j, k] = 1.0 - literal_fraction_inside(lb, rb, rf, lf)
    for i in range(nx):
        for j in range(ny):
            for k in range(nz + 1):
                if k == 0 or k == nz or (F[i, j, k - 1] > 0.0 and F[i, j, k] > 0.0):
                    continue
                p = ((i + 0.5) * h, (j + 0.5) * h, k * h)
                ld = literal_eval(C, h, (p[0] - hh, p[1] - hh, p[2] + 0.0))
                lu = literal_eval(C, h, (p[0] - hh, p[1] + hh, p[2] + 0.0))
                ru = literal_eval(C, h, (p[0] + hh, p[1] + hh, p[2] + 0.0))
                rd = literal_eval(C, h, (p[0] + hh, p[1] - hh, p[2] + 0.0))
                ww[i, j, k] = 1.0 - literal_fraction_inside(ld, lu, ru, rd)
    adiag = np.zeros(dims)
    an = [np.zeros(dims) for _ in range(6)]
    rhs = np.zeros(dims)
    active = np.zeros(dims, np.uint8)
    factor = dt / h
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                if (uw[i, j, k] == 0.0 and uw[i + 1, j, k] == 0.0 and vw[i, j, k] == 0.0 and vw[i, j + 1, k] == 0.0
                        and ww[i, j, k] == 0.0 and ww[i, j, k + 1] == 0.0):
                    continue
                if F[i, j, k] > 0.0:
                    continue
                active[i, j, k] = 1
                sd = F[i, j, k]
                a = 0.0
                if i > 0:
                    if F[i - 1, j, k] > 0.0:
                        th = min(F[i - 1, j, k] / (F[i - 1, j, k] - sd), 0.99)
                        a += uw[i, j, k] * factor / (1.0 - th)
                    else:
                        a += uw[i, j, k] * factor
                        an[LEFT][i, j, k] -= uw[i, j, k] * factor
                    rhs[i, j, k] += uw[i, j, k] * u[i, j, k]
                if i < nx - 1:
                    if F[i + 1, j, k] > 0.0:
                        th = max(sd / (sd - F[i + 1, j, k]), 0.01)
                        a += uw[i + 1, j, k] * factor / th
                    else:
                        a += uw[i + 1, j, k] * factor
                        an[RIGHT][i, j, k] -= uw[i + 1, j, k] * factor
                    rhs[i, j, k] -= uw[i + 1, j, k] * u[i + 1, j, k]
                if j > 0:
                    if F[i, j - 1, k] > 0.0:
                        th = min(F[i, j - 1, k] / (F[i, j - 1, k] - sd), 0.99)
                        a += vw[i, j, k] * factor / (1.0 - th)
                    else:
                        a += vw[i, j, k] * factor
                        an[DOWN][i, j, k] -= vw[i, j, k] * factor
                    rhs[i, j, k] += vw[i, j, k] * v[i, j, k]
                if j < nx - 1:  # the reference bounds `up` by the width (:186)
                    if F[i, j + 1, k] > 0.0:
                        th = max(sd / (sd - F[i, j + 1, k]), 0.01)
                        a += vw[i, j + 1, k] * factor / th
                    else:
                        a += vw[i, j + 1, k] * factor
                        an[UP][i, j, k] -= vw[i, j + 1, k] * factor
                    rhs[i, j, k] -= vw[i, j + 1, k] * v[i, j + 1, k]
                if k > 0:
                    if F[i, j, k - 1] > 0.0:
                        th = min(F[i, j, k - 1] / (F[i, j, k - 1] - sd), 0.99)
                        a += ww[i, j, k] * factor / (1.0 - th)
                    else:
                        a += ww[i, j, k] * factor
                        an[BACK][i, j, k] -= ww[i, j, k] * factor
                    rhs[i, j, k] += ww[i, j, k] * w[i, j, k]
                if k < nz - 1:
                    if F[i, j, k + 1] > 0.0:
                        th = max(sd / (sd - F[i, j, k + 1]), 0.01)
                        a += ww[i, j, k + 1] * factor / th
                    else:
                        a += ww[i, j, k + 1] * factor
                        an[FRONT][i, j, k] -= ww[i, j, k + 1] * factor
                    rhs[i, j, k] -= ww[i, j, k + 1] * w[i, j, k + 1]
                adiag[i, j, k] = a
    return dict(adiag=adiag, an=an, rhs=rhs, active=active, uwt=uw, vwt=vw, wwt=ww)


@pytest.mark.parametrize("case", ["empty_collider", "sphere_collider", "narrow_x"])
def test_build_system_equals_literal(oracle, case):
    dims = (6, 9, 7) if case == "narrow_x" else (8, 8, 7)
    h = 1.0 / 8
    dt = 0.3 * h
    rng = np.random.default_rng(17)
    x = [(np.arange(n) + 0.5) * h for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    F = np.minimum(np.sqrt((X - 0.45) ** 2 + (Y - 0.4) ** 2 + (Z - 0.5) ** 2) - 0.33, Y - 0.3)
    nx, ny, nz = dims
    u, v, w = rng.uniform(-1, 1, (nx + 1, ny, nz)), rng.uniform(-1, 1, (nx, ny + 1, nz)), rng.uniform(-1, 1, (nx, ny, nz + 1))
    if case == "sphere_collider":
        C = np.sqrt((X - 0.6) ** 2 + (Y - 0.35) ** 2 + (Z - 0.45) ** 2) - 0.2
    else:
        C = np.full(dims, 1e9)
    got = oracle.build_system(dims, h, dt, u, v, w, F, C)
    ref = literal_build_system(dims, h, dt, u, v, w, F, C)
    for key in ("adiag", "rhs", "active", "uwt", "vwt", "wwt"):
        assert np.array_equal(got[key], ref[key]), key
    for d in range(6):
        assert np.array_equal(got["an"][d], ref["an"][d]), d
    assert ref["active"].any()
    if case == "sphere_collider":
        assert ((ref["uwt"] > 0) & (ref["uwt"] < 1)).any()  # partial faces


def test_fraction_inside_and_eval_equal_literal(oracle):
    rng = np.random.default_rng(23)
    for c in rng.uniform(-1, 1, (3000, 4)):
        assert oracle.fraction_inside(*c) == literal_fraction_inside(*c), c
    for c in rng.integers(-1, 2, (300, 4)).astype(np.float64):  # exact zeros on corners
        assert oracle.fraction_inside(*c) == literal_fraction_inside(*c), c
    h = 1.0 / 8
    g = rng.uniform(-1, 1, (8, 7, 9))
    for p in rng.uniform(-0.2, 1.2, (500, 3)):  # inside, and clamped outside the grid
        assert oracle.sdf_eval(g, h, p) == literal_eval(g, h, tuple(p)), p


# --- FvmSolver3D::project (project-solver.cc:348-435)

def literal_project(dims, h, dt, u, v, w, pg, F, uw, vw, ww):
    nx, ny, nz = dims
    u, v, w = u.copy(), v.copy(), w.copy()

    def face(vel, idx, wt, n_along, axis_i, lo_idx, hi_idx):
        if wt <= 0.0:
            return
        if axis_i == 0 or axis_i == n_along:
            vel[idx] = 0.0
            return
        sl, sr = F[lo_idx], F[hi_idx]
        if sl >= 0.0 and sr >= 0.0:
            return
        if sl < 0.0 and sr < 0.0:
            vel[idx] -= (pg[hi_idx] - pg[lo_idx]) * dt / h
            return
        if sl < 0.0:
            th = max(sl / (sl - sr), 0.01)
            vel[idx] += pg[lo_idx] * dt / h / th
        else:
            th = min(sl / (sl - sr), 0.99)
            vel[idx] -= pg[hi_idx] * dt / h / (1.0 - th)

    for i in range(nx + 1):
        for j in range(ny):
            for k in range(nz):
                face(u, (i, j, k), uw[i, j, k], nx, i, (i - 1, j, k), (i, j, k))
    for i in range(nx):
        for j in range(ny + 1):
            for k in range(nz):
                face(v, (i, j, k), vw[i, j, k], ny, j, (i, j - 1, k), (i, j, k))
    for i in range(nx):
        for j in range(ny):
            for k in range(nz + 1):
                face(w, (i, j, k), ww[i, j, k], nz, k, (i, j, k - 1), (i, j, k))
    return u, v, w


def test_project_equals_literal(oracle):
    dims = (8, 9, 7)
    h = 1.0 / 9
    dt = 0.4 * h
    rng = np.random.default_rng(29)
    x = [(np.arange(n) + 0.5) * h for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    F = np.minimum(np.sqrt((X - 0.4) ** 2 + (Y - 0.45) ** 2 + (Z - 0.4) ** 2) - 0.3, Y - 0.35)
    C = np.sqrt((X - 0.55) ** 2 + (Y - 0.3) ** 2 + (Z - 0.4) ** 2) - 0.17
    nx, ny, nz = dims
    u, v, w = rng.uniform(-1, 1, (nx + 1, ny, nz)), rng.uniform(-1, 1, (nx, ny + 1, nz)), rng.uniform(-1, 1, (nx, ny, nz + 1))
    S = oracle.build_system(dims, h, dt, u, v, w, F, C)
    pg = rng.uniform(-2, 2, dims)
    got = oracle.project(dims, h, dt, u, v, w, pg, F, S["uwt"], S["vwt"], S["wwt"])
    ref = literal_project(dims, h, dt, u, v, w, pg, F, S["uwt"], S["vwt"], S["wwt"])
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    # every branch is reached: fluid-fluid, both ghost sides, walls
    sl, sr = F[:-1], F[1:]
    assert ((sl < 0) & (sr < 0)).any() and ((sl < 0) & (sr >= 0)).any() and ((sl >= 0) & (sr < 0)).any()
