"""The oracle's pressure solver pinned on the CPU against plain-Python
restatements that follow the reference statement by statement, in the same
loop orders and the same operation order (IEEE doubles):

* applyCompressedMatrix (FluidSim/src/cpu/project-solver.cc:16-39);
* ModifiedIncompleteCholesky3D::precond (project-solver.cc:230-306): the pivot
  pass with its divide-by-E^2 tau terms, the Adiag != 0 guards and the sigma
  fallback, then the forward and the reversed backward sweep;
* CgSolver3D::solve (project-solver.cc:308-346) with dotProduct, saxpy,
  scaleAndAdd and LinfNorm (util.cc:380-410, util.h:56-63): zero start,
  absolute L-inf stop, `iter` from 1, the first preconditioner applied to rhs.

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
