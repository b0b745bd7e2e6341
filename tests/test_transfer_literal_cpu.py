"""The oracle's particle-grid transfers pinned on the CPU against plain-Python
restatements that follow the reference statement by statement (IEEE doubles,
the same operation order):

* sampleVelocity (FluidSim/src/cpu/util.cc:40-85): per face grid the 4^3 nodes
  nearest + {-1..2} inside the grid, weights normalised by their sum, with
  nearest() (Spatify/include/Spatify/grids.h:287-292) truncating toward zero;
* FlipAdvectionSolver3D::solveG2P (advect-solver.cc:157-169) and the PIC form
  (advect-solver.cc:7-17);
* solveP2G (advect-solver.cc:188-271) in serial particle order: splat, weight
  sums, normalisation, validity, u_last;
* advect (advect-solver.cc:170-187): Ralston RK3 through sampleVelocity, then
  handleCollision (advect-solver.cc:100-137) with SDF<3>::grad
  (FluidSim/include/FluidSim/cpu/sdf.h:62-118: the mirrored trilinear blend of
  one-sided/central node gradients, unclamped weights) and the box clamp.

The transfer kernel CubicKernel::weight lives in a header missing from the
reference tree; both sides use the oracle's documented B-spline policy for it
(pinned separately), so these tests pin everything around the weight."""
import math

import numpy as np
import pytest


def _nearest(p, off, h):
    return tuple(int(((p[a] - 0.0) - off[a] * h) / h + 0.5) for a in range(3))


OFFSETS = ((0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0))


def literal_sample(oracle, p, h, grids):
    out = []
    for g, off in zip(grids, OFFSETS):
        idx = _nearest(p, off, h)
        s, ws = 0.0, 0.0
        for i in range(-1, 3):
            for j in range(-1, 3):
                for k in range(-1, 3):
                    n = (idx[0] + i, idx[1] + j, idx[2] + k)
                    if not all(0 <= n[a] < g.shape[a] for a in range(3)):
                        continue
                    pn = [(n[a] + off[a]) * h + 0.0 for a in range(3)]
                    wt = oracle.cubic_weight(h, [p[a] - pn[a] for a in range(3)])
                    s += g[n] * wt
                    ws += wt
        out.append(s / ws if ws > 0.0 else 0.0)
    return out


def literal_grad(C, h, p):
    W, H, D = C.shape

    def clamp(a, lo, hi):
        return lo if a < lo else (hi if a > hi else a)

    def node_grad(x, y, z):
        xn = x + 1 if x < W - 1 else x
        xp = x - 1 if x > 0 else x
        yn = y + 1 if y < H - 1 else y
        yp = y - 1 if y > 0 else y
        zn = z + 1 if z < D - 1 else z
        zp = z - 1 if z > 0 else z
        dx = 2 * h if 0 < x < W - 1 else h
        dy = 2 * h if 0 < y < H - 1 else h
        dz = 2 * h if 0 < z < D - 1 else h
        return ((C[xn, y, z] - C[xp, y, z]) / dx, (C[x, yn, z] - C[x, yp, z]) / dy, (C[x, y, zn] - C[x, y, zp]) / dz)

    ix, iy, iz = (int(c / h - 0.5) for c in p)
    x, y, z = clamp(ix, 0, W - 1), clamp(iy, 0, H - 1), clamp(iz, 0, D - 1)
    xn, yn, zn = clamp(ix + 1, 0, W - 1), clamp(iy + 1, 0, H - 1), clamp(iz + 1, 0, D - 1)
    tx = (p[0] - (x + 0.5) * h) / h
    ty = (p[1] - (y + 0.5) * h) / h
    tz = (p[2] - (z + 0.5) * h) / h
    terms = [(tx * ty * tz, (x, y, z)), (tx * ty * (1 - tz), (x, y, zn)), (tx * (1 - ty) * tz, (x, yn, z)),
             (tx * (1 - ty) * (1 - tz), (x, yn, zn)), ((1 - tx) * ty * tz, (xn, y, z)),
             ((1 - tx) * ty * (1 - tz), (xn, y, zn)), ((1 - tx) * (1 - ty) * tz, (xn, yn, z)),
             ((1 - tx) * (1 - ty) * (1 - tz), (xn, yn, zn))]
    g = None
    for wgt, node in terms:
        gn = node_grad(*node)
        t = [wgt * gn[a] for a in range(3)]
        g = t if g is None else [g[a] + t[a] for a in range(3)]
    return g


def _eval(C, h, p):
    from test_solver_literal_cpu import literal_eval

    return literal_eval(C, h, p)


def literal_collide(C, h, box, p, v, fired=None):
    p, v = list(p), list(v)
    if C is not None:
        d = _eval(C, h, tuple(p))
        if d < 0.0:
            if fired is not None:
                fired["collider"] += 1
            g = literal_grad(C, h, p)
            inv = 1.0 / math.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
            nrm = [g[a] * inv for a in range(3)]
            p = [p[a] - d * nrm[a] for a in range(3)]
            m = min(v[0] * nrm[0] + v[1] * nrm[1] + v[2] * nrm[2], 0.0)
            if fired is not None and m < 0.0:
                fired["inflow"] += 1
            v = [v[a] - m * nrm[a] for a in range(3)]
    for a in range(3):
        if fired is not None and (p[a] < 0.0 or p[a] > box[a]):
            fired["box"] += 1
        if p[a] < 0.0:
            p[a] = 0.0
            if v[a] < 0.0:
                v[a] = 0.0
        if p[a] > box[a]:
            p[a] = box[a]
            if v[a] > 0.0:
                v[a] = 0.0
    return p, v


def literal_advect(oracle, p, v, h, grids, C, box, dt, fired=None):
    k1 = list(v)
    p1 = [p[a] + 0.5 * dt * k1[a] for a in range(3)]
    k2 = literal_sample(oracle, p1, h, grids)
    p2 = [p[a] + 0.75 * dt * k2[a] for a in range(3)]
    k3 = literal_sample(oracle, p2, h, grids)
    q = [p[a] + 2.0 / 9.0 * dt * k1[a] + 1.0 / 3.0 * dt * k2[a] + 4.0 / 9.0 * dt * k3[a] for a in range(3)]
    return literal_collide(C, h, box, q, v, fired)


@pytest.fixture(scope="module")
def scene():
    dims = (7, 8, 6)
    h = 1.0 / 8
    rng = np.random.default_rng(41)
    nx, ny, nz = dims
    grids = (rng.uniform(-1, 1, (nx + 1, ny, nz)), rng.uniform(-1, 1, (nx, ny + 1, nz)),
             rng.uniform(-1, 1, (nx, ny, nz + 1)))
    last = tuple(g + rng.uniform(-0.2, 0.2, g.shape) for g in grids)
    ext = np.array(dims) * h
    pos = rng.uniform(-0.05, 1.05, (40, 3)) * ext  # some outside the box, some at the walls
    pos[:4] = [[0.0, 0.3, 0.2], [ext[0], 0.1, 0.1], [0.2, ext[1], 0.4], [0.1, 0.1, ext[2]]]
    vel = rng.uniform(-2, 2, (40, 3))
    x = [(np.arange(n) + 0.5) * h for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    C = np.sqrt((X - 0.45) ** 2 + (Y - 0.5) ** 2 + (Z - 0.35) ** 2) - 0.22
    return dict(dims=dims, h=h, grids=grids, last=last, pos=pos, vel=vel, C=C, box=tuple(n * h for n in dims))


def test_sample_velocity_equals_literal(oracle, scene):
    S = scene
    got = oracle.sample_velocity(S["pos"], S["dims"], S["h"], *S["grids"])
    for p, g in zip(S["pos"], got):
        assert list(g) == literal_sample(oracle, p, S["h"], S["grids"]), p


@pytest.mark.parametrize("alpha", [0.95, -1.0])
def test_g2p_equals_literal(oracle, scene, alpha):
    S = scene
    if alpha >= 0:
        got = oracle.g2p(S["pos"], S["vel"], S["dims"], S["h"], *S["grids"], *S["last"], alpha=alpha)
    else:
        got = oracle.g2p(S["pos"], S["vel"], S["dims"], S["h"], *S["grids"], alpha=alpha)
    for p, v, g in zip(S["pos"], S["vel"], got):
        pic = literal_sample(oracle, p, S["h"], S["grids"])
        if alpha < 0:
            ref = pic
        else:
            old = literal_sample(oracle, p, S["h"], S["last"])
            flip = [v[a] + pic[a] - old[a] for a in range(3)]
            ref = [alpha * flip[a] + (1.0 - alpha) * pic[a] for a in range(3)]
        assert list(g) == ref, p


@pytest.mark.parametrize("collider", [False, True])
def test_advect_and_collision_equal_literal(oracle, scene, collider):
    S = scene
    C = S["C"] if collider else None
    dt = 0.05
    rng = np.random.default_rng(47)
    centre = np.array([0.45, 0.5, 0.35])
    inside = centre + rng.uniform(-0.1, 0.1, (20, 3))  # in the collider sphere (radius 0.22)
    pos = np.concatenate([S["pos"], inside])
    vel = np.concatenate([S["vel"], (centre - inside) * 5.0])  # moving inward
    gp, gv = oracle.advect(pos, vel, S["dims"], S["h"], *S["grids"], C, dt)
    fired = {"collider": 0, "box": 0, "inflow": 0}
    for i, (p, v) in enumerate(zip(pos, vel)):
        rp, rv = literal_advect(oracle, p, v, S["h"], S["grids"], C, S["box"], dt, fired)
        assert list(gp[i]) == rp and list(gv[i]) == rv, i
    # the push-out and the removal of the inflowing velocity both ran
    assert fired["box"] > 0 and (fired["collider"] > 0) == collider and (fired["inflow"] > 0) == collider, fired


def literal_p2g(oracle, pos, vel, dims, h):
    """FlipAdvectionSolver3D::solveP2G (advect-solver.cc:188-271) with the
    particles taken in order (the reference's parallel loop races on shared
    nodes; serial order is the oracle's parity mode)."""
    nx, ny, nz = dims
    shapes = ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))
    g = [np.zeros(s) for s in shapes]
    wsum = [np.zeros(s) for s in shapes]
    for p, v in zip(pos.tolist(), vel.tolist()):
        idx = [_nearest(p, off, h) for off in OFFSETS]
        for i in range(-1, 3):
            for j in range(-1, 3):
                for k in range(-1, 3):
                    for a in range(3):
                        n = (idx[a][0] + i, idx[a][1] + j, idx[a][2] + k)
                        if not all(0 <= n[b] < shapes[a][b] for b in range(3)):
                            continue
                        pn = [(n[b] + OFFSETS[a][b]) * h + 0.0 for b in range(3)]
                        wt = oracle.cubic_weight(h, [p[b] - pn[b] for b in range(3)])
                        g[a][n] += v[a] * wt
                        wsum[a][n] += wt
    valid = []
    for a in range(3):
        pos_w = wsum[a] > 0.0
        g[a] = np.where(pos_w, g[a] / np.where(pos_w, wsum[a], 1.0), 0.0)
        valid.append(pos_w.astype(np.uint8))
    return g, wsum, valid


def test_p2g_equals_literal(oracle, scene):
    S = scene
    rng = np.random.default_rng(43)
    ext = np.array(S["dims"]) * S["h"]
    pos = rng.uniform(0.0, 1.0, (60, 3)) * ext * np.array([0.6, 1.0, 1.0])  # leaves empty faces
    vel = rng.uniform(-1, 1, (60, 3))
    got = oracle.p2g(pos, vel, S["dims"], S["h"], flip=True)
    g, wsum, valid = literal_p2g(oracle, pos, vel, S["dims"], S["h"])
    for a, c in enumerate("uvw"):
        assert np.array_equal(got[c], g[a]), c
        assert np.array_equal(got[c + "w"], wsum[a]), c
        assert np.array_equal(got[c + "valid"], valid[a]), c
        assert np.array_equal(got[c + "last"], g[a]), c  # u_last: the normalised grid itself
        assert valid[a].any() and not valid[a].all()
