"""The oracle's manifold2SDF (util.cc:203-310) pinned on the CPU.  The reference
ships no test or fixture for this function, so the pins are (1) a plain-Python
restatement of its point-triangle arithmetic (util.cc:87-125) evaluated over
every triangle where the exact band covers the whole grid, which the oracle
must equal bit for bit, and (2) geometric properties: true distances in the
band in exact-distance mode, the inside/outside sign of a closed mesh, and even
crossing counts per column."""
import math

import numpy as np
import pytest

from simcraft_b200 import scenes


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _mul(s, a):
    return (s * a[0], s * a[1], s * a[2])


def ref_dist(p, a, b, c, exact):
    """distancePointTriangle (util.cc:87-125), operation for operation; the
    reference adds the edge/face offsets (exact=False)."""
    pm = _sub if exact else _add
    ab, ac, ap = _sub(b, a), _sub(c, a), _sub(p, a)
    d1, d2 = _dot(ab, ap), _dot(ac, ap)
    if d1 <= 0 and d2 <= 0:
        return math.sqrt(_dot(ap, ap))
    bp = _sub(p, b)
    d3, d4 = _dot(ab, bp), _dot(ac, bp)
    if d3 >= 0 and d4 <= d3:
        return math.sqrt(_dot(bp, bp))
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        q = pm(ap, _mul(d1 / (d1 - d3), ab))
        return math.sqrt(_dot(q, q))
    cp = _sub(p, c)
    d5, d6 = _dot(ab, cp), _dot(ac, cp)
    if d6 >= 0 and d5 <= d6:
        return math.sqrt(_dot(cp, cp))
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        q = pm(ap, _mul(d2 / (d2 - d6), ac))
        return math.sqrt(_dot(q, q))
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        w = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        q = _add(bp, _mul(w, _sub(cp, bp)))
        return math.sqrt(_dot(q, q))
    denom = 1.0 / (va + vb + vc)
    q = pm(pm(ap, _mul(vb * denom, ab)), _mul(vc * denom, ac))
    return math.sqrt(_dot(q, q))


def _cells(dims, h, origin=(0.0, 0.0, 0.0)):
    for x in range(dims[0]):
        for y in range(dims[1]):
            for z in range(dims[2]):
                yield (x, y, z), ((x + 0.5) * h + origin[0], (y + 0.5) * h + origin[1], (z + 0.5) * h + origin[2])


@pytest.mark.parametrize("exact", [False, True])
def test_full_band_equals_restated_minimum(oracle, exact):
    """With the band covering the grid every cell sees every triangle exactly,
    so |sdf| is the minimum of the restated distance and `closest` the first
    triangle attaining it."""
    n = 12
    h = 1.0 / n
    v, t = scenes.box_mesh((0.27, 0.31, 0.22), (0.71, 0.66, 0.74))
    sdf, cl, _ = oracle.manifold_to_sdf(v, t, (n, n, n), h, exact_band=n, exact_distance=exact)
    tris = [tuple(tuple(v[k]) for k in tri) for tri in t]
    for (x, y, z), p in _cells((n, n, n), h):
        ds = [ref_dist(p, *tri, exact) for tri in tris]
        m = min(ds)
        assert abs(sdf[x, y, z]) == m, ((x, y, z), sdf[x, y, z], m)
        assert cl[x, y, z] == ds.index(m)


def test_reference_distance_overstates_faces(oracle):
    """The reference's face and AB/AC-edge distances add the offsets: inside a
    box they come out larger than the true distance, never smaller; the sign is
    the same in both modes."""
    n = 16
    h = 1.0 / n
    lo, hi = np.array([0.3, 0.3, 0.3]), np.array([0.7, 0.7, 0.7])
    v, t = scenes.box_mesh(lo, hi)
    ref, _, _ = oracle.manifold_to_sdf(v, t, (n, n, n), h)
    ex, cl, _ = oracle.manifold_to_sdf(v, t, (n, n, n), h, exact_distance=True)
    x = (np.arange(n) + 0.5) * h
    P = np.stack(np.meshgrid(x, x, x, indexing="ij"), -1)
    inside = ((P > lo) & (P < hi)).all(-1)
    assert ((ref < 0) == inside).all() and ((ex < 0) == inside).all()
    # exact mode: interior distance to the nearest face
    d_in = np.minimum(P - lo, hi - P).min(-1)
    np.testing.assert_allclose(-ex[inside], d_in[inside], rtol=0, atol=1e-12)
    assert (np.abs(ref) >= np.abs(ex) - 1e-15).all()
    assert (np.abs(ref) > np.abs(ex) + 0.1 * h).any()
    assert (cl >= 0).all()


def _pt_tri(p, a, b, c):
    """True point-triangle distance, vectorised (independent of the C code)."""
    ab, ac = b - a, c - a
    n = np.cross(ab, ac)
    n2 = n @ n
    ap = p - a
    w = (np.cross(ab, ap) @ n) / n2
    v = (np.cross(ap, ac) @ n) / n2
    inside = (v >= 0) & (w >= 0) & (v + w <= 1)
    d_in = np.linalg.norm(p - (a + np.outer(v, ab) + np.outer(w, ac)), axis=1)

    def seg(x, y):
        d = y - x
        s = np.clip(((p - x) @ d) / (d @ d), 0, 1)
        return np.linalg.norm(p - (x + np.outer(s, d)), axis=1)

    return np.where(inside, d_in, np.minimum(np.minimum(seg(a, b), seg(b, c)), seg(c, a)))


@pytest.mark.parametrize("band", [1, 3])
def test_exact_band_distances_equal_brute_force(oracle, band):
    n = 20
    h = 1.0 / n
    centre = np.array([0.52, 0.47, 0.5])
    v, t = scenes.icosphere(2, 0.27, centre)
    sdf, cl, _ = oracle.manifold_to_sdf(v, t, (n, n, n), h, exact_band=band, exact_distance=True)
    x = (np.arange(n) + 0.5) * h
    P = np.stack([a.ravel() for a in np.meshgrid(x, x, x, indexing="ij")], 1)
    brute = np.full(len(P), np.inf)
    for tri in t:
        brute = np.minimum(brute, _pt_tri(P, v[tri[0]], v[tri[1]], v[tri[2]]))
    brute = brute.reshape(n, n, n)
    near = brute < 0.5 * h  # within the band of the nearest triangle
    np.testing.assert_allclose(np.abs(sdf[near]), brute[near], rtol=0, atol=1e-12)
    assert (np.abs(sdf) >= brute - 1e-12).all()  # always a distance to some triangle
    r = np.linalg.norm(P - centre, axis=1).reshape(n, n, n)
    clear = np.abs(r - 0.27) > 0.05
    assert ((sdf < 0) == (r < 0.27))[clear].all()


def test_torus_with_origin_and_partial_grid(oracle):
    v, t = scenes.torus(16, 8, 0.3, 0.1, (0.5, 0.5, 0.5))
    dims, h, origin = (18, 14, 22), 1.0 / 18, (0.05, 0.1, -0.07)
    sdf, cl, icnt = oracle.manifold_to_sdf(v, t, dims, h, origin=origin)
    assert np.isfinite(sdf).all() and (cl >= 0).all()
    assert (sdf < 0).sum() > 0 and (sdf > 0).sum() > 0
    # each column crosses a closed surface an even number of times
    assert (icnt.sum(axis=2) % 2 == 0).all()


def test_empty_mesh(oracle):
    sdf, cl, icnt = oracle.manifold_to_sdf(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (4, 5, 6), 0.25)
    assert (sdf == 1e9).all() and (cl == -1).all() and not icnt.any()


def literal_manifold_to_sdf(v, t, dims, h, origin, exact_band):
    """manifold2SDF (util.cc:203-310) with checkNeighbour/sweep (:159-201),
    insideTraingle2D/solveEquations/calcBiocentricCoord (:128-157), statement
    by statement in plain Python floats, reference point-triangle distance."""
    W, H, D = dims
    ox, oy, oz = origin
    V = [tuple(float(c) for c in p) for p in v]
    T = [tuple(int(c) for c in tri) for tri in t]
    sdf = np.full(dims, 1e9)
    closest = np.full(dims, -1, np.int32)
    cnt = np.zeros(dims, np.int32)

    def clamp(a, lo, hi):
        return lo if a < lo else (hi if a > hi else a)

    def centre(x, y, z):
        return ((x + 0.5) * h + ox, (y + 0.5) * h + oy, (z + 0.5) * h + oz)

    def cross2(a, b):
        return a[0] * b[1] - b[0] * a[1]

    def inside2(p, a, b, c):
        ap, ab = (p[0] - a[0], p[1] - a[1]), (b[0] - a[0], b[1] - a[1])
        bp, bc = (p[0] - b[0], p[1] - b[1]), (c[0] - b[0], c[1] - b[1])
        cp, ca = (p[0] - c[0], p[1] - c[1]), (a[0] - c[0], a[1] - c[1])
        n = int(cross2(ap, ab) >= 0.0) + int(cross2(bp, bc) >= 0.0) + int(cross2(cp, ca) >= 0.0)
        return n == 3 or n == 0

    for i, (ia, ib, ic) in enumerate(T):
        a, b, c = V[ia], V[ib], V[ic]
        lo = [clamp(int(math.floor(min(min(a[q] - o, b[q] - o), c[q] - o) / h - 0.5)) - exact_band, 0, n - 1)
              for q, (o, n) in enumerate(zip(origin, dims))]
        hi = [clamp(int(math.ceil(max(max(a[q] - o, b[q] - o), c[q] - o) / h - 0.5)) + exact_band, 0, n - 1)
              for q, (o, n) in enumerate(zip(origin, dims))]
        for x in range(lo[0], hi[0] + 1):
            for y in range(lo[1], hi[1] + 1):
                for z in range(lo[2], hi[2] + 1):
                    d = ref_dist(centre(x, y, z), a, b, c, False)
                    if d < sdf[x, y, z]:
                        sdf[x, y, z] = d
                        closest[x, y, z] = i
        lo = [clamp(int(math.floor(min(min(a[q] - o, b[q] - o), c[q] - o) / h - 0.5)), 0, n - 1)
              for q, (o, n) in enumerate(zip(origin[:2], dims[:2]))]
        hi = [clamp(int(math.ceil(max(max(a[q] - o, b[q] - o), c[q] - o) / h - 0.5)), 0, n - 1)
              for q, (o, n) in enumerate(zip(origin[:2], dims[:2]))]
        for j in range(lo[0], hi[0] + 1):
            for k in range(lo[1], hi[1] + 1):
                orig = centre(j, k, -1)
                pp = (orig[0], orig[1])
                if not inside2(pp, a, b, c):
                    continue
                a1, b1, c1 = a[0] - c[0], b[0] - c[0], pp[0] - c[0]
                a2, b2, c2 = a[1] - c[1], b[1] - c[1], pp[1] - c[1]
                det = a1 * b2 - a2 * b1
                u = (c1 * b2 - c2 * b1) / det
                vv = (a1 * c2 - a2 * c1) / det
                w = 1.0 - u - vv
                inter_z = a[2] * u + b[2] * vv + c[2] * w
                l = int(math.ceil((inter_z - oz) / h - 0.5))
                if l < 0:
                    cnt[j, k, 0] += 1
                elif l < D:
                    cnt[j, k, l] += 1

    def check(dx, dy, dz, x, y, z):
        nx_, ny_, nz_ = x + dx, y + dy, z + dz
        if nx_ < 0 or nx_ >= W or ny_ < 0 or ny_ >= H or nz_ < 0 or nz_ >= D:
            return
        tri = closest[nx_, ny_, nz_]
        if tri == -1:
            return
        ia, ib, ic = T[tri]
        d1 = ref_dist(centre(x, y, z), V[ia], V[ib], V[ic], False)
        if abs(d1) < abs(sdf[x, y, z]):
            sdf[x, y, z] = d1
            closest[x, y, z] = tri

    def sweep(dx, dy, dz):
        xs = range(W - 1, -1, -1) if dx > 0 else range(W)
        ys = range(H - 1, -1, -1) if dy > 0 else range(H)
        zs = range(D - 1, -1, -1) if dz > 0 else range(D)
        for x in xs:
            for y in ys:
                for z in zs:
                    check(0, dy, dz, x, y, z)
                    check(dx, 0, dz, x, y, z)
                    check(dx, dy, 0, x, y, z)
                    check(0, 0, dz, x, y, z)
                    check(0, dy, 0, x, y, z)
                    check(dx, 0, 0, x, y, z)
                    check(dx, dy, dz, x, y, z)

    for _ in range(2):
        for dx, dy, dz in ((1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1),
                           (-1, -1, -1)):
            sweep(dx, dy, dz)
    for i in range(W):
        for j in range(H):
            tot = 0
            for k in range(D):
                tot += int(cnt[i, j, k])
                if tot & 1:
                    sdf[i, j, k] = -sdf[i, j, k]
    return sdf, closest, cnt


@pytest.mark.parametrize("case", ["icosphere_band1", "torus_origin"])
def test_manifold_to_sdf_equals_literal(oracle, case):
    if case == "icosphere_band1":
        v, t = scenes.icosphere(1, 0.3, (0.48, 0.52, 0.5))
        dims, h, origin, band = (10, 11, 9), 0.1, (0.0, 0.0, 0.0), 1
    else:
        v, t = scenes.torus(10, 6, 0.28, 0.1, (0.5, 0.5, 0.5))
        dims, h, origin, band = (11, 9, 10), 1.0 / 10, (0.03, 0.06, -0.02), 2
    sdf, cl, icnt = oracle.manifold_to_sdf(v, t, dims, h, origin=origin, exact_band=band)
    ls, lc, li = literal_manifold_to_sdf(v, t, dims, h, origin, band)
    assert np.array_equal(icnt, li)
    assert np.array_equal(cl, lc)
    assert np.array_equal(sdf, ls)
    assert (ls < 0).any() and (lc >= 0).all()
