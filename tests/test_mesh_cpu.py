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
