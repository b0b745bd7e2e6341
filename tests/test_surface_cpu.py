"""The marching-cubes surface export (rebuildSurface,
FluidSim/src/cpu/rebuild-surface.cc:643-741) pinned on the CPU.

The reference ships no test or fixture for this function and cannot be built
here (glm and Core are missing), so the pins are:
(1) the case table: the library's packed table decodes to the reference's
    vertexOffset / edgeConnection / triangleConnectionTable3D, checked by
    SHA-256 digests generated from the reference source
    (tests/golden/make_mc_table_pin.py);
(2) a plain-Python restatement of singleCube / rebuildSurface that follows the
    reference statement by statement (hash map keyed by globalVertexIdx, evalSdf
    returning 1000 outside, the one-sided grad at the border), which the C
    oracle must equal bit for bit;
(3) geometric properties: a closed surface comes out watertight with Euler
    characteristic 2, its vertices lie on the sign-change edges, and its
    normals point outward."""
import json
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLE_H = os.path.join(ROOT, "simcraft_b200", "csrc", "sc_mc_table.h")


def decode_table():
    """(cases, corners, edges) decoded from the library's packed header."""
    text = open(TABLE_H).read()
    body = text[text.index("#define SC_MC_CASES_INIT"):]
    words = [int(w, 16) for w in re.findall(r"0x([0-9a-f]{16})ull", body)]
    assert len(words) == 256
    cases = [[(w >> (4 + 4 * i)) & 15 for i in range(w & 15)] for w in words]

    def macro_const(name):
        return int(re.search(r"#define %s\(c\) \(\((0x[0-9a-f]+) >>" % name, text).group(1), 16)

    mx, my, mz = (macro_const("SC_MC_CORNER_" + a) for a in "XYZ")
    corners = [((mx >> c) & 1, (my >> c) & 1, (mz >> c) & 1) for c in range(8)]
    ea = int(re.search(r"#define SC_MC_EDGE_A\(e\) \(\(int\)\(\((0x[0-9a-f]+)ull", text).group(1), 16)
    eb = int(re.search(r"#define SC_MC_EDGE_B\(e\) \(\(int\)\(\((0x[0-9a-f]+)ull", text).group(1), 16)
    edges = [((ea >> (4 * e)) & 15, (eb >> (4 * e)) & 15) for e in range(12)]
    return cases, corners, edges


CASES, CORNERS, EDGES = decode_table()


def test_table_digests_match_reference():
    import importlib.util

    spec = importlib.util.spec_from_file_location("mkpin", os.path.join(ROOT, "tests", "golden", "make_mc_table_pin.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    pin = json.load(open(os.path.join(ROOT, "tests", "golden", "mc_table_pin.json")))
    got = mk.digests(CASES, CORNERS, EDGES)
    for k in ("cases", "corners", "edges"):
        assert got[k] == pin[k], k


def test_table_cases_list_exactly_the_crossing_edges():
    for m, case in enumerate(CASES):
        assert len(case) % 3 == 0 and len(case) <= 15
        crossing = {e for e, (a, b) in enumerate(EDGES) if ((m >> a) & 1) != ((m >> b) & 1)}
        assert set(case) == crossing, m
        for t in range(0, len(case), 3):
            assert len(set(case[t:t + 3])) == 3
    # every edge runs along +x, +y or +z between two corners one apart
    for a, b in EDGES:
        d = [CORNERS[b][k] - CORNERS[a][k] for k in range(3)]
        assert sorted(d) == [0, 0, 1]


def literal_rebuild_surface(sdf, spacing, origin):
    """rebuildSurface / singleCube (rebuild-surface.cc:643-741), statement by
    statement, in plain Python floats (IEEE doubles, same operation order)."""
    W, H, D = sdf.shape
    hx, hy, hz = spacing
    ox, oy, oz = origin
    S = sdf.tolist()

    def eval_sdf(x, y, z):
        if x < 0 or x >= W or y < 0 or y >= H or z < 0 or z >= D:
            return 1000.0
        return S[x][y][z]

    def grad(x, y, z):
        xn = x + 1 if x < W else x
        xp = x - 1 if x > -1 else x
        yn = y + 1 if y < H else y
        yp = y - 1 if y > -1 else y
        zn = z + 1 if z < D else z
        zp = z - 1 if z > -1 else z
        dx = 2 * hx if (x > -1 and x < W - 1) else hx
        dy = 2 * hy if (y > -1 and y < H - 1) else hy
        dz = 2 * hz if (z > -1 and z < D - 1) else hz
        gx = eval_sdf(xn, y, z) - eval_sdf(xp, y, z)
        gy = eval_sdf(x, yn, z) - eval_sdf(x, yp, z)
        gz = eval_sdf(x, y, zn) - eval_sdf(x, y, zp)
        return (gx / dx, gy / dy, gz / dz)

    off3 = [(1, 0, 0), (2, 0, 1), (1, 0, 2), (0, 0, 1), (1, 2, 0), (2, 2, 1),
            (1, 2, 2), (0, 2, 1), (0, 1, 0), (2, 1, 0), (2, 1, 2), (0, 1, 2)]

    def global_vertex_idx(x, y, z, e):
        return (2 * (y + 1) + off3[e][1] + (2 * (x + 1) + off3[e][0]) * (2 * H + 3)) * (2 * D + 3) \
            + 2 * (z + 1) + off3[e][2]

    verts, norms, idx, vmap = [], [], [], {}
    for x in range(-1, W):
        for y in range(-1, H):
            for z in range(-1, D):
                mask = 0
                for i in range(8):
                    c = CORNERS[i]
                    if eval_sdf(x + c[0], y + c[1], z + c[2]) < 0.0:
                        mask |= 1 << i
                for e in CASES[mask]:
                    g = global_vertex_idx(x, y, z, e)
                    if g not in vmap:
                        a, b = CORNERS[EDGES[e][0]], CORNERS[EDGES[e][1]]
                        i1 = (x + a[0], y + a[1], z + a[2])
                        i2 = (x + b[0], y + b[1], z + b[2])
                        pa = ((i1[0] + 0.5) * hx + ox, (i1[1] + 0.5) * hy + oy, (i1[2] + 0.5) * hz + oz)
                        pb = ((i2[0] + 0.5) * hx + ox, (i2[1] + 0.5) * hy + oy, (i2[2] + 0.5) * hz + oz)
                        na, nb = grad(*i1), grad(*i2)
                        va, vb = eval_sdf(*i1), eval_sdf(*i2)
                        assert va * vb <= 0.0
                        frac = va / (va - vb)
                        p = tuple(pa[k] * (1 - frac) + pb[k] * frac for k in range(3))
                        n = tuple(na[k] * (1 - frac) + nb[k] * frac for k in range(3))
                        dot = n[0] * n[0] + n[1] * n[1] + n[2] * n[2]
                        # 1 / sqrt(dot) with IEEE semantics: 1/0 = inf, NaN stays NaN
                        inv = math.nan if dot != dot else (math.inf if dot == 0.0 else 1.0 / math.sqrt(dot))
                        vmap[g] = len(verts)
                        verts.append(p)
                        norms.append(tuple(c * inv for c in n))
                    idx.append(vmap[g])
    return (np.array(verts, np.float64).reshape(-1, 3), np.array(norms, np.float64).reshape(-1, 3),
            np.array(idx, np.uint32))


def sphere_sdf(dims, spacing, origin, centre, r):
    axes = [(np.arange(n) + 0.5) * s + o for n, s, o in zip(dims, spacing, origin)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2) - r


def scenes():
    rng = np.random.default_rng(11)
    yield "sphere_aniso", sphere_sdf((9, 7, 8), (0.11, 0.13, 0.12), (0.05, -0.1, 0.2), (0.55, 0.35, 0.7), 0.33), \
        (0.11, 0.13, 0.12), (0.05, -0.1, 0.2)
    yield "noise", rng.uniform(-1, 1, (6, 5, 7)), (0.1, 0.1, 0.1), (0.0, 0.0, 0.0)
    yield "zeros", rng.integers(-1, 2, (5, 6, 4)).astype(np.float64), (0.25, 0.25, 0.25), (0.0, 0.0, 0.0)
    yield "all_inside", -np.ones((3, 3, 3)), (0.5, 0.5, 0.5), (0.0, 0.0, 0.0)
    yield "empty", np.ones((4, 3, 5)), (0.5, 0.5, 0.5), (0.0, 0.0, 0.0)
    yield "single_cell", -np.ones((1, 1, 1)), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)
    holes = sphere_sdf((8, 9, 7), (0.125, 0.125, 0.125), (0, 0, 0), (0.5, 0.55, 0.45), 0.3)
    holes[rng.random(holes.shape) < 0.15] = np.inf  # +inf samples: positive, non-finite gradients
    yield "inf_holes", holes, (0.125, 0.125, 0.125), (0.0, 0.0, 0.0)


@pytest.mark.parametrize("name", [s[0] for s in scenes()])
def test_oracle_equals_literal_restatement(oracle, name):
    sdf, sp, org = next((s[1], s[2], s[3]) for s in scenes() if s[0] == name)
    V, N, I = oracle.rebuild_surface(sdf, sp, org)
    v, n, i = literal_rebuild_surface(sdf, sp, org)
    assert V.shape == v.shape and I.shape == i.shape
    assert np.array_equal(V, v, equal_nan=True) and np.array_equal(I, i)
    assert np.array_equal(N, n, equal_nan=True)
    if name == "empty":
        assert len(V) == 0 and len(I) == 0


def _edges(I):
    t = I.reshape(-1, 3).astype(np.int64)
    und = {}
    directed = set()
    for a, b, c in t:
        for u, v in ((a, b), (b, c), (c, a)):
            und[(min(u, v), max(u, v))] = und.get((min(u, v), max(u, v)), 0) + 1
            directed.add((u, v))
    return und, directed, len(t)


@pytest.mark.parametrize("n", [12, 17])
def test_closed_sphere_is_watertight_and_outward(oracle, n):
    h = 1.0 / n
    centre, r = (0.47, 0.52, 0.5), 0.3
    sdf = sphere_sdf((n, n, n), (h, h, h), (0, 0, 0), centre, r)
    V, N, I = oracle.rebuild_surface(sdf, h)
    assert len(I) % 3 == 0 and I.max() < len(V)
    und, directed, F = _edges(I)
    assert set(und.values()) == {2}  # every edge shared by exactly two triangles
    assert len(V) - len(und) + F == 2  # a sphere
    assert len(directed) == 2 * len(und)  # consistently oriented
    rad = np.linalg.norm(V - np.array(centre), axis=1)
    assert np.abs(rad - r).max() < h
    np.testing.assert_allclose(np.linalg.norm(N, axis=1), 1.0, rtol=0, atol=1e-12)
    assert (np.einsum("ij,ij->i", N, V - np.array(centre)) > 0).all()


def test_vertices_lie_on_sign_change_edges(oracle):
    rng = np.random.default_rng(3)
    sdf = rng.uniform(-1, 1, (5, 6, 7))
    V, N, I = oracle.rebuild_surface(sdf, 1.0)
    # each vertex sits on a grid edge between cell centres (one coordinate
    # strictly between two centres, the others on centres)
    frac = V - 0.5 - np.floor(V - 0.5)
    on_centre = np.isclose(frac, 0.0, atol=1e-12) | np.isclose(frac, 1.0, atol=1e-12)
    assert (on_centre.sum(1) >= 2).all()
    assert len(np.unique(I)) == len(V)  # every vertex is used


_REPLAY = r'''
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "sc_surface_dev.cuh"
static const uint64_t kCases[256] = {SC_MC_CASES_INIT};
struct Cases { uint64_t operator()(int m) const { return kCases[m]; } };
int main(int argc, char** argv) {
  FILE* f = fopen(argv[1], "rb");
  int dims[3]; double sp[3], org[3];
  if (fread(dims, 4, 3, f) != 3 || fread(sp, 8, 3, f) != 3 || fread(org, 8, 3, f) != 3) return 2;
  const size_t n = (size_t)dims[0] * dims[1] * dims[2];
  std::vector<double> sdf(n);
  if (fread(sdf.data(), 8, n, f) != n) return 2;
  fclose(f);
  sc::mc::Grid g{dims[0], dims[1], dims[2], sp[0], sp[1], sp[2], org[0], org[1], org[2], sdf.data()};
  const int64_t nc = g.ncubes();
  std::vector<uint8_t> mask(nc);
  std::vector<uint32_t> vbase(nc, 0xffffffffu);
  std::vector<int64_t> ibase(nc);
  int64_t nv = 0, ni = 0;
  for (int64_t c = 0; c < nc; c++) {  // count pass and exclusive scans, in cube order
    int i, j, k;
    g.cube(c, i, j, k);
    if (g.cube_index(i, j, k) != c) return 3;
    mask[c] = (uint8_t)g.mask(i, j, k);
    const uint64_t w = kCases[mask[c]];
    const int cv = sc::mc::owned_count(w);
    if (cv) vbase[c] = (uint32_t)nv;
    ibase[c] = ni;
    nv += cv;
    ni += SC_MC_COUNT(w);
  }
  std::vector<double> V(3 * nv), N(3 * nv);
  std::vector<uint32_t> I(ni);
  bool ok = true;
  for (int64_t c = nc - 1; c >= 0; c--) {  // emit in reverse: no order dependence
    int i, j, k;
    g.cube(c, i, j, k);
    const uint64_t w = kCases[mask[c]];
    if (vbase[c] != 0xffffffffu) sc::mc::emit_vertices(g, i, j, k, w, vbase[c], V.data(), N.data());
    ok &= sc::mc::emit_indices(g, i, j, k, w, Cases(), mask.data(), vbase.data(), ibase[c], I.data());
  }
  FILE* o = fopen(argv[2], "wb");
  fwrite(&nv, 8, 1, o); fwrite(&ni, 8, 1, o);
  fwrite(V.data(), 8, V.size(), o); fwrite(N.data(), 8, N.size(), o); fwrite(I.data(), 4, I.size(), o);
  fclose(o);
  return ok ? 0 : 4;
}
'''


@pytest.fixture(scope="module")
def replay(tmp_path_factory):
    """The kernels' per-cube functions (sc_surface_dev.cuh) built as host C++
    and driven in cube order: count, exclusive scan, emit."""
    import shutil
    import subprocess

    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("mc_replay")
    (d / "replay.cc").write_text(_REPLAY)
    exe = d / "replay"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-ffp-contract=off", "-Wall", "-Werror",
                           "-I", os.path.join(ROOT, "simcraft_b200", "csrc"), str(d / "replay.cc"), "-o", str(exe)])

    def run(sdf, spacing, origin):
        sdf = np.ascontiguousarray(sdf, np.float64)
        inp, out = d / "in.bin", d / "out.bin"
        with open(inp, "wb") as f:
            f.write(np.array(sdf.shape, np.int32).tobytes())
            f.write(np.array(spacing, np.float64).tobytes())
            f.write(np.array(origin, np.float64).tobytes())
            f.write(sdf.tobytes())
        subprocess.check_call([str(exe), str(inp), str(out)])
        raw = out.read_bytes()
        nv, ni = np.frombuffer(raw[:16], np.int64)
        off = 16
        V = np.frombuffer(raw[off:off + 24 * nv], np.float64).reshape(-1, 3)
        off += 24 * nv
        N = np.frombuffer(raw[off:off + 24 * nv], np.float64).reshape(-1, 3)
        off += 24 * nv
        return V, N, np.frombuffer(raw[off:off + 4 * ni], np.uint32)

    return run


def _nan_inf_field():
    f = sphere_sdf((12, 11, 13), (0.09,) * 3, (0, 0, 0), (0.5, 0.5, 0.55), 0.33)
    u = np.random.default_rng(8).random(f.shape)
    f[u < 0.06] = np.nan
    f[(u >= 0.06) & (u < 0.12)] = np.inf
    f[(u >= 0.12) & (u < 0.15)] = -np.inf
    return f


@pytest.mark.parametrize("name", [s[0] for s in scenes()] + ["sphere_32", "noise_20", "nan_inf"])
def test_kernel_numbering_replayed_on_cpu_equals_oracle(oracle, replay, name):
    """Owner cubes, ranks and the scan order give the reference's vertex
    numbering: the replay equals the oracle bit for bit (NaN where it has NaN)."""
    extra = {
        "sphere_32": (sphere_sdf((32, 30, 28), (1 / 32,) * 3, (0, 0, 0), (0.5, 0.45, 0.4), 0.31), (1 / 32,) * 3,
                      (0.0, 0.0, 0.0)),
        "noise_20": (np.random.default_rng(4).standard_normal((20, 21, 19)), (0.05, 0.06, 0.07), (0.3, 0.2, 0.1)),
        "nan_inf": (_nan_inf_field(), (0.09,) * 3, (0.0, 0.0, 0.0)),
    }
    if name in extra:
        sdf, sp, org = extra[name]
    else:
        sdf, sp, org = next((s[1], s[2], s[3]) for s in scenes() if s[0] == name)
    V, N, I = oracle.rebuild_surface(sdf, sp, org)
    v, n, i = replay(sdf, sp, org)
    assert np.array_equal(V, v, equal_nan=True) and np.array_equal(I, i)
    assert np.array_equal(N, n, equal_nan=True)


def test_wrapper_call_protocol_against_a_fake_library(oracle, monkeypatch):
    """simcraft_b200.surface.rebuild_surface drives the C-ABI contract: a
    counting call then a filling call the first time; one call when the mesh
    fits the remembered size; on a capacity failure the counts that call
    returned, then one filling call.  The fake library implements the contract
    with the oracle (no GPU)."""
    import ctypes

    import simcraft_b200.surface as S

    calls = []

    def as_array(p, ctype, shape):
        addr = p.value if isinstance(p, ctypes.c_void_p) else p
        return np.ctypeslib.as_array(ctypes.cast(addr, ctypes.POINTER(ctype)), shape)

    class FakeLib:
        def sc_rebuild_surface_host(self, h, nx, ny, nz, sp, org, sdf_p, vp, np_, ip, cv, ci, pnv, pni):
            sdf = as_array(sdf_p, ctypes.c_double, (nx, ny, nz)).copy()
            V, N, I = oracle.rebuild_surface(sdf, list(sp), list(org))
            pnv._obj.value, pni._obj.value = len(V), len(I)
            if vp is None:
                calls.append("count")
                return 0
            if cv < len(V) or ci < len(I):
                calls.append("short")
                return -1
            calls.append("fill")
            if len(V):
                as_array(vp, ctypes.c_double, (cv, 3))[:len(V)] = V
                as_array(np_, ctypes.c_double, (cv, 3))[:len(V)] = N
            if len(I):
                as_array(ip, ctypes.c_uint32, (ci,))[:len(I)] = I
            return 0

    class FakeCtx:
        handle = ctypes.c_void_p(0x5C)

    monkeypatch.setattr(S, "lib", lambda: FakeLib())
    monkeypatch.setattr(S, "_last_counts", {})
    ctx = FakeCtx()
    h = 1.0 / 14
    small = sphere_sdf((14, 14, 14), (h, h, h), (0, 0, 0), (0.5, 0.5, 0.5), 0.2)
    big = sphere_sdf((14, 14, 14), (h, h, h), (0, 0, 0), (0.5, 0.5, 0.5), 0.38)
    other = sphere_sdf((10, 12, 9), (h, h, h), (0, 0, 0), (0.3, 0.4, 0.3), 0.2)

    def run(sdf, expect):
        calls.clear()
        got = S.rebuild_surface(sdf, h, context=ctx)
        assert calls == expect
        ref = oracle.rebuild_surface(sdf, h)
        for a, b in zip(got, ref):
            assert a.shape == b.shape and np.array_equal(a, b, equal_nan=True)

    run(small, ["count", "fill"])
    run(small, ["fill"])
    run(big, ["short", "fill"])
    run(small, ["fill"])  # the remembered size is now the bigger mesh
    run(other, ["count", "fill"])
    run(np.ones((14, 14, 14)), ["fill"])  # an empty mesh fits any size


def test_export_obj_layout_and_round_trip(oracle, tmp_path):
    """export_obj writes exportObj's layout (Core/src/obj-io.cc:66-91) and the
    numbers read back to the same doubles; an unopenable path returns False."""
    from simcraft_b200.surface import export_obj

    h = 1.0 / 11
    V, N, I = oracle.rebuild_surface(sphere_sdf((11, 11, 11), (h, h, h), (0, 0, 0), (0.5, 0.5, 0.5), 0.3), h)
    path = tmp_path / "fluid.obj"
    assert export_obj(str(path), V, N, I)
    lines = path.read_text().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    nv, nt = len(V), len(I) // 3
    assert len(lines) == 2 * nv + nt
    v = np.array([[float(x) for x in ln.split()[1:]] for ln in lines[:nv] if ln.startswith("v ")])
    n = np.array([[float(x) for x in ln.split()[1:]] for ln in lines[nv:2 * nv] if ln.startswith("vn ")])
    assert np.array_equal(v, V) and np.array_equal(n, N)
    faces = lines[2 * nv:]
    assert all(ln.startswith("f ") and ln.endswith(" ") for ln in faces)
    f = np.array([[int(tok.split("//")[0]) for tok in ln.split()[1:]] for ln in faces])
    g = np.array([[int(tok.split("//")[1]) for tok in ln.split()[1:]] for ln in faces])
    assert np.array_equal(f, g) and np.array_equal(f - 1, I.reshape(-1, 3).astype(np.int64))
    assert export_obj(str(tmp_path), V, N, I) is False  # a directory cannot be opened for writing
