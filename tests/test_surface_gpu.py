"""The marching-cubes surface export (rebuildSurface,
FluidSim/src/cpu/rebuild-surface.cc:686-741) on the GPU, through the C-ABI,
against the CPU oracle: vertices, normals and index entries bit for bit (the
vertex numbering and triangle order included) on spheres with anisotropic
spacing and an origin, random fields full of ambiguous cases, exact zeros,
regions touching the border, a single cell, an empty field, and the fluid SDF
of a simulated dam break; then properties at 256^3 (watertight, Euler
characteristic 2) and the capacity error path."""
import numpy as np
import pytest

from test_surface_cpu import scenes, sphere_sdf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod(gpu):
    import torch
    return torch


def _same(got, ref):
    V, N, I = (x.cpu().numpy() if hasattr(x, "cpu") else x for x in got)
    v, n, i = ref
    assert V.shape == v.shape and I.shape == i.shape
    np.testing.assert_array_equal(V, v)
    np.testing.assert_array_equal(N, n)  # NaN where the gradient vanishes, on both sides
    np.testing.assert_array_equal(I.astype(np.int64), i.astype(np.int64))


@pytest.mark.parametrize("name", [s[0] for s in scenes()])
@pytest.mark.parametrize("path", ["host", "device"])
def test_small_scenes_bit_exact(oracle, torch_mod, name, path):
    from simcraft_b200.surface import rebuild_surface

    sdf, sp, org = next((s[1], s[2], s[3]) for s in scenes() if s[0] == name)
    ref = oracle.rebuild_surface(sdf, sp, org)
    arg = torch_mod.from_numpy(np.ascontiguousarray(sdf)).cuda() if path == "device" else sdf
    _same(rebuild_surface(arg, sp, org), ref)


def _spheres(dims, sp, seed, count):
    rng = np.random.default_rng(seed)
    axes = [(np.arange(n) + 0.5) * s for n, s in zip(dims, sp)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    ext = [n * s for n, s in zip(dims, sp)]
    d = np.full(dims, np.inf)
    for _ in range(count):
        c = rng.uniform(0, 1, 3) * ext
        r = rng.uniform(0.05, 0.2) * min(ext)
        d = np.minimum(d, np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r)
    return d


@pytest.mark.parametrize("case", ["noise_64", "spheres_96x80x72", "spheres_160"])
def test_larger_grids_bit_exact(oracle, torch_mod, case):
    from simcraft_b200.surface import rebuild_surface

    if case == "noise_64":
        sdf, sp, org = np.random.default_rng(21).standard_normal((64, 64, 64)), (1 / 64,) * 3, (0.0, 0.0, 0.0)
    elif case == "spheres_96x80x72":
        sp = (0.011, 0.013, 0.012)
        sdf, org = _spheres((96, 80, 72), sp, 22, 24), (-0.2, 0.1, 0.3)
    else:
        sp = (1 / 160,) * 3
        sdf, org = _spheres((160, 160, 160), sp, 23, 24), (0.0, 0.0, 0.0)
    ref = oracle.rebuild_surface(sdf, sp, org)
    assert len(ref[2]) > 0
    _same(rebuild_surface(torch_mod.from_numpy(sdf).cuda(), sp, org), ref)


def test_simulated_fluid_surface_bit_exact(oracle, torch_mod):
    """rebuildSurface(mesh, exportFluidSurface()) after two frames of a 16^3
    dam break, as the reference's app exports the fluid."""
    from simcraft_b200 import scenes as S
    from simcraft_b200.fluid import FluidSimulator

    n = 16
    pos, _, h = S.dam_break(n, seed=1)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), pcg_tol=1e-6, pcg_max_iter=200)
    sim.set_initial_fluid(pos)
    for _ in range(2):
        sim.step(1.0 / 120)
    sdf = sim.export_fluid_surface()
    got = sim.rebuild_surface()
    ref = oracle.rebuild_surface(sdf, h)
    assert len(ref[2]) > 0
    _same(got, ref)


def test_sphere_256_watertight(torch_mod):
    """At full size, through size-independent properties: every edge in two
    triangles, consistently oriented, Euler characteristic 2, vertices within a
    cell of the sphere, unit outward normals."""
    from simcraft_b200.surface import rebuild_surface

    n, centre, r = 256, (0.5, 0.47, 0.53), 0.37
    h = 1.0 / n
    sdf = torch_mod.from_numpy(sphere_sdf((n, n, n), (h, h, h), (0, 0, 0), centre, r)).cuda()
    V, N, I = (x.cpu().numpy() for x in rebuild_surface(sdf, h))
    t = I.astype(np.int64).reshape(-1, 3)
    directed = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    key = np.minimum(directed[:, 0], directed[:, 1]) * len(V) + np.maximum(directed[:, 0], directed[:, 1])
    uniq, cnt = np.unique(key, return_counts=True)
    assert (cnt == 2).all()
    assert len(np.unique(directed[:, 0] * len(V) + directed[:, 1])) == len(directed)
    assert len(V) - len(uniq) + len(t) == 2
    assert np.abs(np.linalg.norm(V - np.array(centre), axis=1) - r).max() < h
    np.testing.assert_allclose(np.linalg.norm(N, axis=1), 1.0, rtol=0, atol=1e-12)
    assert (np.einsum("ij,ij->i", N, V - np.array(centre)) > 0).all()


SC_ERR_INVALID = -1


def test_capacity_below_mesh_is_an_error(torch_mod):
    import ctypes

    from simcraft_b200._capi import lib
    from simcraft_b200.solver import default_context

    ctx = default_context()
    h = 1.0 / 12
    sdf = np.ascontiguousarray(sphere_sdf((12, 12, 12), (h, h, h), (0, 0, 0), (0.5, 0.5, 0.5), 0.3))
    sp = (ctypes.c_double * 3)(h, h, h)
    nv, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    assert lib().sc_rebuild_surface_host(ctx.handle, 12, 12, 12, sp, None, sdf.ctypes.data, None, None, None, 0, 0,
                                         ctypes.byref(nv), ctypes.byref(ni)) == 0
    assert nv.value > 0 and ni.value > 0
    V = np.zeros((nv.value, 3))
    Nn = np.zeros((nv.value, 3))
    I = np.zeros(ni.value, np.uint32)
    rc = lib().sc_rebuild_surface_host(ctx.handle, 12, 12, 12, sp, None, sdf.ctypes.data, V.ctypes.data,
                                       Nn.ctypes.data, I.ctypes.data, nv.value, ni.value - 3, ctypes.byref(nv),
                                       ctypes.byref(ni))
    assert rc == SC_ERR_INVALID and not V.any() and not I.any()
    # one output missing
    rc = lib().sc_rebuild_surface_host(ctx.handle, 12, 12, 12, sp, None, sdf.ctypes.data, V.ctypes.data, None,
                                       I.ctypes.data, nv.value, ni.value, ctypes.byref(nv), ctypes.byref(ni))
    assert rc == SC_ERR_INVALID
    # the context still works
    assert lib().sc_rebuild_surface_host(ctx.handle, 12, 12, 12, sp, None, sdf.ctypes.data, V.ctypes.data,
                                         Nn.ctypes.data, I.ctypes.data, nv.value, ni.value, ctypes.byref(nv),
                                         ctypes.byref(ni)) == 0
    assert I.max() == nv.value - 1


@pytest.mark.parametrize("path", ["host", "device"])
def test_repeated_exports_single_call_path(oracle, torch_mod, path):
    """Exports of one grid in a row (the wrapper's one-call path, then a mesh
    larger than the remembered size, then smaller again) stay bit-exact."""
    from simcraft_b200.solver import Context
    from simcraft_b200.surface import rebuild_surface

    ctx = Context(0)
    h = 1.0 / 40
    for r in (0.2, 0.2, 0.41, 0.15, 0.3):
        sdf = sphere_sdf((40, 40, 40), (h, h, h), (0, 0, 0), (0.5, 0.52, 0.48), r)
        arg = torch_mod.from_numpy(sdf).cuda() if path == "device" else sdf
        _same(rebuild_surface(arg, h, context=ctx), oracle.rebuild_surface(sdf, h))
