"""manifold2SDF on the GPU (through the C-ABI) against the oracle: bit-exact
distances and closest triangles for closed meshes on cubic and non-cubic grids,
with origins, narrow and wide exact bands, meshes reaching outside the grid, in
the reference's arithmetic and in exact-distance mode; then the simulator with
a mesh collider against the oracle simulator given the oracle's collider SDF."""
import numpy as np
import pytest

from simcraft_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod(gpu):
    import torch
    return torch


CASES = {
    "icosphere": (lambda: scenes.icosphere(2, 0.3, (0.5, 0.48, 0.52)), (20, 20, 20), 1 / 20, (0.0, 0.0, 0.0), 3),
    "torus": (lambda: scenes.torus(16, 8, 0.3, 0.1, (0.5, 0.5, 0.5)), (18, 14, 22), 1 / 18, (0.05, 0.1, -0.07), 1),
    "box_band0": (lambda: scenes.box_mesh((0.27, 0.31, 0.22), (0.71, 0.66, 0.74)), (16, 16, 16), 1 / 16,
                  (0.0, 0.0, 0.0), 0),
    "outside": (lambda: scenes.icosphere(3, 0.3, (0.9, 0.5, 0.45)), (24, 16, 20), 1 / 24, (0.0, 0.0, 0.0), 3),
}


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("case", sorted(CASES))
def test_mesh_to_sdf_bit_exact(oracle, torch_mod, case, exact):
    torch = torch_mod
    from simcraft_b200.mesh import manifold_to_sdf
    make, dims, h, origin, band = CASES[case]
    v, t = make()
    sdf_ref, cl_ref, _ = oracle.manifold_to_sdf(v, t, dims, h, origin=origin, exact_band=band, exact_distance=exact)
    sdf, cl = manifold_to_sdf(torch.from_numpy(v).cuda(), torch.from_numpy(t).cuda(), dims, h, origin=origin,
                              exact_band=band, exact_distance=exact, closest=True)
    np.testing.assert_array_equal(sdf.cpu().numpy(), sdf_ref)
    np.testing.assert_array_equal(cl.cpu().numpy(), cl_ref)
    assert (sdf_ref < 0).any() and (sdf_ref > 0).any()


def test_mesh_to_sdf_host_path_twice_and_errors(oracle, torch_mod):
    from simcraft_b200._capi import CapiError
    from simcraft_b200.mesh import manifold_to_sdf
    v, t = scenes.icosphere(2, 0.25)
    dims, h = (12, 14, 10), 1 / 12
    ref, _, _ = oracle.manifold_to_sdf(v, t, dims, h)
    for _ in range(2):  # scratch is re-initialised on every call
        np.testing.assert_array_equal(manifold_to_sdf(v, t, dims, h), ref)
    # empty mesh: nothing reaches any cell
    e, cl = manifold_to_sdf(np.zeros((0, 3)), np.zeros((0, 3), np.int32), dims, h, closest=True)
    assert (e == 1e9).all() and (cl == -1).all()
    bad = t.copy()
    bad[3, 1] = len(v)
    with pytest.raises(CapiError):
        manifold_to_sdf(v, bad, dims, h)
    bad[3, 1] = -1
    with pytest.raises(CapiError):
        manifold_to_sdf(v, bad, dims, h)


def test_simulator_with_mesh_collider(oracle, torch_mod):
    """setCollider(mesh) on the GPU simulator against the oracle simulator given
    the oracle's manifold2SDF of the same mesh: 24^3 PIC dam break, 4 frames."""
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2
    n = 24
    pos, vel, h = scenes.dam_break(n, seed=3)
    v, t = scenes.icosphere(2, 0.12, (0.3, 0.15, 0.5))
    col, _, _ = oracle.manifold_to_sdf(v, t, (n, n, n), h)
    ocfg = oracle.default_config(n, n, n, h, flip=0, flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200,
                                 pcg_criterion=CRIT_REL_L2)
    ref = oracle.Sim(**ocfg)
    ref.set_particles(pos, vel)
    ref.set_collider(col)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), advection="pic", flip_alpha=0.95, pcg_tol=1e-6,
                         pcg_max_iter=200, pcg_criterion=CRIT_REL_L2)
    sim.set_initial_fluid(pos, vel)
    sim.set_collider_mesh(v, t)
    for _ in range(4):
        ref.step(1.0 / 120)
        sim.step(1.0 / 120)
        p_ref = ref.pressure()
        assert np.linalg.norm(sim.pressure() - p_ref) <= 1e-5 * np.linalg.norm(p_ref)
    x_ref, _ = ref.particles()
    x, _ = sim.particles()
    assert np.abs(x - x_ref).max() <= 1e-4 * h
