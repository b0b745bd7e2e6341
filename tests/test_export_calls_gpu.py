"""The simulator's export calls on the GPU against the oracle simulator:
FluidSimulator::reconstruct() (FluidSim/include/FluidSim/cpu/fluid-simulator.h
:115-119, radius 1.2 h / sqrt 2) and smoothFluidSurface(5)
(FluidSim/src/cpu/fluid-simulator.cc:39-74), called between frames as the
reference's export path calls them (FluidSim/disabled/fluid-sim.cc:231-235).
Both act on the simulator's own surface buffers, so the next frame must still
follow the oracle; then the mesh of the exported surface (rebuildSurface) is
the oracle's mesh of the same SDF."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_export_calls_between_frames_follow_the_oracle(oracle, gpu):
    from simcraft_b200 import scenes
    from simcraft_b200.fluid import FluidSimulator

    n = 16
    pos, vel, h = scenes.dam_break(n, seed=1)
    cfg = oracle.default_config(n, n, n, h, flip_alpha=0.95, pcg_tol=1e-8, pcg_criterion=1)
    ref = oracle.Sim(**cfg)
    ref.set_particles(pos, vel)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), flip_alpha=0.95, pcg_tol=1e-8, pcg_criterion=1)
    sim.set_initial_fluid(pos, vel)
    ref.step(1.0 / 120)
    sim.step(1.0 / 120)
    ref.reconstruct()
    sim.reconstruct()
    np.testing.assert_allclose(sim.export_fluid_surface(), ref.fluid_sdf(), rtol=0, atol=1e-9 * h)
    ref.smooth_fluid_surface(5)
    sim.smooth_fluid_surface(5)
    s_ref = ref.fluid_sdf()
    s_gpu = sim.export_fluid_surface()
    np.testing.assert_allclose(s_gpu, s_ref, rtol=0, atol=1e-9 * h)
    V, N, I = sim.rebuild_surface()
    Vr, Nr, Ir = oracle.rebuild_surface(s_gpu, h)
    assert len(Ir) > 0 and np.array_equal(V, Vr) and np.array_equal(I, Ir)
    ref.step(1.0 / 120)
    sim.step(1.0 / 120)
    p_ref, p_gpu = ref.pressure(), sim.pressure()
    assert np.linalg.norm(p_gpu - p_ref) / np.linalg.norm(p_ref) < 1e-5
    assert np.abs(sim.positions() - ref.particles()[0]).max() < 1e-4 * h
    np.testing.assert_allclose(sim.export_fluid_surface(), ref.fluid_sdf(), rtol=0, atol=1e-6 * h)


def test_export_collider_surface(gpu):
    """exportColliderSurface(): 1e9 everywhere without a collider, the given
    SDF after setCollider(sdf), and empty again after removing it."""
    from simcraft_b200 import scenes
    from simcraft_b200.fluid import FluidSimulator

    n = 12
    pos, vel, h = scenes.dam_break(n, seed=2)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n))
    assert (sim.export_collider_surface() == 1e9).all()
    x = (np.arange(n) + 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    C = np.sqrt((X - 0.6) ** 2 + (Y - 0.3) ** 2 + (Z - 0.5) ** 2) - 0.2
    sim.set_collider(C)
    assert np.array_equal(sim.export_collider_surface(), C)
    sim.set_collider(None)
    assert (sim.export_collider_surface() == 1e9).all()


@pytest.mark.parametrize("passes", [(7, 2), (1, 4, 3)])
def test_smoothing_pass_counts_follow_the_oracle(oracle, gpu, passes):
    """smoothFluidSurface with pass counts other than five, odd and even, on a
    non-cubic grid: the surface after each call, and the next substep, whose
    SDF extrapolation keeps the older buffer's values in valid cells, so the
    buffer the pass before the last one wrote must hold what the oracle's
    holds."""
    from simcraft_b200 import scenes
    from simcraft_b200.fluid import FluidSimulator

    dims = (24, 20, 36)
    pos, vel, h = scenes.dam_break(24, seed=4)  # the block x, y < 1/2, z < 1
    cfg = oracle.default_config(*dims, h, flip_alpha=0.95, pcg_tol=1e-8, pcg_criterion=1)
    ref = oracle.Sim(**cfg)
    ref.set_particles(pos, vel)
    ext = tuple(d * h for d in dims)
    sim = FluidSimulator(len(pos), ext, dims, flip_alpha=0.95, pcg_tol=1e-8, pcg_criterion=1)
    sim.set_initial_fluid(pos, vel)
    ref.step(1.0 / 120)
    sim.step(1.0 / 120)
    for k in passes:
        ref.smooth_fluid_surface(k)
        sim.smooth_fluid_surface(k)
        np.testing.assert_allclose(sim.export_fluid_surface(), ref.fluid_sdf(), rtol=0, atol=1e-9 * h)
    ref.step(1.0 / 120)
    sim.step(1.0 / 120)
    assert np.abs(sim.positions() - ref.particles()[0]).max() < 1e-4 * h
    np.testing.assert_allclose(sim.export_fluid_surface(), ref.fluid_sdf(), rtol=0, atol=1e-6 * h)
