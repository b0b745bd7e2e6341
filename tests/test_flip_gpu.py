"""FLIP/PIC step parity: the CUDA path (through the C-ABI) against the oracle.

Per-stage tests compare one call of each transfer with the oracle on the same
seeded inputs; the simulator tests run the 32^3 dam break of the reference's
scalar type for 10 frames and compare the pressure after every frame and the
particle positions at the end."""
import numpy as np
import pytest

from simcraft_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod(gpu):
    import torch
    return torch


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _grids(dims, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    return [scale * rng.uniform(-1, 1, s) for s in ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))]


def _points(dims, h, n, seed, margin=0.1):
    rng = np.random.default_rng(seed)
    ext = np.array(dims) * h
    return rng.uniform(-margin, 1 + margin, (n, 3)) * ext


# The transfers restate the CPU arithmetic operation by operation (no FMA
# contraction, the same loop and summation order), so gathers are bit-exact.
@pytest.mark.parametrize("dims,h", [((13, 9, 11), 1 / 13), ((16, 16, 16), 1 / 16), ((5, 7, 3), 0.3)])
def test_sample_velocity_bit_exact(oracle, torch_mod, dims, h):
    from simcraft_b200 import fluid
    u, v, w = _grids(dims, 1)
    pts = _points(dims, h, 4000, 2)
    # nodes and cell faces exactly, where nearest() rounds
    ii = np.random.default_rng(3).integers(0, 2 * max(dims) + 1, (500, 3))
    pts = np.concatenate([pts, ii * (h / 2)])
    ref = oracle.sample_velocity(pts, dims, h, u, v, w)
    t = torch_mod
    got = fluid.sample_velocity(_dev(t, pts), dims, h, _dev(t, u), _dev(t, v), _dev(t, w)).cpu().numpy()
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("alpha", [0.97, 0.95, -1.0])
def test_g2p_bit_exact(oracle, torch_mod, alpha):
    from simcraft_b200 import fluid
    dims, h = (12, 10, 14), 1 / 12
    u, v, w = _grids(dims, 4)
    ul, vl, wl = _grids(dims, 5)
    pos = _points(dims, h, 5000, 6, margin=0.0)
    vel = np.random.default_rng(7).normal(size=pos.shape)
    ref = oracle.g2p(pos, vel, dims, h, u, v, w, ul, vl, wl, alpha=alpha)
    t = torch_mod
    got = fluid.g2p(_dev(t, pos), _dev(t, vel), dims, h, _dev(t, u), _dev(t, v), _dev(t, w),
                    _dev(t, ul) if alpha >= 0 else None, _dev(t, vl) if alpha >= 0 else None,
                    _dev(t, wl) if alpha >= 0 else None, alpha=alpha).cpu().numpy()
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("with_collider", [False, True])
def test_advect_bit_exact(oracle, torch_mod, with_collider):
    from simcraft_b200 import fluid
    n = 16
    dims, h = (n, n, n), 1 / n
    u, v, w = _grids(dims, 8, scale=3.0)
    pos = _points(dims, h, 6000, 9, margin=0.0)
    # velocities large enough to leave the box (box clamp) and to enter the collider
    vel = np.random.default_rng(10).normal(scale=4.0, size=pos.shape)
    col = None
    if with_collider:
        col = scenes.sphere_union_sdf(n, np.array([[0.5, 0.3, 0.5], [0.2, 0.8, 0.7]]), np.array([0.2, 0.15]))
    dt = 1 / 30
    p_ref, v_ref = oracle.advect(pos, vel, dims, h, u, v, w, col, dt)
    t = torch_mod
    p, vv = fluid.advect(_dev(t, pos), _dev(t, vel), dims, h, _dev(t, u), _dev(t, v), _dev(t, w),
                         _dev(t, col) if col is not None else None, dt)
    np.testing.assert_array_equal(p.cpu().numpy(), p_ref)
    np.testing.assert_array_equal(vv.cpu().numpy(), v_ref)
    assert (p_ref == 0).any() and (p_ref == 1.0).any()  # the box clamp fired
    if with_collider:
        p_free, _ = oracle.advect(pos, vel, dims, h, u, v, w, None, dt)
        assert (np.abs(p_free - p_ref).max(axis=1) > 0).any()  # so did the collider push-out


def _p2g_inputs(n, seed):
    pos, _, h = scenes.dam_break(n, seed=seed)
    rng = np.random.default_rng(seed + 100)
    vel = rng.normal(size=pos.shape)
    # particles on the domain walls and on cell faces, and a few outside the box
    extra = rng.integers(0, 2 * n + 1, (200, 3)) * (h / 2)
    outside = rng.uniform(-1.5 * h, 1 + 1.5 * h, (60, 3))
    extra = np.concatenate([extra, outside])
    pos = np.concatenate([pos, extra])
    vel = np.concatenate([vel, rng.normal(size=extra.shape)])
    return pos, vel, h


@pytest.mark.parametrize("n", [8, 16])
def test_p2g_matches_oracle(oracle, torch_mod, n):
    from simcraft_b200 import fluid
    pos, vel, h = _p2g_inputs(n, 11)
    dims = (n, n, n)
    ref = oracle.p2g(pos, vel, dims, h, flip=True)
    t = torch_mod
    got = {k: a.cpu().numpy() for k, a in fluid.p2g(_dev(t, pos), _dev(t, vel), dims, h, flip=True).items()}
    for g in "uvw":
        # validity is exact; values differ from the serial splat only by summation order
        np.testing.assert_array_equal(got[g + "valid"], ref[g + "valid"])
        np.testing.assert_allclose(got[g + "w"], ref[g + "w"], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(got[g], ref[g], rtol=1e-12, atol=1e-13)
        np.testing.assert_array_equal(got[g + "last"], got[g])


def _p2g_box_inputs(dims, h, seed, ppc=3):
    """Jittered particles in every cell of a non-cubic grid, plus particles on
    cell faces and centres (where the nearest-node tests round) and outside."""
    rng = np.random.default_rng(seed)
    ext = np.array(dims) * h
    n = int(np.prod(dims)) * ppc
    pos = rng.uniform(0, 1, (n, 3)) * ext
    faces = rng.integers(0, 2 * min(dims) + 1, (300, 3)) * (h / 2)
    outside = rng.uniform(-1.5 * h, ext + 1.5 * h, (60, 3))
    pos = np.concatenate([pos, faces, outside])
    return pos, rng.normal(size=pos.shape)


@pytest.mark.parametrize("dims", [(40, 24, 33), (9, 17, 8)])
def test_p2g_non_cubic_matches_oracle_and_repeats_bit_for_bit(oracle, torch_mod, dims):
    """Several 8^3 tiles with partial tiles at the far faces; the sums are the
    same bit for bit on every run (no atomics on the regular path)."""
    from simcraft_b200 import fluid
    t = torch_mod
    h = 1.0 / max(dims)
    pos, vel = _p2g_box_inputs(dims, h, 31)
    ref = oracle.p2g(pos, vel, dims, h, flip=True)
    runs = [{k: a.cpu().numpy() for k, a in fluid.p2g(_dev(t, pos), _dev(t, vel), dims, h, flip=True).items()}
            for _ in range(3)]
    for g in "uvw":
        np.testing.assert_array_equal(runs[0][g + "valid"], ref[g + "valid"])
        np.testing.assert_allclose(runs[0][g + "w"], ref[g + "w"], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(runs[0][g], ref[g], rtol=1e-12, atol=1e-13)
    for r in runs[1:]:
        for k in runs[0]:
            np.testing.assert_array_equal(r[k], runs[0][k])


def test_p2g_empty_and_permutation_invariant(oracle, torch_mod):
    from simcraft_b200 import fluid
    t = torch_mod
    n = 8
    dims = (n, n, n)
    pos, vel, h = _p2g_inputs(n, 12)
    a = fluid.p2g(_dev(t, pos), _dev(t, vel), dims, h, flip=False)
    perm = np.random.default_rng(13).permutation(len(pos))
    b = fluid.p2g(_dev(t, pos[perm]), _dev(t, vel[perm]), dims, h, flip=False)
    for k in a:
        # particles are sorted by (cell, index) first, so only the index tie-break changes
        np.testing.assert_allclose(a[k].cpu().numpy(), b[k].cpu().numpy(), rtol=1e-12, atol=1e-14)
    e = fluid.p2g(_dev(t, np.zeros((0, 3))), _dev(t, np.zeros((0, 3))), dims, h, flip=False)
    for k in e:
        assert not e[k].any()


@pytest.mark.parametrize("n,radius_factor", [(16, 0.8), (12, 1.2 / np.sqrt(2))])
def test_reconstruct_bit_exact(oracle, torch_mod, n, radius_factor):
    from simcraft_b200 import fluid
    pos, _, h = scenes.dam_break(n, frac_x=0.6, frac_y=0.4, ppc=3, seed=14)
    rng = np.random.default_rng(15)
    # lone particles (buckets of one are never visited) and particles outside the box
    pos = np.concatenate([pos, rng.uniform(-0.05, 1.05, (300, 3))])
    dims = (n, n, n)
    s_ref, v_ref = oracle.reconstruct(pos, dims, h, radius_factor * h)
    t = torch_mod
    s, v = fluid.reconstruct(_dev(t, pos), dims, h, radius_factor * h)
    np.testing.assert_array_equal(v.cpu().numpy(), v_ref)
    np.testing.assert_array_equal(s.cpu().numpy(), s_ref)
    assert v_ref.any() and not v_ref.all()


def test_reconstruct_dense_buckets_bit_exact(oracle, torch_mod):
    """Buckets far fuller than the dam breaks' (about 20 to 25 particles, past
    the 16 that are ordered through shared memory, so the sort's in-place
    path): the bucket order, which fixes the particle the reference's loop
    skips, and so the SDF, bit for bit."""
    from simcraft_b200 import fluid
    n = 16
    h = 1.0 / n
    rng = np.random.default_rng(16)
    # cells (0, 0..7, 0..15): ~2600 particles
    a = rng.uniform(0, 1, (2600, 3)) * np.array([h, 8 * h, 16 * h])
    # cells (5, 8..15, 0..15): ~1500 particles, ~23 a bucket
    b = rng.uniform(0, 1, (1500, 3)) * np.array([h, 8 * h, 16 * h]) + np.array([5 * h, 8 * h, 0.0])
    pos, _, _ = scenes.dam_break(n, frac_x=0.5, frac_y=0.5, ppc=3, seed=17)
    pos = rng.permutation(np.concatenate([pos, a, b]))
    dims = (n, n, n)
    s_ref, v_ref = oracle.reconstruct(pos, dims, h, 0.8 * h)
    s, v = fluid.reconstruct(_dev(torch_mod, pos), dims, h, 0.8 * h)
    np.testing.assert_array_equal(v.cpu().numpy(), v_ref)
    np.testing.assert_array_equal(s.cpu().numpy(), s_ref)


def _config1_sim(oracle, n=32, steps=10, precision="f64", advection="flip", collider=None, seed=1):
    """The 32^3 dam break: block x<0.5, y<0.5, 8 jittered particles per cell,
    frame dt 1/120, FLIP blend 0.95, MIC(0)-PCG to 1e-6 relative, max 200."""
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2
    pos, vel, h = scenes.dam_break(n, seed=seed)
    flip = advection == "flip"
    ocfg = oracle.default_config(n, n, n, h, flip=int(flip), flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200,
                                 pcg_criterion=CRIT_REL_L2)
    ref = oracle.Sim(**ocfg)
    ref.set_particles(pos, vel)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), precision=precision, advection=advection,
                         flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200, pcg_criterion=CRIT_REL_L2)
    sim.set_initial_fluid(pos, vel)
    if collider is not None:
        ref.set_collider(collider)
        sim.set_collider(collider)
    return ref, sim, h


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_dam_break_32_fp64_parity(oracle, torch_mod):
    ref, sim, h = _config1_sim(oracle)
    frame = 1.0 / 120
    for step in range(10):
        n_ref = ref.step(frame)
        st = sim.step(frame)
        assert st["substeps"] == n_ref == 1
        p_ref, p = ref.pressure(), sim.pressure()
        assert np.abs(p_ref).max() > 0
        assert _rel(p, p_ref) <= 1e-5, (step, _rel(p, p_ref))
        assert abs(st["pcg_iterations"] - ref.last_iters()) <= 1
    x_ref, v_ref = ref.particles()
    x, v = sim.particles()
    assert np.abs(x - x_ref).max() <= 1e-4 * h
    assert np.abs(v - v_ref).max() <= 1e-4 * max(1.0, np.abs(v_ref).max())
    # the fluid moved and stayed in the box
    assert np.abs(x - scenes.dam_break(32, seed=1)[0]).max() > 0.1 * h
    assert x.min() >= 0 and x.max() <= 1
    u, vg, w = sim.faces()
    ur, vr, wr = ref.faces()
    for a, b in ((u, ur), (vg, vr), (w, wr)):
        assert _rel(a, b) <= 1e-5
    # the surface follows the particles: same bound as the positions
    np.testing.assert_allclose(sim.export_fluid_surface(), ref.fluid_sdf(), rtol=0, atol=1e-4 * h)


def test_dam_break_pic_with_collider(oracle, torch_mod):
    n = 24
    col = scenes.sphere_union_sdf(n, np.array([[0.3, 0.15, 0.5]]), np.array([0.12]))
    ref, sim, h = _config1_sim(oracle, n=n, advection="pic", collider=col, seed=3)
    for step in range(4):
        ref.step(1.0 / 120)
        sim.step(1.0 / 120)
        assert _rel(sim.pressure(), ref.pressure()) <= 1e-5
    x_ref, _ = ref.particles()
    x, _ = sim.particles()
    assert np.abs(x - x_ref).max() <= 1e-4 * h


def test_dam_break_fp32_and_mixed_solver(oracle, torch_mod):
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2, PREC_MIXED
    n = 32
    pos, vel, h = scenes.dam_break(n, seed=1)
    ocfg = oracle.default_config(n, n, n, h, flip=1, flip_alpha=0.95, pcg_tol=1e-8, pcg_max_iter=400,
                                 pcg_criterion=CRIT_REL_L2)
    ref = oracle.Sim(**ocfg)
    ref.set_particles(pos, vel)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), precision="f32", flip_alpha=0.95,
                         pcg_tol=1e-8, pcg_max_iter=400, pcg_criterion=CRIT_REL_L2, pcg_precision=PREC_MIXED)
    sim.set_initial_fluid(pos, vel)
    for _ in range(5):
        ref.step(1.0 / 120)
        st = sim.step(1.0 / 120)
        assert st["pcg_residual"] < 1e-8
        # FP32 particles and grids: agreement to single-precision rounding
        assert _rel(sim.pressure(), ref.pressure()) <= 1e-3
    x_ref, _ = ref.particles()
    x, _ = sim.particles()
    assert np.abs(x - x_ref).max() <= 1e-2 * h


def test_simulator_edge_cases(oracle, torch_mod):
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200._capi import CapiError
    n = 8
    sim = FluidSimulator(0, (1.0, 1.0, 1.0), (n, n, n))
    # no particles: CFL of a still grid, one substep, zero pressure
    assert sim.cfl() == pytest.approx(5.0 * (1.0 / n) / 1e-6)
    st = sim.substep(1.0 / 120)
    assert st["substeps"] == 1 and st["kernel_launches"] > 0
    assert not sim.pressure().any()
    with pytest.raises(ValueError):
        FluidSimulator(0, (1.0, 2.0, 1.0), (n, n, n))
    with pytest.raises(CapiError):
        sim.substep(-1.0)
    # particles come back in the order they were given, after the per-substep sort
    pos, vel, h = scenes.dam_break(n, seed=5)
    perm = np.random.default_rng(6).permutation(len(pos))
    sim.set_initial_fluid(pos[perm], vel[perm])
    x0, _ = sim.particles()
    np.testing.assert_array_equal(x0, pos[perm])
    sim.step(1.0 / 120)
    x1, _ = sim.particles()
    assert np.abs(x1 - pos[perm]).max() < 0.5 * h


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_dam_break_64_ten_frames(oracle, torch_mod, precision):
    """The largest stand-in for the 256^3 dam break that the CPU oracle runs in
    seconds: 64^3, block x < 0.5, y < 0.5 (262,144 particles), FLIP 0.95, frames
    of 1/240 (dt/h = 0.267, the regime where the reference's MIC(0) converges),
    10 frames.  f64: the FP64 solver, pressure within 1e-5 relative L2 after
    every frame and positions within 1e-4 h after 10 frames.  f32: FP32
    particles and grids with the mixed solver (FP32 Eisenstat CG, FP64
    residual replacement) to 1e-8; single-precision rounding of positions and
    grids bounds the agreement: pressure within 1e-3 relative L2 after every
    frame, positions within 1e-2 h after 10 frames."""
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2, PREC_FP64, PREC_MIXED
    n = 64
    pos, vel, h = scenes.dam_break(n, seed=1)
    ocfg = oracle.default_config(n, n, n, h, flip=1, flip_alpha=0.95, pcg_tol=1e-8, pcg_max_iter=800,
                                 pcg_criterion=CRIT_REL_L2)
    ref = oracle.Sim(**ocfg)
    ref.set_particles(pos, vel)
    f32 = precision == "f32"
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), precision=precision, flip_alpha=0.95,
                         pcg_tol=1e-8, pcg_max_iter=800, pcg_criterion=CRIT_REL_L2,
                         pcg_precision=PREC_MIXED if f32 else PREC_FP64)
    sim.set_initial_fluid(pos, vel)
    errs = []
    for step in range(10):
        assert ref.step(1.0 / 240) == 1
        st = sim.step(1.0 / 240)
        assert st["substeps"] == 1 and st["pcg_residual"] < 1e-8
        errs.append(_rel(sim.pressure(), ref.pressure()))
        assert errs[-1] <= (1e-3 if f32 else 1e-5), (step, errs)
    x_ref, _ = ref.particles()
    x, _ = sim.particles()
    dx = np.abs(x - x_ref).max() / h
    assert dx <= (1e-2 if f32 else 1e-4), (dx, errs)
    assert np.abs(x_ref - pos).max() > 0.2 * h  # the block has started to fall (0.29 h in 10 frames)
