"""The oracle restatement against the reference's OWN code, bit for bit.

oracle/_ref/libsimcraft_ref.so is the reference's FluidSim CPU sources
(FluidSim/src/cpu/*.cc) compiled from the reference tree with the stand-in
headers of oracle/refshim (`make -C oracle ref`).  Every GPU parity test checks
the CUDA path against the oracle; these tests check the oracle against the
reference itself, function by function and for the whole simulator (config 1:
the 32^3 FLIP dam break over 10 frames).

Two readings differ between the reference as compiled here and the oracle, and
the tests state them:
  * bucket order of the reconstruction: the reference sorts with std::sort
    (not stable); the oracle's default, like the GPU path, is (cell, particle
    id).  oracle.set_bucket_order(1) reproduces the reference's sort.
  * unqualified `abs` on doubles (fluid-simulator.cc:190-200 CFL,
    util.cc:174 checkNeighbour) binds to C's int abs(int) with these headers;
    the oracle and the GPU take the floating-point absolute value.
"""
import numpy as np
import pytest

from helpers import poisson_system

R = pytest.importorskip("ref")
pytestmark = pytest.mark.skipif(not R.available(), reason="reference library not built (no reference tree)")


def _eq(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("dims", [(16, 16, 16), (24, 12, 10), (9, 17, 13)])
def test_solver_functions_equal_reference(oracle, dims):
    """applyCompressedMatrix, MIC(0) precond (z and its E, q scratch),
    CgSolver3D::solve (reference stopping test) and the masked BLAS-1."""
    S = poisson_system(oracle, 0, dims=dims, seed=4)
    A, an, act = S["adiag"], S["an"], S["active"]
    rng = np.random.default_rng(5)
    x, y = rng.uniform(-1, 1, dims), rng.uniform(-1, 1, dims)
    assert _eq(oracle.apply_matrix(A, an, x, act), R.apply_matrix(A, an, x, act))
    for tau, sigma in ((0.97, 0.25), (0.0, 0.25), (0.5, 0.9)):
        zo = oracle.mic_precond(A, an, x, act, tau, sigma, return_scratch=True)
        zr = R.mic_precond(A, an, x, act, tau, sigma, return_scratch=True)
        assert all(_eq(a, b) for a, b in zip(zo, zr)), (tau, sigma)
    for tol, mx in ((1e-6, 300), (1e-9, 300), (1e-6, 5)):
        po, reso, _ = oracle.pcg_solve(A, an, S["rhs"], act, tol=tol, max_iter=mx, criterion=0)
        pr, resr = R.cg_solve(A, an, S["rhs"], act, tol=tol, max_iter=mx)
        assert _eq(po, pr) and reso == resr, (tol, mx)
    assert oracle.dot(x, y, act) == R.dot(x, y, act)
    assert oracle.linf(x, act) == R.linf(x, act)
    a1, a2 = x.copy(), x.copy()
    oracle.saxpy(a1, y, 0.37, act)
    R.saxpy(a2, y, 0.37, act)
    assert _eq(a1, a2)
    c1, c2 = y.copy(), y.copy()
    oracle.scale_and_add(c1, x, -1.3, act)
    R.scale_and_add(c2, x, -1.3, act)
    assert _eq(c1, c2)


# buildSystem's `j < width - 1` (project-solver.cc:186) reads out of range when
# nx > ny and leaves the system asymmetric when nx < ny, where the reference's
# own asserts stop it (project-solver.cc:223, :41-57): cubic grids only.
@pytest.mark.parametrize("dims", [(16, 16, 16), (11, 11, 11)])
def test_build_system_and_project_equal_reference(oracle, dims):
    S = poisson_system(oracle, 0, dims=dims, seed=4)
    m = max(dims)
    h = 1.0 / m
    dt = 32.0 / 120.0 * h
    rng = np.random.default_rng(6)
    nx, ny, nz = dims
    u, v, w = rng.uniform(-1, 1, (nx + 1, ny, nz)), rng.uniform(-1, 1, (nx, ny + 1, nz)), rng.uniform(-1, 1, (nx, ny, nz + 1))
    for collider in (None, rng.uniform(-0.3, 1.0, dims) * 3 * h):
        so = oracle.build_system(dims, h, dt, u, v, w, S["sdf"], collider)
        sr = R.build_system(dims, h, dt, u, v, w, S["sdf"], collider)
        for k in ("adiag", "rhs", "active", "uwt", "vwt", "wwt"):
            assert _eq(so[k], sr[k]), k
        assert all(_eq(a, b) for a, b in zip(so["an"], sr["an"]))
        pg = rng.uniform(-1, 1, dims)
        po = oracle.project(dims, h, dt, u, v, w, pg, S["sdf"], so["uwt"], so["vwt"], so["wwt"])
        pr = R.project(dims, h, dt, u, v, w, pg, S["sdf"], sr["uwt"], sr["vwt"], sr["wwt"])
        assert all(_eq(a, b) for a, b in zip(po, pr))


@pytest.mark.parametrize("dims", [(12, 12, 12), (10, 14, 9)])
def test_transfers_equal_reference(oracle, dims):
    """solveP2G (FLIP, PIC), sampleVelocity, solveG2P (FLIP, PIC), advect with
    handleCollision (with and without a collider), SDF eval/grad, fractionInside.
    Particles include some outside the domain box."""
    m = max(dims)
    h = 1.0 / m
    rng = np.random.default_rng(7)
    n = 3000
    pos = rng.uniform(-0.05, 1.05, (n, 3)) * np.array(dims) * h
    vel = rng.normal(0, 1, (n, 3))
    for flip in (True, False):
        o, r = oracle.p2g(pos, vel, dims, h, flip), R.p2g(pos, vel, dims, h, flip)
        assert all(_eq(o[k], r[k]) for k in o), flip
    u, v, w = o["u"], o["v"], o["w"]
    assert _eq(oracle.sample_velocity(pos, dims, h, u, v, w), R.sample_velocity(pos, dims, h, u, v, w))
    ul, vl, wl = (0.5 * a + 0.1 for a in (u, v, w))
    assert _eq(oracle.g2p(pos, vel, dims, h, u, v, w, ul, vl, wl, alpha=0.95),
               R.g2p(pos, vel, dims, h, u, v, w, ul, vl, wl, alpha=0.95))
    assert _eq(oracle.g2p(pos, vel, dims, h, u, v, w, alpha=-1.0), R.g2p(pos, vel, dims, h, u, v, w, alpha=-1.0))
    for collider in (None, rng.uniform(-1, 1, dims) * 2 * h):
        po, vo = oracle.advect(pos, vel, dims, h, u, v, w, collider, 1.0 / 120)
        pr, vr = R.advect(pos, vel, dims, h, u, v, w, collider, 1.0 / 120)
        assert _eq(po, pr) and _eq(vo, vr)
    sdf = rng.uniform(-1, 1, dims) * 3 * h
    for p in rng.uniform(0, 1, (20, 3)) * np.array(dims) * h:
        assert oracle.sdf_eval(sdf, h, p) == R.sdf_eval(sdf, h, p)
        assert _eq(oracle.sdf_grad(sdf, h, p), R.sdf_grad(sdf, h, p))
    for c in rng.uniform(-1, 1, (300, 4)):
        assert oracle.fraction_inside(*c) == R.fraction_inside(*c)


# The reference's neighbour search indexes its bucket table by Morton code
# (ns-util.h:36-45), so it only runs on cubic power-of-two grids.
@pytest.mark.parametrize("n", [8, 16, 32])
def test_reconstruct_equals_reference_in_its_bucket_order(oracle, n):
    dims = (n, n, n)
    h = 1.0 / n
    pos = np.random.default_rng(n).uniform(-0.05, 1.05, (20000, 3))
    sr, vr = R.reconstruct(pos, dims, h, 0.8 * h)
    oracle.set_bucket_order(1)
    try:
        so, vo = oracle.reconstruct(pos, dims, h, 0.8 * h)
    finally:
        oracle.set_bucket_order(0)
    assert _eq(so, sr) and _eq(vo, vr)


@pytest.mark.parametrize("dims", [(12, 12, 12), (10, 14, 9)])
def test_rebuild_surface_equals_reference(oracle, dims):
    h = 1.0 / max(dims)
    sdf = np.random.default_rng(9).uniform(-1, 1, dims) * 3 * h
    c = (np.indices(dims).transpose(1, 2, 3, 0) + 0.5) * h - 0.5
    sphere = np.linalg.norm(c, axis=-1) - 0.3
    for f in (sdf, np.ascontiguousarray(sphere)):
        Vo, No, Io = oracle.rebuild_surface(f, h)
        Vr, Nr, Ir = R.rebuild_surface(f, h)
        assert len(Io) > 0 and _eq(Vo, Vr) and _eq(No, Nr) and _eq(Io, Ir)


def test_manifold_to_sdf_equals_reference_with_a_full_band(oracle):
    """With the exact band covering the grid, every cell holds its minimum over
    all triangles before the sweeps, which then change nothing under either
    reading of `abs`; distances, closest triangles and crossing counts match."""
    from simcraft_b200 import scenes
    cases = [(scenes.box_mesh((0.27, 0.31, 0.22), (0.71, 0.66, 0.74)), (12, 12, 12), 1.0 / 12, (0.0, 0.0, 0.0)),
             (scenes.icosphere(1, 0.3, (0.48, 0.52, 0.5)), (10, 11, 9), 0.1, (0.0, 0.0, 0.0)),
             (scenes.torus(10, 6, 0.28, 0.1, (0.5, 0.5, 0.5)), (11, 9, 10), 0.1, (0.03, 0.06, -0.02))]
    for (v, t), dims, h, origin in cases:
        o = oracle.manifold_to_sdf(v, t, dims, h, origin=origin, exact_band=max(dims))
        r = R.manifold_to_sdf(v, t, dims, h, origin=origin, exact_band=max(dims))
        assert all(_eq(a, b) for a, b in zip(o, r))


def test_reference_abs_on_doubles_binds_to_int(oracle):
    """Compiled here, the reference's CFL() takes int abs(int) of the face
    velocities: below 1 in magnitude they count as 0 and are skipped, so the
    CFL stays 5 * h / 1e-6; the oracle takes |u| (5 * h / max|u|)."""
    from simcraft_b200 import scenes
    m = 16
    pos, vel, h = scenes.dam_break(m, seed=1)
    r = R.Sim((m, m, m), h, len(pos), flip=True, flip_alpha=0.95)
    r.set_particles(pos, vel)
    cfg = oracle.default_config(m, m, m, h, flip_alpha=0.95)
    o = oracle.Sim(**cfg)
    o.set_particles(pos, vel)
    r.substep(1.0 / 120)
    o.substep(1.0 / 120)
    umax = max(np.abs(f).max() for f in o.faces())
    assert 0 < umax < 1
    assert r.cfl() == 5.0 * (h / 1e-6)
    assert o.cfl() == pytest.approx(5.0 * h / umax, rel=1e-12)


@pytest.mark.parametrize("m,frames,flip", [(16, 4, True), (16, 3, False), (32, 10, True)])
def test_simulator_equals_reference(oracle, m, frames, flip):
    """fluid::cpu::FluidSimulator::step itself against the oracle's simulator
    on the dam break (config 1 at 32^3: 65,536 particles, dt 1/120, FLIP 0.95,
    MIC(0)-PCG to the reference's absolute 1e-6, at most 200 iterations):
    pressure, positions, velocities, face grids and fluid SDF equal after every
    frame, with the reference's bucket order in the oracle."""
    from simcraft_b200 import scenes
    pos, vel, h = scenes.dam_break(m, seed=1)
    cfg = oracle.default_config(m, m, m, h, flip=int(flip), flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200)
    o = oracle.Sim(**cfg)
    o.set_particles(pos, vel)
    r = R.Sim((m, m, m), h, len(pos), flip=flip, flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200)
    r.set_particles(pos, vel)
    oracle.set_bucket_order(1)
    try:
        for f in range(frames):
            assert o.step(1.0 / 120) == r.step(1.0 / 120) == 1
            po, vo = o.particles()
            pr, vr = r.particles()
            assert _eq(o.pressure(), r.pressure()), f
            assert _eq(po, pr) and _eq(vo, vr), f
            assert all(_eq(a, b) for a, b in zip(o.faces(), r.faces())), f
            assert _eq(o.fluid_sdf(), r.fluid_sdf()), f
        assert np.abs(o.pressure()).max() > 0
    finally:
        oracle.set_bucket_order(0)
