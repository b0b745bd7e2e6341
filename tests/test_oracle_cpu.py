"""The CPU oracle (a restatement of the reference's CPU path) against
known answers, the semantics the reference's own CUDA test expects
(FluidSim/tests/test-fluid-utils.cu), and committed golden fixtures."""
import os

import numpy as np
import pytest

from helpers import poisson_system

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("corners,expected", [
    ((1.0, 1.0, 1.0, 1.0), 0.0),
    ((-1.0, -1.0, -1.0, -1.0), 1.0),
    ((-1.0, 1.0, 1.0, -1.0), 0.5),      # straight edge through the middle
    ((-1.0, -1.0, 1.0, 1.0), 0.5),
    ((-1.0, 1.0, 1.0, 1.0), 0.125),     # corner triangle with legs 1/2, 1/2
    ((1.0, -1.0, -1.0, -1.0), 0.875),
])
def test_fraction_inside_known_answers(oracle, corners, expected):
    assert abs(oracle.fraction_inside(*corners) - expected) < 1e-15


def test_cubic_bspline_partition_of_unity(oracle):
    rng = np.random.default_rng(0)
    for x in rng.uniform(-3, 3, 50):
        s = sum(oracle.cubic_weight(1.0, (x - i, 0.0, 0.0)) for i in range(-6, 7))
        assert abs(s / oracle.cubic_weight(1.0, (0.0, 0.0, 0.0)) * (2.0 / 3.0) - 1.0) < 1e-12


def test_blas_semantics_match_reference_test(oracle):
    # FluidSim/tests/test-fluid-utils.cu: masked saxpy x + a*y, FP64 dot, masked L-inf.
    rng = np.random.default_rng(1)
    x = rng.uniform(-100, 100, (10, 10, 10))
    y = rng.uniform(-100, 100, (10, 10, 10))
    act = (rng.random((10, 10, 10)) < 0.5).astype(np.uint8)
    a = x.copy()
    oracle.saxpy(a, y, 10.0, act)
    np.testing.assert_allclose(a, np.where(act, x + 10.0 * y, x), rtol=0, atol=1e-12)
    assert abs(oracle.dot(x, y, act) - float(np.sum(x * y * act))) < 1e-8
    assert oracle.linf(x, act) == np.abs(x * act).max()
    # scaleAndAdd follows the CPU (util.cc:404-410): c = a + x*c on active cells
    c = y.copy()
    oracle.scale_and_add(c, x, 0.5, act)
    np.testing.assert_allclose(c, np.where(act, x + 0.5 * y, y), rtol=0, atol=1e-12)


def test_mic_preconditioner_is_symmetric(oracle):
    S = poisson_system(oracle, 12, seed=5)
    rng = np.random.default_rng(2)
    a = rng.standard_normal(S["adiag"].shape) * S["active"]
    b = rng.standard_normal(S["adiag"].shape) * S["active"]
    ma = oracle.mic_precond(S["adiag"], S["an"], a, S["active"])
    mb = oracle.mic_precond(S["adiag"], S["an"], b, S["active"])
    assert abs(np.sum(b * ma) - np.sum(a * mb)) < 1e-10 * np.linalg.norm(ma) * np.linalg.norm(b)
    assert np.sum(a * ma) > 0  # positive definite


def test_pcg_reference_iteration_semantics(oracle):
    S = poisson_system(oracle, 12, seed=5)
    # a tolerance above the initial residual returns before preconditioning (iter 0)
    _, res, it = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e9)
    assert it == 0
    # max_iter bounds the loop at max_iter - 1 SpMVs; `iter` then equals max_iter
    _, res, it = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=0.0, max_iter=5)
    assert it == 5
    p, res, it = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-10, max_iter=500,
                                  criterion=oracle.CRIT_REL_L2)
    r = S["rhs"] - oracle.apply_matrix(S["adiag"], S["an"], p, S["active"])
    act = S["active"].astype(bool)
    assert np.linalg.norm(r[act]) / np.linalg.norm(S["rhs"][act]) < 1e-10


def test_build_system_is_symmetric(oracle):
    S = poisson_system(oracle, 16, seed=7)
    an, act = S["an"], S["active"].astype(bool)
    # A_Right(p) == A_Left(p+x) wherever both cells are active (checkSystemSymmetry)
    both = act[:-1] & act[1:]
    assert np.array_equal(an[1][:-1][both], an[0][1:][both])
    both = act[:, :-1] & act[:, 1:]
    assert np.array_equal(an[2][:, :-1][both], an[3][:, 1:][both])
    both = act[:, :, :-1] & act[:, :, 1:]
    assert np.array_equal(an[4][:, :, :-1][both], an[5][:, :, 1:][both])


def test_golden_fixtures(oracle):
    path = os.path.join(GOLDEN, "oracle_golden.npz")
    g = np.load(path)
    S = poisson_system(oracle, int(g["n"]), seed=int(g["seed"]))
    np.testing.assert_array_equal(S["active"], g["active"])
    np.testing.assert_allclose(S["adiag"], g["adiag"], rtol=0, atol=0)
    p, res, it = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-8, max_iter=500,
                                  criterion=oracle.CRIT_REL_L2)
    assert it == int(g["iters"])
    np.testing.assert_allclose(p, g["pressure"], rtol=1e-12, atol=1e-14)
    pos = g["p2g_pos"]
    out = oracle.p2g(pos, g["p2g_vel"], (8, 8, 8), 1.0 / 8, flip=True)
    for k in ("u", "v", "w", "uw"):
        np.testing.assert_allclose(out[k], g["p2g_" + k], rtol=1e-13, atol=1e-15)


def test_dam_break_step_invariants(oracle):
    from simcraft_b200 import scenes
    n = 16
    pos, vel, h = scenes.dam_break(n, seed=1)
    sim = oracle.Sim(**oracle.default_config(n, n, n, h, flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200,
                                             pcg_criterion=oracle.CRIT_REL_L2))
    sim.set_particles(pos, vel)
    for _ in range(3):
        assert sim.step(1.0 / 120) == 1
    p, v = sim.particles()
    assert np.isfinite(p).all() and np.isfinite(v).all()
    assert p.min() >= 0.0 and p.max() <= 1.0
    assert v[:, 1].mean() < 0  # gravity pulls the column down


def test_timing_mode_does_the_same_work(oracle):
    """bench.py times the oracle in its timing mode (parallel P2G with
    per-thread accumulation, OpenMP where the reference uses TBB).  That mode
    must compute what the parity mode computes, up to summation order: P2G
    grids, then a whole simulated frame."""
    from simcraft_b200 import scenes

    pos, vel, h = scenes.dam_break(16, seed=2)
    vel = np.random.default_rng(3).uniform(-1, 1, pos.shape)
    threads = oracle.get_threads()
    try:
        oracle.set_threads(max(4, threads))
        oracle.set_parity_mode(True)
        a = oracle.p2g(pos, vel, (16, 16, 16), h)
        cfg = oracle.default_config(16, 16, 16, h, pcg_tol=1e-10, pcg_criterion=1)
        s1 = oracle.Sim(**cfg)
        s1.set_particles(pos, vel)
        s1.step(1.0 / 120)
        oracle.set_parity_mode(False)
        b = oracle.p2g(pos, vel, (16, 16, 16), h)
        s2 = oracle.Sim(**cfg)
        s2.set_particles(pos, vel)
        s2.step(1.0 / 120)
    finally:
        oracle.set_parity_mode(True)
        oracle.set_threads(threads)
    for k in ("u", "v", "w", "uw", "vw", "ww"):
        np.testing.assert_allclose(b[k], a[k], rtol=1e-12, atol=1e-14)
    for k in ("uvalid", "vvalid", "wvalid"):
        assert np.array_equal(a[k], b[k])
    p1, p2 = s1.pressure(), s2.pressure()
    assert np.linalg.norm(p2 - p1) / np.linalg.norm(p1) < 1e-8
    assert np.abs(s2.particles()[0] - s1.particles()[0]).max() < 1e-8 * h
