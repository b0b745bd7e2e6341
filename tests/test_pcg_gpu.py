"""MIC(0)-PCG parity: the CUDA path (through the C-ABI) against the oracle."""
import numpy as np
import pytest

from helpers import poisson_system, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_mod(gpu):
    import torch
    return torch


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dims", [(16, 16, 16), (40, 20, 13), (33, 17, 40), (70, 9, 5)])
def test_apply_and_precond_match_oracle(oracle, torch_mod, dims):
    torch = torch_mod
    from simcraft_b200.solver import CgSolver3D
    S = poisson_system(oracle, 0, dims=dims, seed=4)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, dims)
    s = CgSolver3D(*dims)
    s.upload(S["adiag"], S["an"], S["rhs"], S["active"])
    b_ref = oracle.apply_matrix(S["adiag"], S["an"], x, S["active"])
    b = torch.zeros(dims, dtype=torch.float64, device="cuda")
    s.apply(_dev(torch, x), b)
    a = S["active"].astype(bool)
    assert np.abs(b.cpu().numpy() - b_ref)[a].max() <= 1e-12 * max(1.0, np.abs(b_ref).max())
    z_ref = oracle.mic_precond(S["adiag"], S["an"], x, S["active"])
    z = torch.zeros(dims, dtype=torch.float64, device="cuda")
    s.precond(_dev(torch, x), z)
    assert rel_l2(z.cpu().numpy(), z_ref, a) < 1e-12


@pytest.mark.parametrize("n,crit", [(16, 0), (32, 1), (48, 1)])
def test_pcg_fp64_matches_oracle(oracle, torch_mod, n, crit):
    from simcraft_b200.solver import CgSolver3D
    S = poisson_system(oracle, n, seed=2)
    tol = 1e-6 if crit == 0 else 1e-8
    p_ref, res_ref, it_ref = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=tol,
                                              max_iter=500, criterion=crit)
    s = CgSolver3D(n, n, n, tol=tol, max_iter=500, criterion=crit)
    pg = np.zeros((n, n, n))
    res = s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
    st = s.last_stats
    assert abs(st["iterations"] - it_ref) <= 1, (st, it_ref)
    assert res < tol
    a = S["active"].astype(bool)
    assert rel_l2(pg, p_ref, a) < 1e-5


def test_pcg_mixed_reaches_1e10(oracle, torch_mod):
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_MIXED
    n = 32
    S = poisson_system(oracle, n, seed=2)
    p_ref, _, _ = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-12, max_iter=1000,
                                   criterion=1)
    s = CgSolver3D(n, n, n, tol=1e-10, max_iter=1000, criterion=CRIT_REL_L2, precision=PREC_MIXED)
    pg = np.zeros((n, n, n))
    s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
    st = s.last_stats
    assert st["true_rel_l2"] < 1e-10, st
    a = S["active"].astype(bool)
    assert rel_l2(pg, p_ref, a) < 1e-8


@pytest.mark.parametrize("dims", [(32, 32, 32), (40, 20, 13), (33, 17, 40)])
@pytest.mark.parametrize("crit,tol", [(1, 1e-10), (0, 1e-6)])
def test_pcg_mixed_inner_methods(oracle, torch_mod, dims, crit, tol):
    """Both FP32 inner iterations of the mixed solve (the reference's PCG step and
    Eisenstat's split form, which applies L^-1 A L^-T with two sweeps and no
    SpMV) meet the FP64 stopping test and agree with the oracle's solution."""
    from simcraft_b200.solver import CgSolver3D, INNER_EISENSTAT, INNER_PCG, PREC_MIXED
    S = poisson_system(oracle, 0, dims=dims, seed=6)
    p_ref, _, _ = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-13, max_iter=2000,
                                   criterion=1)
    a = S["active"].astype(bool)
    iters = {}
    for meth in (INNER_PCG, INNER_EISENSTAT):
        s = CgSolver3D(*dims, tol=tol, max_iter=2000, criterion=crit, precision=PREC_MIXED, inner_method=meth)
        pg = np.zeros(dims)
        res = s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
        st = s.last_stats
        assert st["status"] == 1 and res < tol, st
        if crit == 1:
            assert st["true_rel_l2"] < tol, st
            assert rel_l2(pg, p_ref, a) < 1e-8
        else:
            assert st["true_linf"] < tol, st
        iters[meth] = st["iterations"]
    assert iters[INNER_EISENSTAT] <= 1.3 * iters[INNER_PCG] + 5, iters


def test_pcg_mixed_eisenstat_zero_rhs(oracle, torch_mod):
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_MIXED
    n = 24
    S = poisson_system(oracle, n, seed=2)
    s = CgSolver3D(n, n, n, tol=1e-8, max_iter=100, criterion=CRIT_REL_L2, precision=PREC_MIXED)
    pg = np.full((n, n, n), 7.0)
    s.solve(S["adiag"], S["an"], np.zeros((n, n, n)), S["active"], pg)
    assert s.last_stats["status"] == 1 and s.last_stats["iterations"] == 0
    assert not pg[S["active"].astype(bool)].any()


def test_pcg_and_precond_match_the_reference_code(oracle, torch_mod):
    """Against the reference's own CgSolver3D::solve and
    ModifiedIncompleteCholesky3D::precond (oracle/_ref, built from the reference
    sources): its stopping test (absolute L-inf 1e-6, at most 300 iterations),
    iteration counts within 1, pressure within 1e-5 relative L2."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import ref as R
    if not R.available():
        pytest.skip("reference library not built")
    torch = torch_mod
    from simcraft_b200.solver import CgSolver3D
    for dims in [(32, 32, 32), (40, 20, 13)]:
        S = poisson_system(oracle, 0, dims=dims, seed=2)
        a = S["active"].astype(bool)
        st = {}
        p_ref, res_ref = R.cg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-6, max_iter=300, stats=st)
        s = CgSolver3D(*dims, tol=1e-6, max_iter=300, criterion=0)
        pg = np.zeros(dims)
        res = s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
        assert st["iterations"] > 10 and abs(s.last_stats["iterations"] - st["iterations"]) <= 1, (st, s.last_stats)
        assert res < 1e-6 and res_ref < 1e-6
        assert rel_l2(pg, p_ref, a) < 1e-5
        x = np.random.default_rng(3).uniform(-1, 1, dims)
        z = torch.zeros(dims, dtype=torch.float64, device="cuda")
        s.precond(_dev(torch, x), z)
        assert rel_l2(z.cpu().numpy(), R.mic_precond(S["adiag"], S["an"], x, S["active"]), a) < 1e-12


def test_config2_128_sphere_pool(oracle, torch_mod):
    """The standalone 128^3 system of the benchmark (24 seeded spheres at 50%
    fill, dt/h = 32/120, rhs U[-1,1] mean-subtracted per enclosed component):
    the FP64 solve to 1e-8 relative within 1 iteration of the oracle and within
    1e-6 of its solution; the mixed solve to 1e-8 within 1e-7 relative L2 of the
    oracle's FP64 solution to 1e-12 (the exact solution to ~1e-12), and to 1e-10
    within 1e-9."""
    from simcraft_b200 import scenes
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_FP64, PREC_MIXED
    n = 128
    h = 1.0 / n
    sdf, info = scenes.sphere_pool(n, count=24, rmin=0.05, rmax=0.2, fill=0.5, seed=2)
    sdf = np.ascontiguousarray(sdf)
    z = np.zeros
    S = oracle.build_system((n, n, n), h, 32.0 / 120.0 * h, z((n + 1, n, n)), z((n, n + 1, n)), z((n, n, n + 1)),
                            sdf)
    rhs, _ = scenes.poisson_rhs(S["active"], sdf, seed=3)
    rhs = np.ascontiguousarray(rhs)
    a = S["active"].astype(bool)
    assert 0.45 < a.mean() < 0.55
    oracle.set_parity_mode(False)
    try:
        p8, _, it8 = oracle.pcg_solve(S["adiag"], S["an"], rhs, S["active"], tol=1e-8, max_iter=2000, criterion=1)
        p12, _, _ = oracle.pcg_solve(S["adiag"], S["an"], rhs, S["active"], tol=1e-12, max_iter=4000, criterion=1)
    finally:
        oracle.set_parity_mode(True)
    s = CgSolver3D(n, n, n, tol=1e-8, max_iter=2000, criterion=CRIT_REL_L2, precision=PREC_FP64)
    pg = np.zeros((n, n, n))
    s.solve(S["adiag"], S["an"], rhs, S["active"], pg)
    assert abs(s.last_stats["iterations"] - it8) <= 1, (s.last_stats, it8)
    assert s.last_stats["true_rel_l2"] < 1e-8
    assert rel_l2(pg, p8, a) < 1e-6
    for tol, bound in ((1e-8, 1e-7), (1e-10, 1e-9)):
        m = CgSolver3D(n, n, n, tol=tol, max_iter=4000, criterion=CRIT_REL_L2, precision=PREC_MIXED)
        pm = np.zeros((n, n, n))
        m.solve(S["adiag"], S["an"], rhs, S["active"], pm)
        assert m.last_stats["status"] == 1 and m.last_stats["true_rel_l2"] < tol, m.last_stats
        assert rel_l2(pm, p12, a) < bound, (tol, rel_l2(pm, p12, a))


# nx >= ny throughout: the reference's buildSystem bounds its up faces by the
# width (project-solver.cc:186), which leaves nx < ny systems asymmetric
@pytest.mark.parametrize("dims", [(64, 64, 40), (72, 72, 40), (128, 128, 24), (136, 136, 20)])
def test_pcg_mixed_cluster_sweeps(oracle, torch_mod, dims):
    """Grids whose column tiles fill thread-block clusters along y (tiles of 8
    rows: ny = 64 fills one cluster of 8, 72 gives a cluster of 8 and a partial
    one, 128 fills one of 16, 136 leaves CTAs of its second cluster of 16
    without a tile), so the FP32 sweeps of the mixed solve hand their y
    boundary rows through distributed shared memory: both inner iterations meet
    the FP64 stopping test and agree with the oracle's solution."""
    from simcraft_b200.solver import CgSolver3D, INNER_EISENSTAT, INNER_PCG, PREC_MIXED
    S = poisson_system(oracle, 0, dims=dims, seed=6)
    assert S["active"].mean() > 0.1
    p_ref, _, _ = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-13, max_iter=3000,
                                   criterion=1)
    a = S["active"].astype(bool)
    for meth in (INNER_EISENSTAT, INNER_PCG):
        s = CgSolver3D(*dims, tol=1e-10, max_iter=3000, criterion=1, precision=PREC_MIXED, inner_method=meth)
        pg = np.zeros(dims)
        s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
        st = s.last_stats
        assert st["status"] == 1 and st["true_rel_l2"] < 1e-10, (meth, st)
        assert rel_l2(pg, p_ref, a) < 1e-8
        # the solve is deterministic: the same handle solves again bit for bit
        pg2 = np.zeros(dims)
        s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg2)
        np.testing.assert_array_equal(pg, pg2)
