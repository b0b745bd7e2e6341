"""Failure detection of the solver and the surface export, with the faults made
on the host (bad inputs), never on the GPU: NaN and Inf in the right-hand side
or the diagonal come back as SC_ERR_NONFINITE in both precisions and under both
stopping tests (never as a false convergence); a NaN outside the active set is
ignored, as the reference never reads it; an asymmetric matrix is refused when
checkSystemSymmetry is asked for; an all-air mask converges at once to zero
pressure; a singular enclosed fluid region never reports convergence; NaN and
Inf samples in an SDF give the oracle's mesh."""
import numpy as np
import pytest

from helpers import poisson_system

pytestmark = pytest.mark.gpu

SC_ERR_NONFINITE = -8
SC_ERR_ASYMMETRIC = -7
SC_ERR_BREAKDOWN = -4
SC_DONE_CONVERGED = 1


@pytest.fixture(scope="module")
def system(oracle, gpu):
    return poisson_system(oracle, 14, seed=6)


def _active_cell(S):
    return tuple(np.argwhere(S["active"] > 0)[len(np.argwhere(S["active"] > 0)) // 2])


def _solver(n, **kw):
    from simcraft_b200.solver import CgSolver3D

    return CgSolver3D(n, n, n, **kw)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("criterion", ["rel_l2", "abs_linf"])
def test_nonfinite_rhs_is_reported(system, bad, precision, criterion):
    from simcraft_b200._capi import CapiError
    from simcraft_b200.solver import CRIT_ABS_LINF, CRIT_REL_L2, PREC_FP64, PREC_MIXED

    S = system
    rhs = S["rhs"].copy()
    rhs[_active_cell(S)] = bad
    s = _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2 if criterion == "rel_l2" else CRIT_ABS_LINF,
                precision=PREC_FP64 if precision == "fp64" else PREC_MIXED)
    with pytest.raises(CapiError) as ei:
        s.solve(S["adiag"], S["an"], rhs, S["active"], np.zeros((14, 14, 14)))
    assert ei.value.status == SC_ERR_NONFINITE


def test_nan_diagonal_is_reported(system):
    from simcraft_b200._capi import CapiError
    from simcraft_b200.solver import CRIT_REL_L2

    S = system
    adiag = S["adiag"].copy()
    adiag[_active_cell(S)] = np.nan
    s = _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2)
    with pytest.raises(CapiError) as ei:
        s.solve(adiag, S["an"], S["rhs"], S["active"], np.zeros((14, 14, 14)))
    assert ei.value.status == SC_ERR_NONFINITE


def test_nan_outside_the_active_set_is_ignored(system):
    from simcraft_b200.solver import CRIT_REL_L2

    S = system
    rhs = S["rhs"].copy()
    inactive = np.argwhere(S["active"] == 0)
    assert len(inactive) > 0
    rhs[tuple(inactive[0])] = np.nan
    p_clean, p_bad = np.zeros((14, 14, 14)), np.zeros((14, 14, 14))
    _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2).solve(S["adiag"], S["an"], S["rhs"], S["active"],
                                                                     p_clean)
    _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2).solve(S["adiag"], S["an"], rhs, S["active"], p_bad)
    assert np.array_equal(p_clean, p_bad)


def test_asymmetric_matrix_is_refused(system):
    from simcraft_b200._capi import CapiError
    from simcraft_b200.solver import CRIT_REL_L2

    S = system
    act = S["active"] > 0
    cells = np.argwhere(act[:-1] & act[1:])  # active with an active +x neighbour
    an = [a.copy() for a in S["an"]]
    an[1][tuple(cells[0])] += 0.5
    s = _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2, check_symmetry=1)
    s.solve(S["adiag"], S["an"], S["rhs"], S["active"], np.zeros((14, 14, 14)))  # the symmetric one passes
    with pytest.raises(CapiError) as ei:
        s.solve(S["adiag"], an, S["rhs"], S["active"], np.zeros((14, 14, 14)))
    assert ei.value.status == SC_ERR_ASYMMETRIC


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_all_air_converges_to_zero(system, precision):
    from simcraft_b200.solver import CRIT_REL_L2, PREC_FP64, PREC_MIXED

    S = system
    s = _solver(14, tol=1e-8, max_iter=300, criterion=CRIT_REL_L2,
                precision=PREC_FP64 if precision == "fp64" else PREC_MIXED)
    pg = np.full((14, 14, 14), 7.0)
    res = s.solve(S["adiag"], S["an"], S["rhs"], np.zeros((14, 14, 14), np.uint8), pg)
    assert res == 0.0 and s.last_stats["iterations"] == 0 and s.last_stats["status"] == SC_DONE_CONVERGED
    assert not pg.any()


def test_singular_enclosed_fluid_never_converges(oracle, gpu):
    """Fluid everywhere, solid walls, no air: A is singular (constants span its
    null space) and a right-hand side with a non-zero mean has no solution.
    The solve stops at max_iter or reports a breakdown or a non-finite value;
    it never claims convergence."""
    from simcraft_b200._capi import CapiError
    from simcraft_b200.solver import CRIT_ABS_LINF

    n = 10
    h = 1.0 / n
    z = np.zeros
    S = oracle.build_system((n, n, n), h, 0.25 * h, z((n + 1, n, n)), z((n, n + 1, n)), z((n, n, n + 1)),
                            -np.ones((n, n, n)))
    assert S["active"].all()
    rhs = np.random.default_rng(12).uniform(0.5, 1.5, (n, n, n))
    s = _solver(n, tol=1e-6, max_iter=150, criterion=CRIT_ABS_LINF)
    try:
        res = s.solve(S["adiag"], S["an"], rhs, S["active"], np.zeros((n, n, n)))
    except CapiError as e:
        assert e.status in (SC_ERR_BREAKDOWN, SC_ERR_NONFINITE)
        return
    assert s.last_stats["status"] != SC_DONE_CONVERGED and not res < 1e-6


@pytest.mark.parametrize("path", ["host", "device"])
def test_surface_with_nan_and_inf_samples(oracle, gpu, path):
    import torch

    from simcraft_b200.surface import rebuild_surface

    rng = np.random.default_rng(31)
    n = 20
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    sdf = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) - 0.3
    u = rng.random(sdf.shape)
    sdf[u < 0.05] = np.nan
    sdf[(u >= 0.05) & (u < 0.1)] = np.inf
    sdf[(u >= 0.1) & (u < 0.12)] = -np.inf
    ref = oracle.rebuild_surface(sdf, h)
    got = rebuild_surface(torch.from_numpy(sdf).cuda() if path == "device" else sdf, h)
    V, N, I = (a.cpu().numpy() if hasattr(a, "cpu") else a for a in got)
    np.testing.assert_array_equal(V, ref[0])  # NaN where the oracle has NaN
    np.testing.assert_array_equal(N, ref[1])
    np.testing.assert_array_equal(I.astype(np.int64), ref[2].astype(np.int64))


SC_ERR_TIMEOUT = -6


def test_wavefront_wait_timeout_is_reported_and_the_solver_recovers(oracle, gpu):
    """The bounded waits of the wavefront sweeps: with the bound cut to one poll
    (sc_context_set_wait_limit), a consumer tile gives up on a mailbox its
    producer has not written yet; the solve returns SC_ERR_TIMEOUT in both
    precisions and through the preconditioner entry point, nothing faults, and
    with the default bound back the same handles solve again, bit for bit as a
    fresh solver does."""
    _timeout_round_trip(oracle, (64, 32, 48))  # 2 x 4 column tiles: mailbox hand-offs


def test_wavefront_wait_timeout_in_cluster_sweeps(oracle, gpu):
    """The same on a grid whose FP32 sweeps run in thread-block clusters (9 tile
    rows: a cluster of 8 and a partial one, 40% fluid): a ring wait, a mailbox wait or the
    backpressure wait gives up, the solve reports SC_ERR_TIMEOUT, and the handle
    solves again bit for bit."""
    _timeout_round_trip(oracle, (72, 72, 40), precond=False)


def _timeout_round_trip(oracle, dims, precond=True):
    import torch
    from simcraft_b200._capi import CapiError
    from simcraft_b200.solver import CgSolver3D, Context, CRIT_REL_L2, PREC_FP64, PREC_MIXED

    S = poisson_system(oracle, 0, dims=dims, seed=6)
    ctx = Context(0)
    fresh = {}
    for prec in (PREC_FP64, PREC_MIXED):
        f = CgSolver3D(*dims, tol=1e-8, max_iter=500, criterion=CRIT_REL_L2, precision=prec)
        fresh[prec] = np.zeros(dims)
        f.solve(S["adiag"], S["an"], S["rhs"], S["active"], fresh[prec])
    for prec in (PREC_FP64, PREC_MIXED):
        s = CgSolver3D(*dims, context=ctx, tol=1e-8, max_iter=500, criterion=CRIT_REL_L2, precision=prec)
        pg = np.zeros(dims)
        s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)  # graphs captured with the default bound
        for _ in range(2):
            ctx.set_wait_limit(1)
            with pytest.raises(CapiError) as ei:
                s.solve(S["adiag"], S["an"], S["rhs"], S["active"], np.zeros(dims))
            assert ei.value.status == SC_ERR_TIMEOUT
            ctx.set_wait_limit(0)
            pg = np.zeros(dims)
            s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
            assert s.last_stats["status"] == SC_DONE_CONVERGED
            np.testing.assert_array_equal(pg, fresh[prec])
    if not precond:
        return
    # the preconditioner entry point
    s = CgSolver3D(*dims, context=ctx)
    s.upload(S["adiag"], S["an"], S["rhs"], S["active"])
    x = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, dims)).cuda()
    z0 = torch.zeros(dims, dtype=torch.float64, device="cuda")
    s.precond(x, z0)
    ctx.set_wait_limit(1)
    with pytest.raises(CapiError) as ei:
        s.precond(x, torch.zeros_like(z0))
    assert ei.value.status == SC_ERR_TIMEOUT
    ctx.set_wait_limit(0)
    z1 = torch.zeros_like(z0)
    s.precond(x, z1)
    assert torch.equal(z0, z1)


def test_mesh_sweep_barrier_timeout_is_reported_and_recovers(gpu):
    """The bounded grid barrier of the collider's fast-sweeping launch: with the
    bound cut to one poll a block gives up waiting for the others; the call
    returns SC_ERR_TIMEOUT, and with the default bound back the same context
    builds the SDF bit for bit as before."""
    from simcraft_b200 import scenes
    from simcraft_b200._capi import CapiError
    from simcraft_b200.mesh import manifold_to_sdf
    from simcraft_b200.solver import Context

    ctx = Context(0)
    v, t = scenes.icosphere(3, 0.3, (0.5, 0.5, 0.5))
    n = 64
    ref = manifold_to_sdf(v, t, (n, n, n), 1.0 / n, context=ctx)
    ctx.set_wait_limit(1)
    with pytest.raises(CapiError) as ei:
        manifold_to_sdf(v, t, (n, n, n), 1.0 / n, context=ctx)
    assert ei.value.status == SC_ERR_TIMEOUT
    ctx.set_wait_limit(0)
    again = manifold_to_sdf(v, t, (n, n, n), 1.0 / n, context=ctx)
    np.testing.assert_array_equal(again, ref)
