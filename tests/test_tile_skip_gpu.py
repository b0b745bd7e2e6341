"""Sweeps over the tiles that hold active cells only.

The iteration sweeps skip every column tile (32 x 8 cells in x-y, all of z)
without an active cell.  These systems put the fluid in a box that leaves most
tiles empty, solve them with the FP64 and the mixed solver against the oracle,
and then give the same solver a second system whose fluid sits elsewhere, so
tiles that were swept become skipped and the reverse."""
import numpy as np
import pytest

from helpers import rel_l2
from simcraft_b200 import scenes

pytestmark = pytest.mark.gpu


def _box_system(O, dims, lo, hi, seed, dt_over_h=32.0 / 120.0):
    """buildSystem for a fluid box [lo, hi] (fractions of the longest side),
    solid walls, no collider, seeded rhs."""
    nx, ny, nz = dims
    h = 1.0 / max(dims)
    c = [(np.arange(k) + 0.5) * h for k in dims]
    X, Y, Z = np.meshgrid(*c, indexing="ij")
    sdf = np.maximum.reduce([lo[0] - X, X - hi[0], lo[1] - Y, Y - hi[1], lo[2] - Z, Z - hi[2]])
    sdf = np.ascontiguousarray(sdf)
    z = np.zeros
    S = O.build_system(dims, h, dt_over_h * h, z((nx + 1, ny, nz)), z((nx, ny + 1, nz)), z((nx, ny, nz + 1)), sdf)
    rhs, _ = scenes.poisson_rhs(S["active"], sdf, seed=seed)
    S["rhs"] = np.ascontiguousarray(rhs)
    return S


def _tiles_with_fluid(active):
    nx, ny, _ = active.shape
    ntx, nty = (nx + 31) // 32, (ny + 7) // 8
    t = np.zeros((ntx, nty), bool)
    for X in range(ntx):
        for Y in range(nty):
            t[X, Y] = active[32 * X:32 * X + 32, 8 * Y:8 * Y + 8].any()
    return t


# (dims, first box, second box): 96 x 64 x 40 has 3 x 8 tiles, the plain
# persistent sweep; 72 x 72 x 40 has 3 x 9 tiles, which the FP32 sweeps take
# in clusters of 8 tiles along y where the GPU runs them.  (nx >= ny: the
# buildSystem being restated gives non-symmetric systems on grids with nx < ny.)
CASES = [
    ((96, 64, 40), ((0.0, 0.0, 0.0), (0.35, 0.3, 1.0)), ((0.5, 0.2, 0.1), (1.0, 0.7, 0.9))),
    ((72, 72, 40), ((0.0, 0.0, 0.0), (0.4, 0.3, 1.0)), ((0.45, 0.5, 0.0), (0.9, 1.0, 0.5))),
]


@pytest.mark.parametrize("dims,box1,box2", CASES)
def test_solves_skip_tiles_without_fluid(oracle, gpu, dims, box1, box2):
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_FP64, PREC_MIXED
    solvers = {
        "fp64": CgSolver3D(*dims, tol=1e-8, max_iter=2000, criterion=CRIT_REL_L2, precision=PREC_FP64),
        "mixed": CgSolver3D(*dims, tol=1e-10, max_iter=2000, criterion=CRIT_REL_L2, precision=PREC_MIXED),
    }
    for k, (lo, hi) in enumerate((box1, box2)):
        S = _box_system(oracle, dims, lo, hi, seed=11 + k)
        a = S["active"].astype(bool)
        t = _tiles_with_fluid(a)
        assert 0 < t.sum() < t.size // 2 + 1, t  # most tiles hold no fluid
        p_ref, _, it_ref = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-8,
                                            max_iter=2000, criterion=1)
        p_tight, _, _ = oracle.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=1e-13,
                                         max_iter=4000, criterion=1)
        for name, s in solvers.items():
            pg = np.full(dims, 7.0)
            s.solve(S["adiag"], S["an"], S["rhs"], S["active"], pg)
            st = s.last_stats
            assert np.all(pg[~a] == 0.0), name  # inactive cells: zero pressure, as the reference leaves them
            if name == "fp64":
                assert abs(st["iterations"] - it_ref) <= 1, (k, st, it_ref)
                assert rel_l2(pg, p_ref, a) < 1e-5, k
            else:
                assert st["true_rel_l2"] < 1e-10, (k, st)
                assert rel_l2(pg, p_tight, a) < 1e-8, k


@pytest.mark.parametrize("dims,box1,box2", CASES[:1])
def test_precond_skips_tiles_without_fluid(oracle, gpu, dims, box1, box2):
    """z = M^-1 r with r non-zero everywhere, inactive cells included: the
    reference's preconditioner reads only active cells and leaves the others
    at zero."""
    import torch
    from simcraft_b200.solver import CgSolver3D
    s = CgSolver3D(*dims)
    rng = np.random.default_rng(3)
    for k, (lo, hi) in enumerate((box1, box2)):
        S = _box_system(oracle, dims, lo, hi, seed=21 + k)
        a = S["active"].astype(bool)
        s.upload(S["adiag"], S["an"], S["rhs"], S["active"])
        x = rng.uniform(-1, 1, dims)
        z_ref = oracle.mic_precond(S["adiag"], S["an"], x, S["active"])
        z = torch.zeros(dims, dtype=torch.float64, device="cuda")
        s.precond(torch.from_numpy(x).cuda(), z)
        zc = z.cpu().numpy()
        assert rel_l2(zc, z_ref, a) < 1e-12, k
        assert np.all(zc[~a] == 0.0), k
