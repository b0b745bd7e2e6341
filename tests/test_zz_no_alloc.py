"""The allocation-free MIC(0) preconditioner (sc_mic_precond_noalloc_device).

It serves callers that cannot call cudaMalloc (engines whose device memory is
owned by their own pool allocator, hot loops that cannot afford cudaMalloc's
device-wide synchronisation): its scratch is a static device array inside the
library.  This checks it against the allocating entry point
(sc_pcg_precond_device) on two calls in a row, and that grids beyond the
array's limit are rejected with a message.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import poisson_system, rel_l2

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("dims", [(32, 32, 32), (40, 20, 13)])
def test_noalloc_precond_matches_allocating_entry_point(oracle, gpu, dims):
    import torch
    from simcraft_b200 import _capi
    from simcraft_b200.solver import CgSolver3D, default_context

    S = poisson_system(oracle, 0, dims=dims, seed=6)
    ctx = default_context()
    L = _capi.lib()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    adiag, act = dev(S["adiag"]), dev(S["active"])
    an = [dev(a) for a in S["an"]]
    an_ptrs = _capi.ptr_array([_p(a) for a in an])
    ref = CgSolver3D(*dims)
    ref.upload(S["adiag"], S["an"], S["rhs"], S["active"])
    rng = np.random.default_rng(12)
    a = S["active"].astype(bool)
    for call in range(2):  # two calls in a row share (and must reset) the static scratch
        r = dev(rng.uniform(-1, 1, dims))
        z_ref = torch.zeros(dims, dtype=torch.float64, device="cuda")
        ref.precond(r, z_ref)
        z = torch.full(dims, float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.sc_mic_precond_noalloc_device(ctx.handle, *dims, _p(adiag), an_ptrs, _p(r), _p(act), _p(z),
                                             0.97, 0.25)
        _capi.check("sc_mic_precond_noalloc_device", rc, ctx.handle)
        zr, zn = z_ref.cpu().numpy(), z.cpu().numpy()
        assert np.isfinite(zn[a]).all()
        assert rel_l2(zn, zr, a) < 1e-12, (call, rel_l2(zn, zr, a))
        # and against the CPU restatement of the reference
        assert rel_l2(zn, oracle.mic_precond(S["adiag"], S["an"], r.cpu().numpy(), S["active"]), a) < 1e-12


def test_noalloc_rejects_grids_beyond_its_limit(gpu):
    import torch
    from simcraft_b200 import _capi
    from simcraft_b200.solver import default_context

    ctx = default_context()
    L = _capi.lib()
    dims = (64, 64, 64)  # 262144 tiled cells > 32768
    x = torch.zeros(dims, dtype=torch.float64, device="cuda")
    act = torch.zeros(dims, dtype=torch.uint8, device="cuda")
    an = _capi.ptr_array([_p(x)] * 6)
    rc = L.sc_mic_precond_noalloc_device(ctx.handle, *dims, _p(x), an, _p(x), _p(act), _p(x), 0.97, 0.25)
    assert rc == -1  # SC_ERR_INVALID
    assert b"too large" in L.sc_context_last_error(ctx.handle)


def test_noalloc_ignores_nonfinite_entries_the_reference_never_reads(oracle, gpu):
    """NaN in an inactive cell's row and in a coupling to an inactive cell:
    the reference never reads them (it tests activity first), so z stays finite
    and equals the allocating entry point's, as for a clean system."""
    import torch
    from simcraft_b200 import _capi
    from simcraft_b200.solver import CgSolver3D, default_context

    dims = (32, 32, 32)
    S = poisson_system(oracle, 0, dims=dims, seed=6)
    act = S["active"].astype(bool)
    inactive = tuple(np.argwhere(~act)[0])
    # an active cell whose x-neighbour below is inactive
    cand = np.argwhere(act[1:] & ~act[:-1])
    cell = (cand[0][0] + 1, cand[0][1], cand[0][2])
    adiag = S["adiag"].copy()
    an = [a.copy() for a in S["an"]]
    adiag[inactive] = np.nan
    for a in an:
        a[inactive] = np.nan
    an[0][cell] = np.nan  # Left coupling of `cell` to the inactive cell below it
    ctx = default_context()
    L = _capi.lib()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_adiag, d_act = dev(adiag), dev(S["active"])
    d_an = [dev(a) for a in an]
    ref = CgSolver3D(*dims)
    ref.upload(adiag, an, S["rhs"], S["active"])
    r = dev(np.random.default_rng(13).uniform(-1, 1, dims))
    z_ref = torch.zeros(dims, dtype=torch.float64, device="cuda")
    ref.precond(r, z_ref)
    z = torch.full(dims, float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.sc_mic_precond_noalloc_device(ctx.handle, *dims, _p(d_adiag), _capi.ptr_array([_p(a) for a in d_an]),
                                         _p(r), _p(d_act), _p(z), 0.97, 0.25)
    _capi.check("sc_mic_precond_noalloc_device", rc, ctx.handle)
    zn, zr = z.cpu().numpy(), z_ref.cpu().numpy()
    assert np.isfinite(zn[act]).all() and np.isfinite(zr[act]).all()
    assert rel_l2(zn, zr, act) < 1e-12
    clean = oracle.mic_precond(S["adiag"], S["an"], r.cpu().numpy(), S["active"])
    assert rel_l2(zn, clean, act) < 1e-12
