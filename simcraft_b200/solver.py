"""Python mirror of the reference's pressure-solver seams, backed by the CUDA
library through the C-ABI.

  CgSolver3D(w, h, d).solve(Adiag, Aneighbour, rhs, active, pg) -> residual
      (FluidSim/include/FluidSim/cpu/project-solver.h:100-131)
  ModifiedIncompleteCholesky3D.precond(Adiag, Aneighbour, r, active, z)
      (project-solver.h:81-98)
  apply_compressed_matrix(Adiag, Aneighbour, x, active, b)
      (FluidSim/src/cpu/project-solver.cc:16-39)

Arrays are numpy (host) or torch CUDA tensors (device), in the reference's
z-fastest layout; Aneighbour is the list of 6 arrays in the Directions order
Left, Right, Up, Down, Front, Back.
"""
import ctypes

import numpy as np

from . import _capi
from ._capi import check, lib, ptr_array

LEFT, RIGHT, UP, DOWN, FRONT, BACK = range(6)
CRIT_ABS_LINF, CRIT_REL_L2 = _capi.SC_CRIT_ABS_LINF, _capi.SC_CRIT_REL_L2
PREC_FP64, PREC_MIXED = _capi.SC_PREC_FP64, _capi.SC_PREC_MIXED
INNER_PCG, INNER_EISENSTAT = _capi.SC_INNER_PCG, _capi.SC_INNER_EISENSTAT

_contexts = {}


class Context:
    """One CUDA stream on one device (sc_context)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check("sc_context_create", lib().sc_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device

    def synchronize(self):
        check("sc_context_synchronize", lib().sc_context_synchronize(self.handle), self.handle)

    def set_stream(self, stream_ptr):
        """Order later work on `stream_ptr` (None/0 = the legacy default stream)."""
        check("sc_context_set_stream", lib().sc_context_set_stream(self.handle, stream_ptr), self.handle)

    def use_own_stream(self):
        check("sc_context_use_own_stream", lib().sc_context_use_own_stream(self.handle), self.handle)

    @property
    def stream(self):
        return lib().sc_context_stream(self.handle)

    def set_wait_limit(self, polls):
        """Bound the device spin-waits of later calls to `polls` polls (<= 0: the
        defaults); a wait that reaches it makes the call fail with SC_ERR_TIMEOUT."""
        check("sc_context_set_wait_limit", lib().sc_context_set_wait_limit(self.handle, int(polls)), self.handle)

    def __del__(self):
        if getattr(self, "handle", None) and _capi._lib is not None:
            _capi._lib.sc_context_destroy(self.handle)
            self.handle = None


def default_context(device=0):
    if device not in _contexts:
        _contexts[device] = Context(device)
    return _contexts[device]


def default_options(**kw):
    o = _capi.sc_pcg_options()
    lib().sc_pcg_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def _is_torch(a):
    return type(a).__module__.startswith("torch")


class _on_torch_stream:
    """Runs device-pointer calls on torch's current CUDA stream, so they are
    ordered with the torch operations that produced and consume the tensors."""

    def __init__(self, ctx, tensor):
        self.ctx, self.tensor = ctx, tensor

    def __enter__(self):
        import torch

        self.ctx.set_stream(ctypes.c_void_p(torch.cuda.current_stream(self.tensor.device).cuda_stream))

    def __exit__(self, *exc):
        self.ctx.use_own_stream()
        return False


def _ptr(a):
    if _is_torch(a):
        assert a.is_cuda and a.is_contiguous(), "device arrays must be contiguous CUDA tensors"
        return ctypes.c_void_p(a.data_ptr())
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


def _prep_host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class CgSolver3D:
    """CgSolver3D + ModifiedIncompleteCholesky3D on the B200.

    `tolerance`/`max_iterations` default to the reference's 1e-6 / 300 and its
    absolute L-inf stopping test; `precision` selects plain FP64 or the mixed
    FP32-inner / FP64-defect-correction solve."""

    def __init__(self, w, h, d, context=None, **opts):
        self.ctx = context or default_context()
        self.shape = (w, h, d)
        self.opts = default_options(**opts)
        hnd = ctypes.c_void_p()
        check("sc_pcg_create", lib().sc_pcg_create(self.ctx.handle, w, h, d, ctypes.byref(self.opts),
                                                   ctypes.byref(hnd)), self.ctx.handle)
        self.handle = hnd
        self.last_stats = None

    def __del__(self):
        if getattr(self, "handle", None) and _capi._lib is not None:
            _capi._lib.sc_pcg_destroy(self.handle)
            self.handle = None

    def set_options(self, **kw):
        for k, v in kw.items():
            setattr(self.opts, k, v)
        check("sc_pcg_set_options", lib().sc_pcg_set_options(self.handle, ctypes.byref(self.opts)),
              self.ctx.handle)

    # -- reference signature -------------------------------------------------
    def solve(self, Adiag, Aneighbour, rhs, active, pg):
        """Solves A pg = rhs in place of pg; returns the residual in the
        configured stopping measure (what CgSolver3D::solve returns)."""
        st = _capi.sc_pcg_stats()
        if _is_torch(pg):
            fn = "sc_pcg_solve_device"
            an = ptr_array([_ptr(a) for a in Aneighbour])
            with _on_torch_stream(self.ctx, pg):
                rc = lib().sc_pcg_solve_device(self.handle, _ptr(Adiag), an, _ptr(rhs), _ptr(active), _ptr(pg),
                                               ctypes.byref(st))
        else:
            fn = "sc_pcg_solve_host"
            Adiag = _prep_host(Adiag, np.float64)
            Aneighbour = [_prep_host(a, np.float64) for a in Aneighbour]
            rhs = _prep_host(rhs, np.float64)
            active = _prep_host(active, np.uint8)
            assert pg.dtype == np.float64 and pg.flags.c_contiguous
            an = ptr_array([_ptr(a) for a in Aneighbour])
            rc = lib().sc_pcg_solve_host(self.handle, _ptr(Adiag), an, _ptr(rhs), _ptr(active), _ptr(pg),
                                         ctypes.byref(st))
        self.last_stats = st.as_dict()
        check(fn, rc, self.ctx.handle)
        return st.residual

    # -- resident form (benchmarks, repeated solves) ------------------------
    def upload(self, Adiag, Aneighbour, rhs, active):
        dev = _is_torch(Adiag)
        if not dev:
            Adiag = _prep_host(Adiag, np.float64)
            Aneighbour = [_prep_host(a, np.float64) for a in Aneighbour]
            rhs = _prep_host(rhs, np.float64)
            active = _prep_host(active, np.uint8)
        self._keep = (Adiag, Aneighbour, rhs, active)
        an = ptr_array([_ptr(a) for a in Aneighbour])
        if dev:
            with _on_torch_stream(self.ctx, Adiag):
                rc = lib().sc_pcg_upload(self.handle, _ptr(Adiag), an, _ptr(rhs), _ptr(active), 1)
                self.ctx.synchronize()
        else:
            rc = lib().sc_pcg_upload(self.handle, _ptr(Adiag), an, _ptr(rhs), _ptr(active), 0)
        check("sc_pcg_upload", rc, self.ctx.handle)

    def upload_rhs(self, rhs):
        dev = _is_torch(rhs)
        if not dev:
            rhs = _prep_host(rhs, np.float64)
            check("sc_pcg_upload_rhs", lib().sc_pcg_upload_rhs(self.handle, _ptr(rhs), 0), self.ctx.handle)
            return
        with _on_torch_stream(self.ctx, rhs):
            check("sc_pcg_upload_rhs", lib().sc_pcg_upload_rhs(self.handle, _ptr(rhs), 1), self.ctx.handle)
            self.ctx.synchronize()

    def solve_resident(self):
        st = _capi.sc_pcg_stats()
        rc = lib().sc_pcg_solve_resident(self.handle, ctypes.byref(st))
        self.last_stats = st.as_dict()
        check("sc_pcg_solve_resident", rc, self.ctx.handle)
        return self.last_stats

    def download(self, pg):
        if _is_torch(pg):
            with _on_torch_stream(self.ctx, pg):
                check("sc_pcg_download", lib().sc_pcg_download(self.handle, _ptr(pg), 1), self.ctx.handle)
        else:
            check("sc_pcg_download", lib().sc_pcg_download(self.handle, _ptr(pg), 0), self.ctx.handle)
        return pg

    def precond(self, r, z):
        """ModifiedIncompleteCholesky3D::precond on the uploaded system (device tensors)."""
        with _on_torch_stream(self.ctx, z):
            check("sc_pcg_precond_device", lib().sc_pcg_precond_device(self.handle, _ptr(r), _ptr(z)),
                  self.ctx.handle)
        return z

    def apply(self, x, b):
        """applyCompressedMatrix on the uploaded system (device tensors)."""
        with _on_torch_stream(self.ctx, b):
            check("sc_pcg_apply_device", lib().sc_pcg_apply_device(self.handle, _ptr(x), _ptr(b)),
                  self.ctx.handle)
        return b
