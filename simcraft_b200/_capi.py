"""ctypes declarations of include/simcraft_fluid_capi.h (the only way Python
reaches the CUDA path).  Loading fails loudly when libsimcraft_fluid.so is
missing: there is no fallback implementation."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsimcraft_fluid.so")

c_int, c_double, c_int64, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p
c_char_p = ctypes.c_char_p
P = ctypes.POINTER


class sc_pcg_options(ctypes.Structure):
    _fields_ = [("tol", c_double), ("max_iter", c_int), ("criterion", c_int), ("precision", c_int),
                ("mic_tau", c_double), ("mic_sigma", c_double), ("inner_rtol", c_double),
                ("max_outer", c_int), ("check_symmetry", c_int), ("true_residual", c_int)]


class sc_pcg_stats(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("outer", c_int), ("status", c_int), ("residual", c_double),
                ("true_rel_l2", c_double), ("true_linf", c_double), ("ms", c_double),
                ("sym_err", c_double), ("device_flags", ctypes.c_uint),
                ("kernel_launches", c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


SC_OK = 0
SC_CRIT_ABS_LINF, SC_CRIT_REL_L2 = 0, 1
SC_PREC_FP64, SC_PREC_MIXED = 0, 1
SC_REAL_F64, SC_REAL_F32 = 0, 1
SC_DONE_CONVERGED, SC_DONE_MAXITER, SC_DONE_BREAKDOWN = 1, 2, 3

_dpp = P(c_void_p)  # array of pointers

# name -> (restype, argtypes)
SIGNATURES = {
    "sc_version": (c_int, []),
    "sc_status_string": (c_char_p, [c_int]),
    "sc_context_create": (c_int, [c_int, P(c_void_p)]),
    "sc_context_destroy": (None, [c_void_p]),
    "sc_context_set_stream": (c_int, [c_void_p, c_void_p]),
    "sc_context_use_own_stream": (c_int, [c_void_p]),
    "sc_context_stream": (c_void_p, [c_void_p]),
    "sc_context_synchronize": (c_int, [c_void_p]),
    "sc_context_last_error": (c_char_p, [c_void_p]),
    "sc_pcg_default_options": (None, [P(sc_pcg_options)]),
    "sc_pcg_create": (c_int, [c_void_p, c_int, c_int, c_int, P(sc_pcg_options), P(c_void_p)]),
    "sc_pcg_destroy": (None, [c_void_p]),
    "sc_pcg_set_options": (c_int, [c_void_p, P(sc_pcg_options)]),
    "sc_pcg_solve_host": (c_int, [c_void_p, c_void_p, _dpp, c_void_p, c_void_p, c_void_p, P(sc_pcg_stats)]),
    "sc_pcg_solve_device": (c_int, [c_void_p, c_void_p, _dpp, c_void_p, c_void_p, c_void_p, P(sc_pcg_stats)]),
    "sc_pcg_upload": (c_int, [c_void_p, c_void_p, _dpp, c_void_p, c_void_p, c_int]),
    "sc_pcg_upload_rhs": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_pcg_solve_resident": (c_int, [c_void_p, P(sc_pcg_stats)]),
    "sc_pcg_download": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_pcg_precond_device": (c_int, [c_void_p, c_void_p, c_void_p]),
    "sc_pcg_apply_device": (c_int, [c_void_p, c_void_p, c_void_p]),
    "sc_pcg_time_kernels": (c_int, [c_void_p, c_int, P(c_double)]),
    "sc_mic_precond_noalloc_device": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, _dpp, c_void_p, c_void_p,
                                              c_void_p, c_double, c_double]),
    "sc_fvm_build_system_device": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_double, c_int,
                                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           _dpp, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "sc_fvm_project_device": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_double, c_int, c_void_p,
                                      c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
}

_lib = None


class CapiError(RuntimeError):
    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} failed with status {status}: {msg}")
        self.status = status


def lib():
    """Load libsimcraft_fluid.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `python -m simcraft_b200.build` "
                          "(the CUDA path has no fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr_array(ptrs):
    return (c_void_p * len(ptrs))(*ptrs)


def check(fn, status, ctx=None):
    if status != SC_OK:
        msg = ""
        if ctx is not None:
            m = lib().sc_context_last_error(ctx)
            msg = m.decode() if m else ""
        if not msg:
            msg = lib().sc_status_string(status).decode()
        raise CapiError(fn, status, msg)
    return status
