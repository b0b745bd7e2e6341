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
                ("max_outer", c_int), ("check_symmetry", c_int), ("true_residual", c_int),
                ("inner_method", c_int), ("reliable_delta", c_double)]


class sc_pcg_stats(ctypes.Structure):
    _fields_ = [("iterations", c_int), ("outer", c_int), ("status", c_int), ("residual", c_double),
                ("true_rel_l2", c_double), ("true_linf", c_double), ("ms", c_double),
                ("sym_err", c_double), ("device_flags", ctypes.c_uint),
                ("kernel_launches", c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class sc_fluid_config(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("h", c_double), ("precision", c_int),
                ("advection", c_int), ("flip_alpha", c_double), ("cfl_factor", c_double),
                ("gravity", c_double), ("recon_factor", c_double), ("sdf_extrap_iters", c_int),
                ("smooth_iters", c_int), ("vel_extrap_iters", c_int), ("pcg", sc_pcg_options)]


class sc_fluid_stats(ctypes.Structure):
    _fields_ = [("substeps", c_int), ("pcg_iterations", c_int), ("pcg_outer", c_int),
                ("pcg_residual", c_double), ("ms_advect", c_double), ("ms_sort_sdf", c_double),
                ("ms_p2g", c_double), ("ms_build", c_double), ("ms_solve", c_double),
                ("ms_project_g2p", c_double), ("ms_total", c_double), ("kernel_launches", c_int64),
                ("pcg_status", c_int), ("pcg_flags", ctypes.c_uint)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class sc_diff_config(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int), ("h", c_double), ("dt", c_double),
                ("precision", c_int), ("advection", c_int), ("flip_alpha", c_double), ("gravity", c_double),
                ("recon_factor", c_double), ("sdf_extrap_iters", c_int), ("smooth_iters", c_int),
                ("vel_extrap_iters", c_int), ("steps", c_int), ("checkpoint_every", c_int),
                ("pcg", sc_pcg_options)]


SC_OK = 0
SC_CRIT_ABS_LINF, SC_CRIT_REL_L2 = 0, 1
SC_PREC_FP64, SC_PREC_MIXED = 0, 1
SC_INNER_PCG, SC_INNER_EISENSTAT = 0, 1
SC_REAL_F64, SC_REAL_F32 = 0, 1
SC_DONE_CONVERGED, SC_DONE_MAXITER, SC_DONE_BREAKDOWN = 1, 2, 3
SC_ADVECT_PIC, SC_ADVECT_FLIP = 0, 1
SC_TAPE_NONE, SC_TAPE_RECORD, SC_TAPE_REPLAY = 0, 1, 2
SC_MESH_REFERENCE_DISTANCE, SC_MESH_EXACT_DISTANCE = 0, 1

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
    "sc_context_set_wait_limit": (c_int, [c_void_p, c_int]),
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
    "sc_flip_p2g_device": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_int, c_int, c_int, c_double]
                           + [c_void_p] * 12),
    "sc_sample_velocity_device": (c_int, [c_void_p, c_int64, c_void_p, c_int, c_int, c_int, c_double,
                                          c_void_p, c_void_p, c_void_p, c_void_p]),
    "sc_flip_g2p_device": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_int, c_int, c_int, c_double]
                           + [c_void_p] * 6 + [c_double]),
    "sc_flip_advect_device": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_int, c_int, c_int, c_double,
                                      c_void_p, c_void_p, c_void_p, c_void_p, c_double]),
    "sc_reconstruct_device": (c_int, [c_void_p, c_int64, c_void_p, c_int, c_int, c_int, c_double, c_double,
                                      c_void_p, c_void_p]),
    "sc_fluid_default_config": (None, [c_int, c_int, c_int, c_double, P(sc_fluid_config)]),
    "sc_fluid_create": (c_int, [c_void_p, P(sc_fluid_config), P(c_void_p)]),
    "sc_fluid_destroy": (None, [c_void_p]),
    "sc_fluid_set_particles": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_int]),
    "sc_fluid_set_collider": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_fluid_set_collider_mesh": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_int, c_int]),
    "sc_mesh_to_sdf_device": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_void_p, c_void_p, c_int64,
                                      c_void_p, c_int64, c_int, c_int, c_void_p, c_void_p]),
    "sc_mesh_to_sdf_host": (c_int, [c_void_p, c_int, c_int, c_int, c_double, c_void_p, c_void_p, c_int64,
                                    c_void_p, c_int64, c_int, c_int, c_void_p, c_void_p]),
    "sc_rebuild_surface_device": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_int64, c_int64, P(c_int64), P(c_int64)]),
    "sc_rebuild_surface_host": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_int64, c_int64, P(c_int64), P(c_int64)]),
    "sc_fluid_reconstruct": (c_int, [c_void_p, c_double]),
    "sc_fluid_get_collider_sdf": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_fluid_smooth_fluid_surface": (c_int, [c_void_p, c_int]),
    "sc_fluid_cfl": (c_int, [c_void_p, P(c_double)]),
    "sc_fluid_substep": (c_int, [c_void_p, c_double, P(sc_fluid_stats)]),
    "sc_fluid_step": (c_int, [c_void_p, c_double, P(sc_fluid_stats)]),
    "sc_fluid_num_particles": (c_int64, [c_void_p]),
    "sc_fluid_get_particles": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "sc_fluid_get_pressure": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_fluid_get_faces": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "sc_fluid_get_fluid_sdf": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_diff_default_config": (None, [c_int, c_int, c_int, c_double, c_double, c_int, P(sc_diff_config)]),
    "sc_diff_create": (c_int, [c_void_p, P(sc_diff_config), P(c_void_p)]),
    "sc_diff_destroy": (None, [c_void_p]),
    "sc_diff_set_particles": (c_int, [c_void_p, c_int64, c_void_p, c_int]),
    "sc_diff_set_target": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_diff_forward": (c_int, [c_void_p, _dpp, c_int, P(c_double)]),
    "sc_diff_backward": (c_int, [c_void_p, _dpp]),
    "sc_diff_get_density": (c_int, [c_void_p, c_void_p, c_int]),
    "sc_diff_get_particles": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "sc_diff_last_pcg_iterations": (c_int, [c_void_p]),
    "sc_diff_get_pressure": (c_int, [c_void_p, c_void_p, c_int]),
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
