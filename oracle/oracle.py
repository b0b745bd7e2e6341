"""ctypes bindings for the CPU oracle (liboracle_fluid.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py -- as the checker, never as the thing
measured on the GPU path.  Every function wraps the C++ restatement in
fluid_oracle.cc, which cites the SimCraft reference line for line.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_fluid.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double

CRIT_ABS_LINF = 0
CRIT_REL_L2 = 1


def build(force=False):
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < max(
        os.path.getmtime(os.path.join(_HERE, f))
        for f in ("fluid_oracle.cc", "fluid_oracle.h", "../simcraft_b200/csrc/sc_mc_table.h")
    ):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


class ora_sim_config(ctypes.Structure):
    _fields_ = [
        ("nx", _int), ("ny", _int), ("nz", _int), ("h", _dbl),
        ("flip", _int), ("flip_alpha", _dbl),
        ("pcg_tol", _dbl), ("pcg_max_iter", _int), ("pcg_criterion", _int),
        ("mic_tau", _dbl), ("mic_sigma", _dbl),
        ("cfl_factor", _dbl), ("gravity", _dbl), ("recon_factor", _dbl),
        ("sdf_extrap_iters", _int), ("smooth_iters", _int), ("vel_extrap_iters", _int),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        sig = {
            "ora_set_threads": (None, [_int]),
            "ora_set_parity_mode": (None, [_int]),
            "ora_set_bucket_order": (None, [_int]),
            "ora_get_threads": (_int, []),
            "ora_cubic_weight": (_dbl, [_dbl, _dbl, _dbl, _dbl]),
            "ora_rebuild_surface": (_i64, [_int, _int, _int, _dp, _dp, _dp, _dp, _dp,
                                           ctypes.POINTER(ctypes.c_uint32), _i64, _i64,
                                           ctypes.POINTER(ctypes.c_int64)]),
            "ora_sim_reconstruct": (None, [ctypes.c_void_p, _dbl]),
            "ora_sim_smooth_fluid_surface": (None, [ctypes.c_void_p, _int]),
            "ora_manifold_to_sdf": (None, [_int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dp,
                                           ctypes.POINTER(ctypes.c_int), _i64, _int, _int, _dp,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
            "ora_p2g": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl] + [_dp] * 6 + [_u8p] * 3 + [_dp] * 3),
            "ora_sample_velocity": (None, [_i64, _dp, _int, _int, _int, _dbl, _dp, _dp, _dp, _dp]),
            "ora_g2p": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl] + [_dp] * 6 + [_dbl]),
            "ora_advect": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl, _dp, _dp, _dp, _dp, _dbl]),
            "ora_sdf_eval": (_dbl, [_dp, _int, _int, _int, _dbl, _dp]),
            "ora_sdf_grad": (None, [_dp, _int, _int, _int, _dbl, _dp, _dp]),
            "ora_reconstruct": (None, [_i64, _dp, _int, _int, _int, _dbl, _dbl, _dp, _u8p]),
            "ora_fraction_inside": (_dbl, [_dbl] * 4),
            "ora_build_system": (None, [_int, _int, _int, _dbl, _dbl, _dp, _dp, _dp, _dp, _dp, _dp,
                                        ctypes.POINTER(_dp), _dp, _u8p, _dp, _dp, _dp]),
            "ora_apply_matrix": (None, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp]),
            "ora_mic_precond": (None, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp,
                                       _dbl, _dbl, _dp, _dp]),
            "ora_dot": (_dbl, [_i64, _dp, _dp, _u8p]),
            "ora_saxpy": (None, [_i64, _dp, _dp, _dbl, _u8p]),
            "ora_scale_and_add": (None, [_i64, _dp, _dp, _dbl, _u8p]),
            "ora_linf": (_dbl, [_i64, _dp, _u8p]),
            "ora_pcg_solve": (_dbl, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp, _dbl,
                                     _int, _int, _dbl, _dbl, ctypes.POINTER(_int)]),
            "ora_project": (None, [_int, _int, _int, _dbl, _dbl, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "ora_sim_create": (ctypes.c_void_p, [ctypes.POINTER(ora_sim_config)]),
            "ora_sim_destroy": (None, [ctypes.c_void_p]),
            "ora_sim_set_particles": (None, [ctypes.c_void_p, _i64, _dp, _dp]),
            "ora_sim_set_collider": (None, [ctypes.c_void_p, _dp]),
            "ora_sim_step": (_int, [ctypes.c_void_p, _dbl]),
            "ora_sim_substep": (None, [ctypes.c_void_p, _dbl]),
            "ora_sim_cfl": (_dbl, [ctypes.c_void_p]),
            "ora_sim_get_particles": (None, [ctypes.c_void_p, _dp, _dp]),
            "ora_sim_get_pressure": (None, [ctypes.c_void_p, _dp]),
            "ora_sim_get_faces": (None, [ctypes.c_void_p, _dp, _dp, _dp]),
            "ora_sim_get_fluid_sdf": (None, [ctypes.c_void_p, _dp]),
            "ora_sim_get_system": (None, [ctypes.c_void_p, _dp, ctypes.POINTER(_dp), _dp, _u8p]),
            "ora_sim_last_iters": (_int, [ctypes.c_void_p]),
            "ora_sim_last_residual": (_dbl, [ctypes.c_void_p]),
            "ora_sim_sdf_tape": (None, [ctypes.c_void_p, _int]),
            "ora_sim_sdf_tape_get": (_int, [ctypes.c_void_p, _i64, _dp]),
            "ora_sim_sdf_tape_put": (_int, [ctypes.c_void_p, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def _ptr_array(arrs):
    return (_dp * len(arrs))(*[_p(a) for a in arrs])


def set_threads(n):
    lib().ora_set_threads(int(n))


def set_bucket_order(mode):
    """0: (cell, particle id) bucket order (the GPU path's); 1: the reference's
    std::sort by Morton key, as ns-util.h:46-79 runs it."""
    lib().ora_set_bucket_order(int(mode))


def get_threads():
    return lib().ora_get_threads()


def set_parity_mode(on):
    lib().ora_set_parity_mode(1 if on else 0)


def face_shapes(nx, ny, nz):
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def cubic_weight(h, d):
    return lib().ora_cubic_weight(h, d[0], d[1], d[2])


def fraction_inside(a, b, c, d):
    return lib().ora_fraction_inside(a, b, c, d)


def p2g(pos, vel, dims, h, flip=True):
    nx, ny, nz = dims
    su, sv, sw = face_shapes(nx, ny, nz)
    out = {k: np.zeros(s) for k, s in (("u", su), ("v", sv), ("w", sw), ("uw", su), ("vw", sv), ("ww", sw))}
    for k, s in (("uvalid", su), ("vvalid", sv), ("wvalid", sw)):
        out[k] = np.zeros(s, np.uint8)
    if flip:
        for k, s in (("ulast", su), ("vlast", sv), ("wlast", sw)):
            out[k] = np.zeros(s)
    pos = np.ascontiguousarray(pos, np.float64)
    vel = np.ascontiguousarray(vel, np.float64)
    lib().ora_p2g(len(pos), _p(pos), _p(vel), nx, ny, nz, h,
                  *[_p(out[k]) for k in ("u", "v", "w", "uw", "vw", "ww", "uvalid", "vvalid", "wvalid")],
                  *[_p(out.get(k)) for k in ("ulast", "vlast", "wlast")])
    return out


def sample_velocity(pts, dims, h, u, v, w):
    pts = np.ascontiguousarray(pts, np.float64)
    out = np.zeros_like(pts)
    lib().ora_sample_velocity(len(pts), _p(pts), *dims, h, _p(u), _p(v), _p(w), _p(out))
    return out


def g2p(pos, vel, dims, h, u, v, w, ulast=None, vlast=None, wlast=None, alpha=0.97):
    """FLIP when alpha >= 0 (needs *last grids); PIC when alpha < 0.  Returns new vel."""
    pos = np.ascontiguousarray(pos, np.float64)
    out = np.array(vel, np.float64, copy=True)
    if alpha < 0:
        ulast, vlast, wlast = u, v, w
    lib().ora_g2p(len(pos), _p(pos), _p(out), *dims, h, _p(u), _p(v), _p(w), _p(ulast), _p(vlast),
                  _p(wlast), alpha)
    return out


def advect(pos, vel, dims, h, u, v, w, collider, dt):
    p = np.array(pos, np.float64, copy=True)
    vv = np.array(vel, np.float64, copy=True)
    lib().ora_advect(len(p), _p(p), _p(vv), *dims, h, _p(u), _p(v), _p(w),
                     _p(np.ascontiguousarray(collider, np.float64)) if collider is not None else None, dt)
    return p, vv


def sdf_eval(sdf, h, p):
    p = np.asarray(p, np.float64)
    return lib().ora_sdf_eval(_p(sdf), *sdf.shape, h, _p(p))


def sdf_grad(sdf, h, p):
    p = np.asarray(p, np.float64)
    g = np.zeros(3)
    lib().ora_sdf_grad(_p(sdf), *sdf.shape, h, _p(p), _p(g))
    return g


def reconstruct(pos, dims, h, radius):
    pos = np.ascontiguousarray(pos, np.float64)
    sdf = np.zeros(dims)
    valid = np.zeros(dims, np.uint8)
    lib().ora_reconstruct(len(pos), _p(pos), *dims, h, radius, _p(sdf), _p(valid))
    return sdf, valid


def build_system(dims, h, dt, u, v, w, fluid_sdf, collider=None):
    nx, ny, nz = dims
    if collider is None:
        collider = np.full(dims, 1e9)
    su, sv, sw = face_shapes(nx, ny, nz)
    adiag = np.zeros(dims)
    an = [np.zeros(dims) for _ in range(6)]
    rhs = np.zeros(dims)
    active = np.zeros(dims, np.uint8)
    uwt, vwt, wwt = np.zeros(su), np.zeros(sv), np.zeros(sw)
    lib().ora_build_system(nx, ny, nz, h, dt, _p(u), _p(v), _p(w), _p(fluid_sdf), _p(collider),
                           _p(adiag), _ptr_array(an), _p(rhs), _p(active), _p(uwt), _p(vwt), _p(wwt))
    return dict(adiag=adiag, an=an, rhs=rhs, active=active, uwt=uwt, vwt=vwt, wwt=wwt)


def apply_matrix(adiag, an, x, active):
    b = np.zeros_like(adiag)
    lib().ora_apply_matrix(*adiag.shape, _p(adiag), _ptr_array(an), _p(x), _p(active), _p(b))
    return b


def mic_precond(adiag, an, r, active, tau=0.97, sigma=0.25, return_scratch=False):
    z = np.zeros_like(adiag)
    E = np.zeros_like(adiag)
    q = np.zeros_like(adiag)
    lib().ora_mic_precond(*adiag.shape, _p(adiag), _ptr_array(an), _p(r), _p(active), _p(z), tau, sigma,
                          _p(E), _p(q))
    return (z, E, q) if return_scratch else z


def manifold_to_sdf(vertices, triangles, dims, h, origin=(0.0, 0.0, 0.0), exact_band=3, exact_distance=False):
    """manifold2SDF (util.cc:203-310) on the CPU: (sdf, closest triangle, crossing counts).
    exact_distance=False keeps the reference's point-triangle arithmetic."""
    v = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
    sdf = np.zeros(dims)
    closest = np.zeros(dims, np.int32)
    icnt = np.zeros(dims, np.int32)
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    lib().ora_manifold_to_sdf(*dims, float(h), *map(float, origin), _p(v), ip(t), len(t), int(exact_band),
                              int(bool(exact_distance)), _p(sdf), ip(closest), ip(icnt))
    return sdf, closest, icnt


def rebuild_surface(sdf, spacing, origin=(0.0, 0.0, 0.0), counts=None):
    """rebuildSurface (rebuild-surface.cc:686-741) on the CPU: (vertices [V,3],
    normals [V,3], indices [I] uint32) of the marching-cubes mesh of a
    cell-centred SDF.  spacing: a number or three.  counts=(vertices, index
    entries) when known makes it one pass (else a counting pass comes first)."""
    sdf = np.ascontiguousarray(sdf, np.float64)
    nx, ny, nz = sdf.shape
    sp = np.array([spacing] * 3 if np.isscalar(spacing) else spacing, np.float64)
    org = np.array(origin, np.float64)
    ni = ctypes.c_int64(0)
    if counts is None:
        nv = lib().ora_rebuild_surface(nx, ny, nz, _p(sp), _p(org), _p(sdf), None, None, None, 0, 0,
                                       ctypes.byref(ni))
    else:
        nv, ni.value = int(counts[0]), int(counts[1])
    V = np.zeros((nv, 3))
    N = np.zeros((nv, 3))
    I = np.zeros(ni.value, np.uint32)
    lib().ora_rebuild_surface(nx, ny, nz, _p(sp), _p(org), _p(sdf), _p(V), _p(N),
                              I.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), nv, ni.value,
                              ctypes.byref(ni))
    assert ni.value == len(I), "counts do not match the mesh"
    return V, N, I


def dot(a, b, active):
    return lib().ora_dot(a.size, _p(a), _p(b), _p(active))


def saxpy(a, b, x, active):
    lib().ora_saxpy(a.size, _p(a), _p(b), x, _p(active))


def scale_and_add(c, a, x, active):
    lib().ora_scale_and_add(c.size, _p(c), _p(a), x, _p(active))


def linf(a, active):
    return lib().ora_linf(a.size, _p(a), _p(active))


def pcg_solve(adiag, an, rhs, active, tol=1e-6, max_iter=300, criterion=CRIT_ABS_LINF, tau=0.97,
              sigma=0.25):
    pg = np.zeros_like(adiag)
    it = _int(0)
    res = lib().ora_pcg_solve(*adiag.shape, _p(adiag), _ptr_array(an), _p(rhs), _p(active), _p(pg), tol,
                              max_iter, criterion, tau, sigma, ctypes.byref(it))
    return pg, res, it.value


def project(dims, h, dt, u, v, w, pg, fluid_sdf, uwt, vwt, wwt):
    u, v, w = (np.array(a, np.float64, copy=True) for a in (u, v, w))
    lib().ora_project(*dims, h, dt, _p(u), _p(v), _p(w), _p(pg), _p(fluid_sdf), _p(uwt), _p(vwt), _p(wwt))
    return u, v, w


def default_config(nx, ny, nz, h, **kw):
    c = dict(nx=nx, ny=ny, nz=nz, h=h, flip=1, flip_alpha=0.97, pcg_tol=1e-6, pcg_max_iter=300,
             pcg_criterion=CRIT_ABS_LINF, mic_tau=0.97, mic_sigma=0.25, cfl_factor=5.0, gravity=9.8,
             recon_factor=0.8, sdf_extrap_iters=10, smooth_iters=5, vel_extrap_iters=10)
    c.update(kw)
    return c


class Sim:
    """fluid::cpu::FluidSimulator restated (FluidSim/src/cpu/fluid-simulator.cc)."""

    def __init__(self, **cfg):
        c = ora_sim_config(**cfg)
        self.cfg = cfg
        self.dims = (cfg["nx"], cfg["ny"], cfg["nz"])
        self._h = lib().ora_sim_create(ctypes.byref(c))
        self.n = 0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_sim_destroy(self._h)
            self._h = None

    def set_particles(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.zeros_like(pos) if vel is None else np.ascontiguousarray(vel, np.float64)
        self.n = len(pos)
        lib().ora_sim_set_particles(self._h, len(pos), _p(pos), _p(vel))

    def set_collider(self, sdf=None):
        lib().ora_sim_set_collider(self._h, _p(np.ascontiguousarray(sdf, np.float64)) if sdf is not None else None)

    def step(self, frame_dt):
        return lib().ora_sim_step(self._h, frame_dt)

    def substep(self, dt):
        lib().ora_sim_substep(self._h, dt)

    def cfl(self):
        return lib().ora_sim_cfl(self._h)

    def particles(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        lib().ora_sim_get_particles(self._h, _p(pos), _p(vel))
        return pos, vel

    def pressure(self):
        p = np.zeros(self.dims)
        lib().ora_sim_get_pressure(self._h, _p(p))
        return p

    def faces(self):
        su, sv, sw = face_shapes(*self.dims)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        lib().ora_sim_get_faces(self._h, _p(u), _p(v), _p(w))
        return u, v, w

    def reconstruct(self, radius=None):
        """FluidSimulator::reconstruct(): radius 1.2 h / sqrt(2) by default."""
        h = self.cfg["h"]
        lib().ora_sim_reconstruct(self._h, 1.2 * h / np.sqrt(2.0) if radius is None else radius)

    def smooth_fluid_surface(self, iters):
        lib().ora_sim_smooth_fluid_surface(self._h, int(iters))

    def fluid_sdf(self):
        s = np.zeros(self.dims)
        lib().ora_sim_get_fluid_sdf(self._h, _p(s))
        return s

    def system(self):
        adiag = np.zeros(self.dims)
        an = [np.zeros(self.dims) for _ in range(6)]
        rhs = np.zeros(self.dims)
        act = np.zeros(self.dims, np.uint8)
        lib().ora_sim_get_system(self._h, _p(adiag), _ptr_array(an), _p(rhs), _p(act))
        return adiag, an, rhs, act

    def last_iters(self):
        return lib().ora_sim_last_iters(self._h)

    def last_residual(self):
        return lib().ora_sim_last_residual(self._h)

    def sdf_tape(self, mode, sdfs=None):
        """Fluid-SDF tape: 1 records the SDF each later substep uses, 2 replays
        the taped ones (or `sdfs`, a list of arrays, when given) instead of
        reconstructing, 0 turns it off."""
        lib().ora_sim_sdf_tape(self._h, 1 if sdfs is not None else int(mode))
        if sdfs is not None:
            for a in sdfs:
                lib().ora_sim_sdf_tape_put(self._h, _p(np.ascontiguousarray(a, np.float64)))
            lib().ora_sim_sdf_tape(self._h, 2)
            # mode 2 rewinds the tape without clearing it

    def taped_sdfs(self):
        out = []
        k = 0
        while True:
            a = np.zeros(self.dims)
            if lib().ora_sim_sdf_tape_get(self._h, k, _p(a)) != 0:
                return out
            out.append(a)
            k += 1
