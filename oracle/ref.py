"""ctypes bindings for oracle/_ref/libsimcraft_ref.so: the reference's OWN
FluidSim CPU code (FluidSim/src/cpu/*.cc), compiled by `make -C oracle ref`
from the reference tree together with the stand-in headers in oracle/refshim.

TEST INFRASTRUCTURE ONLY: the tests use it to pin the oracle restatement
(fluid_oracle.cc) against the reference itself.  The library is built where the
reference tree is present; it travels with the repository as a built file, so
the GPU tests can load it where the tree is absent.  `available()` says whether
it can be used here.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_ref", "libsimcraft_ref.so")
# the timing build: the same sources with oneTBB's loops on OpenMP threads
_LIB_PAR = os.path.join(_HERE, "_ref", "libsimcraft_ref_par.so")
_SRC = ("ref_capi.cc", "refshim/prelude.h", "refshim/glm/glm.hpp", "refshim/tbb/tbb.h",
        "refshim/spdlog/spdlog.h", "refshim/Core/transfer-stencil.h")
_libs = {}

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_ip = ctypes.POINTER(ctypes.c_int)
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double
_vp = ctypes.c_void_p


def reference_tree():
    """The reference source tree the library is built from (REF in oracle/Makefile)."""
    return os.environ.get("SIMCRAFT_REFERENCE", "/root/reference")


def build(force=False):
    """Build the library when the reference tree is present and the library is
    missing or older than its wrapper sources.  Returns the path or None."""
    newest = max(os.path.getmtime(os.path.join(_HERE, f)) for f in _SRC)
    stale = any(not os.path.exists(p) or os.path.getmtime(p) < newest for p in (_LIB, _LIB_PAR))
    if (force or stale) and os.path.isdir(os.path.join(reference_tree(), "FluidSim")):
        subprocess.check_call(["make", "-s", "-C", _HERE, "ref", "REF=" + reference_tree()])
    return _LIB if os.path.exists(_LIB) else None


def available():
    try:
        return build() is not None
    except (OSError, subprocess.CalledProcessError):
        return False


def lib(parallel=False):
    """The parity build (serial), or with parallel=True the timing build."""
    if parallel not in _libs:
        path = _LIB_PAR if parallel else _LIB
        if build() is None or not os.path.exists(path):
            raise RuntimeError(path + " is not built and the reference tree is absent")
        L = ctypes.CDLL(path)
        sig = {
            "ref_apply_matrix": (None, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp]),
            "ref_mic_precond": (None, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp, _dbl, _dbl,
                                       _dp, _dp]),
            "ref_cg_solve": (_dbl, [_int, _int, _int, _dp, ctypes.POINTER(_dp), _dp, _u8p, _dp, _dbl, _int,
                                    ctypes.POINTER(_int), _dp]),
            "ref_set_threads": (None, [_int]),
            "ref_dot": (_dbl, [_int, _int, _int, _dp, _dp, _u8p]),
            "ref_saxpy": (None, [_int, _int, _int, _dp, _dp, _dbl, _u8p]),
            "ref_scale_and_add": (None, [_int, _int, _int, _dp, _dp, _dbl, _u8p]),
            "ref_linf": (_dbl, [_int, _int, _int, _dp, _u8p]),
            "ref_fraction_inside": (_dbl, [_dbl] * 4),
            "ref_build_system": (None, [_int, _int, _int, _dbl, _dbl, _dp, _dp, _dp, _dp, _dp, _dp,
                                        ctypes.POINTER(_dp), _dp, _u8p, _dp, _dp, _dp]),
            "ref_project": (None, [_int, _int, _int, _dbl, _dbl, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "ref_sample_velocity": (None, [_i64, _dp, _int, _int, _int, _dbl, _dp, _dp, _dp, _dp]),
            "ref_p2g": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl] + [_dp] * 6 + [_u8p] * 3 + [_dp] * 3),
            "ref_g2p": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl] + [_dp] * 6 + [_dbl]),
            "ref_advect": (None, [_i64, _dp, _dp, _int, _int, _int, _dbl, _dp, _dp, _dp, _dp, _dbl]),
            "ref_sdf_eval": (_dbl, [_dp, _int, _int, _int, _dbl, _dp]),
            "ref_sdf_grad": (None, [_dp, _int, _int, _int, _dbl, _dp, _dp]),
            "ref_reconstruct": (None, [_i64, _dp, _int, _int, _int, _dbl, _dbl, _dp, _u8p]),
            "ref_manifold_to_sdf": (None, [_int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dp, _i64, _ip, _i64, _int,
                                           _dp, _ip, _ip]),
            "ref_rebuild_surface": (_i64, [_int, _int, _int, _dbl, _dp, _dp, _dp,
                                           ctypes.POINTER(ctypes.c_uint32), _i64, _i64, ctypes.POINTER(_i64)]),
            "ref_sim_create": (_vp, [_int, _int, _int, _dbl, _int, _dbl, _dbl, _int, _i64]),
            "ref_sim_destroy": (None, [_vp]),
            "ref_sim_set_particles": (None, [_vp, _dp, _dp]),
            "ref_sim_set_collider": (None, [_vp, _dp]),
            "ref_sim_substep": (None, [_vp, _dbl]),
            "ref_sim_step": (_int, [_vp, _dbl]),
            "ref_sim_cfl": (_dbl, [_vp]),
            "ref_sim_get_particles": (None, [_vp, _dp, _dp]),
            "ref_sim_get_pressure": (None, [_vp, _dp]),
            "ref_sim_get_faces": (None, [_vp, _dp, _dp, _dp]),
            "ref_sim_get_fluid_sdf": (None, [_vp, _dp]),
            "ref_sim_get_system": (None, [_vp, _dp, ctypes.POINTER(_dp), _dp, _u8p]),
            "ref_sim_reconstruct": (None, [_vp]),
            "ref_sim_smooth_fluid_surface": (None, [_vp, _int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _libs[parallel] = L
    return _libs[parallel]


def _p(a):
    if a is None:
        return None
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_u8p)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_ip)
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def _ptr_array(arrs):
    return (_dp * len(arrs))(*[_p(np.ascontiguousarray(a, np.float64)) for a in arrs])


def face_shapes(nx, ny, nz):
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def apply_matrix(adiag, an, x, active):
    b = np.zeros_like(adiag)
    an = [np.ascontiguousarray(a) for a in an]
    lib().ref_apply_matrix(*adiag.shape, _p(adiag), _ptr_array(an), _p(x), _p(active), _p(b))
    return b


def mic_precond(adiag, an, r, active, tau=0.97, sigma=0.25, return_scratch=False):
    z = np.zeros_like(adiag)
    E = np.zeros_like(adiag)
    q = np.zeros_like(adiag)
    an = [np.ascontiguousarray(a) for a in an]
    lib().ref_mic_precond(*adiag.shape, _p(adiag), _ptr_array(an), _p(np.ascontiguousarray(r)), _p(active),
                          _p(z), tau, sigma, _p(E), _p(q))
    return (z, E, q) if return_scratch else z


def cg_solve(adiag, an, rhs, active, tol=1e-6, max_iter=300, parallel=False, threads=None, stats=None):
    """CgSolver3D::solve: the reference's stopping test (absolute L-inf < tol,
    at most max_iter - 1 iterations).  Returns (pressure, residual); `stats`
    (a dict) receives the reference's iteration count and the solve's wall ms.
    parallel=True runs the timing build on `threads` OpenMP threads."""
    pg = np.zeros_like(adiag)
    an = [np.ascontiguousarray(a) for a in an]
    L = lib(parallel)
    if parallel:
        L.ref_set_threads(int(threads or os.cpu_count() or 1))
    it, ms = _int(0), _dbl(0.0)
    res = L.ref_cg_solve(*adiag.shape, _p(adiag), _ptr_array(an), _p(rhs), _p(active), _p(pg), tol, max_iter,
                         ctypes.byref(it), ctypes.byref(ms))
    if stats is not None:
        stats["iterations"] = it.value
        stats["ms"] = ms.value
    return pg, res


def dot(a, b, active):
    return lib().ref_dot(*a.shape, _p(a), _p(b), _p(active))


def saxpy(a, b, x, active):
    lib().ref_saxpy(*a.shape, _p(a), _p(b), x, _p(active))


def scale_and_add(c, a, x, active):
    lib().ref_scale_and_add(*c.shape, _p(c), _p(a), x, _p(active))


def linf(a, active):
    return lib().ref_linf(*a.shape, _p(a), _p(active))


def fraction_inside(a, b, c, d):
    return lib().ref_fraction_inside(a, b, c, d)


def build_system(dims, h, dt, u, v, w, fluid_sdf, collider=None):
    nx, ny, nz = dims
    su, sv, sw = face_shapes(nx, ny, nz)
    adiag = np.zeros(dims)
    an = [np.zeros(dims) for _ in range(6)]
    rhs = np.zeros(dims)
    active = np.zeros(dims, np.uint8)
    uwt, vwt, wwt = np.zeros(su), np.zeros(sv), np.zeros(sw)
    c = None if collider is None else np.ascontiguousarray(collider, np.float64)
    lib().ref_build_system(nx, ny, nz, h, dt, _p(u), _p(v), _p(w), _p(fluid_sdf), _p(c), _p(adiag),
                           (_dp * 6)(*[_p(a) for a in an]), _p(rhs), _p(active), _p(uwt), _p(vwt), _p(wwt))
    return dict(adiag=adiag, an=an, rhs=rhs, active=active, uwt=uwt, vwt=vwt, wwt=wwt)


def project(dims, h, dt, u, v, w, pg, fluid_sdf, uwt, vwt, wwt):
    u, v, w = (np.array(a, np.float64, copy=True) for a in (u, v, w))
    lib().ref_project(*dims, h, dt, _p(u), _p(v), _p(w), _p(pg), _p(fluid_sdf), _p(uwt), _p(vwt), _p(wwt))
    return u, v, w


def sample_velocity(pts, dims, h, u, v, w):
    pts = np.ascontiguousarray(pts, np.float64)
    out = np.zeros_like(pts)
    lib().ref_sample_velocity(len(pts), _p(pts), *dims, h, _p(u), _p(v), _p(w), _p(out))
    return out


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
    lib().ref_p2g(len(pos), _p(pos), _p(vel), nx, ny, nz, h,
                  *[_p(out[k]) for k in ("u", "v", "w", "uw", "vw", "ww", "uvalid", "vvalid", "wvalid")],
                  *[_p(out.get(k)) for k in ("ulast", "vlast", "wlast")])
    return out


def g2p(pos, vel, dims, h, u, v, w, ulast=None, vlast=None, wlast=None, alpha=0.97):
    """FLIP when alpha >= 0 (with the *last grids); PIC when alpha < 0.  Returns new vel."""
    pos = np.ascontiguousarray(pos, np.float64)
    out = np.array(vel, np.float64, copy=True)
    lib().ref_g2p(len(pos), _p(pos), _p(out), *dims, h, _p(u), _p(v), _p(w), _p(ulast), _p(vlast), _p(wlast),
                  alpha)
    return out


def advect(pos, vel, dims, h, u, v, w, collider, dt):
    p = np.array(pos, np.float64, copy=True)
    vv = np.array(vel, np.float64, copy=True)
    c = None if collider is None else np.ascontiguousarray(collider, np.float64)
    lib().ref_advect(len(p), _p(p), _p(vv), *dims, h, _p(u), _p(v), _p(w), _p(c), dt)
    return p, vv


def sdf_eval(sdf, h, p):
    return lib().ref_sdf_eval(_p(sdf), *sdf.shape, h, _p(np.asarray(p, np.float64)))


def sdf_grad(sdf, h, p):
    g = np.zeros(3)
    lib().ref_sdf_grad(_p(sdf), *sdf.shape, h, _p(np.asarray(p, np.float64)), _p(g))
    return g


def reconstruct(pos, dims, h, radius):
    pos = np.ascontiguousarray(pos, np.float64)
    sdf = np.zeros(dims)
    valid = np.zeros(dims, np.uint8)
    lib().ref_reconstruct(len(pos), _p(pos), *dims, h, radius, _p(sdf), _p(valid))
    return sdf, valid


def manifold_to_sdf(vertices, triangles, dims, h, origin=(0.0, 0.0, 0.0), exact_band=3):
    v = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
    sdf = np.zeros(dims)
    closest = np.zeros(dims, np.int32)
    icnt = np.zeros(dims, np.int32)
    lib().ref_manifold_to_sdf(*dims, float(h), *map(float, origin), _p(v), len(v), _p(t), len(t), int(exact_band),
                              _p(sdf), _p(closest), _p(icnt))
    return sdf, closest, icnt


def rebuild_surface(sdf, h):
    sdf = np.ascontiguousarray(sdf, np.float64)
    ni = _i64(0)
    nv = lib().ref_rebuild_surface(*sdf.shape, h, _p(sdf), None, None, None, 0, 0, ctypes.byref(ni))
    V, N, I = np.zeros((nv, 3)), np.zeros((nv, 3)), np.zeros(ni.value, np.uint32)
    lib().ref_rebuild_surface(*sdf.shape, h, _p(sdf), _p(V), _p(N), I.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                              nv, ni.value, ctypes.byref(ni))
    return V, N, I


class Sim:
    """fluid::cpu::FluidSimulator itself (FluidSim/src/cpu/fluid-simulator.cc),
    set up as the reference's app does: FLIP (or PIC), FVM projection, CG with
    MIC(0), naive reconstruction, the empty-mesh collider (1e9)."""

    def __init__(self, dims, h, n, flip=True, flip_alpha=0.97, pcg_tol=1e-6, pcg_max_iter=300):
        self.dims = tuple(dims)
        self.n = int(n)
        self._h = lib().ref_sim_create(*self.dims, h, int(bool(flip)), flip_alpha, pcg_tol, pcg_max_iter, self.n)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_sim_destroy(self._h)
            self._h = None

    def set_particles(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float64)
        assert len(pos) == self.n
        vel = np.zeros_like(pos) if vel is None else np.ascontiguousarray(vel, np.float64)
        lib().ref_sim_set_particles(self._h, _p(pos), _p(vel))

    def set_collider(self, sdf):
        lib().ref_sim_set_collider(self._h, _p(np.ascontiguousarray(sdf, np.float64)))

    def substep(self, dt):
        lib().ref_sim_substep(self._h, dt)

    def step(self, frame_dt):
        return lib().ref_sim_step(self._h, frame_dt)

    def cfl(self):
        return lib().ref_sim_cfl(self._h)

    def particles(self):
        pos, vel = np.zeros((self.n, 3)), np.zeros((self.n, 3))
        lib().ref_sim_get_particles(self._h, _p(pos), _p(vel))
        return pos, vel

    def pressure(self):
        p = np.zeros(self.dims)
        lib().ref_sim_get_pressure(self._h, _p(p))
        return p

    def faces(self):
        su, sv, sw = face_shapes(*self.dims)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        lib().ref_sim_get_faces(self._h, _p(u), _p(v), _p(w))
        return u, v, w

    def fluid_sdf(self):
        s = np.zeros(self.dims)
        lib().ref_sim_get_fluid_sdf(self._h, _p(s))
        return s

    def system(self):
        adiag, rhs = np.zeros(self.dims), np.zeros(self.dims)
        an = [np.zeros(self.dims) for _ in range(6)]
        act = np.zeros(self.dims, np.uint8)
        lib().ref_sim_get_system(self._h, _p(adiag), (_dp * 6)(*[_p(a) for a in an]), _p(rhs), _p(act))
        return adiag, an, rhs, act

    def reconstruct(self):
        lib().ref_sim_reconstruct(self._h)

    def smooth_fluid_surface(self, iters):
        lib().ref_sim_smooth_fluid_surface(self._h, int(iters))
