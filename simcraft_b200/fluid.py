"""Python mirror of the reference's FLIP/PIC simulator and advection seams, backed
by the CUDA library through the C-ABI.

  FluidSimulator(n, size, resolution)         fluid::cpu::FluidSimulator
      (FluidSim/include/FluidSim/cpu/fluid-simulator.h:25-200,
       FluidSim/src/cpu/fluid-simulator.cc)
  p2g / g2p / advect / sample_velocity         HybridAdvectionSolver3D
      (FluidSim/include/FluidSim/cpu/advect-solver.h:16-140,
       FluidSim/src/cpu/advect-solver.cc, FluidSim/src/cpu/util.cc:40-85)
  reconstruct                                   NaiveReconstructor::reconstruct
      (FluidSim/include/FluidSim/cpu/sdf.h:204-229)

Grids use the reference's z-fastest layout; face grids are (nx+1,ny,nz),
(nx,ny+1,nz), (nx,ny,nz+1).  Particles are (n, 3) float64 arrays.  The stage
functions take torch CUDA float64 tensors and run on torch's current stream.
"""
import ctypes

import numpy as np

from . import _capi
from ._capi import check, lib
from .solver import _is_torch, _on_torch_stream, _ptr, default_context, default_options

PIC, FLIP = _capi.SC_ADVECT_PIC, _capi.SC_ADVECT_FLIP
REAL_F64, REAL_F32 = _capi.SC_REAL_F64, _capi.SC_REAL_F32


def face_shapes(nx, ny, nz):
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def default_config(resolution, h, **kw):
    """sc_fluid_config with the reference's constants; keyword overrides may
    name config fields or (prefixed `pcg_`) pressure-solver options."""
    nx, ny, nz = resolution
    c = _capi.sc_fluid_config()
    lib().sc_fluid_default_config(nx, ny, nz, float(h), ctypes.byref(c))
    for k, v in kw.items():
        if k.startswith("pcg_"):
            if not hasattr(c.pcg, k[4:]):
                raise KeyError(k)
            setattr(c.pcg, k[4:], v)
        elif hasattr(c, k) and k != "pcg":
            setattr(c, k, v)
        else:
            raise KeyError(k)
    return c


class FluidSimulator:
    """fluid::cpu::FluidSimulator on the B200.

    `size` and `resolution` follow the reference constructor (domain extent and
    cell counts; cells must be cubic).  Options: precision ("f64"/"f32"),
    advection ("flip"/"pic"), flip_alpha, cfl_factor, gravity, recon_factor,
    sdf_extrap_iters, smooth_iters, vel_extrap_iters, and pressure-solver
    options prefixed with `pcg_` (pcg_tol, pcg_max_iter, pcg_criterion,
    pcg_precision, pcg_mic_tau, pcg_mic_sigma, ...)."""

    def __init__(self, n, size, resolution, context=None, precision="f64", advection="flip", **opts):
        self.ctx = context or default_context()
        nx, ny, nz = (int(r) for r in resolution)
        hs = [float(s) / r for s, r in zip(size, (nx, ny, nz))]
        if max(hs) - min(hs) > 1e-12 * max(hs):
            raise ValueError("cells must be cubic (the reference asserts equal grid spacing)")
        self.dims = (nx, ny, nz)
        self.h = hs[0]
        self.n = int(n)
        self.cfg = default_config(self.dims, self.h,
                                  precision=REAL_F32 if precision == "f32" else REAL_F64,
                                  advection=PIC if advection == "pic" else FLIP, **opts)
        hnd = ctypes.c_void_p()
        check("sc_fluid_create", lib().sc_fluid_create(self.ctx.handle, ctypes.byref(self.cfg), ctypes.byref(hnd)),
              self.ctx.handle)
        self.handle = hnd
        self.last_stats = None

    def __del__(self):
        if getattr(self, "handle", None) and _capi._lib is not None:
            _capi._lib.sc_fluid_destroy(self.handle)
            self.handle = None

    # -- set-up ---------------------------------------------------------------
    def set_initial_fluid(self, positions, velocities=None):
        """The particles (n, 3); velocities default to rest."""
        if _is_torch(positions):
            with _on_torch_stream(self.ctx, positions):
                rc = lib().sc_fluid_set_particles(self.handle, positions.shape[0], _ptr(positions),
                                                  _ptr(velocities) if velocities is not None else None, 1)
        else:
            positions = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
            if velocities is not None:
                velocities = np.ascontiguousarray(velocities, np.float64).reshape(-1, 3)
            rc = lib().sc_fluid_set_particles(self.handle, len(positions), _ptr(positions),
                                              _ptr(velocities) if velocities is not None else None, 0)
        check("sc_fluid_set_particles", rc, self.ctx.handle)
        self.n = int(positions.shape[0])

    def set_collider(self, sdf=None):
        """Collider SDF sampled at the cell centres (None: no collider)."""
        if sdf is None:
            rc = lib().sc_fluid_set_collider(self.handle, None, 0)
        elif _is_torch(sdf):
            with _on_torch_stream(self.ctx, sdf):
                rc = lib().sc_fluid_set_collider(self.handle, _ptr(sdf), 1)
        else:
            sdf = np.ascontiguousarray(sdf, np.float64)
            assert sdf.shape == self.dims
            rc = lib().sc_fluid_set_collider(self.handle, _ptr(sdf), 0)
        check("sc_fluid_set_collider", rc, self.ctx.handle)

    def set_collider_mesh(self, vertices, triangles, exact_distance=False):
        """setCollider(const Mesh&) (fluid-simulator.h:62-71): the collider SDF
        built on the GPU from a closed triangle mesh (vertices [V,3], triangles
        [T,3] vertex indices), numpy or CUDA tensors, with manifold2SDF's exact
        band of 3 cells; exact_distance as in simcraft_b200.mesh.manifold_to_sdf."""
        flags = int(bool(exact_distance))
        if _is_torch(vertices):
            import torch

            v = vertices.to(torch.float64).contiguous()
            t = triangles.to(torch.int32).contiguous()
            with _on_torch_stream(self.ctx, v):
                rc = lib().sc_fluid_set_collider_mesh(self.handle, _ptr(v), v.shape[0], _ptr(t), t.shape[0], flags, 1)
        else:
            v = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
            t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
            rc = lib().sc_fluid_set_collider_mesh(self.handle, _ptr(v), len(v), _ptr(t), len(t), flags, 0)
        check("sc_fluid_set_collider_mesh", rc, self.ctx.handle)

    # -- time stepping ----------------------------------------------------------
    def cfl(self):
        dt = ctypes.c_double()
        check("sc_fluid_cfl", lib().sc_fluid_cfl(self.handle, ctypes.byref(dt)), self.ctx.handle)
        return dt.value

    def substep(self, dt):
        st = _capi.sc_fluid_stats()
        rc = lib().sc_fluid_substep(self.handle, float(dt), ctypes.byref(st))
        self.last_stats = st.as_dict()
        check("sc_fluid_substep", rc, self.ctx.handle)
        return self.last_stats

    def step(self, frame_dt):
        """One frame: CFL-limited substeps until frame_dt is covered."""
        st = _capi.sc_fluid_stats()
        rc = lib().sc_fluid_step(self.handle, float(frame_dt), ctypes.byref(st))
        self.last_stats = st.as_dict()
        check("sc_fluid_step", rc, self.ctx.handle)
        return self.last_stats

    # -- read-back ----------------------------------------------------------------
    def particles(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        check("sc_fluid_get_particles", lib().sc_fluid_get_particles(self.handle, _ptr(pos), _ptr(vel), 0),
              self.ctx.handle)
        return pos, vel

    def positions(self):
        return self.particles()[0]

    def pressure(self):
        p = np.zeros(self.dims)
        check("sc_fluid_get_pressure", lib().sc_fluid_get_pressure(self.handle, _ptr(p), 0), self.ctx.handle)
        return p

    def faces(self):
        su, sv, sw = face_shapes(*self.dims)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        check("sc_fluid_get_faces", lib().sc_fluid_get_faces(self.handle, _ptr(u), _ptr(v), _ptr(w), 0),
              self.ctx.handle)
        return u, v, w

    def export_fluid_surface(self):
        s = np.zeros(self.dims)
        check("sc_fluid_get_fluid_sdf", lib().sc_fluid_get_fluid_sdf(self.handle, _ptr(s), 0), self.ctx.handle)
        return s

    def export_collider_surface(self):
        """exportColliderSurface() (cpu/fluid-simulator.h:191-193): the collider
        SDF, 1e9 everywhere when there is none."""
        s = np.zeros(self.dims)
        check("sc_fluid_get_collider_sdf", lib().sc_fluid_get_collider_sdf(self.handle, _ptr(s), 0), self.ctx.handle)
        return s

    def reconstruct(self, radius=None):
        """FluidSimulator::reconstruct() (cpu/fluid-simulator.h:115-119): the
        particles' surface into the fluid SDF, radius 1.2 h / sqrt(2) unless
        given."""
        check("sc_fluid_reconstruct", lib().sc_fluid_reconstruct(self.handle, float(radius or 0.0)),
              self.ctx.handle)

    def smooth_fluid_surface(self, iters):
        """smoothFluidSurface(iters) (fluid-simulator.cc:39-74) on the fluid SDF."""
        check("sc_fluid_smooth_fluid_surface", lib().sc_fluid_smooth_fluid_surface(self.handle, int(iters)),
              self.ctx.handle)

    def rebuild_surface(self):
        """rebuildSurface(mesh, exportFluidSurface()) (rebuild-surface.cc:732-741,
        as FluidSim/disabled/fluid-sim.cc:230-238 exports the fluid): the
        marching-cubes mesh of the fluid SDF, (vertices, normals, indices)."""
        from .surface import rebuild_surface

        return rebuild_surface(self.export_fluid_surface(), self.h, context=self.ctx)


# ---------------------------------------------------------------------------
# Stage functions on torch CUDA float64 tensors.

def _ctx(context):
    return context or default_context()


def p2g(pos, vel, dims, h, flip=True, context=None):
    """FlipAdvectionSolver3D::solveP2G; returns a dict of u, v, w, uw, vw, ww,
    uvalid, vvalid, wvalid (and ulast, vlast, wlast when flip)."""
    import torch

    ctx = _ctx(context)
    su, sv, sw = face_shapes(*dims)
    dev = pos.device
    out = {}
    for k, s in (("u", su), ("v", sv), ("w", sw), ("uw", su), ("vw", sv), ("ww", sw)):
        out[k] = torch.zeros(s, dtype=torch.float64, device=dev)
    for k, s in (("uvalid", su), ("vvalid", sv), ("wvalid", sw)):
        out[k] = torch.zeros(s, dtype=torch.uint8, device=dev)
    if flip:
        for k, s in (("ulast", su), ("vlast", sv), ("wlast", sw)):
            out[k] = torch.zeros(s, dtype=torch.float64, device=dev)
    last = [_ptr(out[k]) if flip else None for k in ("ulast", "vlast", "wlast")]
    with _on_torch_stream(ctx, pos):
        rc = lib().sc_flip_p2g_device(ctx.handle, pos.shape[0], _ptr(pos), _ptr(vel), *dims, float(h),
                                      *[_ptr(out[k]) for k in ("u", "v", "w", "uw", "vw", "ww",
                                                               "uvalid", "vvalid", "wvalid")], *last)
    check("sc_flip_p2g_device", rc, ctx.handle)
    return out


def sample_velocity(pts, dims, h, u, v, w, context=None):
    import torch

    ctx = _ctx(context)
    out = torch.empty_like(pts)
    with _on_torch_stream(ctx, pts):
        rc = lib().sc_sample_velocity_device(ctx.handle, pts.shape[0], _ptr(pts), *dims, float(h), _ptr(u),
                                             _ptr(v), _ptr(w), _ptr(out))
    check("sc_sample_velocity_device", rc, ctx.handle)
    return out


def g2p(pos, vel, dims, h, u, v, w, ulast=None, vlast=None, wlast=None, alpha=0.97, context=None):
    """FLIP blend when alpha >= 0 (needs the *last grids), PIC when alpha < 0.
    Returns the new velocities (vel is not modified)."""
    ctx = _ctx(context)
    out = vel.clone()
    lp = [_ptr(a) if a is not None else None for a in (ulast, vlast, wlast)]
    with _on_torch_stream(ctx, pos):
        rc = lib().sc_flip_g2p_device(ctx.handle, pos.shape[0], _ptr(pos), _ptr(out), *dims, float(h), _ptr(u),
                                      _ptr(v), _ptr(w), *lp, float(alpha))
    check("sc_flip_g2p_device", rc, ctx.handle)
    return out


def advect(pos, vel, dims, h, u, v, w, collider, dt, context=None):
    """FlipAdvectionSolver3D::advect; returns new (pos, vel)."""
    ctx = _ctx(context)
    p, vv = pos.clone(), vel.clone()
    with _on_torch_stream(ctx, pos):
        rc = lib().sc_flip_advect_device(ctx.handle, p.shape[0], _ptr(p), _ptr(vv), *dims, float(h), _ptr(u),
                                         _ptr(v), _ptr(w), _ptr(collider) if collider is not None else None,
                                         float(dt))
    check("sc_flip_advect_device", rc, ctx.handle)
    return p, vv


def reconstruct(pos, dims, h, radius, context=None):
    """NaiveReconstructor::reconstruct; returns (sdf, valid)."""
    import torch

    ctx = _ctx(context)
    sdf = torch.empty(dims, dtype=torch.float64, device=pos.device)
    valid = torch.empty(dims, dtype=torch.uint8, device=pos.device)
    with _on_torch_stream(ctx, pos):
        rc = lib().sc_reconstruct_device(ctx.handle, pos.shape[0], _ptr(pos), *dims, float(h), float(radius),
                                         _ptr(sdf), _ptr(valid))
    check("sc_reconstruct_device", rc, ctx.handle)
    return sdf, valid


__all__ = ["FluidSimulator", "default_config", "face_shapes", "p2g", "sample_velocity", "g2p", "advect",
           "reconstruct", "default_options", "PIC", "FLIP", "REAL_F64", "REAL_F32"]
