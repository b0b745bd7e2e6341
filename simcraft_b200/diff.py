"""Differentiable FLIP/PIC substeps: torch bindings of the adjoint kernels.

  DiffFlip(resolution, h, dt, steps, ...)   forward / backward through the C-ABI
  FlipLoss.apply(param, sim)                 torch.autograd.Function over a
                                             (3, nx, ny, nz) velocity parameter
  faces_from_cells / cells_from_faces        the parameter <-> MAC-face map

The model is the simulator's substep with a fixed dt (see
include/simcraft_fluid_capi.h, "Differentiable FLIP/PIC substeps"): particles
start at fixed positions with velocities sampled from the parameter field and
the loss compares the particle density after the last substep with a target.
The gradient is computed by hand-written adjoint kernels (no autograd tape of
torch operations), with states checkpointed every `checkpoint_every` substeps.
"""
import ctypes

import numpy as np
import torch

from . import _capi
from ._capi import check, lib, ptr_array
from .solver import _ptr, default_context

TAPE = {"none": _capi.SC_TAPE_NONE, "record": _capi.SC_TAPE_RECORD, "replay": _capi.SC_TAPE_REPLAY}


def face_shapes(nx, ny, nz):
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def faces_from_cells(param):
    """(3, nx, ny, nz) cell-indexed velocity -> three MAC face grids.  Component a
    fills faces 0..n-1 along axis a; the extra face n (a domain wall) is 0."""
    _, nx, ny, nz = param.shape
    out = []
    for a, shp in enumerate(face_shapes(nx, ny, nz)):
        f = torch.zeros(shp, dtype=torch.float64, device=param.device)
        idx = [slice(None)] * 3
        idx[a] = slice(0, (nx, ny, nz)[a])
        f[tuple(idx)] = param[a].to(torch.float64)
        out.append(f.contiguous())
    return out


def cells_from_faces(faces, dtype):
    """Adjoint of faces_from_cells (drops the extra face)."""
    nx, ny, nz = faces[0].shape[0] - 1, faces[0].shape[1], faces[0].shape[2]
    comps = []
    for a, f in enumerate(faces):
        idx = [slice(None)] * 3
        idx[a] = slice(0, (nx, ny, nz)[a])
        comps.append(f[tuple(idx)])
    return torch.stack(comps).to(dtype)


def default_config(resolution, h, dt, steps, **kw):
    nx, ny, nz = resolution
    c = _capi.sc_diff_config()
    lib().sc_diff_default_config(nx, ny, nz, float(h), float(dt), int(steps), ctypes.byref(c))
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


class DiffFlip:
    """Forward and adjoint of `steps` FLIP/PIC substeps on the GPU."""

    def __init__(self, resolution, h, dt, steps, context=None, precision="f64", advection="flip", **opts):
        self.ctx = context or default_context()
        self.dims = tuple(int(r) for r in resolution)
        self.cfg = default_config(self.dims, h, dt, steps,
                                  precision=_capi.SC_REAL_F32 if precision == "f32" else _capi.SC_REAL_F64,
                                  advection=_capi.SC_ADVECT_PIC if advection == "pic" else _capi.SC_ADVECT_FLIP,
                                  **opts)
        hnd = ctypes.c_void_p()
        check("sc_diff_create", lib().sc_diff_create(self.ctx.handle, ctypes.byref(self.cfg), ctypes.byref(hnd)),
              self.ctx.handle)
        self.handle = hnd
        self.n = 0

    def __del__(self):
        if getattr(self, "handle", None) and _capi._lib is not None:
            _capi._lib.sc_diff_destroy(self.handle)
            self.handle = None

    def set_particles(self, pos):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        check("sc_diff_set_particles", lib().sc_diff_set_particles(self.handle, len(pos), _ptr(pos), 0),
              self.ctx.handle)
        self.n = len(pos)

    def set_target(self, rho):
        rho = np.ascontiguousarray(rho, np.float64)
        assert rho.shape == self.dims
        check("sc_diff_set_target", lib().sc_diff_set_target(self.handle, _ptr(rho), 0), self.ctx.handle)

    def forward(self, faces, tape="none"):
        """Loss for the parameter given as three CUDA float64 face grids.  Runs on
        the context's own stream (the solver captures CUDA graphs there) after
        torch's pending work; returns when the loss is on the host."""
        loss = ctypes.c_double()
        torch.cuda.current_stream(faces[0].device).synchronize()
        rc = lib().sc_diff_forward(self.handle, ptr_array([_ptr(f) for f in faces]), TAPE[tape],
                                   ctypes.byref(loss))
        check("sc_diff_forward", rc, self.ctx.handle)
        return loss.value

    def backward(self):
        """dL/d(face grids) of the last forward (synchronous)."""
        grads = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in face_shapes(*self.dims)]
        torch.cuda.current_stream(grads[0].device).synchronize()
        rc = lib().sc_diff_backward(self.handle, ptr_array([_ptr(g) for g in grads]))
        check("sc_diff_backward", rc, self.ctx.handle)
        return grads

    def density(self):
        rho = np.zeros(self.dims)
        check("sc_diff_get_density", lib().sc_diff_get_density(self.handle, _ptr(rho), 0), self.ctx.handle)
        return rho

    def particles(self):
        pos, vel = np.zeros((self.n, 3)), np.zeros((self.n, 3))
        check("sc_diff_get_particles", lib().sc_diff_get_particles(self.handle, _ptr(pos), _ptr(vel), 0),
              self.ctx.handle)
        return pos, vel

    def last_pcg_iterations(self):
        return lib().sc_diff_last_pcg_iterations(self.handle)

    def pressure(self):
        """Pressure of the last substep of the last forward (reference layout)."""
        p = np.zeros(self.dims)
        check("sc_diff_get_pressure", lib().sc_diff_get_pressure(self.handle, _ptr(p), 0), self.ctx.handle)
        return p


class FlipLoss(torch.autograd.Function):
    """loss = FlipLoss.apply(param, sim): param is a (3, nx, ny, nz) CUDA tensor;
    the backward runs the adjoint kernels of `sim` (a DiffFlip)."""

    @staticmethod
    def forward(ctx, param, sim):
        faces = faces_from_cells(param.detach())
        loss = sim.forward(faces)
        ctx.sim = sim
        ctx.dtype = param.dtype
        return torch.tensor(loss, dtype=torch.float64, device=param.device)

    @staticmethod
    def backward(ctx, gout):
        grads = ctx.sim.backward()
        g = cells_from_faces(grads, ctx.dtype)
        return g * gout.to(ctx.dtype), None


def control_scene(n=64, seed_particles=5, seed_param=6, seed_target=7, ppc=8, param_std=0.1):
    """The differentiable control problem: fluid in the lower quarter (y < 0.25)
    of an n^3 box, `ppc` jittered particles per cell; parameter (3, n, n, n)
    float32 ~ N(0, param_std); target density = ppc on the cells inside a union
    of seeded spheres.  Returns (pos, param (numpy float32), target, h)."""
    from . import scenes

    pos, _, h = scenes.dam_break(n, frac_x=1.0, frac_y=0.25, frac_z=1.0, ppc=ppc, seed=seed_particles)
    param = np.random.default_rng(seed_param).normal(0.0, param_std, (3, n, n, n)).astype(np.float32)
    rng = np.random.default_rng(seed_target)
    centres = rng.uniform(0.2, 0.8, (4, 3))
    centres[:, 1] = rng.uniform(0.1, 0.3, 4)
    radii = rng.uniform(0.08, 0.15, 4)
    sdf = scenes.sphere_union_sdf(n, centres, radii)
    target = np.where(sdf <= 0.0, float(ppc), 0.0)
    return pos, param, target, h


__all__ = ["DiffFlip", "FlipLoss", "faces_from_cells", "cells_from_faces", "default_config", "control_scene"]
