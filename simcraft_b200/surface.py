"""Surface export on the GPU: rebuildSurface (FluidSim/src/cpu/rebuild-surface.cc:686-741),
the marching-cubes mesh of a cell-centred SDF, and exportObj
(Core/src/obj-io.cc:66-91), the file it is written to.

  rebuild_surface(sdf, spacing, origin=(0, 0, 0), context=None)
      -> (vertices [V,3] float64, normals [V,3] float64, indices [I])

`sdf` is an (nx, ny, nz) array of samples at ((x + 0.5) spacing + origin, ...):
numpy (host path; the mesh comes back as numpy, indices uint32) or a CUDA
float64 tensor (device path; the mesh is CUDA tensors, indices int32 holding
the same numbers, ordered on torch's current stream).  The mesh equals the
reference's bit for bit, vertex numbering and triangle order included; every
three index entries are one triangle.
"""
import ctypes

import numpy as np

from ._capi import check, lib
from .solver import _is_torch, _on_torch_stream, _ptr, default_context


def _three(x, name):
    t = [float(x)] * 3 if np.isscalar(x) else [float(v) for v in x]
    if len(t) != 3:
        raise ValueError(name + " needs one or three numbers")
    return (ctypes.c_double * 3)(*t)


def rebuild_surface(sdf, spacing, origin=(0.0, 0.0, 0.0), context=None):
    """The marching-cubes mesh of `sdf` (see the module docstring)."""
    ctx = context or default_context()
    sp, org = _three(spacing, "spacing"), _three(origin, "origin")
    nv, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    if _is_torch(sdf):
        import torch

        s = sdf.to(torch.float64).contiguous()
        if s.dim() != 3:
            raise ValueError("sdf must be 3-D")
        nx, ny, nz = s.shape
        with _on_torch_stream(ctx, s):
            rc = lib().sc_rebuild_surface_device(ctx.handle, nx, ny, nz, sp, org, _ptr(s), None, None, None, 0, 0,
                                                 ctypes.byref(nv), ctypes.byref(ni))
            check("sc_rebuild_surface_device", rc, ctx.handle)
            V = torch.empty((nv.value, 3), dtype=torch.float64, device=s.device)
            N = torch.empty((nv.value, 3), dtype=torch.float64, device=s.device)
            I = torch.empty((ni.value,), dtype=torch.int32, device=s.device)
            if ni.value:
                rc = lib().sc_rebuild_surface_device(ctx.handle, nx, ny, nz, sp, org, _ptr(s), _ptr(V), _ptr(N),
                                                     _ptr(I), nv.value, ni.value, ctypes.byref(nv), ctypes.byref(ni))
                check("sc_rebuild_surface_device", rc, ctx.handle)
        return V, N, I
    s = np.ascontiguousarray(sdf, np.float64)
    if s.ndim != 3:
        raise ValueError("sdf must be 3-D")
    nx, ny, nz = s.shape
    rc = lib().sc_rebuild_surface_host(ctx.handle, nx, ny, nz, sp, org, _ptr(s), None, None, None, 0, 0,
                                       ctypes.byref(nv), ctypes.byref(ni))
    check("sc_rebuild_surface_host", rc, ctx.handle)
    V = np.empty((nv.value, 3))
    N = np.empty((nv.value, 3))
    I = np.empty(ni.value, np.uint32)
    if ni.value:
        rc = lib().sc_rebuild_surface_host(ctx.handle, nx, ny, nz, sp, org, _ptr(s), _ptr(V), _ptr(N), _ptr(I),
                                           nv.value, ni.value, ctypes.byref(nv), ctypes.byref(ni))
        check("sc_rebuild_surface_host", rc, ctx.handle)
    return V, N, I


def export_obj(path, vertices, normals, indices):
    """Writes the mesh as exportObj does (Core/src/obj-io.cc:66-91): `v` lines,
    `vn` lines, then `f a//a b//b c//c ` per triangle with 1-based numbers.
    Numbers are written in the shortest form that reads back to the same
    double.  Returns False if the file cannot be opened, as the reference."""
    V = np.asarray(vertices.cpu() if _is_torch(vertices) else vertices, np.float64).reshape(-1, 3)
    N = np.asarray(normals.cpu() if _is_torch(normals) else normals, np.float64).reshape(-1, 3)
    I = np.asarray(indices.cpu() if _is_torch(indices) else indices).astype(np.int64).reshape(-1)
    try:
        f = open(path, "w")
    except OSError:
        return False
    with f:
        f.writelines("v %r %r %r\n" % (float(a), float(b), float(c)) for a, b, c in V)
        f.writelines("vn %r %r %r\n" % (float(a), float(b), float(c)) for a, b, c in N)
        t = I[: len(I) - len(I) % 3].reshape(-1, 3) + 1
        f.writelines("f %d//%d %d//%d %d//%d \n" % (a, a, b, b, c, c) for a, b, c in t)
    return True


__all__ = ["rebuild_surface", "export_obj"]
