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


# Mesh size of the last export per (context, grid): a repeated export (one per
# frame) first tries a single call with that size plus headroom.
_last_counts = {}


def _headroom(nv, ni):
    return nv + nv // 4 + 64, ni + ni // 4 + 192


def rebuild_surface(sdf, spacing, origin=(0.0, 0.0, 0.0), context=None):
    """The marching-cubes mesh of `sdf` (see the module docstring).

    One C-ABI call when the mesh fits the size remembered from the previous
    export of the same grid on this context (plus a quarter); otherwise a
    counting call, or the failed call's counts, then one filling call."""
    ctx = context or default_context()
    sp, org = _three(spacing, "spacing"), _three(origin, "origin")
    nv, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    device = _is_torch(sdf)
    if device:
        import torch

        s = sdf.to(torch.float64).contiguous()
        shape = tuple(s.shape)
        fn_name = "sc_rebuild_surface_device"

        def alloc(cv, ci):
            return (torch.empty((cv, 3), dtype=torch.float64, device=s.device),
                    torch.empty((cv, 3), dtype=torch.float64, device=s.device),
                    torch.empty((ci,), dtype=torch.int32, device=s.device))
    else:
        s = np.ascontiguousarray(sdf, np.float64)
        shape = s.shape
        fn_name = "sc_rebuild_surface_host"

        def alloc(cv, ci):
            return np.empty((cv, 3)), np.empty((cv, 3)), np.empty(ci, np.uint32)
    if len(shape) != 3:
        raise ValueError("sdf must be 3-D")
    nx, ny, nz = shape
    fn = getattr(lib(), fn_name)
    key = (ctx.handle.value if hasattr(ctx.handle, "value") else ctx.handle, device, shape)

    def call(out, cv, ci):
        ptrs = [_ptr(a) for a in out] if out is not None else [None, None, None]
        return fn(ctx.handle, nx, ny, nz, sp, org, _ptr(s), *ptrs, cv, ci, ctypes.byref(nv), ctypes.byref(ni))

    def run():
        out = None
        if key in _last_counts:
            cv, ci = _headroom(*_last_counts[key])
            out = alloc(cv, ci)
            rc = call(out, cv, ci)
            if rc == 0:
                return out, nv.value, ni.value
            if nv.value <= cv and ni.value <= ci:  # not a capacity failure
                check(fn_name, rc, ctx.handle)
        else:
            check(fn_name, call(None, 0, 0), ctx.handle)  # count only
        cv, ci = nv.value, ni.value
        out = alloc(cv, ci)
        if ci:
            check(fn_name, call(out, cv, ci), ctx.handle)
        return out, cv, ci

    if device:
        with _on_torch_stream(ctx, s):
            (V, N, I), cv, ci = run()
    else:
        (V, N, I), cv, ci = run()
    _last_counts[key] = (cv, ci)
    return V[:cv], N[:cv], I[:ci]


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
