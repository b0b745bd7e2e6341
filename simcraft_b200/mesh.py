"""Mesh -> signed distance grid on the GPU: manifold2SDF
(FluidSim/src/cpu/util.cc:203-310), the collider build of
FluidSimulator::setCollider (FluidSim/include/FluidSim/cpu/fluid-simulator.h:62-71).

  manifold_to_sdf(vertices, triangles, resolution, h, origin=(0, 0, 0),
                  exact_band=3, exact_distance=False, context=None, closest=False)

vertices [V,3] and triangles [T,3] (vertex indices) as numpy arrays (host
path, the result comes back as numpy) or CUDA tensors (device path, the result
is a CUDA tensor, ordered on torch's current stream).  Cell (x, y, z) is
sampled at ((x + 0.5) h + origin[0], ...); the SDF is negative inside.

exact_distance=False reproduces the reference bit for bit, including its
point-triangle distance, which overstates the distance to edges AB and AC and
to the face interior (it adds the edge/face offsets instead of subtracting
them); exact_distance=True measures true point-triangle distances.
"""
import ctypes

import numpy as np

from ._capi import check, lib
from .solver import _is_torch, _on_torch_stream, _ptr, default_context


def manifold_to_sdf(vertices, triangles, resolution, h, origin=(0.0, 0.0, 0.0), exact_band=3,
                    exact_distance=False, context=None, closest=False):
    """Signed distance of a closed triangle mesh on the cell centres of a grid;
    with closest=True also the index of the triangle each distance came from
    (-1 where none reached the cell)."""
    ctx = context or default_context()
    nx, ny, nz = (int(r) for r in resolution)
    org = (ctypes.c_double * 3)(*map(float, origin))
    if _is_torch(vertices):
        import torch

        v = vertices.to(torch.float64).reshape(-1, 3).contiguous()
        t = triangles.to(torch.int32).reshape(-1, 3).contiguous()
        sdf = torch.empty((nx, ny, nz), dtype=torch.float64, device=v.device)
        cl = torch.empty((nx, ny, nz), dtype=torch.int32, device=v.device) if closest else None
        with _on_torch_stream(ctx, v):
            rc = lib().sc_mesh_to_sdf_device(ctx.handle, nx, ny, nz, float(h), org, _ptr(v), v.shape[0], _ptr(t),
                                             t.shape[0], int(exact_band), int(bool(exact_distance)), _ptr(sdf),
                                             _ptr(cl) if cl is not None else None)
        check("sc_mesh_to_sdf_device", rc, ctx.handle)
    else:
        v = np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, np.int32).reshape(-1, 3)
        sdf = np.empty((nx, ny, nz))
        cl = np.empty((nx, ny, nz), np.int32) if closest else None
        rc = lib().sc_mesh_to_sdf_host(ctx.handle, nx, ny, nz, float(h), org, _ptr(v), len(v), _ptr(t), len(t),
                                       int(exact_band), int(bool(exact_distance)), _ptr(sdf),
                                       _ptr(cl) if cl is not None else None)
        check("sc_mesh_to_sdf_host", rc, ctx.handle)
    return (sdf, cl) if closest else sdf


__all__ = ["manifold_to_sdf"]
