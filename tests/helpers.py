"""Shared scene builders for the tests (seeded, small)."""
import numpy as np

from simcraft_b200 import scenes


def poisson_system(O, n, fill=0.5, seed=2, dims=None, dt_over_h=32.0 / 120.0):
    """A standalone pressure system: sphere-union fluid, buildSystem rules
    (empty collider, solid walls), random rhs on active cells."""
    dims = dims or (n, n, n)
    m = max(dims)
    sdf, info = scenes.sphere_pool(m, fill=fill, seed=seed, probe=min(m, 48))
    sdf = np.ascontiguousarray(sdf[: dims[0], : dims[1], : dims[2]])
    h = 1.0 / m
    nx, ny, nz = dims
    z = np.zeros
    S = O.build_system(dims, h, dt_over_h * h, z((nx + 1, ny, nz)), z((nx, ny + 1, nz)), z((nx, ny, nz + 1)), sdf)
    rhs, _ = scenes.poisson_rhs(S["active"], sdf, seed=seed + 1)
    S["rhs"] = np.ascontiguousarray(rhs)
    S["sdf"] = sdf
    S["h"] = h
    return S


def rel_l2(a, b, mask=None):
    if mask is not None:
        a, b = a[mask], b[mask]
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d
