"""Seeded synthetic scenes for the FLIP dam break and the standalone pressure solve.

The reference seeds nothing (`setInitialFluid` draws from an unseeded mt19937,
FluidSim/include/FluidSim/cpu/fluid-simulator.h:73-78, and the orphan CUDA test
uses std::random_device), so every scene here is generated once on the host
from numpy's PCG64 with a fixed seed and fed identically to the CUDA path and
to the CPU oracle.
"""
import numpy as np

# Domain is the unit cube; cells are cubic with h = 1/n.


def dam_break(n, frac_x=0.5, frac_y=0.5, frac_z=1.0, ppc=8, seed=1, dtype=np.float64):
    """Particles jittered uniformly inside every cell of the block
    x < frac_x, y < frac_y, z < frac_z of an n^3 grid; zero velocity.

    Particles are emitted cell by cell in the grid's (x, y, z) lexicographic
    order, `ppc` per cell, each at cell_min + h * U[0,1)^3.
    Returns (pos[P,3], vel[P,3], h)."""
    h = 1.0 / n
    cx, cy, cz = int(round(frac_x * n)), int(round(frac_y * n)), int(round(frac_z * n))
    ii, jj, kk = np.meshgrid(np.arange(cx), np.arange(cy), np.arange(cz), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    rng = np.random.default_rng(seed)
    jitter = rng.random((cells.shape[0], ppc, 3))
    pos = (cells[:, None, :] + jitter) * h
    pos = pos.reshape(-1, 3).astype(dtype)
    return np.ascontiguousarray(pos), np.zeros_like(pos), h


def _spheres(seed, count, rmin, rmax):
    rng = np.random.default_rng(seed)
    centres = rng.random((count, 3))
    radii = rmin + (rmax - rmin) * rng.random(count)
    return centres, radii


def sphere_union_sdf(n, centres, radii, chunk=32, device=None):
    """Signed distance to a union of spheres at the cell centres of an n^3 grid
    (min over spheres of |x - c| - r), float64, shape (n, n, n).  With a torch
    `device` the same double-precision expression is evaluated there, for large
    grids (values agree with the numpy path to within an ulp of the square root)."""
    if device is not None:
        return _sphere_union_sdf_torch(n, centres, radii, chunk, device)
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    out = np.empty((n, n, n))
    for i0 in range(0, n, chunk):
        xs = x[i0:i0 + chunk]
        best = np.full((len(xs), n, n), np.inf)
        for c, r in zip(centres, radii):
            d2 = ((xs - c[0]) ** 2)[:, None, None] + ((x - c[1]) ** 2)[None, :, None] + ((x - c[2]) ** 2)[None, None, :]
            np.minimum(best, np.sqrt(d2) - r, out=best)
        out[i0:i0 + chunk] = best
    return out


def _sphere_union_sdf_torch(n, centres, radii, chunk, device):
    import torch

    h = 1.0 / n
    x = (torch.arange(n, dtype=torch.float64, device=device) + 0.5) * h
    out = np.empty((n, n, n))
    for i0 in range(0, n, chunk):
        xs = x[i0:i0 + chunk]
        best = torch.full((len(xs), n, n), float("inf"), dtype=torch.float64, device=device)
        for c, r in zip(centres, radii):
            d2 = ((xs - float(c[0])) ** 2)[:, None, None] + ((x - float(c[1])) ** 2)[None, :, None] + \
                ((x - float(c[2])) ** 2)[None, None, :]
            torch.minimum(best, torch.sqrt(d2) - float(r), out=best)
        out[i0:i0 + chunk] = best.cpu().numpy()
    return out


def sphere_pool(n, count=24, rmin=0.05, rmax=0.2, fill=0.5, seed=2, probe=64, device=None):
    """Fluid mask of `count` seeded spheres (centres U[0,1)^3, radii U[rmin,rmax]).

    24 spheres of those radii cover only ~25% of the box, so all radii are
    scaled by one common factor, found by bisection on a probe grid, until the
    fluid fraction is `fill`.  Returns (fluid_sdf, info) with info holding the
    scale and the achieved fill on the full grid."""
    centres, radii = _spheres(seed, count, rmin, rmax)
    lo, hi = 0.5, 4.0
    for _ in range(30):
        mid = 0.5 * (lo + hi)
        f = float((sphere_union_sdf(probe, centres, radii * mid) <= 0.0).mean())
        if f < fill:
            lo = mid
        else:
            hi = mid
    scale = 0.5 * (lo + hi)
    sdf = sphere_union_sdf(n, centres, radii * scale, device=device)
    return sdf, dict(scale=scale, fill=float((sdf <= 0.0).mean()), centres=centres, radii=radii * scale)


def icosphere(subdiv=2, radius=0.3, centre=(0.5, 0.5, 0.5)):
    """Closed triangle mesh of a sphere: an icosahedron with each face split in
    four `subdiv` times, vertices pushed to the sphere.  Returns (vertices
    [V,3] float64, triangles [T,3] int32); T = 20 * 4^subdiv."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, float) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache, nf = {}, []

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v = np.array(verts) * radius + np.asarray(centre, float)
    return np.ascontiguousarray(v), np.ascontiguousarray(np.array(faces, np.int32))


def torus(n_major=24, n_minor=12, r_major=0.3, r_minor=0.1, centre=(0.5, 0.5, 0.5)):
    """Closed triangle mesh of a torus around the z axis through `centre`."""
    u = 2 * np.pi * np.arange(n_major) / n_major
    w = 2 * np.pi * np.arange(n_minor) / n_minor
    U, W = np.meshgrid(u, w, indexing="ij")
    rad = r_major + r_minor * np.cos(W)
    v = np.stack([rad * np.cos(U), rad * np.sin(U), r_minor * np.sin(W)], -1).reshape(-1, 3)
    v = v + np.asarray(centre, float)
    tris = []
    for i in range(n_major):
        for j in range(n_minor):
            a, b = i * n_minor + j, ((i + 1) % n_major) * n_minor + j
            c, d = ((i + 1) % n_major) * n_minor + (j + 1) % n_minor, i * n_minor + (j + 1) % n_minor
            tris += [(a, b, c), (a, c, d)]
    return np.ascontiguousarray(v), np.ascontiguousarray(np.array(tris, np.int32))


def box_mesh(lo=(0.3, 0.3, 0.3), hi=(0.7, 0.7, 0.7)):
    """Closed 12-triangle mesh of an axis-aligned box."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    v = np.array([[hi[0] if i & 1 else lo[0], hi[1] if i & 2 else lo[1], hi[2] if i & 4 else lo[2]]
                  for i in range(8)])
    tris = [(0, 2, 1), (1, 2, 3), (4, 5, 6), (5, 7, 6), (0, 1, 4), (1, 5, 4), (2, 6, 3), (3, 6, 7),
            (0, 4, 2), (2, 4, 6), (1, 3, 5), (3, 7, 5)]
    return np.ascontiguousarray(v), np.ascontiguousarray(np.array(tris, np.int32))


def poisson_rhs(active, fluid_sdf, seed=3):
    """Right-hand side U[-1,1] on active cells, mean-subtracted on every
    6-connected active component that has no air (fluid_sdf > 0) face
    neighbour, i.e. every component whose pure-Neumann system is singular."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    act = active.astype(bool)
    rhs = np.where(act, rng.uniform(-1.0, 1.0, size=active.shape), 0.0)
    labels, nlab = ndimage.label(act)
    if nlab == 0:
        return rhs, dict(components=0, enclosed=0)
    air = fluid_sdf > 0.0
    struct = ndimage.generate_binary_structure(3, 1)
    near_air = ndimage.binary_dilation(air, structure=struct) & act
    touches = np.zeros(nlab + 1, bool)
    touches[np.unique(labels[near_air])] = True
    enclosed = [l for l in range(1, nlab + 1) if not touches[l]]
    for l in enclosed:
        m = labels == l
        rhs[m] -= rhs[m].mean()
    return rhs, dict(components=int(nlab), enclosed=len(enclosed))
