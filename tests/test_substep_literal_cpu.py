"""The oracle's whole FLIP substep pinned on the CPU against a plain-Python
restatement of FluidSimulator::substep (FluidSim/src/cpu/fluid-simulator.cc:
139-181) that follows the reference statement by statement, buffers included:

* clear() (:21-38) zeroes the velocity grids, their buffers, weights, validity
  and pressure, but not the fluid-surface buffers, so advect (:143) samples the
  cleared grids and extrapolateFluidSdf / smoothFluidSurface (fluid-simulator.h
  :123-166, fluid-simulator.cc:40-73) read stale buffer values where a cell is
  valid (those cells are never written into the buffer before the swap);
* NaiveReconstructor::reconstruct with the Morton-bucket neighbour search
  (FluidSim/include/FluidSim/cpu/sdf.h:204-229, Spatify/include/Spatify/
  ns-util.h:46-109): the last particle of every bucket is skipped, buckets hold
  particles in ascending index (the reference's std::sort leaves that order
  open; the oracle pins it);
* P2G, the Dirichlet walls (:106-137), extrapolate (fluid-simulator.h:204-253,
  with the same stale-buffer swap), gravity on valid interior v faces
  (:13-18), buildSystem, the MIC(0)-PCG, project, applyCollider (:75-105) and
  FLIP G2P.

The restatement reuses the literal pieces of test_solver_literal_cpu and
test_transfer_literal_cpu; after each of two substeps of a small dam break
(with and without a collider) particles, pressure, faces, the fluid SDF and the
assembled system must equal the oracle's bit for bit.  Also restated: CFL and
the frame loop (fluid-simulator.cc:184-220), and the export path's
reconstruct() / smoothFluidSurface() between substeps."""
import math

import numpy as np
import pytest

from test_solver_literal_cpu import literal_build_system, literal_eval, literal_pcg, literal_project
from test_transfer_literal_cpu import OFFSETS, _nearest, literal_collide, literal_grad, literal_sample


def _morton10(x):
    x = (x | (x << 16)) & 0x030000FF
    x = (x | (x << 8)) & 0x0300F00F
    x = (x | (x << 4)) & 0x030C30C3
    x = (x | (x << 2)) & 0x09249249
    return x


def _morton(x, y, z):
    return _morton10(x) | (_morton10(y) << 1) | (_morton10(z) << 2)


def literal_reconstruct(pos, dims, h, radius):
    W, H, D = dims
    cells = []
    for p in pos:
        idx = []
        for a, n in enumerate(dims):
            c = int(math.floor(p[a] / h))
            idx.append(0 if c < 0 else (n - 1 if c >= n else c))
        cells.append(_morton(*idx))
    order = sorted(range(len(pos)), key=lambda i: (cells[i], i))
    sorted_cells = sorted(cells)
    begin, end = {}, {}
    for i, c in enumerate(sorted_cells):
        if i == 0 or sorted_cells[i - 1] != c:
            begin[c] = i
        if i == len(pos) - 1 or sorted_cells[i + 1] != c:
            end[c] = i
    sdf = np.full(dims, 1e9)
    valid = np.zeros(dims, np.uint8)
    r = 2 * radius

    def dist(a, b):
        d = (a[0] - b[0], a[1] - b[1], a[2] - b[2])
        return math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])

    for i in range(W):
        for j in range(H):
            for k in range(D):
                p = ((i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h)
                lo = [max(0, int(math.floor((p[a] - r) / h))) for a in range(3)]
                hi = [min(dims[a] - 1, int(math.ceil((p[a] + r) / h))) for a in range(3)]
                for x in range(lo[0], hi[0] + 1):
                    for y in range(lo[1], hi[1] + 1):
                        for z in range(lo[2], hi[2] + 1):
                            c = _morton(x, y, z)
                            for l in range(begin.get(c, -1), end.get(c, -1)):
                                q = pos[order[l]]
                                if dist(q, p) <= r:
                                    sdf[i, j, k] = min(sdf[i, j, k], dist(p, q) - radius)
                                    valid[i, j, k] = 1
    return sdf, valid


def _extrapolate(g, gbuf, valid, vbuf, iters, zero_invalid):
    """extrapolate / extrapolateFluidSdf: valid cells are not copied into the
    buffer, then the pair is swapped.  Returns the new (current, buffer) pairs."""
    W, H, D = g.shape
    for _ in range(iters):
        vbuf[...] = 0
        for i in range(W):
            for j in range(H):
                for k in range(D):
                    if valid[i, j, k]:
                        vbuf[i, j, k] = 1
                        continue
                    s, c = 0.0, 0
                    for (a, b, e, ok) in ((i - 1, j, k, i > 0), (i + 1, j, k, i < W - 1), (i, j - 1, k, j > 0),
                                          (i, j + 1, k, j < H - 1), (i, j, k - 1, k > 0), (i, j, k + 1, k < D - 1)):
                        if ok and valid[a, b, e]:
                            s += g[a, b, e]
                            c += 1
                    if c > 0:
                        gbuf[i, j, k] = s / c
                        vbuf[i, j, k] = 1
                    else:
                        if zero_invalid:
                            gbuf[i, j, k] = 0.0
                        vbuf[i, j, k] = 0
        g, gbuf = gbuf, g
        valid, vbuf = vbuf, valid
    return g, gbuf, valid, vbuf


class LiteralSim:
    def __init__(self, oracle, n, h, pos, vel, collider, alpha=0.97, tol=1e-6, max_iter=300):
        self.O, self.n, self.h = oracle, n, h
        self.dims = (n, n, n)
        shapes = ((n + 1, n, n), (n, n + 1, n), (n, n, n + 1))
        self.g = [np.zeros(s) for s in shapes]
        self.gbuf = [np.zeros(s) for s in shapes]
        self.valid = [np.zeros(s, np.uint8) for s in shapes]
        self.vbuf = [np.zeros(s, np.uint8) for s in shapes]
        self.last = [np.zeros(s) for s in shapes]
        self.surf, self.surfbuf = np.zeros(self.dims), np.zeros(self.dims)
        self.sval, self.svalbuf = np.zeros(self.dims, np.uint8), np.zeros(self.dims, np.uint8)
        self.pos = [list(p) for p in pos]
        self.vel = [list(v) for v in vel]
        self.C = collider
        self.alpha, self.tol, self.max_iter = alpha, tol, max_iter

    def smooth(self, iters):
        """smoothFluidSurface (fluid-simulator.cc:39-74)."""
        n = self.n
        for _ in range(iters):
            S, B = self.surf, self.surfbuf
            for i in range(n):
                for j in range(n):
                    for k in range(n):
                        s, c = 0.0, 0
                        for (a, b, e, ok) in ((i - 1, j, k, i > 0), (i + 1, j, k, i < n - 1), (i, j - 1, k, j > 0),
                                              (i, j + 1, k, j < n - 1), (i, j, k - 1, k > 0),
                                              (i, j, k + 1, k < n - 1)):
                            if ok:
                                s += S[a, b, e]
                                c += 1
                        B[i, j, k] = s / c
                        if S[i, j, k] < B[i, j, k]:
                            B[i, j, k] = S[i, j, k]
            self.surf, self.surfbuf = B, S

    def cfl(self, factor):
        """FluidSimulator::CFL (fluid-simulator.cc:184-203): h / |u| over the
        non-zero face velocities, floored at 1e-3, times the CFL factor."""
        h = self.h
        c = h / 1e-6
        for G in self.g:
            for u in G.ravel().tolist():
                if u != 0.0:
                    c = min(c, h / abs(u))
        return factor * max(1e-3, c)

    def step(self, frame_dt, factor):
        """FluidSimulator::step (fluid-simulator.cc:205-220)."""
        t = 0.0
        count = 0
        while t < frame_dt:
            dt = min(self.cfl(factor), frame_dt - t)
            self.substep(dt)
            t += dt
            count += 1
        return count

    def reconstruct(self):
        """FluidSimulator::reconstruct (cpu/fluid-simulator.h:115-119)."""
        sdf, valid = literal_reconstruct(self.pos, self.dims, self.h, 1.2 * self.h / math.sqrt(2.0))
        self.surf[...] = sdf
        self.sval[...] = valid

    def substep(self, dt):
        O, n, h, dims = self.O, self.n, self.h, self.dims
        for a in range(3):  # clear()
            self.g[a][...] = 0.0
            self.gbuf[a][...] = 0.0
            self.valid[a][...] = 0
            self.vbuf[a][...] = 0
        box = (n * h, n * h, n * h)
        C = self.C
        for i in range(len(self.pos)):  # advect through the cleared grids
            p, v = self.pos[i], self.vel[i]
            k1 = list(v)
            p1 = [p[a] + 0.5 * dt * k1[a] for a in range(3)]
            k2 = literal_sample(O, p1, h, self.g)
            p2 = [p[a] + 0.75 * dt * k2[a] for a in range(3)]
            k3 = literal_sample(O, p2, h, self.g)
            q = [p[a] + 2.0 / 9.0 * dt * k1[a] + 1.0 / 3.0 * dt * k2[a] + 4.0 / 9.0 * dt * k3[a] for a in range(3)]
            self.pos[i], self.vel[i] = literal_collide(C, h, box, q, v)
        sdf, valid = literal_reconstruct(self.pos, dims, h, 0.8 * h)
        self.surf[...] = sdf
        self.sval[...] = valid
        self.surf, self.surfbuf, self.sval, self.svalbuf = _extrapolate(self.surf, self.surfbuf, self.sval,
                                                                        self.svalbuf, 10, zero_invalid=False)
        self.smooth(5)
        # P2G into the cleared grids, serial particle order
        wsum = [np.zeros_like(x) for x in self.g]
        for p, v in zip(self.pos, self.vel):
            idx = [_nearest(p, off, h) for off in OFFSETS]
            for i in range(-1, 3):
                for j in range(-1, 3):
                    for k in range(-1, 3):
                        for a in range(3):
                            nd = (idx[a][0] + i, idx[a][1] + j, idx[a][2] + k)
                            if not all(0 <= nd[b] < self.g[a].shape[b] for b in range(3)):
                                continue
                            pn = [(nd[b] + OFFSETS[a][b]) * h + 0.0 for b in range(3)]
                            wt = O.cubic_weight(h, [p[b] - pn[b] for b in range(3)])
                            self.g[a][nd] += v[a] * wt
                            wsum[a][nd] += wt
        for a in range(3):
            ok = wsum[a] > 0.0
            self.g[a][...] = np.where(ok, self.g[a] / np.where(ok, wsum[a], 1.0), 0.0)
            self.valid[a][...] = ok
            self.last[a] = self.g[a].copy()
        # applyDirichletBoundary
        self.g[0][0], self.g[0][-1], self.valid[0][0], self.valid[0][-1] = 0.0, 0.0, 1, 1
        self.g[1][:, 0], self.g[1][:, -1], self.valid[1][:, 0], self.valid[1][:, -1] = 0.0, 0.0, 1, 1
        self.g[2][:, :, 0], self.g[2][:, :, -1], self.valid[2][:, :, 0], self.valid[2][:, :, -1] = 0.0, 0.0, 1, 1
        for a in range(3):
            self.g[a], self.gbuf[a], self.valid[a], self.vbuf[a] = _extrapolate(
                self.g[a], self.gbuf[a], self.valid[a], self.vbuf[a], 10, zero_invalid=True)
        # applyForce
        vg, vv = self.g[1], self.valid[1]
        for i in range(vg.shape[0]):
            for j in range(vg.shape[1]):
                for k in range(vg.shape[2]):
                    if vv[i, j, k] and 0 < j < vg.shape[1] - 1:
                        vg[i, j, k] -= 9.8 * dt
        Cs = C if C is not None else np.full(dims, 1e9)
        self.system = literal_build_system(dims, h, dt, *self.g, self.surf, Cs)
        S = self.system
        self.pg, _, self.iters = literal_pcg(S["adiag"], S["an"], S["rhs"], S["active"], self.tol, self.max_iter,
                                            0.97, 0.25)
        self.g = list(literal_project(dims, h, dt, *self.g, self.pg, self.surf, S["uwt"], S["vwt"], S["wwt"]))
        # applyCollider
        for a in range(3):
            G = self.g[a]
            for i in range(G.shape[0]):
                for j in range(G.shape[1]):
                    for k in range(G.shape[2]):
                        ijk = (i, j, k)
                        if ijk[a] == 0 or ijk[a] == G.shape[a] - 1:
                            G[ijk] = 0.0
                            continue
                        pos = [(ijk[b] + OFFSETS[a][b]) * h + 0.0 for b in range(3)]
                        if literal_eval(Cs, h, tuple(pos)) < 0.0:
                            gr = literal_grad(Cs, h, pos)
                            inv = 1.0 / math.sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2])
                            G[ijk] -= G[ijk] * (gr[a] * inv)
        # FLIP G2P
        for i, p in enumerate(self.pos):
            pic = literal_sample(O, p, h, self.g)
            old = literal_sample(O, p, h, self.last)
            flip = [self.vel[i][a] + pic[a] - old[a] for a in range(3)]
            self.vel[i] = [self.alpha * flip[a] + (1.0 - self.alpha) * pic[a] for a in range(3)]


@pytest.mark.parametrize("collider", [False, True])
def test_substep_equals_literal(oracle, collider):
    from simcraft_b200 import scenes

    n = 8
    pos, vel, h = scenes.dam_break(n, ppc=2, seed=3)
    vel = np.random.default_rng(5).uniform(-0.5, 0.5, pos.shape)
    C = None
    if collider:
        x = (np.arange(n) + 0.5) * h
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        C = np.sqrt((X - 0.62) ** 2 + (Y - 0.2) ** 2 + (Z - 0.5) ** 2) - 0.2
    cfg = oracle.default_config(n, n, n, h)
    sim = oracle.Sim(**cfg)
    sim.set_particles(pos, vel)
    if C is not None:
        sim.set_collider(C)
    lit = LiteralSim(oracle, n, h, pos, vel, C)
    for step in range(2):
        dt = 1.0 / 120
        sim.substep(dt)
        lit.substep(dt)
        p, v = sim.particles()
        assert np.array_equal(p, np.array(lit.pos)), step
        assert np.array_equal(v, np.array(lit.vel)), step
        assert np.array_equal(sim.fluid_sdf(), lit.surf), step
        assert np.array_equal(sim.pressure(), lit.pg), step
        for a, b in zip(sim.faces(), lit.g):
            assert np.array_equal(a, b), step
        adiag, an, rhs, act = sim.system()
        assert np.array_equal(adiag, lit.system["adiag"]) and np.array_equal(rhs, lit.system["rhs"])
        assert np.array_equal(act, lit.system["active"]) and lit.iters > 1


def test_export_calls_between_substeps_equal_literal(oracle):
    """The reference's export path (FluidSim/disabled/fluid-sim.cc:231-235)
    calls reconstruct() and smoothFluidSurface(5) between frames; both act on
    the simulator's surface buffers, so they change the stale values the next
    substep's extrapolation reads.  The oracle follows the literal simulator
    through substep, reconstruct, smooth, substep."""
    from simcraft_b200 import scenes

    n = 8
    pos, vel, h = scenes.dam_break(n, ppc=2, seed=7)
    sim = oracle.Sim(**oracle.default_config(n, n, n, h))
    sim.set_particles(pos, vel)
    lit = LiteralSim(oracle, n, h, pos, vel, None)
    dt = 1.0 / 120
    sim.substep(dt)
    lit.substep(dt)
    sim.reconstruct()
    lit.reconstruct()
    assert np.array_equal(sim.fluid_sdf(), lit.surf)
    sim.smooth_fluid_surface(5)
    lit.smooth(5)
    assert np.array_equal(sim.fluid_sdf(), lit.surf)
    sim.substep(dt)
    lit.substep(dt)
    p, v = sim.particles()
    assert np.array_equal(p, np.array(lit.pos)) and np.array_equal(v, np.array(lit.vel))
    assert np.array_equal(sim.fluid_sdf(), lit.surf) and np.array_equal(sim.pressure(), lit.pg)


def test_frame_loop_equals_literal(oracle):
    """step(frame) (fluid-simulator.cc:205-220): substeps of min(CFL, rest of the
    frame) until the frame is covered; a CFL factor of 0.2 makes the second
    frame take several substeps."""
    from simcraft_b200 import scenes

    n = 8
    pos, vel, h = scenes.dam_break(n, ppc=2, seed=9)
    vel = np.random.default_rng(10).uniform(-0.5, 0.5, pos.shape)
    factor = 0.2
    sim = oracle.Sim(**oracle.default_config(n, n, n, h, cfl_factor=factor))
    sim.set_particles(pos, vel)
    lit = LiteralSim(oracle, n, h, pos, vel, None)
    counts = []
    for frame in range(2):
        sim.step(0.05)
        counts.append(lit.step(0.05, factor))
        p, v = sim.particles()
        assert np.array_equal(p, np.array(lit.pos)) and np.array_equal(v, np.array(lit.vel)), frame
        assert np.array_equal(sim.pressure(), lit.pg), frame
    assert counts[0] == 1 and counts[1] > 1, counts  # the grids are empty before the first substep
    assert sim.cfl() == lit.cfl(factor)
