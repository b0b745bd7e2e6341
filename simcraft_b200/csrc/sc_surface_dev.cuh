// sc_surface_dev.cuh -- per-cube arithmetic of the marching-cubes surface export
// (rebuildSurface, FluidSim/src/cpu/rebuild-surface.cc:643-741), used by the
// kernels in sc_surface.cu.  Host and device: compiled as plain C++ the same
// functions replay the kernels' numbering on the CPU.
//
// Cubes.  Cube (i, j, k) has its lowest corner at sample (i, j, k) with i in
// [-1, nx-1] (likewise j, k), so there are (nx+1)(ny+1)(nz+1) cubes, numbered
// c = ((i+1) (ny+1) + (j+1)) (nz+1) + (k+1): the reference's loop order.  Samples
// outside the grid read 1000.
//
// Vertex numbering.  The reference numbers a vertex when it first meets its
// edge, visiting cubes in the order above and each cube's case entries in table
// order.  Every cube that shares an edge whose corners differ in sign lists that
// edge (each case lists exactly its sign-change edges), so the first cube to meet
// an edge is the lowest-numbered cube sharing it: the one that has the edge at
// its (1,1,1) corner, as its edge 5 (z), 6 (x) or 10 (y).  A cube therefore
// creates the vertices of its own crossing edges among {5, 6, 10}, in the order
// they first appear in its case; an exclusive scan of those counts over the cube
// order gives each cube's first vertex number.
#pragma once
#include <math.h>
#include <stdint.h>

#include "sc_mc_table.h"

#ifdef __CUDACC__
#define SC_HD __host__ __device__ __forceinline__
#else
#define SC_HD inline
#endif

namespace sc {
namespace mc {

// Round-to-nearest double operations that the compiler may not fuse, so that
// device and host evaluate the reference's expressions operation by operation.
#ifdef __CUDA_ARCH__
SC_HD double mul(double a, double b) { return __dmul_rn(a, b); }
SC_HD double add(double a, double b) { return __dadd_rn(a, b); }
SC_HD double sub(double a, double b) { return __dsub_rn(a, b); }
#else
SC_HD double mul(double a, double b) { return a * b; }
SC_HD double add(double a, double b) { return a + b; }
SC_HD double sub(double a, double b) { return a - b; }
#endif

struct Grid {
  int nx, ny, nz;
  double hx, hy, hz, ox, oy, oz;
  const double* sdf;  // reference layout, z fastest
  SC_HD int64_t cy() const { return (int64_t)ny + 1; }
  SC_HD int64_t cz() const { return (int64_t)nz + 1; }
  SC_HD int64_t ncubes() const { return ((int64_t)nx + 1) * cy() * cz(); }
  // evalSdf (rebuild-surface.cc:655-660)
  SC_HD double eval(int x, int y, int z) const {
    if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) return 1000.0;
    return sdf[((int64_t)x * ny + y) * nz + z];
  }
  SC_HD void cube(int64_t c, int& i, int& j, int& k) const {
    k = (int)(c % cz()) - 1;
    const int64_t r = c / cz();
    j = (int)(r % cy()) - 1;
    i = (int)(r / cy()) - 1;
  }
  SC_HD int64_t cube_index(int i, int j, int k) const {
    return ((int64_t)(i + 1) * cy() + (j + 1)) * cz() + (k + 1);
  }
  // bit c set when corner c has sdf < 0 (singleCube, :690-694)
  SC_HD int mask(int i, int j, int k) const {
    int m = 0;
    for (int c = 0; c < 8; c++)
      if (eval(i + SC_MC_CORNER_X(c), j + SC_MC_CORNER_Y(c), k + SC_MC_CORNER_Z(c)) < 0.0) m |= 1 << c;
    return m;
  }
  // grad (rebuild-surface.cc:666-686)
  SC_HD void grad(int x, int y, int z, double g[3]) const {
    const int xn = x < nx ? x + 1 : x, xp = x > -1 ? x - 1 : x;
    const int yn = y < ny ? y + 1 : y, yp = y > -1 ? y - 1 : y;
    const int zn = z < nz ? z + 1 : z, zp = z > -1 ? z - 1 : z;
    const double dx = x > -1 && x < nx - 1 ? 2.0 * hx : hx;
    const double dy = y > -1 && y < ny - 1 ? 2.0 * hy : hy;
    const double dz = z > -1 && z < nz - 1 ? 2.0 * hz : hz;
    g[0] = sub(eval(xn, y, z), eval(xp, y, z)) / dx;
    g[1] = sub(eval(x, yn, z), eval(x, yp, z)) / dy;
    g[2] = sub(eval(x, y, zn), eval(x, y, zp)) / dz;
  }
  // The vertex of edge e of cube (i, j, k) (singleCube, :705-719): position
  // lerp(pa, pb, t) = pa (1 - t) + pb t with t = va / (va - vb) between the
  // sample centres (index + 0.5) spacing + origin; normal
  // normalize(lerp(grad a, grad b, t)) = n * (1 / sqrt((nx nx + ny ny) + nz nz)).
  SC_HD void vertex(int i, int j, int k, int e, double p[3], double n[3]) const {
    const int ca = SC_MC_EDGE_A(e), cb = SC_MC_EDGE_B(e);
    const int ax = i + SC_MC_CORNER_X(ca), ay = j + SC_MC_CORNER_Y(ca), az = k + SC_MC_CORNER_Z(ca);
    const int bx = i + SC_MC_CORNER_X(cb), by = j + SC_MC_CORNER_Y(cb), bz = k + SC_MC_CORNER_Z(cb);
    const double pa[3] = {add(mul(add((double)ax, 0.5), hx), ox), add(mul(add((double)ay, 0.5), hy), oy),
                          add(mul(add((double)az, 0.5), hz), oz)};
    const double pb[3] = {add(mul(add((double)bx, 0.5), hx), ox), add(mul(add((double)by, 0.5), hy), oy),
                          add(mul(add((double)bz, 0.5), hz), oz)};
    double na[3], nb[3];
    grad(ax, ay, az, na);
    grad(bx, by, bz, nb);
    const double va = eval(ax, ay, az), vb = eval(bx, by, bz);
    const double t = va / sub(va, vb);
    const double s = sub(1.0, t);
    double m[3];
    for (int d = 0; d < 3; d++) {
      p[d] = add(mul(pa[d], s), mul(pb[d], t));
      m[d] = add(mul(na[d], s), mul(nb[d], t));
    }
    const double inv = 1.0 / sqrt(add(add(mul(m[0], m[0]), mul(m[1], m[1])), mul(m[2], m[2])));
    for (int d = 0; d < 3; d++) n[d] = mul(m[d], inv);
  }
};

// Edges a cube owns: the three at its (1,1,1) corner.
SC_HD bool owned(int e) { return e == 5 || e == 6 || e == 10; }
SC_HD int owned_bit(int e) { return e == 5 ? 1 : (e == 6 ? 2 : 4); }

// The cube that owns edge e of a cube, as an offset (d[0], d[1], d[2]) from it,
// and the owner's number for the edge.  The owner has the edge at coordinate 1
// on the two axes across it, so its offset there is the edge's coordinate in
// this cube minus 1, and 0 along the edge.
SC_HD int owner_of(int e, int d[3]) {
  const int a = SC_MC_EDGE_A(e), b = SC_MC_EDGE_B(e);
  const int ca[3] = {SC_MC_CORNER_X(a), SC_MC_CORNER_Y(a), SC_MC_CORNER_Z(a)};
  const int cb[3] = {SC_MC_CORNER_X(b), SC_MC_CORNER_Y(b), SC_MC_CORNER_Z(b)};
  int axis = 0;
  for (int q = 0; q < 3; q++) {
    d[q] = ca[q] - 1;
    if (cb[q] != ca[q]) {
      axis = q;
      d[q] = 0;
    }
  }
  return axis == 0 ? 6 : (axis == 1 ? 10 : 5);
}

// Vertices a cube creates: its crossing edges among {5, 6, 10}.
SC_HD int owned_count(uint64_t w) {
  int seen = 0;
  for (int q = 0; q < SC_MC_COUNT(w); q++) {
    const int e = SC_MC_ENTRY(w, q);
    if (owned(e)) seen |= owned_bit(e);
  }
  return (seen & 1) + ((seen >> 1) & 1) + ((seen >> 2) & 1);
}

// Rank of owned edge oe among the cube's own vertices: how many other owned
// edges first appear before oe in the case (-1 if the case lacks oe).
SC_HD int owned_rank(uint64_t w, int oe) {
  int seen = 0;
  for (int q = 0; q < SC_MC_COUNT(w); q++) {
    const int e = SC_MC_ENTRY(w, q);
    if (e == oe) return (seen & 1) + ((seen >> 1) & 1) + ((seen >> 2) & 1);
    if (owned(e)) seen |= owned_bit(e);
  }
  return -1;
}

// Writes the vertices and normals cube (i, j, k) with case word w creates,
// numbered from vbase (arrays of 3 doubles per vertex).
SC_HD void emit_vertices(const Grid& g, int i, int j, int k, uint64_t w, int64_t vbase, double* V,
                         double* N) {
  int seen = 0;
  int64_t v = vbase;
  for (int q = 0; q < SC_MC_COUNT(w); q++) {
    const int e = SC_MC_ENTRY(w, q);
    if (!owned(e) || (seen & owned_bit(e))) continue;
    seen |= owned_bit(e);
    double p[3], n[3];
    g.vertex(i, j, k, e, p, n);
    for (int d = 0; d < 3; d++) {
      V[3 * v + d] = p[d];
      N[3 * v + d] = n[d];
    }
    v++;
  }
}

// Writes the index entries of cube (i, j, k) with case word w from ibase.  The
// vertex of each entry comes from the edge's owner: vbase[owner] (the owner's
// first vertex number) plus the edge's rank in the owner's case.  An owner
// outside the cube range or a case without the edge (neither happens for a
// sign-change edge) writes 0xffffffff and returns false.
template <class Cases>
SC_HD bool emit_indices(const Grid& g, int i, int j, int k, uint64_t w, const Cases& cases,
                        const uint8_t* mask, const uint32_t* vbase, int64_t ibase, uint32_t* I) {
  bool ok = true;
  for (int q = 0; q < SC_MC_COUNT(w); q++) {
    const int e = SC_MC_ENTRY(w, q);
    int d[3];
    const int oe = owner_of(e, d);
    const int oi = i + d[0], oj = j + d[1], ok_ = k + d[2];
    uint32_t vid = 0xffffffffu;
    if (oi >= -1 && oj >= -1 && ok_ >= -1) {
      const int64_t oc = g.cube_index(oi, oj, ok_);
      const int r = owned_rank(cases(mask[oc]), oe);
      if (r >= 0) vid = vbase[oc] + (uint32_t)r;
    }
    if (vid == 0xffffffffu) ok = false;
    I[ibase + q] = vid;
  }
  return ok;
}

}  // namespace mc
}  // namespace sc
