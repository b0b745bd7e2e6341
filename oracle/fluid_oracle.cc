// fluid_oracle.cc -- CPU restatement of SimCraft FluidSim's FLIP/PIC step, FP64.
//
// TEST INFRASTRUCTURE ONLY: the parity checker for simcraft_b200 and the timed
// CPU baseline of bench.py.  Each function follows the cited reference
// function loop for loop (same loop order, same masks, same buffer swaps,
// same arithmetic order); TBB parallel loops become OpenMP loops.  Paths are
// relative to the SimCraft tree.
#include "fluid_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 1;
int g_parity = 1;
// Bucket order of the reconstruction's neighbour search: 0 = (cell, particle
// id), stable; 1 = the reference's own, std::sort of the particle indices by
// Morton key (ns-util.h:46-79), which is not stable.
int g_bucket_order = 0;

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// glm::normalize, which the reference uses (Core/include/Core/utils.h:18):
// v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x).
inline V3 normalize3(V3 a) {
  const double inv = 1.0 / std::sqrt(dot3(a, a));
  return {a.x * inv, a.y * inv, a.z * inv};
}

// Dense 3-D view, spatify::LinearHashXYZ order (Spatify/include/Spatify/hash.h:23-26).
template <class T>
struct A3 {
  T* d;
  int w, h, dp;
  T& operator()(int i, int j, int k) const {
    return d[k + (int64_t)j * dp + (int64_t)i * h * dp];
  }
  int64_t size() const { return (int64_t)w * h * dp; }
};

// Face-centred grid geometry (Spatify/include/Spatify/grids.h:287-308, 479-485).
struct FaceGeom {
  int w, h, d;          // node counts
  double ox, oy, oz;    // offsets in cells
  double sp;            // spacing
  // TGrid::nearest: Vec3i((coord - origin - offset*h)/h + 0.5), truncation.
  void nearest(const V3& p, int& i, int& j, int& k) const {
    i = (int)((p.x - 0.0 - ox * sp) / sp + 0.5);
    j = (int)((p.y - 0.0 - oy * sp) / sp + 0.5);
    k = (int)((p.z - 0.0 - oz * sp) / sp + 0.5);
  }
  // TGrid::indexToCoord: (index + offset) * spacing + origin.
  V3 coord(int i, int j, int k) const {
    return {((double)i + ox) * sp + 0.0, ((double)j + oy) * sp + 0.0,
            ((double)k + oz) * sp + 0.0};
  }
};

FaceGeom ugeom(int nx, int ny, int nz, double h) { return {nx + 1, ny, nz, 0.0, 0.5, 0.5, h}; }
FaceGeom vgeom(int nx, int ny, int nz, double h) { return {nx, ny + 1, nz, 0.5, 0.0, 0.5, h}; }
FaceGeom wgeom(int nx, int ny, int nz, double h) { return {nx, ny, nz + 1, 0.5, 0.5, 0.0, h}; }

// Cubic B-spline N(r), r = |d|/h: the documented policy for the missing
// core::CubicKernel::weight<Real,3>(h, d) (call sites advect-solver.cc:44,214; util.cc:58).
inline double bspline(double r) {
  if (r < 1.0) return 2.0 / 3.0 - r * r + 0.5 * r * r * r;
  if (r < 2.0) {
    double t = 2.0 - r;
    return t * t * t / 6.0;
  }
  return 0.0;
}
inline double kweight(double h, V3 d) {
  return bspline(std::fabs(d.x) / h) * bspline(std::fabs(d.y) / h) *
         bspline(std::fabs(d.z) / h);
}

inline V3 ld3(const double* p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void st3(double* p, int64_t i, V3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

// sampleVelocity (FluidSim/src/cpu/util.cc:40-85).
V3 sample_velocity(V3 p, int nx, int ny, int nz, double h, const double* u, const double* v,
                   const double* w) {
  FaceGeom gu = ugeom(nx, ny, nz, h), gv = vgeom(nx, ny, nz, h), gw = wgeom(nx, ny, nz, h);
  A3<const double> U{u, gu.w, gu.h, gu.d}, Vv{v, gv.w, gv.h, gv.d}, W{w, gw.w, gw.h, gw.d};
  int ui, uj, uk, vi, vj, vk, wi, wj, wk;
  gu.nearest(p, ui, uj, uk);
  gv.nearest(p, vi, vj, vk);
  gw.nearest(p, wi, wj, wk);
  double su = 0.0, sv = 0.0, sw = 0.0, wu = 0.0, wv = 0.0, ww = 0.0;
  for (int i = -1; i <= 2; i++)
    for (int j = -1; j <= 2; j++)
      for (int k = -1; k <= 2; k++) {
        if (ui + i >= 0 && ui + i < gu.w && uj + j >= 0 && uj + j < gu.h && uk + k >= 0 &&
            uk + k < gu.d) {
          double un = U(ui + i, uj + j, uk + k);
          double wt = kweight(h, p - gu.coord(ui + i, uj + j, uk + k));
          su += un * wt;
          wu += wt;
        }
        if (vi + i >= 0 && vi + i < gv.w && vj + j >= 0 && vj + j < gv.h && vk + k >= 0 &&
            vk + k < gv.d) {
          double vn = Vv(vi + i, vj + j, vk + k);
          double wt = kweight(h, p - gv.coord(vi + i, vj + j, vk + k));
          sv += vn * wt;
          wv += wt;
        }
        if (wi + i >= 0 && wi + i < gw.w && wj + j >= 0 && wj + j < gw.h && wk + k >= 0 &&
            wk + k < gw.d) {
          double wn = W(wi + i, wj + j, wk + k);
          double wt = kweight(h, p - gw.coord(wi + i, wj + j, wk + k));
          sw += wn * wt;
          ww += wt;
        }
      }
  return {wu > 0.0 ? su / wu : 0.0, wv > 0.0 ? sv / wv : 0.0, ww > 0.0 ? sw / ww : 0.0};
}

// One particle's splat into one face grid (advect-solver.cc:207-235 inner body).
inline void splat_one(const FaceGeom& g, A3<double>& G, A3<double>& Wt, V3 p, double val) {
  int bi, bj, bk;
  g.nearest(p, bi, bj, bk);
  for (int i = -1; i <= 2; i++)
    for (int j = -1; j <= 2; j++)
      for (int k = -1; k <= 2; k++) {
        if (bi + i >= 0 && bi + i < g.w && bj + j >= 0 && bj + j < g.h && bk + k >= 0 &&
            bk + k < g.d) {
          double wt = kweight(g.sp, p - g.coord(bi + i, bj + j, bk + k));
          G(bi + i, bj + j, bk + k) += val * wt;
          Wt(bi + i, bj + j, bk + k) += wt;
        }
      }
}

// Normalisation pass (advect-solver.cc:238-267).
void normalise(A3<double>& G, const A3<double>& Wt, uint8_t* valid) {
  int64_t n = G.size();
  std::memset(valid, 0, (size_t)n);
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < G.w; i++)
    for (int j = 0; j < G.h; j++)
      for (int k = 0; k < G.dp; k++) {
        int64_t id = k + (int64_t)j * G.dp + (int64_t)i * G.h * G.dp;
        if (Wt.d[id] > 0.0) {
          G.d[id] /= Wt.d[id];
          valid[id] = 1;
        } else {
          G.d[id] = 0.0;
          valid[id] = 0;
        }
      }
}

inline double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }
inline int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// SDF<3>::eval, including the reference's reversed trilinear weights (sdf.h:35-61).
double sdf_eval(const double* sdf, int nx, int ny, int nz, double h, V3 p) {
  A3<const double> S{sdf, nx, ny, nz};
  // coordToSampledCellIndex: Vec3i((coord - origin)/h - offset) (grids.h:298-300).
  int ix = (int)((p.x - 0.0) / h - 0.5), iy = (int)((p.y - 0.0) / h - 0.5),
      iz = (int)((p.z - 0.0) / h - 0.5);
  int x = clampi(ix, 0, nx - 1), y = clampi(iy, 0, ny - 1), z = clampi(iz, 0, nz - 1);
  int xn = clampi(ix + 1, 0, nx - 1), yn = clampi(iy + 1, 0, ny - 1),
      zn = clampi(iz + 1, 0, nz - 1);
  double px = ((double)x + 0.5) * h + 0.0, py = ((double)y + 0.5) * h + 0.0,
         pz = ((double)z + 0.5) * h + 0.0;
  double tx = clampd((p.x - px) / h, 0.0, 1.0);
  double ty = clampd((p.y - py) / h, 0.0, 1.0);
  double tz = clampd((p.z - pz) / h, 0.0, 1.0);
  return tx * ty * tz * S(x, y, z) + tx * ty * (1 - tz) * S(x, y, zn) +
         tx * (1 - ty) * tz * S(x, yn, z) + tx * (1 - ty) * (1 - tz) * S(x, yn, zn) +
         (1 - tx) * ty * tz * S(xn, y, z) + (1 - tx) * ty * (1 - tz) * S(xn, y, zn) +
         (1 - tx) * (1 - ty) * tz * S(xn, yn, z) +
         (1 - tx) * (1 - ty) * (1 - tz) * S(xn, yn, zn);
}

// SDF<3>::gradient(idx) (sdf.h:62-85).
V3 sdf_gradient_at(const double* sdf, int nx, int ny, int nz, double h, int ix, int iy, int iz) {
  A3<const double> S{sdf, nx, ny, nz};
  int xn = ix < nx - 1 ? ix + 1 : ix, xp = ix > 0 ? ix - 1 : ix;
  int yn = iy < ny - 1 ? iy + 1 : iy, yp = iy > 0 ? iy - 1 : iy;
  int zn = iz < nz - 1 ? iz + 1 : iz, zp = iz > 0 ? iz - 1 : iz;
  double dx = ix > 0 && ix < nx - 1 ? 2 * h : h;
  double dy = iy > 0 && iy < ny - 1 ? 2 * h : h;
  double dz = iz > 0 && iz < nz - 1 ? 2 * h : h;
  double gx = S(xn, iy, iz) - S(xp, iy, iz);
  double gy = S(ix, yn, iz) - S(ix, yp, iz);
  double gz = S(ix, iy, zn) - S(ix, iy, zp);
  return {gx / dx, gy / dy, gz / dz};
}

// SDF<3>::grad(p) (sdf.h:86-118).
V3 sdf_grad(const double* sdf, int nx, int ny, int nz, double h, V3 p) {
  int ix = (int)((p.x - 0.0) / h - 0.5), iy = (int)((p.y - 0.0) / h - 0.5),
      iz = (int)((p.z - 0.0) / h - 0.5);
  int x = clampi(ix, 0, nx - 1), y = clampi(iy, 0, ny - 1), z = clampi(iz, 0, nz - 1);
  int xn = clampi(ix + 1, 0, nx - 1), yn = clampi(iy + 1, 0, ny - 1),
      zn = clampi(iz + 1, 0, nz - 1);
  double tx = (p.x - (((double)x + 0.5) * h + 0.0)) / h;
  double ty = (p.y - (((double)y + 0.5) * h + 0.0)) / h;
  double tz = (p.z - (((double)z + 0.5) * h + 0.0)) / h;
  V3 g000 = sdf_gradient_at(sdf, nx, ny, nz, h, x, y, z);
  V3 g001 = sdf_gradient_at(sdf, nx, ny, nz, h, x, y, zn);
  V3 g010 = sdf_gradient_at(sdf, nx, ny, nz, h, x, yn, z);
  V3 g011 = sdf_gradient_at(sdf, nx, ny, nz, h, x, yn, zn);
  V3 g100 = sdf_gradient_at(sdf, nx, ny, nz, h, xn, y, z);
  V3 g101 = sdf_gradient_at(sdf, nx, ny, nz, h, xn, y, zn);
  V3 g110 = sdf_gradient_at(sdf, nx, ny, nz, h, xn, yn, z);
  V3 g111 = sdf_gradient_at(sdf, nx, ny, nz, h, xn, yn, zn);
  return (tx * ty * tz) * g000 + (tx * ty * (1 - tz)) * g001 + (tx * (1 - ty) * tz) * g010 +
         (tx * (1 - ty) * (1 - tz)) * g011 + ((1 - tx) * ty * tz) * g100 +
         ((1 - tx) * ty * (1 - tz)) * g101 + ((1 - tx) * (1 - ty) * tz) * g110 +
         ((1 - tx) * (1 - ty) * (1 - tz)) * g111;
}

// HybridAdvectionSolver3D::handleCollision (advect-solver.cc:100-137).
void handle_collision(const double* collider, int nx, int ny, int nz, double h, V3& p, V3& v) {
  double width = nx * h, height = ny * h, depth = nz * h;
  if (collider) {
    double d = sdf_eval(collider, nx, ny, nz, h, p);
    if (d < 0.0) {
      V3 n = normalize3(sdf_grad(collider, nx, ny, nz, h, p));
      p = p - d * n;
      v = v - std::min(dot3(v, n), 0.0) * n;
    }
  }
  if (p.x < 0.0) {
    p.x = 0.0;
    if (v.x < 0.0) v.x = 0.0;
  }
  if (p.x > width) {
    p.x = width;
    if (v.x > 0.0) v.x = 0.0;
  }
  if (p.y < 0.0) {
    p.y = 0.0;
    if (v.y < 0.0) v.y = 0.0;
  }
  if (p.y > height) {
    p.y = height;
    if (v.y > 0.0) v.y = 0.0;
  }
  if (p.z < 0.0) {
    p.z = 0.0;
    if (v.z < 0.0) v.z = 0.0;
  }
  if (p.z > depth) {
    p.z = depth;
    if (v.z > 0.0) v.z = 0.0;
  }
}

enum { Left = 0, Right = 1, Up = 2, Down = 3, Front = 4, Back = 5 };

// ---------------------------------------------------------------------------
// Mesh -> signed distance grid: manifold2SDF (FluidSim/src/cpu/util.cc:203-310)
// and its helpers, in the reference's operation order.  Grid cell (x, y, z)
// sits at ((x + 0.5) h + ox, ...) (CellCentredGrid::indexToCoord,
// Spatify/include/Spatify/grids.h:303-308).

// distancePointTriangle (util.cc:87-125): closest point by Voronoi regions.
// The reference measures |ap + v ab| on edge AB, |ap + w ac| on edge AC and
// |ap + v ab + w ac| inside the face, where the offset to the closest point is
// ap - v ab (etc.), so it overstates those distances; `exact` selects the
// offsets with the minus signs (vertices and edge BC agree in both).
double dist_point_tri(V3 p, V3 a, V3 b, V3 c, bool exact) {
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0 && d2 <= 0) return std::sqrt(dot3(ap, ap));
  const V3 bp = p - b;
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0 && d4 <= d3) return std::sqrt(dot3(bp, bp));
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const double v = d1 / (d1 - d3);
    const V3 q = exact ? ap - v * ab : ap + v * ab;
    return std::sqrt(dot3(q, q));
  }
  const V3 cp = p - c;
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0 && d5 <= d6) return std::sqrt(dot3(cp, cp));
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const double w = d2 / (d2 - d6);
    const V3 q = exact ? ap - w * ac : ap + w * ac;
    return std::sqrt(dot3(q, q));
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    const V3 q = bp + w * (cp - bp);
    return std::sqrt(dot3(q, q));
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  const V3 q = exact ? (ap - v * ab) - w * ac : (ap + v * ab) + w * ac;
  return std::sqrt(dot3(q, q));
}

// cross / insideTraingle2D (util.cc:127-142): all three edge tests agree.
inline double cross2(double ax, double ay, double bx, double by) { return ax * by - bx * ay; }
bool inside_tri_2d(double px, double py, V3 a, V3 b, V3 c) {
  const int cnt = (cross2(px - a.x, py - a.y, b.x - a.x, b.y - a.y) >= 0.0) +
                  (cross2(px - b.x, py - b.y, c.x - b.x, c.y - b.y) >= 0.0) +
                  (cross2(px - c.x, py - c.y, a.x - c.x, a.y - c.y) >= 0.0);
  return cnt == 3 || cnt == 0;
}

// solveEquations / calcBiocentricCoord (util.cc:144-157).
void bary_2d(double px, double py, V3 a, V3 b, V3 c, double* u, double* v, double* w) {
  const double a1 = a.x - c.x, b1 = b.x - c.x, c1 = px - c.x;
  const double a2 = a.y - c.y, b2 = b.y - c.y, c2 = py - c.y;
  const double det = a1 * b2 - a2 * b1;
  *u = (c1 * b2 - c2 * b1) / det;
  *v = (a1 * c2 - a2 * c1) / det;
  *w = 1.0 - (*u) - (*v);
}

struct MeshGrid {
  int nx, ny, nz;
  double h, ox, oy, oz;
  const double* vert;
  const int* tri;
  bool exact;
  V3 vtx(int t, int k) const { return ld3(vert, tri[3 * t + k]); }
  V3 coord(int x, int y, int z) const {
    return {(x + 0.5) * h + ox, (y + 0.5) * h + oy, (z + 0.5) * h + oz};
  }
  int64_t at(int x, int y, int z) const { return ((int64_t)x * ny + y) * nz + z; }
};

// checkNeighbour (util.cc:159-180).  The reference writes abs(); on doubles
// that is fabs.
void check_neighbour(const MeshGrid& M, double* sdf, int* closest, int dx, int dy, int dz, int x,
                     int y, int z) {
  if (x + dx < 0 || x + dx >= M.nx || y + dy < 0 || y + dy >= M.ny || z + dz < 0 || z + dz >= M.nz)
    return;
  const int t = closest[M.at(x + dx, y + dy, z + dz)];
  if (t == -1) return;
  const int64_t e = M.at(x, y, z);
  const double d1 = dist_point_tri(M.coord(x, y, z), M.vtx(t, 0), M.vtx(t, 1), M.vtx(t, 2), M.exact);
  if (std::fabs(d1) < std::fabs(sdf[e])) {
    sdf[e] = d1;
    closest[e] = t;
  }
}

// sweep (util.cc:182-201): one Gauss-Seidel pass in the direction (-dx, -dy, -dz).
void mesh_sweep(const MeshGrid& M, double* sdf, int* closest, int dx, int dy, int dz) {
  const int xs = dx < 0 ? 0 : M.nx - 1, xe = dx < 0 ? M.nx : -1;
  const int ys = dy < 0 ? 0 : M.ny - 1, ye = dy < 0 ? M.ny : -1;
  const int zs = dz < 0 ? 0 : M.nz - 1, ze = dz < 0 ? M.nz : -1;
  for (int x = xs; x != xe; x -= dx)
    for (int y = ys; y != ye; y -= dy)
      for (int z = zs; z != ze; z -= dz) {
        check_neighbour(M, sdf, closest, 0, dy, dz, x, y, z);
        check_neighbour(M, sdf, closest, dx, 0, dz, x, y, z);
        check_neighbour(M, sdf, closest, dx, dy, 0, x, y, z);
        check_neighbour(M, sdf, closest, 0, 0, dz, x, y, z);
        check_neighbour(M, sdf, closest, 0, dy, 0, x, y, z);
        check_neighbour(M, sdf, closest, dx, 0, 0, x, y, z);
        check_neighbour(M, sdf, closest, dx, dy, dz, x, y, z);
      }
}

}  // namespace

extern "C" {

void ora_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
void ora_set_parity_mode(int on) { g_parity = on; }
void ora_set_bucket_order(int mode) { g_bucket_order = mode; }
int ora_get_threads(void) { return g_threads; }

double ora_cubic_weight(double h, double dx, double dy, double dz) {
  return kweight(h, V3{dx, dy, dz});
}

void ora_p2g(int64_t n, const double* pos, const double* vel, int nx, int ny, int nz, double h,
             double* u, double* v, double* w, double* uw, double* vw, double* ww,
             uint8_t* uvalid, uint8_t* vvalid, uint8_t* wvalid, double* ulast, double* vlast,
             double* wlast) {
  FaceGeom gu = ugeom(nx, ny, nz, h), gv = vgeom(nx, ny, nz, h), gw = wgeom(nx, ny, nz, h);
  A3<double> U{u, gu.w, gu.h, gu.d}, Vv{v, gv.w, gv.h, gv.d}, W{w, gw.w, gw.h, gw.d};
  A3<double> UW{uw, gu.w, gu.h, gu.d}, VW{vw, gv.w, gv.h, gv.d}, WW{ww, gw.w, gw.h, gw.d};
  if (g_parity || g_threads == 1) {
    // Serial particle order (PicAdvector3D::solveP2G is serial; the FLIP version's
    // tbb::parallel_for with plain += is a data race, advect-solver.cc:201-237).
    for (int64_t idx = 0; idx < n; idx++) {
      V3 p = ld3(pos, idx), vv = ld3(vel, idx);
      // The reference interleaves u/v/w inside one (i,j,k) loop; per-grid sums
      // are independent, so splatting grid by grid gives identical sums.
      splat_one(gu, U, UW, p, vv.x);
      splat_one(gv, Vv, VW, p, vv.y);
      splat_one(gw, W, WW, p, vv.z);
    }
  } else {
    // Timing mode: per-thread accumulation, then a reduction.
    int T = g_threads;
    int64_t su = U.size(), sv = Vv.size(), sw = W.size();
    std::vector<std::vector<double>> bufs(T);
#pragma omp parallel num_threads(T)
    {
      int t = 0;
#ifdef _OPENMP
      t = omp_get_thread_num();
#endif
      auto& b = bufs[t];
      b.assign((size_t)(2 * (su + sv + sw)), 0.0);
      A3<double> tu{b.data(), gu.w, gu.h, gu.d}, tuw{b.data() + su, gu.w, gu.h, gu.d};
      A3<double> tv{b.data() + 2 * su, gv.w, gv.h, gv.d},
          tvw{b.data() + 2 * su + sv, gv.w, gv.h, gv.d};
      A3<double> tw{b.data() + 2 * (su + sv), gw.w, gw.h, gw.d},
          tww{b.data() + 2 * (su + sv) + sw, gw.w, gw.h, gw.d};
#pragma omp for schedule(static)
      for (int64_t idx = 0; idx < n; idx++) {
        V3 p = ld3(pos, idx), vv = ld3(vel, idx);
        splat_one(gu, tu, tuw, p, vv.x);
        splat_one(gv, tv, tvw, p, vv.y);
        splat_one(gw, tw, tww, p, vv.z);
      }
    }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < su; i++)
      for (int t = 0; t < T; t++) {
        u[i] += bufs[t][i];
        uw[i] += bufs[t][su + i];
      }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < sv; i++)
      for (int t = 0; t < T; t++) {
        v[i] += bufs[t][2 * su + i];
        vw[i] += bufs[t][2 * su + sv + i];
      }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t i = 0; i < sw; i++)
      for (int t = 0; t < T; t++) {
        w[i] += bufs[t][2 * (su + sv) + i];
        ww[i] += bufs[t][2 * (su + sv) + sw + i];
      }
  }
  normalise(U, UW, uvalid);
  normalise(Vv, VW, vvalid);
  normalise(W, WW, wvalid);
  if (ulast) {  // advect-solver.cc:268-270
    std::memcpy(ulast, u, sizeof(double) * (size_t)U.size());
    std::memcpy(vlast, v, sizeof(double) * (size_t)Vv.size());
    std::memcpy(wlast, w, sizeof(double) * (size_t)W.size());
  }
}

void ora_sample_velocity(int64_t n, const double* pts, int nx, int ny, int nz, double h,
                         const double* u, const double* v, const double* w, double* out) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; i++)
    st3(out, i, sample_velocity(ld3(pts, i), nx, ny, nz, h, u, v, w));
}

void ora_g2p(int64_t n, const double* pos, double* vel, int nx, int ny, int nz, double h,
             const double* u, const double* v, const double* w, const double* ulast,
             const double* vlast, const double* wlast, double alpha) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; i++) {
    V3 p = ld3(pos, i);
    V3 pic = sample_velocity(p, nx, ny, nz, h, u, v, w);
    if (alpha < 0.0) {  // PicAdvector3D::solveG2P (advect-solver.cc:7-17)
      st3(vel, i, pic);
      continue;
    }
    V3 vi = ld3(vel, i);
    V3 flip = (vi + pic) - sample_velocity(p, nx, ny, nz, h, ulast, vlast, wlast);
    st3(vel, i, alpha * flip + (1.0 - alpha) * pic);
  }
}

void ora_advect(int64_t n, double* pos, double* vel, int nx, int ny, int nz, double h,
                const double* u, const double* v, const double* w, const double* collider,
                double dt) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; i++) {
    V3 p = ld3(pos, i), k1 = ld3(vel, i);
    V3 p1 = p + (0.5 * dt) * k1;
    V3 k2 = sample_velocity(p1, nx, ny, nz, h, u, v, w);
    V3 p2 = p + (0.75 * dt) * k2;
    V3 k3 = sample_velocity(p2, nx, ny, nz, h, u, v, w);
    p = p + (2.0 / 9.0 * dt) * k1 + (1.0 / 3.0 * dt) * k2 + (4.0 / 9.0 * dt) * k3;
    V3 vv = k1;
    handle_collision(collider, nx, ny, nz, h, p, vv);
    st3(pos, i, p);
    st3(vel, i, vv);
  }
}

double ora_sdf_eval(const double* sdf, int nx, int ny, int nz, double h, const double* p) {
  return sdf_eval(sdf, nx, ny, nz, h, V3{p[0], p[1], p[2]});
}
void ora_sdf_grad(const double* sdf, int nx, int ny, int nz, double h, const double* p,
                  double* g) {
  V3 r = sdf_grad(sdf, nx, ny, nz, h, V3{p[0], p[1], p[2]});
  g[0] = r.x;
  g[1] = r.y;
  g[2] = r.z;
}

void ora_reconstruct(int64_t n, const double* pos, int nx, int ny, int nz, double h,
                     double radius, double* sdf, uint8_t* valid) {
  // ParticleNeighbourSearcher::update (ns-util.h:46-79): bucket by cell, sorted.
  // Bucket key: linear cell index (the reference's Morton key orders buckets
  // differently but gives the same bucket membership); within a bucket the
  // order is pinned to ascending particle id (stable sort).
  int64_t ncell = (int64_t)nx * ny * nz;
  std::vector<int64_t> key((size_t)n);
  for (int64_t i = 0; i < n; i++) {
    V3 p = ld3(pos, i);
    int ix = (int)std::floor(p.x / h);
    if (ix < 0) ix = 0;
    if (ix >= nx) ix = nx - 1;
    int iy = (int)std::floor(p.y / h);
    if (iy < 0) iy = 0;
    if (iy >= ny) iy = ny - 1;
    int iz = (int)std::floor(p.z / h);
    if (iz < 0) iz = 0;
    if (iz >= nz) iz = nz - 1;
    key[i] = iz + (int64_t)iy * nz + (int64_t)ix * ny * nz;
  }
  std::vector<int64_t> order((size_t)n);
  if (g_bucket_order == 1) {
    // ParticleNeighbourSearcher::update (ns-util.h:36-79): int indices sorted by
    // std::sort on the Morton key of the (clamped) cell.  The permutation inside
    // a bucket, and so the particle that forNeighbours skips, is the one this
    // unstable sort leaves; the buckets themselves are the same either way.
    auto morton10 = [](int x) {
      x = (x | (x << 16)) & 0x030000FF;
      x = (x | (x << 8)) & 0x0300F00F;
      x = (x | (x << 4)) & 0x030C30C3;
      x = (x | (x << 2)) & 0x09249249;
      return x;
    };
    std::vector<int> mkey((size_t)n), idx((size_t)n);
    for (int64_t i = 0; i < n; i++) {
      const int64_t c = key[i];
      const int iz = (int)(c % nz), iy = (int)((c / nz) % ny), ix = (int)(c / ((int64_t)ny * nz));
      mkey[i] = morton10(ix) | (morton10(iy) << 1) | (morton10(iz) << 2);
      idx[i] = (int)i;
    }
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return mkey[a] < mkey[b]; });
    for (int64_t i = 0; i < n; i++) order[i] = idx[i];
  } else {
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  }
  std::vector<int64_t> beg((size_t)ncell, -1), end((size_t)ncell, -1);
  for (int64_t i = 0; i < n; i++) {
    int64_t c = key[order[i]];
    if (i == 0 || key[order[i - 1]] != c) beg[c] = i;
    if (i == n - 1 || key[order[i + 1]] != c) end[c] = i;  // inclusive end
  }
  double r2 = 2 * radius;
  std::fill(sdf, sdf + ncell, 1e9);  // sdf.h:215-216
  std::memset(valid, 0, (size_t)ncell);
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        V3 p{((double)i + 0.5) * h + 0.0, ((double)j + 0.5) * h + 0.0,
             ((double)k + 0.5) * h + 0.0};
        int64_t cid = k + (int64_t)j * nz + (int64_t)i * ny * nz;
        // forNeighbours (ns-util.h:80-109)
        int x_min = std::max(0, (int)std::floor((p.x - r2) / h));
        int x_max = std::min(nx - 1, (int)std::ceil((p.x + r2) / h));
        int y_min = std::max(0, (int)std::floor((p.y - r2) / h));
        int y_max = std::min(ny - 1, (int)std::ceil((p.y + r2) / h));
        int z_min = std::max(0, (int)std::floor((p.z - r2) / h));
        int z_max = std::min(nz - 1, (int)std::ceil((p.z + r2) / h));
        for (int a = x_min; a <= x_max; a++)
          for (int b = y_min; b <= y_max; b++)
            for (int c = z_min; c <= z_max; c++) {
              int64_t cell = c + (int64_t)b * nz + (int64_t)a * ny * nz;
              for (int64_t l = beg[cell]; l < end[cell]; l++) {  // end exclusive: skips last
                V3 q = ld3(pos, order[l]);
                V3 d = q - p;
                double dis = std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
                if (dis <= r2) {
                  sdf[cid] = std::min(sdf[cid], dis - radius);
                  valid[cid] = 1;
                }
              }
            }
      }
}

double ora_fraction_inside(double lu, double ru, double rd, double ld) {
  // util.cc:333-378 (the corner cycle rotates (lu,ru,rd,ld) -> (ld,lu,ru,rd)).
  auto cycle = [](double& a0, double& a1, double& a2, double& a3) {
    double t = a0;
    a0 = a3;
    a3 = a2;
    a2 = a1;
    a1 = t;
  };
  int n_negs = (lu <= 0.0) + (ru <= 0.0) + (rd <= 0.0) + (ld <= 0.0);
  if (n_negs == 0) return 0.0;
  if (n_negs == 4) return 1.0;
  while (lu > 0.0) cycle(lu, ru, rd, ld);
  if (n_negs == 1) {
    double fracu = ru / (ru - lu);
    double fracl = ld / (ld - lu);
    return fracu * fracl * 0.5;
  }
  if (n_negs == 2) {
    if (ru <= 0.0) {
      double fracl = ld / (ld - lu);
      double fracr = rd / (rd - ru);
      return 0.5 * (fracl + fracr);
    }
    if (ld <= 0.0) {
      double fracu = ru / (ru - lu);
      double fracd = rd / (rd - ld);
      return 0.5 * (fracu + fracd);
    }
    if (rd <= 0.0) {
      double fracu = ru / (ru - lu);
      double fracd = ld / (ld - rd);
      double fracl = ld / (ld - lu);
      double fracr = ru / (ru - rd);
      if (lu + ru + rd + ld <= 0.0)
        return 1.0 - 0.5 * ((1.0 - fracu) * (1.0 - fracl) + (1.0 - fracd) * (1.0 - fracr));
      return 0.5 * (fracu * fracl + fracd * fracr);
    }
    return 0.0;  // unreachable (reference prints "numerical error" and falls through)
  }
  // n_negs == 3
  while (lu <= 0.0) cycle(lu, ru, rd, ld);
  double fracu = ru / (ru - lu);
  double fracl = ld / (ld - lu);
  return 1.0 - 0.5 * fracu * fracl;
}

void ora_build_system(int nx, int ny, int nz, double h, double dt, const double* u,
                      const double* v, const double* w, const double* fluid_sdf,
                      const double* collider, double* adiag, double* const* an, double* rhs,
                      uint8_t* active, double* uwt, double* vwt, double* wwt) {
  int64_t N = (int64_t)nx * ny * nz;
  A3<const double> F{fluid_sdf, nx, ny, nz};
  A3<const double> U{u, nx + 1, ny, nz}, Vv{v, nx, ny + 1, nz}, W{w, nx, ny, nz + 1};
  A3<double> UW{uwt, nx + 1, ny, nz}, VW{vwt, nx, ny + 1, nz}, WW{wwt, nx, ny, nz + 1};
  A3<double> AD{adiag, nx, ny, nz}, R{rhs, nx, ny, nz};
  A3<double> AN[6];
  for (int d = 0; d < 6; d++) {
    AN[d] = A3<double>{an[d], nx, ny, nz};
    std::fill(an[d], an[d] + N, 0.0);
  }
  std::fill(adiag, adiag + N, 0.0);
  std::fill(rhs, rhs + N, 0.0);
  std::fill(uwt, uwt + UW.size(), 0.0);
  std::fill(vwt, vwt + VW.size(), 0.0);
  std::fill(wwt, wwt + WW.size(), 0.0);
  std::memset(active, 0, (size_t)N);
  A3<uint8_t> ACT{active, nx, ny, nz};
  auto ceval = [&](V3 p) { return sdf_eval(collider, nx, ny, nz, h, p); };
  FaceGeom gu = ugeom(nx, ny, nz, h), gv = vgeom(nx, ny, nz, h), gw = wgeom(nx, ny, nz, h);
  // u face weights (project-solver.cc:77-93)
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx + 1; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (i == 0 || i == nx) {
          UW(i, j, k) = 0.0;
          continue;
        }
        if (F(i - 1, j, k) > 0.0 && F(i, j, k) > 0.0) continue;
        V3 p = gu.coord(i, j, k);
        double bu = ceval(p + (0.5 * h) * V3{0.0, 1, -1});
        double bd = ceval(p + (0.5 * h) * V3{0.0, -1, -1});
        double fd = ceval(p + (0.5 * h) * V3{0.0, -1, 1});
        double fu = ceval(p + (0.5 * h) * V3{0.0, 1, 1});
        UW(i, j, k) = 1.0 - ora_fraction_inside(bu, bd, fd, fu);
      }
  // v face weights (:94-110)
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny + 1; j++)
      for (int k = 0; k < nz; k++) {
        if (j == 0 || j == ny) {
          VW(i, j, k) = 0.0;
          continue;
        }
        if (F(i, j - 1, k) > 0.0 && F(i, j, k) > 0.0) continue;
        V3 p = gv.coord(i, j, k);
        double lb = ceval(p + (0.5 * h) * V3{-1, 0.0, -1});
        double rb = ceval(p + (0.5 * h) * V3{1, 0.0, -1});
        double rf = ceval(p + (0.5 * h) * V3{1, 0.0, 1});
        double lf = ceval(p + (0.5 * h) * V3{-1, 0.0, 1});
        VW(i, j, k) = 1.0 - ora_fraction_inside(lb, rb, rf, lf);
      }
  // w face weights (:111-127)
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz + 1; k++) {
        if (k == 0 || k == nz) {
          WW(i, j, k) = 0.0;
          continue;
        }
        if (F(i, j, k - 1) > 0.0 && F(i, j, k) > 0.0) continue;
        V3 p = gw.coord(i, j, k);
        double ld = ceval(p + (0.5 * h) * V3{-1, -1, 0.0});
        double lu = ceval(p + (0.5 * h) * V3{-1, 1, 0.0});
        double ru = ceval(p + (0.5 * h) * V3{1, 1, 0.0});
        double rd = ceval(p + (0.5 * h) * V3{1, -1, 0.0});
        WW(i, j, k) = 1.0 - ora_fraction_inside(ld, lu, ru, rd);
      }
  // matrix + rhs (:129-226)
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (UW(i, j, k) == 0.0 && UW(i + 1, j, k) == 0.0 && VW(i, j, k) == 0.0 &&
            VW(i, j + 1, k) == 0.0 && WW(i, j, k) == 0.0 && WW(i, j, k + 1) == 0.0)
          continue;
        if (F(i, j, k) > 0.0) continue;
        ACT(i, j, k) = 1;
        double sd = F(i, j, k);
        double factor = dt / h;
        if (i > 0) {  // left
          if (F(i - 1, j, k) > 0.0) {
            double theta = std::min(F(i - 1, j, k) / (F(i - 1, j, k) - sd), 0.99);
            AD(i, j, k) += UW(i, j, k) * factor / (1.0 - theta);
          } else {
            AD(i, j, k) += UW(i, j, k) * factor;
            AN[Left](i, j, k) -= UW(i, j, k) * factor;
          }
          R(i, j, k) += UW(i, j, k) * U(i, j, k);
        }
        if (i < nx - 1) {  // right
          if (F(i + 1, j, k) > 0.0) {
            double theta = std::max(sd / (sd - F(i + 1, j, k)), 0.01);
            AD(i, j, k) += UW(i + 1, j, k) * factor / theta;
          } else {
            AD(i, j, k) += UW(i + 1, j, k) * factor;
            AN[Right](i, j, k) -= UW(i + 1, j, k) * factor;
          }
          R(i, j, k) -= UW(i + 1, j, k) * U(i + 1, j, k);
        }
        if (j > 0) {  // down
          if (F(i, j - 1, k) > 0.0) {
            double theta = std::min(F(i, j - 1, k) / (F(i, j - 1, k) - sd), 0.99);
            AD(i, j, k) += VW(i, j, k) * factor / (1.0 - theta);
          } else {
            AD(i, j, k) += VW(i, j, k) * factor;
            AN[Down](i, j, k) -= VW(i, j, k) * factor;
          }
          R(i, j, k) += VW(i, j, k) * Vv(i, j, k);
        }
        // up: the reference bounds j by the grid WIDTH (:186); identical on the
        // cubic grids used here, and clipped to the height otherwise.
        if (j < nx - 1 && j < ny - 1) {
          if (F(i, j + 1, k) > 0.0) {
            double theta = std::max(sd / (sd - F(i, j + 1, k)), 0.01);
            AD(i, j, k) += VW(i, j + 1, k) * factor / theta;
          } else {
            AD(i, j, k) += VW(i, j + 1, k) * factor;
            AN[Up](i, j, k) -= VW(i, j + 1, k) * factor;
          }
          R(i, j, k) -= VW(i, j + 1, k) * Vv(i, j + 1, k);
        }
        if (k > 0) {  // back
          if (F(i, j, k - 1) > 0.0) {
            double theta = std::min(F(i, j, k - 1) / (F(i, j, k - 1) - sd), 0.99);
            AD(i, j, k) += WW(i, j, k) * factor / (1.0 - theta);
          } else {
            AD(i, j, k) += WW(i, j, k) * factor;
            AN[Back](i, j, k) -= WW(i, j, k) * factor;
          }
          R(i, j, k) += WW(i, j, k) * W(i, j, k);
        }
        if (k < nz - 1) {  // front
          if (F(i, j, k + 1) > 0.0) {
            double theta = std::max(sd / (sd - F(i, j, k + 1)), 0.01);
            AD(i, j, k) += WW(i, j, k + 1) * factor / theta;
          } else {
            AD(i, j, k) += WW(i, j, k + 1) * factor;
            AN[Front](i, j, k) -= WW(i, j, k + 1) * factor;
          }
          R(i, j, k) -= WW(i, j, k + 1) * W(i, j, k + 1);
        }
      }
}

void ora_apply_matrix(int nx, int ny, int nz, const double* adiag, const double* const* an,
                      const double* x, const uint8_t* active, double* b) {
  A3<const double> AD{adiag, nx, ny, nz}, X{x, nx, ny, nz};
  A3<const uint8_t> ACT{active, nx, ny, nz};
  A3<double> B{b, nx, ny, nz};
  A3<const double> AN[6];
  for (int d = 0; d < 6; d++) AN[d] = A3<const double>{an[d], nx, ny, nz};
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (!ACT(i, j, k)) continue;
        double t = AD(i, j, k) * X(i, j, k);
        if (i > 0 && ACT(i - 1, j, k)) t += AN[Left](i, j, k) * X(i - 1, j, k);
        if (j > 0 && ACT(i, j - 1, k)) t += AN[Down](i, j, k) * X(i, j - 1, k);
        if (k > 0 && ACT(i, j, k - 1)) t += AN[Back](i, j, k) * X(i, j, k - 1);
        if (i < nx - 1 && ACT(i + 1, j, k)) t += AN[Right](i, j, k) * X(i + 1, j, k);
        if (j < ny - 1 && ACT(i, j + 1, k)) t += AN[Up](i, j, k) * X(i, j + 1, k);
        if (k < nz - 1 && ACT(i, j, k + 1)) t += AN[Front](i, j, k) * X(i, j, k + 1);
        B(i, j, k) = t;
      }
}

void ora_mic_precond(int nx, int ny, int nz, const double* adiag, const double* const* an,
                     const double* r, const uint8_t* active, double* z, double tau,
                     double sigma, double* E_out, double* q_out) {
  int64_t N = (int64_t)nx * ny * nz;
  std::vector<double> Ebuf, qbuf;
  double* Ed = E_out;
  double* qd = q_out;
  if (!Ed) {
    Ebuf.assign((size_t)N, 0.0);
    Ed = Ebuf.data();
  }
  if (!qd) {
    qbuf.assign((size_t)N, 0.0);
    qd = qbuf.data();
  }
  A3<const double> AD{adiag, nx, ny, nz}, R{r, nx, ny, nz};
  A3<const uint8_t> ACT{active, nx, ny, nz};
  A3<const double> L{an[Left], nx, ny, nz}, D{an[Down], nx, ny, nz}, Bk{an[Back], nx, ny, nz};
  A3<double> E{Ed, nx, ny, nz}, Q{qd, nx, ny, nz}, Z{z, nx, ny, nz};
  auto sqr = [](double x) { return x * x; };
  std::fill(Ed, Ed + N, 0.0);
  // pivot (project-solver.cc:237-274), serial lexicographic
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (!ACT(i, j, k)) continue;
        double e = AD(i, j, k);
        if (e == 0.0) continue;
        if (i > 0 && ACT(i - 1, j, k) && AD(i - 1, j, k) != 0.0) {
          e -= sqr(L(i, j, k) * E(i - 1, j, k));
          if (j < ny - 1 && ACT(i - 1, j + 1, k))
            e -= tau * L(i, j, k) * L(i - 1, j + 1, k) / sqr(E(i - 1, j, k));
          if (k < nz - 1 && ACT(i - 1, j, k + 1))
            e -= tau * L(i, j, k) * L(i - 1, j, k + 1) / sqr(E(i - 1, j, k));
        }
        if (j > 0 && ACT(i, j - 1, k) && AD(i, j - 1, k) != 0.0) {
          e -= sqr(D(i, j, k) * E(i, j - 1, k));
          if (i < nx - 1 && ACT(i + 1, j - 1, k))
            e -= tau * D(i, j, k) * D(i + 1, j - 1, k) / sqr(E(i, j - 1, k));
          if (k < nz - 1 && ACT(i, j - 1, k + 1))
            e -= tau * D(i, j, k) * D(i, j - 1, k + 1) / sqr(E(i, j - 1, k));
        }
        if (k > 0 && ACT(i, j, k - 1) && AD(i, j, k - 1) != 0.0) {
          e -= sqr(Bk(i, j, k) * E(i, j, k - 1));
          if (i < nx - 1 && ACT(i + 1, j, k - 1))
            e -= tau * Bk(i, j, k) * Bk(i + 1, j, k - 1) / sqr(E(i, j, k - 1));
          if (j < ny - 1 && ACT(i, j + 1, k - 1))
            e -= tau * Bk(i, j, k) * Bk(i, j + 1, k - 1) / sqr(E(i, j, k - 1));
        }
        if (e < sigma * AD(i, j, k)) e = AD(i, j, k);
        E(i, j, k) = 1.0 / std::sqrt(e);
      }
  // forward: L q = r (:276-288)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (!ACT(i, j, k)) continue;
        double t = R(i, j, k);
        if (i > 0 && ACT(i - 1, j, k)) t -= L(i, j, k) * E(i - 1, j, k) * Q(i - 1, j, k);
        if (j > 0 && ACT(i, j - 1, k)) t -= D(i, j, k) * E(i, j - 1, k) * Q(i, j - 1, k);
        if (k > 0 && ACT(i, j, k - 1)) t -= Bk(i, j, k) * E(i, j, k - 1) * Q(i, j, k - 1);
        Q(i, j, k) = t * E(i, j, k);
      }
  // backward: L^T z = q (:293-305), reversed lexicographic
  for (int i = nx - 1; i >= 0; i--)
    for (int j = ny - 1; j >= 0; j--)
      for (int k = nz - 1; k >= 0; k--) {
        if (!ACT(i, j, k)) continue;
        double t = Q(i, j, k);
        if (i < nx - 1 && ACT(i + 1, j, k)) t -= L(i + 1, j, k) * E(i, j, k) * Z(i + 1, j, k);
        if (j < ny - 1 && ACT(i, j + 1, k)) t -= D(i, j + 1, k) * E(i, j, k) * Z(i, j + 1, k);
        if (k < nz - 1 && ACT(i, j, k + 1)) t -= Bk(i, j, k + 1) * E(i, j, k) * Z(i, j, k + 1);
        Z(i, j, k) = t * E(i, j, k);
      }
}

double ora_dot(int64_t n, const double* a, const double* b, const uint8_t* active) {
  double s = 0.0;  // serial, lexicographic (util.cc:380-392)
  for (int64_t i = 0; i < n; i++)
    if (active[i]) s += a[i] * b[i];
  return s;
}
void ora_saxpy(int64_t n, double* a, const double* b, double x, const uint8_t* active) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; i++)
    if (active[i]) a[i] += x * b[i];
}
void ora_scale_and_add(int64_t n, double* c, const double* a, double x,
                       const uint8_t* active) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; i++)
    if (active[i]) c[i] = a[i] + x * c[i];
}
double ora_linf(int64_t n, const double* a, const uint8_t* active) {
  double m = 0.0;
  for (int64_t i = 0; i < n; i++)
    if (active[i]) m = std::max(m, std::fabs(a[i]));
  return m;
}

static double norm2_masked(int64_t n, const double* a, const uint8_t* active) {
  return std::sqrt(ora_dot(n, a, a, active));
}

double ora_pcg_solve(int nx, int ny, int nz, const double* adiag, const double* const* an,
                     const double* rhs, const uint8_t* active, double* pg, double tol,
                     int max_iter, int criterion, double tau, double sigma, int* iters) {
  int64_t N = (int64_t)nx * ny * nz;
  std::vector<double> r(rhs, rhs + N), z((size_t)N, 0.0), s((size_t)N, 0.0);
  std::vector<double> E((size_t)N), q((size_t)N, 0.0);
  std::fill(pg, pg + N, 0.0);
  double bnorm = criterion == ORA_CRIT_REL_L2 ? norm2_masked(N, rhs, active) : 1.0;
  auto measure = [&](const double* rr) {
    if (criterion == ORA_CRIT_REL_L2)
      return bnorm > 0.0 ? norm2_masked(N, rr, active) / bnorm : 0.0;
    return ora_linf(N, rr, active);
  };
  double residual = measure(r.data());
  if (iters) *iters = 0;
  if (residual < tol) return residual;  // "naturally converged" (:317-319)
  ora_mic_precond(nx, ny, nz, adiag, an, rhs, active, z.data(), tau, sigma, E.data(),
                  q.data());
  s = z;
  double sig = ora_dot(N, z.data(), r.data(), active);
  int iter = 1;
  for (; iter < max_iter; iter++) {
    ora_apply_matrix(nx, ny, nz, adiag, an, s.data(), active, z.data());
    double sdotz = ora_dot(N, s.data(), z.data(), active);
    double alpha = sig / sdotz;
    ora_saxpy(N, pg, s.data(), alpha, active);
    ora_saxpy(N, r.data(), z.data(), -alpha, active);
    residual = measure(r.data());
    if (residual < tol) break;
    ora_mic_precond(nx, ny, nz, adiag, an, r.data(), active, z.data(), tau, sigma, E.data(),
                    q.data());
    double sig_new = ora_dot(N, z.data(), r.data(), active);
    double beta = sig_new / sig;
    ora_scale_and_add(N, s.data(), z.data(), beta, active);
    sig = sig_new;
  }
  if (iters) *iters = iter;
  return residual;
}

void ora_project(int nx, int ny, int nz, double h, double dt, double* u, double* v, double* w,
                 const double* pg, const double* fluid_sdf, const double* uwt,
                 const double* vwt, const double* wwt) {
  A3<double> U{u, nx + 1, ny, nz}, Vv{v, nx, ny + 1, nz}, W{w, nx, ny, nz + 1};
  A3<const double> UW{uwt, nx + 1, ny, nz}, VW{vwt, nx, ny + 1, nz}, WW{wwt, nx, ny, nz + 1};
  A3<const double> P{pg, nx, ny, nz}, F{fluid_sdf, nx, ny, nz};
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx + 1; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        if (UW(i, j, k) <= 0.0) continue;
        if (i == 0 || i == nx) {
          U(i, j, k) = 0.0;
          continue;
        }
        double sl = F(i - 1, j, k), sr = F(i, j, k);
        if (sl >= 0.0 && sr >= 0.0) continue;
        if (sl < 0.0 && sr < 0.0) {
          U(i, j, k) -= (P(i, j, k) - P(i - 1, j, k)) * dt / h;
          continue;
        }
        if (sl < 0.0) {
          double theta = std::max(sl / (sl - sr), 0.01);
          U(i, j, k) += P(i - 1, j, k) * dt / h / theta;
        } else {
          double theta = std::min(sl / (sl - sr), 0.99);
          U(i, j, k) -= P(i, j, k) * dt / h / (1.0 - theta);
        }
      }
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny + 1; j++)
      for (int k = 0; k < nz; k++) {
        if (VW(i, j, k) <= 0.0) continue;
        if (j == 0 || j == ny) {
          Vv(i, j, k) = 0.0;
          continue;
        }
        double sd = F(i, j - 1, k), su = F(i, j, k);
        if (sd >= 0.0 && su >= 0.0) continue;
        if (sd < 0.0 && su < 0.0) {
          Vv(i, j, k) -= (P(i, j, k) - P(i, j - 1, k)) * dt / h;
          continue;
        }
        if (sd < 0.0) {
          double theta = std::max(sd / (sd - su), 0.01);
          Vv(i, j, k) += P(i, j - 1, k) * dt / h / theta;
        } else {
          double theta = std::min(sd / (sd - su), 0.99);
          Vv(i, j, k) -= P(i, j, k) * dt / h / (1.0 - theta);
        }
      }
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz + 1; k++) {
        if (WW(i, j, k) <= 0.0) continue;
        if (k == 0 || k == nz) {
          W(i, j, k) = 0.0;
          continue;
        }
        double sb = F(i, j, k - 1), sf = F(i, j, k);
        if (sb >= 0.0 && sf >= 0.0) continue;
        if (sb < 0.0 && sf < 0.0) {
          W(i, j, k) -= (P(i, j, k) - P(i, j, k - 1)) * dt / h;
          continue;
        }
        if (sb < 0.0) {
          double theta = std::max(sb / (sb - sf), 0.01);
          W(i, j, k) += P(i, j, k - 1) * dt / h / theta;
        } else {
          double theta = std::min(sb / (sb - sf), 0.99);
          W(i, j, k) -= P(i, j, k) * dt / h / (1.0 - theta);
        }
      }
}

// ------------------------------------------------------------------------------------
// Whole simulator: fluid::cpu::FluidSimulator (FluidSim/include/FluidSim/cpu/fluid-simulator.h,
// FluidSim/src/cpu/fluid-simulator.cc).  Buffers that the reference swaps through
// unique_ptr are modelled as index pairs so that the stale-buffer behaviour of
// extrapolateFluidSdf / extrapolate (which do not copy valid cells into the
// destination buffer) is reproduced exactly.
struct ora_sim {
  ora_sim_config c;
  int64_t n = 0;
  std::vector<double> pos, vel;
  std::vector<double> g[3][2];       // [u|v|w][primary-or-buffer]
  std::vector<uint8_t> gv[3][2];     // valid / validBuf
  int gcur[3] = {0, 0, 0};
  std::vector<double> gw[3];         // uw, vw, ww
  std::vector<double> last[3];       // u_last, v_last, w_last
  std::vector<double> pg;
  std::vector<double> sdf[2];        // fluidSurface / fluidSurfaceBuf
  std::vector<uint8_t> sdfv[2];      // sdfValid / sdfValidBuf
  int scur = 0, svcur = 0;
  std::vector<double> collider;
  std::vector<double> adiag, an[6], rhs, wt[3];
  std::vector<uint8_t> active;
  int last_iters = 0;
  double last_residual = 0.0;
  int64_t fsize[3];
  // fluid-SDF tape (checker of the differentiable step, not part of the
  // reference): 1 records the fluid SDF each substep uses, 2 uses the recorded
  // ones in their order instead of reconstructing
  int sdf_tape = 0;
  size_t sdf_tape_pos = 0;
  std::vector<std::vector<double>> sdf_tape_data;
};

// smoothFluidSurface (fluid-simulator.cc:39-74): min-preserving neighbour
// average, ping-ponging fluidSurface and fluidSurfaceBuf.
static void sim_smooth(ora_sim* s, int iters) {
  const int nx = s->c.nx, ny = s->c.ny, nz = s->c.nz;
  for (int it = 0; it < iters; it++) {
    const double* src = s->sdf[s->scur].data();
    double* dst = s->sdf[1 - s->scur].data();
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
          int64_t id = k + (int64_t)j * nz + (int64_t)i * ny * nz;
          double sum = 0;
          int cnt = 0;
          if (i > 0) { sum += src[id - (int64_t)ny * nz]; cnt++; }
          if (i < nx - 1) { sum += src[id + (int64_t)ny * nz]; cnt++; }
          if (j > 0) { sum += src[id - nz]; cnt++; }
          if (j < ny - 1) { sum += src[id + nz]; cnt++; }
          if (k > 0) { sum += src[id - 1]; cnt++; }
          if (k < nz - 1) { sum += src[id + 1]; cnt++; }
          dst[id] = sum / cnt;
          if (src[id] < dst[id]) dst[id] = src[id];
        }
    s->scur = 1 - s->scur;
  }
}

static void sim_alloc(ora_sim* s) {
  int nx = s->c.nx, ny = s->c.ny, nz = s->c.nz;
  int64_t N = (int64_t)nx * ny * nz;
  s->fsize[0] = (int64_t)(nx + 1) * ny * nz;
  s->fsize[1] = (int64_t)nx * (ny + 1) * nz;
  s->fsize[2] = (int64_t)nx * ny * (nz + 1);
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) {
      s->g[a][b].assign((size_t)s->fsize[a], 0.0);
      s->gv[a][b].assign((size_t)s->fsize[a], 0);
    }
    s->gw[a].assign((size_t)s->fsize[a], 0.0);
    s->last[a].assign((size_t)s->fsize[a], 0.0);
    s->wt[a].assign((size_t)s->fsize[a], 0.0);
  }
  s->pg.assign((size_t)N, 0.0);
  for (int b = 0; b < 2; b++) {
    s->sdf[b].assign((size_t)N, 0.0);
    s->sdfv[b].assign((size_t)N, 0);
  }
  s->collider.assign((size_t)N, 1e9);  // manifold2SDF of an empty mesh (util.cc:211)
  s->adiag.assign((size_t)N, 0.0);
  for (int d = 0; d < 6; d++) s->an[d].assign((size_t)N, 0.0);
  s->rhs.assign((size_t)N, 0.0);
  s->active.assign((size_t)N, 0);
}

ora_sim* ora_sim_create(const ora_sim_config* cfg) {
  ora_sim* s = new ora_sim();
  s->c = *cfg;
  sim_alloc(s);
  return s;
}
void ora_sim_sdf_tape(ora_sim* s, int mode) {
  s->sdf_tape = mode;
  s->sdf_tape_pos = 0;
  if (mode == 1) s->sdf_tape_data.clear();
}
int ora_sim_sdf_tape_get(ora_sim* s, int64_t k, double* sdf) {
  if (k < 0 || k >= (int64_t)s->sdf_tape_data.size()) return -1;
  std::copy(s->sdf_tape_data[k].begin(), s->sdf_tape_data[k].end(), sdf);
  return 0;
}
int ora_sim_sdf_tape_put(ora_sim* s, const double* sdf) {
  s->sdf_tape_data.emplace_back(sdf, sdf + (int64_t)s->c.nx * s->c.ny * s->c.nz);
  return 0;
}

void ora_sim_destroy(ora_sim* s) { delete s; }
void ora_sim_set_particles(ora_sim* s, int64_t n, const double* pos, const double* vel) {
  s->n = n;
  s->pos.assign(pos, pos + 3 * n);
  if (vel)
    s->vel.assign(vel, vel + 3 * n);
  else
    s->vel.assign((size_t)(3 * n), 0.0);
}
void ora_sim_set_collider(ora_sim* s, const double* sdf) {
  int64_t N = (int64_t)s->c.nx * s->c.ny * s->c.nz;
  if (sdf)
    s->collider.assign(sdf, sdf + N);
  else
    s->collider.assign((size_t)N, 1e9);
}

double ora_sim_cfl(const ora_sim* s) {  // fluid-simulator.cc:184-203
  double h = s->c.h;
  double cfl = h / 1e-6;
  for (int a = 0; a < 3; a++) {
    const std::vector<double>& g = s->g[a][s->gcur[a]];
    for (double x : g)
      if (x != 0.0) cfl = std::min(cfl, h / std::fabs(x));
  }
  return s->c.cfl_factor * std::max(1e-3, cfl);
}

void ora_sim_substep(ora_sim* s, double dt) {  // fluid-simulator.cc:140-182
  const ora_sim_config& c = s->c;
  int nx = c.nx, ny = c.ny, nz = c.nz;
  double h = c.h;
  int64_t N = (int64_t)nx * ny * nz;
  // clear() (:20-37): valid + validBuf, grids + bufs, weights, pg.
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) {
      std::fill(s->g[a][b].begin(), s->g[a][b].end(), 0.0);
      std::fill(s->gv[a][b].begin(), s->gv[a][b].end(), 0);
    }
    std::fill(s->gw[a].begin(), s->gw[a].end(), 0.0);
  }
  std::fill(s->pg.begin(), s->pg.end(), 0.0);
  double* U = s->g[0][s->gcur[0]].data();
  double* Vv = s->g[1][s->gcur[1]].data();
  double* W = s->g[2][s->gcur[2]].data();
  // advect on the just-cleared grids (:143)
  ora_advect(s->n, s->pos.data(), s->vel.data(), nx, ny, nz, h, U, Vv, W, s->collider.data(),
             dt);
  const bool replay = s->sdf_tape == 2 && s->sdf_tape_pos < s->sdf_tape_data.size();
  if (replay) {
    std::copy(s->sdf_tape_data[s->sdf_tape_pos].begin(), s->sdf_tape_data[s->sdf_tape_pos].end(),
              s->sdf[s->scur].begin());
    s->sdf_tape_pos++;
  } else {
  // reconstruct into the current primary SDF (:146-148)
  ora_reconstruct(s->n, s->pos.data(), nx, ny, nz, h, c.recon_factor * h,
                  s->sdf[s->scur].data(), s->sdfv[s->svcur].data());
  // extrapolateFluidSdf (cpu/fluid-simulator.h:123-166): valid cells are NOT
  // copied into the destination buffer.
  for (int it = 0; it < c.sdf_extrap_iters; it++) {
    const double* src = s->sdf[s->scur].data();
    double* dst = s->sdf[1 - s->scur].data();
    const uint8_t* vs = s->sdfv[s->svcur].data();
    uint8_t* vd = s->sdfv[1 - s->svcur].data();
    std::memset(vd, 0, (size_t)N);
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
          int64_t id = k + (int64_t)j * nz + (int64_t)i * ny * nz;
          if (vs[id]) {
            vd[id] = 1;
            continue;
          }
          double sum = 0.0;
          int cnt = 0;
          if (i > 0 && vs[id - (int64_t)ny * nz]) { sum += src[id - (int64_t)ny * nz]; cnt++; }
          if (i < nx - 1 && vs[id + (int64_t)ny * nz]) { sum += src[id + (int64_t)ny * nz]; cnt++; }
          if (j > 0 && vs[id - nz]) { sum += src[id - nz]; cnt++; }
          if (j < ny - 1 && vs[id + nz]) { sum += src[id + nz]; cnt++; }
          if (k > 0 && vs[id - 1]) { sum += src[id - 1]; cnt++; }
          if (k < nz - 1 && vs[id + 1]) { sum += src[id + 1]; cnt++; }
          if (cnt > 0) {
            dst[id] = sum / cnt;
            vd[id] = 1;
          } else
            vd[id] = 0;
        }
    s->scur = 1 - s->scur;
    s->svcur = 1 - s->svcur;
  }
  sim_smooth(s, c.smooth_iters);
  if (s->sdf_tape == 1) s->sdf_tape_data.push_back(s->sdf[s->scur]);
  }
  const double* fluid = s->sdf[s->scur].data();
  // P2G (:155-156)
  U = s->g[0][s->gcur[0]].data();
  Vv = s->g[1][s->gcur[1]].data();
  W = s->g[2][s->gcur[2]].data();
  ora_p2g(s->n, s->pos.data(), s->vel.data(), nx, ny, nz, h, U, Vv, W, s->gw[0].data(),
          s->gw[1].data(), s->gw[2].data(), s->gv[0][s->gcur[0]].data(),
          s->gv[1][s->gcur[1]].data(), s->gv[2][s->gcur[2]].data(),
          c.flip ? s->last[0].data() : nullptr, c.flip ? s->last[1].data() : nullptr,
          c.flip ? s->last[2].data() : nullptr);
  // applyDirichletBoundary (:113-138)
  {
    A3<double> Ua{U, nx + 1, ny, nz}, Va{Vv, nx, ny + 1, nz}, Wa{W, nx, ny, nz + 1};
    A3<uint8_t> uv{s->gv[0][s->gcur[0]].data(), nx + 1, ny, nz};
    A3<uint8_t> vv{s->gv[1][s->gcur[1]].data(), nx, ny + 1, nz};
    A3<uint8_t> wv{s->gv[2][s->gcur[2]].data(), nx, ny, nz + 1};
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        Ua(0, j, k) = 0.0;
        uv(0, j, k) = 1;
        Ua(nx, j, k) = 0.0;
        uv(nx, j, k) = 1;
      }
    for (int i = 0; i < nx; i++)
      for (int k = 0; k < nz; k++) {
        Va(i, 0, k) = 0.0;
        vv(i, 0, k) = 1;
        Va(i, ny, k) = 0.0;
        vv(i, ny, k) = 1;
      }
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++) {
        Wa(i, j, 0) = 0.0;
        wv(i, j, 0) = 1;
        Wa(i, j, nz) = 0.0;
        wv(i, j, nz) = 1;
      }
  }
  // extrapolate u, v, w (cpu/fluid-simulator.h:204-253): valid cells are NOT
  // copied into the destination buffer; cells without valid neighbours get 0.
  for (int a = 0; a < 3; a++) {
    int gw_ = nx + (a == 0), gh = ny + (a == 1), gd = nz + (a == 2);
    for (int it = 0; it < c.vel_extrap_iters; it++) {
      const double* src = s->g[a][s->gcur[a]].data();
      double* dst = s->g[a][1 - s->gcur[a]].data();
      const uint8_t* vs = s->gv[a][s->gcur[a]].data();
      uint8_t* vd = s->gv[a][1 - s->gcur[a]].data();
      std::memset(vd, 0, (size_t)s->fsize[a]);
#pragma omp parallel for num_threads(g_threads) schedule(static)
      for (int i = 0; i < gw_; i++)
        for (int j = 0; j < gh; j++)
          for (int k = 0; k < gd; k++) {
            int64_t id = k + (int64_t)j * gd + (int64_t)i * gh * gd;
            int64_t sx = (int64_t)gh * gd, sy = gd;
            if (vs[id]) {
              vd[id] = 1;
              continue;
            }
            double sum = 0.0;
            int cnt = 0;
            if (i > 0 && vs[id - sx]) { sum += src[id - sx]; cnt++; }
            if (i < gw_ - 1 && vs[id + sx]) { sum += src[id + sx]; cnt++; }
            if (j > 0 && vs[id - sy]) { sum += src[id - sy]; cnt++; }
            if (j < gh - 1 && vs[id + sy]) { sum += src[id + sy]; cnt++; }
            if (k > 0 && vs[id - 1]) { sum += src[id - 1]; cnt++; }
            if (k < gd - 1 && vs[id + 1]) { sum += src[id + 1]; cnt++; }
            if (cnt > 0) {
              dst[id] = sum / cnt;
              vd[id] = 1;
            } else {
              dst[id] = 0.0;
              vd[id] = 0;
            }
          }
      s->gcur[a] = 1 - s->gcur[a];
    }
  }
  U = s->g[0][s->gcur[0]].data();
  Vv = s->g[1][s->gcur[1]].data();
  W = s->g[2][s->gcur[2]].data();
  // applyForce (:13-18): valid v-faces with 0 < j < height-1.
  {
    A3<double> Va{Vv, nx, ny + 1, nz};
    A3<uint8_t> vv{s->gv[1][s->gcur[1]].data(), nx, ny + 1, nz};
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny + 1; j++)
        for (int k = 0; k < nz; k++)
          if (vv(i, j, k) && j > 0 && j < ny) Va(i, j, k) -= c.gravity * dt;
  }
  // buildSystem (:166)
  double* anp[6];
  for (int d = 0; d < 6; d++) anp[d] = s->an[d].data();
  ora_build_system(nx, ny, nz, h, dt, U, Vv, W, fluid, s->collider.data(), s->adiag.data(), anp,
                   s->rhs.data(), s->active.data(), s->wt[0].data(), s->wt[1].data(),
                   s->wt[2].data());
  // solvePressure (:169)
  s->last_residual = ora_pcg_solve(nx, ny, nz, s->adiag.data(), anp, s->rhs.data(),
                                   s->active.data(), s->pg.data(), c.pcg_tol, c.pcg_max_iter,
                                   c.pcg_criterion, c.mic_tau, c.mic_sigma, &s->last_iters);
  // project + applyCollider (:175-176)
  ora_project(nx, ny, nz, h, dt, U, Vv, W, s->pg.data(), fluid, s->wt[0].data(),
              s->wt[1].data(), s->wt[2].data());
  {
    A3<double> Ua{U, nx + 1, ny, nz}, Va{Vv, nx, ny + 1, nz}, Wa{W, nx, ny, nz + 1};
    const double* col = s->collider.data();
    FaceGeom gu = ugeom(nx, ny, nz, h), gv = vgeom(nx, ny, nz, h), gw = wgeom(nx, ny, nz, h);
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < nx + 1; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
          if (i == 0 || i == nx) {
            Ua(i, j, k) = 0.0;
            continue;
          }
          V3 p = gu.coord(i, j, k);
          if (sdf_eval(col, nx, ny, nz, h, p) < 0.0) {
            V3 nrm = normalize3(sdf_grad(col, nx, ny, nz, h, p));
            Ua(i, j, k) -= Ua(i, j, k) * nrm.x;
          }
        }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny + 1; j++)
        for (int k = 0; k < nz; k++) {
          if (j == 0 || j == ny) {
            Va(i, j, k) = 0.0;
            continue;
          }
          V3 p = gv.coord(i, j, k);
          if (sdf_eval(col, nx, ny, nz, h, p) < 0.0) {
            V3 nrm = normalize3(sdf_grad(col, nx, ny, nz, h, p));
            Va(i, j, k) -= Va(i, j, k) * nrm.y;
          }
        }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz + 1; k++) {
          if (k == 0 || k == nz) {
            Wa(i, j, k) = 0.0;
            continue;
          }
          V3 p = gw.coord(i, j, k);
          if (sdf_eval(col, nx, ny, nz, h, p) < 0.0) {
            V3 nrm = normalize3(sdf_grad(col, nx, ny, nz, h, p));
            Wa(i, j, k) -= Wa(i, j, k) * nrm.z;
          }
        }
  }
  // G2P (:179-180)
  ora_g2p(s->n, s->pos.data(), s->vel.data(), nx, ny, nz, h, U, Vv, W, s->last[0].data(),
          s->last[1].data(), s->last[2].data(), c.flip ? c.flip_alpha : -1.0);
}

int ora_sim_step(ora_sim* s, double frame_dt) {  // fluid-simulator.cc:205-220
  double t = 0;
  int cnt = 0;
  while (t < frame_dt) {
    double cfl = ora_sim_cfl(s);
    double dt = std::min(cfl, frame_dt - t);
    cnt++;
    ora_sim_substep(s, dt);
    t += dt;
  }
  return cnt;
}

void ora_sim_get_particles(const ora_sim* s, double* pos, double* vel) {
  if (pos) std::memcpy(pos, s->pos.data(), sizeof(double) * (size_t)(3 * s->n));
  if (vel) std::memcpy(vel, s->vel.data(), sizeof(double) * (size_t)(3 * s->n));
}
void ora_sim_get_pressure(const ora_sim* s, double* p) {
  std::memcpy(p, s->pg.data(), sizeof(double) * s->pg.size());
}
void ora_sim_get_faces(const ora_sim* s, double* u, double* v, double* w) {
  double* out[3] = {u, v, w};
  for (int a = 0; a < 3; a++)
    if (out[a])
      std::memcpy(out[a], s->g[a][s->gcur[a]].data(), sizeof(double) * (size_t)s->fsize[a]);
}
void ora_sim_get_fluid_sdf(const ora_sim* s, double* sdf) {
  std::memcpy(sdf, s->sdf[s->scur].data(), sizeof(double) * s->sdf[s->scur].size());
}
// FluidSimulator::reconstruct (cpu/fluid-simulator.h:115-119): the particles'
// surface into the current fluidSurface and sdfValid; the reference passes
// radius = 1.2 h / sqrt(2).
void ora_sim_reconstruct(ora_sim* s, double radius) {
  ora_reconstruct(s->n, s->pos.data(), s->c.nx, s->c.ny, s->c.nz, s->c.h, radius,
                  s->sdf[s->scur].data(), s->sdfv[s->svcur].data());
}
void ora_sim_smooth_fluid_surface(ora_sim* s, int iters) { sim_smooth(s, iters); }
void ora_sim_get_system(const ora_sim* s, double* adiag, double* const* an, double* rhs,
                        uint8_t* active) {
  size_t N = s->adiag.size();
  if (adiag) std::memcpy(adiag, s->adiag.data(), sizeof(double) * N);
  if (an)
    for (int d = 0; d < 6; d++)
      if (an[d]) std::memcpy(an[d], s->an[d].data(), sizeof(double) * N);
  if (rhs) std::memcpy(rhs, s->rhs.data(), sizeof(double) * N);
  if (active) std::memcpy(active, s->active.data(), N);
}
// manifold2SDF (FluidSim/src/cpu/util.cc:203-310): exact distances in a band of
// `exact_band` cells around each triangle's box, crossing counts of the +z rays
// through the cell centres, two rounds of eight fast sweeps propagating the
// closest triangle, then the sign from the parity of the crossings below.
// exact_distance = 0 keeps the reference's point-triangle arithmetic.
void ora_manifold_to_sdf(int nx, int ny, int nz, double h, double ox, double oy, double oz,
                         const double* vert, const int* tri, int64_t ntri, int exact_band,
                         int exact_distance, double* sdf, int* closest, int* icnt) {
  MeshGrid M{nx, ny, nz, h, ox, oy, oz, vert, tri, exact_distance != 0};
  const int64_t N = (int64_t)nx * ny * nz;
  for (int64_t e = 0; e < N; e++) {
    closest[e] = -1;
    icnt[e] = 0;
    sdf[e] = 1e9;
  }
  for (int64_t i = 0; i < ntri; i++) {
    const V3 a = M.vtx((int)i, 0), b = M.vtx((int)i, 1), c = M.vtx((int)i, 2);
    const double mnx = std::min(std::min(a.x - ox, b.x - ox), c.x - ox);
    const double mxx = std::max(std::max(a.x - ox, b.x - ox), c.x - ox);
    const double mny = std::min(std::min(a.y - oy, b.y - oy), c.y - oy);
    const double mxy = std::max(std::max(a.y - oy, b.y - oy), c.y - oy);
    const double mnz = std::min(std::min(a.z - oz, b.z - oz), c.z - oz);
    const double mxz = std::max(std::max(a.z - oz, b.z - oz), c.z - oz);
    int lx = clampi((int)std::floor(mnx / h - 0.5) - exact_band, 0, nx - 1);
    int hx = clampi((int)std::ceil(mxx / h - 0.5) + exact_band, 0, nx - 1);
    int ly = clampi((int)std::floor(mny / h - 0.5) - exact_band, 0, ny - 1);
    int hy = clampi((int)std::ceil(mxy / h - 0.5) + exact_band, 0, ny - 1);
    const int lz = clampi((int)std::floor(mnz / h - 0.5) - exact_band, 0, nz - 1);
    const int hz = clampi((int)std::ceil(mxz / h - 0.5) + exact_band, 0, nz - 1);
    for (int x = lx; x <= hx; x++)
      for (int y = ly; y <= hy; y++)
        for (int z = lz; z <= hz; z++) {
          const double d = dist_point_tri(M.coord(x, y, z), a, b, c, M.exact);
          const int64_t e = M.at(x, y, z);
          if (d < sdf[e]) {
            sdf[e] = d;
            closest[e] = (int)i;
          }
        }
    lx = clampi((int)std::floor(mnx / h - 0.5), 0, nx - 1);
    hx = clampi((int)std::ceil(mxx / h - 0.5), 0, nx - 1);
    ly = clampi((int)std::floor(mny / h - 0.5), 0, ny - 1);
    hy = clampi((int)std::ceil(mxy / h - 0.5), 0, ny - 1);
    for (int j = lx; j <= hx; j++)
      for (int k = ly; k <= hy; k++) {
        const V3 o = M.coord(j, k, -1);
        if (!inside_tri_2d(o.x, o.y, a, b, c)) continue;
        double u, v, w;
        bary_2d(o.x, o.y, a, b, c, &u, &v, &w);
        const double iz = a.z * u + b.z * v + c.z * w;
        const int l = (int)std::ceil((iz - oz) / h - 0.5);
        if (l < 0)
          icnt[M.at(j, k, 0)]++;
        else if (l < nz)
          icnt[M.at(j, k, l)]++;
      }
  }
  for (int round = 0; round < 2; round++) {
    mesh_sweep(M, sdf, closest, 1, 1, 1);
    mesh_sweep(M, sdf, closest, 1, 1, -1);
    mesh_sweep(M, sdf, closest, 1, -1, 1);
    mesh_sweep(M, sdf, closest, 1, -1, -1);
    mesh_sweep(M, sdf, closest, -1, 1, 1);
    mesh_sweep(M, sdf, closest, -1, 1, -1);
    mesh_sweep(M, sdf, closest, -1, -1, 1);
    mesh_sweep(M, sdf, closest, -1, -1, -1);
  }
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++) {
      int tot = 0;
      for (int k = 0; k < nz; k++) {
        tot += icnt[M.at(i, j, k)];
        if (tot & 1) sdf[M.at(i, j, k)] = -sdf[M.at(i, j, k)];
      }
    }
}

int ora_sim_last_iters(const ora_sim* s) { return s->last_iters; }
double ora_sim_last_residual(const ora_sim* s) { return s->last_residual; }

}  // extern "C"

// ---------------------------------------------------------------------------
// rebuildSurface (FluidSim/src/cpu/rebuild-surface.cc:686-741): marching cubes
// over the cubes whose lowest corner runs from -1 to n-1 on each axis, samples
// outside the grid reading 1000 (evalSdf, :655-664).  Vertices are numbered in
// the order they are first met -- cubes in x, y, z order, a cube's case entries
// in table order -- and shared through a hash map keyed by the doubled
// coordinates of the edge midpoint (globalVertexIdx, :643-653).  Serial, as the
// reference.  The cases come from the library's packed table (the same cases as
// the reference's triangleConnectionTable3D, pinned by a digest test).
#include <unordered_map>

#include "../simcraft_b200/csrc/sc_mc_table.h"

namespace {

const uint64_t kMcCases[256] = {SC_MC_CASES_INIT};

struct McOracle {
  int nx, ny, nz;
  double hx, hy, hz, ox, oy, oz;
  const double* sdf;
  double eval(int x, int y, int z) const {  // evalSdf (:655-660)
    if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) return 1000;
    return sdf[((int64_t)x * ny + y) * nz + z];
  }
  // grad (:666-686): central differences, one-sided where the neighbour index
  // would leave [-1, n]; the spacing doubles only strictly inside [0, n-1).
  void grad(int x, int y, int z, double g[3]) const {
    const int xn = x < nx ? x + 1 : x, xp = x > -1 ? x - 1 : x;
    const int yn = y < ny ? y + 1 : y, yp = y > -1 ? y - 1 : y;
    const int zn = z < nz ? z + 1 : z, zp = z > -1 ? z - 1 : z;
    const double dx = x > -1 && x < nx - 1 ? 2 * hx : hx;
    const double dy = y > -1 && y < ny - 1 ? 2 * hy : hy;
    const double dz = z > -1 && z < nz - 1 ? 2 * hz : hz;
    const double gx = eval(xn, y, z) - eval(xp, y, z);
    const double gy = eval(x, yn, z) - eval(x, yp, z);
    const double gz = eval(x, y, zn) - eval(x, y, zp);
    g[0] = gx / dx;
    g[1] = gy / dy;
    g[2] = gz / dz;
  }
};

}  // namespace

int64_t ora_rebuild_surface(int nx, int ny, int nz, const double* spacing, const double* origin,
                            const double* sdf, double* vertices, double* normals, uint32_t* indices,
                            int64_t vertex_capacity, int64_t index_capacity, int64_t* nindices) {
  McOracle M{nx, ny, nz, spacing[0], spacing[1], spacing[2], origin[0], origin[1], origin[2], sdf};
  std::vector<double> V, Nrm;
  std::vector<uint32_t> I;
  std::unordered_map<int64_t, int64_t> vmap;
  const int64_t ky = 2 * (int64_t)ny + 3, kz = 2 * (int64_t)nz + 3;
  for (int x = -1; x < nx; x++)
    for (int y = -1; y < ny; y++)
      for (int z = -1; z < nz; z++) {
        int mask = 0;
        for (int c = 0; c < 8; c++)
          if (M.eval(x + SC_MC_CORNER_X(c), y + SC_MC_CORNER_Y(c), z + SC_MC_CORNER_Z(c)) < 0.0)
            mask |= 1 << c;
        const uint64_t w = kMcCases[mask];
        for (int q = 0; q < SC_MC_COUNT(w); q++) {
          const int e = SC_MC_ENTRY(w, q), ca = SC_MC_EDGE_A(e), cb = SC_MC_EDGE_B(e);
          const int ax = x + SC_MC_CORNER_X(ca), ay = y + SC_MC_CORNER_Y(ca), az = z + SC_MC_CORNER_Z(ca);
          const int bx = x + SC_MC_CORNER_X(cb), by = y + SC_MC_CORNER_Y(cb), bz = z + SC_MC_CORNER_Z(cb);
          // doubled midpoint, shifted by 2 so that it starts at 0 (globalVertexIdx)
          const int64_t key = ((int64_t)(ax + bx + 2) * ky + (ay + by + 2)) * kz + (az + bz + 2);
          auto it = vmap.find(key);
          int64_t vid;
          if (it == vmap.end()) {
            vid = (int64_t)(V.size() / 3);
            const double pa[3] = {(ax + 0.5) * M.hx + M.ox, (ay + 0.5) * M.hy + M.oy, (az + 0.5) * M.hz + M.oz};
            const double pb[3] = {(bx + 0.5) * M.hx + M.ox, (by + 0.5) * M.hy + M.oy, (bz + 0.5) * M.hz + M.oz};
            double na[3], nb[3];
            M.grad(ax, ay, az, na);
            M.grad(bx, by, bz, nb);
            const double va = M.eval(ax, ay, az), vb = M.eval(bx, by, bz);
            const double t = va / (va - vb);
            double n[3];
            for (int d = 0; d < 3; d++) {  // lerp (util.h:26-29): x (1 - t) + y t
              V.push_back(pa[d] * (1 - t) + pb[d] * t);
              n[d] = na[d] * (1 - t) + nb[d] * t;
            }
            // normalize: v * (1 / sqrt(dot(v, v))), the dot summed x + y, then + z
            const double inv = 1.0 / std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for (int d = 0; d < 3; d++) Nrm.push_back(n[d] * inv);
            vmap.emplace(key, vid);
          } else {
            vid = it->second;
          }
          I.push_back((uint32_t)vid);
        }
      }
  const int64_t nv = (int64_t)(V.size() / 3), ni = (int64_t)I.size();
  if (nindices) *nindices = ni;
  if (vertices && normals && indices && vertex_capacity >= nv && index_capacity >= ni) {
    std::memcpy(vertices, V.data(), sizeof(double) * V.size());
    std::memcpy(normals, Nrm.data(), sizeof(double) * Nrm.size());
    std::memcpy(indices, I.data(), sizeof(uint32_t) * I.size());
  }
  return nv;
}
