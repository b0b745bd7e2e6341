// sc_flip_dev.cuh -- device helpers and kernels of the FLIP/PIC substep,
// shared by the simulator (sc_flip.cu) and its adjoint (sc_diff.cu).  Every
// definition sits in an anonymous namespace: each translation unit that
// includes this header gets its own copy.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "sc_common.cuh"
#include "sc_fvm.cuh"

namespace sc {
namespace {


constexpr int kT = 256;

inline int nblk(int64_t n) {
  int64_t b = (n + kT - 1) / kT;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 1 << 20));
}
#define GRID_LOOP(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// IEEE round-to-nearest operations without contraction, per precision.
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }

// Face-grid geometry (Spatify/include/Spatify/grids.h:287-308, 479-485).
struct Geo {
  int nx, ny, nz;
  __device__ __forceinline__ int fx(int ax) const { return nx + (ax == 0); }
  __device__ __forceinline__ int fy(int ax) const { return ny + (ax == 1); }
  __device__ __forceinline__ int fz(int ax) const { return nz + (ax == 2); }
};

// TGrid::nearest: Vec3i((coord - origin - offset*h)/h + 0.5), truncation.
template <class T>
__device__ __forceinline__ int nearest1(T p, T off, T h) {
  return (int)radd(rdiv(rsub(rsub(p, T(0)), rmul(off, h)), h), T(0.5));
}
// TGrid::indexToCoord: (index + offset) * h + origin.
template <class T>
__device__ __forceinline__ T coord1(int i, T off, T h) {
  return radd(rmul(radd((T)i, off), h), T(0));
}
// Cubic B-spline policy for core::CubicKernel (advect-solver.cc:44): per-axis
// N(|d|/h) with N(r) = 2/3 - r^2 + r^3/2 (r < 1), (2 - r)^3 / 6 (r < 2).
template <class T>
__device__ __forceinline__ T bspline(T r) {
  if (r < T(1)) return radd(rsub(T(2.0 / 3.0), rmul(r, r)), rmul(rmul(rmul(T(0.5), r), r), r));
  if (r < T(2)) {
    T t = rsub(T(2), r);
    return rdiv(rmul(rmul(t, t), t), T(6));
  }
  return T(0);
}
template <class T>
__device__ __forceinline__ T kweight(T h, T dx, T dy, T dz) {
  return rmul(rmul(bspline(rdiv(fabs(dx), h)), bspline(rdiv(fabs(dy), h))),
              bspline(rdiv(fabs(dz), h)));
}

// The kernel weight is a product of per-axis factors, and a face grid uses
// offset 0 along its own axis and 1/2 along the other two, so one position
// needs only 2 x 4 factors per axis for all three grids.  Each factor is
// computed exactly as the per-node expression N(|p - x_node| / h), so the
// products below equal the per-node kernel weights bit for bit.
template <class T>
struct Stencil {
  int base[3][2];  // nearest - 1, per axis, for face offset 0 (index 0) and 1/2 (index 1)
  T w[3][2][4];
};
template <class T>
__device__ __forceinline__ void make_stencil(Stencil<T>& S, T px, T py, T pz, T h) {
  const T p[3] = {px, py, pz};
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const T off = o ? T(0.5) : T(0);
      const int b = nearest1(p[ax], off, h) - 1;
      S.base[ax][o] = b;
#pragma unroll
      for (int i = 0; i < 4; i++) S.w[ax][o][i] = bspline(rdiv(fabs(rsub(p[ax], coord1(b + i, off, h))), h));
    }
}

// The same stencil with its nearest-node bases taken from a record of an
// earlier run (tb: 6 int16 per particle, [axis][offset]); tb == nullptr
// computes them.  The differentiable step replays recorded bases so that the
// map from parameters to loss is smooth around the recorded run.
template <class T>
__device__ __forceinline__ void make_stencil_tb(Stencil<T>& S, T px, T py, T pz, T h,
                                                const int16_t* tb) {
  if (!tb) {
    make_stencil(S, px, py, pz, h);
    return;
  }
  const T p[3] = {px, py, pz};
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const T off = o ? T(0.5) : T(0);
      const int b = tb[ax * 2 + o];
      S.base[ax][o] = b;
#pragma unroll
      for (int i = 0; i < 4; i++) S.w[ax][o][i] = bspline(rdiv(fabs(rsub(p[ax], coord1(b + i, off, h))), h));
    }
}

// sampleVelocity for face grid AX (FluidSim/src/cpu/util.cc:40-85): the same
// nodes in the same order, the same weight and accumulation arithmetic.
template <class T, int AX>
__device__ __forceinline__ T gather(const T* __restrict__ g, const Stencil<T>& S, const Geo& G) {
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  T s = T(0), ws = T(0);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      const T wxy = rmul(S.w[0][ox][i], S.w[1][oy][j]);
      const T* row = g + lin(a, b, 0, fy, fz);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int c = S.base[2][oz] + k;
        if (c < 0 || c >= fz) continue;
        const T wt = rmul(wxy, S.w[2][oz][k]);
        s = radd(s, rmul(__ldg(row + c), wt));
        ws = radd(ws, wt);
      }
    }
  }
  return ws > T(0) ? rdiv(s, ws) : T(0);
}

// SDF<3>::gradient(idx) and grad(p) (FluidSim/include/FluidSim/cpu/sdf.h:62-118).
__device__ void sdf_gradient_at(const double* S, const Geo& G, double h, int ix, int iy, int iz,
                                double* g) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  int xn = ix < nx - 1 ? ix + 1 : ix, xp = ix > 0 ? ix - 1 : ix;
  int yn = iy < ny - 1 ? iy + 1 : iy, yp = iy > 0 ? iy - 1 : iy;
  int zn = iz < nz - 1 ? iz + 1 : iz, zp = iz > 0 ? iz - 1 : iz;
  double dx = ix > 0 && ix < nx - 1 ? 2 * h : h;
  double dy = iy > 0 && iy < ny - 1 ? 2 * h : h;
  double dz = iz > 0 && iz < nz - 1 ? 2 * h : h;
  g[0] = (S[lin(xn, iy, iz, ny, nz)] - S[lin(xp, iy, iz, ny, nz)]) / dx;
  g[1] = (S[lin(ix, yn, iz, ny, nz)] - S[lin(ix, yp, iz, ny, nz)]) / dy;
  g[2] = (S[lin(ix, iy, zn, ny, nz)] - S[lin(ix, iy, zp, ny, nz)]) / dz;
}
__device__ void sdf_grad(const double* S, const Geo& G, double h, double px, double py, double pz,
                         double* out) {
  auto clampi = [](int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); };
  int ix = (int)((px - 0.0) / h - 0.5), iy = (int)((py - 0.0) / h - 0.5), iz = (int)((pz - 0.0) / h - 0.5);
  int x = clampi(ix, 0, G.nx - 1), y = clampi(iy, 0, G.ny - 1), z = clampi(iz, 0, G.nz - 1);
  int xn = clampi(ix + 1, 0, G.nx - 1), yn = clampi(iy + 1, 0, G.ny - 1), zn = clampi(iz + 1, 0, G.nz - 1);
  double tx = (px - (((double)x + 0.5) * h + 0.0)) / h;
  double ty = (py - (((double)y + 0.5) * h + 0.0)) / h;
  double tz = (pz - (((double)z + 0.5) * h + 0.0)) / h;
  double g[8][3];
  sdf_gradient_at(S, G, h, x, y, z, g[0]);
  sdf_gradient_at(S, G, h, x, y, zn, g[1]);
  sdf_gradient_at(S, G, h, x, yn, z, g[2]);
  sdf_gradient_at(S, G, h, x, yn, zn, g[3]);
  sdf_gradient_at(S, G, h, xn, y, z, g[4]);
  sdf_gradient_at(S, G, h, xn, y, zn, g[5]);
  sdf_gradient_at(S, G, h, xn, yn, z, g[6]);
  sdf_gradient_at(S, G, h, xn, yn, zn, g[7]);
  const double w[8] = {tx * ty * tz,       tx * ty * (1 - tz),       tx * (1 - ty) * tz,
                       tx * (1 - ty) * (1 - tz), (1 - tx) * ty * tz, (1 - tx) * ty * (1 - tz),
                       (1 - tx) * (1 - ty) * tz, (1 - tx) * (1 - ty) * (1 - tz)};
  for (int c = 0; c < 3; c++) {
    double s = 0.0;
    for (int k = 0; k < 8; k++) s += w[k] * g[k][c];
    out[c] = s;
  }
}

// HybridAdvectionSolver3D::handleCollision (advect-solver.cc:100-137).
template <class T>
__device__ void handle_collision(const double* col, const Geo& G, double h, T& px, T& py, T& pz,
                                 T& vx, T& vy, T& vz) {
  if (col) {
    const double d = sdf_eval(col, G.nx, G.ny, G.nz, h, (double)px, (double)py, (double)pz);
    if (d < 0.0) {
      double n[3];
      sdf_grad(col, G, h, (double)px, (double)py, (double)pz, n);
      // glm::normalize: n * (1 / sqrt(dot(n, n)))
      const double inv = 1.0 / sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      n[0] *= inv;
      n[1] *= inv;
      n[2] *= inv;
      px = (T)((double)px - d * n[0]);
      py = (T)((double)py - d * n[1]);
      pz = (T)((double)pz - d * n[2]);
      const double vn = fmin((double)vx * n[0] + (double)vy * n[1] + (double)vz * n[2], 0.0);
      vx = (T)((double)vx - vn * n[0]);
      vy = (T)((double)vy - vn * n[1]);
      vz = (T)((double)vz - vn * n[2]);
    }
  }
  const T width = (T)(G.nx * h), height = (T)(G.ny * h), depth = (T)(G.nz * h);
  if (px < T(0)) {
    px = T(0);
    if (vx < T(0)) vx = T(0);
  }
  if (px > width) {
    px = width;
    if (vx > T(0)) vx = T(0);
  }
  if (py < T(0)) {
    py = T(0);
    if (vy < T(0)) vy = T(0);
  }
  if (py > height) {
    py = height;
    if (vy > T(0)) vy = T(0);
  }
  if (pz < T(0)) {
    pz = T(0);
    if (vz < T(0)) vz = T(0);
  }
  if (pz > depth) {
    pz = depth;
    if (vz > T(0)) vz = T(0);
  }
}

struct Parts {
  void *px, *py, *pz, *vx, *vy, *vz;
};
template <class T>
struct PartsT {
  T *px, *py, *pz, *vx, *vy, *vz;
  __host__ __device__ static PartsT from(const Parts& p) {
    return {(T*)p.px, (T*)p.py, (T*)p.pz, (T*)p.vx, (T*)p.vy, (T*)p.vz};
  }
};

// FlipAdvectionSolver3D::advect: RK3 (Ralston) with k2, k3 sampled from the
// grids it is given (advect-solver.cc:170-187), then handleCollision.
template <class T>
__global__ void __launch_bounds__(kT)
    k_advect(int64_t n, PartsT<T> P, const T* __restrict__ u, const T* __restrict__ v,
             const T* __restrict__ w, Geo G, double hd, const double* col, double dtd) {
  const T h = (T)hd, dt = (T)dtd;
  GRID_LOOP(i, n) {
    T px = P.px[i], py = P.py[i], pz = P.pz[i];
    const T k1x = P.vx[i], k1y = P.vy[i], k1z = P.vz[i];
    const T a = rmul(T(0.5), dt);
    const T p1x = radd(px, rmul(a, k1x)), p1y = radd(py, rmul(a, k1y)), p1z = radd(pz, rmul(a, k1z));
    Stencil<T> S;
    make_stencil(S, p1x, p1y, p1z, h);
    const T k2x = gather<T, 0>(u, S, G), k2y = gather<T, 1>(v, S, G), k2z = gather<T, 2>(w, S, G);
    const T b = rmul(T(0.75), dt);
    const T p2x = radd(px, rmul(b, k2x)), p2y = radd(py, rmul(b, k2y)), p2z = radd(pz, rmul(b, k2z));
    make_stencil(S, p2x, p2y, p2z, h);
    const T k3x = gather<T, 0>(u, S, G), k3y = gather<T, 1>(v, S, G), k3z = gather<T, 2>(w, S, G);
    const T c1 = rmul(T(2.0 / 9.0), dt), c2 = rmul(T(1.0 / 3.0), dt), c3 = rmul(T(4.0 / 9.0), dt);
    px = radd(radd(radd(px, rmul(c1, k1x)), rmul(c2, k2x)), rmul(c3, k3x));
    py = radd(radd(radd(py, rmul(c1, k1y)), rmul(c2, k2y)), rmul(c3, k3y));
    pz = radd(radd(radd(pz, rmul(c1, k1z)), rmul(c2, k2z)), rmul(c3, k3z));
    T vx = k1x, vy = k1y, vz = k1z;
    handle_collision(col, G, hd, px, py, pz, vx, vy, vz);
    P.px[i] = px;
    P.py[i] = py;
    P.pz[i] = pz;
    P.vx[i] = vx;
    P.vy[i] = vy;
    P.vz[i] = vz;
  }
}

// advect as the substep runs it: clear() (fluid-simulator.cc:141) has just
// zeroed the grids advect samples, so both RK3 samples are exactly +0 (a
// weighted average of zeros, or 0 where no node is in range) and the update
// reduces to the same rounded sums with zero k2, k3.  Bit-identical to
// k_advect on zero grids.
template <class T>
__global__ void __launch_bounds__(kT)
    k_advect_still(int64_t n, PartsT<T> P, Geo G, double hd, const double* col, double dtd) {
  const T dt = (T)dtd;
  const T zero = T(0);
  GRID_LOOP(i, n) {
    T px = P.px[i], py = P.py[i], pz = P.pz[i];
    const T k1x = P.vx[i], k1y = P.vy[i], k1z = P.vz[i];
    const T c1 = rmul(T(2.0 / 9.0), dt), c2 = rmul(T(1.0 / 3.0), dt), c3 = rmul(T(4.0 / 9.0), dt);
    px = radd(radd(radd(px, rmul(c1, k1x)), rmul(c2, zero)), rmul(c3, zero));
    py = radd(radd(radd(py, rmul(c1, k1y)), rmul(c2, zero)), rmul(c3, zero));
    pz = radd(radd(radd(pz, rmul(c1, k1z)), rmul(c2, zero)), rmul(c3, zero));
    T vx = k1x, vy = k1y, vz = k1z;
    handle_collision(col, G, hd, px, py, pz, vx, vy, vz);
    P.px[i] = px;
    P.py[i] = py;
    P.pz[i] = pz;
    P.vx[i] = vx;
    P.vy[i] = vy;
    P.vz[i] = vz;
  }
}

// FlipAdvectionSolver3D::solveG2P (advect-solver.cc:157-169); alpha < 0 is PIC.
template <class T>
__global__ void __launch_bounds__(kT)
    k_g2p(int64_t n, PartsT<T> P, const T* u, const T* v, const T* w, const T* ul, const T* vl,
          const T* wl, Geo G, double hd, double alphad, const int16_t* tape = nullptr) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    const T px = P.px[i], py = P.py[i], pz = P.pz[i];
    Stencil<T> S;
    make_stencil_tb(S, px, py, pz, h, tape ? tape + 6 * i : nullptr);
    const T pu = gather<T, 0>(u, S, G), pv = gather<T, 1>(v, S, G), pw = gather<T, 2>(w, S, G);
    if (alphad < 0.0) {
      P.vx[i] = pu;
      P.vy[i] = pv;
      P.vz[i] = pw;
      continue;
    }
    const T lu = gather<T, 0>(ul, S, G), lv = gather<T, 1>(vl, S, G), lw = gather<T, 2>(wl, S, G);
    const T al = (T)alphad, bl = rsub(T(1), al);
    const T fx = rsub(radd(P.vx[i], pu), lu), fy = rsub(radd(P.vy[i], pv), lv),
            fz = rsub(radd(P.vz[i], pw), lw);
    P.vx[i] = radd(rmul(al, fx), rmul(bl, pu));
    P.vy[i] = radd(rmul(al, fy), rmul(bl, pv));
    P.vz[i] = radd(rmul(al, fz), rmul(bl, pw));
  }
}

// ---- counting sort by cell (ParticleNeighbourSearcher::update, ns-util.h:46-79) ----
template <class T>
__global__ void __launch_bounds__(kT)
    k_keys(int64_t n, const T* px, const T* py, const T* pz, Geo G, double hd, int* key, int* cnt) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    int ix = (int)floor(rdiv(px[i], h)), iy = (int)floor(rdiv(py[i], h)), iz = (int)floor(rdiv(pz[i], h));
    ix = ix < 0 ? 0 : (ix >= G.nx ? G.nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= G.ny ? G.ny - 1 : iy);
    iz = iz < 0 ? 0 : (iz >= G.nz ? G.nz - 1 : iz);
    const int c = (int)lin(ix, iy, iz, G.ny, G.nz);
    key[i] = c;
    atomicAdd(&cnt[c], 1);
  }
}

// Exclusive scan of `in` into `out` (two-level: 1024-element blocks).
__global__ void __launch_bounds__(1024) k_scan_blocks(int64_t n, const int* in, int* out, int* bsum) {
  __shared__ int s[1024];
  const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  int v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = s[1023];
}
__global__ void __launch_bounds__(1024) k_scan_sums(int nb, int* bsum) {
  __shared__ int s[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) bsum[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
}
__global__ void __launch_bounds__(1024) k_scan_add(int64_t n, int* out, const int* bsum) {
  const int64_t i = (int64_t)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x];
}

template <class T>
__global__ void __launch_bounds__(kT)
    k_scatter(int64_t n, const int* key, const int* start, int* cursor, PartsT<T> src,
              const int64_t* sid, PartsT<T> dst, int64_t* did) {
  GRID_LOOP(i, n) {
    const int c = key[i];
    const int64_t d = (int64_t)start[c] + atomicAdd(&cursor[c], 1);
    dst.px[d] = src.px[i];
    dst.py[d] = src.py[i];
    dst.pz[d] = src.pz[i];
    dst.vx[d] = src.vx[i];
    dst.vy[d] = src.vy[i];
    dst.vz[d] = src.vz[i];
    did[d] = sid[i];
  }
}

// Order each cell's bucket by original particle index (insertion sort); the
// reference's bucket order is then pinned (ns-util.h:65-69 uses std::sort).
template <class T>
__global__ void __launch_bounds__(kT)
    k_sort_cells(int64_t ncell, const int* start, const int* cnt, PartsT<T> P, int64_t* id) {
  GRID_LOOP(c, ncell) {
    const int64_t b = start[c];
    const int m = cnt[c];
    for (int i = 1; i < m; i++) {
      int j = i;
      while (j > 0 && id[b + j - 1] > id[b + j]) {
        const int64_t a = b + j - 1, q = b + j;
        auto sw = [&](auto* arr) {
          auto t = arr[a];
          arr[a] = arr[q];
          arr[q] = t;
        };
        sw(P.px);
        sw(P.py);
        sw(P.pz);
        sw(P.vx);
        sw(P.vy);
        sw(P.vz);
        sw(id);
        j--;
      }
    }
  }
}

// NaiveReconstructor::reconstruct (sdf.h:210-225) over the sorted buckets:
// cell-centred SDF = min over particles within 2r of (|x - p| - r).  Each
// bucket's last particle is skipped, as the reference's forNeighbours loop
// stops one short of its inclusive end index (ns-util.h:76-77, 103).
template <class T>
__global__ void __launch_bounds__(kT)
    k_reconstruct(Geo G, double h, double radius, const int* start, const int* cnt,
                  const T* __restrict__ px, const T* __restrict__ py, const T* __restrict__ pz,
                  double* sdf, uint8_t* valid) {
  const int64_t N = (int64_t)G.nx * G.ny * G.nz;
  const double r2 = 2 * radius;
  GRID_LOOP(id, N) {
    int i, j, k;
    decode3(id, G.ny, G.nz, i, j, k);
    const double cx = radd(rmul(radd((double)i, 0.5), h), 0.0);
    const double cy = radd(rmul(radd((double)j, 0.5), h), 0.0);
    const double cz = radd(rmul(radd((double)k, 0.5), h), 0.0);
    const int x0 = max(0, (int)floor(rdiv(rsub(cx, r2), h))), x1 = min(G.nx - 1, (int)ceil(rdiv(radd(cx, r2), h)));
    const int y0 = max(0, (int)floor(rdiv(rsub(cy, r2), h))), y1 = min(G.ny - 1, (int)ceil(rdiv(radd(cy, r2), h)));
    const int z0 = max(0, (int)floor(rdiv(rsub(cz, r2), h))), z1 = min(G.nz - 1, (int)ceil(rdiv(radd(cz, r2), h)));
    double best = 1e9;
    uint8_t ok = 0;
    const double lim = r2 * r2 * (1.0 + 1e-9);
    // Distance from the cell centre to a bucket's cell box; boundary buckets
    // also hold the particles clamped into them, so their boxes are open.
    auto gap = [&](int a, int n, double c) {
      const double lo = a > 0 ? a * h - c : -1e300, hi = a < n - 1 ? c - (a + 1) * h : -1e300;
      return fmax(0.0, fmax(lo, hi));
    };
    for (int a = x0; a <= x1; a++) {
      const double ex = gap(a, G.nx, cx);
      for (int b = y0; b <= y1; b++) {
        const double ey = gap(b, G.ny, cy);
        if (ex * ex + ey * ey > lim) continue;
        for (int c = z0; c <= z1; c++) {
          const double ez = gap(c, G.nz, cz);
          if (ex * ex + ey * ey + ez * ez > lim) continue;  // no particle of the bucket can be within 2r
          const int cell = (int)lin(a, b, c, G.ny, G.nz);
          const int m = cnt[cell];
          if (m < 2) continue;
          const int s = start[cell];
          for (int l = s; l < s + m - 1; l++) {
            const double dx = rsub((double)px[l], cx), dy = rsub((double)py[l], cy),
                         dz = rsub((double)pz[l], cz);
            const double dis = sqrt(radd(radd(rmul(dx, dx), rmul(dy, dy)), rmul(dz, dz)));
            if (dis <= r2) {
              best = fmin(best, rsub(dis, radius));
              ok = 1;
            }
          }
        }
      }
    }
    sdf[id] = best;
    valid[id] = ok;
  }
}

// extrapolateFluidSdf iteration (cpu/fluid-simulator.h:123-166): valid cells
// keep whatever the destination buffer holds.
__global__ void __launch_bounds__(kT)
    k_extrap_sdf(Geo G, const double* __restrict__ src, double* __restrict__ dst,
                 const uint8_t* __restrict__ vs, uint8_t* __restrict__ vd) {
  const int64_t N = (int64_t)G.nx * G.ny * G.nz;
  const int64_t sx = (int64_t)G.ny * G.nz, sy = G.nz;
  GRID_LOOP(id, N) {
    if (vs[id]) {
      vd[id] = 1;
      continue;
    }
    int i, j, k;
    decode3(id, G.ny, G.nz, i, j, k);
    double sum = 0.0;
    int cnt = 0;
    if (i > 0 && vs[id - sx]) { sum = radd(sum, src[id - sx]); cnt++; }
    if (i < G.nx - 1 && vs[id + sx]) { sum = radd(sum, src[id + sx]); cnt++; }
    if (j > 0 && vs[id - sy]) { sum = radd(sum, src[id - sy]); cnt++; }
    if (j < G.ny - 1 && vs[id + sy]) { sum = radd(sum, src[id + sy]); cnt++; }
    if (k > 0 && vs[id - 1]) { sum = radd(sum, src[id - 1]); cnt++; }
    if (k < G.nz - 1 && vs[id + 1]) { sum = radd(sum, src[id + 1]); cnt++; }
    if (cnt > 0) {
      dst[id] = rdiv(sum, (double)cnt);
      vd[id] = 1;
    } else {
      vd[id] = 0;
    }
  }
}

// smoothFluidSurface iteration (fluid-simulator.cc:39-74).
__global__ void __launch_bounds__(kT)
    k_smooth_sdf(Geo G, const double* __restrict__ src, double* __restrict__ dst) {
  const int64_t N = (int64_t)G.nx * G.ny * G.nz;
  const int64_t sx = (int64_t)G.ny * G.nz, sy = G.nz;
  GRID_LOOP(id, N) {
    int i, j, k;
    decode3(id, G.ny, G.nz, i, j, k);
    double sum = 0.0;
    int cnt = 0;
    if (i > 0) { sum = radd(sum, src[id - sx]); cnt++; }
    if (i < G.nx - 1) { sum = radd(sum, src[id + sx]); cnt++; }
    if (j > 0) { sum = radd(sum, src[id - sy]); cnt++; }
    if (j < G.ny - 1) { sum = radd(sum, src[id + sy]); cnt++; }
    if (k > 0) { sum = radd(sum, src[id - 1]); cnt++; }
    if (k < G.nz - 1) { sum = radd(sum, src[id + 1]); cnt++; }
    double v = rdiv(sum, (double)cnt);
    if (src[id] < v) v = src[id];
    dst[id] = v;
  }
}

// solveP2G (advect-solver.cc:188-271) as a tile splat.  A block owns an
// 8x8x8 tile of cells, one thread per cell; each thread walks its cell's
// particles (contiguous after the per-substep sort), evaluates the per-axis
// kernel factors once per particle and adds the 64 weighted contributions per
// face grid into shared-memory accumulators covering every node the tile's
// particles can reach (nearest + {-1..2}: 12 nodes along a grid's own axis,
// 13 along the others).  The block then adds its accumulators into the global
// sums once.  Threads of a warp own distinct cells, so their shared-memory
// atomics at one stencil offset hit distinct nodes.  Like the reference's
// parallel FLIP splat, the floating-point summation order is not fixed.
constexpr int kPT = 8;                        // cells per tile edge
constexpr int kPThreads = kPT * kPT * kPT;    // one thread per cell
template <int AX, int D>
struct P2GRegion {
  static constexpr int lo = AX == D ? 1 : 2;          // nodes below the tile's first cell
  static constexpr int n = kPT + (AX == D ? 4 : 5);   // nodes along axis D
};
template <int AX>
constexpr int p2g_region() {
  return P2GRegion<AX, 0>::n * P2GRegion<AX, 1>::n * P2GRegion<AX, 2>::n;
}
template <class T>
constexpr size_t p2g_smem_bytes() {
  return sizeof(T) * 2 * (size_t)(p2g_region<0>() + p2g_region<1>() + p2g_region<2>());
}

template <class T, int AX>
__device__ __forceinline__ void p2g_splat_one(const Stencil<T>& S, T val, T* __restrict__ acc,
                                              int x0, int y0, int z0, const Geo& G, T* gsum,
                                              T* gwt) {
  constexpr int o0 = AX == 0 ? 0 : 1, o1 = AX == 1 ? 0 : 1, o2 = AX == 2 ? 0 : 1;
  constexpr int n0 = P2GRegion<AX, 0>::n, n1 = P2GRegion<AX, 1>::n, n2 = P2GRegion<AX, 2>::n;
  constexpr int R = n0 * n1 * n2;
  const int b0 = S.base[0][o0], b1 = S.base[1][o1], b2 = S.base[2][o2];
  const int l0 = b0 - (x0 - P2GRegion<AX, 0>::lo), l1 = b1 - (y0 - P2GRegion<AX, 1>::lo),
            l2 = b2 - (z0 - P2GRegion<AX, 2>::lo);
  if (l0 >= 0 && l0 + 3 < n0 && l1 >= 0 && l1 + 3 < n1 && l2 >= 0 && l2 + 3 < n2) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const T wxy = rmul(S.w[0][o0][i], S.w[1][o1][j]);
        T* row = acc + ((l0 + i) * n1 + (l1 + j)) * n2 + l2;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const T wt = rmul(wxy, S.w[2][o2][k]);
          atomicAdd(row + k, rmul(val, wt));
          atomicAdd(row + k + R, wt);
        }
      }
    return;
  }
  // a particle outside the domain box: straight to the global sums
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  for (int i = 0; i < 4; i++) {
    const int a = b0 + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = b1 + j;
      if (b < 0 || b >= fy) continue;
      const T wxy = rmul(S.w[0][o0][i], S.w[1][o1][j]);
      for (int k = 0; k < 4; k++) {
        const int c = b2 + k;
        if (c < 0 || c >= fz) continue;
        const T wt = rmul(wxy, S.w[2][o2][k]);
        atomicAdd(gsum + lin(a, b, c, fy, fz), rmul(val, wt));
        atomicAdd(gwt + lin(a, b, c, fy, fz), wt);
      }
    }
  }
}

template <class T, int AX>
__device__ __forceinline__ void p2g_merge(const T* __restrict__ acc, int x0, int y0, int z0,
                                          const Geo& G, T* gsum, T* gwt) {
  constexpr int n1 = P2GRegion<AX, 1>::n, n2 = P2GRegion<AX, 2>::n;
  constexpr int R = p2g_region<AX>();
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  for (int e = threadIdx.x; e < R; e += blockDim.x) {
    const T w = acc[R + e];
    if (w == T(0)) continue;
    const int k = e % n2, j = (e / n2) % n1, i = e / (n1 * n2);
    const int a = x0 - P2GRegion<AX, 0>::lo + i, b = y0 - P2GRegion<AX, 1>::lo + j,
              c = z0 - P2GRegion<AX, 2>::lo + k;
    if (a < 0 || a >= fx || b < 0 || b >= fy || c < 0 || c >= fz) continue;  // outside the grid
    const int64_t id = lin(a, b, c, fy, fz);
    atomicAdd(gsum + id, acc[e]);
    atomicAdd(gwt + id, w);
  }
}

// Accumulates sum(v w) and sum(w) of all particles into gsum/gwt (zeroed by
// the caller); k_p2g_normalize finishes solveP2G.
template <class T>
__global__ void __launch_bounds__(kPThreads)
    k_p2g_splat(Geo G, double hd, const int* __restrict__ start, const int* __restrict__ cnt,
                PartsT<T> P, T* su, T* sv, T* sw, T* wu, T* wv, T* ww, const int16_t* tape,
                const int64_t* ids) {
  extern __shared__ __align__(16) unsigned char p2g_dyn[];
  T* acc0 = reinterpret_cast<T*>(p2g_dyn);
  T* acc1 = acc0 + 2 * p2g_region<0>();
  T* acc2 = acc1 + 2 * p2g_region<1>();
  const T h = (T)hd;
  const int ntz = (G.nz + kPT - 1) / kPT, nty = (G.ny + kPT - 1) / kPT;
  const int tz = blockIdx.x % ntz, ty = (blockIdx.x / ntz) % nty, tx = blockIdx.x / (ntz * nty);
  const int x0 = tx * kPT, y0 = ty * kPT, z0 = tz * kPT;
  const int lz = threadIdx.x % kPT, ly = (threadIdx.x / kPT) % kPT, lx = threadIdx.x / (kPT * kPT);
  const int cx = x0 + lx, cy = y0 + ly, cz = z0 + lz;
  int m = 0, s0 = 0;
  if (cx < G.nx && cy < G.ny && cz < G.nz) {
    const int cell = (int)lin(cx, cy, cz, G.ny, G.nz);
    m = cnt[cell];
    s0 = start[cell];
  }
  if (!__syncthreads_or(m > 0)) return;  // no particle in this tile
  constexpr int NACC = 2 * (p2g_region<0>() + p2g_region<1>() + p2g_region<2>());
  for (int e = threadIdx.x; e < NACC; e += blockDim.x) acc0[e] = T(0);
  __syncthreads();
  for (int l = s0; l < s0 + m; l++) {
    Stencil<T> S;
    make_stencil_tb(S, P.px[l], P.py[l], P.pz[l], h, tape ? tape + 6 * ids[l] : nullptr);
    p2g_splat_one<T, 0>(S, P.vx[l], acc0, x0, y0, z0, G, su, wu);
    p2g_splat_one<T, 1>(S, P.vy[l], acc1, x0, y0, z0, G, sv, wv);
    p2g_splat_one<T, 2>(S, P.vz[l], acc2, x0, y0, z0, G, sw, ww);
  }
  __syncthreads();
  p2g_merge<T, 0>(acc0, x0, y0, z0, G, su, wu);
  p2g_merge<T, 1>(acc1, x0, y0, z0, G, sv, wv);
  p2g_merge<T, 2>(acc2, x0, y0, z0, G, sw, ww);
}

// Normalisation of solveP2G (advect-solver.cc:238-267): g = sum / W where
// W > 0 (valid), else 0; FLIP copies the result into `last` (:268-270).
template <class T>
__global__ void __launch_bounds__(kT)
    k_p2g_normalize(int64_t n, T* __restrict__ g, const T* __restrict__ wsum,
                    uint8_t* __restrict__ valid, T* __restrict__ last) {
  GRID_LOOP(i, n) {
    const T w = wsum[i];
    const bool ok = w > T(0);
    const T out = ok ? rdiv(g[i], w) : T(0);
    g[i] = out;
    valid[i] = ok ? 1 : 0;
    if (last) last[i] = out;
  }
}

// Launches the splat over all cell tiles and normalises the three grids; g*
// and w* must hold zeros.
template <class T>
int launch_p2g(cudaStream_t st, const Geo& G, double h, const int* start, const int* cnt,
               PartsT<T> P, T* gu, T* gv, T* gw, T* wu, T* wv, T* ww, uint8_t* vu, uint8_t* vv,
               uint8_t* vw, T* lu, T* lv, T* lw, const int16_t* tape = nullptr,
               const int64_t* ids = nullptr) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_p2g_splat<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)p2g_smem_bytes<T>());
    attr = true;
  }
  const int tiles = ((G.nx + kPT - 1) / kPT) * ((G.ny + kPT - 1) / kPT) * ((G.nz + kPT - 1) / kPT);
  k_p2g_splat<T><<<tiles, kPThreads, p2g_smem_bytes<T>(), st>>>(G, h, start, cnt, P, gu, gv, gw, wu, wv,
                                                                 ww, tape, ids);
  const int64_t f0 = (int64_t)(G.nx + 1) * G.ny * G.nz, f1 = (int64_t)G.nx * (G.ny + 1) * G.nz,
                f2 = (int64_t)G.nx * G.ny * (G.nz + 1);
  k_p2g_normalize<T><<<nblk(f0), kT, 0, st>>>(f0, gu, wu, vu, lu);
  k_p2g_normalize<T><<<nblk(f1), kT, 0, st>>>(f1, gv, wv, vv, lv);
  k_p2g_normalize<T><<<nblk(f2), kT, 0, st>>>(f2, gw, ww, vw, lw);
  return 4;
}

// applyDirichletBoundary for one face grid (fluid-simulator.cc:113-138).
template <class T, int AX>
__global__ void __launch_bounds__(kT) k_dirichlet(Geo G, T* g, uint8_t* valid) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  GRID_LOOP(id, n) {
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    const int q = AX == 0 ? a : (AX == 1 ? b : c), qm = AX == 0 ? fx - 1 : (AX == 1 ? fy - 1 : fz - 1);
    if (q == 0 || q == qm) {
      g[id] = T(0);
      valid[id] = 1;
    }
  }
}

// extrapolate iteration for one face grid (cpu/fluid-simulator.h:204-253):
// valid nodes keep whatever the destination buffer holds; nodes without a
// valid neighbour get 0.
template <class T, int AX>
__global__ void __launch_bounds__(kT)
    k_extrap_face(Geo G, const T* __restrict__ src, T* __restrict__ dst,
                  const uint8_t* __restrict__ vs, uint8_t* __restrict__ vd) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  const int64_t sx = (int64_t)fy * fz, sy = fz;
  GRID_LOOP(id, n) {
    if (vs[id]) {
      vd[id] = 1;
      continue;
    }
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    T sum = T(0);
    int cnt = 0;
    if (a > 0 && vs[id - sx]) { sum = radd(sum, src[id - sx]); cnt++; }
    if (a < fx - 1 && vs[id + sx]) { sum = radd(sum, src[id + sx]); cnt++; }
    if (b > 0 && vs[id - sy]) { sum = radd(sum, src[id - sy]); cnt++; }
    if (b < fy - 1 && vs[id + sy]) { sum = radd(sum, src[id + sy]); cnt++; }
    if (c > 0 && vs[id - 1]) { sum = radd(sum, src[id - 1]); cnt++; }
    if (c < fz - 1 && vs[id + 1]) { sum = radd(sum, src[id + 1]); cnt++; }
    if (cnt > 0) {
      dst[id] = rdiv(sum, (T)cnt);
      vd[id] = 1;
    } else {
      dst[id] = T(0);
      vd[id] = 0;
    }
  }
}

// applyForce (fluid-simulator.cc:13-18): gravity on valid v faces, 0 < j < ny.
template <class T>
__global__ void __launch_bounds__(kT) k_force(Geo G, T* v, const uint8_t* valid, double gdt) {
  const int fy = G.ny + 1;
  const int64_t n = (int64_t)G.nx * fy * G.nz;
  const T d = (T)gdt;
  GRID_LOOP(id, n) {
    int i, j, k;
    decode3(id, fy, G.nz, i, j, k);
    if (valid[id] && j > 0 && j < G.ny) v[id] = rsub(v[id], d);
  }
}

// applyCollider for one face grid (fluid-simulator.cc:76-111).
template <class T, int AX>
__global__ void __launch_bounds__(kT) k_collider(Geo G, double h, T* g, const double* col) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  GRID_LOOP(id, n) {
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    const int q = AX == 0 ? a : (AX == 1 ? b : c), qm = AX == 0 ? fx - 1 : (AX == 1 ? fy - 1 : fz - 1);
    if (q == 0 || q == qm) {
      g[id] = T(0);
      continue;
    }
    if (!col) continue;
    const double px = ((double)a + (AX == 0 ? 0.0 : 0.5)) * h + 0.0;
    const double py = ((double)b + (AX == 1 ? 0.0 : 0.5)) * h + 0.0;
    const double pz = ((double)c + (AX == 2 ? 0.0 : 0.5)) * h + 0.0;
    if (sdf_eval(col, G.nx, G.ny, G.nz, h, px, py, pz) < 0.0) {
      double nrm[3];
      sdf_grad(col, G, h, px, py, pz, nrm);
      // glm::normalize: nrm * (1 / sqrt(dot(nrm, nrm)))
      const double inv = 1.0 / sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
      const double nc = nrm[AX] * inv;
      const double x = (double)g[id];
      g[id] = (T)(x - x * nc);
    }
  }
}

// max |u| over a face grid (for CFL, fluid-simulator.cc:184-203).
template <class T>
__global__ void __launch_bounds__(kT) k_maxabs(int64_t n, const T* g, double* out) {
  double m = 0.0;
  GRID_LOOP(i, n) m = fmax(m, fabs((double)g[i]));
  m = warp_max(m);
  __shared__ double s[kT / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kT / 32; k++) m = fmax(m, s[k]);
    // non-negative doubles order like their bit patterns
    atomicMax((unsigned long long*)out, (unsigned long long)__double_as_longlong(m));
  }
}

template <class T>
__global__ void k_aos_to_soa(int64_t n, const double* pos, const double* vel, PartsT<T> P,
                             int64_t* id) {
  GRID_LOOP(i, n) {
    P.px[i] = (T)pos[3 * i];
    P.py[i] = (T)pos[3 * i + 1];
    P.pz[i] = (T)pos[3 * i + 2];
    P.vx[i] = vel ? (T)vel[3 * i] : T(0);
    P.vy[i] = vel ? (T)vel[3 * i + 1] : T(0);
    P.vz[i] = vel ? (T)vel[3 * i + 2] : T(0);
    if (id) id[i] = i;
  }
}
template <class T>
__global__ void k_soa_to_aos(int64_t n, PartsT<T> P, const int64_t* id, double* pos, double* vel) {
  GRID_LOOP(i, n) {
    const int64_t o = id ? id[i] : i;
    if (pos) {
      pos[3 * o] = (double)P.px[i];
      pos[3 * o + 1] = (double)P.py[i];
      pos[3 * o + 2] = (double)P.pz[i];
    }
    if (vel) {
      vel[3 * o] = (double)P.vx[i];
      vel[3 * o + 1] = (double)P.vy[i];
      vel[3 * o + 2] = (double)P.vz[i];
    }
  }
}
template <class Ts, class Td>
__global__ void k_cast(int64_t n, const Ts* a, Td* b) {
  GRID_LOOP(i, n) b[i] = (Td)a[i];
}

// ---------------------------------------------------------------------------------
// Sorting driver shared by the simulator and the stage functions.
struct SortBufs {
  int *key, *cnt, *start, *cursor, *bsum;
};

template <class T>
int64_t sort_particles(cudaStream_t st, int64_t n, const Geo& G, double h, PartsT<T> src,
                       int64_t* sid, PartsT<T> dst, int64_t* did, const SortBufs& b) {
  const int64_t ncell = (int64_t)G.nx * G.ny * G.nz;
  cudaMemsetAsync(b.cnt, 0, sizeof(int) * ncell, st);
  cudaMemsetAsync(b.cursor, 0, sizeof(int) * ncell, st);
  k_keys<T><<<nblk(n), kT, 0, st>>>(n, src.px, src.py, src.pz, G, h, b.key, b.cnt);
  const int nb = (int)((ncell + 1023) / 1024);
  k_scan_blocks<<<nb, 1024, 0, st>>>(ncell, b.cnt, b.start, b.bsum);
  k_scan_sums<<<1, 1024, 0, st>>>(nb, b.bsum);
  k_scan_add<<<nb, 1024, 0, st>>>(ncell, b.start, b.bsum);
  k_scatter<T><<<nblk(n), kT, 0, st>>>(n, b.key, b.start, b.cursor, src, sid, dst, did);
  k_sort_cells<T><<<nblk(ncell), kT, 0, st>>>(ncell, b.start, b.cnt, dst, did);
  return 7;  // kernels launched
}


}  // namespace
}  // namespace sc
