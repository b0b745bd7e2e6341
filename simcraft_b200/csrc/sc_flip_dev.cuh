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
// The same factor with both pieces evaluated and one selected: the lanes of a
// warp fall in different pieces, and without the branch the G2P tile kernel
// measured 3% faster (project + G2P of 33.5M particles 4.11 -> 3.97 ms); the
// values are the same bit for bit.
template <class T>
__device__ __forceinline__ T bspline_sel(T r) {
  const T inner = radd(rsub(T(2.0 / 3.0), rmul(r, r)), rmul(rmul(rmul(T(0.5), r), r), r));
  const T t = rsub(T(2), r);
  const T outer = rdiv(rmul(rmul(t, t), t), T(6));
  return r < T(1) ? inner : (r < T(2) ? outer : T(0));
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

// make_stencil with every division by h done as a multiplication by 1/h when
// h is a power of two, where the two are the same operation (the bases and
// factors equal make_stencil's bit for bit); pow2 false divides.
template <class T>
__device__ __forceinline__ void make_stencil_pow2(Stencil<T>& S, T px, T py, T pz, T h, T inv, bool pow2) {
  const T p[3] = {px, py, pz};
  auto over = [&](T x) { return pow2 ? rmul(x, inv) : rdiv(x, h); };
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const T off = o ? T(0.5) : T(0);
      const int b = (int)radd(over(rsub(rsub(p[ax], T(0)), rmul(off, h))), T(0.5)) - 1;
      S.base[ax][o] = b;
#pragma unroll
      for (int i = 0; i < 4; i++) S.w[ax][o][i] = bspline_sel(over(fabs(rsub(p[ax], coord1(b + i, off, h)))));
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
__device__ __forceinline__ void handle_collision(const double* col, const Geo& G, double h, T& px, T& py, T& pz,
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
// k_advect on zero grids.  COL: a collider SDF is given; without one the
// kernel is a stream of loads and stores, compiled apart from the collider's
// FP64 sampling so that it needs a fifth of the registers (full occupancy).
template <class T, bool COL>
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
    handle_collision(COL ? col : nullptr, G, hd, px, py, pz, vx, vy, vz);
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

// Order each cell's bucket by original particle index; the reference's
// bucket order is then pinned (ns-util.h:65-69 uses std::sort).  A bucket of
// up to kSortSmall particles is permuted through shared memory (each index's
// rank among the bucket's indices, then one read and one write per array
// element); larger ones take an insertion sort in place.
constexpr int kSortSmall = 16;
__device__ __forceinline__ int64_t to_bits(float v) { return (int64_t)__float_as_uint(v); }
__device__ __forceinline__ int64_t to_bits(double v) { return __double_as_longlong(v); }
template <class T>
__device__ __forceinline__ T from_bits(int64_t b);
template <>
__device__ __forceinline__ float from_bits<float>(int64_t b) { return __uint_as_float((unsigned)b); }
template <>
__device__ __forceinline__ double from_bits<double>(int64_t b) { return __longlong_as_double(b); }
template <class T>
__global__ void __launch_bounds__(kT)
    k_sort_cells(int64_t ncell, const int* start, const int* cnt, PartsT<T> P, int64_t* id) {
  __shared__ int64_t buf[kSortSmall * kT];      // [slot][thread]
  __shared__ unsigned char perm[kSortSmall * kT];  // destination slot -> source slot
  const int t = threadIdx.x;
  GRID_LOOP(c, ncell) {
    const int64_t b = start[c];
    const int m = cnt[c];
    if (m < 2) continue;
    if (m <= kSortSmall) {
      for (int l = 0; l < m; l++) buf[l * kT + t] = id[b + l];
      for (int l = 0; l < m; l++) {
        // rank by index, ties (none in a valid bucket) by slot: a permutation
        const int64_t v = buf[l * kT + t];
        int r = 0;
        for (int k = 0; k < m; k++) {
          const int64_t o = buf[k * kT + t];
          r += o < v || (o == v && k < l);
        }
        perm[r * kT + t] = (unsigned char)l;
      }
      for (int r = 0; r < m; r++) id[b + r] = buf[perm[r * kT + t] * kT + t];
      // values go through the same int64 buffer as their bit patterns (one
      // type for every access: no aliasing between the id and value passes)
      auto permute = [&](T* a) {
        for (int l = 0; l < m; l++) buf[l * kT + t] = to_bits(a[b + l]);
        for (int r = 0; r < m; r++) a[b + r] = from_bits<T>(buf[perm[r * kT + t] * kT + t]);
      };
      permute(P.px);
      permute(P.py);
      permute(P.pz);
      permute(P.vx);
      permute(P.vy);
      permute(P.vz);
      continue;
    }
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
// The buckets a cell's reconstruction visits, as offsets from the cell
// (packed dx + 8 | dy + 8 << 8 | dz + 8 << 16): every offset whose bucket box
// comes within 2r of the cell centre (box distance, in units of h, with a
// margin), the same set for every cell (a boundary bucket's open side faces
// away from the cells that reach it).  A superset of the buckets the
// reference's loop keeps is harmless: only the nearest particle decides the
// result.  They come nearest first, each with a lower bound on the squared
// distance from the cell centre to any particle of that bucket: the box
// distance of the bucket's cell, less a margin for the rounding of the
// particle's cell key (one ulp of the grid size in the particle type, times
// h) and for the rounding of the squared distance.  Particles the sort
// clamped into boundary buckets lie beyond the bucket's box, on the side away
// from every cell centre, so the bound holds for them too.
struct ReconOffsets {
  int n;
  int d[512];
  double g2[512];
};
inline bool recon_offsets(double h, double radius, double key_ulp, ReconOffsets& o) {
  const double R = 2.0 * radius / h;
  const int D = (int)std::ceil(R + 0.5) + 1;
  auto gap = [](int d) { return d == 0 ? 0.0 : std::abs(d) - 0.5; };
  struct Off {
    double g2;
    int d;
  };
  Off all[15 * 15 * 15];
  int n = 0;
  if (D > 7) return false;
  for (int dx = -D; dx <= D; dx++)
    for (int dy = -D; dy <= D; dy++)
      for (int dz = -D; dz <= D; dz++) {
        const double g = gap(dx) * gap(dx) + gap(dy) * gap(dy) + gap(dz) * gap(dz);
        if (g > R * R * (1.0 + 1e-6) + 1e-12) continue;
        double b = 0.0;
        for (int e : {dx, dy, dz}) {
          const double t = std::max(0.0, gap(e) * h - key_ulp * h);
          b += t * t;
        }
        all[n++] = Off{b * (1.0 - 1e-12), (dx + 8) | ((dy + 8) << 8) | ((dz + 8) << 16)};
      }
  if (n > 512) return false;
  // ascending bounds, so that the first bound above the least distance ends the search
  std::stable_sort(all, all + n, [](const Off& a, const Off& b) { return a.g2 < b.g2; });
  o.n = n;
  for (int q = 0; q < n; q++) {
    o.d[q] = all[q].d;
    o.g2[q] = all[q].g2;
  }
  return true;
}
// A block takes one tile of the FP64 extrapolation (8 x 16 x 16 cells) and,
// given `cls`, records the tile's class (a valid cell; all valid), which the
// SDF extrapolation reads instead of scanning every tile's region.
constexpr int kRecTX = 8, kRecTY = 16, kRecTZ = 16;
inline int recon_tiles(const Geo& G) {
  return ((G.nx + kRecTX - 1) / kRecTX) * ((G.ny + kRecTY - 1) / kRecTY) * ((G.nz + kRecTZ - 1) / kRecTZ);
}
template <class T>
__global__ void __launch_bounds__(kT)
    k_reconstruct(Geo G, double h, double radius, const int* start, const int* cnt,
                  const T* __restrict__ px, const T* __restrict__ py, const T* __restrict__ pz,
                  double* sdf, uint8_t* valid, const ReconOffsets off, uint8_t* cls) {
  const double r2 = 2 * radius;
  const int ntz = (G.nz + kRecTZ - 1) / kRecTZ, nty = (G.ny + kRecTY - 1) / kRecTY;
  const int tz = blockIdx.x % ntz, ty = (blockIdx.x / ntz) % nty, tx = blockIdx.x / (ntz * nty);
  int any = 0, all = 1;
  for (int e = threadIdx.x; e < kRecTX * kRecTY * kRecTZ; e += blockDim.x) {
    const int i = tx * kRecTX + e / (kRecTY * kRecTZ), j = ty * kRecTY + (e / kRecTZ) % kRecTY,
              k = tz * kRecTZ + e % kRecTZ;
    if (i >= G.nx || j >= G.ny || k >= G.nz) continue;
    const int64_t id = lin(i, j, k, G.ny, G.nz);
    const double cx = radd(rmul(radd((double)i, 0.5), h), 0.0);
    const double cy = radd(rmul(radd((double)j, 0.5), h), 0.0);
    const double cz = radd(rmul(radd((double)k, 0.5), h), 0.0);
    // min over the candidates of |x - p| - r where |x - p| <= 2r: sqrt and the
    // subtraction are monotone and correctly rounded, so that is sqrt of the
    // least squared distance minus r, when its root passes the test (if the
    // nearest particle fails it, all do): one square root per cell.  The
    // buckets come nearest first; once a bucket's bound exceeds the least
    // squared distance found, no particle of it or of any later bucket can
    // be nearer, and the minimum is exact.
    double m2 = INFINITY;
    for (int q = 0; q < off.n; q++) {
      if (m2 < off.g2[q]) break;
      const int w = off.d[q];
      const int a = i + (w & 255) - 8, b = j + ((w >> 8) & 255) - 8, c = k + ((w >> 16) & 255) - 8;
      if (a < 0 || a >= G.nx || b < 0 || b >= G.ny || c < 0 || c >= G.nz) continue;
      const int cell = (int)lin(a, b, c, G.ny, G.nz);
      const int m = __ldg(cnt + cell);
      if (m < 2) continue;
      const int s = __ldg(start + cell);
      // each bucket's last particle is skipped (the reference's forNeighbours
      // loop stops one short of its inclusive end index)
      for (int l = s; l < s + m - 1; l++) {
        const double dx = rsub((double)px[l], cx), dy = rsub((double)py[l], cy), dz = rsub((double)pz[l], cz);
        m2 = fmin(m2, radd(radd(rmul(dx, dx), rmul(dy, dy)), rmul(dz, dz)));
      }
    }
    double best = 1e9;
    uint8_t ok = 0;
    if (m2 < INFINITY) {
      const double dis = sqrt(m2);
      if (dis <= r2) {
        best = rsub(dis, radius);
        ok = 1;
      }
    }
    sdf[id] = best;
    valid[id] = ok;
    any |= ok;
    all &= ok;
  }
  if (cls) {
    any = __syncthreads_or(any);
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) cls[blockIdx.x] = (any ? 1 : 0) | (all ? 2 : 0);
  }
}
// NaiveReconstructor::reconstruct over the sorted buckets; -1 when the radius
// reaches past the offsets the kernel takes (over ~6 cells).
template <class T>
int launch_reconstruct(cudaStream_t st, const Geo& G, double h, double radius, const int* start, const int* cnt,
                       const T* px, const T* py, const T* pz, double* sdf, uint8_t* valid, uint8_t* cls = nullptr) {
  ReconOffsets off;
  // one ulp of the largest cell index in T: the cell key's rounding, in cells
  const int nmax = std::max(G.nx, std::max(G.ny, G.nz));
  const double key_ulp = std::ldexp(1.0, std::ilogb((double)nmax) + 1 - (sizeof(T) == 4 ? 24 : 53));
  if (!recon_offsets(h, radius, key_ulp, off)) return -1;
  k_reconstruct<T><<<recon_tiles(G), kT, 0, st>>>(G, h, radius, start, cnt, px, py, pz, sdf, valid, off, cls);
  return 0;
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
    // min(own, sum / cnt): when own * cnt < sum exactly (the sign of one fused
    // multiply-add), own is below the rounded quotient or equal to it, so the
    // minimum is own and the division is not needed
    const double own = src[id], cd = (double)cnt;
    double v;
    if (fma(own, cd, -sum) < 0.0) {
      v = own;
    } else {
      v = rdiv(sum, cd);
      if (own < v) v = own;
    }
    dst[id] = v;
  }
}

// `iters` smoothing passes (fluid-simulator.cc:39-74), one launch each: every
// cell changes in every pass, so a tile has nothing to skip, and a
// plane-pipelined kernel running five passes per launch (a ring of planes per
// pass in shared memory) measured slower than five launches of this streaming
// one (256^3: 1.07 ms against 0.60 ms).
inline int launch_smooth(cudaStream_t st, const Geo& G, int iters, double* const sdf[2], int& cur) {
  const int64_t N = (int64_t)G.nx * G.ny * G.nz;
  for (int it = 0; it < iters; it++) {
    k_smooth_sdf<<<nblk(N), kT, 0, st>>>(G, sdf[cur], sdf[1 - cur]);
    cur = 1 - cur;
  }
  return iters;
}

// ---- the iterated grid passes, temporally blocked ----
// extrapolate(.., 10) per face grid (cpu/fluid-simulator.h:204-253) and
// extrapolateFluidSdf(10) (:123-166) are Jacobi-style passes over two buffers:
// pass k reads buffer k mod 2 and writes buffer (k + 1) mod 2, and a cell a
// pass does not write keeps that buffer's older value.  A pass makes valid
// exactly the invalid cells with a valid neighbour, so the cells pass p makes
// valid are those at (6-neighbour) distance p from the cells valid before the
// first pass, and their valid neighbours are all at distance p - 1: made
// valid by pass p - 1, which wrote their values into the very buffer pass p
// reads (or valid from the start, in buffer 0).  So each cell's value is
// computed once, from values computed once, and one value per cell is enough:
// a block loads its tile plus a halo of kIterHalo cells (the values of the
// buffer pass 0 reads, and from the flags the pass that makes each cell valid,
// 0 or not yet) into shared memory, runs up to kIterHalo passes there over a
// region that shrinks by one cell per pass, and writes back, for its tile,
// each new value into the buffer its pass wrote and the last two passes'
// flags (or, for the differentiable step, each pass's flags into their
// history).  Nothing else changes: in the SDF passes a cell without a valid
// neighbour keeps its values; in the face passes it is given zero, which is
// what both face buffers hold there (cleared before P2G, which writes zero
// where it writes no value).  The neighbour order and the arithmetic are
// those of k_extrap_face and k_extrap_sdf, so the results are the same bit
// for bit.  Two kinds of tile need no values: one whose loaded region holds
// no valid flag (the passes change no value; the SDF passes write zero
// flags), and one whose cells are all valid (the passes leave the values and
// set the flags).  Only the tiles along the front of the valid region run the
// passes.
enum { ITER_FACE = 0, ITER_SDF = 1 };
constexpr int kIterThreads = 512;
constexpr int kIterHalo = 5;  // passes per launch at most
template <class T>
struct IterTile;
template <>
struct IterTile<float> {
  static constexpr int X = 16, Y = 16, Z = 16;
};
template <>
struct IterTile<double> {
  static constexpr int X = 8, Y = 16, Z = 16;
};
template <class T>
constexpr int iter_region() {
  return (IterTile<T>::X + 2 * kIterHalo) * (IterTile<T>::Y + 2 * kIterHalo) * (IterTile<T>::Z + 2 * kIterHalo);
}
template <class T>
constexpr size_t iter_smem_bytes() {
  return (size_t)iter_region<T>() * (sizeof(T) + 1);
}
// The pass that makes a cell valid, for cells not valid yet or outside the grid.
constexpr uint8_t kIterNotYet = 255, kIterOutside = 254;
template <class T>
inline int iter_tiles(int dx, int dy, int dz) {
  return ((dx + IterTile<T>::X - 1) / IterTile<T>::X) * ((dy + IterTile<T>::Y - 1) / IterTile<T>::Y) *
         ((dz + IterTile<T>::Z - 1) / IterTile<T>::Z);
}

// One grid's buffers for a launch: values b[2], flags f[2] (ping-pong) or a
// flag history (hist: pass k's flags at hist + k * hstride, f unused); cur:
// the buffer pass 0 reads.
template <class T>
struct IterGrid {
  int dx, dy, dz;
  T* b[2];
  uint8_t* f[2];
  uint8_t* hist;
  int64_t hstride;
  int cur;
  // tile classes (kClsAny: a valid cell in the tile, kClsAll: every in-grid
  // cell of the tile valid) before the launch, and after it; null: the block
  // scans its region's flags instead
  const uint8_t* cin;
  uint8_t* cout;
};
constexpr uint8_t kClsAny = 1, kClsAll = 2;
static_assert(IterTile<double>::X == kRecTX && IterTile<double>::Y == kRecTY && IterTile<double>::Z == kRecTZ,
              "the reconstruction's tiles are the FP64 extrapolation's");

template <class T, int MODE>
__device__ void iter_tile(const IterGrid<T>& G, int tile, int nit, unsigned char* smem) {
  constexpr int TX = IterTile<T>::X, TY = IterTile<T>::Y, TZ = IterTile<T>::Z, H = kIterHalo;
  constexpr int RX = TX + 2 * H, RY = TY + 2 * H, RZ = TZ + 2 * H, RN = RX * RY * RZ;
  T* V = reinterpret_cast<T*>(smem);                  // [RN]: buffer cur, then each cell's new value
  uint8_t* D = reinterpret_cast<uint8_t*>(V + RN);    // [RN]: the pass that makes the cell valid
  const int dx = G.dx, dy = G.dy, dz = G.dz;
  const int ntz = (dz + TZ - 1) / TZ, nty = (dy + TY - 1) / TY;
  const int tz = tile % ntz, ty = (tile / ntz) % nty, tx = tile / (ntz * nty);
  const int x0 = tx * TX - H, y0 = ty * TY - H, z0 = tz * TZ - H;  // region origin
  const T* bs = G.b[G.cur];
  const T* bd = G.b[1 - G.cur];
  const uint8_t* fs = G.hist ? G.hist : G.f[G.cur];
  // region cell e -> global index (or -1 outside the grid)
  auto gidx = [&](int e) -> int64_t {
    const int i = e / (RY * RZ), r = e - i * (RY * RZ), j = r / RZ, k = r - j * RZ;
    const int gx = x0 + i, gy = y0 + j, gz = z0 + k;
    const bool in = gx >= 0 && gx < dx && gy >= 0 && gy < dy && gz >= 0 && gz < dz;
    return in ? lin(gx, gy, gz, dy, dz) : -1;
  };
  const int ntx = (dx + TX - 1) / TX;
  // every tile cell valid: each pass leaves the values and sets the flags
  auto all_valid = [&]() {
    for (int e = threadIdx.x; e < TX * TY * TZ; e += blockDim.x) {
      const int i = e / (TY * TZ), r = e - i * (TY * TZ), j = r / TZ, k = r - j * TZ;
      const int gx = x0 + H + i, gy = y0 + H + j, gz = z0 + H + k;
      if (gx >= dx || gy >= dy || gz >= dz) continue;
      const int64_t gi = lin(gx, gy, gz, dy, dz);
      if (G.hist) {
        for (int p = 1; p <= nit; p++) G.hist[(int64_t)p * G.hstride + gi] = 1;
      } else {
        G.f[0][gi] = 1;
        G.f[1][gi] = 1;
      }
    }
    if (G.cout && threadIdx.x == 0) G.cout[tile] = kClsAny | kClsAll;
  };
  // no valid cell within reach: the face passes would write zeros where the
  // buffers hold zeros already; the SDF passes leave the values and write zero
  // flags into the buffers they write
  auto none_valid = [&]() {
    if (MODE == ITER_SDF && !G.hist)
      for (int e = threadIdx.x; e < TX * TY * TZ; e += blockDim.x) {
        const int i = e / (TY * TZ), r = e - i * (TY * TZ), j = r / TZ, k = r - j * TZ;
        const int gx = x0 + H + i, gy = y0 + H + j, gz = z0 + H + k;
        if (gx >= dx || gy >= dy || gz >= dz) continue;
        const int64_t gi = lin(gx, gy, gz, dy, dz);
        G.f[1 - G.cur][gi] = 0;
        if (nit > 1) G.f[G.cur][gi] = 0;
      }
    if (G.cout && threadIdx.x == 0) G.cout[tile] = 0;
  };
  if (G.cin) {
    // the classes say which tiles are on the front: the halo is shorter than
    // a tile, so a valid cell within reach lies in one of the 27 tiles around
    int nb = 0;
    if (threadIdx.x < 27) {
      const int ax = tx + (int)threadIdx.x % 3 - 1, ay = ty + ((int)threadIdx.x / 3) % 3 - 1,
                az = tz + (int)threadIdx.x / 9 - 1;
      if (ax >= 0 && ax < ntx && ay >= 0 && ay < nty && az >= 0 && az < ntz)
        nb = G.cin[((int64_t)ax * nty + ay) * ntz + az] & kClsAny;
    }
    const bool near = __syncthreads_or(nb);
    if (G.cin[tile] & kClsAll) {
      all_valid();
      return;
    }
    if (!near) {
      none_valid();
      return;
    }
  }
  constexpr int NB = 8;  // loads in flight per thread
  {
    // the flags first: a tile with no valid flag within reach needs no values
    int any = 0, all = 1;  // a valid cell within reach; every in-grid tile cell valid
    for (int e0 = threadIdx.x; e0 < RN; e0 += NB * blockDim.x) {
      uint8_t fv[NB];
      int64_t gv[NB];
#pragma unroll
      for (int u = 0; u < NB; u++) {
        const int e = e0 + u * (int)blockDim.x;
        gv[u] = e < RN ? gidx(e) : -1;
        fv[u] = gv[u] >= 0 ? fs[gv[u]] : 0;
      }
#pragma unroll
      for (int u = 0; u < NB; u++) {
        const int e = e0 + u * (int)blockDim.x;
        if (e < RN) {
          D[e] = fv[u] ? 0 : (gv[u] >= 0 ? kIterNotYet : kIterOutside);
          any |= fv[u];
          const int i = e / (RY * RZ), r = e - i * (RY * RZ), j = r / RZ, k = r - j * RZ;
          if (gv[u] >= 0 && i >= H && i < H + TX && j >= H && j < H + TY && k >= H && k < H + TZ) all &= fv[u];
        }
      }
    }
    if (__syncthreads_and(all)) {
      all_valid();
      return;
    }
    if (!__syncthreads_or(any)) {
      none_valid();
      return;
    }
  }
  for (int e0 = threadIdx.x; e0 < RN; e0 += NB * blockDim.x) {
    T va[NB];
#pragma unroll
    for (int u = 0; u < NB; u++) {
      const int e = e0 + u * (int)blockDim.x;
      const int64_t gi = e < RN ? gidx(e) : -1;
      va[u] = gi >= 0 ? bs[gi] : T(0);
    }
#pragma unroll
    for (int u = 0; u < NB; u++) {
      const int e = e0 + u * (int)blockDim.x;
      if (e < RN) V[e] = va[u];
    }
  }
  __syncthreads();
  constexpr int sX = RY * RZ, sY = RZ;
  constexpr int CL = 8;  // cells of an x run
  for (int p = 1; p <= nit; p++) {
    // the cells whose six neighbours hold the data of p - 1 passes: the box
    // [p, R - p) in each axis, as runs of up to CL cells along x, one run a
    // thread (consecutive threads take consecutive z)
    const int wy = RY - 2 * p, wz = RZ - 2 * p, ncol = wy * wz;
    const int nrun = ncol * ((RX - 2 * p + CL - 1) / CL);
    const int ia = max(p, -x0), ib = min(RX - p, dx - x0);  // in the box and the grid
    const int q = p - 1;  // valid before pass p: D <= q
    for (int it = threadIdx.x; it < nrun; it += blockDim.x) {
      const int ch = it / ncol, col = it - ch * ncol;
      const int jj = col / wz;
      const int j = p + jj, k = p + (col - jj * wz);
      const int gy = y0 + j, gz = z0 + k;
      if (gy < 0 || gy >= dy || gz < 0 || gz >= dz) continue;
      const int i0 = max(ia, p + ch * CL), i1 = min(ib, p + ch * CL + CL);
      for (int i = i0; i < i1; i++) {
        const int e = i * sX + j * sY + k;
        if (D[e] != kIterNotYet) continue;
        // out-of-domain neighbours are never valid and never counted
        T sum = T(0);
        int cnt = 0;
        if (D[e - sX] <= q) { sum = radd(sum, V[e - sX]); cnt++; }
        if (D[e + sX] <= q) { sum = radd(sum, V[e + sX]); cnt++; }
        if (D[e - sY] <= q) { sum = radd(sum, V[e - sY]); cnt++; }
        if (D[e + sY] <= q) { sum = radd(sum, V[e + sY]); cnt++; }
        if (D[e - 1] <= q) { sum = radd(sum, V[e - 1]); cnt++; }
        if (D[e + 1] <= q) { sum = radd(sum, V[e + 1]); cnt++; }
        if (cnt > 0) {
          V[e] = rdiv(sum, (T)cnt);
          D[e] = (uint8_t)p;
        }
      }
    }
    __syncthreads();
  }
  // the tile: a cell made valid by pass d has its value in the buffer that
  // pass wrote, side d mod 2 (the other side keeps what it held: zero in the
  // face grids, which cells without a valid neighbour are given anyway);
  // the last two passes' flags (or every pass's, into the history)
  int any = 0, all = 1;  // the tile's class after the passes
  for (int e = threadIdx.x; e < TX * TY * TZ; e += blockDim.x) {
    const int i = e / (TY * TZ), r = e - i * (TY * TZ), j = r / TZ, k = r - j * TZ;
    const int gx = x0 + H + i, gy = y0 + H + j, gz = z0 + H + k;
    if (gx >= dx || gy >= dy || gz >= dz) continue;
    const int64_t gi = lin(gx, gy, gz, dy, dz);
    const int le = (H + i) * sX + (H + j) * sY + (H + k);
    const int d = D[le];
    if (d >= 1 && d <= nit) G.b[G.cur ^ (d & 1)][gi] = V[le];
    if (G.hist) {
      for (int p = 1; p <= nit; p++) G.hist[(int64_t)p * G.hstride + gi] = d <= p ? 1 : 0;
    } else {
      G.f[G.cur ^ (nit & 1)][gi] = d <= nit ? 1 : 0;
      G.f[G.cur ^ ((nit - 1) & 1)][gi] = d <= nit - 1 ? 1 : 0;
    }
    any |= d <= nit;
    all &= d <= nit;
  }
  if (G.cout) {
    any = __syncthreads_or(any);
    all = __syncthreads_and(all);
    if (threadIdx.x == 0) G.cout[tile] = (any ? kClsAny : 0) | (all ? kClsAll : 0);
  }
}

// The three face grids in one launch (blocks of grid 0, then 1, then 2).
template <class T>
struct IterFaces {
  IterGrid<T> g[3];
  int t0, t1;  // tiles of grid 0, of grids 0 and 1
};
template <class T>
__global__ void __launch_bounds__(kIterThreads) k_iter_faces(IterFaces<T> a, int nit) {
  extern __shared__ __align__(16) unsigned char iter_dyn[];
  const int b = blockIdx.x;
  if (b < a.t0)
    iter_tile<T, ITER_FACE>(a.g[0], b, nit, iter_dyn);
  else if (b < a.t1)
    iter_tile<T, ITER_FACE>(a.g[1], b - a.t0, nit, iter_dyn);
  else
    iter_tile<T, ITER_FACE>(a.g[2], b - a.t1, nit, iter_dyn);
}
template <int MODE>
__global__ void __launch_bounds__(kIterThreads) k_iter_cells(IterGrid<double> g, int nit) {
  extern __shared__ __align__(16) unsigned char iter_dyn[];
  iter_tile<double, MODE>(g, blockIdx.x, nit, iter_dyn);
}

// `iters` passes of extrapolate() over the three face grids; cur[a] is the
// buffer holding grid a's current values, flipped once per pass.  hist[a]:
// the differentiable step's flag history (pass 0 reads hist[a]), or null for
// the ping-pong flags f[a][2].
template <class T>
int launch_extrap_faces(cudaStream_t st, const Geo& G, int iters, T* const b[3][2], uint8_t* const f[3][2],
                        uint8_t* const hist[3], const int64_t fsz[3], int cur[3],
                        uint8_t* const cls[2][3] = nullptr) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_iter_faces<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)iter_smem_bytes<T>());
    attr = true;
  }
  int launches = 0;
  for (int k0 = 0; k0 < iters; k0 += kIterHalo) {
    const int nit = std::min(kIterHalo, iters - k0);
    IterFaces<T> a;
    int acc = 0;
    for (int ax = 0; ax < 3; ax++) {
      IterGrid<T>& g = a.g[ax];
      g.dx = G.nx + (ax == 0);
      g.dy = G.ny + (ax == 1);
      g.dz = G.nz + (ax == 2);
      g.b[0] = b[ax][0];
      g.b[1] = b[ax][1];
      g.f[0] = f ? f[ax][0] : nullptr;
      g.f[1] = f ? f[ax][1] : nullptr;
      g.hist = hist ? hist[ax] + (int64_t)k0 * fsz[ax] : nullptr;
      g.hstride = fsz[ax];
      g.cur = cur[ax];
      // launch k reads the classes launch k - 1 wrote (the first, those of
      // k_dirichlet_tiles) and writes the other array
      const int kl = k0 / kIterHalo;
      g.cin = cls ? cls[kl & 1][ax] : nullptr;
      g.cout = cls ? cls[(kl + 1) & 1][ax] : nullptr;
      acc += iter_tiles<T>(g.dx, g.dy, g.dz);
      if (ax == 0) a.t0 = acc;
      if (ax == 1) a.t1 = acc;
    }
    k_iter_faces<T><<<acc, kIterThreads, iter_smem_bytes<T>(), st>>>(a, nit);
    launches++;
    for (int ax = 0; ax < 3; ax++)
      if (nit & 1) cur[ax] = 1 - cur[ax];
  }
  return launches;
}
// `iters` passes of extrapolateFluidSdf over the cell grid (flags f[2]); cur
// and fcur flip per pass.
template <int MODE>
int launch_iter_cells(cudaStream_t st, const Geo& G, int iters, double* const b[2], uint8_t* const f[2], int& cur,
                      int& fcur, uint8_t* const cls[2] = nullptr) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_iter_cells<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)iter_smem_bytes<double>());
    attr = true;
  }
  int launches = 0;
  for (int k0 = 0; k0 < iters; k0 += kIterHalo) {
    const int nit = std::min(kIterHalo, iters - k0);
    IterGrid<double> g;
    g.dx = G.nx;
    g.dy = G.ny;
    g.dz = G.nz;
    g.b[0] = b[0];
    g.b[1] = b[1];
    // the value and flag buffers flip together, but need not start together:
    // address the flags so that side 0 is the one pass 0 reads
    g.cur = cur;
    g.f[0] = f ? (fcur == cur ? f[0] : f[1]) : nullptr;
    g.f[1] = f ? (fcur == cur ? f[1] : f[0]) : nullptr;
    g.hist = nullptr;
    g.hstride = 0;
    // launch k reads the classes launch k - 1 wrote (the first, the
    // reconstruction's) and writes the other array
    g.cin = cls ? cls[(k0 / kIterHalo) & 1] : nullptr;
    g.cout = cls ? cls[(k0 / kIterHalo + 1) & 1] : nullptr;
    k_iter_cells<MODE><<<iter_tiles<double>(G.nx, G.ny, G.nz), kIterThreads, iter_smem_bytes<double>(), st>>>(g, nit);
    launches++;
    if (nit & 1) {
      cur = 1 - cur;
      if (f) fcur = 1 - fcur;
    }
  }
  return launches;
}

// ---- solveP2G (advect-solver.cc:188-271) ----
// Two kernels, no global atomics and a summation order fixed by the data, so
// the sums are the same bit for bit on every run:
//  k_p2g_tiles:  a block owns an 8x8x8 tile of cells, one thread per cell, and
//                sums its particles' contributions over the nodes they reach
//                (the tile's "region") into shared memory, then writes the
//                region to the tile's slice of a scratch buffer;
//  k_p2g_gather: each face node adds the slices of the tiles whose regions
//                hold it (at most 2 per axis), in tile order, and normalises.
// Within a tile the accumulation is a fixed sequence too.  The weights of a
// particle for face grid AX are the same per-axis factors as the reference's
// (offset 0 along AX, 1/2 along the others).  Along AX the particle's stencil
// starts at its cell - 1 or at its cell (nearest node below or above its
// centre); along the other axes at cell - 1, rounding aside.  So the nodes of
// one cell's particles lie in a 5 x 4 x 4 window.  The tile walks that window
// in 5 passes, one node plane along AX at a time: in a pass each thread sums
// its particles (in bucket order) into 16 registers per quantity for the 4 x 4
// nodes of the plane, stages them, and after a barrier each region node adds
// the staged values of the (up to 16) cells that reach it, in a fixed order.
// Particles whose stencil starts elsewhere (rounding of the half-offset
// nearest-node test, particles outside the grid box, or recorded bases of the
// differentiable step) are added one thread after another, in thread order,
// straight into the region; the region spans cell - 2 .. cell + 3 across AX
// and cell - 1 .. cell + 3 along it, which holds every in-grid node of any
// such particle.  Only a node beyond it (a recorded base far from the
// particle's cell) goes to the global sums with an atomic add, raising the
// spill flag that makes the gather read them.
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
constexpr int kP2GRegion = p2g_region<0>();  // the same for all three grids
static_assert(p2g_region<1>() == kP2GRegion && p2g_region<2>() == kP2GRegion, "region sizes");
template <class T>
constexpr size_t p2g_smem_bytes() {
  // 2 x 16 staged values per thread, the region (sum and weight), outlier list
  return sizeof(T) * (2 * 16 * (size_t)kPThreads + 2 * (size_t)kP2GRegion) + sizeof(int) * (kPThreads + 32);
}

// Device scratch of the two kernels: per tile the three grids' regions (sum
// and weight), per tile a flag (the tile held particles), the spill flag.
struct P2GScratch {
  void* slices = nullptr;
  int* occ = nullptr;
  int* spill = nullptr;
};
inline int64_t p2g_ntiles(const Geo& G) {
  return (int64_t)((G.nx + kPT - 1) / kPT) * ((G.ny + kPT - 1) / kPT) * ((G.nz + kPT - 1) / kPT);
}
inline size_t p2g_scratch_bytes(const Geo& G, size_t elem) {
  const int64_t nt = p2g_ntiles(G);
  const size_t a = (elem * 6 * (size_t)kP2GRegion * nt + 255) & ~(size_t)255;
  return a + ((sizeof(int) * (size_t)(nt + 1) + 255) & ~(size_t)255);
}
inline P2GScratch p2g_scratch_at(void* base, const Geo& G, size_t elem) {
  const int64_t nt = p2g_ntiles(G);
  const size_t a = (elem * 6 * (size_t)kP2GRegion * nt + 255) & ~(size_t)255;
  P2GScratch s;
  s.slices = base;
  s.occ = (int*)((char*)base + a);
  s.spill = s.occ + nt;
  return s;
}

// Spacing of the P2G kernels: a division by h is a multiplication by 1/h,
// exactly, when h is a power of two (the usual 1/2^k grids); otherwise divide.
template <class T>
struct P2GSpacing {
  T h, inv;
  bool pow2;
  __device__ __forceinline__ T over(T x) const { return pow2 ? rmul(x, inv) : rdiv(x, h); }
};
// Nearest-node base along axis D for face grid AX (TGrid::nearest, as
// nearest1 computes it); tb: recorded bases, or null.
template <class T, int AX, int D>
__device__ __forceinline__ int p2g_base(T p, const P2GSpacing<T>& sp, const int16_t* tb) {
  constexpr int o = D == AX ? 0 : 1;
  if (tb) return (int)tb[D * 2 + o];
  return (int)radd(sp.over(rsub(rsub(p, T(0)), rmul(o ? T(0.5) : T(0), sp.h))), T(0.5)) - 1;
}
// The per-axis factor N(|p - x_node| / h) of the cubic B-spline (bspline),
// with the 1/6 of its outer piece as a multiplication: within an ulp of the
// reference's factor, which divides.
template <class T, int AX, int D>
__device__ __forceinline__ T p2g_factor(T p, int node, const P2GSpacing<T>& sp) {
  constexpr T off = D == AX ? T(0) : T(0.5);
  const T r = sp.over(fabs(rsub(p, coord1(node, off, sp.h))));
  if (r < T(1)) return radd(rsub(T(2.0 / 3.0), rmul(r, r)), rmul(rmul(rmul(T(0.5), r), r), r));
  if (r < T(2)) {
    const T t = rsub(T(2), r);
    return rmul(rmul(rmul(t, t), t), T(1.0 / 6.0));
  }
  return T(0);
}
// The same factor from q = p / h and the node's index plus offset c = b + i +
// off: |q - c| is (p - c h) / h rounded once, which on a power-of-two grid is
// the reference's rounding of p - c h scaled exactly, so the factor is the
// same bit for bit; otherwise q carries one more rounding.
// Both pieces are evaluated and one is selected: the lanes of a warp fall in
// different pieces, and the selection keeps them on one path.  (Selecting the
// piece's variable and coefficients first and evaluating once measured slower:
// 256^3 P2G 6.8 -> 7.6 ms, the one evaluation a longer dependent chain.)
template <class T>
__device__ __forceinline__ T p2g_factor_q(T q, T c) {
  const T r = fabs(rsub(q, c));
  const T inner = radd(rsub(T(2.0 / 3.0), rmul(r, r)), rmul(rmul(rmul(T(0.5), r), r), r));
  const T t = rsub(T(2), r);
  const T outer = rmul(rmul(rmul(t, t), t), T(1.0 / 6.0));
  return r < T(1) ? inner : (r < T(2) ? outer : T(0));
}
// The reference's product order: (w_x w_y) w_z.
template <class T>
__device__ __forceinline__ T p2g_weight(T w0, T w1, T w2) {
  return rmul(rmul(w0, w1), w2);
}

template <class T, int AX>
__device__ void p2g_tile_grid(const Geo& G, const P2GSpacing<T>& h, int x0, int y0, int z0, int cx, int cy, int cz, int s0, int m,
                              const PartsT<T>& P, const T* __restrict__ vel, const int16_t* tape,
                              const int64_t* ids, T* stage, T* Rs, int* olist, T* slice, T* gsum, T* gwt,
                              int* spill) {
  constexpr int D1 = AX == 0 ? 1 : 0, D2 = AX == 2 ? 1 : 2;  // the two axes across AX
  constexpr int n0 = P2GRegion<AX, 0>::n, n1 = P2GRegion<AX, 1>::n, n2 = P2GRegion<AX, 2>::n;
  constexpr int lo0 = P2GRegion<AX, 0>::lo, lo1 = P2GRegion<AX, 1>::lo, lo2 = P2GRegion<AX, 2>::lo;
  T* Rw = Rs + kP2GRegion;
  const int tid = threadIdx.x;
  const int c[3] = {cx, cy, cz};
  const int t0[3] = {x0, y0, z0};
  for (int e = tid; e < 2 * kP2GRegion; e += kPThreads) Rs[e] = T(0);
  int nout = 0;
  // the stencil class of the cell's first 32 particles, computed once: bit l
  // of `outm` marks a particle whose stencil starts elsewhere, of `shm` one
  // whose stencil starts at its cell along AX (else at cell - 1)
  unsigned shm = 0u, outm = 0u;
  for (int l = s0; l < s0 + min(m, 32); l++) {
    const T p[3] = {P.px[l], P.py[l], P.pz[l]};
    const int16_t* tb = tape ? tape + 6 * ids[l] : nullptr;
    const int bA = p2g_base<T, AX, AX>(p[AX], h, tb);
    const int b1 = p2g_base<T, AX, D1>(p[D1], h, tb), b2 = p2g_base<T, AX, D2>(p[D2], h, tb);
    const int sh = bA - (c[AX] - 1);
    const unsigned bit = 1u << (l - s0);
    if (sh < 0 || sh > 1 || b1 != c[D1] - 1 || b2 != c[D2] - 1) {
      outm |= bit;
      nout++;
    } else if (sh) {
      shm |= bit;
    }
  }
  // region strides along AX and across it
  constexpr int stA = AX == 0 ? n1 * n2 : (AX == 1 ? n2 : 1);
  constexpr int st1 = D1 == 0 ? n1 * n2 : (D1 == 1 ? n2 : 1);
  constexpr int st2 = D2 == 0 ? n1 * n2 : (D2 == 1 ? n2 : 1);
  for (int ip = 0; ip < 5; ip++) {
    T as[16], aw[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      as[q] = T(0);
      aw[q] = T(0);
    }
    for (int l = s0; l < s0 + m; l++) {
      int sh;
      if (l - s0 < 32) {
        const unsigned bit = 1u << (l - s0);
        if (outm & bit) continue;
        sh = (shm & bit) ? 1 : 0;
      } else {
        const T p[3] = {P.px[l], P.py[l], P.pz[l]};
        const int16_t* tb = tape ? tape + 6 * ids[l] : nullptr;
        const int bA = p2g_base<T, AX, AX>(p[AX], h, tb);
        const int b1 = p2g_base<T, AX, D1>(p[D1], h, tb), b2 = p2g_base<T, AX, D2>(p[D2], h, tb);
        sh = bA - (c[AX] - 1);
        if (sh < 0 || sh > 1 || b1 != c[D1] - 1 || b2 != c[D2] - 1) {
          if (ip == 0) nout++;
          continue;
        }
      }
      const int t = ip - sh;
      if (t < 0 || t > 3) continue;
      const T p[3] = {P.px[l], P.py[l], P.pz[l]};
      const int bA = c[AX] - 1 + sh, b1 = c[D1] - 1, b2 = c[D2] - 1;
      // own axis: offset 0, across: 1/2
      const T wA = p2g_factor_q(h.over(p[AX]), (T)(bA + t));
      const T q1 = h.over(p[D1]), q2 = h.over(p[D2]);
      const T c1 = radd((T)b1, T(0.5)), c2 = radd((T)b2, T(0.5));
      T w1[4], w2[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        w1[j] = p2g_factor_q(q1, radd(c1, (T)j));
        w2[j] = p2g_factor_q(q2, radd(c2, (T)j));
      }
      const T v = vel[l];
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
          // factors in axis order x, y, z
          T f[3];
          f[AX] = wA;
          f[D1] = w1[j];
          f[D2] = w2[k];
          const T wt = p2g_weight(f[0], f[1], f[2]);
          // one fused multiply-add (the sums' order is not the reference's
          // anyway, which adds from a parallel loop)
          as[j * 4 + k] = fma(v, wt, as[j * 4 + k]);
          aw[j * 4 + k] = radd(aw[j * 4 + k], wt);
        }
    }
#pragma unroll
    for (int q = 0; q < 16; q++) {
      stage[q * kPThreads + tid] = as[q];
      stage[(16 + q) * kPThreads + tid] = aw[q];
    }
    __syncthreads();
    // region nodes of this pass: along AX the plane of cell + ip - 1 of each
    // cell of the tile (region index cell + ip), across AX the nodes reached
    // from the tile's cells at their typical bases (region indices 1..11)
    // (the index that runs fastest over the threads is the one along z, in the
    // staged values and in the region alike: consecutive threads read
    // consecutive words)
    constexpr int NA = kPT, NB = kPT + 3;
    for (int e = tid; e < NA * NB * NB; e += kPThreads) {
      int a, b, cc;
      if (AX == 2) {
        a = e % NA;
        const int r = e / NA;
        b = r / NB;
        cc = r - b * NB;
      } else {
        a = e / (NB * NB);
        const int r = e - a * (NB * NB);
        b = r / NB;
        cc = r - b * NB;
      }
      const int rb = b + 1, rc = cc + 1;  // region indices across AX
      T S = T(0), W = T(0);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int q1 = rb - 1 - j;  // the cell along D1 whose window index j is this node
        if (q1 < 0 || q1 >= kPT) continue;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int q2 = rc - 1 - k;
          if (q2 < 0 || q2 >= kPT) continue;
          int lc[3];
          lc[AX] = a;
          lc[D1] = q1;
          lc[D2] = q2;
          const int src = (lc[0] * kPT + lc[1]) * kPT + lc[2];
          S = radd(S, stage[(j * 4 + k) * kPThreads + src]);
          W = radd(W, stage[(16 + j * 4 + k) * kPThreads + src]);
        }
      }
      const int ridx = (a + ip) * stA + rb * st1 + rc * st2;
      Rs[ridx] = radd(Rs[ridx], S);
      Rw[ridx] = radd(Rw[ridx], W);
    }
    __syncthreads();
  }
  // the particles outside the typical windows, thread after thread
  if (__syncthreads_or(nout > 0)) {
    const int lane = tid & 31, warp = tid >> 5;
    int* wcnt = olist + kPThreads;
    const unsigned bal = __ballot_sync(0xffffffffu, nout > 0);
    if (lane == 0) wcnt[warp] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kPThreads / 32; w++) {
      if (w < warp) before += wcnt[w];
      total += wcnt[w];
    }
    if (nout > 0) olist[before + __popc(bal & ((1u << lane) - 1u))] = tid;
    __syncthreads();
    for (int qi = 0; qi < total; qi++) {
      if (olist[qi] == tid) {
        const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
        for (int l = s0; l < s0 + m; l++) {
          const T p[3] = {P.px[l], P.py[l], P.pz[l]};
          const int16_t* tb = tape ? tape + 6 * ids[l] : nullptr;
          int b[3];
          b[AX] = p2g_base<T, AX, AX>(p[AX], h, tb);
          b[D1] = p2g_base<T, AX, D1>(p[D1], h, tb);
          b[D2] = p2g_base<T, AX, D2>(p[D2], h, tb);
          const int sh = b[AX] - (c[AX] - 1);
          if (!(sh < 0 || sh > 1 || b[D1] != c[D1] - 1 || b[D2] != c[D2] - 1)) continue;
          const T v = vel[l];
          T w[3][4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            w[0][i] = p2g_factor<T, AX, 0>(p[0], b[0] + i, h);
            w[1][i] = p2g_factor<T, AX, 1>(p[1], b[1] + i, h);
            w[2][i] = p2g_factor<T, AX, 2>(p[2], b[2] + i, h);
          }
          for (int i = 0; i < 4; i++) {
            const int ga = b[0] + i;
            if (ga < 0 || ga >= fx) continue;
            for (int j = 0; j < 4; j++) {
              const int gb = b[1] + j;
              if (gb < 0 || gb >= fy) continue;
              for (int k = 0; k < 4; k++) {
                const int gc = b[2] + k;
                if (gc < 0 || gc >= fz) continue;
                const T wt = p2g_weight(w[0][i], w[1][j], w[2][k]);
                const int la = ga - (t0[0] - lo0), lb = gb - (t0[1] - lo1), lcc = gc - (t0[2] - lo2);
                if (la >= 0 && la < n0 && lb >= 0 && lb < n1 && lcc >= 0 && lcc < n2) {
                  const int ridx = (la * n1 + lb) * n2 + lcc;
                  Rs[ridx] = radd(Rs[ridx], rmul(v, wt));
                  Rw[ridx] = radd(Rw[ridx], wt);
                } else {
                  const int64_t gi = lin(ga, gb, gc, fy, fz);
                  atomicAdd(gsum + gi, rmul(v, wt));
                  atomicAdd(gwt + gi, wt);
                  *spill = 1;
                }
              }
            }
          }
        }
      }
      __syncthreads();
    }
  }
  for (int e = tid; e < 2 * kP2GRegion; e += kPThreads) slice[e] = Rs[e];
  __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(kPThreads)
    k_p2g_tiles(Geo G, double hd, int pow2, const int* __restrict__ start, const int* __restrict__ cnt, PartsT<T> P,
                T* slices, int* occ, T* su, T* sv, T* sw, T* wu, T* wv, T* ww, int* spill, const int16_t* tape,
                const int64_t* ids) {
  extern __shared__ __align__(16) unsigned char p2g_dyn[];
  T* stage = reinterpret_cast<T*>(p2g_dyn);
  T* Rs = stage + 32 * kPThreads;
  int* olist = reinterpret_cast<int*>(Rs + 2 * kP2GRegion);
  P2GSpacing<T> h;
  h.h = (T)hd;
  h.inv = (T)(1.0 / hd);
  h.pow2 = pow2 != 0;
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
  const bool any = __syncthreads_or(m > 0);
  if (threadIdx.x == 0) occ[blockIdx.x] = any ? 1 : 0;
  if (!any) return;  // no particle in this tile: its slices are never read
  T* slice = slices + (int64_t)blockIdx.x * 6 * kP2GRegion;
  p2g_tile_grid<T, 0>(G, h, x0, y0, z0, cx, cy, cz, s0, m, P, P.vx, tape, ids, stage, Rs, olist, slice, su, wu,
                      spill);
  p2g_tile_grid<T, 1>(G, h, x0, y0, z0, cx, cy, cz, s0, m, P, P.vy, tape, ids, stage, Rs, olist,
                      slice + 2 * kP2GRegion, sv, wv, spill);
  p2g_tile_grid<T, 2>(G, h, x0, y0, z0, cx, cy, cz, s0, m, P, P.vz, tape, ids, stage, Rs, olist,
                      slice + 4 * kP2GRegion, sw, ww, spill);
}

// Tiles along one axis whose regions hold node x: [lo, hi] (empty if lo > hi).
__device__ __forceinline__ void p2g_tiles_of(int x, int rlo, int rn, int ntile, int& lo, int& hi) {
  const int v = x + rlo - rn;  // >= -13
  lo = max(0, (v + 16) / kPT - 16 / kPT + 1);
  hi = min(ntile - 1, (x + rlo) / kPT);
}

// Sum of the tile slices holding each node (tile order), plus the spilled
// global sums when the spill flag is set, then the normalisation of solveP2G
// (advect-solver.cc:238-267): W > 0 -> g = sum / W, valid; else 0, invalid;
// FLIP copies g into `last` (:268-270).  w keeps W.
template <class T, int AX>
__device__ __forceinline__ void p2g_gather_node(const Geo& G, int64_t id, const T* __restrict__ slices,
                                                const int* __restrict__ occ, bool spilled, T* g, T* w,
                                                uint8_t* valid, T* last) {
  const int fy = G.fy(AX), fz = G.fz(AX);
  int a, b, c;
  decode3(id, fy, fz, a, b, c);
  const int ntx = (G.nx + kPT - 1) / kPT, nty = (G.ny + kPT - 1) / kPT, ntz = (G.nz + kPT - 1) / kPT;
  constexpr int lo0 = P2GRegion<AX, 0>::lo, lo1 = P2GRegion<AX, 1>::lo, lo2 = P2GRegion<AX, 2>::lo;
  constexpr int n0 = P2GRegion<AX, 0>::n, n1 = P2GRegion<AX, 1>::n, n2 = P2GRegion<AX, 2>::n;
  int xa, xb, ya, yb, za, zb;
  p2g_tiles_of(a, lo0, n0, ntx, xa, xb);
  p2g_tiles_of(b, lo1, n1, nty, ya, yb);
  p2g_tiles_of(c, lo2, n2, ntz, za, zb);
  T S = T(0), W = T(0);
  for (int tx = xa; tx <= xb; tx++)
    for (int ty = ya; ty <= yb; ty++)
      for (int tz = za; tz <= zb; tz++) {
        const int64_t tile = ((int64_t)tx * nty + ty) * ntz + tz;
        if (!occ[tile]) continue;
        const int la = a - (tx * kPT - lo0), lb = b - (ty * kPT - lo1), lc = c - (tz * kPT - lo2);
        const T* sl = slices + (tile * 6 + 2 * AX) * kP2GRegion + (la * n1 + lb) * n2 + lc;
        S = radd(S, __ldg(sl));
        W = radd(W, __ldg(sl + kP2GRegion));
      }
  if (spilled) {
    S = radd(S, g[id]);
    W = radd(W, w[id]);
  }
  const bool ok = W > T(0);
  const T out = ok ? rdiv(S, W) : T(0);
  g[id] = out;
  w[id] = W;
  valid[id] = ok ? 1 : 0;
  if (last) last[id] = out;
}
template <class T>
__global__ void __launch_bounds__(kT)
    k_p2g_gather(Geo G, const T* __restrict__ slices, const int* __restrict__ occ, const int* __restrict__ spill,
                 T* gu, T* gv, T* gw, T* wu, T* wv, T* ww, uint8_t* vu, uint8_t* vv, uint8_t* vw, T* lu, T* lv,
                 T* lw) {
  const int64_t f0 = (int64_t)(G.nx + 1) * G.ny * G.nz, f1 = (int64_t)G.nx * (G.ny + 1) * G.nz,
                f2 = (int64_t)G.nx * G.ny * (G.nz + 1);
  const bool spilled = *spill != 0;
  GRID_LOOP(i, f0 + f1 + f2) {
    if (i < f0)
      p2g_gather_node<T, 0>(G, i, slices, occ, spilled, gu, wu, vu, lu);
    else if (i < f0 + f1)
      p2g_gather_node<T, 1>(G, i - f0, slices, occ, spilled, gv, wv, vv, lv);
    else
      p2g_gather_node<T, 2>(G, i - f0 - f1, slices, occ, spilled, gw, ww, vw, lw);
  }
}

// solveP2G: the tile sums, then the gather.  g* and w* must hold zeros (the
// spill path adds into them); `scratch` holds p2g_scratch_bytes(G, sizeof(T)).
template <class T>
int launch_p2g(cudaStream_t st, const Geo& G, double h, const int* start, const int* cnt, PartsT<T> P,
               const P2GScratch& scr, T* gu, T* gv, T* gw, T* wu, T* wv, T* ww, uint8_t* vu, uint8_t* vv,
               uint8_t* vw, T* lu, T* lv, T* lw, const int16_t* tape = nullptr, const int64_t* ids = nullptr) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_p2g_tiles<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p2g_smem_bytes<T>());
    attr = true;
  }
  const int64_t tiles = p2g_ntiles(G);
  cudaMemsetAsync(scr.spill, 0, sizeof(int), st);
  int ex = 0;
  const int pow2 = std::frexp(h, &ex) == 0.5 ? 1 : 0;
  k_p2g_tiles<T><<<(unsigned)tiles, kPThreads, p2g_smem_bytes<T>(), st>>>(G, h, pow2, start, cnt, P, (T*)scr.slices,
                                                                          scr.occ, gu, gv, gw, wu, wv, ww,
                                                                          scr.spill, tape, ids);
  const int64_t nf = (int64_t)(G.nx + 1) * G.ny * G.nz + (int64_t)G.nx * (G.ny + 1) * G.nz +
                     (int64_t)G.nx * G.ny * (G.nz + 1);
  k_p2g_gather<T><<<nblk(nf), kT, 0, st>>>(G, (const T*)scr.slices, scr.occ, scr.spill, gu, gv, gw, wu, wv, ww,
                                          vu, vv, vw, lu, lv, lw);
  return 2;
}

// ---- solveG2P over cell tiles (advect-solver.cc:157-169, util.cc:40-85) ----
// A block takes the same 8x8x8 cell tiles as the P2G kernels and first copies
// the P2G region of each face grid it samples (u, v, w and, for FLIP, their
// last values) into shared memory, row by row; the tile's particles then read
// their 4x4x4 stencil nodes from there.  The particles of a column of the tile
// (8 cells along z) are contiguous after the sort; the block numbers the
// tile's particles column after column and gives consecutive particles to
// consecutive threads, so no lane waits on a short column.  The nodes, their
// order and the arithmetic are those of sampleVelocity (gather), so the
// velocities are the same bit for bit; a particle whose stencil leaves the
// region (far outside the grid box, or outside its sorted cell) samples the
// grids in global memory instead.
constexpr int kG2PThreads = 256;
template <class T, int AX>
__device__ __forceinline__ void g2p_stage(T* __restrict__ R, const T* __restrict__ g, const Geo& G, int x0, int y0,
                                          int z0) {
  constexpr int n1 = P2GRegion<AX, 1>::n, n2 = P2GRegion<AX, 2>::n;
  constexpr int lo0 = P2GRegion<AX, 0>::lo, lo1 = P2GRegion<AX, 1>::lo, lo2 = P2GRegion<AX, 2>::lo;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  for (int e = threadIdx.x; e < kP2GRegion; e += blockDim.x) {
    const int i0 = e / (n1 * n2), r = e - i0 * (n1 * n2);
    const int i1 = r / n2, i2 = r - i1 * n2;
    const int a = x0 - lo0 + i0, b = y0 - lo1 + i1, c = z0 - lo2 + i2;
    R[e] = (a >= 0 && a < fx && b >= 0 && b < fy && c >= 0 && c < fz) ? __ldg(g + lin(a, b, c, fy, fz)) : T(0);
  }
}
template <class T, int AX>
__device__ __forceinline__ bool g2p_in_region(const Stencil<T>& S, int x0, int y0, int z0) {
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int r0 = S.base[0][ox] - (x0 - P2GRegion<AX, 0>::lo), r1 = S.base[1][oy] - (y0 - P2GRegion<AX, 1>::lo),
            r2 = S.base[2][oz] - (z0 - P2GRegion<AX, 2>::lo);
  return r0 >= 0 && r0 + 3 < P2GRegion<AX, 0>::n && r1 >= 0 && r1 + 3 < P2GRegion<AX, 1>::n && r2 >= 0 &&
         r2 + 3 < P2GRegion<AX, 2>::n;
}
// Nodes outside the grid get weight zero: the staged region holds zeros
// there, so such a node adds +0 to the value sum and nothing to the weight
// sum, which is what gather's skip of it gives (up to the sign of a zero
// sum, which compares equal).  Along axis d the grid with offset 0 (the face
// grid of axis d) has n_d + 1 nodes, the grids with offset 1/2 have n_d.
template <class T>
__device__ __forceinline__ void g2p_mask_outside(Stencil<T>& S, const Geo& G) {
  const int n[3] = {G.nx, G.ny, G.nz};
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const int ext = n[d] + (o == 0 ? 1 : 0);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int b = S.base[d][o] + i;
        if (b < 0 || b >= ext) S.w[d][o][i] = T(0);
      }
    }
}
// The staged gathers of a particle whose stencils lie inside the region, the
// weights of nodes outside the grid masked: no node is skipped, so the loops
// are branch-free; each grid's sum keeps gather's order.  One grid (and its
// last values) at a time, in a loop over the axes that is not unrolled: with
// all six grids unrolled together the kernel's warps stalled on instruction
// fetch (project + G2P of 33.5M particles 4.3 ms, against 4.1 ms so).
template <class T, bool FLIP>
__device__ __forceinline__ void g2p_gather_axes(const T* __restrict__ R, const Stencil<T>& S, int x0, int y0, int z0,
                                                const PartsT<T>& P, int64_t p, T al, T bl) {
#pragma unroll 1
  for (int ax = 0; ax < 3; ax++) {
    T wx[4], wy[4], wz[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      wx[q] = ax == 0 ? S.w[0][0][q] : S.w[0][1][q];
      wy[q] = ax == 1 ? S.w[1][0][q] : S.w[1][1][q];
      wz[q] = ax == 2 ? S.w[2][0][q] : S.w[2][1][q];
    }
    const int bx = ax == 0 ? S.base[0][0] - (x0 - 1) : S.base[0][1] - (x0 - 2);
    const int by = ax == 1 ? S.base[1][0] - (y0 - 1) : S.base[1][1] - (y0 - 2);
    const int bz = ax == 2 ? S.base[2][0] - (z0 - 1) : S.base[2][1] - (z0 - 2);
    const int n1 = ax == 1 ? kPT + 4 : kPT + 5, n2 = ax == 2 ? kPT + 4 : kPT + 5;
    const T* g = R + ax * kP2GRegion + (bx * n1 + by) * n2 + bz;
    T s = T(0), sl = T(0), ws = T(0);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const T wxy = rmul(wx[i], wy[j]);
        const T* row = g + (i * n1 + j) * n2;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const T wt = rmul(wxy, wz[k]);
          s = radd(s, rmul(row[k], wt));
          if (FLIP) sl = radd(sl, rmul(row[3 * kP2GRegion + k], wt));
          ws = radd(ws, wt);
        }
      }
    T* vp = ax == 0 ? P.vx : (ax == 1 ? P.vy : P.vz);
    const T pic = ws > T(0) ? rdiv(s, ws) : T(0);
    if (!FLIP) {
      vp[p] = pic;
    } else {
      const T last = ws > T(0) ? rdiv(sl, ws) : T(0);
      const T f = rsub(radd(vp[p], pic), last);
      vp[p] = radd(rmul(al, f), rmul(bl, pic));
    }
  }
}
template <class T>
constexpr size_t g2p_smem_bytes(bool flip) {
  return sizeof(T) * (size_t)(flip ? 6 : 3) * kP2GRegion;
}
// Four FP32 blocks of 256 threads per SM (64 registers a thread, no spills)
// measured 25% faster than the register count the compiler picks on its own
// (9.9 -> 7.4 ms for project + G2P of 33.5M particles); the FP64 kernel keeps
// its registers, since its staged regions allow two blocks per SM anyway.
template <class T>
constexpr int g2p_min_blocks() {
  return sizeof(T) == 4 ? 4 : 1;
}
template <class T, bool FLIP>
__global__ void __launch_bounds__(kG2PThreads, g2p_min_blocks<T>())
    k_g2p_tiles(Geo G, double hd, double alphad, int pow2, const int* __restrict__ start,
                const int* __restrict__ cnt, PartsT<T> P, const T* u, const T* v, const T* w, const T* ul,
                const T* vl, const T* wl) {
  extern __shared__ __align__(16) unsigned char g2p_dyn[];
  T* R = reinterpret_cast<T*>(g2p_dyn);  // [grid][region]: u, v, w, then u, v, w last
  __shared__ int cbeg[kPT * kPT], pre[kPT * kPT + 1];
  const T h = (T)hd, hinv = (T)(1.0 / hd);
  constexpr bool flip = FLIP;
  const int ntz = (G.nz + kPT - 1) / kPT, nty = (G.ny + kPT - 1) / kPT;
  const int tz = blockIdx.x % ntz, ty = (blockIdx.x / ntz) % nty, tx = blockIdx.x / (ntz * nty);
  const int x0 = tx * kPT, y0 = ty * kPT, z0 = tz * kPT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    // the particle runs of columns 2 lane and 2 lane + 1 (cells z0 .. z0 + 7
    // of column (x0 + col / 8, y0 + col % 8)), and their exclusive prefix
    int c2[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int col = 2 * lane + q;
      const int x = x0 + col / kPT, y = y0 + col % kPT, zl = min(z0 + kPT, G.nz) - 1;
      int b = 0, e = 0;
      if (x < G.nx && y < G.ny) {
        const int e0 = (int)lin(x, y, z0, G.ny, G.nz), e1 = (int)lin(x, y, zl, G.ny, G.nz);
        b = start[e0];
        e = start[e1] + cnt[e1];
      }
      cbeg[col] = b;
      c2[q] = e - b;
    }
    int inc = c2[0] + c2[1];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += t;
    }
    const int ex = inc - c2[0] - c2[1];
    pre[2 * lane] = ex;
    pre[2 * lane + 1] = ex + c2[0];
    if (lane == 31) pre[kPT * kPT] = inc;
  }
  __syncthreads();
  const int total = pre[kPT * kPT];
  if (total == 0) return;  // no particle in this tile
  g2p_stage<T, 0>(R, u, G, x0, y0, z0);
  g2p_stage<T, 1>(R + kP2GRegion, v, G, x0, y0, z0);
  g2p_stage<T, 2>(R + 2 * kP2GRegion, w, G, x0, y0, z0);
  if (flip) {
    g2p_stage<T, 0>(R + 3 * kP2GRegion, ul, G, x0, y0, z0);
    g2p_stage<T, 1>(R + 4 * kP2GRegion, vl, G, x0, y0, z0);
    g2p_stage<T, 2>(R + 5 * kP2GRegion, wl, G, x0, y0, z0);
  }
  __syncthreads();
  const T al = (T)alphad, bl = rsub(T(1), al);
  // the tile's particles in order, column after column: particle k lies in
  // the last column whose prefix is <= k
  for (int k = threadIdx.x; k < total; k += kG2PThreads) {
    int col = 0;
#pragma unroll
    for (int s = 32; s >= 1; s >>= 1)
      if (pre[col + s] <= k) col += s;
    const int64_t i = (int64_t)cbeg[col] + (k - pre[col]);
    const T px = P.px[i], py = P.py[i], pz = P.pz[i];
    Stencil<T> S;
    make_stencil_pow2(S, px, py, pz, h, hinv, pow2 != 0);
    const bool in = g2p_in_region<T, 0>(S, x0, y0, z0) && g2p_in_region<T, 1>(S, x0, y0, z0) &&
                    g2p_in_region<T, 2>(S, x0, y0, z0);
    if (in) {
      // the common case: every node staged
      g2p_mask_outside(S, G);
      g2p_gather_axes<T, FLIP>(R, S, x0, y0, z0, P, i, al, bl);
      continue;
    }
    // a stencil beyond the staged region: sampleVelocity on the grids in
    // global memory
    const T pu = gather<T, 0>(u, S, G), pv = gather<T, 1>(v, S, G), pw = gather<T, 2>(w, S, G);
    if (!flip) {
      P.vx[i] = pu;
      P.vy[i] = pv;
      P.vz[i] = pw;
      continue;
    }
    const T lu = gather<T, 0>(ul, S, G), lv = gather<T, 1>(vl, S, G), lw = gather<T, 2>(wl, S, G);
    const T fx = rsub(radd(P.vx[i], pu), lu), fy = rsub(radd(P.vy[i], pv), lv), fz = rsub(radd(P.vz[i], pw), lw);
    P.vx[i] = radd(rmul(al, fx), rmul(bl, pu));
    P.vy[i] = radd(rmul(al, fy), rmul(bl, pv));
    P.vz[i] = radd(rmul(al, fz), rmul(bl, pw));
  }
}
// G2P of cell-sorted particles (start/cnt of the sort that ordered P).
template <class T>
int launch_g2p_tiles(cudaStream_t st, const Geo& G, double h, double alpha, const int* start, const int* cnt,
                     PartsT<T> P, const T* u, const T* v, const T* w, const T* ul, const T* vl, const T* wl) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_g2p_tiles<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)g2p_smem_bytes<T>(true));
    cudaFuncSetAttribute(k_g2p_tiles<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)g2p_smem_bytes<T>(false));
    attr = true;
  }
  const bool flip = alpha >= 0.0;
  int ex = 0;
  const int pow2 = std::frexp(h, &ex) == 0.5 ? 1 : 0;
  const unsigned nt = (unsigned)p2g_ntiles(G);
  if (flip)
    k_g2p_tiles<T, true><<<nt, kG2PThreads, g2p_smem_bytes<T>(true), st>>>(G, h, alpha, pow2, start, cnt, P, u, v,
                                                                           w, ul, vl, wl);
  else
    k_g2p_tiles<T, false><<<nt, kG2PThreads, g2p_smem_bytes<T>(false), st>>>(G, h, alpha, pow2, start, cnt, P, u, v,
                                                                            w, ul, vl, wl);
  return 1;
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

// applyDirichletBoundary for the three face grids in one launch, a block per
// extrapolation tile (the tiles of k_iter_faces), which also records each
// tile's class (kClsAny, kClsAll) from its flags after the walls are set: the
// first extrapolation launch reads the classes instead of scanning every
// tile's region.
template <class T>
struct DirTiles {
  T* g[3];
  uint8_t* f[3];
  uint8_t* cls[3];
  int t0, t1;  // tiles of grid 0, of grids 0 and 1
};
constexpr int kDirThreads = 512;
template <class T>
__global__ void __launch_bounds__(kDirThreads) k_dirichlet_tiles(Geo G, DirTiles<T> a) {
  constexpr int TX = IterTile<T>::X, TY = IterTile<T>::Y, TZ = IterTile<T>::Z;
  const int b = blockIdx.x;
  const int ax = b < a.t0 ? 0 : (b < a.t1 ? 1 : 2);
  const int tile = b - (ax == 0 ? 0 : (ax == 1 ? a.t0 : a.t1));
  const int dx = G.fx(ax), dy = G.fy(ax), dz = G.fz(ax);
  const int ntz = (dz + TZ - 1) / TZ, nty = (dy + TY - 1) / TY;
  const int tz = tile % ntz, ty = (tile / ntz) % nty, tx = tile / (ntz * nty);
  T* g = a.g[ax];
  uint8_t* f = a.f[ax];
  const int qm = (ax == 0 ? dx : (ax == 1 ? dy : dz)) - 1;
  int any = 0, all = 1;
  for (int e = threadIdx.x; e < TX * TY * TZ; e += blockDim.x) {
    const int i = e / (TY * TZ), r = e - i * (TY * TZ), j = r / TZ, k = r - j * TZ;
    const int gx = tx * TX + i, gy = ty * TY + j, gz = tz * TZ + k;
    if (gx >= dx || gy >= dy || gz >= dz) continue;
    const int64_t gi = lin(gx, gy, gz, dy, dz);
    const int q = ax == 0 ? gx : (ax == 1 ? gy : gz);
    int v;
    if (q == 0 || q == qm) {
      g[gi] = T(0);
      f[gi] = 1;
      v = 1;
    } else {
      v = f[gi] ? 1 : 0;
    }
    any |= v;
    all &= v;
  }
  any = __syncthreads_or(any);
  all = __syncthreads_and(all);
  if (threadIdx.x == 0) a.cls[ax][tile] = (any ? kClsAny : 0) | (all ? kClsAll : 0);
}
template <class T>
int launch_dirichlet_tiles(cudaStream_t st, const Geo& G, T* const g[3], uint8_t* const f[3], uint8_t* const cls[3]) {
  DirTiles<T> a;
  int acc = 0;
  for (int ax = 0; ax < 3; ax++) {
    a.g[ax] = g[ax];
    a.f[ax] = f[ax];
    a.cls[ax] = cls[ax];
    acc += iter_tiles<T>(G.nx + (ax == 0), G.ny + (ax == 1), G.nz + (ax == 2));
    if (ax == 0) a.t0 = acc;
    if (ax == 1) a.t1 = acc;
  }
  k_dirichlet_tiles<T><<<acc, kDirThreads, 0, st>>>(G, a);
  return 1;
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

// applyCollider without a collider mesh: only the walls along AX change (to
// zero), so the launch covers the two wall planes alone instead of the grid.
template <class T, int AX>
__global__ void __launch_bounds__(kT) k_collider_walls(Geo G, T* g) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int nu = AX == 0 ? fy : fx, nv = AX == 2 ? fy : fz;  // the plane across AX
  const int qm = (AX == 0 ? fx : (AX == 1 ? fy : fz)) - 1;
  const int64_t np = (int64_t)nu * nv;
  GRID_LOOP(t, 2 * np) {
    const int side = t >= np ? 1 : 0;
    const int64_t r = t - side * np;
    const int u = (int)(r / nv), v = (int)(r - (int64_t)u * nv);
    const int q = side ? qm : 0;
    const int a = AX == 0 ? q : u, b = AX == 0 ? u : (AX == 1 ? q : v), c = AX == 2 ? q : v;
    g[lin(a, b, c, fy, fz)] = T(0);
  }
}
// applyCollider on the three face grids (col: the collider SDF, or null for
// the empty-mesh collider); returns the launches.
template <class T>
inline int launch_collider(cudaStream_t st, const Geo& G, double h, T* gu, T* gv, T* gw, const double* col) {
  const int64_t fu = (int64_t)(G.nx + 1) * G.ny * G.nz, fv = (int64_t)G.nx * (G.ny + 1) * G.nz,
                fw = (int64_t)G.nx * G.ny * (G.nz + 1);
  if (col) {
    k_collider<T, 0><<<nblk(fu), kT, 0, st>>>(G, h, gu, col);
    k_collider<T, 1><<<nblk(fv), kT, 0, st>>>(G, h, gv, col);
    k_collider<T, 2><<<nblk(fw), kT, 0, st>>>(G, h, gw, col);
  } else {
    k_collider_walls<T, 0><<<nblk(2 * (int64_t)G.ny * G.nz), kT, 0, st>>>(G, gu);
    k_collider_walls<T, 1><<<nblk(2 * (int64_t)G.nx * G.nz), kT, 0, st>>>(G, gv);
    k_collider_walls<T, 2><<<nblk(2 * (int64_t)G.nx * G.ny), kT, 0, st>>>(G, gw);
  }
  return 3;
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
