// sc_diff.cu -- differentiable FLIP/PIC substeps (forward, checkpoints, adjoint).
//
// Forward stages and their sources in the reference:
//   advect + handleCollision   advect-solver.cc:170-187, 100-137 (zero grids: clear() precedes it)
//   reconstruct / extrapolateFluidSdf / smoothFluidSurface   sdf.h:204-229, fluid-simulator.h:123-166
//   solveP2G, applyDirichletBoundary, extrapolate, applyForce   advect-solver.cc:188-271, fluid-simulator.cc:13-138
//   buildSystem, solvePressure, project, applyCollider   project-solver.cc:59-228, 308-435
//   solveG2P                   advect-solver.cc:157-169
// The adjoint kernels below are the transposes of those maps with the run's
// discrete structure fixed (see sc_diff.cuh).
#include <algorithm>
#include <cstring>

#include "sc_diff.cuh"
#include "sc_flip_dev.cuh"

namespace sc {
namespace {

template <class T>
PartsT<T> parts_of(const void* base, int64_t n) {
  T* b = (T*)base;
  return {b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n};
}

// d N(r) / d r of the cubic B-spline policy (bspline above).
template <class T>
__device__ __forceinline__ T bspline_dr(T r) {
  if (r < T(1)) return T(-2) * r + T(1.5) * r * r;
  if (r < T(2)) {
    const T t = T(2) - r;
    return T(-0.5) * t * t;
  }
  return T(0);
}

// Stencil factors and their x-derivatives d/dp N(|p - x_node| / h).
template <class T>
struct StencilD {
  int base[3][2];
  T w[3][2][4];
  T dw[3][2][4];
};
template <class T>
__device__ __forceinline__ void make_stencil_d(StencilD<T>& S, T px, T py, T pz, T h,
                                               const int16_t* tb) {
  const T p[3] = {px, py, pz};
#pragma unroll
  for (int ax = 0; ax < 3; ax++)
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const T off = o ? T(0.5) : T(0);
      const int b = tb ? (int)tb[ax * 2 + o] : nearest1(p[ax], off, h) - 1;
      S.base[ax][o] = b;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const T d = rsub(p[ax], coord1(b + i, off, h));
        const T r = rdiv(fabs(d), h);
        S.w[ax][o][i] = bspline(r);
        S.dw[ax][o][i] = bspline_dr(r) * (d < T(0) ? T(-1) : T(1)) / h;
      }
    }
}

// Value, weight sum and gradient of sampleVelocity on face grid AX:
// S = sum w g / W, grad S = sum grad w (g - S) / W.
template <class T, int AX>
__device__ __forceinline__ void gather_grad(const T* __restrict__ g, const StencilD<T>& S,
                                            const Geo& G, T& val, T& W, T grad[3]) {
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  T s = T(0), ws = T(0);
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      for (int k = 0; k < 4; k++) {
        const int c = S.base[2][oz] + k;
        if (c < 0 || c >= fz) continue;
        const T wt = S.w[0][ox][i] * S.w[1][oy][j] * S.w[2][oz][k];
        s += g[lin(a, b, c, fy, fz)] * wt;
        ws += wt;
      }
    }
  }
  W = ws;
  val = ws > T(0) ? s / ws : T(0);
  grad[0] = grad[1] = grad[2] = T(0);
  if (!(ws > T(0))) return;
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      for (int k = 0; k < 4; k++) {
        const int c = S.base[2][oz] + k;
        if (c < 0 || c >= fz) continue;
        const T d = (g[lin(a, b, c, fy, fz)] - val) / ws;
        grad[0] += S.dw[0][ox][i] * S.w[1][oy][j] * S.w[2][oz][k] * d;
        grad[1] += S.w[0][ox][i] * S.dw[1][oy][j] * S.w[2][oz][k] * d;
        grad[2] += S.w[0][ox][i] * S.w[1][oy][j] * S.dw[2][oz][k] * d;
      }
    }
  }
}

// lambda_g[n] += c * w_n / W over the in-grid stencil nodes of grid AX.
template <class T, int AX>
__device__ __forceinline__ void scatter_sample(T* __restrict__ lg, const StencilD<T>& S, const Geo& G,
                                               T W, T c) {
  if (!(W > T(0)) || c == T(0)) return;
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const T cw = c / W;
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      for (int k = 0; k < 4; k++) {
        const int c2 = S.base[2][oz] + k;
        if (c2 < 0 || c2 >= fz) continue;
        atomicAdd(lg + lin(a, b, c2, fy, fz), cw * S.w[0][ox][i] * S.w[1][oy][j] * S.w[2][oz][k]);
      }
    }
  }
}

// ---- forward kernels ----

// advect as the substep runs it (zero grids, see k_advect_still) with the
// domain-box clamp; records or replays the clamp decisions.
template <class T>
__global__ void __launch_bounds__(kT)
    k_diff_advect(int64_t n, PartsT<T> I, PartsT<T> O, uint16_t* flags, const uint16_t* replay,
                  uint16_t* record, Geo G, double hd, double dtd) {
  const T dt = (T)dtd, zero = T(0);
  const T ext[3] = {(T)(G.nx * hd), (T)(G.ny * hd), (T)(G.nz * hd)};
  GRID_LOOP(i, n) {
    const T c1 = rmul(T(2.0 / 9.0), dt), c2 = rmul(T(1.0 / 3.0), dt), c3 = rmul(T(4.0 / 9.0), dt);
    T p[3] = {I.px[i], I.py[i], I.pz[i]};
    T v[3] = {I.vx[i], I.vy[i], I.vz[i]};
    uint16_t f = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      T q = radd(radd(radd(p[a], rmul(c1, v[a])), rmul(c2, zero)), rmul(c3, zero));
      bool lo, hi, vz;
      if (replay) {
        const uint16_t r = replay[i];
        lo = (r >> a) & 1 && !((r >> (6 + a)) & 1);
        hi = (r >> a) & 1 && ((r >> (6 + a)) & 1);
        vz = (r >> (3 + a)) & 1;
      } else {
        lo = q < T(0);
        hi = !lo && q > ext[a];
        vz = (lo && v[a] < T(0)) || (hi && v[a] > T(0));
      }
      if (lo) q = T(0);
      if (hi) q = ext[a];
      if (vz) v[a] = T(0);
      p[a] = q;
      f |= (uint16_t)((((lo || hi) ? 1 : 0) << a) | ((vz ? 1 : 0) << (3 + a)) | ((hi ? 1 : 0) << (6 + a)));
    }
    flags[i] = f;
    if (record) record[i] = f;
    O.px[i] = p[0];
    O.py[i] = p[1];
    O.pz[i] = p[2];
    O.vx[i] = v[0];
    O.vy[i] = v[1];
    O.vz[i] = v[2];
  }
}

template <class T>
__global__ void __launch_bounds__(kT)
    k_record_bases(int64_t n, const T* px, const T* py, const T* pz, double hd, int16_t* tape) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    const T p[3] = {px[i], py[i], pz[i]};
#pragma unroll
    for (int ax = 0; ax < 3; ax++)
#pragma unroll
      for (int o = 0; o < 2; o++) tape[6 * i + ax * 2 + o] = (int16_t)(nearest1(p[ax], o ? T(0.5) : T(0), h) - 1);
  }
}

// PIC sample of the parameter grids at the initial positions.
template <class T>
__global__ void __launch_bounds__(kT)
    k_sample_into(int64_t n, const T* px, const T* py, const T* pz, const T* u, const T* v,
                  const T* w, Geo G, double hd, T* vx, T* vy, T* vz) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    Stencil<T> S;
    make_stencil(S, px[i], py[i], pz[i], h);
    vx[i] = gather<T, 0>(u, S, G);
    vy[i] = gather<T, 1>(v, S, G);
    vz[i] = gather<T, 2>(w, S, G);
  }
}

// Particle density on the cell centres: rho_c = sum_p N(x_p - x_c) over the
// stencil nearest + {-1..2} (cell-centred nodes: offset 1/2 on every axis).
template <class T>
__global__ void __launch_bounds__(kT)
    k_density(int64_t n, const T* px, const T* py, const T* pz, const int16_t* tape, int16_t* record,
              Geo G, double hd, double* rho) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    Stencil<T> S;
    make_stencil_tb(S, px[i], py[i], pz[i], h, tape ? tape + 6 * i : nullptr);
    if (record)
      for (int q = 0; q < 6; q++) record[6 * i + q] = (int16_t)S.base[q / 2][q % 2];
    for (int a = 0; a < 4; a++) {
      const int x = S.base[0][1] + a;
      if (x < 0 || x >= G.nx) continue;
      for (int b = 0; b < 4; b++) {
        const int y = S.base[1][1] + b;
        if (y < 0 || y >= G.ny) continue;
        const T wxy = S.w[0][1][a] * S.w[1][1][b];
        for (int c = 0; c < 4; c++) {
          const int z = S.base[2][1] + c;
          if (z < 0 || z >= G.nz) continue;
          atomicAdd(rho + lin(x, y, z, G.ny, G.nz), (double)(wxy * S.w[2][1][c]));
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kT) k_loss(int64_t N, const double* rho, const double* target, double* out) {
  double s = 0.0;
  GRID_LOOP(i, N) {
    const double d = rho[i] - target[i];
    s += d * d;
  }
  s = warp_sum(s);
  __shared__ double sh[kT / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kT / 32; k++) t += sh[k];
    atomicAdd(out, t);
  }
}

// ---- adjoint kernels ----

// d loss / d x_p = sum_c 2 (rho_c - rho*_c) grad N_c(x_p)
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_density(int64_t n, PartsT<T> X, const int16_t* tape, Geo G, double hd, const double* rho,
                  const double* target, PartsT<T> L) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    StencilD<T> S;
    make_stencil_d(S, X.px[i], X.py[i], X.pz[i], h, tape ? tape + 6 * i : nullptr);
    T gx = T(0), gy = T(0), gz = T(0);
    for (int a = 0; a < 4; a++) {
      const int x = S.base[0][1] + a;
      if (x < 0 || x >= G.nx) continue;
      for (int b = 0; b < 4; b++) {
        const int y = S.base[1][1] + b;
        if (y < 0 || y >= G.ny) continue;
        for (int c = 0; c < 4; c++) {
          const int z = S.base[2][1] + c;
          if (z < 0 || z >= G.nz) continue;
          const int64_t id = lin(x, y, z, G.ny, G.nz);
          const T l = (T)(2.0 * (rho[id] - target[id]));
          gx += l * S.dw[0][1][a] * S.w[1][1][b] * S.w[2][1][c];
          gy += l * S.w[0][1][a] * S.dw[1][1][b] * S.w[2][1][c];
          gz += l * S.w[0][1][a] * S.w[1][1][b] * S.dw[2][1][c];
        }
      }
    }
    L.px[i] = gx;
    L.py[i] = gy;
    L.pz[i] = gz;
    L.vx[i] = T(0);
    L.vy[i] = T(0);
    L.vz[i] = T(0);
  }
}

// G2P: v'' = alpha v' + S(u) - alpha S(u_last) (FLIP), v'' = S(u) (PIC).
// In: L.x = d/dx', L.v = d/dv''.  Out: L.x += ..., L.v = d/dv' (G2P part);
// scatters into lu (d/du) and lul (d/du_last).
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_g2p(int64_t n, PartsT<T> A, const T* u, const T* v, const T* w, const T* ul, const T* vl,
              const T* wl, const int16_t* tape, Geo G, double hd, double alphad, PartsT<T> L,
              T* lu, T* lv, T* lw, T* lul, T* lvl, T* lwl) {
  const T h = (T)hd;
  const bool flip = alphad >= 0.0;
  const T al = flip ? (T)alphad : T(0);
  GRID_LOOP(i, n) {
    StencilD<T> S;
    make_stencil_d(S, A.px[i], A.py[i], A.pz[i], h, tape ? tape + 6 * i : nullptr);
    const T lvv[3] = {L.vx[i], L.vy[i], L.vz[i]};
    T gx = L.px[i], gy = L.py[i], gz = L.pz[i];
    const T* gr[3] = {u, v, w};
    const T* gl[3] = {ul, vl, wl};
    T* lgr[3] = {lu, lv, lw};
    T* lgl[3] = {lul, lvl, lwl};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      T val, W, grad[3];
      if (a == 0) gather_grad<T, 0>(gr[0], S, G, val, W, grad);
      else if (a == 1) gather_grad<T, 1>(gr[1], S, G, val, W, grad);
      else gather_grad<T, 2>(gr[2], S, G, val, W, grad);
      gx += lvv[a] * grad[0];
      gy += lvv[a] * grad[1];
      gz += lvv[a] * grad[2];
      if (a == 0) scatter_sample<T, 0>(lgr[0], S, G, W, lvv[0]);
      else if (a == 1) scatter_sample<T, 1>(lgr[1], S, G, W, lvv[1]);
      else scatter_sample<T, 2>(lgr[2], S, G, W, lvv[2]);
      if (flip) {
        T vl2, Wl, gradl[3];
        if (a == 0) gather_grad<T, 0>(gl[0], S, G, vl2, Wl, gradl);
        else if (a == 1) gather_grad<T, 1>(gl[1], S, G, vl2, Wl, gradl);
        else gather_grad<T, 2>(gl[2], S, G, vl2, Wl, gradl);
        gx -= al * lvv[a] * gradl[0];
        gy -= al * lvv[a] * gradl[1];
        gz -= al * lvv[a] * gradl[2];
        if (a == 0) scatter_sample<T, 0>(lgl[0], S, G, Wl, -al * lvv[0]);
        else if (a == 1) scatter_sample<T, 1>(lgl[1], S, G, Wl, -al * lvv[1]);
        else scatter_sample<T, 2>(lgl[2], S, G, Wl, -al * lvv[2]);
      }
    }
    L.px[i] = gx;
    L.py[i] = gy;
    L.pz[i] = gz;
    L.vx[i] = al * lvv[0];
    L.vy[i] = al * lvv[1];
    L.vz[i] = al * lvv[2];
  }
}

// applyCollider with no collider: the walls are set to zero.
template <class T, int AX>
__global__ void __launch_bounds__(kT) k_adj_walls(Geo G, T* lg) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  GRID_LOOP(id, n) {
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    const int q = AX == 0 ? a : (AX == 1 ? b : c), qm = AX == 0 ? fx - 1 : (AX == 1 ? fy - 1 : fz - 1);
    if (q == 0 || q == qm) lg[id] = T(0);
  }
}

// Coefficient of p(cell on side `right` of face id) in project's update of
// that face (project-solver.cc:355-420): 0 when the face is not updated.
__device__ __forceinline__ double project_coef(const double* F, const double* wt, int64_t id,
                                               int64_t lcell, int64_t rcell, bool wall, bool right,
                                               double dt_h) {
  if (!(wt[id] > 0.0) || wall) return 0.0;
  const double sl = F[lcell], sr = F[rcell];
  if (sl >= 0.0 && sr >= 0.0) return 0.0;
  if (sl < 0.0 && sr < 0.0) return right ? -dt_h : dt_h;
  if (sl < 0.0) {
    const double theta = fmax(sl / (sl - sr), 0.01);
    return right ? 0.0 : dt_h / theta;
  }
  const double theta = fmin(sl / (sl - sr), 0.99);
  return right ? -dt_h / (1.0 - theta) : 0.0;
}

// d/dp of the projection: per active cell, the sum over its six faces of the
// face's p-coefficient times d/du(face).  Written into the solver's tiled rhs.
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_project(Geo G, double h, double dt, Tiled tg, const uint8_t* __restrict__ act,
                  const double* __restrict__ F, const double* __restrict__ wu, const double* __restrict__ wv,
                  const double* __restrict__ ww, const T* __restrict__ lu, const T* __restrict__ lv,
                  const T* __restrict__ lw, double* __restrict__ rhs) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const int64_t N = (int64_t)nx * ny * nz;
  const double dt_h = dt / h;
  GRID_LOOP(id, N) {
    const int k = (int)(id % nz);
    const int j = (int)((id / nz) % ny);
    const int i = (int)(id / ((int64_t)ny * nz));
    const int64_t e = tg.off(i, j, k);
    if (!act[e]) continue;
    double s = 0.0;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    {  // u faces i (this cell on the right) and i+1 (on the left)
      const int64_t f0 = lin(i, j, k, ny, nz), f1 = lin(i + 1, j, k, ny, nz);
      if (i > 0) s += project_coef(F, wu, f0, id - sx, id, false, true, dt_h) * (double)lu[f0];
      if (i + 1 < nx) s += project_coef(F, wu, f1, id, id + sx, false, false, dt_h) * (double)lu[f1];
    }
    {
      const int64_t f0 = lin(i, j, k, ny + 1, nz), f1 = lin(i, j + 1, k, ny + 1, nz);
      if (j > 0) s += project_coef(F, wv, f0, id - sy, id, false, true, dt_h) * (double)lv[f0];
      if (j + 1 < ny) s += project_coef(F, wv, f1, id, id + sy, false, false, dt_h) * (double)lv[f1];
    }
    {
      const int64_t f0 = lin(i, j, k, ny, nz + 1), f1 = lin(i, j, k + 1, ny, nz + 1);
      if (k > 0) s += project_coef(F, ww, f0, id - 1, id, false, true, dt_h) * (double)lw[f0];
      if (k + 1 < nz) s += project_coef(F, ww, f1, id, id + 1, false, false, dt_h) * (double)lw[f1];
    }
    rhs[e] = s;
  }
}

// d/du of buildSystem's right-hand side (project-solver.cc:129-226): the
// face is +uw u in its right cell's row (i > 0) and -uw u in its left cell's
// row (i < nx-1; the up face of v uses the reference's width/height bound).
template <class T, int AX>
__global__ void __launch_bounds__(kT)
    k_adj_rhs(Geo G, Tiled tg, const double* __restrict__ mu, const double* __restrict__ wt,
              T* __restrict__ lg) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  GRID_LOOP(id, n) {
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    const int q = AX == 0 ? a : (AX == 1 ? b : c);
    const int qn = AX == 0 ? nx : (AX == 1 ? ny : nz);
    double s = 0.0;
    // right cell (index q) has this face as its low face when q > 0
    if (q > 0 && q < qn) s += mu[tg.off(a, b, c)];
    // left cell (index q-1) has it as its high face when q-1 < qn-1 (and for v, q-1 < nx-1)
    if (q >= 1 && q - 1 < qn - 1 && (AX != 1 || q - 1 < nx - 1))
      s -= mu[tg.off(a - (AX == 0), b - (AX == 1), c - (AX == 2))];
    if (s != 0.0) lg[id] += (T)(wt[id] * s);
  }
}

// Transpose of one extrapolation iteration (k_extrap_face): cells invalid in
// vs took the mean of their valid neighbours from src; valid cells kept dst.
template <class T, int AX>
__global__ void __launch_bounds__(kT)
    k_adj_extrap_src(Geo G, T* __restrict__ ls, const T* __restrict__ ld, const uint8_t* __restrict__ vs) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  const int64_t sx = (int64_t)fy * fz, sy = fz;
  auto count = [&](int64_t i, int a, int b, int c) {
    int m = 0;
    if (a > 0 && vs[i - sx]) m++;
    if (a < fx - 1 && vs[i + sx]) m++;
    if (b > 0 && vs[i - sy]) m++;
    if (b < fy - 1 && vs[i + sy]) m++;
    if (c > 0 && vs[i - 1]) m++;
    if (c < fz - 1 && vs[i + 1]) m++;
    return m;
  };
  GRID_LOOP(id, n) {
    if (!vs[id]) continue;
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    T s = T(0);
    if (a > 0 && !vs[id - sx]) s += ld[id - sx] / (T)count(id - sx, a - 1, b, c);
    if (a < fx - 1 && !vs[id + sx]) s += ld[id + sx] / (T)count(id + sx, a + 1, b, c);
    if (b > 0 && !vs[id - sy]) s += ld[id - sy] / (T)count(id - sy, a, b - 1, c);
    if (b < fy - 1 && !vs[id + sy]) s += ld[id + sy] / (T)count(id + sy, a, b + 1, c);
    if (c > 0 && !vs[id - 1]) s += ld[id - 1] / (T)count(id - 1, a, b, c - 1);
    if (c < fz - 1 && !vs[id + 1]) s += ld[id + 1] / (T)count(id + 1, a, b, c + 1);
    ls[id] += s;
  }
}
template <class T>
__global__ void __launch_bounds__(kT) k_adj_extrap_dst(int64_t n, T* __restrict__ ld, const uint8_t* __restrict__ vs) {
  GRID_LOOP(id, n) if (!vs[id]) ld[id] = T(0);
}

// applyDirichletBoundary overwrote the walls after P2G; u_last kept the raw P2G
// result: d/d(P2G output) = (walls ? 0 : d/d(after Dirichlet)) + d/du_last.
template <class T, int AX>
__global__ void __launch_bounds__(kT) k_adj_dirichlet(Geo G, T* lg, const T* lul) {
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  const int64_t n = (int64_t)fx * fy * fz;
  GRID_LOOP(id, n) {
    int a, b, c;
    decode3(id, fy, fz, a, b, c);
    const int q = AX == 0 ? a : (AX == 1 ? b : c), qm = AX == 0 ? fx - 1 : (AX == 1 ? fy - 1 : fz - 1);
    lg[id] = ((q == 0 || q == qm) ? T(0) : lg[id]) + lul[id];
  }
}

// P2G: g_n = sum_p w_np v_p / W_n.  d/dv_p += sum_n lg_n w_np / W_n;
// d/dx_p += sum_n lg_n (v_p - g_n) grad w_np / W_n.
template <class T, int AX>
__device__ __forceinline__ void adj_p2g_grid(const StencilD<T>& S, T vp, const T* __restrict__ g,
                                             const T* __restrict__ W, const T* __restrict__ lg,
                                             const Geo& G, T& lv, T& gx, T& gy, T& gz) {
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      for (int k = 0; k < 4; k++) {
        const int c = S.base[2][oz] + k;
        if (c < 0 || c >= fz) continue;
        const int64_t id = lin(a, b, c, fy, fz);
        const T Wn = W[id];
        if (!(Wn > T(0))) continue;
        const T l = lg[id] / Wn;
        if (l == T(0)) continue;
        const T wx = S.w[0][ox][i], wy = S.w[1][oy][j], wz = S.w[2][oz][k];
        lv += l * wx * wy * wz;
        const T d = l * (vp - g[id]);
        gx += d * S.dw[0][ox][i] * wy * wz;
        gy += d * wx * S.dw[1][oy][j] * wz;
        gz += d * wx * wy * S.dw[2][oz][k];
      }
    }
  }
}
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_p2g(int64_t n, PartsT<T> A, const int16_t* tape, Geo G, double hd, const T* gu,
              const T* gv, const T* gw, const T* Wu, const T* Wv, const T* Ww, const T* lu,
              const T* lv, const T* lw, PartsT<T> L) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    StencilD<T> S;
    make_stencil_d(S, A.px[i], A.py[i], A.pz[i], h, tape ? tape + 6 * i : nullptr);
    T gx = T(0), gy = T(0), gz = T(0), l0 = T(0), l1 = T(0), l2 = T(0);
    adj_p2g_grid<T, 0>(S, A.vx[i], gu, Wu, lu, G, l0, gx, gy, gz);
    adj_p2g_grid<T, 1>(S, A.vy[i], gv, Wv, lv, G, l1, gx, gy, gz);
    adj_p2g_grid<T, 2>(S, A.vz[i], gw, Ww, lw, G, l2, gx, gy, gz);
    L.px[i] += gx;
    L.py[i] += gy;
    L.pz[i] += gz;
    L.vx[i] += l0;
    L.vy[i] += l1;
    L.vz[i] += l2;
  }
}

// advect: x' = x + c1 v unless clamped (then constant); v' = v unless zeroed.
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_advect(int64_t n, const uint16_t* __restrict__ flags, double dtd, PartsT<T> L) {
  const T c1 = rmul(T(2.0 / 9.0), (T)dtd);
  GRID_LOOP(i, n) {
    const uint16_t f = flags[i];
    T* lx[3] = {L.px, L.py, L.pz};
    T* lv[3] = {L.vx, L.vy, L.vz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const bool clamped = (f >> a) & 1, vz = (f >> (3 + a)) & 1;
      const T gx = lx[a][i], gv = lv[a][i];
      lx[a][i] = clamped ? T(0) : gx;
      lv[a][i] = (clamped ? T(0) : c1 * gx) + (vz ? T(0) : gv);
    }
  }
}

// Sum of the in-grid stencil weights of grid AX (sampleVelocity's normaliser).
template <class T, int AX>
__device__ __forceinline__ T stencil_weight(const StencilD<T>& S, const Geo& G) {
  constexpr int ox = AX == 0 ? 0 : 1, oy = AX == 1 ? 0 : 1, oz = AX == 2 ? 0 : 1;
  const int fx = G.fx(AX), fy = G.fy(AX), fz = G.fz(AX);
  T ws = T(0);
  for (int i = 0; i < 4; i++) {
    const int a = S.base[0][ox] + i;
    if (a < 0 || a >= fx) continue;
    for (int j = 0; j < 4; j++) {
      const int b = S.base[1][oy] + j;
      if (b < 0 || b >= fy) continue;
      for (int k = 0; k < 4; k++) {
        const int c = S.base[2][oz] + k;
        if (c < 0 || c >= fz) continue;
        ws += S.w[0][ox][i] * S.w[1][oy][j] * S.w[2][oz][k];
      }
    }
  }
  return ws;
}

// initial velocities v0 = S(x0; U): dL/dU += scatter of dL/dv0.
template <class T>
__global__ void __launch_bounds__(kT)
    k_adj_init(int64_t n, const T* px, const T* py, const T* pz, PartsT<T> L, Geo G, double hd, T* gu,
               T* gv, T* gw) {
  const T h = (T)hd;
  GRID_LOOP(i, n) {
    StencilD<T> S;
    make_stencil_d(S, px[i], py[i], pz[i], h, nullptr);
    scatter_sample<T, 0>(gu, S, G, stencil_weight<T, 0>(S, G), L.vx[i]);
    scatter_sample<T, 1>(gv, S, G, stencil_weight<T, 1>(S, G), L.vy[i]);
    scatter_sample<T, 2>(gw, S, G, stencil_weight<T, 2>(S, G), L.vz[i]);
  }
}

}  // namespace

// =================================================================================

void* DiffSim::alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  allocs_.push_back(p);
  cudaMemsetAsync(p, 0, bytes, ctx_->stream);
  return p;
}

int DiffSim::err(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ctx_->set_error(-2, std::string(where) + ": " + cudaGetErrorString(e));
  return 0;
}

DiffSim::DiffSim(Context* ctx, const DiffConfig& cfg) : ctx_(ctx), c_(cfg) {
  if (c_.nx < 1 || c_.ny < 1 || c_.nz < 1 || !(c_.h > 0) || !(c_.dt > 0) || c_.steps < 1 ||
      c_.checkpoint_every < 1) {
    status_ = -1;
    return;
  }
  rs_ = c_.f32 ? sizeof(float) : sizeof(double);
  N_ = (int64_t)c_.nx * c_.ny * c_.nz;
  fsz_[0] = (int64_t)(c_.nx + 1) * c_.ny * c_.nz;
  fsz_[1] = (int64_t)c_.nx * (c_.ny + 1) * c_.nz;
  fsz_[2] = (int64_t)c_.nx * c_.ny * (c_.nz + 1);
  nck_ = (c_.steps + c_.checkpoint_every - 1) / c_.checkpoint_every;
  bool ok = true;
  const int it = c_.vel_extrap_iters;
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) {
      ok &= (g_[a][b] = alloc(rs_ * fsz_[a])) != nullptr;
      ok &= (lg_[a][b] = alloc(rs_ * fsz_[a])) != nullptr;
    }
    ok &= (W_[a] = alloc(rs_ * fsz_[a])) != nullptr;
    ok &= (last_[a] = alloc(rs_ * fsz_[a])) != nullptr;
    ok &= (lul_[a] = alloc(rs_ * fsz_[a])) != nullptr;
    ok &= (mask_[a] = (uint8_t*)alloc((size_t)fsz_[a] * (it + 1))) != nullptr;
    ok &= (wt_[a] = (double*)alloc(sizeof(double) * fsz_[a])) != nullptr;
  }
  for (int b = 0; b < 2; b++) {
    ok &= (sdf_[b] = (double*)alloc(sizeof(double) * N_)) != nullptr;
    ok &= (sdfv_[b] = (uint8_t*)alloc(N_)) != nullptr;
  }
  ok &= (sdf_ck_ = (double*)alloc(sizeof(double) * N_ * 2 * (size_t)nck_)) != nullptr;
  ok &= (sdfv_ck_ = (uint8_t*)alloc((size_t)N_ * 2 * nck_)) != nullptr;
  ok &= (cnt_ = (int*)alloc(sizeof(int) * N_)) != nullptr;
  ok &= (start_ = (int*)alloc(sizeof(int) * N_)) != nullptr;
  ok &= (cursor_ = (int*)alloc(sizeof(int) * N_)) != nullptr;
  ok &= (bsum_ = (int*)alloc(sizeof(int) * ((N_ + 1023) / 1024 + 1))) != nullptr;
  ok &= (rho_ = (double*)alloc(sizeof(double) * N_)) != nullptr;
  ok &= (target_ = (double*)alloc(sizeof(double) * N_)) != nullptr;
  ok &= (red_ = (double*)alloc(sizeof(double) * 4)) != nullptr;
  ok &= (p2g_scr_ = alloc(p2g_scratch_bytes(Geo{c_.nx, c_.ny, c_.nz}, rs_))) != nullptr;
  if (ok && cudaMallocHost(&host_red_, sizeof(double) * 4) != cudaSuccess) ok = false;
  scur_ck_.assign(nck_, 0);
  svcur_ck_.assign(nck_, 0);
  if (!ok) {
    status_ = -3;
    return;
  }
  pcg_ = new PcgSolver(ctx, c_.nx, c_.ny, c_.nz, c_.pcg);
  if (pcg_->status()) {
    status_ = pcg_->status();
    return;
  }
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) status_ = -2;
}

DiffSim::~DiffSim() {
  cudaStreamSynchronize(ctx_->stream);
  delete pcg_;
  if (host_red_) cudaFreeHost(host_red_);
  for (void* p : allocs_) cudaFree(p);
}

int DiffSim::set_particles(int64_t n, const double* pos, bool device) {
  if (n < 1) return ctx_->set_error(-1, "the differentiable step needs particles");
  if (n_ != 0) return ctx_->set_error(-1, "particles are already set");
  cudaStream_t st = ctx_->stream;
  const size_t P = (size_t)n;
  const int K = c_.checkpoint_every;
  bool ok = true;
  ok &= (x0_ = alloc(rs_ * 3 * P)) != nullptr;
  ok &= (ids0_ = (int64_t*)alloc(sizeof(int64_t) * P)) != nullptr;
  ok &= (sid_ = (int64_t*)alloc(sizeof(int64_t) * P)) != nullptr;
  ok &= (key_ = (int*)alloc(sizeof(int) * P)) != nullptr;
  ok &= (ck_ = alloc(rs_ * 6 * P * (size_t)nck_)) != nullptr;
  ok &= (seg_ = alloc(rs_ * 6 * P * (size_t)(K + 1))) != nullptr;
  ok &= (cur_[0] = alloc(rs_ * 6 * P)) != nullptr;
  ok &= (cur_[1] = alloc(rs_ * 6 * P)) != nullptr;
  ok &= (fin_ = alloc(rs_ * 6 * P)) != nullptr;
  ok &= (xa_ = alloc(rs_ * 6 * P)) != nullptr;
  ok &= (srt_ = alloc(rs_ * 6 * P)) != nullptr;
  ok &= (flags_ = (uint16_t*)alloc(sizeof(uint16_t) * P)) != nullptr;
  ok &= (lx_ = alloc(rs_ * 6 * P)) != nullptr;
  if (!ok) return ctx_->set_error(-3, "particle allocation failed");
  lv_ = nullptr;
  n_ = n;
  double* stage = nullptr;
  const double* dp = pos;
  if (!device) {
    if (cudaMallocAsync(&stage, sizeof(double) * 3 * P, st) != cudaSuccess)
      return ctx_->set_error(-3, "staging allocation failed");
    cudaMemcpyAsync(stage, pos, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, st);
    dp = stage;
  }
  if (c_.f32) {
    float* x = (float*)x0_;
    k_aos_to_soa<float><<<nblk(n), kT, 0, st>>>(
        n, dp, nullptr, PartsT<float>{x, x + P, x + 2 * P, (float*)cur_[0] + 3 * P, (float*)cur_[0] + 4 * P,
                                      (float*)cur_[0] + 5 * P},
        ids0_);
  } else {
    double* x = (double*)x0_;
    k_aos_to_soa<double><<<nblk(n), kT, 0, st>>>(
        n, dp, nullptr, PartsT<double>{x, x + P, x + 2 * P, (double*)cur_[0] + 3 * P, (double*)cur_[0] + 4 * P,
                                       (double*)cur_[0] + 5 * P},
        ids0_);
  }
  if (stage) cudaFreeAsync(stage, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("set_particles");
  return err("set_particles");
}

int DiffSim::set_target(const double* rho, bool device) {
  cudaMemcpyAsync(target_, rho, sizeof(double) * N_, device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                  ctx_->stream);
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return err("set_target");
  return err("set_target");
}

void DiffSim::save_sdf(int slot) {
  cudaStream_t st = ctx_->stream;
  for (int b = 0; b < 2; b++) {
    cudaMemcpyAsync(sdf_ck_ + ((size_t)slot * 2 + b) * N_, sdf_[b], sizeof(double) * N_, cudaMemcpyDeviceToDevice,
                    st);
    cudaMemcpyAsync(sdfv_ck_ + ((size_t)slot * 2 + b) * N_, sdfv_[b], N_, cudaMemcpyDeviceToDevice, st);
  }
  scur_ck_[slot] = scur_;
  svcur_ck_[slot] = svcur_;
}

void DiffSim::load_sdf(int slot) {
  cudaStream_t st = ctx_->stream;
  for (int b = 0; b < 2; b++) {
    cudaMemcpyAsync(sdf_[b], sdf_ck_ + ((size_t)slot * 2 + b) * N_, sizeof(double) * N_, cudaMemcpyDeviceToDevice,
                    st);
    cudaMemcpyAsync(sdfv_[b], sdfv_ck_ + ((size_t)slot * 2 + b) * N_, N_, cudaMemcpyDeviceToDevice, st);
  }
  scur_ = scur_ck_[slot];
  svcur_ = svcur_ck_[slot];
}

// One substep from state `in` to state `out`.  mode TAPE_REPLAY takes the
// clamps, bases and fluid SDF of substep t from the record; `sdf_in`
// (non-null) supplies the fluid SDF instead of reconstructing it; `sdf_out`
// (non-null) receives the fluid SDF used.
template <class T>
int DiffSim::step_t(int t, int mode, const void* in, void* out) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  const double h = c_.h, dt = c_.dt;
  const int64_t n = n_, N = N_;
  const int it = c_.vel_extrap_iters;
  PartsT<T> I = parts_of<T>(in, n), O = parts_of<T>(out, n), A = parts_of<T>(xa_, n), S = parts_of<T>(srt_, n);
  const int16_t* tb = mode == TAPE_REPLAY ? tape_bases_ + (size_t)t * 6 * n : nullptr;
  // clear() (fluid-simulator.cc:20-37)
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) cudaMemsetAsync(g_[a][b], 0, rs_ * fsz_[a], st);
    cudaMemsetAsync(W_[a], 0, rs_ * fsz_[a], st);
    cudaMemsetAsync(mask_[a], 0, (size_t)fsz_[a] * (it + 1), st);
  }
  k_diff_advect<T><<<nblk(n), kT, 0, st>>>(n, I, A, flags_,
                                          mode == TAPE_REPLAY ? tape_flags_ + (size_t)t * n : nullptr,
                                          mode == TAPE_RECORD ? tape_flags_ + (size_t)t * n : nullptr, G, h, dt);
  if (mode == TAPE_RECORD)
    k_record_bases<T><<<nblk(n), kT, 0, st>>>(n, A.px, A.py, A.pz, h, tape_bases_ + (size_t)t * 6 * n);
  SortBufs sb{key_, cnt_, start_, cursor_, bsum_};
  launches_ += 3 + sort_particles<T>(st, n, G, h, A, ids0_, S, sid_, sb);
  // fluid SDF
  if (mode == TAPE_REPLAY || seg_sdf_in_) {
    const double* src = mode == TAPE_REPLAY ? tape_sdf_ + (size_t)t * N : seg_sdf_in_;
    cudaMemcpyAsync(sdf_[scur_], src, sizeof(double) * N, cudaMemcpyDeviceToDevice, st);
  } else {
    if (launch_reconstruct<T>(st, G, h, c_.recon_factor * h, start_, cnt_, S.px, S.py, S.pz, sdf_[scur_],
                              sdfv_[svcur_]))
      return ctx_->set_error(-1, "reconstruct: radius reaches past 6 cells");
    launches_ += 1 + launch_iter_cells<ITER_SDF>(st, G, c_.sdf_extrap_iters, sdf_, sdfv_, scur_, svcur_);
    for (int k = 0; k < c_.smooth_iters; k++) {
      k_smooth_sdf<<<nblk(N), kT, 0, st>>>(G, sdf_[scur_], sdf_[1 - scur_]);
      scur_ = 1 - scur_;
    }
    launches_ += c_.smooth_iters;
    if (mode == TAPE_RECORD)
      cudaMemcpyAsync(tape_sdf_ + (size_t)t * N, sdf_[scur_], sizeof(double) * N, cudaMemcpyDeviceToDevice, st);
  }
  if (seg_sdf_out_) cudaMemcpyAsync(seg_sdf_out_, sdf_[scur_], sizeof(double) * N, cudaMemcpyDeviceToDevice, st);
  const double* fluid = sdf_[scur_];
  // P2G, Dirichlet, extrapolation, gravity
  for (int a = 0; a < 3; a++) gstart_[a] = gcur_[a];
  launches_ += launch_p2g<T>(st, G, h, start_, cnt_, S, p2g_scratch_at(p2g_scr_, G, rs_), (T*)g_[0][gcur_[0]],
                             (T*)g_[1][gcur_[1]],
                             (T*)g_[2][gcur_[2]], (T*)W_[0], (T*)W_[1], (T*)W_[2], mask_[0], mask_[1], mask_[2],
                             (T*)last_[0], (T*)last_[1], (T*)last_[2], tb, sid_);
  k_dirichlet<T, 0><<<nblk(fsz_[0]), kT, 0, st>>>(G, (T*)g_[0][gcur_[0]], mask_[0]);
  k_dirichlet<T, 1><<<nblk(fsz_[1]), kT, 0, st>>>(G, (T*)g_[1][gcur_[1]], mask_[1]);
  k_dirichlet<T, 2><<<nblk(fsz_[2]), kT, 0, st>>>(G, (T*)g_[2][gcur_[2]], mask_[2]);
  // extrapolation, temporally blocked, each pass's flags kept for the adjoint
  {
    T* const fb[3][2] = {{(T*)g_[0][0], (T*)g_[0][1]}, {(T*)g_[1][0], (T*)g_[1][1]}, {(T*)g_[2][0], (T*)g_[2][1]}};
    launches_ += launch_extrap_faces<T>(st, G, it, fb, nullptr, mask_, fsz_, gcur_);
  }
  k_force<T><<<nblk(fsz_[1]), kT, 0, st>>>(G, (T*)g_[1][gcur_[1]], mask_[1] + (size_t)it * fsz_[1], c_.gravity * dt);
  launches_ += 4;
  // buildSystem, solve, project, walls
  SystemOut so;
  so.g = pcg_->geom();
  so.t_adiag = pcg_->adiag64();
  so.t_al = pcg_->al64();
  so.t_ad = pcg_->ad64();
  so.t_ab = pcg_->ab64();
  so.t_rhs = pcg_->rhs64();
  so.t_active = pcg_->active();
  T* gu = (T*)g_[0][gcur_[0]];
  T* gv = (T*)g_[1][gcur_[1]];
  T* gw = (T*)g_[2][gcur_[2]];
  if (fvm_build_system<T>(st, c_.nx, c_.ny, c_.nz, h, dt, gu, gv, gw, fluid, nullptr, wt_[0], wt_[1], wt_[2], so))
    return err("buildSystem");
  pcg_->mark_system_changed();
  PcgStats ps;
  int e = pcg_->solve(&ps);
  if (e) return e;
  last_iters_ = ps.iterations;
  launches_ += 4 + ps.kernel_launches;
  const Tiled tg = pcg_->geom();
  if (fvm_project<T>(st, c_.nx, c_.ny, c_.nz, h, dt, gu, gv, gw, pcg_->pressure64(), &tg, fluid, wt_[0], wt_[1],
                     wt_[2]))
    return err("project");
  launch_collider<T>(st, G, h, gu, gv, gw, nullptr);
  // G2P into out
  cudaMemcpyAsync(out, xa_, rs_ * 6 * (size_t)n, cudaMemcpyDeviceToDevice, st);
  k_g2p<T><<<nblk(n), kT, 0, st>>>(n, O, gu, gv, gw, (T*)last_[0], (T*)last_[1], (T*)last_[2], G, h,
                                   c_.flip ? c_.flip_alpha : -1.0, tb);
  launches_ += 7;
  return err("substep");
}

// Adjoint of the substep just run by step_t: (lx, lv) hold d/d(out state) on
// entry and d/d(in state) on exit.
template <class T>
int DiffSim::adjoint_step_t(int t, void* lxv, void*) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  const double h = c_.h, dt = c_.dt;
  const int64_t n = n_;
  const int it = c_.vel_extrap_iters;
  PartsT<T> A = parts_of<T>(xa_, n), L = parts_of<T>(lxv, n);
  const int16_t* tb = last_mode_ == TAPE_REPLAY ? tape_bases_ + (size_t)t * 6 * n : nullptr;
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) cudaMemsetAsync(lg_[a][b], 0, rs_ * fsz_[a], st);
    cudaMemsetAsync(lul_[a], 0, rs_ * fsz_[a], st);
  }
  const int fin[3] = {gcur_[0], gcur_[1], gcur_[2]};
  T* lu[3] = {(T*)lg_[0][fin[0]], (T*)lg_[1][fin[1]], (T*)lg_[2][fin[2]]};
  // G2P
  k_adj_g2p<T><<<nblk(n), kT, 0, st>>>(n, A, (const T*)g_[0][fin[0]], (const T*)g_[1][fin[1]],
                                       (const T*)g_[2][fin[2]], (const T*)last_[0], (const T*)last_[1],
                                       (const T*)last_[2], tb, G, h, c_.flip ? c_.flip_alpha : -1.0, L, lu[0],
                                       lu[1], lu[2], (T*)lul_[0], (T*)lul_[1], (T*)lul_[2]);
  // applyCollider (walls), then project: d/dp into the solver's rhs
  k_adj_walls<T, 0><<<nblk(fsz_[0]), kT, 0, st>>>(G, lu[0]);
  k_adj_walls<T, 1><<<nblk(fsz_[1]), kT, 0, st>>>(G, lu[1]);
  k_adj_walls<T, 2><<<nblk(fsz_[2]), kT, 0, st>>>(G, lu[2]);
  const Tiled tg = pcg_->geom();
  cudaMemsetAsync(pcg_->rhs64(), 0, sizeof(double) * (size_t)tg.total, st);
  k_adj_project<T><<<nblk(N_), kT, 0, st>>>(G, h, dt, tg, pcg_->active(), sdf_[scur_], wt_[0], wt_[1], wt_[2],
                                            lu[0], lu[1], lu[2], pcg_->rhs64());
  // the pressure solve is self-adjoint: mu = A^-1 d/dp
  PcgStats ps;
  int e = pcg_->solve(&ps);
  if (e) return e;
  launches_ += 5 + ps.kernel_launches;
  k_adj_rhs<T, 0><<<nblk(fsz_[0]), kT, 0, st>>>(G, tg, pcg_->pressure64(), wt_[0], lu[0]);
  k_adj_rhs<T, 1><<<nblk(fsz_[1]), kT, 0, st>>>(G, tg, pcg_->pressure64(), wt_[1], lu[1]);
  k_adj_rhs<T, 2><<<nblk(fsz_[2]), kT, 0, st>>>(G, tg, pcg_->pressure64(), wt_[2], lu[2]);
  // gravity adds a constant; extrapolation iterations in reverse
  for (int k = it - 1; k >= 0; k--) {
    for (int a = 0; a < 3; a++) {
      const int s = (k % 2 == 0) ? gstart_[a] : 1 - gstart_[a], d = 1 - s;
      const uint8_t* vs = mask_[a] + (size_t)k * fsz_[a];
      if (a == 0) k_adj_extrap_src<T, 0><<<nblk(fsz_[0]), kT, 0, st>>>(G, (T*)lg_[0][s], (const T*)lg_[0][d], vs);
      if (a == 1) k_adj_extrap_src<T, 1><<<nblk(fsz_[1]), kT, 0, st>>>(G, (T*)lg_[1][s], (const T*)lg_[1][d], vs);
      if (a == 2) k_adj_extrap_src<T, 2><<<nblk(fsz_[2]), kT, 0, st>>>(G, (T*)lg_[2][s], (const T*)lg_[2][d], vs);
      k_adj_extrap_dst<T><<<nblk(fsz_[a]), kT, 0, st>>>(fsz_[a], (T*)lg_[a][d], vs);
    }
  }
  // Dirichlet and u_last, then P2G, then advect
  T* lp[3] = {(T*)lg_[0][gstart_[0]], (T*)lg_[1][gstart_[1]], (T*)lg_[2][gstart_[2]]};
  k_adj_dirichlet<T, 0><<<nblk(fsz_[0]), kT, 0, st>>>(G, lp[0], (const T*)lul_[0]);
  k_adj_dirichlet<T, 1><<<nblk(fsz_[1]), kT, 0, st>>>(G, lp[1], (const T*)lul_[1]);
  k_adj_dirichlet<T, 2><<<nblk(fsz_[2]), kT, 0, st>>>(G, lp[2], (const T*)lul_[2]);
  k_adj_p2g<T><<<nblk(n), kT, 0, st>>>(n, A, tb, G, h, (const T*)last_[0], (const T*)last_[1], (const T*)last_[2],
                                       (const T*)W_[0], (const T*)W_[1], (const T*)W_[2], lp[0], lp[1], lp[2], L);
  k_adj_advect<T><<<nblk(n), kT, 0, st>>>(n, flags_, dt, L);
  launches_ += 12 + 6 * it;
  return err("adjoint substep");
}

template <class T>
int DiffSim::forward_t(const double* const U[3], int mode, double* loss) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  const int64_t n = n_;
  const size_t P = (size_t)n;
  if (mode == TAPE_RECORD && !have_tape_) {
    tape_sdf_ = (double*)alloc(sizeof(double) * N_ * (size_t)c_.steps);
    tape_flags_ = (uint16_t*)alloc(sizeof(uint16_t) * P * (size_t)c_.steps);
    tape_bases_ = (int16_t*)alloc(sizeof(int16_t) * 6 * P * (size_t)c_.steps);
    tape_final_ = (int16_t*)alloc(sizeof(int16_t) * 6 * P);
    if (!tape_sdf_ || !tape_flags_ || !tape_bases_ || !tape_final_)
      return ctx_->set_error(-3, "record allocation failed");
  }
  if (mode == TAPE_REPLAY && !have_tape_) return ctx_->set_error(-1, "no recorded run to replay");
  // initial state: x0 and v0 = S(x0; U)
  for (int a = 0; a < 3; a++)
    k_cast<double, T><<<nblk(fsz_[a]), kT, 0, st>>>(fsz_[a], U[a], (T*)g_[a][0]);
  T* x0 = (T*)x0_;
  T* s0 = (T*)cur_[0];
  cudaMemcpyAsync(s0, x0, rs_ * 3 * P, cudaMemcpyDeviceToDevice, st);
  k_sample_into<T><<<nblk(n), kT, 0, st>>>(n, x0, x0 + P, x0 + 2 * P, (T*)g_[0][0], (T*)g_[1][0], (T*)g_[2][0], G,
                                           c_.h, s0 + 3 * P, s0 + 4 * P, s0 + 5 * P);
  // the simulator starts with zeroed SDF buffers
  for (int b = 0; b < 2; b++) {
    cudaMemsetAsync(sdf_[b], 0, sizeof(double) * N_, st);
    cudaMemsetAsync(sdfv_[b], 0, N_, st);
  }
  scur_ = svcur_ = 0;
  gcur_[0] = gcur_[1] = gcur_[2] = 0;
  seg_sdf_in_ = seg_sdf_out_ = nullptr;
  int a = 0, b = 1;
  for (int t = 0; t < c_.steps; t++) {
    if (t % c_.checkpoint_every == 0) {
      const int slot = t / c_.checkpoint_every;
      cudaMemcpyAsync((char*)ck_ + rs_ * 6 * P * slot, cur_[a], rs_ * 6 * P, cudaMemcpyDeviceToDevice, st);
      save_sdf(slot);
    }
    int e = step_t<T>(t, mode, cur_[a], cur_[b]);
    if (e) return e;
    std::swap(a, b);
  }
  cudaMemcpyAsync(fin_, cur_[a], rs_ * 6 * P, cudaMemcpyDeviceToDevice, st);
  // density and loss
  T* xf = (T*)fin_;
  cudaMemsetAsync(rho_, 0, sizeof(double) * N_, st);
  k_density<T><<<nblk(n), kT, 0, st>>>(n, xf, xf + P, xf + 2 * P, mode == TAPE_REPLAY ? tape_final_ : nullptr,
                                       mode == TAPE_RECORD ? tape_final_ : nullptr, G, c_.h, rho_);
  cudaMemsetAsync(red_, 0, sizeof(double), st);
  k_loss<<<nblk(N_), kT, 0, st>>>(N_, rho_, target_, red_);
  cudaMemcpyAsync(host_red_, red_, sizeof(double), cudaMemcpyDeviceToHost, st);
  launches_ += 7;
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("forward");
  if (mode == TAPE_RECORD) have_tape_ = true;
  last_mode_ = mode;
  have_forward_ = true;
  *loss = host_red_[0];
  return err("forward");
}

template <class T>
int DiffSim::backward_t(double* const gU[3]) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  const int64_t n = n_;
  const size_t P = (size_t)n;
  const int K = c_.checkpoint_every;
  const int mode = last_mode_ == TAPE_REPLAY ? TAPE_REPLAY : TAPE_NONE;
  if (!seg_sdf_) {
    seg_sdf_ = (double*)alloc(sizeof(double) * N_ * (size_t)K);
    if (!seg_sdf_) return ctx_->set_error(-3, "segment allocation failed");
  }
  // d loss / d x_final
  T* xf = (T*)fin_;
  k_adj_density<T><<<nblk(n), kT, 0, st>>>(n, parts_of<T>(fin_, n), last_mode_ == TAPE_REPLAY ? tape_final_ : nullptr,
                                           G, c_.h, rho_, target_, parts_of<T>(lx_, n));
  (void)xf;
  for (int s = nck_ - 1; s >= 0; s--) {
    const int t0 = s * K, t1 = std::min(t0 + K, c_.steps);
    // recompute the segment's states and the fluid SDF each substep used
    load_sdf(s);
    gcur_[0] = gcur_[1] = gcur_[2] = (t0 * c_.vel_extrap_iters) & 1;
    cudaMemcpyAsync(seg_, (char*)ck_ + rs_ * 6 * P * s, rs_ * 6 * P, cudaMemcpyDeviceToDevice, st);
    for (int t = t0; t < t1; t++) {
      seg_sdf_in_ = nullptr;
      seg_sdf_out_ = seg_sdf_ + (size_t)(t - t0) * N_;
      int e = step_t<T>(t, mode, (char*)seg_ + rs_ * 6 * P * (t - t0), (char*)seg_ + rs_ * 6 * P * (t - t0 + 1));
      if (e) return e;
    }
    // adjoint substeps in reverse, each after re-running its forward
    for (int t = t1 - 1; t >= t0; t--) {
      seg_sdf_in_ = seg_sdf_ + (size_t)(t - t0) * N_;
      seg_sdf_out_ = nullptr;
      gcur_[0] = gcur_[1] = gcur_[2] = (t * c_.vel_extrap_iters) & 1;
      int e = step_t<T>(t, mode, (char*)seg_ + rs_ * 6 * P * (t - t0), cur_[0]);
      if (e) return e;
      e = adjoint_step_t<T>(t, lx_, nullptr);
      if (e) return e;
    }
  }
  seg_sdf_in_ = seg_sdf_out_ = nullptr;
  // v0 = S(x0; U)
  for (int a = 0; a < 3; a++) cudaMemsetAsync(lg_[a][0], 0, rs_ * fsz_[a], st);
  T* x0 = (T*)x0_;
  k_adj_init<T><<<nblk(n), kT, 0, st>>>(n, x0, x0 + P, x0 + 2 * P, parts_of<T>(lx_, n), G, c_.h, (T*)lg_[0][0],
                                        (T*)lg_[1][0], (T*)lg_[2][0]);
  for (int a = 0; a < 3; a++)
    k_cast<T, double><<<nblk(fsz_[a]), kT, 0, st>>>(fsz_[a], (const T*)lg_[a][0], gU[a]);
  launches_ += 5;
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("backward");
  return err("backward");
}

int DiffSim::forward(const double* const U[3], int tape, double* loss) {
  if (n_ < 1) return ctx_->set_error(-1, "no particles");
  return c_.f32 ? forward_t<float>(U, tape, loss) : forward_t<double>(U, tape, loss);
}

int DiffSim::backward(double* const gU[3]) {
  if (!have_forward_) return ctx_->set_error(-1, "backward needs a forward first");
  return c_.f32 ? backward_t<float>(gU) : backward_t<double>(gU);
}

int DiffSim::get_density(double* rho, bool device) {
  cudaMemcpyAsync(rho, rho_, sizeof(double) * N_, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                  ctx_->stream);
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return err("get_density");
  return err("get_density");
}

int DiffSim::get_pressure(double* p, bool device) {
  if (!have_forward_) return ctx_->set_error(-1, "get_pressure needs a forward first");
  return pcg_->download_pressure(p, device);
}

int DiffSim::get_particles(double* pos, double* vel, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t n = n_;
  double* stage = nullptr;
  double *dp = pos, *dv = vel;
  if (!device) {
    if (cudaMallocAsync(&stage, sizeof(double) * 6 * (size_t)n, st) != cudaSuccess)
      return ctx_->set_error(-3, "staging allocation failed");
    dp = pos ? stage : nullptr;
    dv = vel ? stage + 3 * n : nullptr;
  }
  if (c_.f32)
    k_soa_to_aos<float><<<nblk(n), kT, 0, st>>>(n, parts_of<float>(fin_, n), nullptr, dp, dv);
  else
    k_soa_to_aos<double><<<nblk(n), kT, 0, st>>>(n, parts_of<double>(fin_, n), nullptr, dp, dv);
  if (!device) {
    if (pos) cudaMemcpyAsync(pos, stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (vel) cudaMemcpyAsync(vel, stage + 3 * n, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(stage, st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("get_particles");
  return err("get_particles");
}

}  // namespace sc
