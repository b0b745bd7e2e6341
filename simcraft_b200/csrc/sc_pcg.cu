// sc_pcg.cu -- MIC(0)-PCG pressure solver on B200 (sm_100a).
//
// Restates, on the GPU, the reference's CgSolver3D::solve
// (FluidSim/src/cpu/project-solver.cc:308-346), applyCompressedMatrix (:16-39),
// ModifiedIncompleteCholesky3D::precond (:230-306) and the masked BLAS-1 of
// FluidSim/src/cpu/util.cc:380-410.  The preconditioner's arithmetic is the
// reference's own (its non-standard pivot recurrence included); only the
// evaluation order changes: the lexicographic sweeps become i+j+k wavefronts.
//
// Structure of one PCG iteration (all kernels read their scalars from device
// memory, so a chunk of iterations is captured once as a CUDA graph):
//   k_spmv   Az = A s, partial s.Az          -> alpha      (project-solver.cc:328-331)
//   k_axpy   p += alpha s, r -= alpha Az     -> residual   (:332-335)
//   k_wave   forward sweep  q = K^-1 r                     (:276-288)
//   k_wave   backward sweep z = K^-T q, z.r -> beta        (:293-305, :338-341)
//   k_sa     s = z + beta s                  -> iter++     (:342, util.cc:404-410)
// The MIC(0) pivots E = 1/sqrt(e) are computed once per solve by a wavefront
// kernel; the reference recomputes them on every call with identical values.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include <mutex>
#include <string>

#include <cooperative_groups.h>

#include "sc_pcg.cuh"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kRing = 32;     // boundary ring entries per wavefront CTA
// Nanoseconds a waiting warp of a sweep (the control warp, the mailbox
// loaders) sleeps between two polls that found nothing (0: back to back).
// 16 took ~1.5% off the 128^3 mixed solve (A/B of two builds, two runs each:
// 40.4 -> 39.8 ms); the spinning warps were taking issue slots from the row
// warps of the same SM.
#ifndef SC_WAVE_CTL_NS
#define SC_WAVE_CTL_NS 16
#endif
// 1: the iterations sweep only the tiles holding an active cell; 0: every tile
#ifndef SC_SKIP_EMPTY_TILES
#define SC_SKIP_EMPTY_TILES 1
#endif
#ifndef SC_WAVE_STAGE_MAX
#define SC_WAVE_STAGE_MAX 8
#endif
// Bytes per cp.async chunk of the staged sweep input (4, 8 or 16); 8 measured
// best for both precisions at 128^3 and 512^3 (16 costs FP64 sweeps ~4%).
#ifndef SC_WAVE_CHUNK64
#define SC_WAVE_CHUNK64 8
#endif
#ifndef SC_WAVE_CHUNK32
#define SC_WAVE_CHUNK32 8
#endif
// Ring slots of staged sweep input (steps in flight per compute warp): as many
// as fit in ~180 KB of shared memory, at most SC_WAVE_STAGE_MAX.
template <class T, int NV>
constexpr int wave_stages() {
  constexpr int fit = (int)(180 * 1024 / ((size_t)Tiled::TY * NV * 32 * sizeof(T)));
  return fit < SC_WAVE_STAGE_MAX ? fit : SC_WAVE_STAGE_MAX;
}
constexpr int kSpinLimit = 1 << 22;  // default bound of the waits: ~0.1-1 s, far above any legitimate wait

enum { FIN_NONE = 0, FIN_INIT, FIN_SPMV, FIN_AXPY, FIN_BWD, FIN_SA, FIN_NORMS, FIN_EINIT, FIN_EAXPY, FIN_EREPLACE };

__device__ void finalize(int kind, PcgScalars* sc, double sum, double mx) {
  switch (kind) {
    case FIN_INIT: {  // r = rhs; residual check before the first preconditioner (:313-319)
      sc->rn2 = sum;
      sc->rinf = mx;
      sc->bnorm = sqrt(sum);
      double res = sc->criterion == CRIT_REL_L2 ? (sc->bnorm > 0.0 ? 1.0 : 0.0) : mx;
      sc->res = res;
      sc->first = 1;
      if (!isfinite(sum) || !(res == res)) {  // NaN/Inf in the right-hand side
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
        sc->iter = 0;
      } else if (res < sc->tol) {
        sc->done = DONE_CONVERGED;
        sc->iter = 0;
      } else {
        sc->done = DONE_RUNNING;
        sc->iter = 1;
      }
      break;
    }
    case FIN_SPMV: {  // alpha = sigma / (s . z)  (:329-331)
      sc->sdotz = sum;
      if (sum == 0.0 || !isfinite(sum)) {
        sc->err |= (sum == 0.0) ? DEV_ERR_BREAKDOWN : DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      } else {
        sc->alpha = sc->sigma / sum;
      }
      break;
    }
    case FIN_AXPY: {  // residual = LinfNorm(r) (or relative L2); break when < tol (:334-335)
      sc->rn2 = sum;
      sc->rinf = mx;
      double res = sc->criterion == CRIT_REL_L2 ? (sc->bnorm > 0.0 ? sqrt(sum) / sc->bnorm : 0.0)
                                                : mx;
      sc->res = res;
      if (!isfinite(res)) {
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      } else if (res < sc->tol) {
        sc->done = DONE_CONVERGED;
      }
      break;
    }
    case FIN_BWD: {  // sigma_new = z . r ; beta = sigma_new / sigma (:338-341)
      if (sc->first) {
        sc->sigma = sum;
        sc->first = 0;
      } else {
        sc->beta = sum / sc->sigma;
        sc->sigma = sum;
      }
      if (!isfinite(sum)) {
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      }
      break;
    }
    case FIN_SA: {  // for-loop increment and bound (:327)
      sc->iter += 1;
      if (sc->iter >= sc->max_iter) sc->done = DONE_MAXITER;
      break;
    }
    case FIN_NORMS: {
      sc->rn2 = sum;
      sc->rinf = mx;
      break;
    }
    // Eisenstat iteration (FP32 inner solve): the residual of the split system is
    // rh = L^-1 r, rho = rh.rh = r.M^-1 r plays sigma's part and the stopping
    // measure is ||rh|| / ||rh_0||.
    case FIN_EINIT: {  // rho_0 = rh_0.rh_0 ; the first search direction is rh_0 (beta = 0)
      sc->sigma = sum;
      sc->beta = 0.0;
      sc->bnorm = sqrt(sum);
      sc->first = 0;
      if (!isfinite(sum)) {
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      } else if (sum == 0.0 && sc->done == DONE_RUNNING) {
        sc->done = DONE_CONVERGED;
        sc->iter = 0;
      }
      break;
    }
    case FIN_EREPLACE: {  // rh replaced by L^-1 of the FP64 residual: rho = rh.rh
      sc->sigma = sum;
      sc->res = sc->bnorm > 0.0 ? sqrt(sum) / sc->bnorm : 0.0;
      if (!isfinite(sum)) {
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      }
      break;
    }
    case FIN_EAXPY: {  // rho_new; convergence; beta = rho_new / rho
      sc->rn2 = sum;
      sc->rinf = mx;
      const double res = sc->bnorm > 0.0 ? sqrt(sum) / sc->bnorm : 0.0;
      sc->res = res;
      if (!isfinite(res)) {
        sc->err |= DEV_ERR_NONFINITE;
        sc->done = DONE_BREAKDOWN;
      } else if (res < sc->tol) {
        sc->done = DONE_CONVERGED;
      }
      sc->beta = sum / sc->sigma;
      sc->sigma = sum;
      break;
    }
    default:
      break;
  }
}

// Block reduce (sum, max) -> per-block partial -> last block reduces the
// partials in fixed order (deterministic) and runs the finalizer.
__device__ void reduce_finalize(double sum, double mx, double* partials, PcgScalars* sc,
                                int kind) {
  __shared__ double ss[32], sm[32];
  __shared__ bool last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  sum = warp_sum(sum);
  mx = warp_max(mx);
  if (l == 0) {
    ss[w] = sum;
    sm[w] = mx;
  }
  __syncthreads();
  if (w == 0) {
    sum = l < nw ? ss[l] : 0.0;
    mx = l < nw ? sm[l] : 0.0;
    sum = warp_sum(sum);
    mx = warp_max(mx);
    if (l == 0) {
      partials[2 * blockIdx.x] = sum;
      partials[2 * blockIdx.x + 1] = mx;
      __threadfence();
      unsigned prev = atomicAdd(&sc->count, 1u);
      last = (prev == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double s2 = 0.0, m2 = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
      s2 += __ldcg(&partials[2 * b]);
      m2 = fmax(m2, __ldcg(&partials[2 * b + 1]));
    }
    s2 = warp_sum(s2);
    m2 = warp_max(m2);
    __syncthreads();
    if (l == 0) {
      ss[w] = s2;
      sm[w] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double S = 0.0, M = 0.0;
      for (int i = 0; i < nw; i++) {
        S += ss[i];
        M = fmax(M, sm[i]);
      }
      sc->count = 0;
      finalize(kind, sc, S, M);
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------------------------
// Layout conversion (reference layout <-> tiled).  Row-block kernels: one
// 256-thread block owns the TY*32 elements of one (tile, slot) row block.
#define SC_ROWBLOCK_LOOP(g) \
  for (int rb = blockIdx.x, nrb_ = (g).ntiles() * (g).nz; rb < nrb_; rb += gridDim.x)

template <class Ts, class Td>
__global__ void __launch_bounds__(kThreads) k_to_tiled(Tiled g, const Ts* __restrict__ src,
                                                       Td* __restrict__ dst,
                                                       const uint8_t* __restrict__ mask_ref) {
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    Td v = Td(0);
    if (c.inside) {
      const int64_t r = lin(c.x, c.y, c.z, g.ny, g.nz);
      if (!mask_ref || mask_ref[r]) v = (Td)src[r];
    }
    dst[c.e] = v;
  }
}
template <class Ts, class Td>
__global__ void __launch_bounds__(kThreads) k_from_tiled(Tiled g, const Ts* __restrict__ src,
                                                         Td* __restrict__ dst) {
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    if (c.inside) dst[lin(c.x, c.y, c.z, g.ny, g.nz)] = (Td)src[c.e];
  }
}
template <class Ts, class Td>
__global__ void k_convert(int64_t n, const Ts* __restrict__ src, Td* __restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    dst[e] = (Td)src[e];
}
template <class T>
__global__ void k_fill(int64_t n, T* __restrict__ dst, T v) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) dst[e] = v;
}

// max |A_Right(p) - A_Left(p+x)| (and Up/Down, Front/Back) over active pairs,
// the relation checkSystemSymmetry asserts (project-solver.cc:41-57).
__global__ void k_symmetry(int nx, int ny, int nz, const double* const* an,
                           const uint8_t* act, double* partials, PcgScalars* sc) {
  double mx = 0.0;
  const int64_t N = (int64_t)nx * ny * nz;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < N; id += stride) {
    if (!act[id]) continue;
    int k = (int)(id % nz);
    int j = (int)((id / nz) % ny);
    int i = (int)(id / ((int64_t)ny * nz));
    if (i < nx - 1 && act[id + (int64_t)ny * nz])
      mx = fmax(mx, fabs(an[1][id] - an[0][id + (int64_t)ny * nz]));
    if (j < ny - 1 && act[id + nz]) mx = fmax(mx, fabs(an[2][id] - an[3][id + nz]));
    if (k < nz - 1 && act[id + 1]) mx = fmax(mx, fabs(an[4][id] - an[5][id + 1]));
  }
  reduce_finalize(0.0, mx, partials, sc, FIN_NORMS);
}

// ---------------------------------------------------------------------------------
// Elementwise PCG kernels (tiled layout).
template <class T>
__global__ void __launch_bounds__(kThreads) k_init(Tiled g, const double* __restrict__ src,
                                                   double scale, const uint8_t* __restrict__ act,
                                                   T* __restrict__ r, T* __restrict__ p,
                                                   double* partials, PcgScalars* sc,
                                                   int fin = FIN_INIT) {
  double s2 = 0.0, mx = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    T v = act[e] ? (T)(src[e] * scale) : T(0);
    r[e] = v;
    p[e] = T(0);
    double dv = (double)v;
    s2 += dv * dv;
    mx = fmax(mx, fabs(dv));
  }
  reduce_finalize(s2, mx, partials, sc, fin);
}

// The iteration kernels below visit only the tiles of a sweep order list
// (tiles[-1].x entries; the tiles holding an active cell): the vectors they
// update are zero on every other tile and stay so.  Work unit: one slot of a
// tile, its TY x 32 = 256 consecutive elements, one per thread of the block.
static_assert(Tiled::TY * 32 == kThreads, "a tile slot is one element per thread");
__device__ __forceinline__ int slot_count(const Tiled& g, const int2* __restrict__ tiles) {
  return tiles[-1].x * g.nz;
}
__device__ __forceinline__ int64_t slot_elem(const Tiled& g, const int2* __restrict__ tiles, int c) {
  const int t = c / g.nz, sl = c - t * g.nz;
  const int2 XY = tiles[t];
  return ((int64_t)(XY.y * g.ntx + (XY.x & 0xffff)) * g.nz + sl) * kThreads + threadIdx.x;
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_copy(Tiled g, const int2* __restrict__ tiles, const T* __restrict__ a,
                                                   T* __restrict__ b, const PcgScalars* sc) {
  if (sc->done != DONE_RUNNING) return;
  const int nch = slot_count(g, tiles);
  for (int c = blockIdx.x; c < nch; c += gridDim.x) {
    const int64_t e = slot_elem(g, tiles, c);
    b[e] = a[e];
  }
}

// applyCompressedMatrix (project-solver.cc:16-39) on the tiled layout.  The
// upper couplings come from the neighbours' lower ones (A symmetric,
// checkSystemSymmetry, :41-57).
template <class T, class X>
__device__ __forceinline__ T apply_row(const Tiled& g, const Cell& c, const T* __restrict__ adiag,
                                       const T* __restrict__ al, const T* __restrict__ ad,
                                       const T* __restrict__ ab, const uint8_t* __restrict__ act,
                                       const X* __restrict__ x) {
  const int64_t e = c.e;
  T t = adiag[e] * (T)x[e];
  if (c.x > 0) {
    int64_t o = c.xm(g);
    if (act[o]) t += al[e] * (T)x[o];
  }
  if (c.y > 0) {
    int64_t o = c.ym(g);
    if (act[o]) t += ad[e] * (T)x[o];
  }
  if (c.z > 0) {
    int64_t o = c.zm(g);
    if (act[o]) t += ab[e] * (T)x[o];
  }
  if (c.x < g.nx - 1) {
    int64_t o = c.xp(g);
    if (act[o]) t += al[o] * (T)x[o];
  }
  if (c.y < g.ny - 1) {
    int64_t o = c.yp(g);
    if (act[o]) t += ad[o] * (T)x[o];
  }
  if (c.z < g.nz - 1) {
    int64_t o = c.zp(g);
    if (act[o]) t += ab[o] * (T)x[o];
  }
  return t;
}

// The PCG's own SpMV.  The PCG vectors are zero on inactive cells and the
// couplings are finite (k_mask_system), so the neighbour activity tests of
// apply_row drop out: every load is unconditional and independent, and the
// result equals applyCompressedMatrix.
template <class T>
__device__ __forceinline__ T apply_row_pcg(const Tiled& g, const Cell& c, const T* __restrict__ adiag,
                                           const T* __restrict__ al, const T* __restrict__ ad,
                                           const T* __restrict__ ab, const T* __restrict__ x) {
  const int64_t e = c.e;
  const bool hx = c.x > 0, hy = c.y > 0, hz = c.z > 0;
  const bool px = c.x < g.nx - 1, py = c.y < g.ny - 1, pz = c.z < g.nz - 1;
  const int64_t oxm = hx ? c.xm(g) : e, oym = hy ? c.ym(g) : e, ozm = hz ? c.zm(g) : e;
  const int64_t oxp = px ? c.xp(g) : e, oyp = py ? c.yp(g) : e, ozp = pz ? c.zp(g) : e;
  const T cxm = hx ? al[e] : T(0), cym = hy ? ad[e] : T(0), czm = hz ? ab[e] : T(0);
  const T cxp = px ? al[oxp] : T(0), cyp = py ? ad[oyp] : T(0), czp = pz ? ab[ozp] : T(0);
  T t = adiag[e] * x[e];
  t += cxm * x[oxm];
  t += cym * x[oym];
  t += czm * x[ozm];
  t += cxp * x[oxp];
  t += cyp * x[oyp];
  t += czp * x[ozp];
  return t;
}

// Each block walks a contiguous range of row blocks (consecutive slots of a
// tile), so the neighbour rows it reads (x and z neighbours, the upper
// couplings) were just loaded by the same block; two row blocks per pass.
// (Measured against two alternatives at 128^3-512^3: per-warp row streaming
// with register windows, and a multistage cp.async slab pipeline; both were
// slower.)
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_spmv(Tiled g, const T* __restrict__ adiag, const T* __restrict__ al,
           const T* __restrict__ ad, const T* __restrict__ ab, const uint8_t* __restrict__ act,
           const T* __restrict__ x, T* __restrict__ y, double* partials, PcgScalars* sc,
           int use_skip) {
  if (use_skip && sc->done != DONE_RUNNING) return;
  double acc = 0.0;
  const int nrb = g.ntiles() * g.nz;
  const int chunk = (nrb + gridDim.x - 1) / gridDim.x;
  const int rb_end = min(nrb, (int)(blockIdx.x + 1) * chunk);
  for (int rb0 = blockIdx.x * chunk; rb0 < rb_end; rb0 += 2) {
    const int rb1 = rb0 + 1;
    Cell c0, c1;
    c0.init(g, rb0, threadIdx.x);
    c1.init(g, rb1 < rb_end ? rb1 : rb0, threadIdx.x);
    const T t0 = apply_row_pcg(g, c0, adiag, al, ad, ab, x);
    const T t1 = apply_row_pcg(g, c1, adiag, al, ad, ab, x);
    const bool a0 = c0.inside && act[c0.e], a1 = rb1 < rb_end && c1.inside && act[c1.e];
    const T o0 = a0 ? t0 : T(0), o1 = a1 ? t1 : T(0);
    acc += (double)x[c0.e] * (double)o0;
    y[c0.e] = o0;
    if (rb1 < rb_end) {
      acc += (double)x[c1.e] * (double)o1;
      y[c1.e] = o1;
    }
  }
  reduce_finalize(acc, 0.0, partials, sc, FIN_SPMV);
}

// The PCG's SpMV as a stream over the z-slots of each tile.  In the tiled
// layout the z-neighbours of a cell are its own lane's entries at the previous
// and next slot, and its x-neighbours are the previous and next lanes' entries
// at those slots.  A warp that owns row ty of a tile and walks the slots in
// order therefore holds every x and z neighbour in a three-slot register window
// (x neighbours by shuffle); the y neighbours are the adjacent rows of the same
// slot, read through L1 where the block's other warps have just loaded them.
// Each array element comes from HBM once, and no cell pays for a division or a
// tile-edge branch: only the two edge lanes of a row reach into the next tiles.
// The sum is the same as apply_row_pcg's, term for term.  A work item is the
// TY row warps of one tile over a run of consecutive slots.
template <class T>
__global__ void __launch_bounds__(kThreads, 3)
    k_spmv_stream(Tiled g, const int2* __restrict__ tiles, const T* __restrict__ adiag, const T* __restrict__ al,
                  const T* __restrict__ ad, const T* __restrict__ ab, const uint8_t* __restrict__ act,
                  const T* __restrict__ x, T* __restrict__ y, double* partials, PcgScalars* sc, int use_skip,
                  int chunks) {
  if (use_skip && sc->done != DONE_RUNNING) return;
  constexpr int TY = Tiled::TY, RS = Tiled::TY * 32;  // elements per slot of a tile
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nz = g.nz;
  double acc = 0.0;
  // the listed tiles (those with an active cell; y stays zero on the others)
  const int items = tiles[-1].x * chunks;
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const int li = it / chunks, ch = it - li * chunks;
    const int tile = tiles[li].y * g.ntx + (tiles[li].x & 0xffff);
    const int s0 = (int)((int64_t)nz * ch / chunks), s1 = (int)((int64_t)nz * (ch + 1) / chunks);
    const int Y = tile / g.ntx, X = tile - Y * g.ntx;
    const int xg = X * 32 + tx, yg = Y * TY + ty;
    const bool inside = xg < g.nx && yg < g.ny;
    const bool hx = xg > 0, px = xg < g.nx - 1, hy = yg > 0, py = yg < g.ny - 1;
    const int64_t tb = (int64_t)tile * g.tile_elems;
    const int64_t row = tb + ty * 32 + tx;
    // the rows of the same slot at y - 1 and y + 1 (read only when hy / py)
    const int64_t rym = ty > 0 ? row - 32 : tb - (int64_t)g.ntx * g.tile_elems + (TY - 1) * 32 + tx;
    const int64_t ryp = ty < TY - 1 ? row + 32 : tb + (int64_t)g.ntx * g.tile_elems + tx;
    // the lanes across the x edges: lane 0's x - 1 is lane 31 of tile X - 1 at
    // slot s + 31, lane 31's x + 1 is lane 0 of tile X + 1 at slot s - 31
    const int64_t rxm = tb - g.tile_elems + ty * 32 + 31, rxp = tb + g.tile_elems + ty * 32;
    auto wrap = [nz](int v) { return v >= nz ? v - nz : (v < 0 ? v + nz : v); };
    int sm = wrap(s0 - 1), sp = wrap(s0 + 1), s31 = wrap(wrap(s0 + 31 % nz)), sm31 = wrap(wrap(s0 - 31 % nz));
    int z = wrap(s0 - tx % nz);
    T x_m = __ldg(x + row + (int64_t)sm * RS), x_c = __ldg(x + row + (int64_t)s0 * RS),
      x_p = __ldg(x + row + (int64_t)sp * RS);
    T al_c = __ldg(al + row + (int64_t)s0 * RS), al_p = __ldg(al + row + (int64_t)sp * RS);
    T ab_c = __ldg(ab + row + (int64_t)s0 * RS), ab_p = __ldg(ab + row + (int64_t)sp * RS);
    // the other loads of a slot are issued one slot ahead too (slot sp is a
    // valid slot index at the end of the run as well, so they stay in bounds)
    const bool ex0 = tx == 0 && hx, ex31 = tx == 31 && px;
    T d_n = __ldg(adiag + row + (int64_t)s0 * RS), adc_n = __ldg(ad + row + (int64_t)s0 * RS);
    uint8_t a_n = __ldg(act + row + (int64_t)s0 * RS);
    T ym_n = hy ? __ldg(x + rym + (int64_t)s0 * RS) : T(0), yp_n = py ? __ldg(x + ryp + (int64_t)s0 * RS) : T(0),
      adp_n = py ? __ldg(ad + ryp + (int64_t)s0 * RS) : T(0);
    T xme_n = ex0 ? __ldg(x + rxm + (int64_t)s31 * RS) : T(0), xpe_n = ex31 ? __ldg(x + rxp + (int64_t)sm31 * RS) : T(0),
      alpe_n = ex31 ? __ldg(al + rxp + (int64_t)sm31 * RS) : T(0);
    for (int s = s0; s < s1; s++) {
      const int64_t e = row + (int64_t)s * RS;
      const int s2 = wrap(sp + 1);
      const T d = d_n, adc = adc_n, ymv = ym_n, ypv = yp_n, adp = adp_n, xme = xme_n, xpe = xpe_n, alpe = alpe_n;
      const bool a = inside && a_n;
      // next window entries and the next slot's loads first: their latency
      // overlaps this slot's work
      const T x_n = __ldg(x + row + (int64_t)s2 * RS), al_n = __ldg(al + row + (int64_t)s2 * RS),
              ab_n = __ldg(ab + row + (int64_t)s2 * RS);
      {
        const int64_t en = row + (int64_t)sp * RS;
        const int s31n = wrap(s31 + 1), sm31n = wrap(sm31 + 1);
        d_n = __ldg(adiag + en);
        adc_n = __ldg(ad + en);
        a_n = __ldg(act + en);
        ym_n = hy ? __ldg(x + rym + (int64_t)sp * RS) : T(0);
        yp_n = py ? __ldg(x + ryp + (int64_t)sp * RS) : T(0);
        adp_n = py ? __ldg(ad + ryp + (int64_t)sp * RS) : T(0);
        xme_n = ex0 ? __ldg(x + rxm + (int64_t)s31n * RS) : T(0);
        xpe_n = ex31 ? __ldg(x + rxp + (int64_t)sm31n * RS) : T(0);
        alpe_n = ex31 ? __ldg(al + rxp + (int64_t)sm31n * RS) : T(0);
      }
      const bool hz = z > 0, pz = z < nz - 1;
      const T ym = hy ? ymv : x_c;
      const T yp = py ? ypv : x_c;
      T xm = __shfl_up_sync(kFull, x_m, 1), xp = __shfl_down_sync(kFull, x_p, 1),
        alp = __shfl_down_sync(kFull, al_p, 1);
      if (tx == 0) xm = hx ? xme : x_c;
      if (tx == 31) {
        xp = px ? xpe : x_c;
        alp = px ? alpe : T(0);
      }
      if (!hx) xm = x_c;
      if (!px) xp = x_c;
      const T cxm = hx ? al_c : T(0), cym = hy ? adc : T(0), czm = hz ? ab_c : T(0);
      const T cxp = px ? alp : T(0), cyp = py ? adp : T(0), czp = pz ? ab_p : T(0);
      T t = d * x_c;
      t += cxm * xm;
      t += cym * ym;
      t += czm * (hz ? x_m : x_c);
      t += cxp * xp;
      t += cyp * yp;
      t += czp * (pz ? x_p : x_c);
      const T o = a ? t : T(0);
      y[e] = o;
      acc += (double)x_c * (double)o;
      x_m = x_c;
      x_c = x_p;
      x_p = x_n;
      al_c = al_p;
      al_p = al_n;
      ab_c = ab_p;
      ab_p = ab_n;
      sm = s;
      sp = s2;
      s31 = wrap(s31 + 1);
      sm31 = wrap(sm31 + 1);
      z = wrap(z + 1);
    }
  }
  reduce_finalize(acc, 0.0, partials, sc, FIN_SPMV);
}

// b = A x with the reference's activity tests (x may be non-zero on inactive
// cells): applyCompressedMatrix for the apply entry point.
__global__ void __launch_bounds__(kThreads)
    k_apply_checked(Tiled g, const double* __restrict__ adiag, const double* __restrict__ al,
                    const double* __restrict__ ad, const double* __restrict__ ab,
                    const uint8_t* __restrict__ act, const double* __restrict__ x, double* __restrict__ b) {
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    b[c.e] = (c.inside && act[c.e]) ? apply_row(g, c, adiag, al, ad, ab, act, x) : 0.0;
  }
}

// Entries that couple to an inactive cell, and whole inactive rows, are never
// read by applyCompressedMatrix (it tests the neighbour's activity first).  The
// PCG kernels multiply them by zeros instead of testing, so any non-finite
// value there is replaced by 0 before the solve; finite values stay as given.
__global__ void __launch_bounds__(kThreads)
    k_mask_system(Tiled g, const uint8_t* __restrict__ act, double* __restrict__ adiag,
                  double* __restrict__ al, double* __restrict__ ad, double* __restrict__ ab) {
  auto fix = [](double* a, int64_t e) {
    if (!isfinite(a[e])) a[e] = 0.0;
  };
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    const int64_t e = c.e;
    if (!(c.inside && act[e])) {
      fix(adiag, e);
      fix(al, e);
      fix(ad, e);
      fix(ab, e);
      continue;
    }
    if (c.x == 0 || !act[c.xm(g)]) fix(al, e);
    if (c.y == 0 || !act[c.ym(g)]) fix(ad, e);
    if (c.z == 0 || !act[c.zm(g)]) fix(ab, e);
  }
}

// saxpy(pg, s, alpha); saxpy(r, z, -alpha); residual (:332-335, util.cc:394-402).
// s and Az are zero on inactive cells, so the masked updates of the reference
// are the plain updates here; four independent elements per thread per pass.
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_axpy(Tiled g, const int2* __restrict__ tiles, const T* __restrict__ s,
           const T* __restrict__ Az, T* __restrict__ p, T* __restrict__ r, double* partials,
           PcgScalars* sc, int fin = FIN_AXPY) {
  if (sc->done != DONE_RUNNING) return;
  const T alpha = (T)sc->alpha;
  double s2 = 0.0, mx = 0.0;
  const int nch = slot_count(g, tiles);
  for (int c0 = blockIdx.x; c0 < nch; c0 += 4 * gridDim.x) {
    T sv[4], av[4], pv[4], rv[4];
    int64_t ee[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int c = c0 + k * (int)gridDim.x;
      const bool in = c < nch;
      const int64_t e = in ? slot_elem(g, tiles, c) : 0;
      ee[k] = in ? e : -1;
      sv[k] = in ? s[e] : T(0);
      av[k] = in ? Az[e] : T(0);
      pv[k] = in ? p[e] : T(0);
      rv[k] = in ? r[e] : T(0);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int64_t e = ee[k];
      if (e < 0) continue;
      p[e] = pv[k] + alpha * sv[k];
      const T rn = rv[k] + (-alpha) * av[k];
      r[e] = rn;
      const double dv = (double)rn;
      s2 += dv * dv;
      mx = fmax(mx, fabs(dv));
    }
  }
  reduce_finalize(s2, mx, partials, sc, fin);
}

// scaleAndAdd(s, z, beta): s = z + beta s (util.cc:404-410); z and s are zero
// on inactive cells.
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_sa(Tiled g, const int2* __restrict__ tiles, const T* __restrict__ z, T* __restrict__ s,
         double* partials, PcgScalars* sc) {
  if (sc->done != DONE_RUNNING) return;
  const T beta = (T)sc->beta;
  const int nch = slot_count(g, tiles);
  for (int c0 = blockIdx.x; c0 < nch; c0 += 4 * gridDim.x) {
    T zv[4], sv[4];
    int64_t ee[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int c = c0 + k * (int)gridDim.x;
      const bool in = c < nch;
      const int64_t e = in ? slot_elem(g, tiles, c) : 0;
      ee[k] = in ? e : -1;
      zv[k] = in ? z[e] : T(0);
      sv[k] = in ? s[e] : T(0);
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (ee[k] >= 0) s[ee[k]] = zv[k] + beta * sv[k];
  }
  reduce_finalize(0.0, 0.0, partials, sc, FIN_SA);
}

// Upper couplings in own-cell form for the backward sweep:
// uR(p) = cL(p+x) = A_L(p+x) E(p), etc. (the products of project-solver.cc:296-302).
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_upper(Tiled g, const T* __restrict__ cL, const T* __restrict__ cD,
            const T* __restrict__ cB, T* __restrict__ uR, T* __restrict__ uU, T* __restrict__ uF) {
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    T a = T(0), b = T(0), d = T(0);
    if (c.inside) {
      if (c.x < g.nx - 1) a = cL[c.xp(g)];
      if (c.y < g.ny - 1) b = cD[c.yp(g)];
      if (c.z < g.nz - 1) d = cB[c.zp(g)];
    }
    uR[c.e] = a;
    uU[c.e] = b;
    uF[c.e] = d;
  }
}

// Diagonals of the Eisenstat operator (FwdEisenstatOp), from the FP64 pivots:
// Pinv = 1/E and Dt = 2/E^2 - Adiag where E != 0, else 0.
__global__ void __launch_bounds__(kThreads)
    k_eisenstat_diag(int64_t n, const double* __restrict__ E, const double* __restrict__ adiag,
                     float* __restrict__ pinv, float* __restrict__ dt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const double v = E[e];
    const double pi = v != 0.0 ? 1.0 / v : 0.0;
    pinv[e] = (float)pi;
    dt[e] = v != 0.0 ? (float)(2.0 * pi * pi - adiag[e]) : 0.0f;
  }
}

// b - A x in FP64 (norms only): the true residual of the final iterate.
__global__ void __launch_bounds__(kThreads)
    k_true_residual(Tiled g, const double* __restrict__ adiag, const double* __restrict__ al,
                    const double* __restrict__ ad, const double* __restrict__ ab,
                    const uint8_t* __restrict__ act, const double* __restrict__ x,
                    const double* __restrict__ b, double* partials, PcgScalars* sc) {
  double s2 = 0.0, mx = 0.0;
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    if (c.inside && act[c.e]) {
      double rv = b[c.e] - apply_row(g, c, adiag, al, ad, ab, act, x);
      s2 += rv * rv;
      mx = fmax(mx, fabs(rv));
    }
  }
  reduce_finalize(s2, mx, partials, sc, FIN_NORMS);
}

// Mixed precision defect correction: x += scale d ; r -= scale A d (FP64 A, FP64 r).
__global__ void __launch_bounds__(kThreads)
    k_mixed_update(Tiled g, const double* __restrict__ adiag, const double* __restrict__ al,
                   const double* __restrict__ ad, const double* __restrict__ ab,
                   const uint8_t* __restrict__ act, const float* __restrict__ d, double scale,
                   double* __restrict__ x, double* __restrict__ r, double* partials,
                   PcgScalars* sc) {
  double s2 = 0.0, mx = 0.0;
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    if (!(c.inside && act[c.e])) continue;
    const double t = apply_row(g, c, adiag, al, ad, ab, act, d);
    x[c.e] += scale * (double)d[c.e];
    const double rv = r[c.e] - scale * t;
    r[c.e] = rv;
    s2 += rv * rv;
    mx = fmax(mx, fabs(rv));
  }
  reduce_finalize(s2, mx, partials, sc, FIN_NORMS);
}

// ---------------------------------------------------------------------------------
// Wavefront sweeps.
//
// A persistent kernel: each CTA repeatedly takes a ticket, maps it to a tile in
// dependency order, and sweeps the tile's i+j+k wavefront with TY compute warps
// (warp = tile row ty, lane = tx).  At step s, lane tx of warp ty owns cell
// z = s - ty - tx (forward) and reads one contiguous row of the tiled arrays.
// Neighbour values inside the tile travel by shuffle (x), shared memory (y) and
// registers (z).  Values from the neighbouring tiles arrive through a
// communication warp that polls the neighbours' published progress and streams
// their boundary rows into shared-memory rings; the same warp publishes this
// tile's progress.  Every wait is bounded: on timeout the kernel raises
// DEV_ERR_TIMEOUT, releases its dependants and finishes.

// Cell operations of the three sweeps.  Each reads NV arrays at its own cell
// (staged into shared memory by cp.async) plus the three already-computed
// neighbour values xn, yn, zn.
// compute() returns the value the recurrence passes on to the neighbours and
// stores the op's outputs at element e itself.
template <class T, bool SELFDOT = false>
struct FwdOp {  // L q = r (project-solver.cc:276-288), c* = A_* E(neighbour); SELFDOT: acc q.q
  static constexpr int NV = 5;
  const T* src[NV];  // r, cL, cD, cB, E
  T* out;            // q
  __device__ __forceinline__ T compute(const T* v, T xn, T yn, T zn, int64_t e, double& acc) const {
    T t = v[0];
    t -= v[1] * xn;
    t -= v[2] * yn;
    t -= v[3] * zn;
    const T q = t * v[4];
    out[e] = q;
    if (SELFDOT) acc += (double)q * (double)q;
    return q;
  }
};

template <class T>
struct BwdOp {  // L^T z = q (project-solver.cc:293-305), u* = A_*(p+dir) E(p); sigma = z.r
  static constexpr int NV = 6;
  const T* src[NV];  // q, E, uR, uU, uF, r
  T* out;            // z
  __device__ __forceinline__ T compute(const T* v, T xn, T yn, T zn, int64_t e, double& acc) const {
    T t = v[0];
    t -= v[2] * xn;
    t -= v[3] * yn;
    t -= v[4] * zn;
    T z = t * v[1];
    out[e] = z;
    acc += (double)z * (double)v[5];
    return z;
  }
};

// Eisenstat backward sweep with the search-direction update folded in:
//   s = rh + beta s  (scaleAndAdd of the CG step), then t = L^-T s.
// beta comes from the device scalars, read once per CTA (prepare).
template <class T>
struct BwdEisenstatOp {
  static constexpr int NV = 6;
  const T* src[NV];  // rh, s (previous), E, uR, uU, uF
  T* out;            // t
  T* s_out;          // s (in place of src[1]: each element is read before it is written)
  T beta;
  __device__ __forceinline__ void prepare(const PcgScalars* sc) { beta = (T)sc->beta; }
  __device__ __forceinline__ T compute(const T* v, T xn, T yn, T zn, int64_t e, double&) const {
    const T sv = v[0] + beta * v[1];
    s_out[e] = sv;
    T u = sv;
    u -= v[3] * xn;
    u -= v[4] * yn;
    u -= v[5] * zn;
    const T t = u * v[2];
    out[e] = t;
    return t;
  }
};

// Ops without per-launch scalars.
template <class Op, class = void>
struct HasPrepare : std::false_type {};
template <class Op>
struct HasPrepare<Op, std::void_t<decltype(std::declval<Op&>().prepare(nullptr))>> : std::true_type {};

// Eisenstat's form of the preconditioned operator (S. C. Eisenstat, "Efficient
// implementation of a class of preconditioned conjugate gradient methods",
// SIAM J. Sci. Stat. Comput. 2 (1981) 1-4).  With the MIC(0) factor
// L = (P^-2 + F) P (P = diag(E), F the strictly lower part of A) and
// A = K + K^T - Dt, K = P^-2 + F, Dt = 2 P^-2 - diag(A), the split operator is
//   L^-1 A L^-T v = P^-1 t + L^-1 (P^-1 v - Dt t),   t = L^-T v,
// so one backward sweep (t) and this forward sweep apply it: no SpMV.  The
// recurrence carries q = L^-1 (P^-1 v - Dt t); the output is w = P^-1 t + q
// and acc gathers v.w.  Pinv = 1/E and Dt are 0 on cells where E = 0.
template <class T>
struct FwdEisenstatOp {
  static constexpr int NV = 8;
  const T* src[NV];  // v, t, Pinv, Dt, cL, cD, cB, E
  T* out;            // w
  __device__ __forceinline__ T compute(const T* v, T xn, T yn, T zn, int64_t e, double& acc) const {
    T u = v[2] * v[0];
    u -= v[3] * v[1];
    u -= v[4] * xn;
    u -= v[5] * yn;
    u -= v[6] * zn;
    const T q = u * v[7];
    const T w = v[2] * v[1] + q;
    out[e] = w;
    acc += (double)v[0] * (double)w;
    return q;
  }
};

// MIC(0) pivot (project-solver.cc:237-274), FP64.  The exchanged value is E.
// E(q) != 0 exactly when q is active with Adiag(q) != 0, which is the guard the
// reference tests before using E(q).  adm is Adiag masked by the active flag;
// dL/dD/dB hold the tau-weighted products with the diagonal neighbours'
// couplings (k_pivot_diag), so the sweep only streams its own row.
struct PivotOp {
  static constexpr int NV = 7;
  const double* src[NV];  // adm, al, ad, ab, dL, dD, dB
  double sigma;
  double *out, *cL, *cD, *cB;
  __device__ __forceinline__ double compute(const double* v, double EL, double ED, double EB,
                                            int64_t e, double&) const {
    const double adiag = v[0], al = v[1], ad = v[2], ab = v[3];
    double E = 0.0;
    if (adiag != 0.0) {
      double ee = adiag;
      if (EL != 0.0) {
        ee -= (al * EL) * (al * EL);
        ee -= v[4] / (EL * EL);
      }
      if (ED != 0.0) {
        ee -= (ad * ED) * (ad * ED);
        ee -= v[5] / (ED * ED);
      }
      if (EB != 0.0) {
        ee -= (ab * EB) * (ab * EB);
        ee -= v[6] / (EB * EB);
      }
      if (ee < sigma * adiag) ee = adiag;
      E = 1.0 / sqrt(ee);
    }
    out[e] = E;
    cL[e] = al * EL;
    cD[e] = ad * ED;
    cB[e] = ab * EB;
    return E;
  }
};

// The tau-weighted neighbour products of the pivot recurrence
// (project-solver.cc:244-265): for the Left term
//   tau*A_L(p)*A_L(p-x+y) [if p-x+y active] + tau*A_L(p)*A_L(p-x+z) [if p-x+z active]
// and likewise for Down and Back.  They only depend on A.
__global__ void __launch_bounds__(kThreads)
    k_pivot_diag(Tiled g, const double* __restrict__ adiag, const double* __restrict__ al,
                 const double* __restrict__ ad, const double* __restrict__ ab,
                 const uint8_t* __restrict__ act, double tau, double* __restrict__ adm,
                 double* __restrict__ dL, double* __restrict__ dD, double* __restrict__ dB) {
  SC_ROWBLOCK_LOOP(g) {
    Cell c;
    c.init(g, rb, threadIdx.x);
    double l = 0.0, d = 0.0, b = 0.0;
    if (c.inside) {
      const int x = c.x, y = c.y, z = c.z;
      if (x > 0) {
        const double a = al[c.e];
        if (y < g.ny - 1) {
          int64_t o = g.off(x - 1, y + 1, z);
          if (act[o]) l += tau * a * al[o];
        }
        if (z < g.nz - 1) {
          int64_t o = g.off(x - 1, y, z + 1);
          if (act[o]) l += tau * a * al[o];
        }
      }
      if (y > 0) {
        const double a = ad[c.e];
        if (x < g.nx - 1) {
          int64_t o = g.off(x + 1, y - 1, z);
          if (act[o]) d += tau * a * ad[o];
        }
        if (z < g.nz - 1) {
          int64_t o = g.off(x, y - 1, z + 1);
          if (act[o]) d += tau * a * ad[o];
        }
      }
      if (z > 0) {
        const double a = ab[c.e];
        if (x < g.nx - 1) {
          int64_t o = g.off(x + 1, y, z - 1);
          if (act[o]) b += tau * a * ab[o];
        }
        if (y < g.ny - 1) {
          int64_t o = g.off(x, y + 1, z - 1);
          if (act[o]) b += tau * a * ab[o];
        }
      }
    }
    dL[c.e] = l;
    dD[c.e] = d;
    dB[c.e] = b;
    adm[c.e] = (c.inside && act[c.e]) ? adiag[c.e] : 0.0;
  }
}

template <int TY, bool FWD>
__device__ __forceinline__ int wave_slot(const Tiled& g, int s, int ty) {
  return FWD ? wrap_mod(s - ty, g.nz) : wrap_mod(g.nz + 29 + TY - s - ty, g.nz);
}

// Mailbox sentinel: a NaN payload that arithmetic never produces (the GPU's
// canonical NaN has all mantissa bits set).
template <class T>
struct Sentinel;
template <>
struct Sentinel<double> {
  using Bits = unsigned long long;
  static constexpr Bits bits = 0x7ff4deadbeefcafeull;
};
template <>
struct Sentinel<float> {
  using Bits = unsigned int;
  static constexpr Bits bits = 0x7fa5deadu;
};
template <class T>
__device__ __forceinline__ typename Sentinel<T>::Bits mb_load(const T* p) {
  typename Sentinel<T>::Bits v;
  if constexpr (sizeof(T) == 8)
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  else
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
template <class T>
__device__ __forceinline__ T mb_value(typename Sentinel<T>::Bits b) {
  T v;
  memcpy(&v, &b, sizeof(T));
  return v;
}
// Every mailbox access is a strong (relaxed, gpu-scope) operation, so writes by
// one CTA and polls by another are coherent under the PTX memory model.
template <class T>
__device__ __forceinline__ void mb_store_bits(T* p, typename Sentinel<T>::Bits b) {
  if constexpr (sizeof(T) == 8)
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(b) : "memory");
  else
    asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(b) : "memory");
}
template <class T>
__device__ __forceinline__ void mb_store(T* p, T v) {
  typename Sentinel<T>::Bits b;
  memcpy(&b, &v, sizeof(T));
  mb_store_bits(p, b);
}
template <class T>
__device__ __forceinline__ void mb_reset(T* p) {
  mb_store_bits(p, Sentinel<T>::bits);
}

// B-byte copy global -> shared (B = 4, 8 or 16; both addresses B-byte aligned);
// 16-byte copies bypass L1.
template <int B, class T>
__device__ __forceinline__ void cp_async_bytes(T* dst, const T* src) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared state of one wavefront CTA.
template <class T, int TY>
struct WaveShared {
  T xch[2][TY][32];
  T bufX[kRing][TY];
  T bufY[kRing][32];
  volatile int done;     // compute steps completed
  volatile int availX;   // ring entries loaded
  volatile int availY;
  volatile int abort;
  int tile;
  bool last;
  double ssum[TY + 3];
};

// Hand-off ring between the CTAs of a thread-block cluster (distributed shared
// memory): the y-boundary row a tile passes to the next tile of the same
// cluster goes straight into that CTA's ring.  One 64-bit word per lane and
// entry holds the FP32 value in its low half and a stamp (the cluster tile's
// ticket << 12 | the entry) in its high half, written with one store, so a
// consumer that sees the stamp it expects sees the value: no fence and no
// reset.  Each CTA fills its ring with an impossible stamp at launch.
constexpr int kClRing = 32;
constexpr unsigned kClNoStamp = 0xffffffffu;
__device__ __forceinline__ unsigned cl_stamp(int ticket, int e) { return ((unsigned)ticket << 12) | (unsigned)e; }
__device__ __forceinline__ void st_relaxed_cluster_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.cluster.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_cluster_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.cluster.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_cluster_s32(const int* p) {
  int v;
  asm volatile("ld.relaxed.cluster.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
template <class T>
__device__ __forceinline__ T cl_value(unsigned long long w) {
  if constexpr (sizeof(T) == 4)
    return __uint_as_float((unsigned)(w & 0xffffffffull));
  else
    return T(0);
}
template <class T>
__device__ __forceinline__ unsigned long long cl_word(int ticket, int e, T v) {
  if constexpr (sizeof(T) == 4)
    return ((unsigned long long)cl_stamp(ticket, e) << 32) | (unsigned long long)__float_as_uint(v);
  else
    return 0ull;
}

// Give up: flag the error and release the compute warps.
template <class T, int TY>
__device__ __forceinline__ void wave_abort(const WaveArgs& a, WaveShared<T, TY>& sh, int NS) {
  atomicOr(&a.sc->err, DEV_ERR_TIMEOUT);
  sh.abort = 1;
  sh.availX = NS;
  sh.availY = NS;
}

// A wait ends early only when another wait of the sweep gave up (the timeout
// bit): the other status bits (a breakdown, a non-finite dot product) belong
// to the iteration, and a sweep run after one of them still completes.
__device__ __forceinline__ bool wave_should_stop(const WaveArgs& a, int& spins,
                                                 volatile int* s_abort, int limit) {
  if (*s_abort) return true;
#if SC_WAVE_CTL_NS > 0
  __nanosleep(SC_WAVE_CTL_NS);
#endif
  ++spins;
  if ((spins & 63) == 0 && (ld_relaxed_gpu_u32(&a.sc->err) & DEV_ERR_TIMEOUT)) return true;
  return spins > limit;
}

// Mailboxes.  The producer tile writes each boundary value it computes into
// the mailbox of the tile that consumes it, at the consumer's ring-entry index:
//   x: mbx[consumer][e][ty]  (e = producer step - 31)
//   y: mby[consumer][e][tx]  (e = producer step - (TY-1))
// The consumer's loader warps poll those words until they stop holding the
// sentinel, copy them to the shared-memory rings and write the sentinel back,
// which leaves the mailboxes ready for the next sweep.  No fences are needed:
// every mailbox word carries exactly one value per sweep.
template <class T, int TY, bool FWD>
__device__ void wave_load_x(const WaveArgs& a, WaveShared<T, TY>& sh, T* mb, int NS, int limit) {
  const Tiled& g = a.g;
  const int lane = threadIdx.x & 31;
  constexpr int EPB = 32 / TY;  // entries per 32 lanes
  int lx = 0, spins = 0;
  while (lx < NS) {
    const int want = min(NS, sh.done + kRing);
    if (lx >= want) {
      if (wave_should_stop(a, spins, &sh.abort, limit)) break;
      continue;
    }
    // poll up to 8*EPB entries: lane handles (entry lx + k*EPB + lane/TY, ty = lane%TY)
    const int ty = lane % TY;
    typename Sentinel<T>::Bits v[8];
    unsigned ready = 0;  // bit k*EPB+j: entry lx+k*EPB+j fully ready
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int e = lx + k * EPB + lane / TY;
      const int z = FWD ? e - ty : g.nz - 1 - e + (TY - 1 - ty);
      const bool need = e < want && z >= 0 && z < g.nz;
      v[k] = need ? mb_load(mb + (int64_t)e * TY + ty) : (typename Sentinel<T>::Bits)0;
      const bool ok = e < want && (!need || v[k] != Sentinel<T>::bits);
      const unsigned bal = __ballot_sync(kFull, ok);
#pragma unroll
      for (int j = 0; j < EPB; j++)
        if (((bal >> (j * TY)) & ((1u << TY) - 1u)) == ((1u << TY) - 1u)) ready |= 1u << (k * EPB + j);
    }
    const int nready = __ffs(~ready) - 1;  // leading ready entries
    const int take = nready < 0 ? 8 * EPB : nready;
    if (take > 0) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int j = k * EPB + lane / TY;
        if (j < take) {
          const int e = lx + j;
          const int z = FWD ? e - ty : g.nz - 1 - e + (TY - 1 - ty);
          const bool need = z >= 0 && z < g.nz;
          sh.bufX[e % kRing][ty] = need ? mb_value<T>(v[k]) : T(0);
          if (need) mb_reset(mb + (int64_t)e * TY + ty);
        }
      }
      __syncwarp();
      __threadfence_block();
      if (lane == 0) sh.availX = lx + take;
      lx += take;
      spins = 0;
      continue;
    }
    if (wave_should_stop(a, spins, &sh.abort, limit)) break;
  }
  if (lx < NS && lane == 0) wave_abort(a, sh, NS);
}

template <class T, int TY, bool FWD>
__device__ void wave_load_y(const WaveArgs& a, WaveShared<T, TY>& sh, T* mb, int NS, int limit) {
  const Tiled& g = a.g;
  const int lane = threadIdx.x & 31;
  int ly = 0, spins = 0;
  while (ly < NS) {
    const int want = min(NS, sh.done + kRing);
    if (ly >= want) {
      if (wave_should_stop(a, spins, &sh.abort, limit)) break;
      continue;
    }
    typename Sentinel<T>::Bits v[8];
    unsigned ready = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int e = ly + k;
      // the consumer is warp 0 (forward) or warp TY-1 (backward), lane = tx
      const int z = FWD ? e - lane : g.nz - 1 - (e - (31 - lane));
      const bool need = e < want && z >= 0 && z < g.nz;
      v[k] = need ? mb_load(mb + (int64_t)e * 32 + lane) : (typename Sentinel<T>::Bits)0;
      const bool ok = e < want && (!need || v[k] != Sentinel<T>::bits);
      if (__all_sync(kFull, ok)) ready |= 1u << k;
    }
    const int nready = __ffs(~ready) - 1;
    const int take = nready < 0 ? 8 : nready;
    if (take > 0) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (k < take) {
          const int e = ly + k;
          const int z = FWD ? e - lane : g.nz - 1 - (e - (31 - lane));
          const bool need = z >= 0 && z < g.nz;
          sh.bufY[e % kRing][lane] = need ? mb_value<T>(v[k]) : T(0);
          if (need) mb_reset(mb + (int64_t)e * 32 + lane);
        }
      }
      __syncwarp();
      __threadfence_block();
      if (lane == 0) sh.availY = ly + take;
      ly += take;
      spins = 0;
      continue;
    }
    if (wave_should_stop(a, spins, &sh.abort, limit)) break;
  }
  if (ly < NS && lane == 0) wave_abort(a, sh, NS);
}

// One CTA per SM: the sweep is issue-bound, and capping registers for two
// CTAs per SM measured slower at 128^3, 256^3 and 512^3.
//
// CL > 0 (FP32 only): the grid is made of thread-block clusters of CL CTAs.  A
// ticket then names a cluster tile, CL tiles stacked along y in one column
// (X, Yc * CL + rank), and a tile hands its y-boundary row to the next tile of
// its cluster through that CTA's shared memory (kClRing) instead of a global
// mailbox; only the hand-offs between clusters (along y at the cluster edges,
// and along x) use the mailboxes.  The CTAs of a cluster take each ticket
// together and meet at a cluster barrier after each cluster tile.
template <class T, int TY, bool FWD, class Op, int CL = 0>
__global__ void __launch_bounds__((TY + 3) * 32, 1) k_wave(const WaveArgs a, const Op op_arg) {
  // warps 0..TY-1: tile rows (compute only, no fences: a fence would wait for
  // the prefetch loads in flight); warp TY: control (flags, ring waits);
  // warps TY+1, TY+2: x and y mailbox loaders.
  constexpr bool CLU = CL > 0;
  static_assert(!CLU || sizeof(T) == 4, "cluster hand-off rings carry FP32 values");
  constexpr int NBAR = (TY + 1) * 32;
  __shared__ WaveShared<T, TY> sh;
  __shared__ unsigned long long ringY[CLU ? kClRing : 1][32];
  extern __shared__ __align__(16) unsigned char wave_dyn[];
  T* stage = reinterpret_cast<T*>(wave_dyn);  // [kStage][TY][NV][32]
  if (a.use_skip && a.sc->done != DONE_RUNNING) return;
  // an earlier sweep gave up: do not wait again (a cluster decides together,
  // below, since CTAs could read the status word at different moments)
  if (!CLU && (a.sc->err & DEV_ERR_TIMEOUT)) return;
  int rank = 0;
  if constexpr (CLU) {
    rank = (int)cooperative_groups::this_cluster().block_rank();
    for (int i = threadIdx.x; i < kClRing * 32; i += blockDim.x) ringY[i / 32][i % 32] = (unsigned long long)kClNoStamp << 32;
    cooperative_groups::this_cluster().sync();  // every CTA of the cluster runs before any remote access
  }
  Op op = op_arg;
  if constexpr (HasPrepare<Op>::value) op.prepare(a.sc);
  const int slim = a.sc->spin_limit > 0 ? a.sc->spin_limit : kSpinLimit;  // bound of every wait
  const Tiled& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = g.ntiles();
  const int NS = g.nz + 31 + TY - 1;
  T* mbx = reinterpret_cast<T*>(a.mbx);
  T* mby = reinterpret_cast<T*>(a.mby);
  double acc = 0.0;
  // the tickets: entries of the order list (tiles, or cluster tiles of CL
  // tiles along y), whose length sits in the header entry before the first
  const int nticket = a.order[-1].x;
  for (;;) {
    if constexpr (CLU) {
      if (threadIdx.x == 0) {
        sh.done = 0;
        sh.availX = 0;
        sh.availY = 0;
        sh.abort = 0;
      }
      if (rank == 0 && threadIdx.x == 0) {
        const int tk = atomicAdd(a.ticket, 1);
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        for (int r = 0; r < CL; r++) *cl.map_shared_rank(&sh.tile, r) = tk;
      }
      cooperative_groups::this_cluster().sync();
    } else {
      if (threadIdx.x == 0) {
        sh.tile = atomicAdd(a.ticket, 1);
        sh.done = 0;
        sh.availX = 0;
        sh.availY = 0;
        sh.abort = 0;
      }
      __syncthreads();
    }
    const int t = sh.tile;
    if (t >= nticket) break;
    // entry: x = X | neighbour bits << 16, y = the tile row (cluster tile row);
    // bit 0/1: the unit at X - 1 / X + 1 is swept, bit 2/3: the unit below /
    // above.  A unit that is not swept (no active cell) holds zeros and has
    // zero couplings to this one, so its boundary values are zeros.
    const int2 XY = a.order[FWD ? t : nticket - 1 - t];
    const int X = XY.x & 0xffff, nb = XY.x >> 16;
    const int Y = CLU ? XY.y * CL + rank : XY.y;
    // a cluster tile at the top edge can have CTAs without a tile
    if (Y < g.nty) {
    const int tid = Y * g.ntx + X;
    // producers within this cluster tile (along y, through the rings), and
    // consumers within it
    const bool inner_in = CLU && (FWD ? rank > 0 : rank < CL - 1);
    const bool inner_out = CLU && (FWD ? rank < CL - 1 : rank > 0);
    const bool hasX = FWD ? (nb & 1) : (nb & 2);
    const bool hasY = (FWD ? Y > 0 : Y < g.nty - 1) && (inner_in || (FWD ? (nb & 4) : (nb & 8)));
    // consumers of this tile's boundary values
    const bool outX = FWD ? (nb & 2) : (nb & 1);
    const bool outY = (FWD ? Y < g.nty - 1 : Y > 0) && (inner_out || (FWD ? (nb & 8) : (nb & 4)));
    const int cX = FWD ? tid + 1 : tid - 1, cY = FWD ? tid + g.ntx : tid - g.ntx;
    // y boundary rows within a cluster travel through the rings
    const bool ydin = CLU && hasY && inner_in;
    const bool ydout = CLU && outY && inner_out;
    const int64_t base = g.tile_base(X, Y);
    if (warp == TY) {
      // control warp: keeps the compute warps one step behind the rings; it
      // waits up to four times the loaders' bound
      const int ctl_limit = slim > (1 << 28) ? (1 << 30) : 4 * slim;
      auto wait_avail = [&](int s) {
        int spins = 0;
        if (ydin) {
          // this lane's word of ring entry s, where the consumer row needs it
          // (the same z test as the mailbox loader's)
          const int zc = FWD ? s - lane : g.nz - 1 - (s - (31 - lane));
          const bool need = zc >= 0 && zc < g.nz;
          const unsigned want = cl_stamp(t, s);
          const unsigned long long* w = &ringY[s % kClRing][lane];
          for (;;) {
            const bool mine = !need || (unsigned)(ld_relaxed_cluster_u64(w) >> 32) == want;
            const bool ok = mine && !(hasX && sh.availX <= s);
            if (__all_sync(kFull, ok) || __any_sync(kFull, sh.abort)) break;
            if (++spins > ctl_limit) {
              if (lane == 0) wave_abort(a, sh, NS);
              break;
            }
#if SC_WAVE_CTL_NS > 0
            __nanosleep(SC_WAVE_CTL_NS);
#endif
          }
        } else {
          while (((hasX && sh.availX <= s) || (hasY && sh.availY <= s)) && !sh.abort) {
            if (++spins > ctl_limit) {
              if (lane == 0) wave_abort(a, sh, NS);
              break;
            }
#if SC_WAVE_CTL_NS > 0
            __nanosleep(SC_WAVE_CTL_NS);
#endif
          }
        }
        __syncwarp();
        __threadfence_block();
      };
      wait_avail(0);
      named_bar_sync(1, NBAR);
      for (int s = 0; s < NS; s++) {
        if (lane == 0) sh.done = s;  // steps < s are complete
        if (s + 1 < NS) wait_avail(s + 1);
        named_bar_sync(1, NBAR);
      }
      if (lane == 0) sh.done = NS;
    } else if (warp == TY + 1) {
      if (hasX) wave_load_x<T, TY, FWD>(a, sh, mbx + (int64_t)tid * a.mb_stride_x, NS, slim);
    } else if (warp == TY + 2) {
      if (hasY && !ydin) wave_load_y<T, TY, FWD>(a, sh, mby + (int64_t)tid * a.mb_stride_y, NS, slim);
    } else {
      const int ty = warp;
      T* outx = outX ? mbx + (int64_t)cX * a.mb_stride_x : nullptr;
      T* outy = (outY && !ydout) ? mby + (int64_t)cY * a.mb_stride_y : nullptr;
      const bool xsrc = FWD ? (lane == 31) : (lane == 0);        // lane feeding the x consumer
      const bool ysrc = FWD ? (ty == TY - 1) : (ty == 0);        // warp feeding the y consumer
      // the ring of the cluster CTA this tile feeds along y, and its progress
      unsigned long long* rring = nullptr;
      const int* rdone = nullptr;
      int cdone = 0;  // the consumer's completed steps, as last read
      if constexpr (CLU) {
        if (ydout && ysrc) {
          cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
          const int cr = FWD ? rank + 1 : rank - 1;
          rring = cl.map_shared_rank(&ringY[0][0], cr);
          rdone = const_cast<const int*>(cl.map_shared_rank(const_cast<int*>(&sh.done), cr));
        }
      }
      // slot of the row this warp touches at step s: forward (s - ty) mod nz,
      // backward (nz + 29 + TY - s - ty) mod nz; advanced incrementally.
      int cslot = wave_slot<TY, FWD>(g, 0, ty);
      int pslot = cslot;
      const int64_t rowbase = base + (int64_t)ty * 32 + lane;
      const int64_t rstride = (int64_t)TY * 32;
      auto advance = [&](int& sl) {
        if (FWD) {
          if (++sl == g.nz) sl = 0;
        } else {
          if (--sl < 0) sl = g.nz - 1;
        }
      };
      // The warp stages the NV input rows of step s + kStage into ring slot
      // s mod kStage at the end of step s, as kChunk-byte cp.async chunks spread
      // over the lanes (CPL per lane, pointers fixed per tile): after the step's
      // dependent chain, so the copies are issued while the other warps are
      // still on theirs.  The warp's lanes read that slot at the start of step s
      // (a __syncwarp orders the reads before the refill); each lane waits for
      // its own chunks of step s + 1 before the barrier of step s, and the
      // barrier makes every lane's chunks visible to the warp.
      constexpr int kStage = wave_stages<T, Op::NV>();
      constexpr int kChunk = sizeof(T) == 8 ? SC_WAVE_CHUNK64 : SC_WAVE_CHUNK32;  // bytes
      constexpr int EPC = kChunk / (int)sizeof(T);           // elements per chunk
      constexpr int CPR = 32 / EPC;                          // chunks per row
      constexpr int CPL = (Op::NV * CPR + 31) / 32;          // chunks per lane
      constexpr size_t kStageStride = (size_t)TY * Op::NV * 32;  // elements per ring slot
      const T* my_stage = stage + (size_t)ty * Op::NV * 32 + lane;
      const T* cg[CPL];
      int coff[CPL];
#pragma unroll
      for (int i = 0; i < CPL; i++) {
        const int j = lane + 32 * i;
        const int k = j / CPR, c = j - k * CPR;
        const T* src = op.src[0];
#pragma unroll
        for (int kk = 1; kk < Op::NV; kk++)
          if (k == kk) src = op.src[kk];
        cg[i] = j < Op::NV * CPR ? src + base + (int64_t)ty * 32 + c * EPC : nullptr;
        coff[i] = (ty * Op::NV + k) * 32 + c * EPC;
      }
      auto issue = [&](int sl, int ridx) {
        const int64_t so = (int64_t)sl * rstride;
#pragma unroll
        for (int i = 0; i < CPL; i++)
          if (Op::NV * CPR % 32 == 0 || cg[i]) cp_async_bytes<kChunk>(stage + ridx * kStageStride + coff[i], cg[i] + so);
      };
#pragma unroll
      for (int r = 0; r < kStage; r++) {
        if (r < NS) issue(pslot, r);
        cp_async_commit();
        advance(pslot);
      }
      cp_async_wait<kStage - 1>();
      T prev = T(0);
      named_bar_sync(1, NBAR);
      for (int s0 = 0; s0 < NS; s0 += kStage) {
#pragma unroll
        for (int u = 0; u < kStage; u++) {
          const int s = s0 + u;
          if (s < NS) {
            T v[Op::NV];
#pragma unroll
            for (int k = 0; k < Op::NV; k++) v[k] = my_stage[u * kStageStride + k * 32];
            const int z = FWD ? (s - ty - lane) : (g.nz - 1 - (s - (TY - 1 - ty) - (31 - lane)));
            const bool valid = (z >= 0) && (z < g.nz);
            const T shv = FWD ? __shfl_up_sync(kFull, prev, 1) : __shfl_down_sync(kFull, prev, 1);
            const bool xedge = FWD ? (lane == 0) : (lane == 31);
            const T xn = xedge ? (hasX ? sh.bufX[s % kRing][ty] : T(0)) : shv;
            T yn;
            // the y neighbour across the tile edge: a cluster ring entry or the
            // mailbox ring the loader filled
            T yedge = T(0);
            if (hasY) {
              if (CLU && ydin)
                yedge = cl_value<T>(*(volatile unsigned long long*)&ringY[s % kClRing][lane]);
              else
                yedge = sh.bufY[s % kRing][lane];
            }
            if (FWD)
              yn = ty > 0 ? sh.xch[(s + 1) & 1][ty - 1][lane] : yedge;
            else
              yn = ty < TY - 1 ? sh.xch[(s + 1) & 1][ty + 1][lane] : yedge;
            if constexpr (CLU) {
              // before writing entry s - (TY-1) into the consumer's ring, that
              // slot's previous entry must have been used (its step completed)
              if (rring && s >= TY - 1 && s - (TY - 1) - kClRing >= cdone) {
                int spins = 0;
                for (;;) {
                  cdone = ld_relaxed_cluster_s32(rdone);
                  if (s - (TY - 1) - kClRing < cdone) break;
                  if (++spins > slim) {
                    atomicOr(&a.sc->err, DEV_ERR_TIMEOUT);
                    break;
                  }
                }
              }
            }
            T val = T(0);
            if (valid) {
              const int64_t e = rowbase + (int64_t)cslot * rstride;
              val = op.compute(v, xn, yn, prev, e, acc);
              if (xsrc && outx) mb_store(outx + (int64_t)(s - 31) * TY + ty, val);
              if (ysrc) {
                if (CLU && rring) {
                  const int en = s - (TY - 1);
                  st_relaxed_cluster_u64(rring + (en % kClRing) * 32 + lane, cl_word<T>(t, en, val));
                } else if (outy) {
                  mb_store(outy + (int64_t)(s - (TY - 1)) * 32 + lane, val);
                }
              }
            }
            sh.xch[s & 1][ty][lane] = val;
            prev = val;
            advance(cslot);
            __syncwarp();
            if (s + kStage < NS) issue(pslot, u);
            cp_async_commit();
            advance(pslot);
            cp_async_wait<kStage - 1>();
            named_bar_sync(1, NBAR);
          }
        }
      }
      cp_async_wait<0>();
    }
    // this tile's share of the dot product (summed later in tile order, so the
    // result does not depend on which CTA swept which tile)
    {
      double v = warp_sum(acc);
      acc = 0.0;
      if (lane == 0) sh.ssum[warp] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double S = 0.0;
        for (int i = 0; i < TY + 3; i++) S += sh.ssum[i];
        a.tile_partials[tid] = S;
      }
    }
    __syncthreads();
    }  // Y < nty
    if constexpr (CLU) cooperative_groups::this_cluster().sync();  // no ring traffic crosses cluster tiles
  }
  // CTA partial of the accumulated dot product, then exit accounting.  The last
  // CTA to exit finalizes the reduction and resets the ticket counters.
  {
    if (threadIdx.x == 0) {
      __threadfence();
      int prev = atomicAdd(a.exits, 1);
      sh.last = (prev == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (sh.last && warp == 0) {
      // the tiles' shares, lane l summing tiles l, l + 32, ... in order, then a
      // fixed shuffle tree: the same sum whichever CTA gets here
      __threadfence();
      double S = 0.0;
      for (int b = lane; b < ntiles; b += 32) S += __ldcg(&a.tile_partials[b]);
      S = warp_sum(S);
      if (lane == 0) {
        *a.ticket = 0;
        *a.exits = 0;
        if (a.fin_kind != FIN_NONE) finalize(a.fin_kind, a.sc, S, 0.0);
        if (a.sc->err & DEV_ERR_TIMEOUT) a.sc->done = DONE_BREAKDOWN;
        __threadfence();
      }
    }
  }
}

template <class T, bool FWD, class Op>
constexpr size_t wave_dyn_smem() {
  return sizeof(T) * (size_t)wave_stages<T, Op::NV>() * Tiled::TY * Op::NV * 32;
}
template <class T, bool FWD, class Op>
void wave_set_attr() {
  cudaFuncSetAttribute(k_wave<T, Tiled::TY, FWD, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)wave_dyn_smem<T, FWD, Op>());
}
// Wavefront CTAs resident per SM (shared memory and registers permitting).
// Tiles are handed out in ticket order to running CTAs only, so a grid larger
// than what fits at once cannot deadlock; it just queues.
template <class T, bool FWD, class Op>
int wave_occupancy() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_wave<T, Tiled::TY, FWD, Op>, (Tiled::TY + 3) * 32,
                                                    wave_dyn_smem<T, FWD, Op>()) != cudaSuccess)
    nb = 1;
  return std::max(1, nb);
}
template <class T, bool FWD, class Op>
void launch_wave(const WaveArgs& a, const Op& op, cudaStream_t st, int grid) {
  k_wave<T, Tiled::TY, FWD, Op><<<grid, (Tiled::TY + 3) * 32, wave_dyn_smem<T, FWD, Op>(), st>>>(a, op);
}

// Cluster launches of the FP32 sweeps (CL CTAs per cluster along y).
template <int CL>
cudaLaunchAttribute cluster_attr() {
  cudaLaunchAttribute at{};
  at.id = cudaLaunchAttributeClusterDimension;
  at.val.clusterDim.x = CL;
  at.val.clusterDim.y = 1;
  at.val.clusterDim.z = 1;
  return at;
}
template <class T, bool FWD, class Op, int CL>
void wave_set_attr_cl() {
  cudaFuncSetAttribute(k_wave<T, Tiled::TY, FWD, Op, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)wave_dyn_smem<T, FWD, Op>());
  if (CL > 8) cudaFuncSetAttribute(k_wave<T, Tiled::TY, FWD, Op, CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}
// Clusters of the sweep that fit on the GPU at once (0: cannot launch).
template <class T, bool FWD, class Op, int CL>
int wave_max_clusters() {
  wave_set_attr_cl<T, FWD, Op, CL>();
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(CL * 64);
  cfg.blockDim = dim3((Tiled::TY + 3) * 32);
  cfg.dynamicSmemBytes = wave_dyn_smem<T, FWD, Op>();
  cudaLaunchAttribute at = cluster_attr<CL>();
  cfg.attrs = &at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_wave<T, Tiled::TY, FWD, Op, CL>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
template <class T, bool FWD, class Op, int CL>
void launch_wave_cl(const WaveArgs& a, const Op& op, cudaStream_t st, int nclusters) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(nclusters * CL);
  cfg.blockDim = dim3((Tiled::TY + 3) * 32);
  cfg.dynamicSmemBytes = wave_dyn_smem<T, FWD, Op>();
  cfg.stream = st;
  cudaLaunchAttribute at = cluster_attr<CL>();
  cfg.attrs = &at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_wave<T, Tiled::TY, FWD, Op, CL>, a, op);
}
// The FP32 sweep kinds (all of them take the cluster path together).
template <int CL>
int fp32_max_clusters() {
  return std::min({wave_max_clusters<float, true, FwdOp<float>, CL>(),
                   wave_max_clusters<float, false, BwdOp<float>, CL>(),
                   wave_max_clusters<float, true, FwdOp<float, true>, CL>(),
                   wave_max_clusters<float, false, BwdEisenstatOp<float>, CL>(),
                   wave_max_clusters<float, true, FwdEisenstatOp<float>, CL>()});
}

// Fill the mailboxes with the sentinel (at allocation and after an error).
template <class T>
__global__ void k_mb_reset(int64_t n, T* mb) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    mb_reset(mb + e);
}

// Per tile: 1 when any of its cells is active (one block per tile).
__global__ void __launch_bounds__(kThreads) k_tile_activity(Tiled g, const uint8_t* __restrict__ act,
                                                            uint8_t* __restrict__ tile_act) {
  // tile_elems = 256 nz bytes, and each tile starts 256-byte aligned
  const uint32_t* w = reinterpret_cast<const uint32_t*>(act + (int64_t)blockIdx.x * g.tile_elems);
  const int64_t nw = g.tile_elems / 4;
  int any = 0;
  for (int64_t i = threadIdx.x; i < nw; i += blockDim.x) any |= __ldg(w + i) != 0u;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) tile_act[blockIdx.x] = any ? 1 : 0;
}

// The sweep order of the iterations: the entries of `all` (n units in
// dependency order, tiles when CL == 0, else cluster tiles of CL tiles along
// y) whose unit holds an active tile, in the same order, each with the bits
// of its swept neighbours (x: X | bits << 16), and their count in the header
// entry dst[-1].  The dot-product shares of tiles left out are set to zero
// (nothing writes them while their unit is left out).  One block.
__global__ void __launch_bounds__(1024) k_compact_order(int ntx, int nty, int CL, const uint8_t* __restrict__ tile_act,
                                                        const int2* __restrict__ all, int n, int2* __restrict__ dst,
                                                        double* __restrict__ tile_partials) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int nyu = CL ? (nty + CL - 1) / CL : nty;
  auto swept = [&](int X, int Yu) -> bool {
    if (X < 0 || X >= ntx || Yu < 0 || Yu >= nyu) return false;
    if (!CL) return tile_act[Yu * ntx + X] != 0;
    for (int r = 0; r < CL; r++) {
      const int Y = Yu * CL + r;
      if (Y < nty && tile_act[Y * ntx + X]) return true;
    }
    return false;
  };
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int b0 = 0; b0 < n; b0 += blockDim.x) {
    const int i = b0 + threadIdx.x;
    bool on = false;
    int2 e = make_int2(0, 0);
    if (i < n) {
      const int X = all[i].x & 0xffff, Yu = all[i].y;
      on = swept(X, Yu);
      const int bits = (swept(X - 1, Yu) ? 1 : 0) | (swept(X + 1, Yu) ? 2 : 0) | (swept(X, Yu - 1) ? 4 : 0) |
                       (swept(X, Yu + 1) ? 8 : 0);
      e = make_int2(X | (bits << 16), Yu);
      if (!on)
        for (int r = 0; r < (CL ? CL : 1); r++) {
          const int Y = CL ? Yu * CL + r : Yu;
          if (Y < nty) tile_partials[Y * ntx + X] = 0.0;
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (lane == 0) wsum[warp] = __popc(m);
    __syncthreads();
    int before = carry;
    for (int w = 0; w < warp; w++) before += wsum[w];
    before += __popc(m & ((1u << lane) - 1u));
    if (on) dst[before] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += wsum[w];
      carry += t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) dst[-1] = make_int2(carry, 0);
}

// Writes a header entry (the count) followed by the units of an ntx x nyu
// grid in anti-diagonal order, each with the bits of the neighbours that
// exist, into `o` (ntx nyu + 1 entries).
void all_units_order(int ntx, int nyu, int2* o) {
  int n = 0;
  o[n++] = make_int2(ntx * nyu, 0);
  for (int d = 0; d <= ntx + nyu - 2; d++)
    for (int X = 0; X < ntx; X++) {
      const int Y = d - X;
      if (Y < 0 || Y >= nyu) continue;
      const int bits = (X > 0 ? 1 : 0) | (X < ntx - 1 ? 2 : 0) | (Y > 0 ? 4 : 0) | (Y < nyu - 1 ? 8 : 0);
      o[n++] = make_int2(X | (bits << 16), Y);
    }
}
std::vector<int2> all_units_order(int ntx, int nyu) {
  std::vector<int2> o((size_t)ntx * nyu + 1);
  all_units_order(ntx, nyu, o.data());
  return o;
}

inline int grid_for(int64_t n, int sm) {
  int64_t b = (n + kThreads - 1) / kThreads;
  int64_t cap = (int64_t)sm * 4;
  return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

// =================================================================================
// PcgSolver (host)

template <>
cudaGraphExec_t& PcgSolver::graph_for<double>(bool) {
  return graph64_;
}
template <>
cudaGraphExec_t& PcgSolver::graph_for<float>(bool eis) {
  return eis ? graph32e_ : graph32_;
}

void PcgSolver::reset_mailboxes(bool f32) {
  const int ntiles = g_.ntiles();
  const int64_t nx_ = mb_stride_x_ * ntiles, ny_ = mb_stride_y_ * ntiles;
  const int grid = grid_for(std::max(nx_, ny_), ctx_->sm_count);
  if (f32) {
    k_mb_reset<float><<<grid, kThreads, 0, ctx_->stream>>>(nx_, mbx32_);
    k_mb_reset<float><<<grid, kThreads, 0, ctx_->stream>>>(ny_, mby32_);
  } else {
    k_mb_reset<double><<<grid, kThreads, 0, ctx_->stream>>>(nx_, mbx64_);
    k_mb_reset<double><<<grid, kThreads, 0, ctx_->stream>>>(ny_, mby64_);
  }
}

// FP32 sweeps go through clusters when the solver set them up; everything
// else (FP64, or no clusters) through the plain persistent grid.
template <class T, bool FWD, class Op>
void PcgSolver::launch_sweep(const WaveArgs& a, const Op& op, cudaStream_t st, int grid) {
  if constexpr (sizeof(T) == 4) {
    if (cl_size_ > 0) {
      WaveArgs c = a;
      c.order = a.order == ws_.order_all ? order_cl_all_ : order_cl_;
      if (cl_size_ == 16)
        launch_wave_cl<T, FWD, Op, 16>(c, op, st, cl_grid_);
      else
        launch_wave_cl<T, FWD, Op, 8>(c, op, st, cl_grid_);
      return;
    }
  }
  launch_wave<T, FWD>(a, op, st, grid);
}

WaveArgs PcgSolver::wave_args(bool f32, int use_skip, int fin, bool all_tiles) const {
  WaveArgs w{};
  w.g = g_;
  w.mbx = f32 ? (void*)mbx32_ : (void*)mbx64_;
  w.mby = f32 ? (void*)mby32_ : (void*)mby64_;
  w.mb_stride_x = mb_stride_x_;
  w.mb_stride_y = mb_stride_y_;
  w.ticket = ws_.ticket;
  w.exits = ws_.exits;
  w.order = all_tiles ? ws_.order_all : ws_.order_fwd;
  w.sc = sc_;
  w.partials = partials_;
  w.tile_partials = tile_partials_;
  w.use_skip = use_skip;
  w.fin_kind = fin;
  return w;
}

int PcgSolver::spin_limit() const { return ctx_->wait_limit > 0 ? ctx_->wait_limit : kSpinLimit; }

int PcgSolver::recover_after_timeout() {
  cudaStream_t st = ctx_->stream;
  reset_mailboxes(false);
  if (have_f32_) reset_mailboxes(true);
  cudaMemsetAsync(sc_, 0, sizeof(PcgScalars), st);
  pivots_valid_ = false;
  cudaStreamSynchronize(st);
  return ctx_->set_error(-6, "wavefront wait timed out");
}

PcgSolver::PcgSolver(Context* ctx, int nx, int ny, int nz, const PcgOptions& opt)
    : ctx_(ctx), opt_(opt) {
  if (nx < 1 || ny < 1 || nz < 1) {
    init_status_ = -1;
    return;
  }
  g_ = Tiled::make(nx, ny, nz);
  wave_set_attr<double, true, PivotOp>();
  wave_set_attr<double, true, FwdOp<double>>();
  wave_set_attr<double, false, BwdOp<double>>();
  wave_set_attr<float, true, FwdOp<float>>();
  wave_set_attr<float, false, BwdOp<float>>();
  wave_set_attr<float, true, FwdOp<float, true>>();
  wave_set_attr<float, false, BwdEisenstatOp<float>>();
  wave_set_attr<float, true, FwdEisenstatOp<float>>();
  nblocks_ = ctx->sm_count * 8;
  const int ntiles = g_.ntiles();
  wave_grid_ = std::min(ntiles, ctx->sm_count);
  {
    const int occ64 = std::min(wave_occupancy<double, true, FwdOp<double>>(),
                               wave_occupancy<double, false, BwdOp<double>>());
    const int occ32 = std::min({wave_occupancy<float, true, FwdOp<float>>(),
                                wave_occupancy<float, false, BwdOp<float>>(),
                                wave_occupancy<float, true, FwdEisenstatOp<float>>(),
                                wave_occupancy<float, false, BwdEisenstatOp<float>>()});
    wave_grid64_ = std::min(ntiles, ctx->sm_count * occ64);
    wave_grid32_ = std::min(ntiles, ctx->sm_count * occ32);
  }
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    allocs_.push_back(p);
    return p;
  };
  const size_t n64 = sizeof(double) * (size_t)g_.total;
  double** arr64[] = {&d64_.adiag, &d64_.al, &d64_.ad, &d64_.ab, &d64_.E, &d64_.cL,
                      &d64_.cD,    &d64_.cB, &d64_.uR, &d64_.uU, &d64_.uF, &d64_.r,
                      &d64_.p,     &d64_.z,  &d64_.s,  &d64_.q,  &d64_.Az, &rhs_};
  for (double** a : arr64) {
    *a = (double*)alloc(n64);
    if (!*a) {
      init_status_ = -3;
      return;
    }
  }
  active_ = (uint8_t*)alloc((size_t)g_.total);
  partials_ = (double*)alloc(sizeof(double) * 2 *
                             (size_t)std::max({nblocks_, wave_grid_, wave_grid64_, wave_grid32_}));
  sc_ = (PcgScalars*)alloc(sizeof(PcgScalars));
  ws_.ticket = (int*)alloc(sizeof(int) * 2);
  tile_partials_ = (double*)alloc(sizeof(double) * (size_t)ntiles);
  tile_act_ = (uint8_t*)alloc((size_t)ntiles);
  // order lists: a header entry (the count) and up to ntiles entries
  int2* order_all = (int2*)alloc(sizeof(int2) * (size_t)(ntiles + 1));
  int2* order = (int2*)alloc(sizeof(int2) * (size_t)(ntiles + 1));
  // mailboxes (FP64; the FP32 ones are allocated with the FP32 arrays)
  const int NS = nz + 31 + Tiled::TY - 1;
  mb_stride_x_ = (int64_t)NS * Tiled::TY;
  mb_stride_y_ = (int64_t)NS * 32;
  mbx64_ = (double*)alloc(sizeof(double) * (size_t)(mb_stride_x_ * ntiles));
  mby64_ = (double*)alloc(sizeof(double) * (size_t)(mb_stride_y_ * ntiles));
  if (!active_ || !partials_ || !sc_ || !ws_.ticket || !order || !order_all || !mbx64_ || !mby64_ ||
      !tile_partials_ || !tile_act_) {
    init_status_ = -3;
    return;
  }
  ws_.exits = ws_.ticket + 1;
  ws_.order_all = order_all + 1;
  ws_.order_fwd = order + 1;
  cudaMemsetAsync(ws_.ticket, 0, sizeof(int) * 2, ctx->stream);
  for (double** a : arr64) cudaMemsetAsync(*a, 0, n64, ctx->stream);
  cudaMemsetAsync(active_, 0, (size_t)g_.total, ctx->stream);
  cudaMemsetAsync(sc_, 0, sizeof(PcgScalars), ctx->stream);
  cudaMemsetAsync(partials_, 0,
                  sizeof(double) * 2 * (size_t)std::max({nblocks_, wave_grid_, wave_grid64_, wave_grid32_}),
                  ctx->stream);
  reset_mailboxes(false);
  // tile order: anti-diagonals of the tile grid, so every tile's forward
  // predecessors (X-1,Y), (X,Y-1) hold smaller tickets; reversed for backward.
  // Until the first system selects its active tiles, both lists hold all.
  std::vector<int2> ord = all_units_order(g_.ntx, g_.nty);
  cudaMemcpyAsync(order_all, ord.data(), sizeof(int2) * ord.size(), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(order, ord.data(), sizeof(int2) * ord.size(), cudaMemcpyHostToDevice, ctx->stream);
  // FP32 sweeps in clusters of 16 (or 8) CTAs along y, when the tile rows fill
  // such clusters, the GPU can run all of them at once, and the ring stamps
  // hold the entries.  A cluster holds its CTAs until its last tile ends, so
  // when cluster tiles have to queue for free clusters (256^3 and up) the
  // plain persistent grid is faster: with clusters of 16 the 512^3 mixed solve
  // measured 2.93 s against 1.80 s without, each FP32 sweep 2.3 ms.
  if (NS < 4096) {
    for (int CL : {16, 8}) {
      if (g_.nty < CL) continue;
      const int n = CL == 16 ? fp32_max_clusters<16>() : fp32_max_clusters<8>();
      if (n < 1) continue;
      const int nyc = (g_.nty + CL - 1) / CL;
      if (g_.ntx * nyc > n) continue;
      std::vector<int2> oc = all_units_order(g_.ntx, nyc);
      int2* ca = (int2*)alloc(sizeof(int2) * oc.size());
      int2* cc = (int2*)alloc(sizeof(int2) * oc.size());
      if (!ca || !cc) break;
      cudaMemcpyAsync(ca, oc.data(), sizeof(int2) * oc.size(), cudaMemcpyHostToDevice, ctx->stream);
      cudaMemcpyAsync(cc, oc.data(), sizeof(int2) * oc.size(), cudaMemcpyHostToDevice, ctx->stream);
      order_cl_all_ = ca + 1;
      order_cl_ = cc + 1;
      cl_size_ = CL;
      cl_grid_ = std::min(n, g_.ntx * nyc);
      break;
    }
  }
  if (cudaMallocHost(&sc_host_, sizeof(PcgScalars) * 2) != cudaSuccess) {
    init_status_ = -3;
    return;
  }
  cudaEventCreate(&ev0_);
  cudaEventCreate(&ev1_);
  cudaEventCreate(&evt0_);
  cudaEventCreate(&evt1_);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) init_status_ = -2;
}

PcgSolver::~PcgSolver() {
  if (graph64_) cudaGraphExecDestroy(graph64_);
  if (graph32_) cudaGraphExecDestroy(graph32_);
  if (graph32e_) cudaGraphExecDestroy(graph32e_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (evt0_) cudaEventDestroy(evt0_);
  if (evt1_) cudaEventDestroy(evt1_);
  if (sc_host_) cudaFreeHost(sc_host_);
  for (void* p : allocs_) cudaFree(p);
}

int PcgSolver::check_dev_error(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
    return ctx_->set_error(-2, buf);
  }
  return 0;
}

// Staging buffers of the host-array entry points, allocated on first use and
// kept: a per-call stream-ordered allocation can hand its pages back at the
// solve's synchronisations and pay for mapping them again on the next call.
int PcgSolver::ensure_host_stage() {
  if (hstage_) return 0;
  const size_t N = (size_t)g_.nx * g_.ny * g_.nz;
  void *a = nullptr, *b = nullptr;
  if (cudaMalloc(&a, sizeof(double) * N) != cudaSuccess) return ctx_->set_error(-3, "staging allocation failed");
  if (cudaMalloc(&b, N) != cudaSuccess) {
    cudaFree(a);
    return ctx_->set_error(-3, "staging allocation failed");
  }
  allocs_.push_back(a);
  allocs_.push_back(b);
  hstage_ = (double*)a;
  hstage_act_ = (uint8_t*)b;
  return 0;
}

int PcgSolver::upload(const double* adiag, const double* const an[6], const double* rhs,
                      const uint8_t* active, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t N = (int64_t)g_.nx * g_.ny * g_.nz;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  const double* src[5] = {adiag, an[0], an[3], an[5], rhs};
  double* dst[5] = {d64_.adiag, d64_.al, d64_.ad, d64_.ab, rhs_};
  // staging buffers for host input (one array at a time)
  double* stage = nullptr;
  uint8_t* stage_act = nullptr;
  if (!device) {
    if (int e = ensure_host_stage()) return e;
    stage = hstage_;
    stage_act = hstage_act_;
    cudaMemcpyAsync(stage_act, active, (size_t)N, cudaMemcpyHostToDevice, st);
  }
  const uint8_t* act_ref = device ? active : stage_act;
  k_to_tiled<uint8_t, uint8_t><<<grid, kThreads, 0, st>>>(g_, act_ref, active_, nullptr);
  launches_ += 6;
  for (int a = 0; a < 5; a++) {
    const double* s = src[a];
    if (!device) {
      cudaMemcpyAsync(stage, src[a], sizeof(double) * (size_t)N, cudaMemcpyHostToDevice, st);
      s = stage;
    }
    // rhs is zeroed outside the active set (the reference never reads it there)
    k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, s, dst[a], a == 4 ? act_ref : nullptr);
  }
  int rc = 0;
  if (opt_.check_symmetry) {
    const double** dan = nullptr;
    std::vector<double*> tmp;
    double* all = nullptr;
    if (cudaMallocAsync((void**)&dan, sizeof(double*) * 6, st) != cudaSuccess)
      return ctx_->set_error(-3, "upload: allocation failed");
    const double* ptrs[6];
    if (device) {
      for (int d = 0; d < 6; d++) ptrs[d] = an[d];
    } else {
      if (cudaMallocAsync((void**)&all, sizeof(double) * (size_t)N * 6, st) != cudaSuccess)
        return ctx_->set_error(-3, "upload: allocation failed");
      for (int d = 0; d < 6; d++) {
        cudaMemcpyAsync(all + (size_t)N * d, an[d], sizeof(double) * (size_t)N,
                        cudaMemcpyHostToDevice, st);
        ptrs[d] = all + (size_t)N * d;
      }
    }
    cudaMemcpyAsync(dan, ptrs, sizeof(ptrs), cudaMemcpyHostToDevice, st);
    k_symmetry<<<nblocks_, kThreads, 0, st>>>(g_.nx, g_.ny, g_.nz, dan, act_ref, partials_, sc_);
    cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    sym_err_ = sc_host_->rinf;
    cudaFreeAsync(dan, st);
    if (all) cudaFreeAsync(all, st);
    if (sym_err_ > 1e-4) rc = -7;
  }
  pivots_valid_ = false;
  int e = check_dev_error("upload");
  if (e) return e;
  if (rc) return ctx_->set_error(rc, "upload: the matrix is not symmetric (checkSystemSymmetry)");
  return 0;
}

int PcgSolver::upload_rhs(const double* rhs, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t N = (int64_t)g_.nx * g_.ny * g_.nz;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  // active_ is already tiled; build a reference-layout mask on the fly is not
  // needed: zero rhs where the tiled mask is 0 after conversion.
  const double* s = rhs;
  double* stage = nullptr;
  if (!device) {
    if (int e = ensure_host_stage()) return e;
    stage = hstage_;
    cudaMemcpyAsync(stage, rhs, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice, st);
    s = stage;
  }
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, s, rhs_, nullptr);
  return check_dev_error("upload_rhs");
}

int PcgSolver::download_pressure(double* pg, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t N = (int64_t)g_.nx * g_.ny * g_.nz;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  const double* src = d64_.p;  // the mixed solve copies its FP64 accumulator here
  if (device) {
    k_from_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, src, pg);
    launches_ += 1;
    return check_dev_error("download_pressure");
  }
  if (int e = ensure_host_stage()) return e;
  double* stage = hstage_;
  k_from_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, src, stage);
  launches_ += 1;
  cudaMemcpyAsync(pg, stage, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_dev_error("download_pressure");
  return check_dev_error("download_pressure");
}

int PcgSolver::ensure_pivots() {
  if (pivots_valid_) return 0;
  cudaStream_t st = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  WaveArgs wa = wave_args(false, 0, FIN_NONE, true);
  // the pivot sweep reports a timeout through the status word: start it clean,
  // with this context's wait bound
  cudaMemsetAsync(&sc_->err, 0, sizeof(unsigned), st);
  pivot_limit_ = spin_limit();
  cudaMemcpyAsync(&sc_->spin_limit, &pivot_limit_, sizeof(int), cudaMemcpyHostToDevice, st);
  k_mask_system<<<grid, kThreads, 0, st>>>(g_, active_, d64_.adiag, d64_.al, d64_.ad, d64_.ab);
  // uR/uU/uF hold the pivot's diagonal products until k_upper overwrites them
  // q holds Adiag masked by the active flag until the forward sweep overwrites it
  k_pivot_diag<<<grid, kThreads, 0, st>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_,
                                          opt_.tau, d64_.q, d64_.uR, d64_.uU, d64_.uF);
  PivotOp op{{d64_.q, d64_.al, d64_.ad, d64_.ab, d64_.uR, d64_.uU, d64_.uF},
             opt_.sigma, d64_.E, d64_.cL, d64_.cD, d64_.cB};
  launch_wave<double, true>(wa, op, st, wave_grid_);
  k_upper<double><<<grid, kThreads, 0, st>>>(g_, d64_.cL, d64_.cD, d64_.cB, d64_.uR, d64_.uU,
                                              d64_.uF);
  launches_ += 4;
  {
    // the solve's scalars are set over the status word next: read it first
    unsigned* herr = reinterpret_cast<unsigned*>(sc_host_ + 1);
    cudaMemcpyAsync(herr, &sc_->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_dev_error("pivots");
    if (*herr & DEV_ERR_TIMEOUT) return recover_after_timeout();
  }
  if (opt_.precision == PREC_MIXED) {
    if (!have_f32_) {
      const size_t n32 = sizeof(float) * (size_t)g_.total;
      float** arr32[] = {&d32_.adiag, &d32_.al, &d32_.ad, &d32_.ab, &d32_.E,    &d32_.cL,
                         &d32_.cD,    &d32_.cB, &d32_.uR, &d32_.uU, &d32_.uF,   &d32_.r,
                         &d32_.p,     &d32_.z,  &d32_.s,  &d32_.q,  &d32_.Az,   &d32_.Pinv,
                         &d32_.Dt};
      for (float** a : arr32) {
        void* p = nullptr;
        if (cudaMalloc(&p, n32) != cudaSuccess) return ctx_->set_error(-3, "FP32 allocation failed");
        allocs_.push_back(p);
        *a = (float*)p;
        cudaMemsetAsync(p, 0, n32, st);
      }
      void* p = nullptr;
      if (cudaMalloc(&p, sizeof(double) * (size_t)g_.total) != cudaSuccess)
        return ctx_->set_error(-3, "FP64 accumulator allocation failed");
      allocs_.push_back(p);
      xacc_ = (double*)p;
      const int ntiles = g_.ntiles();
      void *px = nullptr, *py = nullptr;
      if (cudaMalloc(&px, sizeof(float) * (size_t)(mb_stride_x_ * ntiles)) != cudaSuccess ||
          cudaMalloc(&py, sizeof(float) * (size_t)(mb_stride_y_ * ntiles)) != cudaSuccess)
        return ctx_->set_error(-3, "FP32 mailbox allocation failed");
      allocs_.push_back(px);
      allocs_.push_back(py);
      mbx32_ = (float*)px;
      mby32_ = (float*)py;
      reset_mailboxes(true);
      have_f32_ = true;
    }
    const double* s64[] = {d64_.adiag, d64_.al, d64_.ad, d64_.ab, d64_.E, d64_.cL,
                           d64_.cD,    d64_.cB, d64_.uR, d64_.uU, d64_.uF};
    float* d32[] = {d32_.adiag, d32_.al, d32_.ad, d32_.ab, d32_.E, d32_.cL,
                    d32_.cD,    d32_.cB, d32_.uR, d32_.uU, d32_.uF};
    for (int i = 0; i < 11; i++)
      k_convert<double, float><<<grid, kThreads, 0, st>>>(g_.total, s64[i], d32[i]);
    k_eisenstat_diag<<<grid, kThreads, 0, st>>>(g_.total, d64_.E, d64_.adiag, d32_.Pinv, d32_.Dt);
    launches_ += 12;
  }
  select_active_tiles();
  int e = check_dev_error("pivots");
  if (e) return e;
  pivots_valid_ = true;
  return 0;
}

// The tiles the iteration sweeps visit: those with an active cell (with
// clusters: the cluster tiles holding one).  A tile left out is never written
// by a sweep, so the vectors the iterations carry start at zero everywhere;
// on a tile without an active cell they then stay zero, as a sweep over it
// would leave them (its pivots and couplings are zero).
void PcgSolver::select_active_tiles() {
  cudaStream_t st = ctx_->stream;
  const int ntiles = g_.ntiles();
#if SC_SKIP_EMPTY_TILES
  k_tile_activity<<<ntiles, kThreads, 0, st>>>(g_, active_, tile_act_);
#else
  cudaMemsetAsync(tile_act_, 1, (size_t)ntiles, st);  // every tile swept
#endif
  k_compact_order<<<1, 1024, 0, st>>>(g_.ntx, g_.nty, 0, tile_act_, ws_.order_all, ntiles, ws_.order_fwd,
                                      tile_partials_);
  launches_ += 2;
  if (cl_size_ > 0) {
    const int nyc = (g_.nty + cl_size_ - 1) / cl_size_;
    k_compact_order<<<1, 1024, 0, st>>>(g_.ntx, g_.nty, cl_size_, tile_act_, order_cl_all_, g_.ntx * nyc,
                                        order_cl_, tile_partials_);
    launches_ += 1;
  }
  const size_t n64 = sizeof(double) * (size_t)g_.total, n32 = sizeof(float) * (size_t)g_.total;
  for (double* v : {d64_.r, d64_.p, d64_.z, d64_.s, d64_.q, d64_.Az}) cudaMemsetAsync(v, 0, n64, st);
  if (have_f32_)
    for (float* v : {d32_.r, d32_.p, d32_.z, d32_.s, d32_.q, d32_.Az}) cudaMemsetAsync(v, 0, n32, st);
}

template <class T>
void PcgSolver::launch_spmv(SysArrays<T>& A, cudaStream_t st, int use_skip) {
  // slot runs per tile: about 12 work items per SM (3 resident blocks x 4),
  // runs of at least 16 slots; whole tiles as items left a partial last wave
  // at 512^3 (1024 tiles over 592 block slots)
  const int ntiles = g_.ntiles();
  const int want = 12 * ctx_->sm_count;
  const int chunks = std::max(1, std::min((want + ntiles - 1) / ntiles, g_.nz / 16));
  const int grid = std::min(3 * ctx_->sm_count, ntiles * chunks);
  k_spmv_stream<T><<<grid, kThreads, 0, st>>>(g_, ws_.order_fwd, A.adiag, A.al, A.ad, A.ab, active_, A.s, A.Az, partials_, sc_,
                                              use_skip, chunks);
}

template <class T>
void PcgSolver::launch_iteration(SysArrays<T>& A, bool eis) {
  cudaStream_t st = ctx_->stream;
  const bool f32 = sizeof(T) == 4;
  const int wg = sizeof(T) == 4 ? wave_grid32_ : wave_grid64_;
  if constexpr (sizeof(T) == 4) {
    if (eis) {
      // CG on L^-1 A L^-T: s = search direction, z = t = L^-T s,
      // Az = w = L^-1 A L^-T s, q = rh (split residual), p = d (FP32 correction).
      // s = rh + beta s ; t = L^-T s ; iteration count and bound
      BwdEisenstatOp<T> bo{{A.q, A.s, A.E, A.uR, A.uU, A.uF}, A.z, A.s, T(0)};
      launch_sweep<T, false>(wave_args(true, 1, FIN_SA), bo, st, wg);
      FwdEisenstatOp<T> fo{{A.s, A.z, A.Pinv, A.Dt, A.cL, A.cD, A.cB, A.E}, A.Az};
      launch_sweep<T, true>(wave_args(true, 1, FIN_SPMV), fo, st, wg);  // alpha = rho / s.w
      // x += alpha t ; rh -= alpha w ; beta = rho_new / rho
      k_axpy<T><<<nblocks_, kThreads, 0, st>>>(g_, ws_.order_fwd, A.z, A.Az, A.p, A.q, partials_, sc_,
                                               FIN_EAXPY);
      return;
    }
  }
  WaveArgs wf = wave_args(f32, 1, FIN_NONE);
  WaveArgs wb = wave_args(f32, 1, FIN_BWD);
  launch_spmv<T>(A, st, 1);
  k_axpy<T><<<nblocks_, kThreads, 0, st>>>(g_, ws_.order_fwd, A.s, A.Az, A.p, A.r, partials_, sc_);
  FwdOp<T> fo{{A.r, A.cL, A.cD, A.cB, A.E}, A.q};
  launch_sweep<T, true>(wf, fo, st, wg);
  BwdOp<T> bo{{A.q, A.E, A.uR, A.uU, A.uF, A.r}, A.z};
  launch_sweep<T, false>(wb, bo, st, wg);
  k_sa<T><<<nblocks_, kThreads, 0, st>>>(g_, ws_.order_fwd, A.z, A.s, partials_, sc_);
}

// A CUDA graph of `chunk` iterations, captured on first use.  The legacy
// default stream cannot be captured: the graph stays null then and callers
// launch the same kernels directly.
template <class T>
int PcgSolver::ensure_graph(SysArrays<T>& A, bool eis) {
  cudaGraphExec_t& gx = graph_for<T>(eis);
  if (gx) return 0;
  cudaStream_t s = ctx_->stream;
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int i = 0; i < opt_.chunk; i++) launch_iteration<T>(A, eis);
  if (cudaStreamEndCapture(s, &graph) != cudaSuccess || !graph) return check_dev_error("end capture");
  if (cudaGraphInstantiate(&gx, graph, 0) != cudaSuccess) {
    cudaGraphDestroy(graph);
    gx = nullptr;
    return check_dev_error("instantiate");
  }
  cudaGraphDestroy(graph);
  return 0;
}

template <class T>
int PcgSolver::run_pcg(SysArrays<T>& A, double tol, int criterion, int max_iter, bool scale_rhs,
                       PcgStats* st, bool eis) {
  cudaStream_t s = ctx_->stream;
  // scalars
  PcgScalars init{};
  init.spin_limit = spin_limit();
  init.tol = tol;
  init.max_iter = max_iter;
  init.criterion = criterion;
  init.done = DONE_RUNNING;
  init.first = 1;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  // r = rhs (or the scaled FP64 residual for the mixed inner solve), p = 0
  const double* src = scale_rhs ? d64_.r : rhs_;
  const double scale = scale_rhs ? 1.0 / inner_scale_ : 1.0;
  k_init<T><<<nblocks_, kThreads, 0, s>>>(g_, src, scale, active_, A.r, A.p, partials_, sc_);
  const bool f32 = sizeof(T) == 4;
  const int wg = sizeof(T) == 4 ? wave_grid32_ : wave_grid64_;
  eis = eis && f32;
  if (eis) {
    // rh = L^-1 r ; s = rh ; rho = rh.rh
    if constexpr (sizeof(T) == 4) {
      FwdOp<T, true> fo{{A.r, A.cL, A.cD, A.cB, A.E}, A.q};
      launch_sweep<T, true>(wave_args(true, 1, FIN_EINIT), fo, s, wg);
    }
    k_copy<T><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.q, A.s, sc_);
  } else {
    // z = M^-1 r ; s = z ; sigma = z.r
    FwdOp<T> fo{{A.r, A.cL, A.cD, A.cB, A.E}, A.q};
    launch_sweep<T, true>(wave_args(f32, 1, FIN_NONE), fo, s, wg);
    BwdOp<T> bo{{A.q, A.E, A.uR, A.uU, A.uF, A.r}, A.z};
    launch_sweep<T, false>(wave_args(f32, 1, FIN_BWD), bo, s, wg);
    k_copy<T><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.z, A.s, sc_);
  }
  launches_ += eis ? 3 : 4;
  int e = check_dev_error("pcg init");
  if (e) return e;
  e = ensure_graph<T>(A, eis);
  if (e) return e;
  cudaGraphExec_t gx = graph_for<T>(eis);
  const int per_iter = eis ? 3 : 5;
  // launch chunks, two in flight, until the device reports done
  const int max_chunks = max_iter / std::max(1, opt_.chunk) + 3;
  cudaEvent_t evs[2] = {ev0_, ev1_};
  int launched = 0;
  auto launch_chunk = [&](int c) {
    if (gx)
      cudaGraphLaunch(gx, s);
    else
      for (int i = 0; i < opt_.chunk; i++) launch_iteration<T>(A, eis);
    launches_ += per_iter * (uint64_t)opt_.chunk;
    cudaMemcpyAsync(&sc_host_[c & 1], sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(evs[c & 1], s);
  };
  launch_chunk(launched++);
  if (launched < max_chunks) launch_chunk(launched++);
  for (int c = 0;; c++) {
    if (cudaEventSynchronize(evs[c & 1]) != cudaSuccess) return check_dev_error("pcg chunk");
    if (sc_host_[c & 1].done != DONE_RUNNING) break;
    if (launched >= max_chunks) break;
    launch_chunk(launched++);
  }
  cudaMemcpyAsync(&sc_host_[0], sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("pcg sync");
  last_ = sc_host_[0];
  if (st) {
    st->iterations += last_.iter;
    st->status = last_.done;
    st->residual = last_.res;
    st->device_flags |= last_.err;
  }
  if (last_.err & DEV_ERR_TIMEOUT) return recover_after_timeout();
  return check_dev_error("pcg");
}

int PcgSolver::solve_fp64(PcgStats* st) {
  int e = ensure_pivots();
  if (e) return e;
  e = run_pcg<double>(d64_, opt_.tol, opt_.criterion, opt_.max_iter, false, st);
  if (e == 0 && (last_.err & DEV_ERR_NONFINITE))
    return ctx_->set_error(-8, "pcg: NaN or Inf in the system or the right-hand side");
  return e;
}

// Mixed precision with reliable updates: FP32 CG on the split system
// L^-1 A L^-T (Eisenstat's iteration) that never restarts, with the FP64
// solution and residual carried beside it.  After each graph chunk the host
// reads the recursive split residual ||rh|| / ||rh_0||; once it has dropped by
// reliable_delta since the last update (or predicts convergence), the FP32
// correction d is folded into the FP64 state, x += scale d, r -= scale A d,
// and the split residual is replaced by L^-1 r / scale, keeping the search
// direction (residual replacement in the manner of H. A. van der Vorst and
// Q. Ye, "Residual replacement strategies for Krylov subspace iterative methods
// for the convergence of true residuals", SIAM J. Sci. Comput. 22 (2000)).
// The solve stops when the FP64 residual meets the stopping test.  Replacing
// the residual breaks the identity rh.s = rh.rh that CG's step length relies
// on, so an update that did not lower the FP64 residual, or a recursion whose
// residual grew a hundredfold, restarts the search direction (s = rh).
int PcgSolver::solve_mixed_reliable(PcgStats* st) {
  int e = ensure_pivots();
  if (e) return e;
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  SysArrays<float>& A = d32_;
  const int wg = wave_grid32_;
  // x = 0 ; r = b (FP64)
  k_fill<double><<<grid, kThreads, 0, s>>>(g_.total, xacc_, 0.0);
  PcgScalars init{};
  init.spin_limit = spin_limit();
  init.tol = 0.0;  // the FP32 recursion never stops itself
  init.max_iter = opt_.max_iter;
  init.criterion = CRIT_REL_L2;
  init.done = DONE_RUNNING;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  k_init<double><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d64_.r, d64_.p, partials_, sc_,
                                               FIN_NORMS);
  launches_ += 2;
  cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed init");
  if (!std::isfinite(sc_host_->rn2)) return ctx_->set_error(-8, "mixed solve: NaN or Inf in the right-hand side");
  const bool abs_crit = opt_.criterion == CRIT_ABS_LINF;
  const double bnorm = sqrt(sc_host_->rn2);
  double meas = abs_crit ? sc_host_->rinf : (bnorm > 0 ? 1.0 : 0.0);
  int updates = 0, status = DONE_RUNNING, iters = 0, restarts = 0;
  unsigned flags = 0;
  if (meas < opt_.tol) status = DONE_CONVERGED;
  const double scale = bnorm;
  if (status == DONE_RUNNING) {
    // d = 0 ; r32 = r / scale ; rh = L^-1 r32 ; s = rh ; rho = rh.rh
    k_init<float><<<nblocks_, kThreads, 0, s>>>(g_, d64_.r, 1.0 / scale, active_, A.r, A.p, partials_, sc_);
    FwdOp<float, true> fo{{A.r, A.cL, A.cD, A.cB, A.E}, A.q};
    launch_sweep<float, true>(wave_args(true, 1, FIN_EINIT), fo, s, wg);
    k_copy<float><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.q, A.s, sc_);
    launches_ += 3;
    e = ensure_graph<float>(A, true);
    if (e) return e;
  }
  cudaGraphExec_t gx = graph_for<float>(true);
  cudaEvent_t evs[2] = {ev0_, ev1_};
  auto launch_chunk = [&](int slot) {
    if (gx)
      cudaGraphLaunch(gx, s);
    else
      for (int i = 0; i < opt_.chunk; i++) launch_iteration<float>(A, true);
    launches_ += 3 * (uint64_t)opt_.chunk;
    cudaMemcpyAsync(&sc_host_[slot], sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(evs[slot], s);
  };
  double res_u = 1.0, meas_u = meas;  // split and stopping residuals at the last update
  const int max_chunks = opt_.max_iter / std::max(1, opt_.chunk) + 3;
  int launched = 0, seen = 0;
  while (status == DONE_RUNNING) {
    // keep two chunks in flight; look at the older one
    while (launched - seen < 2 && launched < max_chunks) launch_chunk(launched++ & 1);
    if (seen == launched) {
      status = DONE_MAXITER;
      break;
    }
    if (cudaEventSynchronize(evs[seen & 1]) != cudaSuccess) return check_dev_error("mixed chunk");
    const PcgScalars h = sc_host_[seen & 1];
    seen++;
    const bool dev_stop = h.done != DONE_RUNNING || launched >= max_chunks;
    const double predicted = meas_u * h.res / res_u;
    const bool grew = !(h.res <= 100.0 * res_u);
    if (!(dev_stop || grew || h.res < opt_.reliable_delta * res_u || predicted < 0.5 * opt_.tol)) continue;
    // residual replacement after the chunks in flight
    if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed chunk");
    seen = launched;
    k_mixed_update<<<nblocks_, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_, A.p,
                                                 scale, xacc_, d64_.r, partials_, sc_);
    k_init<float><<<nblocks_, kThreads, 0, s>>>(g_, d64_.r, 1.0 / scale, active_, A.r, A.p, partials_, sc_,
                                                FIN_NONE);
    FwdOp<float, true> fo{{A.r, A.cL, A.cD, A.cB, A.E}, A.q};
    launch_sweep<float, true>(wave_args(true, 0, FIN_EREPLACE), fo, s, wg);
    launches_ += 3;
    cudaMemcpyAsync(&sc_host_[0], sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed update");
    const PcgScalars u = sc_host_[0];
    updates++;
    iters = u.iter;
    flags |= u.err;
    const double rel = bnorm > 0 ? sqrt(u.rn2) / bnorm : 0.0;
    meas = abs_crit ? u.rinf : rel;
    if (!std::isfinite(rel)) return ctx_->set_error(-8, "mixed solve: non-finite residual");
    if (u.err & DEV_ERR_TIMEOUT) return recover_after_timeout();
    if (meas < opt_.tol) {
      status = DONE_CONVERGED;
    } else if (u.done == DONE_BREAKDOWN && (!(u.err & DEV_ERR_BREAKDOWN) || (u.err & DEV_ERR_NONFINITE) ||
                                            restarts >= 4 || updates >= opt_.max_outer)) {
      status = DONE_BREAKDOWN;
    } else if (u.done == DONE_BREAKDOWN) {
      // s.w == 0: the FP32 recursion lost its search direction before the FP64
      // residual met the test; restart it from the replaced residual (s = rh)
      const int running = DONE_RUNNING;
      const unsigned keep = u.err & ~(unsigned)DEV_ERR_BREAKDOWN;
      cudaMemcpyAsync(&sc_->done, &running, sizeof(int), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(&sc_->err, &keep, sizeof(unsigned), cudaMemcpyHostToDevice, s);
      k_copy<float><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.q, A.s, sc_);
      cudaMemsetAsync(&sc_->beta, 0, sizeof(double), s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed restart");
      launches_ += 1;
      restarts++;
    } else if (u.done == DONE_MAXITER || launched >= max_chunks || updates >= opt_.max_outer) {
      status = DONE_MAXITER;
    } else if (grew || !(meas < meas_u)) {
      k_copy<float><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.q, A.s, sc_);
      cudaMemsetAsync(&sc_->beta, 0, sizeof(double), s);
      launches_ += 1;
    }
    res_u = u.res;
    meas_u = meas;
  }
  if (st) {
    st->iterations += iters;
    st->outer = updates;
    st->residual = meas;
    st->status = status;
    st->device_flags |= flags;
  }
  cudaMemcpyAsync(d64_.p, xacc_, sizeof(double) * (size_t)g_.total, cudaMemcpyDeviceToDevice, s);
  return check_dev_error("mixed");
}

int PcgSolver::solve_mixed(PcgStats* st) {
  if (opt_.inner_method == INNER_EISENSTAT) return solve_mixed_reliable(st);
  // Defect correction: FP64 residual and solution, FP32 inner MIC-PCG whose
  // pivots were computed in FP64, restarted after each correction.  Stops on
  // the FP64 residual's stopping test.
  int e = ensure_pivots();
  if (e) return e;
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  // x = 0, r = b
  k_fill<double><<<grid, kThreads, 0, s>>>(g_.total, xacc_, 0.0);
  launches_ += 2;
  PcgScalars init{};
  init.spin_limit = spin_limit();
  init.tol = 0.0;
  init.max_iter = 1;
  init.criterion = CRIT_REL_L2;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  k_init<double><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d64_.r, d64_.p, partials_,
                                               sc_);
  cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed init");
  if (!std::isfinite(sc_host_->rn2)) return ctx_->set_error(-8, "mixed solve: NaN or Inf in the right-hand side");
  const double bnorm = sqrt(sc_host_->rn2);
  double rnorm = bnorm;
  double rel = bnorm > 0 ? 1.0 : 0.0;
  int outer = 0;
  const bool abs_crit = opt_.criterion == CRIT_ABS_LINF;
  double meas = abs_crit ? sc_host_->rinf : rel;
  while (meas >= opt_.tol && outer < opt_.max_outer) {
    inner_scale_ = rnorm;
    // the inner solve only needs to reach what is still missing (with margin)
    double want = abs_crit ? opt_.inner_rtol : std::max(opt_.inner_rtol, 0.25 * opt_.tol / rel);
    PcgStats inner{};
    e = run_pcg<float>(d32_, std::min(want, 0.5), CRIT_REL_L2, opt_.max_iter, true, &inner,
                       opt_.inner_method == INNER_EISENSTAT);
    if (e) return e;
    if (st) {
      st->iterations += inner.iterations;
      st->device_flags |= inner.device_flags;
    }
    outer++;
    // x += rnorm d ; r -= rnorm A d   (FP64)
    launches_ += 1;
    k_mixed_update<<<nblocks_, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab,
                                                 active_, d32_.p, rnorm, xacc_, d64_.r, partials_,
                                                 sc_);
    cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed update");
    rnorm = sqrt(sc_host_->rn2);
    rel = bnorm > 0 ? rnorm / bnorm : 0.0;
    meas = abs_crit ? sc_host_->rinf : rel;
    if (!std::isfinite(rel)) return ctx_->set_error(-8, "mixed solve: non-finite residual");
    if (inner.status == DONE_BREAKDOWN) break;
  }
  if (st) {
    st->outer = outer;
    st->residual = meas;
    st->status = meas < opt_.tol ? DONE_CONVERGED : DONE_MAXITER;
  }
  // copy the FP64 solution into p64 for the consumers of pressure64()
  cudaMemcpyAsync(d64_.p, xacc_, sizeof(double) * (size_t)g_.total, cudaMemcpyDeviceToDevice, s);
  return check_dev_error("mixed");
}

int PcgSolver::true_residual(PcgStats* st) {
  cudaStream_t s = ctx_->stream;
  launches_ += 2;
  k_true_residual<<<nblocks_, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_,
                                                d64_.p, rhs_, partials_, sc_);
  PcgScalars* h = sc_host_ + 1;
  cudaMemcpyAsync(h, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  // ||b||
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("true residual");
  const double rn = sqrt(h->rn2), rinf = h->rinf;
  k_init<double><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d64_.Az, d64_.q, partials_,
                                               sc_);
  cudaMemcpyAsync(h, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("true residual");
  const double bn = sqrt(h->rn2);
  if (st) {
    st->true_rel_l2 = bn > 0 ? rn / bn : 0.0;
    st->true_linf = rinf;
  }
  return check_dev_error("true residual");
}

int PcgSolver::solve(PcgStats* st) {
  PcgStats local{};
  if (!st) st = &local;
  *st = PcgStats{};
  const uint64_t launches0 = launches_;
  cudaEventRecord(evt0_, ctx_->stream);
  int e = opt_.precision == PREC_MIXED ? solve_mixed(st) : solve_fp64(st);
  if (e) return e;
  if (opt_.precision == PREC_MIXED && st->status == DONE_BREAKDOWN && (st->device_flags & DEV_ERR_NONFINITE)) {
    // The FP32 recursion left the FP32 range (a preconditioner with very large
    // eigenvalues: the reference's tau terms at some dt/h) while the system is
    // finite: solve it again with the FP64 iteration.
    PcgStats f{};
    e = solve_fp64(&f);
    if (e) return e;
    st->iterations += f.iterations;
    st->status = f.status;
    st->residual = f.residual;
    st->device_flags |= f.device_flags | DEV_FLAG_FP64_RERUN;
  }
  cudaEventRecord(evt1_, ctx_->stream);
  cudaEventSynchronize(evt1_);
  float ms = 0;
  cudaEventElapsedTime(&ms, evt0_, evt1_);
  st->ms = ms;
  st->sym_err = sym_err_;
  if (opt_.true_residual) {
    e = true_residual(st);
    if (e) return e;
  }
  st->kernel_launches = (int64_t)(launches_ - launches0);
  return 0;
}

int PcgSolver::precond_only(const double* r, double* z) {
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  int e = ensure_pivots();
  if (e) return e;
  k_to_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, r, d64_.r, nullptr);
  PcgScalars init{};
  init.spin_limit = spin_limit();
  init.done = DONE_RUNNING;
  init.first = 1;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  WaveArgs wf = wave_args(false, 0, FIN_NONE);
  WaveArgs wb = wave_args(false, 0, FIN_BWD);
  FwdOp<double> fo{{d64_.r, d64_.cL, d64_.cD, d64_.cB, d64_.E}, d64_.q};
  launch_wave<double, true>(wf, fo, s, wave_grid64_);
  BwdOp<double> bo{{d64_.q, d64_.E, d64_.uR, d64_.uU, d64_.uF, d64_.r}, d64_.z};
  launch_wave<double, false>(wb, bo, s, wave_grid64_);
  k_from_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, d64_.z, z);
  cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("precond");
  last_ = *sc_host_;
  if (sc_host_->err & DEV_ERR_TIMEOUT) return recover_after_timeout();
  return check_dev_error("precond");
}

int PcgSolver::apply_only(const double* x, double* b) {
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  k_to_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, x, d64_.s, nullptr);
  k_apply_checked<<<grid, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_, d64_.s,
                                            d64_.Az);
  k_from_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, d64_.Az, b);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("apply");
  return check_dev_error("apply");
}


int PcgSolver::time_kernels(int reps, double* ms) {
  cudaStream_t s = ctx_->stream;
  int e = ensure_pivots();
  if (e) return e;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  // a benign state: r = rhs, s = r, scalars running with a tiny alpha/beta
  PcgScalars init{};
  init.spin_limit = spin_limit();
  init.done = DONE_RUNNING;
  init.first = 1;
  init.max_iter = 1 << 30;
  init.alpha = 0.0;
  init.beta = 0.0;
  init.sigma = 1.0;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  k_init<double><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d64_.r, d64_.p, partials_,
                                               sc_);
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  k_copy<double><<<grid, kThreads, 0, s>>>(g_, ws_.order_fwd, d64_.r, d64_.s, sc_);
  // The mixed solver iterates in FP32: time its FP32 kernels (the pivot sweep
  // is FP64 in both).
  const bool f32 = opt_.precision == PREC_MIXED && have_f32_;
  if (f32) {
    k_init<float><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d32_.r, d32_.p, partials_, sc_);
    cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
    k_copy<float><<<grid, kThreads, 0, s>>>(g_, ws_.order_fwd, d32_.r, d32_.s, sc_);
  }
  auto kernel = [&](auto& A, int which) {
    using T = std::remove_reference_t<decltype(*A.r)>;
    const bool is32 = sizeof(T) == 4;
    const int wg = is32 ? wave_grid32_ : wave_grid64_;
    switch (which) {
      case 1:
        this->template launch_sweep<T, true>(wave_args(is32, 0, FIN_NONE), FwdOp<T>{{A.r, A.cL, A.cD, A.cB, A.E}, A.q}, s, wg);
        break;
      case 2:
        this->template launch_sweep<T, false>(wave_args(is32, 0, FIN_NONE), BwdOp<T>{{A.q, A.E, A.uR, A.uU, A.uF, A.r}, A.z},
                              s, wg);
        break;
      case 3:
        launch_spmv<T>(A, s, 0);
        break;
      case 4:
        k_axpy<T><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.s, A.Az, A.p, A.r, partials_, sc_);
        break;
      case 5:
        k_sa<T><<<nblocks_, kThreads, 0, s>>>(g_, ws_.order_fwd, A.z, A.s, partials_, sc_);
        break;
      case 6:
        if constexpr (sizeof(T) == 4)
          this->template launch_sweep<T, false>(wave_args(true, 0, FIN_NONE),
                                BwdEisenstatOp<T>{{A.q, A.s, A.E, A.uR, A.uU, A.uF}, A.z, A.s, T(0)}, s, wg);
        break;
      case 7:
        if constexpr (sizeof(T) == 4)
          this->template launch_sweep<T, true>(wave_args(true, 0, FIN_NONE),
                               FwdEisenstatOp<T>{{A.s, A.z, A.Pinv, A.Dt, A.cL, A.cD, A.cB, A.E}, A.Az}, s, wg);
        break;
    }
  };
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  auto timed = [&](int which) -> double {
    cudaEventRecord(a, s);
    for (int i = 0; i < reps; i++) {
      switch (which) {
        case 0: {
          WaveArgs wa = wave_args(false, 0, FIN_NONE, true);
          PivotOp op{{d64_.q, d64_.al, d64_.ad, d64_.ab, d64_.uR, d64_.uU, d64_.uF},
                     opt_.sigma, d64_.E, d64_.cL, d64_.cD, d64_.cB};
          // the diag terms live in uR/uU/uF only until k_upper; rebuild them
          k_pivot_diag<<<grid, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab,
                                                 active_, opt_.tau, d64_.q, d64_.uR, d64_.uU,
                                                 d64_.uF);
          launch_wave<double, true>(wa, op, s, wave_grid_);
          k_upper<double><<<grid, kThreads, 0, s>>>(g_, d64_.cL, d64_.cD, d64_.cB, d64_.uR,
                                                    d64_.uU, d64_.uF);
          break;
        }
        default:
          if (f32)
            kernel(d32_, which);
          else
            kernel(d64_, which);
          break;
      }
    }
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    return (double)t / reps;
  };
  for (int k = 0; k < 8; k++) {
    cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
    ms[k] = (k < 6 || f32) ? timed(k) : 0.0;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  pivots_valid_ = true;
  return check_dev_error("time_kernels");
}

}  // namespace sc

// =================================================================================
// Allocation-free MIC(0) preconditioner (sc_mic_precond_noalloc_device).
//
// Some callers cannot call cudaMalloc: engines whose device memory is owned up
// front by their own pool allocator (no third-party allocations allowed), and
// hot loops where cudaMalloc's implicit device-wide synchronisation is not
// acceptable.  For them this variant of ModifiedIncompleteCholesky3D::precond
// keeps every scratch buffer it needs (the tiled copies of A, the pivots, the
// sweep couplings, the sweep outputs, the tile mailboxes and the scheduling
// counters) in the file-scope array below instead of allocating.  It launches
// the same kernels as sc_pcg_precond_device.
//
// The array is kNoAllocBytes (about 4.4 MB) and lives on every GPU that loads
// this library, until the process exits.  It bounds the problem size: at most
// kNoAllocMaxTiled tiled elements (ceil(nx/32)*32 * ceil(ny/8)*8 * nz, e.g. a
// 32^3 grid) in at most kNoAllocMaxTiles column tiles.  Every call shares the
// one array, so calls whose work overlaps on the GPU (other streams, other
// host threads) race and corrupt each other's results.
namespace sc {
namespace {

constexpr int64_t kNoAllocMaxTiled = 32768;
constexpr int kNoAllocMaxTiles = 8;
constexpr int kNoAllocMaxNS = (int)(kNoAllocMaxTiled / (Tiled::TY * 32)) + 31 + Tiled::TY - 1;
constexpr int kNoAllocArrays = 15;  // adiag al ad ab E cL cD cB uR uU uF r q z (spare)

constexpr size_t na_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kNaArrBytes = na_align(sizeof(double) * kNoAllocMaxTiled);
constexpr size_t kNaActBytes = na_align(kNoAllocMaxTiled);
constexpr size_t kNaMbxBytes = na_align(sizeof(double) * kNoAllocMaxTiles * kNoAllocMaxNS * Tiled::TY);
constexpr size_t kNaMbyBytes = na_align(sizeof(double) * kNoAllocMaxTiles * kNoAllocMaxNS * 32);
constexpr size_t kNaSmallBytes =
    na_align(sizeof(double) * kNoAllocMaxTiles + sizeof(int) * 2 + sizeof(int2) * (kNoAllocMaxTiles + 1)) +
    na_align(sizeof(PcgScalars));
constexpr size_t kNoAllocBytes =
    kNaArrBytes * kNoAllocArrays + kNaActBytes + kNaMbxBytes + kNaMbyBytes + kNaSmallBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_base[64] = {};  // device address of g_noalloc_scratch, per device

}  // namespace

// Returns 0, or a negative status with `msg` set.
int mic_precond_noalloc(cudaStream_t st, int device, int sm_count, int nx, int ny, int nz,
                        const double* adiag, const double* const* an, const double* r,
                        const uint8_t* active, double* z, double tau, double sigma,
                        std::string* msg) {
  const Tiled g = Tiled::make(nx, ny, nz);
  if (g.total > kNoAllocMaxTiled || g.ntiles() > kNoAllocMaxTiles) {
    *msg = "grid too large for the allocation-free preconditioner: at most " +
           std::to_string(kNoAllocMaxTiled) + " tiled cells (ceil(nx/32)*32 * ceil(ny/8)*8 * nz) in " +
           std::to_string(kNoAllocMaxTiles) + " tiles of 32x8 columns";
    return -1;
  }
  if (device < 0 || device >= 64) {
    *msg = "device ordinal out of range";
    return -1;
  }
  unsigned char* base = nullptr;
  {
    // One-time set-up per device (the device is current here): the device
    // address of the static array, and the shared-memory attribute of the sweeps.
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_base[device]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) {
        *msg = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
        return -2;
      }
      wave_set_attr<double, true, PivotOp>();
      wave_set_attr<double, true, FwdOp<double>>();
      wave_set_attr<double, false, BwdOp<double>>();
      g_noalloc_base[device] = ptr;
    }
    base = (unsigned char*)g_noalloc_base[device];
  }
  double* arr[kNoAllocArrays];
  for (int i = 0; i < kNoAllocArrays; i++) arr[i] = (double*)(base + kNaArrBytes * i);
  unsigned char* q = base + kNaArrBytes * kNoAllocArrays;
  uint8_t* act = (uint8_t*)q;
  q += kNaActBytes;
  double* mbx = (double*)q;
  q += kNaMbxBytes;
  double* mby = (double*)q;
  q += kNaMbyBytes;
  double* tile_partials = (double*)q;
  int* ticket = (int*)(tile_partials + kNoAllocMaxTiles);
  int2* order = (int2*)(ticket + 2);  // header entry, then the tiles
  PcgScalars* scal = (PcgScalars*)(q + na_align(sizeof(double) * kNoAllocMaxTiles + sizeof(int) * 2 +
                                                sizeof(int2) * (kNoAllocMaxTiles + 1)));
  double *t_adiag = arr[0], *t_al = arr[1], *t_ad = arr[2], *t_ab = arr[3], *t_E = arr[4],
         *t_cL = arr[5], *t_cD = arr[6], *t_cB = arr[7], *t_uR = arr[8], *t_uU = arr[9],
         *t_uF = arr[10], *t_r = arr[11], *t_q = arr[12], *t_z = arr[13];
  // The array keeps the previous call's contents: reset what must start at
  // zero (scheduling counters, scalars) and the mailbox sentinels.
  const int ntiles = g.ntiles();
  const int NS = g.nz + 31 + Tiled::TY - 1;
  const int64_t sx = (int64_t)NS * Tiled::TY, sy = (int64_t)NS * 32;
  // An error left pending by earlier, unrelated work is not this call's.
  cudaGetLastError();
  auto failed = [&](cudaError_t e, const char* step) {
    if (e == cudaSuccess) return false;
    *msg = std::string(step) + ": " + cudaGetErrorString(e);
    return true;
  };
  if (failed(cudaMemsetAsync(ticket, 0, sizeof(int) * 2, st), "clearing the tile tickets") ||
      failed(cudaMemsetAsync(scal, 0, sizeof(PcgScalars), st), "clearing the status word"))
    return -2;
  const int rgrid = grid_for(sy * ntiles, sm_count);
  k_mb_reset<double><<<rgrid, kThreads, 0, st>>>(sx * ntiles, mbx);
  k_mb_reset<double><<<rgrid, kThreads, 0, st>>>(sy * ntiles, mby);
  if (failed(cudaGetLastError(), "resetting the mailboxes")) return -2;
  // every tile is swept (the order of all tiles, its count in the header)
  int2 ord[kNoAllocMaxTiles + 1];
  all_units_order(g.ntx, g.nty, ord);
  if (failed(cudaMemcpyAsync(order, ord, sizeof(int2) * (ntiles + 1), cudaMemcpyHostToDevice, st),
             "uploading the tile order"))
    return -2;
  // system and right-hand side into the tiled layout, then the entries the
  // reference never reads (couplings to inactive cells, inactive rows) cleared
  // of non-finite values, as the allocating entry point does
  const int grid = grid_for(g.total, sm_count);
  k_to_tiled<uint8_t, uint8_t><<<grid, kThreads, 0, st>>>(g, active, act, nullptr);
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g, adiag, t_adiag, nullptr);
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g, an[0], t_al, nullptr);
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g, an[3], t_ad, nullptr);
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g, an[5], t_ab, nullptr);
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g, r, t_r, nullptr);
  k_mask_system<<<grid, kThreads, 0, st>>>(g, act, t_adiag, t_al, t_ad, t_ab);
  if (failed(cudaGetLastError(), "converting the system to the tiled layout")) return -2;
  // pivots, couplings, forward and backward sweeps
  WaveArgs wa{};
  wa.g = g;
  wa.mbx = mbx;
  wa.mby = mby;
  wa.mb_stride_x = sx;
  wa.mb_stride_y = sy;
  wa.ticket = ticket;
  wa.exits = ticket + 1;
  wa.order = order + 1;
  wa.sc = scal;
  wa.partials = tile_partials;
  wa.tile_partials = tile_partials;
  wa.use_skip = 0;
  wa.fin_kind = FIN_NONE;
  const int wgrid = std::min(ntiles, sm_count);
  k_pivot_diag<<<grid, kThreads, 0, st>>>(g, t_adiag, t_al, t_ad, t_ab, act, tau, t_q, t_uR, t_uU,
                                          t_uF);
  PivotOp pop{{t_q, t_al, t_ad, t_ab, t_uR, t_uU, t_uF}, sigma, t_E, t_cL, t_cD, t_cB};
  launch_wave<double, true>(wa, pop, st, wgrid);
  k_upper<double><<<grid, kThreads, 0, st>>>(g, t_cL, t_cD, t_cB, t_uR, t_uU, t_uF);
  FwdOp<double> fo{{t_r, t_cL, t_cD, t_cB, t_E}, t_q};
  launch_wave<double, true>(wa, fo, st, wgrid);
  BwdOp<double> bo{{t_q, t_E, t_uR, t_uU, t_uF, t_r}, t_z};
  launch_wave<double, false>(wa, bo, st, wgrid);
  k_from_tiled<double, double><<<grid, kThreads, 0, st>>>(g, t_z, z);
  if (failed(cudaGetLastError(), "launching the pivot and sweep kernels")) return -2;
  unsigned err = 0;
  if (failed(cudaMemcpyAsync(&err, &scal->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st),
             "reading the status word") ||
      failed(cudaStreamSynchronize(st), "running the preconditioner") ||
      failed(cudaGetLastError(), "running the preconditioner"))
    return -2;
  if (err & DEV_ERR_TIMEOUT) {
    *msg = "wavefront wait timed out";
    return -6;
  }
  return 0;
}

}  // namespace sc
