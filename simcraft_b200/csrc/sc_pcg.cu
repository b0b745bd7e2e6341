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
#include <vector>

#include "sc_pcg.cuh"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kRing = 64;     // boundary ring entries per wavefront CTA
constexpr int kPrefetch = 8;  // steps of input prefetch per compute warp
constexpr int kSpinLimit = 1 << 22;  // bounded waits: ~0.1-1 s, far above any legitimate wait

enum { FIN_NONE = 0, FIN_INIT, FIN_SPMV, FIN_AXPY, FIN_BWD, FIN_SA, FIN_NORMS };

__device__ void finalize(int kind, PcgScalars* sc, double sum, double mx) {
  switch (kind) {
    case FIN_INIT: {  // r = rhs; residual check before the first preconditioner (:313-319)
      sc->rn2 = sum;
      sc->rinf = mx;
      sc->bnorm = sqrt(sum);
      double res = sc->criterion == CRIT_REL_L2 ? (sc->bnorm > 0.0 ? 1.0 : 0.0) : mx;
      sc->res = res;
      sc->first = 1;
      if (!(res == res)) {
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
// Layout conversion (reference layout <-> tiled).
template <class Ts, class Td>
__global__ void k_to_tiled(Tiled g, const Ts* __restrict__ src, Td* __restrict__ dst,
                           const uint8_t* __restrict__ mask_ref) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    Td v = Td(0);
    if (g.coords(e, i, j, k)) {
      int64_t r = lin(i, j, k, g.ny, g.nz);
      if (!mask_ref || mask_ref[r]) v = (Td)src[r];
    }
    dst[e] = v;
  }
}
template <class Ts, class Td>
__global__ void k_from_tiled(Tiled g, const Ts* __restrict__ src, Td* __restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    if (g.coords(e, i, j, k)) dst[lin(i, j, k, g.ny, g.nz)] = (Td)src[e];
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
                                                   double* partials, PcgScalars* sc) {
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
  reduce_finalize(s2, mx, partials, sc, FIN_INIT);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_copy(int64_t n, const T* __restrict__ a,
                                                   T* __restrict__ b, const PcgScalars* sc) {
  if (sc->done != DONE_RUNNING) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) b[e] = a[e];
}

// applyCompressedMatrix (project-solver.cc:16-39) on the tiled layout.  The
// upper couplings come from the neighbours' lower ones (A symmetric,
// checkSystemSymmetry, :41-57).  Also accumulates x . (A x).
template <class T>
__device__ __forceinline__ T apply_row(const Tiled& g, int64_t e, int i, int j, int k,
                                       const T* __restrict__ adiag, const T* __restrict__ al,
                                       const T* __restrict__ ad, const T* __restrict__ ab,
                                       const uint8_t* __restrict__ act, const T* __restrict__ x) {
  T t = adiag[e] * x[e];
  if (i > 0) {
    int64_t o = g.off(i - 1, j, k);
    if (act[o]) t += al[e] * x[o];
  }
  if (j > 0) {
    int64_t o = g.off(i, j - 1, k);
    if (act[o]) t += ad[e] * x[o];
  }
  if (k > 0) {
    int64_t o = g.off(i, j, k - 1);
    if (act[o]) t += ab[e] * x[o];
  }
  if (i < g.nx - 1) {
    int64_t o = g.off(i + 1, j, k);
    if (act[o]) t += al[o] * x[o];
  }
  if (j < g.ny - 1) {
    int64_t o = g.off(i, j + 1, k);
    if (act[o]) t += ad[o] * x[o];
  }
  if (k < g.nz - 1) {
    int64_t o = g.off(i, j, k + 1);
    if (act[o]) t += ab[o] * x[o];
  }
  return t;
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    k_spmv(Tiled g, const T* __restrict__ adiag, const T* __restrict__ al,
           const T* __restrict__ ad, const T* __restrict__ ab, const uint8_t* __restrict__ act,
           const T* __restrict__ x, T* __restrict__ y, double* partials, PcgScalars* sc,
           int use_skip) {
  if (use_skip && sc->done != DONE_RUNNING) return;
  double acc = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    T out = T(0);
    if (g.coords(e, i, j, k) && act[e]) {
      out = apply_row(g, e, i, j, k, adiag, al, ad, ab, act, x);
      acc += (double)x[e] * (double)out;
    }
    y[e] = out;
  }
  reduce_finalize(acc, 0.0, partials, sc, FIN_SPMV);
}

// saxpy(pg, s, alpha); saxpy(r, z, -alpha); residual (:332-335, util.cc:394-402)
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_axpy(int64_t n, const uint8_t* __restrict__ act, const T* __restrict__ s,
           const T* __restrict__ Az, T* __restrict__ p, T* __restrict__ r, double* partials,
           PcgScalars* sc) {
  if (sc->done != DONE_RUNNING) return;
  const T alpha = (T)sc->alpha;
  double s2 = 0.0, mx = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    if (!act[e]) continue;
    p[e] += alpha * s[e];
    T rv = r[e] + (-alpha) * Az[e];
    r[e] = rv;
    double dv = (double)rv;
    s2 += dv * dv;
    mx = fmax(mx, fabs(dv));
  }
  reduce_finalize(s2, mx, partials, sc, FIN_AXPY);
}

// scaleAndAdd(s, z, beta): s = z + beta s (util.cc:404-410)
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_sa(int64_t n, const uint8_t* __restrict__ act, const T* __restrict__ z, T* __restrict__ s,
         double* partials, PcgScalars* sc) {
  if (sc->done != DONE_RUNNING) return;
  const T beta = (T)sc->beta;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    if (act[e]) s[e] = z[e] + beta * s[e];
  reduce_finalize(0.0, 0.0, partials, sc, FIN_SA);
}

// Upper couplings in own-cell form for the backward sweep:
// uR(p) = cL(p+x) = A_L(p+x) E(p), etc. (the products of project-solver.cc:296-302).
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_upper(Tiled g, const T* __restrict__ cL, const T* __restrict__ cD,
            const T* __restrict__ cB, T* __restrict__ uR, T* __restrict__ uU, T* __restrict__ uF) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    T a = T(0), b = T(0), c = T(0);
    if (g.coords(e, i, j, k)) {
      if (i < g.nx - 1) a = cL[g.off(i + 1, j, k)];
      if (j < g.ny - 1) b = cD[g.off(i, j + 1, k)];
      if (k < g.nz - 1) c = cB[g.off(i, j, k + 1)];
    }
    uR[e] = a;
    uU[e] = b;
    uF[e] = c;
  }
}

// b - A x in FP64 (norms only): the true residual of the final iterate.
__global__ void __launch_bounds__(kThreads)
    k_true_residual(Tiled g, const double* __restrict__ adiag, const double* __restrict__ al,
                    const double* __restrict__ ad, const double* __restrict__ ab,
                    const uint8_t* __restrict__ act, const double* __restrict__ x,
                    const double* __restrict__ b, double* partials, PcgScalars* sc) {
  double s2 = 0.0, mx = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    if (g.coords(e, i, j, k) && act[e]) {
      double rv = b[e] - apply_row(g, e, i, j, k, adiag, al, ad, ab, act, x);
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
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < g.total; e += stride) {
    int i, j, k;
    if (!(g.coords(e, i, j, k) && act[e])) continue;
    double t = adiag[e] * (double)d[e];
    if (i > 0) {
      int64_t o = g.off(i - 1, j, k);
      if (act[o]) t += al[e] * (double)d[o];
    }
    if (j > 0) {
      int64_t o = g.off(i, j - 1, k);
      if (act[o]) t += ad[e] * (double)d[o];
    }
    if (k > 0) {
      int64_t o = g.off(i, j, k - 1);
      if (act[o]) t += ab[e] * (double)d[o];
    }
    if (i < g.nx - 1) {
      int64_t o = g.off(i + 1, j, k);
      if (act[o]) t += al[o] * (double)d[o];
    }
    if (j < g.ny - 1) {
      int64_t o = g.off(i, j + 1, k);
      if (act[o]) t += ad[o] * (double)d[o];
    }
    if (k < g.nz - 1) {
      int64_t o = g.off(i, j, k + 1);
      if (act[o]) t += ab[o] * (double)d[o];
    }
    x[e] += scale * (double)d[e];
    double rv = r[e] - scale * t;
    r[e] = rv;
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

struct WaveArgs {
  Tiled g;
  int* progress;
  int* ticket;
  int* exits;
  const int2* order;
  PcgScalars* sc;
  double* partials;
  int use_skip;
  int fin_kind;
};

template <class T>
struct FwdOp {  // L q = r (project-solver.cc:276-288), c* = A_* E(neighbour)
  const T *r, *cL, *cD, *cB, *E;
  T* out;
  struct In {
    T r, cL, cD, cB, E;
  };
  __device__ __forceinline__ In load(int64_t e) const {
    return In{__ldg(r + e), __ldg(cL + e), __ldg(cD + e), __ldg(cB + e), __ldg(E + e)};
  }
  __device__ __forceinline__ T compute(const In& in, T xn, T yn, T zn, int, int, int, int64_t,
                                       double&) const {
    T t = in.r;
    t -= in.cL * xn;
    t -= in.cD * yn;
    t -= in.cB * zn;
    return t * in.E;
  }
};

template <class T>
struct BwdOp {  // L^T z = q (project-solver.cc:293-305), u* = A_*(p+dir) E(p); sigma = z.r
  const T *q, *E, *uR, *uU, *uF, *r;
  T* out;
  struct In {
    T q, E, uR, uU, uF, r;
  };
  __device__ __forceinline__ In load(int64_t e) const {
    return In{__ldg(q + e), __ldg(E + e), __ldg(uR + e), __ldg(uU + e), __ldg(uF + e), __ldg(r + e)};
  }
  __device__ __forceinline__ T compute(const In& in, T xn, T yn, T zn, int, int, int, int64_t,
                                       double& acc) const {
    T t = in.q;
    t -= in.uR * xn;
    t -= in.uU * yn;
    t -= in.uF * zn;
    T v = t * in.E;
    acc += (double)v * (double)in.r;
    return v;
  }
};

// MIC(0) pivot (project-solver.cc:237-274), FP64.  The exchanged value is E.
// E(q) != 0 exactly when q is active with Adiag(q) != 0, which is the guard the
// reference tests before using E(q).
struct PivotOp {
  Tiled g;
  const double *adiag, *al, *ad, *ab;
  const uint8_t* act;
  double tau, sigma;
  double *out, *cL, *cD, *cB;
  struct In {
    double adiag, al, ad, ab;
    int act;
  };
  __device__ __forceinline__ In load(int64_t e) const {
    return In{__ldg(adiag + e), __ldg(al + e), __ldg(ad + e), __ldg(ab + e), (int)__ldg(act + e)};
  }
  __device__ __forceinline__ double compute(const In& in, double EL, double ED, double EB, int x,
                                            int y, int z, int64_t e, double&) const {
    double E = 0.0;
    if (in.act && in.adiag != 0.0) {
      double ee = in.adiag;
      if (EL != 0.0) {
        ee -= (in.al * EL) * (in.al * EL);
        if (y < g.ny - 1) {
          int64_t o = g.off(x - 1, y + 1, z);
          if (act[o]) ee -= tau * in.al * al[o] / (EL * EL);
        }
        if (z < g.nz - 1) {
          int64_t o = g.off(x - 1, y, z + 1);
          if (act[o]) ee -= tau * in.al * al[o] / (EL * EL);
        }
      }
      if (ED != 0.0) {
        ee -= (in.ad * ED) * (in.ad * ED);
        if (x < g.nx - 1) {
          int64_t o = g.off(x + 1, y - 1, z);
          if (act[o]) ee -= tau * in.ad * ad[o] / (ED * ED);
        }
        if (z < g.nz - 1) {
          int64_t o = g.off(x, y - 1, z + 1);
          if (act[o]) ee -= tau * in.ad * ad[o] / (ED * ED);
        }
      }
      if (EB != 0.0) {
        ee -= (in.ab * EB) * (in.ab * EB);
        if (x < g.nx - 1) {
          int64_t o = g.off(x + 1, y, z - 1);
          if (act[o]) ee -= tau * in.ab * ab[o] / (EB * EB);
        }
        if (y < g.ny - 1) {
          int64_t o = g.off(x, y + 1, z - 1);
          if (act[o]) ee -= tau * in.ab * ab[o] / (EB * EB);
        }
      }
      if (ee < sigma * in.adiag) ee = in.adiag;
      E = 1.0 / sqrt(ee);
    }
    cL[e] = in.al * EL;
    cD[e] = in.ad * ED;
    cB[e] = in.ab * EB;
    return E;
  }
};

template <class T, int TY, bool FWD>
__device__ __forceinline__ int wave_slot(const Tiled& g, int s, int ty) {
  return FWD ? wrap_mod(s - ty, g.nz) : wrap_mod(g.nz + 29 + TY - s - ty, g.nz);
}

template <class T, int TY, bool FWD>
__device__ void wave_comm(const WaveArgs& a, const T* out, int tile_id, int tileX_id,
                          int tileY_id, int64_t baseX, int64_t baseY, bool hasX, bool hasY,
                          int NS, T (*bufX)[TY], T (*bufY)[32], volatile int* s_done,
                          volatile int* s_availX, volatile int* s_availY, volatile int* s_abort) {
  const Tiled& g = a.g;
  const int lane = threadIdx.x & 31;
  int pub = 0;
  int lx = hasX ? 0 : NS, ly = hasY ? 0 : NS;
  int seenX = 0, seenY = 0;
  int spins = 0;
  int* my_prog = a.progress + tile_id;
  for (;;) {
    bool worked = false;
    const int d = *s_done;
    if (d > pub) {
      __threadfence();
      if (lane == 0) st_release_gpu(my_prog, d);
      pub = d;
      worked = true;
    }
    const int want = min(NS, d + kRing);
    if (lx < want) {
      // entry e needs the neighbour's step e+31 done (progress >= e+32); the
      // neighbour's final progress NS releases every remaining entry.
      int availX = seenX >= NS ? NS : seenX - 31;
      if (lx >= availX) {
        int v = lane == 0 ? ld_acquire_gpu(a.progress + tileX_id) : 0;
        seenX = __shfl_sync(kFull, v, 0);
        __syncwarp();
        availX = seenX >= NS ? NS : seenX - 31;
      }
      const int hi = min(want, availX);
      if (hi > lx) {
        const int cnt = (hi - lx) * TY;
        for (int i = lane; i < cnt; i += 32) {
          const int e = lx + i / TY, ty = i % TY;
          T val = T(0);
          if (FWD) {
            const int z = e - ty;
            if (z >= 0 && z < g.nz)
              val = ld_cg(out + baseX + ((int64_t)wrap_mod(z + 31, g.nz) * TY + ty) * 32 + 31);
          } else {
            const int z = g.nz - 1 - e + (TY - 1 - ty);
            if (z >= 0 && z < g.nz) val = ld_cg(out + baseX + ((int64_t)z * TY + ty) * 32);
          }
          bufX[e % kRing][ty] = val;
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) *s_availX = hi;
        lx = hi;
        worked = true;
      }
    }
    if (ly < want) {
      // entry e needs the neighbour's step e+TY-1 done (progress >= e+TY)
      int availY = seenY >= NS ? NS : seenY - TY + 1;
      if (ly >= availY) {
        int v = lane == 0 ? ld_acquire_gpu(a.progress + tileY_id) : 0;
        seenY = __shfl_sync(kFull, v, 0);
        __syncwarp();
        availY = seenY >= NS ? NS : seenY - TY + 1;
      }
      const int hi = min(want, availY);
      if (hi > ly) {
        for (int e = ly; e < hi; e++) {
          const int slot = FWD ? wrap_mod(e, g.nz) : wrap_mod(g.nz + 30 - e, g.nz);
          const int row = FWD ? TY - 1 : 0;
          bufY[e % kRing][lane] = ld_cg(out + baseY + ((int64_t)slot * TY + row) * 32 + lane);
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) *s_availY = hi;
        ly = hi;
        worked = true;
      }
    }
    if (pub >= NS && lx >= NS && ly >= NS) break;
    if (*s_abort) {
      if (lane == 0) {
        st_release_gpu(my_prog, NS);
        *s_availX = NS;
        *s_availY = NS;
      }
      break;
    }
    if (worked) {
      spins = 0;
    } else {
      if (++spins > kSpinLimit || (((spins & 255) == 0) && ld_relaxed_gpu_u32(&a.sc->err))) {
        if (lane == 0) {
          atomicOr(&a.sc->err, DEV_ERR_TIMEOUT);
          *s_abort = 1;
          st_release_gpu(my_prog, NS);
          *s_availX = NS;
          *s_availY = NS;
        }
        break;
      }
      __nanosleep(32);
    }
  }
}

template <class T, int TY, bool FWD, class Op>
__global__ void __launch_bounds__((TY + 1) * 32, 1) k_wave(const WaveArgs a, const Op op) {
  constexpr int NTC = TY * 32;
  __shared__ T xch[2][TY][32];
  __shared__ T bufX[kRing][TY];
  __shared__ T bufY[kRing][32];
  __shared__ volatile int s_done, s_availX, s_availY, s_abort;
  __shared__ int s_tile;
  __shared__ bool s_last;
  if (a.use_skip && a.sc->done != DONE_RUNNING) return;
  if (a.sc->err & DEV_ERR_TIMEOUT) return;  // an earlier sweep gave up: do not wait again
  const Tiled& g = a.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = g.ntx * g.nty;
  const int NS = g.nz + 31 + TY - 1;
  double acc = 0.0;
  for (;;) {
    if (threadIdx.x == 0) {
      s_tile = atomicAdd(a.ticket, 1);
      s_done = 0;
      s_availX = 0;
      s_availY = 0;
      s_abort = 0;
    }
    __syncthreads();
    const int t = s_tile;
    if (t >= ntiles) break;
    const int2 XY = a.order[FWD ? t : ntiles - 1 - t];
    const int X = XY.x, Y = XY.y;
    const bool hasX = FWD ? (X > 0) : (X < g.ntx - 1);
    const bool hasY = FWD ? (Y > 0) : (Y < g.nty - 1);
    const int Xn = FWD ? X - 1 : X + 1, Yn = FWD ? Y - 1 : Y + 1;
    const int64_t base = g.tile_base(X, Y);
    if (warp == TY) {
      wave_comm<T, TY, FWD>(a, op.out, Y * g.ntx + X, hasX ? Y * g.ntx + Xn : 0,
                            hasY ? Yn * g.ntx + X : 0, hasX ? g.tile_base(Xn, Y) : 0,
                            hasY ? g.tile_base(X, Yn) : 0, hasX, hasY, NS, bufX, bufY, &s_done,
                            &s_availX, &s_availY, &s_abort);
    } else {
      const int ty = warp;
      const int x = X * 32 + lane, y = Y * TY + ty;
      typename Op::In ring[kPrefetch];
#pragma unroll
      for (int u = 0; u < kPrefetch; u++)
        if (u < NS)
          ring[u] = op.load(base + ((int64_t)wave_slot<T, TY, FWD>(g, u, ty) * TY + ty) * 32 + lane);
      T prev = T(0);
      auto wait_avail = [&](int s) {
        int spins = 0;
        while (((hasX && s_availX <= s) || (hasY && s_availY <= s)) && !s_abort) {
          if (++spins > kSpinLimit) {
            atomicOr(&a.sc->err, DEV_ERR_TIMEOUT);
            s_abort = 1;
            break;
          }
          __nanosleep(20);
        }
        __threadfence_block();
      };
      if (threadIdx.x == 0) wait_avail(0);
      named_bar_sync(1, NTC);
      for (int s0 = 0; s0 < NS; s0 += kPrefetch) {
#pragma unroll
        for (int u = 0; u < kPrefetch; u++) {
          const int s = s0 + u;
          if (s < NS) {
            const typename Op::In in = ring[u];
            if (s + kPrefetch < NS)
              ring[u] = op.load(
                  base + ((int64_t)wave_slot<T, TY, FWD>(g, s + kPrefetch, ty) * TY + ty) * 32 + lane);
            const int z = FWD ? (s - ty - lane) : (g.nz - 1 - (s - (TY - 1 - ty) - (31 - lane)));
            const bool valid = (z >= 0) && (z < g.nz);
            const T sh = FWD ? __shfl_up_sync(kFull, prev, 1) : __shfl_down_sync(kFull, prev, 1);
            const bool xedge = FWD ? (lane == 0) : (lane == 31);
            const T xn = xedge ? (hasX ? bufX[s % kRing][ty] : T(0)) : sh;
            T yn;
            if (FWD)
              yn = ty > 0 ? xch[(s + 1) & 1][ty - 1][lane] : (hasY ? bufY[s % kRing][lane] : T(0));
            else
              yn = ty < TY - 1 ? xch[(s + 1) & 1][ty + 1][lane]
                               : (hasY ? bufY[s % kRing][lane] : T(0));
            T val = T(0);
            if (valid) {
              const int64_t e = base + ((int64_t)wave_slot<T, TY, FWD>(g, s, ty) * TY + ty) * 32 + lane;
              val = op.compute(in, xn, yn, prev, x, y, z, e, acc);
              op.out[e] = val;
            }
            xch[s & 1][ty][lane] = val;
            prev = val;
            if (threadIdx.x == 0) {
              __threadfence_block();
              s_done = s;
              if (s + 1 < NS) wait_avail(s + 1);
            }
            named_bar_sync(1, NTC);
          }
        }
      }
      if (threadIdx.x == 0) {
        __threadfence_block();
        s_done = NS;
      }
    }
    __syncthreads();
  }
  // CTA partial of the accumulated dot product, then exit accounting.  The last
  // CTA to exit finalizes the reduction and resets the scheduling state.
  {
    __shared__ double ssum[(TY + 1)];
    double v = warp_sum(acc);
    if (lane == 0) ssum[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double S = 0.0;
      for (int i = 0; i < TY + 1; i++) S += ssum[i];
      a.partials[2 * blockIdx.x] = S;
      a.partials[2 * blockIdx.x + 1] = 0.0;
      __threadfence();
      int prev = atomicAdd(a.exits, 1);
      s_last = (prev == (int)gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      for (int i = threadIdx.x; i < ntiles; i += blockDim.x) a.progress[i] = 0;
      if (threadIdx.x == 0) {
        double S = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) S += __ldcg(&a.partials[2 * b]);
        *a.ticket = 0;
        *a.exits = 0;
        if (a.fin_kind != FIN_NONE) finalize(a.fin_kind, a.sc, S, 0.0);
        if (a.sc->err & DEV_ERR_TIMEOUT) a.sc->done = DONE_BREAKDOWN;
      }
      __threadfence();
    }
  }
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
cudaGraphExec_t& PcgSolver::graph_for<double>() {
  return graph64_;
}
template <>
cudaGraphExec_t& PcgSolver::graph_for<float>() {
  return graph32_;
}

PcgSolver::PcgSolver(Context* ctx, int nx, int ny, int nz, const PcgOptions& opt)
    : ctx_(ctx), opt_(opt) {
  if (nx < 1 || ny < 1 || nz < 1) {
    init_status_ = -1;
    return;
  }
  g_ = Tiled::make(nx, ny, nz, kTY);
  nblocks_ = ctx->sm_count * 4;
  const int ntiles = g_.ntx * g_.nty;
  wave_grid_ = std::min(ntiles, ctx->sm_count);
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
  partials_ = (double*)alloc(sizeof(double) * 2 * (size_t)std::max(nblocks_, wave_grid_));
  sc_ = (PcgScalars*)alloc(sizeof(PcgScalars));
  ws_.progress = (int*)alloc(sizeof(int) * (size_t)(ntiles + 2));
  int2* order = (int2*)alloc(sizeof(int2) * (size_t)ntiles);
  if (!active_ || !partials_ || !sc_ || !ws_.progress || !order) {
    init_status_ = -3;
    return;
  }
  ws_.ticket = ws_.progress + ntiles;
  ws_.exits = ws_.progress + ntiles + 1;
  ws_.order_fwd = order;
  cudaMemsetAsync(ws_.progress, 0, sizeof(int) * (size_t)(ntiles + 2), ctx->stream);
  cudaMemsetAsync(d64_.adiag, 0, n64, ctx->stream);
  for (double** a : arr64) cudaMemsetAsync(*a, 0, n64, ctx->stream);
  cudaMemsetAsync(active_, 0, (size_t)g_.total, ctx->stream);
  cudaMemsetAsync(sc_, 0, sizeof(PcgScalars), ctx->stream);
  // tile order: anti-diagonals of the tile grid, so every tile's forward
  // predecessors (X-1,Y), (X,Y-1) hold smaller tickets; reversed for backward.
  std::vector<int2> ord;
  ord.reserve(ntiles);
  for (int d = 0; d <= g_.ntx + g_.nty - 2; d++)
    for (int X = 0; X < g_.ntx; X++) {
      int Y = d - X;
      if (Y >= 0 && Y < g_.nty) ord.push_back(make_int2(X, Y));
    }
  cudaMemcpyAsync(order, ord.data(), sizeof(int2) * ord.size(), cudaMemcpyHostToDevice,
                  ctx->stream);
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
    if (cudaMallocAsync(&stage, sizeof(double) * (size_t)N, st) != cudaSuccess ||
        cudaMallocAsync(&stage_act, (size_t)N, st) != cudaSuccess)
      return ctx_->set_error(-3, "upload: staging allocation failed");
    cudaMemcpyAsync(stage_act, active, (size_t)N, cudaMemcpyHostToDevice, st);
  }
  const uint8_t* act_ref = device ? active : stage_act;
  k_to_tiled<uint8_t, uint8_t><<<grid, kThreads, 0, st>>>(g_, act_ref, active_, nullptr);
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
  if (stage) cudaFreeAsync(stage, st);
  if (stage_act) cudaFreeAsync(stage_act, st);
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
    if (cudaMallocAsync(&stage, sizeof(double) * (size_t)N, st) != cudaSuccess)
      return ctx_->set_error(-3, "upload_rhs: staging allocation failed");
    cudaMemcpyAsync(stage, rhs, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice, st);
    s = stage;
  }
  k_to_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, s, rhs_, nullptr);
  if (stage) cudaFreeAsync(stage, st);
  return check_dev_error("upload_rhs");
}

int PcgSolver::download_pressure(double* pg, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t N = (int64_t)g_.nx * g_.ny * g_.nz;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  const double* src = d64_.p;  // the mixed solve copies its FP64 accumulator here
  if (device) {
    k_from_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, src, pg);
    return check_dev_error("download_pressure");
  }
  double* stage = nullptr;
  if (cudaMallocAsync(&stage, sizeof(double) * (size_t)N, st) != cudaSuccess)
    return ctx_->set_error(-3, "download: staging allocation failed");
  k_from_tiled<double, double><<<grid, kThreads, 0, st>>>(g_, src, stage);
  cudaMemcpyAsync(pg, stage, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(stage, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_dev_error("download_pressure");
  return check_dev_error("download_pressure");
}

int PcgSolver::ensure_pivots() {
  if (pivots_valid_) return 0;
  cudaStream_t st = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  WaveArgs wa{g_, ws_.progress, ws_.ticket, ws_.exits, ws_.order_fwd, sc_, partials_, 0, FIN_NONE};
  PivotOp op{g_,         d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_, opt_.tau,
             opt_.sigma, d64_.E,     d64_.cL, d64_.cD, d64_.cB};
  k_wave<double, kTY, true, PivotOp><<<wave_grid_, (kTY + 1) * 32, 0, st>>>(wa, op);
  k_upper<double><<<grid, kThreads, 0, st>>>(g_, d64_.cL, d64_.cD, d64_.cB, d64_.uR, d64_.uU,
                                              d64_.uF);
  if (opt_.precision == PREC_MIXED) {
    if (!have_f32_) {
      const size_t n32 = sizeof(float) * (size_t)g_.total;
      float** arr32[] = {&d32_.adiag, &d32_.al, &d32_.ad, &d32_.ab, &d32_.E, &d32_.cL,
                         &d32_.cD,    &d32_.cB, &d32_.uR, &d32_.uU, &d32_.uF, &d32_.r,
                         &d32_.p,     &d32_.z,  &d32_.s,  &d32_.q,  &d32_.Az};
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
      have_f32_ = true;
    }
    const double* s64[] = {d64_.adiag, d64_.al, d64_.ad, d64_.ab, d64_.E, d64_.cL,
                           d64_.cD,    d64_.cB, d64_.uR, d64_.uU, d64_.uF};
    float* d32[] = {d32_.adiag, d32_.al, d32_.ad, d32_.ab, d32_.E, d32_.cL,
                    d32_.cD,    d32_.cB, d32_.uR, d32_.uU, d32_.uF};
    for (int i = 0; i < 11; i++)
      k_convert<double, float><<<grid, kThreads, 0, st>>>(g_.total, s64[i], d32[i]);
  }
  int e = check_dev_error("pivots");
  if (e) return e;
  pivots_valid_ = true;
  return 0;
}

template <class T>
void PcgSolver::launch_iteration(SysArrays<T>& A) {
  cudaStream_t st = ctx_->stream;
  WaveArgs wf{g_, ws_.progress, ws_.ticket, ws_.exits, ws_.order_fwd, sc_, partials_, 1, FIN_NONE};
  WaveArgs wb = wf;
  wb.fin_kind = FIN_BWD;
  k_spmv<T><<<nblocks_, kThreads, 0, st>>>(g_, A.adiag, A.al, A.ad, A.ab, active_, A.s, A.Az,
                                            partials_, sc_, 1);
  k_axpy<T><<<nblocks_, kThreads, 0, st>>>(g_.total, active_, A.s, A.Az, A.p, A.r, partials_, sc_);
  FwdOp<T> fo{A.r, A.cL, A.cD, A.cB, A.E, A.q};
  k_wave<T, kTY, true, FwdOp<T>><<<wave_grid_, (kTY + 1) * 32, 0, st>>>(wf, fo);
  BwdOp<T> bo{A.q, A.E, A.uR, A.uU, A.uF, A.r, A.z};
  k_wave<T, kTY, false, BwdOp<T>><<<wave_grid_, (kTY + 1) * 32, 0, st>>>(wb, bo);
  k_sa<T><<<nblocks_, kThreads, 0, st>>>(g_.total, active_, A.z, A.s, partials_, sc_);
}

template <class T>
int PcgSolver::run_pcg(SysArrays<T>& A, double tol, int criterion, int max_iter, bool scale_rhs,
                       PcgStats* st) {
  cudaStream_t s = ctx_->stream;
  // scalars
  PcgScalars init{};
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
  // z = M^-1 r ; s = z ; sigma = z.r
  WaveArgs wf{g_, ws_.progress, ws_.ticket, ws_.exits, ws_.order_fwd, sc_, partials_, 1, FIN_NONE};
  WaveArgs wb = wf;
  wb.fin_kind = FIN_BWD;
  FwdOp<T> fo{A.r, A.cL, A.cD, A.cB, A.E, A.q};
  k_wave<T, kTY, true, FwdOp<T>><<<wave_grid_, (kTY + 1) * 32, 0, s>>>(wf, fo);
  BwdOp<T> bo{A.q, A.E, A.uR, A.uU, A.uF, A.r, A.z};
  k_wave<T, kTY, false, BwdOp<T>><<<wave_grid_, (kTY + 1) * 32, 0, s>>>(wb, bo);
  k_copy<T><<<nblocks_, kThreads, 0, s>>>(g_.total, A.z, A.s, sc_);
  int e = check_dev_error("pcg init");
  if (e) return e;
  // graph of `chunk` iterations
  cudaGraphExec_t& gx = graph_for<T>();
  if (!gx) {
    cudaGraph_t graph;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return check_dev_error("begin capture");
    for (int i = 0; i < opt_.chunk; i++) launch_iteration<T>(A);
    if (cudaStreamEndCapture(s, &graph) != cudaSuccess) return check_dev_error("end capture");
    if (cudaGraphInstantiate(&gx, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      return check_dev_error("instantiate");
    }
    cudaGraphDestroy(graph);
  }
  // launch chunks, two in flight, until the device reports done
  const int max_chunks = max_iter / std::max(1, opt_.chunk) + 3;
  cudaEvent_t evs[2] = {ev0_, ev1_};
  int launched = 0;
  auto launch_chunk = [&](int c) {
    cudaGraphLaunch(gx, s);
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
  }
  if (last_.err & DEV_ERR_TIMEOUT) return ctx_->set_error(-6, "wavefront wait timed out");
  return check_dev_error("pcg");
}

int PcgSolver::solve_fp64(PcgStats* st) {
  int e = ensure_pivots();
  if (e) return e;
  return run_pcg<double>(d64_, opt_.tol, opt_.criterion, opt_.max_iter, false, st);
}

int PcgSolver::solve_mixed(PcgStats* st) {
  // Defect correction: FP64 residual and solution, FP32 inner MIC-PCG whose
  // pivots were computed in FP64.  Stops on ||b - A x||_2 / ||b||_2 < tol.
  int e = ensure_pivots();
  if (e) return e;
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  // x = 0, r = b
  k_fill<double><<<grid, kThreads, 0, s>>>(g_.total, xacc_, 0.0);
  PcgScalars init{};
  init.tol = 0.0;
  init.max_iter = 1;
  init.criterion = CRIT_REL_L2;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  k_init<double><<<nblocks_, kThreads, 0, s>>>(g_, rhs_, 1.0, active_, d64_.r, d64_.p, partials_,
                                               sc_);
  cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("mixed init");
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
    e = run_pcg<float>(d32_, std::min(want, 0.5), CRIT_REL_L2, opt_.max_iter, true, &inner);
    if (e) return e;
    if (st) st->iterations += inner.iterations;
    outer++;
    // x += rnorm d ; r -= rnorm A d   (FP64)
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
  cudaEventRecord(evt0_, ctx_->stream);
  int e = opt_.precision == PREC_MIXED ? solve_mixed(st) : solve_fp64(st);
  if (e) return e;
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
  return 0;
}

int PcgSolver::precond_only(const double* r, double* z) {
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  int e = ensure_pivots();
  if (e) return e;
  k_to_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, r, d64_.r, nullptr);
  PcgScalars init{};
  init.done = DONE_RUNNING;
  init.first = 1;
  cudaMemcpyAsync(sc_, &init, sizeof(PcgScalars), cudaMemcpyHostToDevice, s);
  WaveArgs wf{g_, ws_.progress, ws_.ticket, ws_.exits, ws_.order_fwd, sc_, partials_, 0, FIN_NONE};
  WaveArgs wb = wf;
  wb.fin_kind = FIN_BWD;
  FwdOp<double> fo{d64_.r, d64_.cL, d64_.cD, d64_.cB, d64_.E, d64_.q};
  k_wave<double, kTY, true, FwdOp<double>><<<wave_grid_, (kTY + 1) * 32, 0, s>>>(wf, fo);
  BwdOp<double> bo{d64_.q, d64_.E, d64_.uR, d64_.uU, d64_.uF, d64_.r, d64_.z};
  k_wave<double, kTY, false, BwdOp<double>><<<wave_grid_, (kTY + 1) * 32, 0, s>>>(wb, bo);
  k_from_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, d64_.z, z);
  cudaMemcpyAsync(sc_host_, sc_, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("precond");
  if (sc_host_->err & DEV_ERR_TIMEOUT) return ctx_->set_error(-6, "wavefront wait timed out");
  return check_dev_error("precond");
}

int PcgSolver::apply_only(const double* x, double* b) {
  cudaStream_t s = ctx_->stream;
  const int grid = grid_for(g_.total, ctx_->sm_count);
  k_to_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, x, d64_.s, nullptr);
  k_spmv<double><<<nblocks_, kThreads, 0, s>>>(g_, d64_.adiag, d64_.al, d64_.ad, d64_.ab, active_,
                                               d64_.s, d64_.Az, partials_, sc_, 0);
  k_from_tiled<double, double><<<grid, kThreads, 0, s>>>(g_, d64_.Az, b);
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_dev_error("apply");
  return check_dev_error("apply");
}

}  // namespace sc
