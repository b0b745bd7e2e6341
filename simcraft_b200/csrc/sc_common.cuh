// sc_common.cuh -- shared device helpers for the SimCraft FluidSim B200 path.
//
// Grid layout conventions (identical to spatify::LinearHashXYZ,
// Spatify/include/Spatify/hash.h:25):  idx(i,j,k) = k + j*sz + i*sy*sz.
// Face grids: u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1)
// (Spatify/include/Spatify/grids.h:245-256, 479-485).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

// Device error bits written into a status word by kernels; the host turns them
// into C-ABI status codes.  No kernel traps or asserts.
enum : unsigned {
  DEV_ERR_TIMEOUT = 1u,     // a bounded spin-wait gave up
  DEV_ERR_NONFINITE = 2u,   // NaN/Inf in a reduction
  DEV_ERR_BREAKDOWN = 4u,   // PCG breakdown (s.As == 0)
  DEV_ERR_BOUNDS = 8u,      // index check failed (bounds-checked build only)
};

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Global-memory accessors with explicit scope, used for cross-CTA hand-offs.
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_gpu_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Loads that bypass L1 (data written by other CTAs during this kernel).
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ int wrap_mod(int v, int n) {
  // v in [-2n, 3n): returns v mod n in [0, n)
  while (v < 0) v += n;
  while (v >= n) v -= n;
  return v;
}

// -------------------------------------------------------------------------------
// Tiled, circularly skewed layout used by the pressure solver.
//
// The grid is cut into column tiles of 32 (x) by TY (y) cells spanning all of z.
// Inside a tile, cell (x, y, z) with tx = x mod 32, ty = y mod TY is stored at
//     ((slot * TY + ty) * 32 + tx),   slot = (z + tx) mod nz.
// A warp that owns row ty of a tile walks the i+j+k wavefront with lane tx at
// z = s - ty - tx, so at every step all 32 lanes touch one contiguous row of
// 32 elements: the MIC(0) sweeps become coalesced streams.  Tiles are ordered
// tile = Y * ntx + X.  Cells outside the grid (x >= nx or y >= ny) are padding
// and hold zeros.
struct Tiled {
  int nx, ny, nz;
  int TY;
  int ntx, nty;
  int64_t tile_elems;  // nz * TY * 32
  int64_t total;       // ntx * nty * tile_elems

  static Tiled make(int nx, int ny, int nz, int TY) {
    Tiled t;
    t.nx = nx;
    t.ny = ny;
    t.nz = nz;
    t.TY = TY;
    t.ntx = (nx + 31) / 32;
    t.nty = (ny + TY - 1) / TY;
    t.tile_elems = (int64_t)nz * TY * 32;
    t.total = (int64_t)t.ntx * t.nty * t.tile_elems;
    return t;
  }
  __host__ __device__ __forceinline__ int64_t tile_base(int X, int Y) const {
    return (int64_t)(Y * ntx + X) * tile_elems;
  }
  __host__ __device__ __forceinline__ int64_t off(int x, int y, int z) const {
    int X = x >> 5, tx = x & 31, Y = y / TY, ty = y - Y * TY;
    int slot = z + tx;
    while (slot >= nz) slot -= nz;
    return tile_base(X, Y) + ((int64_t)slot * TY + ty) * 32 + tx;
  }
  // Inverse map; returns false for padding.
  __host__ __device__ __forceinline__ bool coords(int64_t e, int& x, int& y, int& z) const {
    int64_t t = e / tile_elems;
    int64_t r = e - t * tile_elems;
    int tx = (int)(r & 31);
    int64_t rr = r >> 5;
    int slot = (int)(rr / TY);
    int ty = (int)(rr - (int64_t)slot * TY);
    int X = (int)(t % ntx), Y = (int)(t / ntx);
    x = X * 32 + tx;
    y = Y * TY + ty;
    int zz = slot - tx;
    while (zz < 0) zz += nz;
    z = zz;
    return x < nx && y < ny;
  }
};

// Reference-layout index helpers.
__host__ __device__ __forceinline__ int64_t lin(int i, int j, int k, int sy, int sz) {
  return (int64_t)k + (int64_t)j * sz + (int64_t)i * sy * sz;
}

}  // namespace sc
