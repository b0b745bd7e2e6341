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
  DEV_FLAG_FP64_RERUN = 8u, // (host) the mixed solve left the FP32 range and was solved again in FP64
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

// Named barrier over a subset of the CTA.  The non-aligned `barrier.sync` form
// is used on purpose: `bar.sync` is `barrier.sync.aligned`, which counts a whole
// warp as arrived when its first lanes arrive.
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
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
  static constexpr int TY = 8;
  int nx, ny, nz;
  int ntx, nty;
  int64_t tile_elems;  // nz * TY * 32
  int64_t total;       // ntx * nty * tile_elems

  static Tiled make(int nx, int ny, int nz) {
    Tiled t;
    t.nx = nx;
    t.ny = ny;
    t.nz = nz;
    t.ntx = (nx + 31) / 32;
    t.nty = (ny + TY - 1) / TY;
    t.tile_elems = (int64_t)nz * TY * 32;
    t.total = (int64_t)t.ntx * t.nty * t.tile_elems;
    return t;
  }
  __host__ __device__ __forceinline__ int ntiles() const { return ntx * nty; }
  __host__ __device__ __forceinline__ int64_t tile_base(int X, int Y) const {
    return (int64_t)(Y * ntx + X) * tile_elems;
  }
  __host__ __device__ __forceinline__ int64_t off(int x, int y, int z) const {
    int X = x >> 5, tx = x & 31, Y = y / TY, ty = y - Y * TY;
    int slot = z + tx;
    while (slot >= nz) slot -= nz;
    return tile_base(X, Y) + ((int64_t)slot * TY + ty) * 32 + tx;
  }
  // Inverse map; returns false for padding.  (Slow path: 64-bit divisions.)
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

// One element of a tiled array seen from a thread of a TY*32-thread block that
// owns the row block (tile, slot): thread (ty, tx) = (threadIdx.x / 32, % 32).
// Gives the coordinates and the element offsets of the six face neighbours
// without any division per element.  Host and device, so that the index
// arithmetic can be checked on the CPU.
struct Cell {
  int x, y, z;
  int tx, ty, slot, X, Y;
  int64_t tbase, e;
  bool inside;
  __host__ __device__ __forceinline__ void init(const Tiled& g, int rb, int tid) {
    const int tile = rb / g.nz;
    slot = rb - tile * g.nz;
    Y = tile / g.ntx;
    X = tile - Y * g.ntx;
    tx = tid & 31;
    ty = tid >> 5;
    x = X * 32 + tx;
    y = Y * Tiled::TY + ty;
    int zz = slot - tx;
    while (zz < 0) zz += g.nz;
    z = zz;
    tbase = (int64_t)tile * g.tile_elems;
    e = (int64_t)rb * (Tiled::TY * 32) + tid;
    inside = x < g.nx && y < g.ny;
  }
  __host__ __device__ __forceinline__ int64_t at(int64_t base, int s, int ty_, int tx_) const {
    return base + ((int64_t)s * Tiled::TY + ty_) * 32 + tx_;
  }
  // neighbour offsets; callers check the domain bounds first
  __host__ __device__ __forceinline__ int64_t xm(const Tiled& g) const {
    if (tx > 0) return at(tbase, slot == 0 ? g.nz - 1 : slot - 1, ty, tx - 1);
    int s = slot + 31;
    while (s >= g.nz) s -= g.nz;
    return at(tbase - g.tile_elems, s, ty, 31);
  }
  __host__ __device__ __forceinline__ int64_t xp(const Tiled& g) const {
    if (tx < 31) return at(tbase, slot == g.nz - 1 ? 0 : slot + 1, ty, tx + 1);
    int s = slot - 31;
    while (s < 0) s += g.nz;
    return at(tbase + g.tile_elems, s, ty, 0);
  }
  __host__ __device__ __forceinline__ int64_t ym(const Tiled& g) const {
    if (ty > 0) return e - 32;
    return at(tbase - (int64_t)g.ntx * g.tile_elems, slot, Tiled::TY - 1, tx);
  }
  __host__ __device__ __forceinline__ int64_t yp(const Tiled& g) const {
    if (ty < Tiled::TY - 1) return e + 32;
    return at(tbase + (int64_t)g.ntx * g.tile_elems, slot, 0, tx);
  }
  __host__ __device__ __forceinline__ int64_t zm(const Tiled& g) const {
    return at(tbase, slot == 0 ? g.nz - 1 : slot - 1, ty, tx);
  }
  __host__ __device__ __forceinline__ int64_t zp(const Tiled& g) const {
    return at(tbase, slot == g.nz - 1 ? 0 : slot + 1, ty, tx);
  }
};

// (x, y, z) of a linear index in an nx x ny x nz grid, z fastest, with
// 32-bit divisions (every grid here holds fewer than 2^31 cells)
__host__ __device__ __forceinline__ void decode3(int64_t id, int ny, int nz, int& x, int& y, int& z) {
  const unsigned u = (unsigned)id, q = u / (unsigned)nz, r = q / (unsigned)ny;
  z = (int)(u - q * (unsigned)nz);
  y = (int)(q - r * (unsigned)ny);
  x = (int)r;
}

// Reference-layout index helpers.
__host__ __device__ __forceinline__ int64_t lin(int i, int j, int k, int sy, int sz) {
  return (int64_t)k + (int64_t)j * sz + (int64_t)i * sy * sz;
}

}  // namespace sc
