// sc_surface.cu -- marching cubes (rebuildSurface, FluidSim/src/cpu/rebuild-surface.cc:686-741).
//
// The reference walks the (nx+1)(ny+1)(nz+1) cubes serially and numbers each
// vertex the first time a cube meets its edge, through a hash map.  Here the
// numbering is recomputed in parallel (sc_surface_dev.cuh): each cube creates
// the vertices of its crossing edges among {5, 6, 10}, and exclusive scans of
// the per-cube vertex and index counts, in the reference's cube order, place
// every vertex and index entry where the serial loop puts it.
//
//   k_mc_count     one pass over the SDF: case mask per cube (1 byte), per-block
//                  totals of vertices and index entries
//   k_mc_scan      one block: exclusive scan of the block totals, grand totals
//   k_mc_vertices  per-block scan of vertex counts; writes each creating cube's
//                  first vertex number and its vertices and normals
//   k_mc_indices   per-block scan of index counts; each entry is the owner
//                  cube's first vertex number plus the edge's rank in its case
//
// Blocks own contiguous runs of kChunk cubes; inside a block the cubes are
// visited in kPer rounds of 256 consecutive cubes (z fastest, so the SDF reads
// of a warp are contiguous).  HBM-bound: the SDF is read once (8 bytes per
// sample), the masks three times (1 byte per cube), plus the mesh itself.
#include <string>

#include "sc_surface.cuh"
#include "sc_surface_dev.cuh"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kPer = 16;
constexpr int64_t kChunk = (int64_t)kThreads * kPer;

__constant__ uint64_t c_mc_cases[256] = {SC_MC_CASES_INIT};

// The case table in shared memory: a warp's cubes index it divergently.
struct SharedCases {
  const uint64_t* t;
  __host__ __device__ uint64_t operator()(int m) const { return t[m]; }
};

__device__ __forceinline__ void load_cases(uint64_t* s) {
  for (int m = threadIdx.x; m < 256; m += blockDim.x) s[m] = c_mc_cases[m];
  __syncthreads();
}

// Exclusive scan of one int per thread over the 256-thread block; *total gets
// the block's sum.  `sh` holds 8 ints; the trailing barrier lets the caller
// reuse it at once.
__device__ __forceinline__ int block_exclusive_scan(int v, int* total, int* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = lane < kThreads / 32 ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < kThreads / 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kThreads / 32) sh[lane] = s;
  }
  __syncthreads();
  const int before = warp ? sh[warp - 1] : 0;
  *total = sh[kThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

struct Scratch {
  uint8_t* mask;       // per cube
  uint32_t* vbase;     // per cube: first vertex number (creating cubes only)
  longlong2* bsum;     // per block: (index entries, vertices), then their exclusive prefix
  long long* totals;   // (index entries, vertices)
  unsigned* status;    // 1: an index entry found no vertex
};

__host__ __device__ inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

Scratch carve(void* base, int64_t ncubes, int64_t nblocks) {
  char* p = (char*)base;
  Scratch s;
  s.mask = (uint8_t*)p;
  p += align256((size_t)ncubes);
  s.vbase = (uint32_t*)p;
  p += align256(sizeof(uint32_t) * (size_t)ncubes);
  s.bsum = (longlong2*)p;
  p += align256(sizeof(longlong2) * (size_t)nblocks);
  s.totals = (long long*)p;
  s.status = (unsigned*)(p + 2 * sizeof(long long));
  return s;
}

__global__ void __launch_bounds__(kThreads) k_mc_count(mc::Grid g, Scratch s) {
  __shared__ uint64_t cases[256];
  __shared__ long long red[2][kThreads / 32];
  load_cases(cases);
  const int64_t nc = g.ncubes(), base = blockIdx.x * kChunk;
  long long nv = 0, ni = 0;
  for (int r = 0; r < kPer; r++) {
    const int64_t c = base + (int64_t)r * kThreads + threadIdx.x;
    if (c >= nc) break;
    int i, j, k;
    g.cube(c, i, j, k);
    const int m = g.mask(i, j, k);
    s.mask[c] = (uint8_t)m;
    const uint64_t w = cases[m];
    nv += mc::owned_count(w);
    ni += SC_MC_COUNT(w);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    nv += __shfl_xor_sync(0xffffffffu, nv, o);
    ni += __shfl_xor_sync(0xffffffffu, ni, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = ni;
    red[1][warp] = nv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long a = 0, b = 0;
    for (int q = 0; q < kThreads / 32; q++) {
      a += red[0][q];
      b += red[1][q];
    }
    s.bsum[blockIdx.x] = make_longlong2(a, b);
  }
}

// One block of 1024 threads: exclusive scan of the per-block totals in place.
__global__ void __launch_bounds__(1024) k_mc_scan(int64_t nb, Scratch s) {
  __shared__ long long sa[1024], sb[1024];
  __shared__ long long carry[2];
  if (threadIdx.x == 0) carry[0] = carry[1] = 0;
  __syncthreads();
  for (int64_t base = 0; base < nb; base += 1024) {
    const int64_t q = base + threadIdx.x;
    const longlong2 v = q < nb ? s.bsum[q] : make_longlong2(0, 0);
    sa[threadIdx.x] = v.x;
    sb[threadIdx.x] = v.y;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const long long ta = threadIdx.x >= o ? sa[threadIdx.x - o] : 0;
      const long long tb = threadIdx.x >= o ? sb[threadIdx.x - o] : 0;
      __syncthreads();
      sa[threadIdx.x] += ta;
      sb[threadIdx.x] += tb;
      __syncthreads();
    }
    if (q < nb) s.bsum[q] = make_longlong2(carry[0] + sa[threadIdx.x] - v.x, carry[1] + sb[threadIdx.x] - v.y);
    __syncthreads();
    if (threadIdx.x == 1023) {
      carry[0] += sa[1023];
      carry[1] += sb[1023];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    s.totals[0] = carry[0];
    s.totals[1] = carry[1];
    *s.status = 0;
  }
}

__global__ void __launch_bounds__(kThreads) k_mc_vertices(mc::Grid g, Scratch s, double* V, double* N) {
  __shared__ uint64_t cases[256];
  __shared__ int sh[kThreads / 32];
  load_cases(cases);
  const int64_t nc = g.ncubes(), base = blockIdx.x * kChunk;
  long long next = s.bsum[blockIdx.x].y;
  for (int r = 0; r < kPer; r++) {
    if (base + (int64_t)r * kThreads >= nc) break;  // uniform over the block
    const int64_t c = base + (int64_t)r * kThreads + threadIdx.x;
    const bool in = c < nc;
    const uint64_t w = cases[in ? s.mask[c] : 0];
    const int cnt = mc::owned_count(w);
    int total;
    const int pre = block_exclusive_scan(cnt, &total, sh);
    if (cnt) {
      int i, j, k;
      g.cube(c, i, j, k);
      const long long vb = next + pre;
      s.vbase[c] = (uint32_t)vb;
      mc::emit_vertices(g, i, j, k, w, vb, V, N);
    }
    next += total;
  }
}

__global__ void __launch_bounds__(kThreads) k_mc_indices(mc::Grid g, Scratch s, uint32_t* I) {
  __shared__ uint64_t cases[256];
  __shared__ int sh[kThreads / 32];
  load_cases(cases);
  const int64_t nc = g.ncubes(), base = blockIdx.x * kChunk;
  long long next = s.bsum[blockIdx.x].x;
  bool ok = true;
  for (int r = 0; r < kPer; r++) {
    if (base + (int64_t)r * kThreads >= nc) break;  // uniform over the block
    const int64_t c = base + (int64_t)r * kThreads + threadIdx.x;
    const bool in = c < nc;
    const uint64_t w = cases[in ? s.mask[c] : 0];
    const int cnt = SC_MC_COUNT(w);
    int total;
    const int pre = block_exclusive_scan(cnt, &total, sh);
    if (cnt) {
      int i, j, k;
      g.cube(c, i, j, k);
      ok &= mc::emit_indices(g, i, j, k, w, SharedCases{cases}, s.mask, s.vbase, next + pre, I);
    }
    next += total;
  }
  if (!ok) atomicOr(s.status, 1u);
}

mc::Grid to_grid(const SurfaceArgs& a) {
  return mc::Grid{a.nx, a.ny, a.nz, a.hx, a.hy, a.hz, a.ox, a.oy, a.oz, a.sdf};
}

int64_t nblocks(const mc::Grid& g) { return (g.ncubes() + kChunk - 1) / kChunk; }

}  // namespace

size_t surface_scratch_bytes(const SurfaceArgs& a) {
  const mc::Grid g = to_grid(a);
  const int64_t nc = g.ncubes();
  return align256((size_t)nc) + align256(sizeof(uint32_t) * (size_t)nc) +
         align256(sizeof(longlong2) * (size_t)nblocks(g)) + 256;
}

int surface_count(cudaStream_t st, const SurfaceArgs& a, void* scratch, int64_t* nvertices,
                  int64_t* nindices) {
  const mc::Grid g = to_grid(a);
  const int64_t nb = nblocks(g);
  const Scratch s = carve(scratch, g.ncubes(), nb);
  k_mc_count<<<(unsigned)nb, kThreads, 0, st>>>(g, s);
  k_mc_scan<<<1, 1024, 0, st>>>(nb, s);
  long long tot[2] = {0, 0};
  cudaMemcpyAsync(tot, s.totals, sizeof(tot), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return -2;
  *nindices = tot[0];
  *nvertices = tot[1];
  return 0;
}

int surface_fill(cudaStream_t st, const SurfaceArgs& a, void* scratch, double* vertices, double* normals,
                 uint32_t* indices, std::string* msg) {
  const mc::Grid g = to_grid(a);
  const int64_t nb = nblocks(g);
  const Scratch s = carve(scratch, g.ncubes(), nb);
  k_mc_vertices<<<(unsigned)nb, kThreads, 0, st>>>(g, s, vertices, normals);
  k_mc_indices<<<(unsigned)nb, kThreads, 0, st>>>(g, s, indices);
  unsigned status = 0;
  cudaMemcpyAsync(&status, s.status, sizeof(status), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return -2;
  if (status) {
    if (msg) *msg = "rebuild_surface: an index entry found no vertex";
    return -1;
  }
  return 0;
}

}  // namespace sc
