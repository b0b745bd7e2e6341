// sc_mesh.cu -- manifold2SDF (FluidSim/src/cpu/util.cc:203-310) on the GPU.
//
// The reference builds the collider SDF in four stages; each maps to kernels
// that reproduce its result exactly (compiled without FMA contraction, every
// expression in the reference's operation order):
// The point-triangle distance is the reference's arithmetic unless the caller
// asks for exact distances (MeshSdfArgs::exact_distance).
//  1. exact band (:215-259): every triangle lowers the distance of the cells in
//     its bounding box grown by `exact_band`.  Sequentially the first triangle
//     reaching a cell's minimum keeps it (strict <), so the GPU takes the
//     minimum distance with a 64-bit atomicMin on the (non-negative) double's
//     bits, then, in a second pass, the smallest triangle index that attains it.
//  2. crossing counts (:260-290): atomic integer increments, order-free.
//  3. fast sweeping (:291-300, sweep/checkNeighbour :159-201): 2 rounds x 8
//     directional Gauss-Seidel passes.  In a pass every cell reads only
//     neighbours that are behind it along all three axes, so the cells of one
//     hyperplane x' + y' + z' = p (coordinates oriented along the pass) are
//     independent and the planes in increasing p give the sequential result.
//  4. sign (:301-309): parity of the crossings at or below each cell, per column.
#include <algorithm>
#include <climits>

#include "sc_mesh.cuh"

namespace sc {
namespace {

constexpr int kMeshThreads = 256;

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 d3add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 d3scale(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double d3dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double d3len(D3 a) { return sqrt(d3dot(a, a)); }
// std::min / std::max semantics
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct MeshGeo {
  int nx, ny, nz;
  double h, ox, oy, oz;
  bool exact;  // true point-triangle distances (else the reference's arithmetic)
  __device__ __forceinline__ D3 coord(int x, int y, int z) const {
    return {((double)x + 0.5) * h + ox, ((double)y + 0.5) * h + oy, ((double)z + 0.5) * h + oz};
  }
  __device__ __forceinline__ int64_t at(int x, int y, int z) const {
    return ((int64_t)x * ny + y) * nz + z;
  }
};

__device__ __forceinline__ D3 vtx(const double* V, const int32_t* T, int64_t t, int k) {
  const int64_t v = T[3 * t + k];
  return {V[3 * v], V[3 * v + 1], V[3 * v + 2]};
}

// distancePointTriangle (util.cc:87-125).  The reference measures |ap + v ab|
// on edge AB, |ap + w ac| on edge AC and |ap + v ab + w ac| inside the face;
// `exact` takes the offsets to the closest point (minus signs) instead.
__device__ double dist_point_tri(D3 p, D3 a, D3 b, D3 c, bool exact) {
  const D3 ab = d3sub(b, a), ac = d3sub(c, a), ap = d3sub(p, a);
  const double d1 = d3dot(ab, ap), d2 = d3dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return d3len(ap);
  const D3 bp = d3sub(p, b);
  const double d3 = d3dot(ab, bp), d4 = d3dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) return d3len(bp);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const double v = d1 / (d1 - d3);
    return d3len(exact ? d3sub(ap, d3scale(v, ab)) : d3add(ap, d3scale(v, ab)));
  }
  const D3 cp = d3sub(p, c);
  const double d5 = d3dot(ab, cp), d6 = d3dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return d3len(cp);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const double w = d2 / (d2 - d6);
    return d3len(exact ? d3sub(ap, d3scale(w, ac)) : d3add(ap, d3scale(w, ac)));
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return d3len(d3add(bp, d3scale(w, d3sub(cp, bp))));
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  return d3len(exact ? d3sub(d3sub(ap, d3scale(v, ab)), d3scale(w, ac))
                     : d3add(d3add(ap, d3scale(v, ab)), d3scale(w, ac)));
}

// Triangle bounding box in cells (util.cc:219-244), grown by `band`.
struct Box {
  int lx, hx, ly, hy, lz, hz;
};
__device__ __forceinline__ Box tri_box(const MeshGeo& g, D3 a, D3 b, D3 c, int band) {
  const double mnx = dmin(dmin(a.x - g.ox, b.x - g.ox), c.x - g.ox);
  const double mxx = dmax(dmax(a.x - g.ox, b.x - g.ox), c.x - g.ox);
  const double mny = dmin(dmin(a.y - g.oy, b.y - g.oy), c.y - g.oy);
  const double mxy = dmax(dmax(a.y - g.oy, b.y - g.oy), c.y - g.oy);
  const double mnz = dmin(dmin(a.z - g.oz, b.z - g.oz), c.z - g.oz);
  const double mxz = dmax(dmax(a.z - g.oz, b.z - g.oz), c.z - g.oz);
  Box r;
  r.lx = iclamp((int)floor(mnx / g.h - 0.5) - band, 0, g.nx - 1);
  r.hx = iclamp((int)ceil(mxx / g.h - 0.5) + band, 0, g.nx - 1);
  r.ly = iclamp((int)floor(mny / g.h - 0.5) - band, 0, g.ny - 1);
  r.hy = iclamp((int)ceil(mxy / g.h - 0.5) + band, 0, g.ny - 1);
  r.lz = iclamp((int)floor(mnz / g.h - 0.5) - band, 0, g.nz - 1);
  r.hz = iclamp((int)ceil(mxz / g.h - 0.5) + band, 0, g.nz - 1);
  return r;
}

// Vertex coordinates of every triangle, 9 doubles each (one dependent load per
// neighbour in the sweeps instead of two).
__global__ void k_mesh_pack(const double* V, const int32_t* T, int64_t ntri, double* P) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 9 * ntri; i += stride) {
    const int64_t t = i / 9, r = i - 9 * t;
    P[i] = V[3 * (int64_t)T[3 * t + r / 3] + r % 3];
  }
}

__global__ void k_mesh_check(const int32_t* T, int64_t ntri, int64_t nvert, int* flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * ntri; i += stride)
    if (T[i] < 0 || T[i] >= nvert) atomicOr(flag, 1);
}

__global__ void k_mesh_init(int64_t n, unsigned long long* dist, int* closest, int* cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const unsigned long long far = (unsigned long long)__double_as_longlong(1e9);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    dist[e] = far;
    closest[e] = INT_MAX;
    cnt[e] = 0;
  }
}

// Exact band.  PASS 0: distance minimum; PASS 1: smallest triangle index at it.
// Blocks stride over triangles (x) and split each box's cells (y).
template <int PASS>
__global__ void __launch_bounds__(kMeshThreads)
    k_mesh_band(MeshGeo g, const double* V, const int32_t* T, int64_t ntri, int band,
                unsigned long long* dist, int* closest) {
  for (int64_t t = blockIdx.x; t < ntri; t += gridDim.x) {
    const D3 a = vtx(V, T, t, 0), b = vtx(V, T, t, 1), c = vtx(V, T, t, 2);
    const Box bx = tri_box(g, a, b, c, band);
    const int sy = bx.hy - bx.ly + 1, sz = bx.hz - bx.lz + 1;
    const int64_t vol = (int64_t)(bx.hx - bx.lx + 1) * sy * sz;
    for (int64_t q = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; q < vol;
         q += (int64_t)gridDim.y * blockDim.x) {
      const int z = bx.lz + (int)(q % sz);
      const int64_t r = q / sz;
      const int y = bx.ly + (int)(r % sy), x = bx.lx + (int)(r / sy);
      const double d = dist_point_tri(g.coord(x, y, z), a, b, c, g.exact);
      const int64_t e = g.at(x, y, z);
      if (PASS == 0) {
        if (d < 1e9) atomicMin(&dist[e], (unsigned long long)__double_as_longlong(d));
      } else {
        if (d < 1e9 && __longlong_as_double((long long)dist[e]) == d) atomicMin(&closest[e], (int)t);
      }
    }
  }
}

// Crossings of the +z rays through the cell-centre columns with each triangle
// (util.cc:260-290).
__global__ void __launch_bounds__(kMeshThreads)
    k_mesh_cross(MeshGeo g, const double* V, const int32_t* T, int64_t ntri, int* cnt) {
  for (int64_t t = blockIdx.x; t < ntri; t += gridDim.x) {
    const D3 a = vtx(V, T, t, 0), b = vtx(V, T, t, 1), c = vtx(V, T, t, 2);
    const Box bx = tri_box(g, a, b, c, 0);
    const int sy = bx.hy - bx.ly + 1;
    const int64_t area = (int64_t)(bx.hx - bx.lx + 1) * sy;
    for (int64_t q = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; q < area;
         q += (int64_t)gridDim.y * blockDim.x) {
      const int j = bx.lx + (int)(q / sy), k = bx.ly + (int)(q % sy);
      const D3 o = g.coord(j, k, -1);
      // insideTraingle2D (util.cc:131-142)
      const double c0 = (o.x - a.x) * (b.y - a.y) - (b.x - a.x) * (o.y - a.y);
      const double c1 = (o.x - b.x) * (c.y - b.y) - (c.x - b.x) * (o.y - b.y);
      const double c2 = (o.x - c.x) * (a.y - c.y) - (a.x - c.x) * (o.y - c.y);
      const int inside = (c0 >= 0.0) + (c1 >= 0.0) + (c2 >= 0.0);
      if (!(inside == 3 || inside == 0)) continue;
      // calcBiocentricCoord / solveEquations (util.cc:144-157)
      const double a1 = a.x - c.x, b1 = b.x - c.x, e1 = o.x - c.x;
      const double a2 = a.y - c.y, b2 = b.y - c.y, e2 = o.y - c.y;
      const double det = a1 * b2 - a2 * b1;
      const double u = (e1 * b2 - e2 * b1) / det;
      const double v = (a1 * e2 - a2 * e1) / det;
      const double w = 1.0 - u - v;
      const double iz = a.z * u + b.z * v + c.z * w;
      const int l = (int)ceil((iz - g.oz) / g.h - 0.5);
      if (l < 0)
        atomicAdd(&cnt[g.at(j, k, 0)], 1);
      else if (l < g.nz)
        atomicAdd(&cnt[g.at(j, k, l)], 1);
    }
  }
}

__global__ void k_mesh_closest(int64_t n, int* closest) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    if (closest[e] == INT_MAX) closest[e] = -1;
}

// One cell of sweep(dx, dy, dz) (util.cc:182-201) on hyperplane p: the pass
// visits x from the far end when dx > 0 (x = nx-1 first) and from 0 when
// dx < 0, likewise y and z; oriented coordinates x' = dx < 0 ? x : nx-1-x, etc.
// q enumerates (x', y'); z' = p - x' - y'.  Neighbour values written by other
// blocks in earlier planes are read past L1 (__ldcg).
__device__ __forceinline__ void sweep_cell(const MeshGeo& g, const double* P, double* sdf, int* closest,
                                           int64_t q, int p, int dx, int dy, int dz) {
  const int xp = (int)(q / g.ny), yp = (int)(q % g.ny), zp = p - xp - yp;
  if (zp < 0 || zp >= g.nz) return;
  const int x = dx < 0 ? xp : g.nx - 1 - xp;
  const int y = dy < 0 ? yp : g.ny - 1 - yp;
  const int z = dz < 0 ? zp : g.nz - 1 - zp;
  const int64_t e = g.at(x, y, z);
  const D3 pc = g.coord(x, y, z);
  // checkNeighbour (util.cc:159-180).  The loads of the seven neighbours'
  // triangles and then of their packed vertices are issued together (two round
  // trips instead of 21 dependent ones); a triangle already
  // measured for this cell reuses its distance (same inputs, same result); the
  // comparisons then run in the reference's order.
  const int off[7][3] = {{0, dy, dz}, {dx, 0, dz}, {dx, dy, 0}, {0, 0, dz},
                         {0, dy, 0},  {dx, 0, 0},  {dx, dy, dz}};
  int tn[7];
#pragma unroll
  for (int k = 0; k < 7; k++) {
    const int nx_ = x + off[k][0], ny_ = y + off[k][1], nz_ = z + off[k][2];
    const bool in = nx_ >= 0 && nx_ < g.nx && ny_ >= 0 && ny_ < g.ny && nz_ >= 0 && nz_ < g.nz;
    tn[k] = in ? __ldcg(&closest[g.at(nx_, ny_, nz_)]) : -1;
  }
  double d = __ldcg(&sdf[e]);
  int cl = __ldcg(&closest[e]);
  double dk[7];
#pragma unroll
  for (int k = 0; k < 7; k++) {
    dk[k] = 0.0;
    if (tn[k] < 0) continue;
    int same = -1;
#pragma unroll
    for (int j = 0; j < k; j++)
      if (same < 0 && tn[j] == tn[k]) same = j;
    if (same >= 0) {
#pragma unroll
      for (int j = 0; j < k; j++)
        if (j == same) dk[k] = dk[j];
      continue;
    }
    const double* tp = P + 9 * (int64_t)tn[k];
    const D3 ta{__ldg(tp), __ldg(tp + 1), __ldg(tp + 2)};
    const D3 tb{__ldg(tp + 3), __ldg(tp + 4), __ldg(tp + 5)};
    const D3 tc{__ldg(tp + 6), __ldg(tp + 7), __ldg(tp + 8)};
    dk[k] = dist_point_tri(pc, ta, tb, tc, g.exact);
  }
#pragma unroll
  for (int k = 0; k < 7; k++)
    if (tn[k] != -1 && fabs(dk[k]) < fabs(d)) {
      d = dk[k];
      cl = tn[k];
    }
  sdf[e] = d;
  closest[e] = cl;
}

// The reference's pass order: (1,1,1), (1,1,-1), (1,-1,1), ..., (-1,-1,-1), twice.
__device__ __host__ __forceinline__ void pass_dir(int d, int& dx, int& dy, int& dz) {
  dx = (d & 4) ? -1 : 1;
  dy = (d & 2) ? -1 : 1;
  dz = (d & 1) ? -1 : 1;
}

// One plane per launch (fallback when cooperative launches are unavailable).
__global__ void __launch_bounds__(kMeshThreads)
    k_mesh_sweep(MeshGeo g, const double* P, double* sdf, int* closest, int p, int dx, int dy, int dz) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < (int64_t)g.nx * g.ny) sweep_cell(g, P, sdf, closest, q, p, dx, dy, dz);
}

// Grid-wide barrier of a cooperative launch (all blocks co-resident): arrival
// by a release add, the last arriver publishes the next generation with a
// release add, the others poll it with acquire loads.  The wait is bounded:
// after `limit` polls (kSweepSpin by default) the block raises *err and stops
// waiting, and every later barrier returns at once.
constexpr int kSweepSpin = 1 << 24;
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void grid_barrier(unsigned* count, unsigned* gen, int* err, int limit) {
  __syncthreads();
  if (threadIdx.x == 0 && !*(volatile int*)err) {
    const unsigned g0 = ld_acquire(gen);
    if (add_acq_rel(count, 1u) == gridDim.x - 1) {
      *(volatile unsigned*)count = 0;
      add_acq_rel(gen, 1u);
    } else {
      int spins = 0;
      while (ld_acquire(gen) == g0) {
        if (++spins > limit || *(volatile int*)err) {
          atomicOr(err, 1);
          break;
        }
      }
    }
  }
  __syncthreads();
}

// All 16 passes in one cooperative launch, a grid barrier after every plane.
__global__ void __launch_bounds__(kMeshThreads)
    k_mesh_sweep_all(MeshGeo g, const double* P, double* sdf, int* closest, unsigned* count, unsigned* gen,
                     int* err, int limit) {
  const int planes = g.nx + g.ny + g.nz - 2;
  const int64_t cols = (int64_t)g.nx * g.ny;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int pass = 0; pass < 16; pass++) {
    int dx, dy, dz;
    pass_dir(pass & 7, dx, dy, dz);
    for (int p = 0; p < planes; p++) {
      // (x', y') pairs whose z' = p - x' - y' lies in [0, nz)
      const int xlo = max(0, p - (g.ny - 1) - (g.nz - 1)), xhi = min(g.nx - 1, p);
      for (int64_t q = (int64_t)xlo * g.ny + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
           q < (int64_t)(xhi + 1) * g.ny && q < cols; q += stride)
        sweep_cell(g, P, sdf, closest, q, p, dx, dy, dz);
      grid_barrier(count, gen, err, limit);
      if (*(volatile int*)err) return;
    }
  }
}

// Sign from the parity of the crossings counted at or below each cell (util.cc:301-309).
__global__ void k_mesh_sign(MeshGeo g, double* sdf, const int* cnt) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (int64_t)g.nx * g.ny) return;
  const int64_t base = q * g.nz;
  int tot = 0;
  for (int k = 0; k < g.nz; k++) {
    tot += cnt[base + k];
    if (tot & 1) sdf[base + k] = -sdf[base + k];
  }
}

}  // namespace

namespace {
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
}  // namespace

size_t mesh_to_sdf_scratch_bytes(const MeshSdfArgs& a, bool need_closest) {
  const size_t N = (size_t)a.nx * a.ny * a.nz;
  return align256(sizeof(int) * N) + align256(4 * sizeof(int)) +
         align256(sizeof(double) * 9 * (size_t)std::max<int64_t>(a.ntriangles, 1)) +
         (need_closest ? align256(sizeof(int) * N) : 0);
}

int mesh_to_sdf(cudaStream_t st, const MeshSdfArgs& a, double* sdf, int32_t* closest, void* scratch,
                size_t scratch_bytes, std::string* msg) {
  const int64_t N = (int64_t)a.nx * a.ny * a.nz;
  const int64_t cols = (int64_t)a.nx * a.ny;
  int* cl = closest;
  int *cnt = nullptr, *flag = nullptr;
  double* packed = nullptr;
  const bool own = scratch == nullptr;  // allocate per call
  auto fail = [&](int rc, const char* what) {
    if (msg) *msg = what;
    if (own) {
      if (packed) cudaFreeAsync(packed, st);
      if (cnt) cudaFreeAsync(cnt, st);
      if (flag) cudaFreeAsync(flag, st);
      if (cl && cl != closest) cudaFreeAsync(cl, st);
    }
    return rc;
  };
  if (own) {
    if (cudaMallocAsync(&cnt, sizeof(int) * (size_t)N, st) != cudaSuccess ||
        cudaMallocAsync(&flag, 4 * sizeof(int), st) != cudaSuccess ||
        cudaMallocAsync(&packed, sizeof(double) * 9 * (size_t)std::max<int64_t>(a.ntriangles, 1), st) !=
            cudaSuccess ||
        (!cl && cudaMallocAsync(&cl, sizeof(int) * (size_t)N, st) != cudaSuccess))
      return fail(-3, "mesh_to_sdf: scratch allocation failed");
  } else {
    if (scratch_bytes < mesh_to_sdf_scratch_bytes(a, closest == nullptr))
      return fail(-1, "mesh_to_sdf: scratch too small");
    char* p = static_cast<char*>(scratch);
    cnt = reinterpret_cast<int*>(p);
    p += align256(sizeof(int) * (size_t)N);
    flag = reinterpret_cast<int*>(p);
    p += align256(4 * sizeof(int));
    packed = reinterpret_cast<double*>(p);
    p += align256(sizeof(double) * 9 * (size_t)std::max<int64_t>(a.ntriangles, 1));
    if (!cl) cl = reinterpret_cast<int*>(p);
  }
  // triangle indices must name vertices
  int hflag = 0;
  cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (a.ntriangles > 0)
    k_mesh_check<<<(int)std::min<int64_t>((3 * a.ntriangles + kMeshThreads - 1) / kMeshThreads, 4096),
                   kMeshThreads, 0, st>>>(a.triangles, a.ntriangles, a.nvertices, flag);
  cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(-2, "mesh_to_sdf: index check failed");
  if (hflag) return fail(-1, "mesh_to_sdf: a triangle index is outside [0, nvertices)");
  const MeshGeo g{a.nx, a.ny, a.nz, a.h, a.ox, a.oy, a.oz, a.exact_distance != 0};
  const int eblocks = (int)std::min<int64_t>((N + kMeshThreads - 1) / kMeshThreads, 65536);
  unsigned long long* dist = reinterpret_cast<unsigned long long*>(sdf);
  k_mesh_init<<<eblocks, kMeshThreads, 0, st>>>(N, dist, cl, cnt);
  if (a.ntriangles > 0) {
    const dim3 tg((unsigned)std::min<int64_t>(a.ntriangles, 1 << 20), a.ntriangles < 4096 ? 16 : 1);
    k_mesh_band<0><<<tg, kMeshThreads, 0, st>>>(g, a.vertices, a.triangles, a.ntriangles, a.exact_band,
                                                 dist, cl);
    k_mesh_band<1><<<tg, kMeshThreads, 0, st>>>(g, a.vertices, a.triangles, a.ntriangles, a.exact_band,
                                                 dist, cl);
    k_mesh_cross<<<tg, kMeshThreads, 0, st>>>(g, a.vertices, a.triangles, a.ntriangles, cnt);
  }
  k_mesh_closest<<<eblocks, kMeshThreads, 0, st>>>(N, cl);
  if (a.ntriangles > 0)
    k_mesh_pack<<<(int)std::min<int64_t>((9 * a.ntriangles + kMeshThreads - 1) / kMeshThreads, 4096), kMeshThreads,
                  0, st>>>(a.vertices, a.triangles, a.ntriangles, packed);
  // sweep(1,1,1), (1,1,-1), (1,-1,1), (1,-1,-1), (-1,1,1), ..., twice (util.cc:291-300):
  // one cooperative launch with a grid barrier per plane (co-resident grid),
  // else one launch per plane
  const int planes = a.nx + a.ny + a.nz - 2;
  const int sblocks = (int)((cols + kMeshThreads - 1) / kMeshThreads);
  bool coop = false;
  {
    int dev = 0, sms = 0, can = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&can, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (can && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mesh_sweep_all, kMeshThreads, 0) ==
                   cudaSuccess && occ > 0) {
      // one block per SM: a plane holds at most ~(3/4) nx ny cells, and fewer
      // arrivals make the per-plane barrier cheaper
      const int grid = (int)std::min<int64_t>((int64_t)sms, (int64_t)sblocks);
      unsigned* bar = reinterpret_cast<unsigned*>(flag + 1);
      cudaMemsetAsync(flag, 0, 4 * sizeof(int), st);
      const double* P = packed;
      unsigned* gen = bar + 1;
      int limit = a.wait_limit > 0 ? a.wait_limit : kSweepSpin;
      void* args[] = {(void*)&g, (void*)&P, (void*)&sdf, (void*)&cl, (void*)&bar, (void*)&gen, (void*)&flag,
                      (void*)&limit};
      coop = cudaLaunchCooperativeKernel((const void*)k_mesh_sweep_all, grid, kMeshThreads, args, 0, st) ==
             cudaSuccess;
      if (!coop) cudaGetLastError();
    }
  }
  if (!coop)
    for (int pass = 0; pass < 16; pass++) {
      int dx, dy, dz;
      pass_dir(pass & 7, dx, dy, dz);
      for (int p = 0; p < planes; p++)
        k_mesh_sweep<<<sblocks, kMeshThreads, 0, st>>>(g, packed, sdf, cl, p, dx, dy, dz);
    }
  k_mesh_sign<<<sblocks, kMeshThreads, 0, st>>>(g, sdf, cnt);
  // the sweep's wait status
  cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (own) {
    cudaFreeAsync(cnt, st);
    cudaFreeAsync(flag, st);
    cudaFreeAsync(packed, st);
    if (cl != closest) cudaFreeAsync(cl, st);
  }
  cnt = flag = nullptr;
  packed = nullptr;
  cl = closest;
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(-2, "mesh_to_sdf");
  if (coop && hflag) return fail(-6, "mesh_to_sdf: a sweep barrier wait timed out");
  return 0;
}

}  // namespace sc
