// sc_fvm.cu -- FvmSolver3D::buildSystem and ::project on the GPU.
//
// One thread per face for the face weights and for the pressure-gradient
// update, one thread per cell for the matrix row; all in the reference's
// z-fastest layout (face grids (nx+1,ny,nz), (nx,ny+1,nz), (nx,ny,nz+1)).
// Arithmetic follows FluidSim/src/cpu/project-solver.cc:59-228 and :348-435
// term by term; every row is independent, so no atomics are involved.
#include "sc_fvm.cuh"

namespace sc {
namespace {

constexpr int kT = 256;

inline int blocks_for(int64_t n) {
  int64_t b = (n + kT - 1) / kT;
  return (int)(b < 1 ? 1 : (b > 65535 * 32 ? 65535 * 32 : b));
}

// Face weights (project-solver.cc:77-127): 1 - fractionInside(collider at the
// four face corners); walls 0; faces between two air cells are left at 0.
// COL: a collider SDF is given (without one the kernel is compiled apart from
// the collider's sampling, a quarter of the registers).
template <int AX, bool COL>
__global__ void __launch_bounds__(kT)
    k_face_weights(int nx, int ny, int nz, double h, const double* __restrict__ fluid,
                   const double* __restrict__ collider, double* __restrict__ wt) {
  const int fx = nx + (AX == 0), fy = ny + (AX == 1), fz = nz + (AX == 2);
  const int64_t n = (int64_t)fx * fy * fz;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n;
       id += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(id, fy, fz, i, j, k);
    const int c = AX == 0 ? i : (AX == 1 ? j : k);
    const int cmax = AX == 0 ? nx : (AX == 1 ? ny : nz);
    double out = 0.0;
    if (c != 0 && c != cmax) {
      const int64_t lo = AX == 0 ? lin(i - 1, j, k, ny, nz)
                                 : (AX == 1 ? lin(i, j - 1, k, ny, nz) : lin(i, j, k - 1, ny, nz));
      const int64_t hi = lin(i, j, k, ny, nz);
      if (fluid[lo] > 0.0 && fluid[hi] > 0.0) {
        out = 0.0;  // untouched by the reference: stays at its fill value 0
      } else if (!COL || !collider) {
        out = 1.0 - 0.0;  // empty-mesh collider: all corners positive, fraction 0
      } else {
        // face centre (indexToCoord with the face offset), corners at +-h/2
        const double px = ((double)i + (AX == 0 ? 0.0 : 0.5)) * h + 0.0;
        const double py = ((double)j + (AX == 1 ? 0.0 : 0.5)) * h + 0.0;
        const double pz = ((double)k + (AX == 2 ? 0.0 : 0.5)) * h + 0.0;
        const double hh = 0.5 * h;
        double a, b, cc, d;
        if (AX == 0) {  // bu, bd, fd, fu
          a = sdf_eval(collider, nx, ny, nz, h, px + hh * 0.0, py + hh * 1, pz + hh * -1);
          b = sdf_eval(collider, nx, ny, nz, h, px + hh * 0.0, py + hh * -1, pz + hh * -1);
          cc = sdf_eval(collider, nx, ny, nz, h, px + hh * 0.0, py + hh * -1, pz + hh * 1);
          d = sdf_eval(collider, nx, ny, nz, h, px + hh * 0.0, py + hh * 1, pz + hh * 1);
        } else if (AX == 1) {  // lb, rb, rf, lf
          a = sdf_eval(collider, nx, ny, nz, h, px + hh * -1, py + hh * 0.0, pz + hh * -1);
          b = sdf_eval(collider, nx, ny, nz, h, px + hh * 1, py + hh * 0.0, pz + hh * -1);
          cc = sdf_eval(collider, nx, ny, nz, h, px + hh * 1, py + hh * 0.0, pz + hh * 1);
          d = sdf_eval(collider, nx, ny, nz, h, px + hh * -1, py + hh * 0.0, pz + hh * 1);
        } else {  // ld, lu, ru, rd
          a = sdf_eval(collider, nx, ny, nz, h, px + hh * -1, py + hh * -1, pz + hh * 0.0);
          b = sdf_eval(collider, nx, ny, nz, h, px + hh * -1, py + hh * 1, pz + hh * 0.0);
          cc = sdf_eval(collider, nx, ny, nz, h, px + hh * 1, py + hh * 1, pz + hh * 0.0);
          d = sdf_eval(collider, nx, ny, nz, h, px + hh * 1, py + hh * -1, pz + hh * 0.0);
        }
        out = 1.0 - fraction_inside(a, b, cc, d);
      }
    }
    wt[id] = out;
  }
}

// Matrix row, rhs and active flag of one cell (project-solver.cc:129-226).
struct CellRow {
  double ad, aL, aR, aU, aD, aF, aB, r;
  uint8_t act;
};
template <class T>
__device__ __forceinline__ CellRow build_cell(int nx, int ny, int nz, double h, double dt, int i, int j, int k,
                                              const T* __restrict__ u, const T* __restrict__ v,
                                              const T* __restrict__ w, const double* __restrict__ F,
                                              const double* __restrict__ uw, const double* __restrict__ vw,
                                              const double* __restrict__ ww) {
  const int64_t id = lin(i, j, k, ny, nz);
  {
    // face indices of this cell
    const int64_t uL = lin(i, j, k, ny, nz), uR = lin(i + 1, j, k, ny, nz);
    const int64_t vD = lin(i, j, k, ny + 1, nz), vU = lin(i, j + 1, k, ny + 1, nz);
    const int64_t wB = lin(i, j, k, ny, nz + 1), wF = lin(i, j, k + 1, ny, nz + 1);
    double ad = 0.0, aL = 0.0, aR = 0.0, aU = 0.0, aD = 0.0, aF = 0.0, aB = 0.0, r = 0.0;
    uint8_t act = 0;
    const bool any = !(uw[uL] == 0.0 && uw[uR] == 0.0 && vw[vD] == 0.0 && vw[vU] == 0.0 &&
                       ww[wB] == 0.0 && ww[wF] == 0.0);
    const double sd = F[id];
    if (any && !(sd > 0.0)) {
      act = 1;
      const double factor = dt / h;
      if (i > 0) {  // left
        const double fn = F[id - (int64_t)ny * nz];
        if (fn > 0.0) {
          double theta = fmin(fn / (fn - sd), 0.99);
          ad += uw[uL] * factor / (1.0 - theta);
        } else {
          ad += uw[uL] * factor;
          aL -= uw[uL] * factor;
        }
        r += uw[uL] * (double)u[uL];
      }
      if (i < nx - 1) {  // right
        const double fn = F[id + (int64_t)ny * nz];
        if (fn > 0.0) {
          double theta = fmax(sd / (sd - fn), 0.01);
          ad += uw[uR] * factor / theta;
        } else {
          ad += uw[uR] * factor;
          aR -= uw[uR] * factor;
        }
        r -= uw[uR] * (double)u[uR];
      }
      if (j > 0) {  // down
        const double fn = F[id - nz];
        if (fn > 0.0) {
          double theta = fmin(fn / (fn - sd), 0.99);
          ad += vw[vD] * factor / (1.0 - theta);
        } else {
          ad += vw[vD] * factor;
          aD -= vw[vD] * factor;
        }
        r += vw[vD] * (double)v[vD];
      }
      // up: the reference bounds j by the grid WIDTH (project-solver.cc:186);
      // identical on cubic grids, clipped to the height otherwise
      if (j < nx - 1 && j < ny - 1) {
        const double fn = F[id + nz];
        if (fn > 0.0) {
          double theta = fmax(sd / (sd - fn), 0.01);
          ad += vw[vU] * factor / theta;
        } else {
          ad += vw[vU] * factor;
          aU -= vw[vU] * factor;
        }
        r -= vw[vU] * (double)v[vU];
      }
      if (k > 0) {  // back
        const double fn = F[id - 1];
        if (fn > 0.0) {
          double theta = fmin(fn / (fn - sd), 0.99);
          ad += ww[wB] * factor / (1.0 - theta);
        } else {
          ad += ww[wB] * factor;
          aB -= ww[wB] * factor;
        }
        r += ww[wB] * (double)w[wB];
      }
      if (k < nz - 1) {  // front
        const double fn = F[id + 1];
        if (fn > 0.0) {
          double theta = fmax(sd / (sd - fn), 0.01);
          ad += ww[wF] * factor / theta;
        } else {
          ad += ww[wF] * factor;
          aF -= ww[wF] * factor;
        }
        r -= ww[wF] * (double)w[wF];
      }
    }
    return CellRow{ad, aL, aR, aU, aD, aF, aB, r, act};
  }
}
__device__ __forceinline__ void store_row_linear(const SystemOut& out, int64_t id, const CellRow& c) {
  if (out.adiag) out.adiag[id] = c.ad;
  if (out.an[0]) out.an[0][id] = c.aL;
  if (out.an[1]) out.an[1][id] = c.aR;
  if (out.an[2]) out.an[2][id] = c.aU;
  if (out.an[3]) out.an[3][id] = c.aD;
  if (out.an[4]) out.an[4][id] = c.aF;
  if (out.an[5]) out.an[5][id] = c.aB;
  if (out.rhs) out.rhs[id] = c.r;
  if (out.active) out.active[id] = c.act;
}
__device__ __forceinline__ void store_row_tiled(const SystemOut& out, int64_t e, const CellRow& c) {
  out.t_adiag[e] = c.ad;
  out.t_al[e] = c.aL;
  out.t_ad[e] = c.aD;
  out.t_ab[e] = c.aB;
  out.t_rhs[e] = c.act ? c.r : 0.0;
  out.t_active[e] = c.act;
}
// Cells in the reference's order: the rows in the reference layout.
template <class T>
__global__ void __launch_bounds__(kT)
    k_build_cells(int nx, int ny, int nz, double h, double dt, const T* __restrict__ u,
                  const T* __restrict__ v, const T* __restrict__ w,
                  const double* __restrict__ F, const double* __restrict__ uw,
                  const double* __restrict__ vw, const double* __restrict__ ww, SystemOut out) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n;
       id += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(id % nz);
    const int j = (int)((id / nz) % ny);
    const int i = (int)(id / ((int64_t)ny * nz));
    const CellRow c = build_cell<T>(nx, ny, nz, h, dt, i, j, k, u, v, w, F, uw, vw, ww);
    store_row_linear(out, id, c);
    if (out.t_adiag) store_row_tiled(out, out.g.off(i, j, k), c);
  }
}
// Cells in the solver's tiled order, a block per row block (tile, slot), so
// that the tiled rows are written in whole 256-element runs (in the
// reference's order consecutive cells lie a tile row apart there).
template <class T>
__global__ void __launch_bounds__(kT)
    k_build_cells_tiled(int nx, int ny, int nz, double h, double dt, const T* __restrict__ u,
                        const T* __restrict__ v, const T* __restrict__ w,
                        const double* __restrict__ F, const double* __restrict__ uw,
                        const double* __restrict__ vw, const double* __restrict__ ww, SystemOut out) {
  static_assert(Tiled::TY * 32 == kT, "one thread per element of a row block");
  const int64_t nrb = (int64_t)out.g.ntiles() * out.g.nz;
  for (int64_t rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
    Cell cl;
    cl.init(out.g, (int)rb, threadIdx.x);
    if (!cl.inside) continue;
    const CellRow c = build_cell<T>(nx, ny, nz, h, dt, cl.x, cl.y, cl.z, u, v, w, F, uw, vw, ww);
    store_row_linear(out, lin(cl.x, cl.y, cl.z, ny, nz), c);
    store_row_tiled(out, cl.e, c);
  }
}

// Ghost-fluid pressure gradient on one face grid (project-solver.cc:355-420).
template <class T, int AX>
__global__ void __launch_bounds__(kT)
    k_project(int nx, int ny, int nz, double h, double dt, T* __restrict__ vel,
              const double* __restrict__ pg, Tiled tg, bool tiled, const double* __restrict__ F,
              const double* __restrict__ wt) {
  const int fx = nx + (AX == 0), fy = ny + (AX == 1), fz = nz + (AX == 2);
  const int64_t n = (int64_t)fx * fy * fz;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n;
       id += (int64_t)gridDim.x * blockDim.x) {
    if (wt[id] <= 0.0) continue;
    int i, j, k;
    decode3(id, fy, fz, i, j, k);
    const int c = AX == 0 ? i : (AX == 1 ? j : k);
    const int cmax = AX == 0 ? nx : (AX == 1 ? ny : nz);
    if (c == 0 || c == cmax) {
      vel[id] = T(0);
      continue;
    }
    const int li = i - (AX == 0), lj = j - (AX == 1), lk = k - (AX == 2);
    const double sl = F[lin(li, lj, lk, ny, nz)], sr = F[lin(i, j, k, ny, nz)];
    if (sl >= 0.0 && sr >= 0.0) continue;
    const double pr = tiled ? pg[tg.off(i, j, k)] : pg[lin(i, j, k, ny, nz)];
    const double pl = tiled ? pg[tg.off(li, lj, lk)] : pg[lin(li, lj, lk, ny, nz)];
    double x = (double)vel[id];
    if (sl < 0.0 && sr < 0.0) {
      x -= (pr - pl) * dt / h;
    } else if (sl < 0.0) {
      const double theta = fmax(sl / (sl - sr), 0.01);
      x += pl * dt / h / theta;
    } else {
      const double theta = fmin(sl / (sl - sr), 0.99);
      x -= pr * dt / h / (1.0 - theta);
    }
    vel[id] = (T)x;
  }
}

}  // namespace

template <class T>
int fvm_build_system(cudaStream_t st, int nx, int ny, int nz, double h, double dt, const T* u,
                     const T* v, const T* w, const double* fluid_sdf, const double* collider,
                     double* uwt, double* vwt, double* wwt, const SystemOut& out) {
  const int64_t fu = (int64_t)(nx + 1) * ny * nz, fv = (int64_t)nx * (ny + 1) * nz,
                fw = (int64_t)nx * ny * (nz + 1);
  if (collider) {
    k_face_weights<0, true><<<blocks_for(fu), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, collider, uwt);
    k_face_weights<1, true><<<blocks_for(fv), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, collider, vwt);
    k_face_weights<2, true><<<blocks_for(fw), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, collider, wwt);
  } else {
    k_face_weights<0, false><<<blocks_for(fu), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, nullptr, uwt);
    k_face_weights<1, false><<<blocks_for(fv), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, nullptr, vwt);
    k_face_weights<2, false><<<blocks_for(fw), kT, 0, st>>>(nx, ny, nz, h, fluid_sdf, nullptr, wwt);
  }
  const int64_t n = (int64_t)nx * ny * nz;
  if (out.t_adiag)
    k_build_cells_tiled<T><<<blocks_for((int64_t)out.g.ntiles() * out.g.nz * kT), kT, 0, st>>>(
        nx, ny, nz, h, dt, u, v, w, fluid_sdf, uwt, vwt, wwt, out);
  else
    k_build_cells<T><<<blocks_for(n), kT, 0, st>>>(nx, ny, nz, h, dt, u, v, w, fluid_sdf, uwt, vwt, wwt, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template <class T>
int fvm_project(cudaStream_t st, int nx, int ny, int nz, double h, double dt, T* u, T* v, T* w,
                const double* pg, const Tiled* tiled, const double* fluid_sdf,
                const double* uwt, const double* vwt, const double* wwt) {
  const int64_t fu = (int64_t)(nx + 1) * ny * nz, fv = (int64_t)nx * (ny + 1) * nz,
                fw = (int64_t)nx * ny * (nz + 1);
  Tiled tg = tiled ? *tiled : Tiled{};
  const bool t = tiled != nullptr;
  k_project<T, 0><<<blocks_for(fu), kT, 0, st>>>(nx, ny, nz, h, dt, u, pg, tg, t, fluid_sdf, uwt);
  k_project<T, 1><<<blocks_for(fv), kT, 0, st>>>(nx, ny, nz, h, dt, v, pg, tg, t, fluid_sdf, vwt);
  k_project<T, 2><<<blocks_for(fw), kT, 0, st>>>(nx, ny, nz, h, dt, w, pg, tg, t, fluid_sdf, wwt);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

template int fvm_build_system<double>(cudaStream_t, int, int, int, double, double, const double*,
                                      const double*, const double*, const double*, const double*,
                                      double*, double*, double*, const SystemOut&);
template int fvm_build_system<float>(cudaStream_t, int, int, int, double, double, const float*,
                                     const float*, const float*, const double*, const double*,
                                     double*, double*, double*, const SystemOut&);
template int fvm_project<double>(cudaStream_t, int, int, int, double, double, double*, double*,
                                 double*, const double*, const Tiled*, const double*,
                                 const double*, const double*, const double*);
template int fvm_project<float>(cudaStream_t, int, int, int, double, double, float*, float*,
                                float*, const double*, const Tiled*, const double*, const double*,
                                const double*, const double*);

}  // namespace sc
