// sc_fvm.cuh -- finite-volume pressure system (FvmSolver3D) on the GPU.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sc_common.cuh"

namespace sc {

// Where buildSystem writes the matrix: the reference layout (6 neighbour
// arrays, Directions order Left, Right, Up, Down, Front, Back) or the tiled
// layout of the pressure solver (Left/Down/Back only).
struct SystemOut {
  // reference layout (any may be null)
  double* adiag = nullptr;
  double* an[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double* rhs = nullptr;
  uint8_t* active = nullptr;
  // tiled layout (used when tiled_adiag != null)
  Tiled g{};
  double *t_adiag = nullptr, *t_al = nullptr, *t_ad = nullptr, *t_ab = nullptr, *t_rhs = nullptr;
  uint8_t* t_active = nullptr;
};

// FvmSolver3D::buildSystem (FluidSim/src/cpu/project-solver.cc:59-228).
// collider == nullptr is the empty-mesh collider (manifold2SDF fills 1e9,
// FluidSim/src/cpu/util.cc:211): every interior face weight is then 1.
template <class T>
int fvm_build_system(cudaStream_t st, int nx, int ny, int nz, double h, double dt, const T* u,
                     const T* v, const T* w, const double* fluid_sdf, const double* collider,
                     double* uwt, double* vwt, double* wwt, const SystemOut& out);

// FvmSolver3D::project (project-solver.cc:348-435).  pg is in the reference
// layout, or tiled when `tiled` is non-null.
template <class T>
int fvm_project(cudaStream_t st, int nx, int ny, int nz, double h, double dt, T* u, T* v, T* w,
                const double* pg, const Tiled* tiled, const double* fluid_sdf,
                const double* uwt, const double* vwt, const double* wwt);

// SDF<3>::eval with the reference's reversed trilinear weights
// (FluidSim/include/FluidSim/cpu/sdf.h:35-61).
__host__ __device__ inline double sdf_eval(const double* s, int nx, int ny, int nz, double h,
                                           double px, double py, double pz) {
  auto clampi = [](int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); };
  auto clampd = [](double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); };
  int ix = (int)((px - 0.0) / h - 0.5), iy = (int)((py - 0.0) / h - 0.5),
      iz = (int)((pz - 0.0) / h - 0.5);
  int x = clampi(ix, 0, nx - 1), y = clampi(iy, 0, ny - 1), z = clampi(iz, 0, nz - 1);
  int xn = clampi(ix + 1, 0, nx - 1), yn = clampi(iy + 1, 0, ny - 1), zn = clampi(iz + 1, 0, nz - 1);
  double cx = ((double)x + 0.5) * h + 0.0, cy = ((double)y + 0.5) * h + 0.0,
         cz = ((double)z + 0.5) * h + 0.0;
  double tx = clampd((px - cx) / h, 0.0, 1.0);
  double ty = clampd((py - cy) / h, 0.0, 1.0);
  double tz = clampd((pz - cz) / h, 0.0, 1.0);
  auto S = [&](int i, int j, int k) { return s[lin(i, j, k, ny, nz)]; };
  return tx * ty * tz * S(x, y, z) + tx * ty * (1 - tz) * S(x, y, zn) +
         tx * (1 - ty) * tz * S(x, yn, z) + tx * (1 - ty) * (1 - tz) * S(x, yn, zn) +
         (1 - tx) * ty * tz * S(xn, y, z) + (1 - tx) * ty * (1 - tz) * S(xn, y, zn) +
         (1 - tx) * (1 - ty) * tz * S(xn, yn, z) + (1 - tx) * (1 - ty) * (1 - tz) * S(xn, yn, zn);
}

// fractionInside (FluidSim/src/cpu/util.cc:333-378).
__host__ __device__ inline double fraction_inside(double lu, double ru, double rd, double ld) {
  int n_negs = (lu <= 0.0) + (ru <= 0.0) + (rd <= 0.0) + (ld <= 0.0);
  if (n_negs == 0) return 0.0;
  if (n_negs == 4) return 1.0;
  auto cycle = [](double& a0, double& a1, double& a2, double& a3) {
    double t = a0;
    a0 = a3;
    a3 = a2;
    a2 = a1;
    a1 = t;
  };
  for (int g = 0; g < 4 && lu > 0.0; g++) cycle(lu, ru, rd, ld);
  if (n_negs == 1) {
    double fracu = ru / (ru - lu);
    double fracl = ld / (ld - lu);
    return fracu * fracl * 0.5;
  }
  if (n_negs == 2) {
    if (ru <= 0.0) {
      double fracl = ld / (ld - lu);
      double fracr = rd / (rd - ru);
      return 0.5 * (fracl + fracr);
    }
    if (ld <= 0.0) {
      double fracu = ru / (ru - lu);
      double fracd = rd / (rd - ld);
      return 0.5 * (fracu + fracd);
    }
    if (rd <= 0.0) {
      double fracu = ru / (ru - lu);
      double fracd = ld / (ld - rd);
      double fracl = ld / (ld - lu);
      double fracr = ru / (ru - rd);
      if (lu + ru + rd + ld <= 0.0)
        return 1.0 - 0.5 * ((1.0 - fracu) * (1.0 - fracl) + (1.0 - fracd) * (1.0 - fracr));
      return 0.5 * (fracu * fracl + fracd * fracr);
    }
    return 0.0;
  }
  for (int g = 0; g < 4 && lu <= 0.0; g++) cycle(lu, ru, rd, ld);
  double fracu = ru / (ru - lu);
  double fracl = ld / (ld - lu);
  return 1.0 - 0.5 * fracu * fracl;
}

}  // namespace sc
