// sc_flip.cuh -- FLIP/PIC particle-grid step of SimCraft FluidSim on the GPU.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "sc_common.cuh"
#include "sc_pcg.cuh"

namespace sc {

struct FluidConfig {
  int nx, ny, nz;
  double h;
  int f32;                // particles and grids in FP32 (else FP64)
  int flip;               // 1 FLIP, 0 PIC
  double flip_alpha;      // advect-solver.h:129 (0.97)
  PcgOptions pcg;         // project-solver.h:129-130 + MIC(0) constants
  double cfl_factor;      // fluid-simulator.cc:202 (5)
  double gravity;         // fluid-simulator.cc:16 (9.8)
  double recon_factor;    // fluid-simulator.cc:147 (0.8)
  int sdf_extrap_iters, smooth_iters, vel_extrap_iters;  // 10, 5, 10
};

struct StepStats {
  int substeps = 0;
  int pcg_iterations = 0;  // last substep
  int pcg_outer = 0;
  double pcg_residual = 0.0;
  double ms_advect = 0, ms_sort_sdf = 0, ms_p2g = 0, ms_build = 0, ms_solve = 0, ms_project_g2p = 0;
  double ms_total = 0;
  int64_t kernel_launches = 0;
  int pcg_status = 0;        // last substep's solve (DONE_*)
  unsigned pcg_flags = 0;    // device flags of the solves, OR-ed
};

// Grids and particles in precision T.  The particle arrays are kept sorted by
// cell (then by original index) after every substep's sort; `id` maps back.
class FluidSim {
 public:
  FluidSim(Context* ctx, const FluidConfig& cfg);
  ~FluidSim();
  int status() const { return status_; }
  int set_particles(int64_t n, const double* pos, const double* vel, bool device);
  int set_collider(const double* sdf, bool device);
  int step(double frame_dt, StepStats* st);
  int substep(double dt, StepStats* st);
  double cfl();
  int get_particles(double* pos, double* vel, bool device);
  int get_pressure(double* p, bool device);
  int get_faces(double* u, double* v, double* w, bool device);
  int get_fluid_sdf(double* s, bool device);
  int get_collider_sdf(double* s, bool device);  // 1e9 everywhere when there is none
  // FluidSimulator::reconstruct() and smoothFluidSurface(iters) on the
  // simulator's own surface buffers (cpu/fluid-simulator.h:115-121).
  int reconstruct(double radius);
  int smooth_fluid_surface(int iters);
  int64_t num_particles() const { return n_; }
  const FluidConfig& config() const { return c_; }

 private:
  template <class T>
  int substep_t(double dt, StepStats* st);
  template <class T>
  int reconstruct_t(double radius);
  int alloc_particles(int64_t n);
  int err(const char* where);

  Context* ctx_;
  FluidConfig c_;
  int status_ = 0;
  int64_t n_ = 0, cap_ = 0;
  size_t rs_;  // sizeof(real)
  // particles (SoA, sorted) and sort scratch
  void *px_ = nullptr, *py_ = nullptr, *pz_ = nullptr, *vx_ = nullptr, *vy_ = nullptr, *vz_ = nullptr;
  void *spx_ = nullptr, *spy_ = nullptr, *spz_ = nullptr, *svx_ = nullptr, *svy_ = nullptr,
       *svz_ = nullptr;
  int64_t *id_ = nullptr, *sid_ = nullptr;
  int *key_ = nullptr, *cnt_ = nullptr, *start_ = nullptr, *cursor_ = nullptr, *bsum_ = nullptr;
  // grids: [axis][buffer]
  void* g_[3][2] = {};
  uint8_t* gv_[3][2] = {};
  int gcur_[3] = {0, 0, 0};
  void* gw_[3] = {};     // weight sums
  void* p2g_scr_ = nullptr;  // P2G tile slices (p2g_scratch_bytes)
  uint8_t* cls_[2][3] = {};  // extrapolation tile classes, per face grid (two launches' worth)
  uint8_t* clsS_[2] = {};    // the same for the fluid SDF's extrapolation
  void* last_[3] = {};   // FLIP u_last/v_last/w_last
  double* wt_[3] = {};   // FVM face weights
  double* sdf_[2] = {};
  uint8_t* sdfv_[2] = {};
  int scur_ = 0, svcur_ = 0;
  double* collider_ = nullptr;  // null: empty-mesh collider
  double* redbuf_ = nullptr;    // CFL reduction scratch
  double* host_red_ = nullptr;  // pinned
  PcgSolver* pcg_ = nullptr;
  int64_t fsz_[3];
  std::vector<void*> allocs_;
  cudaEvent_t ev_[8];
  int64_t launches_ = 0;
};

// ---- stage functions on device arrays (reference layout, AoS double particles) ----
// Used by the per-function C ABI (HybridAdvectionSolver3D seams).
int flip_p2g(cudaStream_t st, int64_t n, const double* pos, const double* vel, int nx, int ny,
             int nz, double h, double* u, double* v, double* w, double* uw, double* vw, double* ww,
             uint8_t* uvalid, uint8_t* vvalid, uint8_t* wvalid, double* ulast, double* vlast,
             double* wlast);
int flip_sample(cudaStream_t st, int64_t n, const double* pts, int nx, int ny, int nz, double h,
                const double* u, const double* v, const double* w, double* out);
int flip_g2p(cudaStream_t st, int64_t n, const double* pos, double* vel, int nx, int ny, int nz,
             double h, const double* u, const double* v, const double* w, const double* ulast,
             const double* vlast, const double* wlast, double alpha);
int flip_advect(cudaStream_t st, int64_t n, double* pos, double* vel, int nx, int ny, int nz,
                double h, const double* u, const double* v, const double* w,
                const double* collider, double dt);
int flip_reconstruct(cudaStream_t st, int64_t n, const double* pos, int nx, int ny, int nz,
                     double h, double radius, double* sdf, uint8_t* valid);

}  // namespace sc
