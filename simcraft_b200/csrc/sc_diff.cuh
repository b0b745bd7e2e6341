// sc_diff.cuh -- differentiable FLIP/PIC substeps: forward with checkpoints and
// a hand-written adjoint (reverse mode) of every stage.
//
// The model is the simulator's substep (fluid-simulator.cc:140-182) with a fixed
// dt, run for `steps` substeps from particles at rest on their initial
// positions whose velocities are sampled from a parameter field U (three face
// grids).  The loss is sum_c (rho_c - rho*_c)^2 over the particle density rho
// splatted to the cell centres with the transfer kernel after the last substep.
//
// The adjoint differentiates every continuous dependence on U: G2P, P2G
// (weights depend on positions), advection, velocity extrapolation, gravity,
// the divergence right-hand side, the pressure solve (a second solve with the
// same MIC(0)-PCG, A being symmetric) and the ghost-fluid projection.  The
// discrete structure of a run -- the nearest-node bases of every transfer, the
// wall clamps of advection and the fluid SDF that fixes the active set and the
// ghost-fluid fractions -- is held fixed, as the derivative of a piecewise
// smooth map is taken within the piece of the run.  A run can record that
// structure (TAPE_RECORD) and later runs can replay it (TAPE_REPLAY), which
// makes the loss a smooth function of U around the recorded run (what central
// finite differences check).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "sc_pcg.cuh"

namespace sc {

struct DiffConfig {
  int nx, ny, nz;
  double h, dt;
  int f32;                  // particles and velocity grids in FP32 (else FP64)
  int flip;                 // FLIP (1) or PIC (0) G2P
  double flip_alpha, gravity, recon_factor;
  int sdf_extrap_iters, smooth_iters, vel_extrap_iters;
  int steps;                // substeps per forward
  int checkpoint_every;     // states kept every k substeps; the backward recomputes the rest
  PcgOptions pcg;           // forward and adjoint pressure solves
};

enum { TAPE_NONE = 0, TAPE_RECORD = 1, TAPE_REPLAY = 2 };

class DiffSim {
 public:
  DiffSim(Context* ctx, const DiffConfig& cfg);
  ~DiffSim();
  int status() const { return status_; }
  int set_particles(int64_t n, const double* pos, bool device);
  // rho* on the cell centres (nx*ny*nz doubles)
  int set_target(const double* rho, bool device);
  // loss for the parameter U (three device FP64 face grids, reference layout)
  int forward(const double* const U[3], int tape, double* loss);
  // dL/dU of the last forward, into three device FP64 face grids
  int backward(double* const gU[3]);
  int get_density(double* rho, bool device);
  int get_particles(double* pos, double* vel, bool device);
  // pressure of the last pressure solve run (reference layout)
  int get_pressure(double* p, bool device);
  int64_t num_particles() const { return n_; }
  int last_pcg_iterations() const { return last_iters_; }
  int64_t launches() const { return launches_; }

 private:
  template <class T>
  int forward_t(const double* const U[3], int tape, double* loss);
  template <class T>
  int backward_t(double* const gU[3]);
  template <class T>
  int step_t(int t, int mode, const void* in, void* out);
  template <class T>
  int adjoint_step_t(int t, void* lx, void* lv);
  int err(const char* where);
  void* alloc(size_t bytes);
  void save_sdf(int slot);
  void load_sdf(int slot);

  Context* ctx_;
  DiffConfig c_;
  int status_ = 0;
  size_t rs_ = 8;
  int64_t n_ = 0, N_ = 0, fsz_[3] = {0, 0, 0};
  int nck_ = 0;
  std::vector<void*> allocs_;
  // particles: initial positions x0 (T, 3 arrays), identity ids
  void* x0_ = nullptr;
  int64_t *ids0_ = nullptr, *sid_ = nullptr;
  // states: 6 arrays of n_ each (x, y, z, vx, vy, vz)
  void* ck_ = nullptr;    // checkpoints (nck_ states)
  void* seg_ = nullptr;   // one segment (checkpoint_every + 1 states)
  void* cur_[2] = {nullptr, nullptr};
  void* fin_ = nullptr;   // state after the last substep
  // per-substep intermediates
  void *xa_ = nullptr, *srt_ = nullptr;  // post-advect state (6 arrays), sorted copy
  uint16_t* flags_ = nullptr;  // advect clamps: bit a clamped, bit 3+a velocity zeroed, bit 6+a at the upper wall
  int *key_ = nullptr, *cnt_ = nullptr, *start_ = nullptr, *cursor_ = nullptr, *bsum_ = nullptr;
  void* g_[3][2] = {};                   // velocity grids (ping-pong of the extrapolation)
  int gcur_[3] = {0, 0, 0};
  int gstart_[3] = {0, 0, 0};            // buffer P2G wrote in the last substep
  void* W_[3] = {};                      // P2G weight sums
  void* p2g_scr_ = nullptr;              // P2G tile slices (p2g_scratch_bytes)
  void* last_[3] = {};                   // P2G result (FLIP u_last)
  uint8_t* mask_[3] = {};                // extrapolation masks: (vel_extrap_iters + 1) per grid
  double* wt_[3] = {};                   // face weights of buildSystem
  double* sdf_[2] = {};
  uint8_t* sdfv_[2] = {};
  int scur_ = 0, svcur_ = 0;
  double* sdf_ck_ = nullptr;             // SDF buffers at each checkpoint (2 per checkpoint)
  uint8_t* sdfv_ck_ = nullptr;
  std::vector<int> scur_ck_, svcur_ck_;
  double* seg_sdf_ = nullptr;            // fluid SDF of each substep of the segment being reversed
  const double* seg_sdf_in_ = nullptr;   // use this fluid SDF instead of reconstructing
  double* seg_sdf_out_ = nullptr;        // copy the fluid SDF used here
  PcgSolver* pcg_ = nullptr;
  // adjoint buffers
  void *lx_ = nullptr, *lv_ = nullptr;  // d/d(state) (6 arrays)
  void* lg_[3][2] = {};                 // d/d(grid buffers)
  void* lul_[3] = {};                   // d/d(u_last)
  // density and loss
  double* rho_ = nullptr;
  double* target_ = nullptr;
  double* red_ = nullptr;
  double* host_red_ = nullptr;
  // replay record: per substep SDF, clamps and bases; bases of the final splat
  double* tape_sdf_ = nullptr;
  uint16_t* tape_flags_ = nullptr;
  int16_t* tape_bases_ = nullptr;
  int16_t* tape_final_ = nullptr;
  bool have_tape_ = false;
  int last_mode_ = TAPE_NONE;
  bool have_forward_ = false;
  int last_iters_ = 0;
  int64_t launches_ = 0;
};

}  // namespace sc
