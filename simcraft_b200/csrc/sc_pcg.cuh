// sc_pcg.cuh -- MIC(0)-preconditioned CG pressure solver (FP64 and mixed FP32/FP64).
//
// Host-side interface of the solver behind CgSolver3D::solve
// (FluidSim/include/FluidSim/cpu/project-solver.h:100-131,
//  FluidSim/src/cpu/project-solver.cc:308-346) and
// ModifiedIncompleteCholesky3D::precond (project-solver.cc:230-306).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "sc_common.cuh"

namespace sc {


struct Context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // Bound of the device's spin-waits (wavefront mailboxes, grid barriers), in
  // polls; 0 selects each wait's default.  A wait that reaches it gives up and
  // the call returns SC_ERR_TIMEOUT.
  int wait_limit = 0;
  std::string last_error;
  int set_error(int code, const std::string& msg) {
    last_error = msg;
    return code;
  }
};

enum { CRIT_ABS_LINF = 0, CRIT_REL_L2 = 1 };
enum { PREC_FP64 = 0, PREC_MIXED = 1 };
enum { INNER_PCG = 0, INNER_EISENSTAT = 1 };
enum { DONE_RUNNING = 0, DONE_CONVERGED = 1, DONE_MAXITER = 2, DONE_BREAKDOWN = 3 };

struct PcgOptions {
  double tol = 1e-6;       // project-solver.h:129
  int max_iter = 300;      // project-solver.h:130
  int criterion = CRIT_ABS_LINF;
  int precision = PREC_FP64;
  double tau = 0.97, sigma = 0.25;  // project-solver.h:83-84
  double inner_rtol = 1e-4;  // mixed: relative reduction asked of each FP32 inner solve
  int max_outer = 50;        // mixed: defect corrections (FP64 residual replacements)
  int chunk = 8;             // PCG iterations per CUDA-graph launch
  int check_symmetry = 0;    // verify Right/Up/Front == shifted Left/Down/Back
  int true_residual = 1;     // recompute ||b - A p|| in FP64 at the end
  int inner_method = INNER_EISENSTAT;  // mixed: iteration of the FP32 inner solve
  double reliable_delta = 0.1;  // mixed, Eisenstat: split-residual reduction between FP64 replacements
};

struct PcgStats {
  int iterations = 0;        // the reference's `iter` (FP64); total inner iterations (mixed)
  int outer = 0;             // mixed: defect-correction passes
  int status = 0;            // DONE_* of the final (inner) solve
  double residual = 0;       // stopping measure at exit (recurrence residual)
  double true_rel_l2 = 0;    // ||b - A p||_2 / ||b||_2 in FP64
  double true_linf = 0;      // ||b - A p||_inf in FP64
  double ms = 0;             // device time of the solve (events)
  double sym_err = 0;        // max |A_R(p) - A_L(p+x)| etc. when checked
  unsigned device_flags = 0; // DEV_ERR_* bits raised on the device
  int64_t kernel_launches = 0;  // kernels launched by the solve (graph nodes counted)
};

// Device scalars shared by the kernels of one PCG run.
struct PcgScalars {
  double sigma, alpha, beta;
  double res, bnorm, tol, rscale;
  double rn2, rinf, sdotz;
  int iter, max_iter, done, criterion;
  unsigned err;
  unsigned count;  // last-block counter
  int first;       // 1 until the first preconditioner application has set sigma
  int spin_limit;  // polls before a sweep's wait gives up (0: the default bound)
};

struct PcgScalars;
// Arguments of one wavefront sweep kernel launch.
struct WaveArgs {
  Tiled g;
  void* mbx;           // x mailboxes: per consumer tile, mb_stride_x elements
  void* mby;           // y mailboxes: per consumer tile, mb_stride_y elements
  int64_t mb_stride_x, mb_stride_y;
  int* ticket;
  int* exits;
  const int2* order;
  PcgScalars* sc;
  double* partials;
  double* tile_partials;  // per tile share of the sweep's dot product
  int use_skip;
  int fin_kind;
  // Nothing more: growing this parameter block past its 128 bytes measured the
  // sweeps ~30% slower.  The wait bound travels in PcgScalars::spin_limit, a
  // cluster launch passes its cluster-tile order through `order`, and the
  // order's length sits in the header entry order[-1].x.
};

// Wavefront scheduling state (one per sweep kernel; reset by the kernel's last CTA).
struct WaveSync {
  int* ticket;        // next tile ticket
  int* exits;         // CTAs that found no more tiles
  // ticket -> tile for forward sweeps, entries after a header entry holding
  // their count: every tile (pivot sweep), and the tiles with an active cell
  int2* order_all;
  int2* order_fwd;
};

template <class T>
struct SysArrays {  // one precision's copy of everything the PCG touches (tiled layout)
  T *adiag = nullptr, *al = nullptr, *ad = nullptr, *ab = nullptr;
  T *E = nullptr, *cL = nullptr, *cD = nullptr, *cB = nullptr, *uR = nullptr, *uU = nullptr,
    *uF = nullptr;
  T *r = nullptr, *p = nullptr, *z = nullptr, *s = nullptr, *q = nullptr, *Az = nullptr;
  T *Pinv = nullptr, *Dt = nullptr;  // Eisenstat diagonals (FP32 copy only)
};

class PcgSolver {
 public:
  PcgSolver(Context* ctx, int nx, int ny, int nz, const PcgOptions& opt);
  ~PcgSolver();
  int status() const { return init_status_; }
  // Load a system given in the reference layout (6 neighbour arrays, Left..Back
  // order of project-solver.cc:7-14).  `device` selects device or host pointers.
  int upload(const double* adiag, const double* const an[6], const double* rhs,
             const uint8_t* active, bool device);
  // Replace only the right-hand side (reference layout).
  int upload_rhs(const double* rhs, bool device);
  int solve(PcgStats* st);
  int download_pressure(double* pg, bool device);
  // ModifiedIncompleteCholesky3D::precond on the uploaded system: z = M^-1 r
  // (reference layout in and out, device pointers).
  int precond_only(const double* r, double* z);
  // applyCompressedMatrix on the uploaded system (device pointers, reference layout).
  int apply_only(const double* x, double* b);
  // Device time per launch of each kernel class (see sc_pcg_time_kernels).
  int time_kernels(int reps, double* ms);

  const Tiled& geom() const { return g_; }
  uint64_t launches() const { return launches_; }
  // Direct access for in-device producers (FLIP buildSystem writes these).
  double* adiag64() { return d64_.adiag; }
  double* al64() { return d64_.al; }
  double* ad64() { return d64_.ad; }
  double* ab64() { return d64_.ab; }
  double* rhs64() { return rhs_; }
  uint8_t* active() { return active_; }
  double* pressure64() { return d64_.p; }
  // Called after a producer wrote adiag/al/ad/ab/active/rhs in tiled layout.
  void mark_system_changed() { pivots_valid_ = false; }
  void set_options(const PcgOptions& o) { opt_ = o; }
  const PcgOptions& options() const { return opt_; }

 private:
  int ensure_pivots();
  // eis: Eisenstat iteration (FP32 inner solve of the mixed path only)
  template <class T>
  int run_pcg(SysArrays<T>& A, double tol, int criterion, int max_iter, bool scale_rhs,
              PcgStats* st, bool eis = false);
  int solve_fp64(PcgStats* st);
  int solve_mixed(PcgStats* st);
  int solve_mixed_reliable(PcgStats* st);
  template <class T>
  int ensure_graph(SysArrays<T>& A, bool eis);
  int true_residual(PcgStats* st);
  template <class T>
  void launch_iteration(SysArrays<T>& A, bool eis);
  template <class T>
  void launch_spmv(SysArrays<T>& A, cudaStream_t st, int use_skip);
  int check_dev_error(const char* where);
  // After a wavefront wait gave up: refill the mailboxes with the sentinel
  // (an aborted consumer leaves entries unconsumed), clear the status word and
  // drop the pivots, so the next solve starts from a clean state.
  int recover_after_timeout();
  int spin_limit() const;
  int pivot_limit_ = 0;  // host copy of the bound uploaded for the pivot sweep
  // FP32 sweeps in thread-block clusters of cl_size_ CTAs along y (0: none),
  // cl_grid_ clusters; the cluster tile order (anti-diagonals of (X, Yc))
  int cl_size_ = 0, cl_grid_ = 0;
  int2* order_cl_all_ = nullptr;  // every cluster tile (header + entries)
  int2* order_cl_ = nullptr;      // the cluster tiles with an active cell
  // Per tile: any active cell (set with the pivots); the sweeps of the
  // iterations visit only those tiles (or cluster tiles holding one).
  uint8_t* tile_act_ = nullptr;
  void select_active_tiles();
  template <class T, bool FWD, class Op>
  void launch_sweep(const WaveArgs& a, const Op& op, cudaStream_t st, int grid);
  int ensure_host_stage();
  double* hstage_ = nullptr;     // staging of the host-array entry points (N doubles)
  uint8_t* hstage_act_ = nullptr;  // and of the active flags (N bytes)

  Context* ctx_;
  PcgOptions opt_;
  Tiled g_;
  int init_status_ = 0;
  bool pivots_valid_ = false;
  bool have_f32_ = false;
  int nblocks_ = 0;     // elementwise grid
  int wave_grid_ = 0;   // persistent wavefront grid (pivot sweep)
  int wave_grid64_ = 0, wave_grid32_ = 0;  // iteration sweeps: SMs x resident CTAs, capped at the tiles
  SysArrays<double> d64_;
  SysArrays<float> d32_;
  double* rhs_ = nullptr;   // tiled rhs (FP64)
  double* xacc_ = nullptr;  // mixed: FP64 solution accumulator
  uint8_t* active_ = nullptr;
  double* partials_ = nullptr;  // 2 per block
  double* tile_partials_ = nullptr;
  PcgScalars* sc_ = nullptr;
  PcgScalars* sc_host_ = nullptr;  // pinned
  WaveSync ws_{};
  // wavefront mailboxes (per consumer tile), FP64 and FP32
  double *mbx64_ = nullptr, *mby64_ = nullptr;
  float *mbx32_ = nullptr, *mby32_ = nullptr;
  int64_t mb_stride_x_ = 0, mb_stride_y_ = 0;
  void reset_mailboxes(bool f32);
  // all_tiles: sweep every tile (the pivot sweep), else the active ones
  WaveArgs wave_args(bool f32, int use_skip, int fin, bool all_tiles = false) const;
  std::vector<void*> allocs_;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;    // chunk polling
  cudaEvent_t evt0_ = nullptr, evt1_ = nullptr;  // solve timing
  double sym_err_ = 0.0;
  double inner_scale_ = 1.0;
  PcgScalars last_{};
  uint64_t launches_ = 0;  // kernels launched so far (graph nodes counted)
  // graphs: one chunk of iterations per precision
  cudaGraphExec_t graph64_ = nullptr, graph32_ = nullptr, graph32e_ = nullptr;
  template <class T>
  cudaGraphExec_t& graph_for(bool eis);
};

// Allocation-free ModifiedIncompleteCholesky3D::precond on device arrays in the
// reference layout, using a static device array as scratch (sc_pcg.cu).
int mic_precond_noalloc(cudaStream_t st, int device, int sm_count, int nx, int ny, int nz,
                        const double* adiag, const double* const* an, const double* r,
                        const uint8_t* active, double* z, double tau, double sigma,
                        std::string* msg);

}  // namespace sc
