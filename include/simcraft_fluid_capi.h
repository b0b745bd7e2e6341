/*
 * simcraft_fluid_capi.h -- C ABI of the B200 (sm_100a) implementation of
 * SimCraft FluidSim's FLIP/PIC step and MIC(0)-PCG pressure projection.
 *
 * Plain C types only: pointers, sizes and POD structs.  Every entry point
 * returns an int status (SC_OK == 0, negative on error) and never throws;
 * sc_context_last_error() gives a message for the last failure.
 *
 * Array layout everywhere is the reference's spatify::LinearHashXYZ order
 * (Spatify/include/Spatify/hash.h:25): idx(i,j,k) = k + j*sz + i*sy*sz, z fastest.
 * Face grids: u (nx+1,ny,nz), v (nx,ny+1,nz), w (nx,ny,nz+1).
 * Neighbour-coefficient arrays are passed as 6 pointers in the reference's
 * Directions order {Left, Right, Up, Down, Front, Back}
 * (FluidSim/src/cpu/project-solver.cc:7-14).
 *
 * Functions suffixed _host take host pointers (copy semantics, synchronous);
 * functions suffixed _device take device pointers and are ordered on the
 * context's stream.
 */
#ifndef SIMCRAFT_FLUID_CAPI_H
#define SIMCRAFT_FLUID_CAPI_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_OK 0
#define SC_ERR_INVALID -1      /* bad argument */
#define SC_ERR_CUDA -2         /* CUDA runtime error */
#define SC_ERR_NOMEM -3        /* device allocation failed */
#define SC_ERR_BREAKDOWN -4    /* PCG breakdown (s.As == 0) */
#define SC_ERR_NOT_CONVERGED -5
#define SC_ERR_TIMEOUT -6      /* a bounded device wait gave up */
#define SC_ERR_ASYMMETRIC -7   /* matrix fails checkSystemSymmetry */
#define SC_ERR_NONFINITE -8    /* NaN/Inf reached a reduction */
#define SC_ERR_UNSUPPORTED -9

/* Stopping criteria for the pressure solve. */
#define SC_CRIT_ABS_LINF 0     /* reference: ||r||_inf < tol (project-solver.cc:334) */
#define SC_CRIT_REL_L2 1       /* ||r||_2 / ||b||_2 < tol */

/* Solver precision. */
#define SC_PREC_FP64 0         /* plain FP64 MIC(0)-PCG */
#define SC_PREC_MIXED 1        /* FP32 inner MIC-PCG + FP64 defect correction */

/* Final state of a solve (sc_pcg_stats.status). */
#define SC_DONE_CONVERGED 1
#define SC_DONE_MAXITER 2
#define SC_DONE_BREAKDOWN 3

typedef struct sc_context sc_context;
typedef struct sc_pcg sc_pcg;

/* Library identity: major * 10000 + minor * 100 (1.1 added the surface export
 * and the simulator's reconstruct / smoothing calls). */
int sc_version(void);
const char* sc_status_string(int status);

/* A context owns one CUDA stream on one device.  Replaces nothing in the
 * reference (which is single-threaded host code); every handle below is bound
 * to a context. */
int sc_context_create(int device, sc_context** out);
/* Frees the context once every handle created from it is destroyed too (in
 * any order). */
void sc_context_destroy(sc_context* ctx);
/* Order all later work on an external stream (a cudaStream_t passed as void*;
 * NULL is the legacy default stream). */
int sc_context_set_stream(sc_context* ctx, void* stream);
/* Go back to the context's own stream. */
int sc_context_use_own_stream(sc_context* ctx);
void* sc_context_stream(sc_context* ctx);
int sc_context_synchronize(sc_context* ctx);
const char* sc_context_last_error(sc_context* ctx);
/* Bound of the device-side spin-waits of this context's later calls (the
 * pressure solver's wavefront mailboxes, the mesh collider's sweep barriers),
 * in polls; polls <= 0 restores each wait's default (about 0.1-1 s).  A wait
 * that reaches the bound gives up: the call returns SC_ERR_TIMEOUT and the
 * handle stays usable (the solver refills its mailboxes and recomputes its
 * pivots on the next call).  No reference counterpart: the reference waits on
 * nothing.  Meant for failure-detection tests and watchdog settings. */
int sc_context_set_wait_limit(sc_context* ctx, int polls);

/* ---------------------------------------------------------------------------
 * Pressure solver: CgSolver3D + ModifiedIncompleteCholesky3D
 * (FluidSim/include/FluidSim/cpu/project-solver.h:71-131).
 */
typedef struct {
  double tol;          /* CgSolver3D::tolerance, 1e-6 (project-solver.h:129) */
  int max_iter;        /* CgSolver3D::max_iterations, 300 (project-solver.h:130) */
  int criterion;       /* SC_CRIT_*; the reference uses SC_CRIT_ABS_LINF */
  int precision;       /* SC_PREC_* */
  double mic_tau;      /* ModifiedIncompleteCholesky3D tuning, 0.97 (project-solver.h:83) */
  double mic_sigma;    /* ModifiedIncompleteCholesky3D safety, 0.25 (project-solver.h:84) */
  double inner_rtol;   /* mixed, SC_INNER_PCG: residual reduction asked of each FP32 inner solve */
  int max_outer;       /* mixed: maximum defect corrections (FP64 residual replacements) */
  int check_symmetry;  /* verify A_Right(p) == A_Left(p+x) etc. on upload */
  int true_residual;   /* recompute ||b - A p|| in FP64 after the solve */
  int inner_method;    /* mixed: SC_INNER_* iteration of the FP32 inner solve */
  double reliable_delta; /* mixed, SC_INNER_EISENSTAT: reduction of the FP32 recursive
                            residual between FP64 residual replacements, 0.1 */
} sc_pcg_options;

/* Iterations of the mixed solve's FP32 inner MIC(0)-PCG.  SC_INNER_PCG is the
 * reference's iteration (SpMV, axpy, forward and backward sweep, scale-add).
 * It restarts after each FP64 defect correction, asking each FP32 solve for a
 * residual reduction of inner_rtol.  SC_INNER_EISENSTAT (the default) runs CG
 * on the split system L^-1 A L^-T with Eisenstat's trick (one backward and one
 * forward sweep apply the operator, so the iteration has no SpMV) and never
 * restarts: whenever its recursive residual has dropped by reliable_delta, the
 * FP32 correction is added to the FP64 solution, the residual is recomputed in
 * FP64 and replaces the FP32 one, and the search direction is kept.  Values of
 * reliable_delta much below 0.01 let the FP32 recursion drift too far between
 * replacements.  Both stop on the FP64 residual's test (criterion, tol). */
enum { SC_INNER_PCG = 0, SC_INNER_EISENSTAT = 1 };

typedef struct {
  int iterations;        /* FP64: the reference's `iter` counter; mixed: inner iterations */
  int outer;             /* mixed: defect-correction passes */
  int status;            /* SC_DONE_* */
  double residual;       /* stopping measure at exit (what CgSolver3D::solve returns) */
  double true_rel_l2;    /* ||b - A p||_2 / ||b||_2 recomputed in FP64 */
  double true_linf;      /* ||b - A p||_inf recomputed in FP64 */
  double ms;             /* device time of the solve */
  double sym_err;        /* max asymmetry found when check_symmetry is set */
  unsigned device_flags; /* device-side error bits: 1 wait timeout, 2 non-finite, 4 breakdown;
                            8: a mixed solve whose FP32 iteration left the FP32 range, solved again in FP64 */
  int64_t kernel_launches; /* kernels this call launched (CUDA-graph nodes counted) */
} sc_pcg_stats;

/* Defaults equal to the reference's constants. */
void sc_pcg_default_options(sc_pcg_options* opt);

/* CgSolver3D(w, h, d) + setPreconditioner(ModifiedIncompleteCholesky)
 * (project-solver.h:100-121).  opt may be NULL for the defaults. */
int sc_pcg_create(sc_context* ctx, int nx, int ny, int nz, const sc_pcg_options* opt,
                  sc_pcg** out);
void sc_pcg_destroy(sc_pcg* pcg);
int sc_pcg_set_options(sc_pcg* pcg, const sc_pcg_options* opt);

/* CgSolver3D::solve(Adiag, Aneighbour, rhs, active, pg) -> residual
 * (project-solver.h:107-111, project-solver.cc:308-346), host arrays.
 * an: 6 arrays in Directions order; only Left/Down/Back are read (the others
 * may be NULL) unless check_symmetry is set, which reads all six and returns
 * SC_ERR_INVALID if one is missing (the matrix must be symmetric,
 * project-solver.cc:41-57). */
int sc_pcg_solve_host(sc_pcg* pcg, const double* adiag, const double* const* an,
                      const double* rhs, const uint8_t* active, double* pg,
                      sc_pcg_stats* stats);
/* Same with device pointers (an: host array of 6 device pointers). */
int sc_pcg_solve_device(sc_pcg* pcg, const double* adiag, const double* const* an,
                        const double* rhs, const uint8_t* active, double* pg,
                        sc_pcg_stats* stats);
/* Split form for repeated solves of one resident system: upload (host or
 * device pointers), solve on the device, then read the pressure back. */
int sc_pcg_upload(sc_pcg* pcg, const double* adiag, const double* const* an,
                  const double* rhs, const uint8_t* active, int device_pointers);
int sc_pcg_upload_rhs(sc_pcg* pcg, const double* rhs, int device_pointers);
int sc_pcg_solve_resident(sc_pcg* pcg, sc_pcg_stats* stats);
int sc_pcg_download(sc_pcg* pcg, double* pg, int device_pointer);

/* ModifiedIncompleteCholesky3D::precond(Adiag, Aneighbour, r, active, z)
 * (project-solver.h:88-92, project-solver.cc:230-306) on the system last
 * uploaded to `pcg`; r and z are device pointers in the reference layout. */
int sc_pcg_precond_device(sc_pcg* pcg, const double* r, double* z);
/* applyCompressedMatrix (project-solver.cc:16-39) on the uploaded system:
 * b = A x, device pointers. */
int sc_pcg_apply_device(sc_pcg* pcg, const double* x, double* b);

/* Per-kernel device time of the solver's kernels on the uploaded system (each
 * kernel launched `reps` times, CUDA events on the context stream), in ms per
 * launch, into ms_out[8]: [0] pivot sweep, [1] forward sweep, [2] backward
 * sweep, [3] SpMV, [4] axpy pair, [5] scale-and-add, and the two sweeps of the
 * Eisenstat inner iteration: [6] backward sweep with the search-direction
 * update, [7] fused forward sweep.  With SC_PREC_MIXED (after a solve) [1]-[7]
 * are FP32 kernels and the mixed iteration is [6] + [7] + [4]; otherwise [6]
 * and [7] are 0.  For profiling; leaves the solution untouched. */
int sc_pcg_time_kernels(sc_pcg* pcg, int reps, double* ms_out);

/* Library-only entry point, no counterpart in the reference: the same MIC(0)
 * preconditioner z = M^-1 r as sc_pcg_precond_device, computed without
 * allocating, on device arrays in the reference layout; an is a host array of
 * 6 device pointers (only Left, Down and Back are read).  It exists for callers
 * that cannot call cudaMalloc, such as engines whose device memory is owned by
 * their own pool allocator, or hot loops where cudaMalloc's device-wide
 * synchronisation is not acceptable.  As in sc_pcg_precond_device, entries the
 * reference never reads (couplings to inactive cells, inactive rows) may hold
 * any value, NaN included.  It allocates nothing: its scratch is one static device array
 * of about 4.4 MB that every GPU loading the library holds until exit, which
 * limits the grid to 32768 tiled cells (ceil(nx/32)*32 * ceil(ny/8)*8 * nz,
 * e.g. 32^3) in at most 8 column tiles; larger grids return SC_ERR_INVALID with
 * a message.  The first call on each device performs a one-time set-up on that
 * device (it looks up the array's device address); make that first call before
 * any stream capture.  All calls share the array, so calls that overlap on the
 * GPU race.  Synchronous on the context's stream. */
int sc_mic_precond_noalloc_device(sc_context* ctx, int nx, int ny, int nz, const double* adiag,
                                  const double* const* an, const double* r,
                                  const uint8_t* active, double* z, double tau, double sigma);

/* ---------------------------------------------------------------------------
 * Finite-volume pressure system: FvmSolver3D
 * (FluidSim/include/FluidSim/cpu/project-solver.h:133-182).
 * `precision` is the type of the face velocity arrays (SC_REAL_F64 / SC_REAL_F32);
 * the matrix, weights and pressure are always double.  collider_sdf == NULL is
 * the empty-mesh collider (all face weights 1 except the domain walls).
 * Cells are cubic with spacing h; device pointers, reference layout.
 */
#define SC_REAL_F64 0
#define SC_REAL_F32 1

/* FvmSolver3D::buildSystem(ug, vg, wg, fluidSdf, colliderSdf, dt)
 * (project-solver.cc:59-228): face weights u/v/w_wt, Adiag, Aneighbour[6]
 * (Directions order), rhs and active.  Any of adiag/an[i]/rhs/active may be
 * NULL to skip that output. */
int sc_fvm_build_system_device(sc_context* ctx, int nx, int ny, int nz, double h, double dt,
                               int precision, const void* u, const void* v, const void* w,
                               const double* fluid_sdf, const double* collider_sdf,
                               double* adiag, double* const* an, double* rhs, uint8_t* active,
                               double* u_wt, double* v_wt, double* w_wt);
/* FvmSolver3D::project(ug, vg, wg, pg, fluidSdf, colliderSdf, dt)
 * (project-solver.cc:348-435), in place on u, v, w. */
int sc_fvm_project_device(sc_context* ctx, int nx, int ny, int nz, double h, double dt,
                          int precision, void* u, void* v, void* w, const double* pg,
                          const double* fluid_sdf, const double* u_wt, const double* v_wt,
                          const double* w_wt);

/* ---------------------------------------------------------------------------
 * Particle/grid transfers of HybridAdvectionSolver3D
 * (FluidSim/include/FluidSim/cpu/advect-solver.h:40-140) as stand-alone device
 * calls, FP64.  Particles are arrays of n xyz triples (pos[3*i+0..2]); grids
 * are face grids in the reference layout with cubic cells of spacing h and the
 * origin at 0.  Transfer kernel: cubic B-spline per axis over the stencil
 * nearest + {-1, 0, 1, 2} of each face grid (advect-solver.cc:44, 207-235).
 */

/* FlipAdvectionSolver3D::solveP2G (advect-solver.cc:188-271): u/v/w = weighted
 * averages of the particle velocities, u_wt/v_wt/w_wt the weight sums,
 * *_valid = weight sum > 0; when u_last is non-NULL the results are also copied
 * into u_last/v_last/w_last (the FLIP reference grids).  Results do not depend
 * on the particle order beyond floating-point summation order. */
int sc_flip_p2g_device(sc_context* ctx, int64_t n, const double* pos, const double* vel, int nx,
                       int ny, int nz, double h, double* u, double* v, double* w, double* u_wt,
                       double* v_wt, double* w_wt, uint8_t* u_valid, uint8_t* v_valid,
                       uint8_t* w_valid, double* u_last, double* v_last, double* w_last);
/* sampleVelocity(p, ug, vg, wg) (FluidSim/src/cpu/util.cc:40-85) at n points. */
int sc_sample_velocity_device(sc_context* ctx, int64_t n, const double* pts, int nx, int ny,
                              int nz, double h, const double* u, const double* v,
                              const double* w, double* out);
/* FlipAdvectionSolver3D::solveG2P (advect-solver.cc:157-169):
 * vel = alpha*(vel + pic - sample(last)) + (1-alpha)*pic; alpha < 0 selects
 * PicAdvector3D::solveG2P (vel = pic, advect-solver.cc:7-17). */
int sc_flip_g2p_device(sc_context* ctx, int64_t n, const double* pos, double* vel, int nx, int ny,
                       int nz, double h, const double* u, const double* v, const double* w,
                       const double* u_last, const double* v_last, const double* w_last,
                       double alpha);
/* FlipAdvectionSolver3D::advect (advect-solver.cc:170-187): Ralston RK3 through
 * the given grids, then handleCollision (advect-solver.cc:100-137) against the
 * collider SDF (NULL: no collider) and the domain box. */
int sc_flip_advect_device(sc_context* ctx, int64_t n, double* pos, double* vel, int nx, int ny,
                          int nz, double h, const double* u, const double* v, const double* w,
                          const double* collider_sdf, double dt);
/* NaiveReconstructor::reconstruct (FluidSim/include/FluidSim/cpu/sdf.h:204-229)
 * with the ParticleNeighbourSearcher buckets (ns-util.h:46-109): cell-centred
 * SDF = min over particles within 2*radius of (distance - radius), 1e9 and
 * valid = 0 where there is none.  Buckets are cells; inside a bucket particles
 * are ordered by index and the last one is not visited, as in the reference. */
int sc_reconstruct_device(sc_context* ctx, int64_t n, const double* pos, int nx, int ny, int nz,
                          double h, double radius, double* sdf, uint8_t* valid);

/* manifold2SDF(exact_band, closest, intersection_cnt, mesh, sdf)
 * (FluidSim/src/cpu/util.cc:203-310): signed distance from a closed triangle
 * mesh at the cell centres ((x + 0.5) h + origin[0], ...) of an nx x ny x nz
 * grid, reference layout.  Exact point-triangle distances within exact_band
 * cells of each triangle's box, then two rounds of eight fast-sweeping passes
 * that propagate the closest triangle, then the sign from the parity of the +z
 * ray crossings below each cell (negative inside).  vertices: nvertices x 3
 * doubles; triangles: ntriangles x 3 vertex indices.  closest (may be NULL)
 * receives the triangle each distance came from (-1 for none).  origin is a
 * host array of 3 doubles (NULL: 0).  flags = SC_MESH_REFERENCE_DISTANCE
 * reproduces the reference bit for bit, including its distancePointTriangle
 * (util.cc:87-125), which measures |ap + v ab|, |ap + w ac| and
 * |ap + v ab + w ac| where the offsets to the closest point on edge AB, edge AC
 * and the face are ap - v ab, ap - w ac and ap - v ab - w ac, so those
 * distances come out too large (the sign is unaffected);
 * SC_MESH_EXACT_DISTANCE uses the true point-triangle distances.  A triangle
 * index outside [0, nvertices) returns SC_ERR_INVALID.  _device: device
 * arrays, on the context stream; _host: host arrays (copied in and out).  The
 * context keeps the scratch it needs (about 8 bytes per cell) until it is
 * destroyed; calls on one context use it one at a time, like its stream. */
enum { SC_MESH_REFERENCE_DISTANCE = 0, SC_MESH_EXACT_DISTANCE = 1 };
int sc_mesh_to_sdf_device(sc_context* ctx, int nx, int ny, int nz, double h, const double* origin,
                          const double* vertices, int64_t nvertices, const int32_t* triangles,
                          int64_t ntriangles, int exact_band, int flags, double* sdf, int32_t* closest);
int sc_mesh_to_sdf_host(sc_context* ctx, int nx, int ny, int nz, double h, const double* origin,
                        const double* vertices, int64_t nvertices, const int32_t* triangles,
                        int64_t ntriangles, int exact_band, int flags, double* sdf, int32_t* closest);

/* rebuildSurface(mesh, sdf) (FluidSim/src/cpu/rebuild-surface.cc:686-741): the
 * marching-cubes mesh of a cell-centred SDF of nx x ny x nz samples (reference
 * layout; sample (x, y, z) at ((x + 0.5) spacing[0] + origin[0], ...); spacing
 * and origin are host arrays of 3 doubles, origin NULL: 0).  The cubes run
 * from -1 to n-1 on each axis, samples outside the grid reading 1000, so a
 * region touching the border is closed there.  The mesh equals the reference's
 * bit for bit: vertices and normals (nvertices x 3 doubles each; normal =
 * normalised interpolated central-difference gradient, not finite where that
 * gradient vanishes) in the order the reference creates them, and index
 * entries (3 per triangle, vertex numbers from 0) in its order.  Both counts
 * are written whenever the arguments are valid.  With vertices, normals and
 * indices all NULL the call only counts; with all three given it fills them,
 * returning SC_ERR_INVALID (nothing written) if a capacity (vertices, index
 * entries) is below the count.  The reference appends to the mesh it is given:
 * a caller doing that adds its earlier vertex count to the indices.  _device:
 * device arrays, on the context stream; _host: host arrays (copied in and
 * out).  The context keeps its scratch (about 5 bytes per cell; _host adds the
 * SDF and the mesh) until it is destroyed; calls on one context use it one at
 * a time. */
int sc_rebuild_surface_device(sc_context* ctx, int nx, int ny, int nz, const double* spacing,
                              const double* origin, const double* sdf, double* vertices, double* normals,
                              uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity,
                              int64_t* nvertices, int64_t* nindices);
int sc_rebuild_surface_host(sc_context* ctx, int nx, int ny, int nz, const double* spacing,
                            const double* origin, const double* sdf, double* vertices, double* normals,
                            uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity,
                            int64_t* nvertices, int64_t* nindices);

/* ---------------------------------------------------------------------------
 * Whole simulator: fluid::cpu::FluidSimulator
 * (FluidSim/include/FluidSim/cpu/fluid-simulator.h:25-200,
 *  FluidSim/src/cpu/fluid-simulator.cc).  Particles and grids live on the
 * device; particles are re-sorted by cell every substep, and the getters return
 * them in the order they were given.
 */
#define SC_ADVECT_PIC 0
#define SC_ADVECT_FLIP 1

typedef struct {
  int nx, ny, nz;        /* resolution (cells) */
  double h;              /* cubic cell size; the domain is [0, n*h] per axis */
  int precision;         /* SC_REAL_F64 / SC_REAL_F32: particles and velocity grids */
  int advection;         /* SC_ADVECT_FLIP (reference default) / SC_ADVECT_PIC */
  double flip_alpha;     /* FLIP blend, 0.97 (advect-solver.h:129) */
  double cfl_factor;     /* CFL() multiplier, 5 (fluid-simulator.cc:202) */
  double gravity;        /* applyForce, 9.8 (fluid-simulator.cc:16) */
  double recon_factor;   /* reconstruction radius / h, 0.8 (fluid-simulator.cc:147) */
  int sdf_extrap_iters;  /* extrapolateFluidSdf(10) (fluid-simulator.cc:151) */
  int smooth_iters;      /* smoothFluidSurface(5) (fluid-simulator.cc:152) */
  int vel_extrap_iters;  /* extrapolate(.., 10) (fluid-simulator.cc:160-162) */
  sc_pcg_options pcg;    /* pressure solve */
} sc_fluid_config;

typedef struct {
  int substeps;          /* substeps taken by this call */
  int pcg_iterations;    /* last substep's solve */
  int pcg_outer;
  double pcg_residual;   /* what solvePressure returned (fluid-simulator.cc:169) */
  double ms_advect, ms_sort_sdf, ms_p2g, ms_build, ms_solve, ms_project_g2p;
  double ms_total;       /* device time, CUDA events, summed over substeps */
  int64_t kernel_launches;
  int pcg_status;        /* last substep's solve: SC_DONE_* */
  unsigned pcg_flags;    /* device_flags of the solves, OR-ed over the substeps */
} sc_fluid_stats;

typedef struct sc_fluid sc_fluid;

/* Reference defaults for an nx*ny*nz grid of spacing h. */
void sc_fluid_default_config(int nx, int ny, int nz, double h, sc_fluid_config* cfg);
/* FluidSimulator(n, size, resolution) (fluid-simulator.h:28-57). */
int sc_fluid_create(sc_context* ctx, const sc_fluid_config* cfg, sc_fluid** out);
void sc_fluid_destroy(sc_fluid* sim);
/* Initial particles (setInitialFluid, fluid-simulator.h:73-78, takes them from
 * the caller); vel == NULL starts them at rest. */
int sc_fluid_set_particles(sc_fluid* sim, int64_t n, const double* pos, const double* vel,
                           int device_pointers);
/* setCollider (fluid-simulator.h:62-72) given the collider SDF on the cell
 * centres (what manifold2SDF produces); NULL removes it. */
int sc_fluid_set_collider(sc_fluid* sim, const double* sdf, int device_pointers);
/* setCollider(const Mesh&) itself (fluid-simulator.h:62-71): the collider SDF
 * built from a closed triangle mesh with manifold2SDF(3, ...) on the
 * simulator's grid (origin 0), as sc_mesh_to_sdf_* computes it with `flags`
 * (SC_MESH_REFERENCE_DISTANCE for the reference's collider). */
int sc_fluid_set_collider_mesh(sc_fluid* sim, const double* vertices, int64_t nvertices,
                               const int32_t* triangles, int64_t ntriangles, int flags,
                               int device_pointers);
/* CFL() (fluid-simulator.cc:184-203). */
int sc_fluid_cfl(sc_fluid* sim, double* dt);
/* substep(dt) (fluid-simulator.cc:140-182). */
int sc_fluid_substep(sc_fluid* sim, double dt, sc_fluid_stats* stats);
/* step(frame): substeps of min(CFL(), remaining) until frame_dt is covered
 * (fluid-simulator.cc:205-220). */
int sc_fluid_step(sc_fluid* sim, double frame_dt, sc_fluid_stats* stats);
int64_t sc_fluid_num_particles(sc_fluid* sim);
/* positions() and the advector's velocities, n*3 doubles each (either may be NULL). */
int sc_fluid_get_particles(sc_fluid* sim, double* pos, double* vel, int device_pointers);
/* pg after the last substep (nx*ny*nz doubles). */
int sc_fluid_get_pressure(sc_fluid* sim, double* pg, int device_pointers);
/* ug/vg/wg after the last substep, as doubles (any may be NULL). */
int sc_fluid_get_faces(sc_fluid* sim, double* u, double* v, double* w, int device_pointers);
/* exportFluidSurface() (fluid-simulator.h:187-189): the smoothed fluid SDF. */
int sc_fluid_get_fluid_sdf(sc_fluid* sim, double* sdf, int device_pointers);
/* FluidSimulator::reconstruct() (FluidSim/include/FluidSim/cpu/fluid-simulator.h
 * :115-119): the surface of the particles as they are now, into the
 * simulator's fluid SDF (what sc_fluid_get_fluid_sdf returns).  radius <= 0
 * selects the reference's 1.2 h / sqrt(2).  smoothFluidSurface(iters)
 * (FluidSim/src/cpu/fluid-simulator.cc:39-74): min-preserving neighbour
 * averaging of that SDF.  Both act on the simulator's own surface buffers, as
 * the reference's, so calling them between steps (as its export path does)
 * changes the stale buffer values the next substep's SDF extrapolation reads,
 * exactly as in the reference. */
int sc_fluid_reconstruct(sc_fluid* sim, double radius);
/* exportColliderSurface() (cpu/fluid-simulator.h:191-193): the collider SDF on
 * the simulator's grid, reference layout; 1e9 everywhere when no collider is
 * set (what manifold2SDF leaves for an empty mesh). */
int sc_fluid_get_collider_sdf(sc_fluid* sim, double* sdf, int device_pointers);
int sc_fluid_smooth_fluid_surface(sc_fluid* sim, int iters);

/* ---------------------------------------------------------------------------
 * Differentiable FLIP/PIC substeps (no counterpart in the reference).
 * Forward: particles at their initial positions take velocities sampled from a
 * parameter field U (three face grids), then `steps` substeps of the
 * simulator's step with a fixed dt; loss = sum_c (rho_c - rho*_c)^2 over the
 * particle density splatted to the cell centres with the transfer kernel.
 * Backward: dL/dU by hand-written adjoint kernels of G2P, P2G, advection,
 * extrapolation, the divergence, the pressure solve (a second MIC(0)-PCG
 * solve; A is symmetric) and the projection, with the run's discrete
 * structure (transfer stencils, wall clamps, fluid SDF) held fixed.  States are
 * kept every `checkpoint_every` substeps; the backward recomputes the others.
 * A forward may record its structure (SC_TAPE_RECORD) and later forwards may
 * replay it (SC_TAPE_REPLAY): with the structure fixed the loss is smooth in U,
 * which is what finite-difference checks of the gradient need.
 */
#define SC_TAPE_NONE 0
#define SC_TAPE_RECORD 1
#define SC_TAPE_REPLAY 2

typedef struct {
  int nx, ny, nz;
  double h, dt;            /* cubic cell size, fixed substep */
  int precision;           /* SC_REAL_F64 / SC_REAL_F32 particles and velocity grids */
  int advection;           /* SC_ADVECT_FLIP / SC_ADVECT_PIC */
  double flip_alpha, gravity, recon_factor;
  int sdf_extrap_iters, smooth_iters, vel_extrap_iters;
  int steps;               /* substeps per forward */
  int checkpoint_every;    /* substeps between stored states */
  sc_pcg_options pcg;      /* forward and adjoint pressure solves */
} sc_diff_config;

typedef struct sc_diff sc_diff;

/* The simulator's defaults, except the pressure solves: relative L2 to 1e-10
 * with the MIC(0) tau = 0 (the reference's tau = 0.97 stalls PCG at
 * dt/h ~ 0.5, and the adjoint needs converged solves). */
void sc_diff_default_config(int nx, int ny, int nz, double h, double dt, int steps,
                            sc_diff_config* cfg);
int sc_diff_create(sc_context* ctx, const sc_diff_config* cfg, sc_diff** out);
void sc_diff_destroy(sc_diff* d);
int sc_diff_set_particles(sc_diff* d, int64_t n, const double* pos, int device_pointers);
/* rho* on the cell centres (nx*ny*nz doubles) */
int sc_diff_set_target(sc_diff* d, const double* rho, int device_pointers);
/* U: host array of 3 device pointers to FP64 face grids (reference layout) */
int sc_diff_forward(sc_diff* d, const double* const* U, int tape, double* loss);
/* dL/dU of the last forward into 3 device FP64 face grids */
int sc_diff_backward(sc_diff* d, double* const* grad_U);
int sc_diff_get_density(sc_diff* d, double* rho, int device_pointers);
/* particles after the last forward (either may be NULL) */
int sc_diff_get_particles(sc_diff* d, double* pos, double* vel, int device_pointers);
/* pressure-solve iterations of the last substep run */
int sc_diff_last_pcg_iterations(sc_diff* d);
/* pressure of the last substep run (nx*ny*nz doubles, reference layout) */
int sc_diff_get_pressure(sc_diff* d, double* p, int device_pointers);

#ifdef __cplusplus
}
#endif
#endif /* SIMCRAFT_FLUID_CAPI_H */
