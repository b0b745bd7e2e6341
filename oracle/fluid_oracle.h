/*
 * fluid_oracle.h -- CPU restatement of SimCraft FluidSim's FLIP/PIC step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path in simcraft_b200 and the timed CPU baseline of bench.py; nothing in the
 * product links or calls it.  Every function follows the reference CPU code
 * loop for loop (file:line cited beside each declaration, paths relative to the
 * SimCraft tree).  It is pinned bit for bit against the reference's own
 * sources, compiled from the reference tree by `make ref` (ref_capi.cc,
 * oracle/_ref, tests/test_ref_pin_cpu.py) with stand-ins for the absent
 * glm/oneTBB/spdlog headers.  Core/transfer-stencil.h is absent from the
 * reference snapshot, so the transfer kernel's shape is the one unpinned part:
 * the cubic B-spline below is the documented policy for the missing
 * CubicKernel::weight, and the reference build uses the same policy.
 *
 * Layout (identical to spatify::LinearHashXYZ, Spatify/include/Spatify/hash.h:25):
 *   idx(i,j,k) = k + j*sz + i*sy*sz      (z fastest)
 * Face grids: u (nx+1,ny,nz) offset (0,.5,.5); v (nx,ny+1,nz) offset (.5,0,.5);
 *             w (nx,ny,nz+1) offset (.5,.5,0)   (Spatify/include/Spatify/grids.h:479-485).
 * Cells are cubic with spacing h; the origin is 0.
 * Particles: AoS double[3] per particle.
 */
#ifndef SIMCRAFT_FLUID_ORACLE_H
#define SIMCRAFT_FLUID_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Threads used by loops that the reference runs with tbb::parallel_for.
 * parity_mode=1 keeps FLIP P2G serial (the reference's parallel P2G is racy). */
void ora_set_threads(int n);
void ora_set_parity_mode(int on);
/* Bucket order of the reconstruction (ora_reconstruct, the simulator's
 * substep): 0 (default) = (cell, particle id), the order the GPU path uses;
 * 1 = the reference's std::sort by Morton key (ns-util.h:46-79), not stable,
 * so the skipped last particle of a bucket is the one that sort leaves last. */
void ora_set_bucket_order(int mode);
int ora_get_threads(void);

/* Cubic B-spline weight policy for the missing Core/transfer-stencil.h. */
double ora_cubic_weight(double h, double dx, double dy, double dz);

/* FlipAdvectionSolver3D::solveP2G (FluidSim/src/cpu/advect-solver.cc:188-271) and
 * PicAdvector3D::solveP2G (:18-98, last==NULL). */
void ora_p2g(int64_t n, const double* pos, const double* vel, int nx, int ny, int nz,
             double h, double* u, double* v, double* w, double* uw, double* vw,
             double* ww, uint8_t* uvalid, uint8_t* vvalid, uint8_t* wvalid,
             double* ulast, double* vlast, double* wlast);
/* sampleVelocity (FluidSim/src/cpu/util.cc:40-85) for a batch of points. */
void ora_sample_velocity(int64_t n, const double* pts, int nx, int ny, int nz, double h,
                         const double* u, const double* v, const double* w, double* out);
/* FlipAdvectionSolver3D::solveG2P (advect-solver.cc:157-169); alpha<0 => PIC (:7-17). */
void ora_g2p(int64_t n, const double* pos, double* vel, int nx, int ny, int nz, double h,
             const double* u, const double* v, const double* w, const double* ulast,
             const double* vlast, const double* wlast, double alpha);
/* advect + handleCollision (advect-solver.cc:170-187, 100-137). collider: cell SDF. */
void ora_advect(int64_t n, double* pos, double* vel, int nx, int ny, int nz, double h,
                const double* u, const double* v, const double* w,
                const double* collider, double dt);
/* SDF<3>::eval / grad (FluidSim/include/FluidSim/cpu/sdf.h:35-118). */
double ora_sdf_eval(const double* sdf, int nx, int ny, int nz, double h, const double* p);
void ora_sdf_grad(const double* sdf, int nx, int ny, int nz, double h, const double* p,
                  double* g);
/* NaiveReconstructor::reconstruct (sdf.h:210-225) with ParticleNeighbourSearcher
 * (Spatify/include/Spatify/ns-util.h:46-109).  Bucket order pinned to (cell, id),
 * so the skipped "last" particle of each bucket is the highest id. */
void ora_reconstruct(int64_t n, const double* pos, int nx, int ny, int nz, double h,
                     double radius, double* sdf, uint8_t* valid);
/* fractionInside (FluidSim/src/cpu/util.cc:333-378). */
double ora_fraction_inside(double lu, double ru, double rd, double ld);
/* FvmSolver3D::buildSystem (FluidSim/src/cpu/project-solver.cc:59-228).
 * An: 6 arrays in the order Left,Right,Up,Down,Front,Back (project-solver.cc:7-14). */
void ora_build_system(int nx, int ny, int nz, double h, double dt, const double* u,
                      const double* v, const double* w, const double* fluid_sdf,
                      const double* collider, double* adiag, double* const* an,
                      double* rhs, uint8_t* active, double* uwt, double* vwt, double* wwt);
/* applyCompressedMatrix (project-solver.cc:16-39). */
void ora_apply_matrix(int nx, int ny, int nz, const double* adiag, const double* const* an,
                      const double* x, const uint8_t* active, double* b);
/* ModifiedIncompleteCholesky3D::precond (project-solver.cc:230-306). E, q: scratch
 * outputs (the pivot 1/sqrt(e) and the forward-sweep result), may be NULL. */
void ora_mic_precond(int nx, int ny, int nz, const double* adiag, const double* const* an,
                     const double* r, const uint8_t* active, double* z, double tau,
                     double sigma, double* E_out, double* q_out);
/* Masked BLAS-1 (FluidSim/src/cpu/util.cc:380-410, FluidSim/include/FluidSim/cpu/util.h:56-63). */
double ora_dot(int64_t n, const double* a, const double* b, const uint8_t* active);
void ora_saxpy(int64_t n, double* a, const double* b, double x, const uint8_t* active);
void ora_scale_and_add(int64_t n, double* c, const double* a, double x,
                       const uint8_t* active);
double ora_linf(int64_t n, const double* a, const uint8_t* active);

/* Stopping criteria. 0 = reference (absolute L-inf of r < tol), 1 = ||r||_2/||b||_2 < tol. */
enum { ORA_CRIT_ABS_LINF = 0, ORA_CRIT_REL_L2 = 1 };
/* CgSolver3D::solve (project-solver.cc:308-346).  Returns the final residual in
 * the chosen criterion; *iters receives the reference's `iter` counter. */
double ora_pcg_solve(int nx, int ny, int nz, const double* adiag, const double* const* an,
                     const double* rhs, const uint8_t* active, double* pg, double tol,
                     int max_iter, int criterion, double tau, double sigma, int* iters);
/* FvmSolver3D::project (project-solver.cc:348-435). */
void ora_project(int nx, int ny, int nz, double h, double dt, double* u, double* v,
                 double* w, const double* pg, const double* fluid_sdf, const double* uwt,
                 const double* vwt, const double* wwt);

/* ---- whole simulator: fluid::cpu::FluidSimulator (FluidSim/src/cpu/fluid-simulator.cc) ---- */
typedef struct ora_sim ora_sim;
typedef struct {
  int nx, ny, nz;
  double h;
  int flip;               /* 1 = FLIP, 0 = PIC */
  double flip_alpha;      /* advect-solver.h:129 (0.97) */
  double pcg_tol;         /* project-solver.h:129 (1e-6) */
  int pcg_max_iter;       /* project-solver.h:130 (300) */
  int pcg_criterion;      /* ORA_CRIT_* */
  double mic_tau, mic_sigma;      /* project-solver.h:83-84 */
  double cfl_factor;      /* fluid-simulator.cc:202 (5) */
  double gravity;         /* fluid-simulator.cc:16 (9.8) */
  double recon_factor;    /* fluid-simulator.cc:147 (0.8) */
  int sdf_extrap_iters, smooth_iters, vel_extrap_iters;  /* 10, 5, 10 */
} ora_sim_config;

ora_sim* ora_sim_create(const ora_sim_config* cfg);
void ora_sim_destroy(ora_sim* s);
void ora_sim_set_particles(ora_sim* s, int64_t n, const double* pos, const double* vel);
void ora_sim_set_collider(ora_sim* s, const double* sdf); /* NULL => empty mesh (1e9) */
/* FluidSimulator::step (fluid-simulator.cc:205-220); returns the number of substeps. */
int ora_sim_step(ora_sim* s, double frame_dt);
void ora_sim_substep(ora_sim* s, double dt);
double ora_sim_cfl(const ora_sim* s);
void ora_sim_get_particles(const ora_sim* s, double* pos, double* vel);
void ora_sim_get_pressure(const ora_sim* s, double* p);
void ora_sim_get_faces(const ora_sim* s, double* u, double* v, double* w);
void ora_sim_get_fluid_sdf(const ora_sim* s, double* sdf);
/* FluidSimulator::reconstruct() (cpu/fluid-simulator.h:115-119, radius
 * 1.2 h / sqrt 2 in the reference) and smoothFluidSurface(iters)
 * (fluid-simulator.cc:39-74) on the simulator's own surface buffers, as the
 * reference's export path calls them between steps. */
void ora_sim_reconstruct(ora_sim* s, double radius);
void ora_sim_smooth_fluid_surface(ora_sim* s, int iters);
void ora_sim_get_system(const ora_sim* s, double* adiag, double* const* an, double* rhs,
                        uint8_t* active);
int ora_sim_last_iters(const ora_sim* s);
/* manifold2SDF (util.cc:203-310): triangle mesh (vert n x 3, tri ntri x 3, int)
 * -> signed distance at the cell centres of an nx x ny x nz grid of spacing h
 * and origin (ox, oy, oz); closest triangle per cell and crossing counts too.
 * exact_distance = 0: the reference's point-triangle arithmetic (which
 * overstates edge-AB, edge-AC and face distances); 1: true distances. */
void ora_manifold_to_sdf(int nx, int ny, int nz, double h, double ox, double oy, double oz,
                         const double* vert, const int* tri, int64_t ntri, int exact_band,
                         int exact_distance, double* sdf, int* closest, int* icnt);
double ora_sim_last_residual(const ora_sim* s);
/* Fluid-SDF tape of the simulator (for checking the differentiable step, which
 * holds the fluid SDF of its recorded run fixed; the reference has no such
 * mode): mode 1 clears the tape and records the fluid SDF each later substep
 * uses; mode 2 makes the later substeps use the taped SDFs in order, skipping
 * reconstruction, SDF extrapolation and smoothing; 0 turns the tape off.
 * _get copies taped SDF k out, _put appends one. */
void ora_sim_sdf_tape(ora_sim* s, int mode);
int ora_sim_sdf_tape_get(ora_sim* s, int64_t k, double* sdf);
int ora_sim_sdf_tape_put(ora_sim* s, const double* sdf);
/* rebuildSurface (FluidSim/src/cpu/rebuild-surface.cc:686-741): marching
 * cubes over the cell-centred SDF (reference layout; sample (x, y, z) at
 * ((x + 0.5) spacing[0] + origin[0], ...)).  Returns the vertex count and
 * writes the index count to *nindices; vertices and normals (count x 3) and
 * indices (3 per triangle) are written only when all three are given and the
 * capacities hold them. */
int64_t ora_rebuild_surface(int nx, int ny, int nz, const double* spacing, const double* origin,
                            const double* sdf, double* vertices, double* normals, uint32_t* indices,
                            int64_t vertex_capacity, int64_t index_capacity, int64_t* nindices);

#ifdef __cplusplus
}
#endif
#endif
