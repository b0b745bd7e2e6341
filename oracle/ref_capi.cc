/*
 * ref_capi.cc -- C entry points over the reference's OWN FluidSim CPU code.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile (target `ref`) compiles this file
 * into oracle/_ref/libsimcraft_ref.so.  This translation unit includes the
 * reference's sources where they lie (FluidSim/src/cpu/{project-solver,
 * advect-solver,util,fluid-simulator,rebuild-surface}.cc, Core/src/rand-gen.cc),
 * together with the stand-in headers under oracle/refshim (glm, oneTBB served
 * serially, spdlog, the missing Core/transfer-stencil.h with the documented
 * B-spline policy, and a prelude for the snapshot's source rot).  Nothing of the
 * reference is copied here: the functions below only marshal plain arrays in
 * and out of the reference's own classes and call them.  The tests use it to pin
 * the oracle restatement (fluid_oracle.cc) bit for bit against the reference.
 *
 * Access: the reference keeps the state these calls need (the FVM system, the
 * FLIP advector's velocities and u_last grids, the simulator's grids) in
 * protected or private members, so the reference's headers are read with
 * `private` and `protected` spelled `public`.
 *
 * Layout and argument meaning are those of fluid_oracle.h (ora_* counterparts).
 */
#include "refshim/prelude.h"

#include <chrono>

#define private public
#define protected public
#include <FluidSim/src/cpu/project-solver.cc>
#include <FluidSim/src/cpu/advect-solver.cc>
#include <FluidSim/src/cpu/util.cc>
#include <FluidSim/src/cpu/fluid-simulator.cc>
#include <FluidSim/src/cpu/rebuild-surface.cc>
#include <Core/src/rand-gen.cc>
#undef private
#undef protected

namespace {
using namespace fluid;
using namespace fluid::cpu;
using spatify::Array3D;

template <class T>
void put(Array3D<T>& a, const T* src) {
  std::memcpy(a.data(), src, sizeof(T) * (size_t)a.size());
}
template <class T>
void get(const Array3D<T>& a, T* dst) {
  std::memcpy(dst, a.data(), sizeof(T) * (size_t)a.size());
}
template <class G>
void put_grid(G& g, const double* src) {
  std::memcpy(g.array().data(), src, sizeof(double) * (size_t)g.array().size());
}
template <class G>
void get_grid(const G& g, double* dst) {
  std::memcpy(dst, g.array().data(), sizeof(double) * (size_t)g.array().size());
}
void put_u8_as_char(Array3D<char>& a, const uint8_t* src) {
  for (int i = 0; i < a.size(); i++) a.data()[i] = (char)src[i];
}
void get_char_as_u8(const Array3D<char>& a, uint8_t* dst) {
  for (int i = 0; i < a.size(); i++) dst[i] = (uint8_t)a.data()[i];
}

struct System {
  Array3D<Real> adiag;
  std::array<Array3D<Real>, 6> an;
  Array3D<uint8_t> active;
  System(int nx, int ny, int nz, const double* a, const double* const* n, const uint8_t* act)
      : adiag(nx, ny, nz),
        an{Array3D<Real>(nx, ny, nz), Array3D<Real>(nx, ny, nz), Array3D<Real>(nx, ny, nz),
           Array3D<Real>(nx, ny, nz), Array3D<Real>(nx, ny, nz), Array3D<Real>(nx, ny, nz)},
        active(nx, ny, nz) {
    put(adiag, a);
    for (int d = 0; d < 6; d++) put(an[d], n[d]);
    put(active, act);
  }
};

Vec3d cube(int nx, int ny, int nz, double h) { return Vec3d(nx * h, ny * h, nz * h); }

// An SDF<3> over nx x ny x nz cells of spacing h (origin 0); NULL -> 1e9 (no collider).
std::unique_ptr<SDF<3>> make_sdf(int nx, int ny, int nz, double h, const double* v) {
  auto s = std::make_unique<SDF<3>>(Vec3i(nx, ny, nz), cube(nx, ny, nz, h));
  if (v)
    put_grid(s->grid, v);
  else
    s->grid.fill(1e9);
  return s;
}

template <int Axis>
std::unique_ptr<FaceCentredGrid<Real, Real, 3, Axis>> make_face(int nx, int ny, int nz, double h,
                                                                const double* v) {
  auto g = std::make_unique<FaceCentredGrid<Real, Real, 3, Axis>>(Vec3i(nx, ny, nz), cube(nx, ny, nz, h));
  if (v)
    put_grid(*g, v);
  else
    g->fill(0.0);
  return g;
}
}  // namespace

extern "C" {

/* applyCompressedMatrix (project-solver.cc:16-39). */
void ref_apply_matrix(int nx, int ny, int nz, const double* adiag, const double* const* an,
                      const double* x, const uint8_t* active, double* b) {
  System S(nx, ny, nz, adiag, an, active);
  Array3D<Real> X(nx, ny, nz), B(nx, ny, nz);
  put(X, x);
  put(B, b);  // applyCompressedMatrix leaves inactive cells untouched
  fluid::cpu::applyCompressedMatrix(S.adiag, S.an, X, S.active, B);
  get(B, b);
}

/* ModifiedIncompleteCholesky3D::precond (project-solver.cc:230-306). */
void ref_mic_precond(int nx, int ny, int nz, const double* adiag, const double* const* an,
                     const double* r, const uint8_t* active, double* z, double tau, double sigma,
                     double* E_out, double* q_out) {
  System S(nx, ny, nz, adiag, an, active);
  Array3D<Real> R(nx, ny, nz), Z(nx, ny, nz);
  put(R, r);
  put(Z, z);
  ModifiedIncompleteCholesky3D mic(nx, ny, nz, tau, sigma);
  mic.precond(S.adiag, S.an, R, S.active, Z);
  get(Z, z);
  if (E_out) get(mic.E, E_out);
  if (q_out) get(mic.q, q_out);
}

/* CgSolver3D::solve (project-solver.cc:308-346) with the MIC(0) preconditioner;
 * tolerance and max_iterations replace the defaults of project-solver.h:129-130.
 * Returns the reference's residual (absolute L-inf); *iters (may be NULL)
 * receives the count the reference prints ("PCG iterations: N", :344), 0 when
 * it converged before iterating.  ms (may be NULL) receives the wall time of
 * the solve call alone. */
double ref_cg_solve(int nx, int ny, int nz, const double* adiag, const double* const* an,
                    const double* rhs, const uint8_t* active, double* pg, double tol, int max_iter,
                    int* iters, double* ms) {
  System S(nx, ny, nz, adiag, an, active);
  Array3D<Real> RHS(nx, ny, nz), P(nx, ny, nz);
  put(RHS, rhs);
  put(P, pg);
  CgSolver3D cg(nx, ny, nz);
  cg.setPreconditioner(PreconditionerMethod::ModifiedIncompleteCholesky);
  cg.tolerance = tol;
  cg.max_iterations = max_iter;
  std::ostringstream sink;
  std::streambuf* o = std::cout.rdbuf(sink.rdbuf());
  const auto t0 = std::chrono::steady_clock::now();
  const Real res = cg.solve(S.adiag, S.an, RHS, S.active, P);
  const auto t1 = std::chrono::steady_clock::now();
  std::cout.rdbuf(o);
  if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (iters) {
    *iters = 0;
    const std::string out = sink.str(), key = "PCG iterations: ";
    const size_t at = out.rfind(key);
    if (at != std::string::npos) *iters = std::atoi(out.c_str() + at + key.size());
  }
  get(P, pg);
  return res;
}

/* Threads of the timing build (SIMCRAFT_REF_PARALLEL); the parity build is serial. */
void ref_set_threads(int n) {
#ifdef SIMCRAFT_REF_PARALLEL
  omp_set_num_threads(n < 1 ? 1 : n);
#else
  (void)n;
#endif
}

/* Masked BLAS-1 (util.cc:380-410, util.h:56-63) on an nx x ny x nz array. */
double ref_dot(int nx, int ny, int nz, const double* a, const double* b, const uint8_t* active) {
  Array3D<Real> A(nx, ny, nz), B(nx, ny, nz);
  Array3D<uint8_t> act(nx, ny, nz);
  put(A, a);
  put(B, b);
  put(act, active);
  return fluid::dotProduct(A, B, act);
}
void ref_saxpy(int nx, int ny, int nz, double* a, const double* b, double x, const uint8_t* active) {
  Array3D<Real> A(nx, ny, nz), B(nx, ny, nz);
  Array3D<uint8_t> act(nx, ny, nz);
  put(A, a);
  put(B, b);
  put(act, active);
  fluid::saxpy(A, B, x, act);
  get(A, a);
}
void ref_scale_and_add(int nx, int ny, int nz, double* c, const double* a, double x,
                       const uint8_t* active) {
  Array3D<Real> C(nx, ny, nz), A(nx, ny, nz);
  Array3D<uint8_t> act(nx, ny, nz);
  put(C, c);
  put(A, a);
  put(act, active);
  fluid::scaleAndAdd(C, A, x, act);
  get(C, c);
}
double ref_linf(int nx, int ny, int nz, const double* a, const uint8_t* active) {
  Array3D<Real> A(nx, ny, nz);
  Array3D<uint8_t> act(nx, ny, nz);
  put(A, a);
  put(act, active);
  return fluid::LinfNorm(A, act);
}

/* fractionInside (util.cc:333-378). */
double ref_fraction_inside(double lu, double ru, double rd, double ld) {
  return fluid::fractionInside(lu, ru, rd, ld);
}

/* FvmSolver3D::buildSystem (project-solver.cc:59-228). collider NULL -> 1e9. */
void ref_build_system(int nx, int ny, int nz, double h, double dt, const double* u, const double* v,
                      const double* w, const double* fluid_sdf, const double* collider, double* adiag,
                      double* const* an, double* rhs, uint8_t* active, double* uwt, double* vwt,
                      double* wwt) {
  auto ug = make_face<0>(nx, ny, nz, h, u);
  auto vg = make_face<1>(nx, ny, nz, h, v);
  auto wg = make_face<2>(nx, ny, nz, h, w);
  auto fs = make_sdf(nx, ny, nz, h, fluid_sdf);
  auto cs = make_sdf(nx, ny, nz, h, collider);
  FvmSolver3D fvm(nx, ny, nz);
  fvm.buildSystem(*ug, *vg, *wg, *fs, *cs, dt);
  get(fvm.Adiag, adiag);
  for (int d = 0; d < 6; d++) get(fvm.Aneighbour[d], an[d]);
  get(fvm.rhs, rhs);
  get(fvm.active, active);
  if (uwt) get(fvm.uWeights, uwt);
  if (vwt) get(fvm.vWeights, vwt);
  if (wwt) get(fvm.wWeights, wwt);
}

/* FvmSolver3D::project (project-solver.cc:348-435) with given face weights. */
void ref_project(int nx, int ny, int nz, double h, double dt, double* u, double* v, double* w,
                 const double* pg, const double* fluid_sdf, const double* uwt, const double* vwt,
                 const double* wwt) {
  auto ug = make_face<0>(nx, ny, nz, h, u);
  auto vg = make_face<1>(nx, ny, nz, h, v);
  auto wg = make_face<2>(nx, ny, nz, h, w);
  auto fs = make_sdf(nx, ny, nz, h, fluid_sdf);
  auto cs = make_sdf(nx, ny, nz, h, nullptr);
  FvmSolver3D fvm(nx, ny, nz);
  put(fvm.uWeights, uwt);
  put(fvm.vWeights, vwt);
  put(fvm.wWeights, wwt);
  Array3D<Real> P(nx, ny, nz);
  put(P, pg);
  fvm.project(*ug, *vg, *wg, P, *fs, *cs, dt);
  get_grid(*ug, u);
  get_grid(*vg, v);
  get_grid(*wg, w);
}

/* sampleVelocity (util.cc:40-85) for a batch of points. */
void ref_sample_velocity(int64_t n, const double* pts, int nx, int ny, int nz, double h, const double* u,
                         const double* v, const double* w, double* out) {
  auto ug = make_face<0>(nx, ny, nz, h, u);
  auto vg = make_face<1>(nx, ny, nz, h, v);
  auto wg = make_face<2>(nx, ny, nz, h, w);
  for (int64_t i = 0; i < n; i++) {
    Vec3d r = fluid::sampleVelocity(Vec3d(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), *ug, *vg, *wg);
    out[3 * i] = r.x;
    out[3 * i + 1] = r.y;
    out[3 * i + 2] = r.z;
  }
}

namespace {
std::vector<Vec3d> load_points(int64_t n, const double* p) {
  std::vector<Vec3d> v((size_t)n);
  for (int64_t i = 0; i < n; i++) v[i] = Vec3d(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
  return v;
}
void store_points(const std::vector<Vec3d>& v, double* p) {
  for (size_t i = 0; i < v.size(); i++) {
    p[3 * i] = v[i].x;
    p[3 * i + 1] = v[i].y;
    p[3 * i + 2] = v[i].z;
  }
}
std::unique_ptr<HybridAdvectionSolver3D> make_advector(bool flip, int64_t n, int nx, int ny, int nz, double h,
                                                       const double* vel) {
  std::unique_ptr<HybridAdvectionSolver3D> a;
  if (flip)
    a = std::make_unique<FlipAdvectionSolver3D>((int)n, Vec3i(nx, ny, nz), nx * h, ny * h, nz * h);
  else
    a = std::make_unique<PicAdvector3D>((int)n, Vec3i(nx, ny, nz), nx * h, ny * h, nz * h);
  a->velocities = load_points(n, vel);
  return a;
}
}  // namespace

/* FlipAdvectionSolver3D::solveP2G (advect-solver.cc:188-271) when ulast is given,
 * else PicAdvector3D::solveP2G.  Serial (refshim/tbb), i.e. in particle order. */
void ref_p2g(int64_t n, const double* pos, const double* vel, int nx, int ny, int nz, double h, double* u,
             double* v, double* w, double* uw, double* vw, double* ww, uint8_t* uvalid, uint8_t* vvalid,
             uint8_t* wvalid, double* ulast, double* vlast, double* wlast) {
  const bool flip = ulast != nullptr;
  auto adv = make_advector(flip, n, nx, ny, nz, h, vel);
  auto ug = make_face<0>(nx, ny, nz, h, nullptr);
  auto vg = make_face<1>(nx, ny, nz, h, nullptr);
  auto wg = make_face<2>(nx, ny, nz, h, nullptr);
  auto cs = make_sdf(nx, ny, nz, h, nullptr);
  Array3D<Real> UW(nx + 1, ny, nz), VW(nx, ny + 1, nz), WW(nx, ny, nz + 1);
  UW.fill(0.0);
  VW.fill(0.0);
  WW.fill(0.0);
  Array3D<char> UV(nx + 1, ny, nz), VV(nx, ny + 1, nz), WV(nx, ny, nz + 1);
  std::vector<Vec3d> P = load_points(n, pos);
  adv->solveP2G(std::span(P), *ug, *vg, *wg, *cs, UW, VW, WW, UV, VV, WV, 0.0);
  get_grid(*ug, u);
  get_grid(*vg, v);
  get_grid(*wg, w);
  get(UW, uw);
  get(VW, vw);
  get(WW, ww);
  get_char_as_u8(UV, uvalid);
  get_char_as_u8(VV, vvalid);
  get_char_as_u8(WV, wvalid);
  if (flip) {
    auto* f = static_cast<FlipAdvectionSolver3D*>(adv.get());
    get_grid(*f->u_last, ulast);
    get_grid(*f->v_last, vlast);
    get_grid(*f->w_last, wlast);
  }
}

/* FlipAdvectionSolver3D::solveG2P (advect-solver.cc:157-169) with the given
 * u_last grids and blend alpha; alpha < 0 selects PicAdvector3D::solveG2P. */
void ref_g2p(int64_t n, const double* pos, double* vel, int nx, int ny, int nz, double h, const double* u,
             const double* v, const double* w, const double* ulast, const double* vlast, const double* wlast,
             double alpha) {
  const bool flip = alpha >= 0.0;
  auto adv = make_advector(flip, n, nx, ny, nz, h, vel);
  if (flip) {
    auto* f = static_cast<FlipAdvectionSolver3D*>(adv.get());
    put_grid(*f->u_last, ulast);
    put_grid(*f->v_last, vlast);
    put_grid(*f->w_last, wlast);
    f->alpha = alpha;
  }
  auto ug = make_face<0>(nx, ny, nz, h, u);
  auto vg = make_face<1>(nx, ny, nz, h, v);
  auto wg = make_face<2>(nx, ny, nz, h, w);
  auto cs = make_sdf(nx, ny, nz, h, nullptr);
  std::vector<Vec3d> P = load_points(n, pos);
  adv->solveG2P(std::span(P), *ug, *vg, *wg, *cs, 0.0);
  store_points(adv->velocities, vel);
}

/* FlipAdvectionSolver3D::advect + handleCollision (advect-solver.cc:170-187, 100-137). */
void ref_advect(int64_t n, double* pos, double* vel, int nx, int ny, int nz, double h, const double* u,
                const double* v, const double* w, const double* collider, double dt) {
  auto adv = make_advector(true, n, nx, ny, nz, h, vel);
  auto ug = make_face<0>(nx, ny, nz, h, u);
  auto vg = make_face<1>(nx, ny, nz, h, v);
  auto wg = make_face<2>(nx, ny, nz, h, w);
  auto cs = make_sdf(nx, ny, nz, h, collider);
  std::vector<Vec3d> P = load_points(n, pos);
  adv->advect(std::span(P), *ug, *vg, *wg, *cs, dt);
  store_points(P, pos);
  store_points(adv->velocities, vel);
}

/* SDF<3>::eval / grad (sdf.h:35-118). */
double ref_sdf_eval(const double* sdf, int nx, int ny, int nz, double h, const double* p) {
  auto s = make_sdf(nx, ny, nz, h, sdf);
  return s->eval(Vec3d(p[0], p[1], p[2]));
}
void ref_sdf_grad(const double* sdf, int nx, int ny, int nz, double h, const double* p, double* g) {
  auto s = make_sdf(nx, ny, nz, h, sdf);
  Vec3d r = s->grad(Vec3d(p[0], p[1], p[2]));
  g[0] = r.x;
  g[1] = r.y;
  g[2] = r.z;
}

/* NaiveReconstructor<Real,3>::reconstruct (sdf.h:210-225) with its
 * ParticleNeighbourSearcher (ns-util.h:46-109), bucket order as std::sort leaves it. */
void ref_reconstruct(int64_t n, const double* pos, int nx, int ny, int nz, double h, double radius, double* sdf,
                     uint8_t* valid) {
  NaiveReconstructor<Real, 3> rec((int)n, nx, ny, nz, cube(nx, ny, nz, h));
  auto s = make_sdf(nx, ny, nz, h, nullptr);
  Array3D<char> V(nx, ny, nz);
  std::vector<Vec3d> P = load_points(n, pos);
  rec.reconstruct(std::span(P), radius, *s, V);
  get_grid(s->grid, sdf);
  get_char_as_u8(V, valid);
}

/* manifold2SDF (util.cc:203-317). */
void ref_manifold_to_sdf(int nx, int ny, int nz, double h, double ox, double oy, double oz, const double* vert,
                         int64_t nvert, const int* tri, int64_t ntri, int exact_band, double* sdf, int* closest,
                         int* icnt) {
  sim::core::Mesh mesh;
  mesh.triangleCount = (int)ntri;
  mesh.vertices = load_points(nvert, vert);
  mesh.indices.resize((size_t)ntri * 3);
  for (int64_t i = 0; i < ntri * 3; i++) mesh.indices[i] = (unsigned)tri[i];
  SDF<3> s(Vec3i(nx, ny, nz), cube(nx, ny, nz, h), Vec3d(ox, oy, oz));
  Array3D<int> C(nx, ny, nz), I(nx, ny, nz);
  fluid::manifold2SDF(exact_band, C, I, mesh, &s);
  get_grid(s.grid, sdf);
  get(C, closest);
  get(I, icnt);
}

/* rebuildSurface (rebuild-surface.cc:643-741) over a cell-centred SDF of cubic
 * spacing h, origin 0.  Returns the vertex count, writes the index count; the
 * arrays are written when the capacities hold them. */
int64_t ref_rebuild_surface(int nx, int ny, int nz, double h, const double* sdf, double* vertices, double* normals,
                            uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity, int64_t* nindices) {
  auto s = make_sdf(nx, ny, nz, h, sdf);
  sim::core::Mesh mesh;
  fluid::cpu::rebuildSurface(mesh, *s);
  const int64_t nv = (int64_t)mesh.vertices.size(), ni = (int64_t)mesh.indices.size();
  *nindices = ni;
  if (vertices && normals && indices && nv <= vertex_capacity && ni <= index_capacity) {
    store_points(mesh.vertices, vertices);
    store_points(mesh.normals, normals);
    for (int64_t i = 0; i < ni; i++) indices[i] = mesh.indices[i];
  }
  return nv;
}

/* ---- fluid::cpu::FluidSimulator (FluidSim/src/cpu/fluid-simulator.cc) ---- */
struct ref_sim {
  std::unique_ptr<fluid::cpu::FluidSimulator> fs;
  int nx, ny, nz;
  double h;
  int64_t n;
  std::ostringstream sink;
};

/* The reference's own set-up (FLIP or PIC advector, FVM projector, CG with the
 * MIC(0) preconditioner, naive reconstructor) with the given FLIP blend, CG
 * tolerance and iteration bound; the collider starts as the empty mesh (1e9). */
ref_sim* ref_sim_create(int nx, int ny, int nz, double h, int flip, double flip_alpha, double pcg_tol,
                        int pcg_max_iter, int64_t n) {
  auto* s = new ref_sim;
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  s->h = h;
  s->n = n;
  s->fs = std::make_unique<fluid::cpu::FluidSimulator>((int)n, cube(nx, ny, nz, h), Vec3i(nx, ny, nz));
  fluid::cpu::FluidSimulator& f = *s->fs;
  f.setAdvector(flip ? AdvectionMethod::FLIP : AdvectionMethod::PIC);
  f.setProjector(ProjectSolver::FVM);
  f.setCompressedSolver(CompressedSolverMethod::CG, PreconditionerMethod::ModifiedIncompleteCholesky);
  f.setReconstructor(ReconstructorMethod::Naive);
  f.colliderSdf->grid.fill(1e9);
  if (flip) static_cast<FlipAdvectionSolver3D*>(f.advector.get())->alpha = flip_alpha;
  auto* fvm = static_cast<FvmSolver3D*>(f.projector.get());
  auto* cg = static_cast<CgSolver3D*>(fvm->solver.get());
  cg->tolerance = pcg_tol;
  cg->max_iterations = pcg_max_iter;
  return s;
}
void ref_sim_destroy(ref_sim* s) { delete s; }
void ref_sim_set_particles(ref_sim* s, const double* pos, const double* vel) {
  s->fs->m_particles.positions = load_points(s->n, pos);
  s->fs->advector->velocities = load_points(s->n, vel);
}
void ref_sim_set_collider(ref_sim* s, const double* sdf) { put_grid(s->fs->colliderSdf->grid, sdf); }
/* FluidSimulator::substep(dt) (fluid-simulator.cc:140-182); its console output is discarded. */
void ref_sim_substep(ref_sim* s, double dt) {
  std::streambuf* o = std::cout.rdbuf(s->sink.rdbuf());
  std::streambuf* e = std::cerr.rdbuf(s->sink.rdbuf());
  s->fs->substep(dt);
  std::cout.rdbuf(o);
  std::cerr.rdbuf(e);
  s->sink.str("");
}
/* FluidSimulator::step (fluid-simulator.cc:205-220); returns the substep count. */
int ref_sim_step(ref_sim* s, double frame_dt) {
  std::streambuf* o = std::cout.rdbuf(s->sink.rdbuf());
  std::streambuf* e = std::cerr.rdbuf(s->sink.rdbuf());
  sim::core::Frame frame;
  frame.dt = frame_dt;
  // the substep count is not returned by the reference; count CFL-limited
  // substeps the way step() takes them
  int count = 0;
  Real t = 0;
  while (t < frame.dt) {
    Real cfl = s->fs->CFL();
    Real dt = std::min(cfl, frame.dt - t);
    count++;
    s->fs->substep(dt);
    t += dt;
  }
  frame.onAdvance();
  std::cout.rdbuf(o);
  std::cerr.rdbuf(e);
  s->sink.str("");
  return count;
}
double ref_sim_cfl(ref_sim* s) { return s->fs->CFL(); }
void ref_sim_get_particles(ref_sim* s, double* pos, double* vel) {
  store_points(s->fs->m_particles.positions, pos);
  store_points(s->fs->advector->velocities, vel);
}
void ref_sim_get_pressure(ref_sim* s, double* p) { get(s->fs->pg, p); }
void ref_sim_get_faces(ref_sim* s, double* u, double* v, double* w) {
  get_grid(*s->fs->ug, u);
  get_grid(*s->fs->vg, v);
  get_grid(*s->fs->wg, w);
}
void ref_sim_get_fluid_sdf(ref_sim* s, double* sdf) { get_grid(s->fs->fluidSurface->grid, sdf); }
void ref_sim_get_system(ref_sim* s, double* adiag, double* const* an, double* rhs, uint8_t* active) {
  auto* fvm = static_cast<FvmSolver3D*>(s->fs->projector.get());
  get(fvm->Adiag, adiag);
  for (int d = 0; d < 6; d++) get(fvm->Aneighbour[d], an[d]);
  get(fvm->rhs, rhs);
  get(fvm->active, active);
}
void ref_sim_reconstruct(ref_sim* s) { s->fs->reconstruct(); }
void ref_sim_smooth_fluid_surface(ref_sim* s, int iters) { s->fs->smoothFluidSurface(iters); }

}  // extern "C"
