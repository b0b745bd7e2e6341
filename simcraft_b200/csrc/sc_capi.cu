// sc_capi.cu -- extern "C" boundary.  No C++ exception or CUDA type crosses it.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "../../include/simcraft_fluid_capi.h"
#include "sc_diff.cuh"
#include "sc_flip.cuh"
#include "sc_fvm.cuh"
#include "sc_mesh.cuh"
#include "sc_pcg.cuh"
#include "sc_surface.cuh"

// A context is freed when its user handle and every handle created from it
// have been destroyed, whatever the order of the destroy calls.
struct sc_context {
  sc::Context c;
  cudaStream_t own = nullptr;
  std::atomic<int> refs{1};
  void* mesh_scratch = nullptr;  // mesh-to-SDF scratch, grown on demand, kept until destroy
  size_t mesh_scratch_bytes = 0;
  void* surf_scratch = nullptr;  // surface export: SDF staging + counting scratch, likewise
  size_t surf_scratch_bytes = 0;
  void* surf_stage = nullptr;    // surface export: mesh staging of the host entry point
  size_t surf_stage_bytes = 0;
};

static sc_context* ctx_retain(sc_context* c) {
  c->refs.fetch_add(1);
  return c;
}
static void ctx_release(sc_context* c) {
  if (c->refs.fetch_sub(1) == 1) {
    cudaSetDevice(c->c.device);
    if (c->mesh_scratch || c->surf_scratch || c->surf_stage) cudaStreamSynchronize(c->c.stream);
    if (c->mesh_scratch) cudaFree(c->mesh_scratch);
    if (c->surf_scratch) cudaFree(c->surf_scratch);
    if (c->surf_stage) cudaFree(c->surf_stage);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
  }
}

struct sc_pcg {
  sc_context* ctx;
  sc::PcgSolver* solver;
};

struct sc_fluid {
  sc_context* ctx;
  sc::FluidSim* sim;
};

struct sc_diff {
  sc_context* ctx;
  sc::DiffSim* sim;
};

namespace {

sc::PcgOptions to_internal(const sc_pcg_options* o) {
  sc::PcgOptions p;
  if (!o) return p;
  p.tol = o->tol;
  p.max_iter = o->max_iter;
  p.criterion = o->criterion;
  p.precision = o->precision;
  p.tau = o->mic_tau;
  p.sigma = o->mic_sigma;
  p.inner_rtol = o->inner_rtol;
  p.max_outer = o->max_outer;
  p.check_symmetry = o->check_symmetry;
  p.true_residual = o->true_residual;
  p.inner_method = o->inner_method;
  p.reliable_delta = o->reliable_delta;
  return p;
}

void to_public(const sc::PcgStats& s, sc_pcg_stats* o) {
  if (!o) return;
  o->iterations = s.iterations;
  o->outer = s.outer;
  o->status = s.status;
  o->residual = s.residual;
  o->true_rel_l2 = s.true_rel_l2;
  o->true_linf = s.true_linf;
  o->ms = s.ms;
  o->sym_err = s.sym_err;
  o->device_flags = s.device_flags;
  o->kernel_launches = s.kernel_launches;
}

int validate_options(const sc_pcg_options* o) {
  if (!o) return SC_OK;
  if (!(o->tol >= 0.0) || o->max_iter < 1 || o->criterion < 0 || o->criterion > 1 ||
      o->precision < 0 || o->precision > 1 || !(o->inner_rtol > 0.0) || o->max_outer < 1 ||
      o->inner_method < 0 || o->inner_method > 1 || !(o->reliable_delta > 0.0 && o->reliable_delta < 1.0))
    return SC_ERR_INVALID;
  return SC_OK;
}

}  // namespace

extern "C" {

int sc_version(void) { return 10100; }  // 1.1: surface export, simulator export calls

const char* sc_status_string(int status) {
  switch (status) {
    case SC_OK: return "ok";
    case SC_ERR_INVALID: return "invalid argument";
    case SC_ERR_CUDA: return "CUDA error";
    case SC_ERR_NOMEM: return "out of device memory";
    case SC_ERR_BREAKDOWN: return "PCG breakdown";
    case SC_ERR_NOT_CONVERGED: return "not converged";
    case SC_ERR_TIMEOUT: return "device wait timed out";
    case SC_ERR_ASYMMETRIC: return "matrix is not symmetric";
    case SC_ERR_NONFINITE: return "non-finite value";
    case SC_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int sc_context_create(int device, sc_context** out) {
  if (!out) return SC_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return SC_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return SC_ERR_CUDA;
  sc_context* c = new (std::nothrow) sc_context();
  if (!c) return SC_ERR_NOMEM;
  c->c.device = device;
  cudaDeviceGetAttribute(&c->c.sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SC_ERR_CUDA;
  }
  c->c.stream = c->own;
  *out = c;
  return SC_OK;
}

void sc_context_destroy(sc_context* ctx) {
  if (!ctx) return;
  ctx_release(ctx);
}

int sc_context_set_stream(sc_context* ctx, void* stream) {
  if (!ctx) return SC_ERR_INVALID;
  ctx->c.stream = (cudaStream_t)stream;
  return SC_OK;
}

int sc_context_use_own_stream(sc_context* ctx) {
  if (!ctx) return SC_ERR_INVALID;
  ctx->c.stream = ctx->own;
  return SC_OK;
}

void* sc_context_stream(sc_context* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

int sc_context_synchronize(sc_context* ctx) {
  if (!ctx) return SC_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(ctx->c.stream);
  if (e != cudaSuccess) return ctx->c.set_error(SC_ERR_CUDA, cudaGetErrorString(e));
  return SC_OK;
}

int sc_context_set_wait_limit(sc_context* ctx, int polls) {
  if (!ctx) return SC_ERR_INVALID;
  ctx->c.wait_limit = polls > 0 ? polls : 0;
  return SC_OK;
}

const char* sc_context_last_error(sc_context* ctx) {
  return ctx ? ctx->c.last_error.c_str() : "no context";
}

void sc_pcg_default_options(sc_pcg_options* o) {
  if (!o) return;
  sc::PcgOptions d;
  o->tol = d.tol;
  o->max_iter = d.max_iter;
  o->criterion = d.criterion;
  o->precision = d.precision;
  o->mic_tau = d.tau;
  o->mic_sigma = d.sigma;
  o->inner_rtol = d.inner_rtol;
  o->max_outer = d.max_outer;
  o->check_symmetry = d.check_symmetry;
  o->true_residual = d.true_residual;
  o->inner_method = d.inner_method;
  o->reliable_delta = d.reliable_delta;
}

int sc_pcg_create(sc_context* ctx, int nx, int ny, int nz, const sc_pcg_options* opt,
                  sc_pcg** out) {
  if (!ctx || !out || nx < 1 || ny < 1 || nz < 1) return SC_ERR_INVALID;
  *out = nullptr;
  if (validate_options(opt)) return ctx->c.set_error(SC_ERR_INVALID, "invalid options");
  if ((int64_t)nx * ny * nz >= ((int64_t)1 << 31))
    return ctx->c.set_error(SC_ERR_UNSUPPORTED, "grid too large (int indices, as the reference)");
  cudaSetDevice(ctx->c.device);
  sc::PcgSolver* s = new (std::nothrow) sc::PcgSolver(&ctx->c, nx, ny, nz, to_internal(opt));
  if (!s) return SC_ERR_NOMEM;
  if (s->status()) {
    int st = s->status();
    delete s;
    return ctx->c.set_error(st == -3 ? SC_ERR_NOMEM : SC_ERR_CUDA, "pcg create failed");
  }
  sc_pcg* h = new (std::nothrow) sc_pcg{ctx, s};
  if (!h) {
    delete s;
    return SC_ERR_NOMEM;
  }
  ctx_retain(ctx);
  *out = h;
  return SC_OK;
}

void sc_pcg_destroy(sc_pcg* pcg) {
  if (!pcg) return;
  cudaSetDevice(pcg->ctx->c.device);
  cudaStreamSynchronize(pcg->ctx->c.stream);
  delete pcg->solver;
  sc_context* c = pcg->ctx;
  delete pcg;
  ctx_release(c);
}

int sc_pcg_set_options(sc_pcg* pcg, const sc_pcg_options* opt) {
  if (!pcg || !opt) return SC_ERR_INVALID;
  if (validate_options(opt)) return pcg->ctx->c.set_error(SC_ERR_INVALID, "invalid options");
  sc::PcgOptions o = to_internal(opt);
  bool pivots_change = o.tau != pcg->solver->options().tau ||
                       o.sigma != pcg->solver->options().sigma ||
                       o.precision != pcg->solver->options().precision;
  pcg->solver->set_options(o);
  if (pivots_change) pcg->solver->mark_system_changed();
  return SC_OK;
}

static int map_status(int rc) {
  switch (rc) {
    case 0: return SC_OK;
    case -1: return SC_ERR_INVALID;
    case -3: return SC_ERR_NOMEM;
    case -6: return SC_ERR_TIMEOUT;
    case -7: return SC_ERR_ASYMMETRIC;
    case -8: return SC_ERR_NONFINITE;
    default: return SC_ERR_CUDA;
  }
}

static int solve_status(const sc::PcgStats& st) {
  if (st.status == sc::DONE_BREAKDOWN) return SC_ERR_BREAKDOWN;
  return SC_OK;  // like the reference, non-convergence is reported through the residual
}

int sc_pcg_upload(sc_pcg* pcg, const double* adiag, const double* const* an, const double* rhs,
                  const uint8_t* active, int device_pointers) {
  if (!pcg || !adiag || !an || !rhs || !active || !an[0] || !an[3] || !an[5])
    return SC_ERR_INVALID;
  // the symmetry check reads the upper couplings too
  if (pcg->solver->options().check_symmetry && (!an[1] || !an[2] || !an[4]))
    return pcg->ctx->c.set_error(SC_ERR_INVALID, "check_symmetry needs all six neighbour arrays");
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->upload(adiag, an, rhs, active, device_pointers != 0));
}

int sc_pcg_upload_rhs(sc_pcg* pcg, const double* rhs, int device_pointers) {
  if (!pcg || !rhs) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->upload_rhs(rhs, device_pointers != 0));
}

int sc_pcg_solve_resident(sc_pcg* pcg, sc_pcg_stats* stats) {
  if (!pcg) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  sc::PcgStats st;
  int rc = map_status(pcg->solver->solve(&st));
  to_public(st, stats);
  if (rc) return rc;
  return solve_status(st);
}

int sc_pcg_download(sc_pcg* pcg, double* pg, int device_pointer) {
  if (!pcg || !pg) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->download_pressure(pg, device_pointer != 0));
}

static int solve_common(sc_pcg* pcg, const double* adiag, const double* const* an,
                        const double* rhs, const uint8_t* active, double* pg,
                        sc_pcg_stats* stats, int device) {
  const uint64_t l0 = pcg->solver->launches();
  int rc = sc_pcg_upload(pcg, adiag, an, rhs, active, device);
  if (rc) return rc;
  sc::PcgStats st;
  rc = map_status(pcg->solver->solve(&st));
  to_public(st, stats);
  if (rc) return rc;
  rc = map_status(pcg->solver->download_pressure(pg, device != 0));
  if (rc) return rc;
  if (stats) stats->kernel_launches = (int64_t)(pcg->solver->launches() - l0);
  if (device) {
    cudaError_t e = cudaStreamSynchronize(pcg->ctx->c.stream);
    if (e != cudaSuccess) return pcg->ctx->c.set_error(SC_ERR_CUDA, cudaGetErrorString(e));
  }
  return solve_status(st);
}

int sc_pcg_solve_host(sc_pcg* pcg, const double* adiag, const double* const* an,
                      const double* rhs, const uint8_t* active, double* pg,
                      sc_pcg_stats* stats) {
  if (!pg) return SC_ERR_INVALID;
  return solve_common(pcg, adiag, an, rhs, active, pg, stats, 0);
}

int sc_pcg_solve_device(sc_pcg* pcg, const double* adiag, const double* const* an,
                        const double* rhs, const uint8_t* active, double* pg,
                        sc_pcg_stats* stats) {
  if (!pg) return SC_ERR_INVALID;
  return solve_common(pcg, adiag, an, rhs, active, pg, stats, 1);
}

int sc_pcg_precond_device(sc_pcg* pcg, const double* r, double* z) {
  if (!pcg || !r || !z) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->precond_only(r, z));
}

int sc_pcg_apply_device(sc_pcg* pcg, const double* x, double* b) {
  if (!pcg || !x || !b) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->apply_only(x, b));
}

int sc_pcg_time_kernels(sc_pcg* pcg, int reps, double* ms_out) {
  if (!pcg || reps < 1 || !ms_out) return SC_ERR_INVALID;
  cudaSetDevice(pcg->ctx->c.device);
  return map_status(pcg->solver->time_kernels(reps, ms_out));
}

int sc_fvm_build_system_device(sc_context* ctx, int nx, int ny, int nz, double h, double dt,
                               int precision, const void* u, const void* v, const void* w,
                               const double* fluid_sdf, const double* collider_sdf,
                               double* adiag, double* const* an, double* rhs, uint8_t* active,
                               double* u_wt, double* v_wt, double* w_wt) {
  if (!ctx || nx < 1 || ny < 1 || nz < 1 || !(h > 0.0) || !u || !v || !w || !fluid_sdf ||
      !u_wt || !v_wt || !w_wt || (precision != SC_REAL_F64 && precision != SC_REAL_F32))
    return SC_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  sc::SystemOut out;
  out.adiag = adiag;
  if (an)
    for (int d = 0; d < 6; d++) out.an[d] = an[d];
  out.rhs = rhs;
  out.active = active;
  int rc = precision == SC_REAL_F64
               ? sc::fvm_build_system<double>(ctx->c.stream, nx, ny, nz, h, dt, (const double*)u,
                                              (const double*)v, (const double*)w, fluid_sdf,
                                              collider_sdf, u_wt, v_wt, w_wt, out)
               : sc::fvm_build_system<float>(ctx->c.stream, nx, ny, nz, h, dt, (const float*)u,
                                             (const float*)v, (const float*)w, fluid_sdf,
                                             collider_sdf, u_wt, v_wt, w_wt, out);
  if (rc) return ctx->c.set_error(SC_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  return SC_OK;
}

int sc_fvm_project_device(sc_context* ctx, int nx, int ny, int nz, double h, double dt,
                          int precision, void* u, void* v, void* w, const double* pg,
                          const double* fluid_sdf, const double* u_wt, const double* v_wt,
                          const double* w_wt) {
  if (!ctx || nx < 1 || ny < 1 || nz < 1 || !(h > 0.0) || !u || !v || !w || !pg || !fluid_sdf ||
      !u_wt || !v_wt || !w_wt || (precision != SC_REAL_F64 && precision != SC_REAL_F32))
    return SC_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  int rc = precision == SC_REAL_F64
               ? sc::fvm_project<double>(ctx->c.stream, nx, ny, nz, h, dt, (double*)u, (double*)v,
                                         (double*)w, pg, nullptr, fluid_sdf, u_wt, v_wt, w_wt)
               : sc::fvm_project<float>(ctx->c.stream, nx, ny, nz, h, dt, (float*)u, (float*)v,
                                        (float*)w, pg, nullptr, fluid_sdf, u_wt, v_wt, w_wt);
  if (rc) return ctx->c.set_error(SC_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  return SC_OK;
}

int sc_mic_precond_noalloc_device(sc_context* ctx, int nx, int ny, int nz, const double* adiag,
                                  const double* const* an, const double* r,
                                  const uint8_t* active, double* z, double tau, double sigma) {
  if (!ctx || nx < 1 || ny < 1 || nz < 1 || !adiag || !an || !an[0] || !an[3] || !an[5] || !r ||
      !active || !z)
    return SC_ERR_INVALID;
  if (cudaSetDevice(ctx->c.device) != cudaSuccess) return SC_ERR_CUDA;
  std::string msg;
  int rc = sc::mic_precond_noalloc(ctx->c.stream, ctx->c.device, ctx->c.sm_count, nx, ny, nz, adiag,
                                   an, r, active, z, tau, sigma, &msg);
  if (rc) return ctx->c.set_error(map_status(rc), msg);
  return SC_OK;
}

// ---------------------------------------------------------------------------------
// Particle/grid transfers (device, FP64).

static bool grid_ok(int nx, int ny, int nz, double h) {
  return nx >= 1 && ny >= 1 && nz >= 1 && h > 0.0 && (int64_t)(nx + 1) * (ny + 1) * (nz + 1) < ((int64_t)1 << 31);
}

static int finish(sc_context* ctx, int rc, const char* what) {
  if (rc == 0) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return SC_OK;
    return ctx->c.set_error(SC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  return ctx->c.set_error(map_status(rc), std::string(what) + " failed");
}

int sc_flip_p2g_device(sc_context* ctx, int64_t n, const double* pos, const double* vel, int nx,
                       int ny, int nz, double h, double* u, double* v, double* w, double* u_wt,
                       double* v_wt, double* w_wt, uint8_t* u_valid, uint8_t* v_valid,
                       uint8_t* w_valid, double* u_last, double* v_last, double* w_last) {
  if (!ctx || n < 0 || (n > 0 && (!pos || !vel)) || !grid_ok(nx, ny, nz, h) || !u || !v || !w ||
      !u_wt || !v_wt || !w_wt || !u_valid || !v_valid || !w_valid ||
      ((u_last || v_last || w_last) && !(u_last && v_last && w_last)))
    return SC_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return finish(ctx,
                sc::flip_p2g(ctx->c.stream, n, pos, vel, nx, ny, nz, h, u, v, w, u_wt, v_wt, w_wt,
                             u_valid, v_valid, w_valid, u_last, v_last, w_last),
                "p2g");
}

int sc_sample_velocity_device(sc_context* ctx, int64_t n, const double* pts, int nx, int ny,
                              int nz, double h, const double* u, const double* v,
                              const double* w, double* out) {
  if (!ctx || n < 0 || (n > 0 && (!pts || !out)) || !grid_ok(nx, ny, nz, h) || !u || !v || !w)
    return SC_ERR_INVALID;
  if (n == 0) return SC_OK;
  cudaSetDevice(ctx->c.device);
  return finish(ctx, sc::flip_sample(ctx->c.stream, n, pts, nx, ny, nz, h, u, v, w, out),
                "sample_velocity");
}

int sc_flip_g2p_device(sc_context* ctx, int64_t n, const double* pos, double* vel, int nx, int ny,
                       int nz, double h, const double* u, const double* v, const double* w,
                       const double* u_last, const double* v_last, const double* w_last,
                       double alpha) {
  if (!ctx || n < 0 || (n > 0 && (!pos || !vel)) || !grid_ok(nx, ny, nz, h) || !u || !v || !w ||
      (alpha >= 0.0 && (!u_last || !v_last || !w_last)) || alpha > 1.0)
    return SC_ERR_INVALID;
  if (n == 0) return SC_OK;
  cudaSetDevice(ctx->c.device);
  return finish(ctx,
                sc::flip_g2p(ctx->c.stream, n, pos, vel, nx, ny, nz, h, u, v, w, u_last, v_last,
                             w_last, alpha),
                "g2p");
}

int sc_flip_advect_device(sc_context* ctx, int64_t n, double* pos, double* vel, int nx, int ny,
                          int nz, double h, const double* u, const double* v, const double* w,
                          const double* collider_sdf, double dt) {
  if (!ctx || n < 0 || (n > 0 && (!pos || !vel)) || !grid_ok(nx, ny, nz, h) || !u || !v || !w ||
      !(dt >= 0.0))
    return SC_ERR_INVALID;
  if (n == 0) return SC_OK;
  cudaSetDevice(ctx->c.device);
  return finish(ctx,
                sc::flip_advect(ctx->c.stream, n, pos, vel, nx, ny, nz, h, u, v, w, collider_sdf,
                                dt),
                "advect");
}

int sc_reconstruct_device(sc_context* ctx, int64_t n, const double* pos, int nx, int ny, int nz,
                          double h, double radius, double* sdf, uint8_t* valid) {
  if (!ctx || n < 0 || (n > 0 && !pos) || !grid_ok(nx, ny, nz, h) || !(radius > 0.0) || !sdf ||
      !valid)
    return SC_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return finish(ctx, sc::flip_reconstruct(ctx->c.stream, n, pos, nx, ny, nz, h, radius, sdf, valid),
                "reconstruct");
}

// ---------------------------------------------------------------------------------
// Mesh -> SDF.

static int mesh_sdf(sc_context* ctx, int nx, int ny, int nz, double h, const double* origin,
                    const double* vertices, int64_t nvertices, const int32_t* triangles,
                    int64_t ntriangles, int exact_band, int flags, double* sdf, int32_t* closest,
                    bool device) {
  if (!ctx || !grid_ok(nx, ny, nz, h) || nvertices < 0 || ntriangles < 0 || ntriangles > INT_MAX ||
      (ntriangles > 0 && (!vertices || !triangles)) || exact_band < 0 || !sdf ||
      (flags != SC_MESH_REFERENCE_DISTANCE && flags != SC_MESH_EXACT_DISTANCE))
    return SC_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  cudaStream_t st = ctx->c.stream;
  const int64_t N = (int64_t)nx * ny * nz;
  sc::MeshSdfArgs a{nx, ny, nz, h, origin ? origin[0] : 0.0, origin ? origin[1] : 0.0,
                    origin ? origin[2] : 0.0, vertices, nvertices, triangles, ntriangles, exact_band,
                    flags == SC_MESH_EXACT_DISTANCE, ctx->c.wait_limit};
  double* d_sdf = sdf;
  int32_t* d_cl = closest;
  void *dv = nullptr, *dt = nullptr;
  if (!device) {
    if (cudaMallocAsync(&d_sdf, sizeof(double) * (size_t)N, st) != cudaSuccess ||
        (closest && cudaMallocAsync((void**)&d_cl, sizeof(int32_t) * (size_t)N, st) != cudaSuccess) ||
        cudaMallocAsync(&dv, sizeof(double) * 3 * (size_t)std::max<int64_t>(nvertices, 1), st) != cudaSuccess ||
        cudaMallocAsync(&dt, sizeof(int32_t) * 3 * (size_t)std::max<int64_t>(ntriangles, 1), st) != cudaSuccess)
      return ctx->c.set_error(SC_ERR_NOMEM, "mesh_to_sdf: staging allocation failed");
    if (nvertices > 0)
      cudaMemcpyAsync(dv, vertices, sizeof(double) * 3 * (size_t)nvertices, cudaMemcpyHostToDevice, st);
    if (ntriangles > 0)
      cudaMemcpyAsync(dt, triangles, sizeof(int32_t) * 3 * (size_t)ntriangles, cudaMemcpyHostToDevice, st);
    a.vertices = (const double*)dv;
    a.triangles = (const int32_t*)dt;
  }
  // scratch kept by the context: a per-call stream-ordered allocation can hand
  // its pages back at the synchronisations and map them again on the next call
  const size_t need = sc::mesh_to_sdf_scratch_bytes(a, d_cl == nullptr);
  if (ctx->mesh_scratch_bytes < need) {
    cudaStreamSynchronize(st);
    if (ctx->mesh_scratch) cudaFree(ctx->mesh_scratch);
    ctx->mesh_scratch = nullptr;
    ctx->mesh_scratch_bytes = 0;
    if (cudaMalloc(&ctx->mesh_scratch, need) != cudaSuccess) {
      ctx->mesh_scratch = nullptr;
      cudaGetLastError();
      return ctx->c.set_error(SC_ERR_NOMEM, "mesh_to_sdf: scratch allocation failed");
    }
    ctx->mesh_scratch_bytes = need;
  }
  std::string msg;
  int rc = sc::mesh_to_sdf(st, a, d_sdf, d_cl, ctx->mesh_scratch, ctx->mesh_scratch_bytes, &msg);
  if (!device) {
    if (rc == 0) {
      cudaMemcpyAsync(sdf, d_sdf, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, st);
      if (closest) cudaMemcpyAsync(closest, d_cl, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(d_sdf, st);
    if (closest) cudaFreeAsync(d_cl, st);
    cudaFreeAsync(dv, st);
    cudaFreeAsync(dt, st);
    cudaStreamSynchronize(st);
  }
  if (rc) return ctx->c.set_error(map_status(rc), msg);
  return finish(ctx, 0, "mesh_to_sdf");
}

int sc_mesh_to_sdf_device(sc_context* ctx, int nx, int ny, int nz, double h, const double* origin,
                          const double* vertices, int64_t nvertices, const int32_t* triangles,
                          int64_t ntriangles, int exact_band, int flags, double* sdf, int32_t* closest) {
  return mesh_sdf(ctx, nx, ny, nz, h, origin, vertices, nvertices, triangles, ntriangles, exact_band,
                  flags, sdf, closest, true);
}

int sc_mesh_to_sdf_host(sc_context* ctx, int nx, int ny, int nz, double h, const double* origin,
                        const double* vertices, int64_t nvertices, const int32_t* triangles,
                        int64_t ntriangles, int exact_band, int flags, double* sdf, int32_t* closest) {
  return mesh_sdf(ctx, nx, ny, nz, h, origin, vertices, nvertices, triangles, ntriangles, exact_band,
                  flags, sdf, closest, false);
}

// ---------------------------------------------------------------------------------
// Surface export (marching cubes).

// Grows a device buffer the context keeps to at least `need` bytes (its
// contents are dropped).
static bool ctx_grow(sc_context* ctx, void** buf, size_t* have, size_t need) {
  if (*have >= need) return true;
  cudaStreamSynchronize(ctx->c.stream);
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  if (cudaMalloc(buf, need) != cudaSuccess) {
    *buf = nullptr;
    cudaGetLastError();
    return false;
  }
  *have = need;
  return true;
}

static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

static int rebuild_surface(sc_context* ctx, int nx, int ny, int nz, const double* spacing,
                           const double* origin, const double* sdf, double* vertices, double* normals,
                           uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity,
                           int64_t* nvertices, int64_t* nindices, bool device) {
  if (!ctx) return SC_ERR_INVALID;
  const bool any = vertices || normals || indices, all = vertices && normals && indices;
  bool ok = nx >= 1 && ny >= 1 && nz >= 1 && (int64_t)(nx + 1) * (ny + 1) * (nz + 1) < ((int64_t)1 << 31) &&
            spacing && sdf && nvertices && nindices && any == all && vertex_capacity >= 0 && index_capacity >= 0;
  for (int d = 0; ok && d < 3; d++) ok = spacing[d] > 0.0 && spacing[d] < 1e300;
  if (!ok) return ctx->c.set_error(SC_ERR_INVALID, "rebuild_surface: invalid argument");
  cudaSetDevice(ctx->c.device);
  cudaStream_t st = ctx->c.stream;
  const size_t N = (size_t)nx * ny * nz;
  sc::SurfaceArgs a{nx, ny, nz, spacing[0], spacing[1], spacing[2], origin ? origin[0] : 0.0,
                    origin ? origin[1] : 0.0, origin ? origin[2] : 0.0, sdf};
  const size_t sdf_bytes = device ? 0 : round256(sizeof(double) * N);
  if (!ctx_grow(ctx, &ctx->surf_scratch, &ctx->surf_scratch_bytes, sdf_bytes + sc::surface_scratch_bytes(a)))
    return ctx->c.set_error(SC_ERR_NOMEM, "rebuild_surface: scratch allocation failed");
  char* scratch = (char*)ctx->surf_scratch;
  if (!device) {
    cudaMemcpyAsync(scratch, sdf, sizeof(double) * N, cudaMemcpyHostToDevice, st);
    a.sdf = (const double*)scratch;
    scratch += sdf_bytes;
  }
  int64_t nv = 0, ni = 0;
  if (sc::surface_count(st, a, scratch, &nv, &ni))
    return ctx->c.set_error(SC_ERR_CUDA, std::string("rebuild_surface: ") + cudaGetErrorString(cudaGetLastError()));
  *nvertices = nv;
  *nindices = ni;
  if (!any) return SC_OK;
  if (vertex_capacity < nv || index_capacity < ni)
    return ctx->c.set_error(SC_ERR_INVALID, "rebuild_surface: capacity below the mesh size");
  if (nv > (int64_t)UINT32_MAX - 1)
    return ctx->c.set_error(SC_ERR_UNSUPPORTED, "rebuild_surface: more vertices than uint32 indices address");
  if (ni == 0) return SC_OK;
  double *dv = vertices, *dn = normals;
  uint32_t* di = indices;
  const size_t vb = round256(sizeof(double) * 3 * (size_t)nv), ib = round256(sizeof(uint32_t) * (size_t)ni);
  if (!device) {
    if (!ctx_grow(ctx, &ctx->surf_stage, &ctx->surf_stage_bytes, 2 * vb + ib))
      return ctx->c.set_error(SC_ERR_NOMEM, "rebuild_surface: staging allocation failed");
    dv = (double*)ctx->surf_stage;
    dn = (double*)((char*)ctx->surf_stage + vb);
    di = (uint32_t*)((char*)ctx->surf_stage + 2 * vb);
  }
  std::string msg;
  int rc = sc::surface_fill(st, a, scratch, dv, dn, di, &msg);
  if (rc == 0 && !device) {
    cudaMemcpyAsync(vertices, dv, sizeof(double) * 3 * (size_t)nv, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(normals, dn, sizeof(double) * 3 * (size_t)nv, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(indices, di, sizeof(uint32_t) * (size_t)ni, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
  }
  if (rc) return ctx->c.set_error(map_status(rc), msg.empty() ? "rebuild_surface failed" : msg);
  return finish(ctx, 0, "rebuild_surface");
}

int sc_rebuild_surface_device(sc_context* ctx, int nx, int ny, int nz, const double* spacing,
                              const double* origin, const double* sdf, double* vertices, double* normals,
                              uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity,
                              int64_t* nvertices, int64_t* nindices) {
  return rebuild_surface(ctx, nx, ny, nz, spacing, origin, sdf, vertices, normals, indices, vertex_capacity,
                         index_capacity, nvertices, nindices, true);
}

int sc_rebuild_surface_host(sc_context* ctx, int nx, int ny, int nz, const double* spacing,
                            const double* origin, const double* sdf, double* vertices, double* normals,
                            uint32_t* indices, int64_t vertex_capacity, int64_t index_capacity,
                            int64_t* nvertices, int64_t* nindices) {
  return rebuild_surface(ctx, nx, ny, nz, spacing, origin, sdf, vertices, normals, indices, vertex_capacity,
                         index_capacity, nvertices, nindices, false);
}

// ---------------------------------------------------------------------------------
// Simulator.

void sc_fluid_default_config(int nx, int ny, int nz, double h, sc_fluid_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->h = h;
  c->precision = SC_REAL_F64;
  c->advection = SC_ADVECT_FLIP;
  c->flip_alpha = 0.97;
  c->cfl_factor = 5.0;
  c->gravity = 9.8;
  c->recon_factor = 0.8;
  c->sdf_extrap_iters = 10;
  c->smooth_iters = 5;
  c->vel_extrap_iters = 10;
  sc_pcg_default_options(&c->pcg);
}

int sc_fluid_create(sc_context* ctx, const sc_fluid_config* cfg, sc_fluid** out) {
  if (!ctx || !cfg || !out) return SC_ERR_INVALID;
  *out = nullptr;
  if (!grid_ok(cfg->nx, cfg->ny, cfg->nz, cfg->h) ||
      (cfg->precision != SC_REAL_F64 && cfg->precision != SC_REAL_F32) ||
      (cfg->advection != SC_ADVECT_FLIP && cfg->advection != SC_ADVECT_PIC) ||
      !(cfg->flip_alpha >= 0.0 && cfg->flip_alpha <= 1.0) || !(cfg->cfl_factor > 0.0) ||
      !(cfg->recon_factor > 0.0) || cfg->sdf_extrap_iters < 0 || cfg->smooth_iters < 0 ||
      cfg->vel_extrap_iters < 0 || validate_options(&cfg->pcg))
    return ctx->c.set_error(SC_ERR_INVALID, "invalid simulator configuration");
  sc::FluidConfig fc;
  fc.nx = cfg->nx;
  fc.ny = cfg->ny;
  fc.nz = cfg->nz;
  fc.h = cfg->h;
  fc.f32 = cfg->precision == SC_REAL_F32;
  fc.flip = cfg->advection == SC_ADVECT_FLIP;
  fc.flip_alpha = cfg->flip_alpha;
  fc.pcg = to_internal(&cfg->pcg);
  fc.cfl_factor = cfg->cfl_factor;
  fc.gravity = cfg->gravity;
  fc.recon_factor = cfg->recon_factor;
  fc.sdf_extrap_iters = cfg->sdf_extrap_iters;
  fc.smooth_iters = cfg->smooth_iters;
  fc.vel_extrap_iters = cfg->vel_extrap_iters;
  cudaSetDevice(ctx->c.device);
  sc::FluidSim* s = new (std::nothrow) sc::FluidSim(&ctx->c, fc);
  if (!s) return SC_ERR_NOMEM;
  if (s->status()) {
    int st = s->status();
    delete s;
    return ctx->c.set_error(map_status(st), "simulator create failed");
  }
  sc_fluid* f = new (std::nothrow) sc_fluid{ctx, s};
  if (!f) {
    delete s;
    return SC_ERR_NOMEM;
  }
  ctx_retain(ctx);
  *out = f;
  return SC_OK;
}

void sc_fluid_destroy(sc_fluid* sim) {
  if (!sim) return;
  cudaSetDevice(sim->ctx->c.device);
  delete sim->sim;
  sc_context* c = sim->ctx;
  delete sim;
  ctx_release(c);
}

static int fl_rc(sc_fluid* f, int rc) {
  if (rc == 0) return SC_OK;
  if (f->ctx->c.last_error.empty()) f->ctx->c.last_error = "simulator call failed";
  return map_status(rc);
}

int sc_fluid_set_particles(sc_fluid* sim, int64_t n, const double* pos, const double* vel,
                           int device_pointers) {
  if (!sim || n < 0 || (n > 0 && !pos) || n >= ((int64_t)1 << 31)) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->set_particles(n, pos, vel, device_pointers != 0));
}

int sc_fluid_set_collider(sc_fluid* sim, const double* sdf, int device_pointers) {
  if (!sim) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->set_collider(sdf, device_pointers != 0));
}

int sc_fluid_set_collider_mesh(sc_fluid* sim, const double* vertices, int64_t nvertices,
                               const int32_t* triangles, int64_t ntriangles, int flags,
                               int device_pointers) {
  if (!sim) return SC_ERR_INVALID;
  sc_context* ctx = sim->ctx;
  cudaSetDevice(ctx->c.device);
  const sc::FluidConfig& c = sim->sim->config();
  double* d_sdf = nullptr;
  if (cudaMallocAsync(&d_sdf, sizeof(double) * (size_t)c.nx * c.ny * c.nz, ctx->c.stream) != cudaSuccess)
    return ctx->c.set_error(SC_ERR_NOMEM, "set_collider_mesh: allocation failed");
  // setCollider uses an exact band of 3 cells (fluid-simulator.h:69)
  int rc = device_pointers
               ? sc_mesh_to_sdf_device(ctx, c.nx, c.ny, c.nz, c.h, nullptr, vertices, nvertices, triangles,
                                       ntriangles, 3, flags, d_sdf, nullptr)
               : -1;
  if (!device_pointers) {
    // host mesh: stage it, then build on the device
    void *dv = nullptr, *dt = nullptr;
    cudaStream_t st = ctx->c.stream;
    if (cudaMallocAsync(&dv, sizeof(double) * 3 * (size_t)std::max<int64_t>(nvertices, 1), st) != cudaSuccess ||
        cudaMallocAsync(&dt, sizeof(int32_t) * 3 * (size_t)std::max<int64_t>(ntriangles, 1), st) != cudaSuccess) {
      cudaFreeAsync(d_sdf, st);
      return ctx->c.set_error(SC_ERR_NOMEM, "set_collider_mesh: allocation failed");
    }
    if (nvertices > 0 && vertices)
      cudaMemcpyAsync(dv, vertices, sizeof(double) * 3 * (size_t)nvertices, cudaMemcpyHostToDevice, st);
    if (ntriangles > 0 && triangles)
      cudaMemcpyAsync(dt, triangles, sizeof(int32_t) * 3 * (size_t)ntriangles, cudaMemcpyHostToDevice, st);
    rc = sc_mesh_to_sdf_device(ctx, c.nx, c.ny, c.nz, c.h, nullptr, vertices ? (const double*)dv : nullptr,
                               nvertices, triangles ? (const int32_t*)dt : nullptr, ntriangles, 3, flags,
                               d_sdf, nullptr);
    cudaFreeAsync(dv, st);
    cudaFreeAsync(dt, st);
  }
  if (rc == SC_OK) rc = fl_rc(sim, sim->sim->set_collider(d_sdf, true));
  cudaFreeAsync(d_sdf, ctx->c.stream);
  cudaStreamSynchronize(ctx->c.stream);
  return rc;
}

int sc_fluid_cfl(sc_fluid* sim, double* dt) {
  if (!sim || !dt) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  *dt = sim->sim->cfl();
  return finish(sim->ctx, 0, "cfl");
}

static void stats_out(const sc::StepStats& s, sc_fluid_stats* o) {
  if (!o) return;
  o->substeps = s.substeps;
  o->pcg_iterations = s.pcg_iterations;
  o->pcg_outer = s.pcg_outer;
  o->pcg_residual = s.pcg_residual;
  o->ms_advect = s.ms_advect;
  o->ms_sort_sdf = s.ms_sort_sdf;
  o->ms_p2g = s.ms_p2g;
  o->ms_build = s.ms_build;
  o->ms_solve = s.ms_solve;
  o->ms_project_g2p = s.ms_project_g2p;
  o->ms_total = s.ms_total;
  o->kernel_launches = s.kernel_launches;
  o->pcg_status = s.pcg_status;
  o->pcg_flags = s.pcg_flags;
}

int sc_fluid_substep(sc_fluid* sim, double dt, sc_fluid_stats* stats) {
  if (!sim || !(dt > 0.0)) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  sc::StepStats s;
  int rc = sim->sim->substep(dt, &s);
  stats_out(s, stats);
  return fl_rc(sim, rc);
}

int sc_fluid_step(sc_fluid* sim, double frame_dt, sc_fluid_stats* stats) {
  if (!sim || !(frame_dt > 0.0)) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  sc::StepStats s;
  int rc = sim->sim->step(frame_dt, &s);
  stats_out(s, stats);
  return fl_rc(sim, rc);
}

int64_t sc_fluid_num_particles(sc_fluid* sim) { return sim ? sim->sim->num_particles() : 0; }

int sc_fluid_get_particles(sc_fluid* sim, double* pos, double* vel, int device_pointers) {
  if (!sim) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->get_particles(pos, vel, device_pointers != 0));
}

int sc_fluid_get_pressure(sc_fluid* sim, double* pg, int device_pointers) {
  if (!sim || !pg) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->get_pressure(pg, device_pointers != 0));
}

int sc_fluid_get_faces(sc_fluid* sim, double* u, double* v, double* w, int device_pointers) {
  if (!sim) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->get_faces(u, v, w, device_pointers != 0));
}

int sc_fluid_get_fluid_sdf(sc_fluid* sim, double* sdf, int device_pointers) {
  if (!sim || !sdf) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->get_fluid_sdf(sdf, device_pointers != 0));
}

int sc_fluid_get_collider_sdf(sc_fluid* sim, double* sdf, int device_pointers) {
  if (!sim || !sdf) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->get_collider_sdf(sdf, device_pointers != 0));
}

int sc_fluid_reconstruct(sc_fluid* sim, double radius) {
  if (!sim || !(radius < 1e300)) return SC_ERR_INVALID;  // rejects NaN and Inf
  cudaSetDevice(sim->ctx->c.device);
  const double h = sim->sim->config().h;
  return fl_rc(sim, sim->sim->reconstruct(radius > 0.0 ? radius : 1.2 * h / std::sqrt(2.0)));
}

int sc_fluid_smooth_fluid_surface(sc_fluid* sim, int iters) {
  if (!sim || iters < 0) return SC_ERR_INVALID;
  cudaSetDevice(sim->ctx->c.device);
  return fl_rc(sim, sim->sim->smooth_fluid_surface(iters));
}

// ---------------------------------------------------------------------------------
// Differentiable substeps.

void sc_diff_default_config(int nx, int ny, int nz, double h, double dt, int steps, sc_diff_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->h = h;
  c->dt = dt;
  c->precision = SC_REAL_F64;
  c->advection = SC_ADVECT_FLIP;
  c->flip_alpha = 0.97;
  c->gravity = 9.8;
  c->recon_factor = 0.8;
  c->sdf_extrap_iters = 10;
  c->smooth_iters = 5;
  c->vel_extrap_iters = 10;
  c->steps = steps;
  c->checkpoint_every = 5;
  sc_pcg_default_options(&c->pcg);
  c->pcg.tol = 1e-10;
  c->pcg.criterion = SC_CRIT_REL_L2;
  c->pcg.max_iter = 2000;
  c->pcg.mic_tau = 0.0;
}

int sc_diff_create(sc_context* ctx, const sc_diff_config* cfg, sc_diff** out) {
  if (!ctx || !cfg || !out) return SC_ERR_INVALID;
  *out = nullptr;
  if (!grid_ok(cfg->nx, cfg->ny, cfg->nz, cfg->h) || !(cfg->dt > 0.0) || cfg->steps < 1 ||
      cfg->checkpoint_every < 1 || (cfg->precision != SC_REAL_F64 && cfg->precision != SC_REAL_F32) ||
      (cfg->advection != SC_ADVECT_FLIP && cfg->advection != SC_ADVECT_PIC) ||
      !(cfg->flip_alpha >= 0.0 && cfg->flip_alpha <= 1.0) || !(cfg->recon_factor > 0.0) ||
      cfg->sdf_extrap_iters < 0 || cfg->smooth_iters < 0 || cfg->vel_extrap_iters < 0 ||
      validate_options(&cfg->pcg))
    return ctx->c.set_error(SC_ERR_INVALID, "invalid differentiable-step configuration");
  sc::DiffConfig dc;
  dc.nx = cfg->nx;
  dc.ny = cfg->ny;
  dc.nz = cfg->nz;
  dc.h = cfg->h;
  dc.dt = cfg->dt;
  dc.f32 = cfg->precision == SC_REAL_F32;
  dc.flip = cfg->advection == SC_ADVECT_FLIP;
  dc.flip_alpha = cfg->flip_alpha;
  dc.gravity = cfg->gravity;
  dc.recon_factor = cfg->recon_factor;
  dc.sdf_extrap_iters = cfg->sdf_extrap_iters;
  dc.smooth_iters = cfg->smooth_iters;
  dc.vel_extrap_iters = cfg->vel_extrap_iters;
  dc.steps = cfg->steps;
  dc.checkpoint_every = cfg->checkpoint_every;
  dc.pcg = to_internal(&cfg->pcg);
  cudaSetDevice(ctx->c.device);
  sc::DiffSim* s = new (std::nothrow) sc::DiffSim(&ctx->c, dc);
  if (!s) return SC_ERR_NOMEM;
  if (s->status()) {
    int st = s->status();
    delete s;
    return ctx->c.set_error(map_status(st), "differentiable step create failed");
  }
  sc_diff* d = new (std::nothrow) sc_diff{ctx, s};
  if (!d) {
    delete s;
    return SC_ERR_NOMEM;
  }
  ctx_retain(ctx);
  *out = d;
  return SC_OK;
}

void sc_diff_destroy(sc_diff* d) {
  if (!d) return;
  cudaSetDevice(d->ctx->c.device);
  delete d->sim;
  sc_context* c = d->ctx;
  delete d;
  ctx_release(c);
}

static int df_rc(sc_diff* d, int rc) {
  if (rc == 0) return SC_OK;
  if (d->ctx->c.last_error.empty()) d->ctx->c.last_error = "differentiable step call failed";
  return map_status(rc);
}

int sc_diff_set_particles(sc_diff* d, int64_t n, const double* pos, int device_pointers) {
  if (!d || n < 1 || !pos || n >= ((int64_t)1 << 31)) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  return df_rc(d, d->sim->set_particles(n, pos, device_pointers != 0));
}

int sc_diff_set_target(sc_diff* d, const double* rho, int device_pointers) {
  if (!d || !rho) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  return df_rc(d, d->sim->set_target(rho, device_pointers != 0));
}

int sc_diff_forward(sc_diff* d, const double* const* U, int tape, double* loss) {
  if (!d || !U || !U[0] || !U[1] || !U[2] || !loss || tape < SC_TAPE_NONE || tape > SC_TAPE_REPLAY)
    return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  const double* u[3] = {U[0], U[1], U[2]};
  return df_rc(d, d->sim->forward(u, tape, loss));
}

int sc_diff_backward(sc_diff* d, double* const* grad_U) {
  if (!d || !grad_U || !grad_U[0] || !grad_U[1] || !grad_U[2]) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  double* g[3] = {grad_U[0], grad_U[1], grad_U[2]};
  return df_rc(d, d->sim->backward(g));
}

int sc_diff_get_density(sc_diff* d, double* rho, int device_pointers) {
  if (!d || !rho) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  return df_rc(d, d->sim->get_density(rho, device_pointers != 0));
}

int sc_diff_get_particles(sc_diff* d, double* pos, double* vel, int device_pointers) {
  if (!d) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  return df_rc(d, d->sim->get_particles(pos, vel, device_pointers != 0));
}

int sc_diff_get_pressure(sc_diff* d, double* p, int device_pointers) {
  if (!d || !p) return SC_ERR_INVALID;
  cudaSetDevice(d->ctx->c.device);
  return df_rc(d, d->sim->get_pressure(p, device_pointers != 0));
}

int sc_diff_last_pcg_iterations(sc_diff* d) { return d ? d->sim->last_pcg_iterations() : 0; }

}  // extern "C"
