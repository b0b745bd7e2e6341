// sc_flip.cu -- the FLIP/PIC substep of SimCraft FluidSim on B200 (sm_100a).
//
// Restates fluid::cpu::FluidSimulator::substep (FluidSim/src/cpu/fluid-simulator.cc:140-182)
// and its callees on the GPU:
//   advect + handleCollision    advect-solver.cc:100-137, 170-187   k_advect
//   NaiveReconstructor          sdf.h:204-229, ns-util.h:46-109      k_keys/scan/scatter + k_reconstruct
//   extrapolateFluidSdf/smooth  cpu/fluid-simulator.h:123-166, fluid-simulator.cc:39-74
//   solveP2G                    advect-solver.cc:188-271             k_p2g_splat + k_p2g_normalize
//   applyDirichletBoundary, extrapolate, applyForce, buildSystem, solvePressure, project,
//   applyCollider, solveG2P     fluid-simulator.cc:13-138, advect-solver.cc:157-169
//
// Particles are re-sorted by cell every substep (counting sort; inside a cell by
// original index).  The sort gives the reconstruction the reference's bucket
// order, lets P2G splat a tile of cells into shared memory, and keeps the
// gathers of neighbouring threads on the same grid nodes.  Arithmetic that
// decides discrete outcomes (nearest node, reconstruction distances, kernel
// weights, sampling sums) uses explicitly rounded operations in the reference's
// order so that it matches the CPU bit for bit; only P2G's summation order
// differs (as in the reference's parallel splat).
#include <algorithm>
#include <cmath>
#include <cstring>

#include <vector>
#include "sc_flip.cuh"
#include "sc_fvm.cuh"

#include "sc_flip_dev.cuh"

namespace sc {


// =================================================================================
// FluidSim

FluidSim::FluidSim(Context* ctx, const FluidConfig& cfg) : ctx_(ctx), c_(cfg) {
  if (c_.nx < 1 || c_.ny < 1 || c_.nz < 1 || !(c_.h > 0)) {
    status_ = -1;
    return;
  }
  rs_ = c_.f32 ? sizeof(float) : sizeof(double);
  const int nx = c_.nx, ny = c_.ny, nz = c_.nz;
  const int64_t N = (int64_t)nx * ny * nz;
  fsz_[0] = (int64_t)(nx + 1) * ny * nz;
  fsz_[1] = (int64_t)nx * (ny + 1) * nz;
  fsz_[2] = (int64_t)nx * ny * (nz + 1);
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    allocs_.push_back(p);
    cudaMemsetAsync(p, 0, bytes, ctx_->stream);
    return p;
  };
  bool ok = true;
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) {
      ok &= (g_[a][b] = alloc(rs_ * fsz_[a])) != nullptr;
      ok &= (gv_[a][b] = (uint8_t*)alloc(fsz_[a])) != nullptr;
    }
    ok &= (gw_[a] = alloc(rs_ * fsz_[a])) != nullptr;
    ok &= (last_[a] = alloc(rs_ * fsz_[a])) != nullptr;
    ok &= (wt_[a] = (double*)alloc(sizeof(double) * fsz_[a])) != nullptr;
  }
  for (int b = 0; b < 2; b++) {
    ok &= (sdf_[b] = (double*)alloc(sizeof(double) * N)) != nullptr;
    ok &= (sdfv_[b] = (uint8_t*)alloc(N)) != nullptr;
  }
  ok &= (cnt_ = (int*)alloc(sizeof(int) * N)) != nullptr;
  ok &= (start_ = (int*)alloc(sizeof(int) * N)) != nullptr;
  ok &= (cursor_ = (int*)alloc(sizeof(int) * N)) != nullptr;
  ok &= (bsum_ = (int*)alloc(sizeof(int) * ((N + 1023) / 1024 + 1))) != nullptr;
  ok &= (redbuf_ = (double*)alloc(sizeof(double) * 4)) != nullptr;
  ok &= (p2g_scr_ = alloc(p2g_scratch_bytes(Geo{nx, ny, nz}, rs_))) != nullptr;
  for (int k = 0; k < 2; k++) ok &= (clsS_[k] = (uint8_t*)alloc((size_t)iter_tiles<double>(nx, ny, nz))) != nullptr;
  for (int k = 0; k < 2; k++)
    for (int a = 0; a < 3; a++)  // the FP64 tiles are the smaller ones: enough for either
      ok &= (cls_[k][a] = (uint8_t*)alloc((size_t)iter_tiles<double>(nx + (a == 0), ny + (a == 1), nz + (a == 2)))) !=
            nullptr;
  if (ok && cudaMallocHost(&host_red_, sizeof(double) * 4) != cudaSuccess) ok = false;
  if (!ok) {
    status_ = -3;
    return;
  }
  pcg_ = new PcgSolver(ctx, nx, ny, nz, c_.pcg);
  if (pcg_->status()) {
    status_ = pcg_->status();
    return;
  }
  for (auto& e : ev_) cudaEventCreate(&e);
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) status_ = -2;
}

FluidSim::~FluidSim() {
  cudaStreamSynchronize(ctx_->stream);
  delete pcg_;
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  if (host_red_) cudaFreeHost(host_red_);
  for (void* p : allocs_) cudaFree(p);
  for (void* p : {px_, py_, pz_, vx_, vy_, vz_, spx_, spy_, spz_, svx_, svy_, svz_, (void*)id_,
                  (void*)sid_, (void*)key_})
    if (p) cudaFree(p);
}

int FluidSim::err(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ctx_->set_error(-2, std::string(where) + ": " + cudaGetErrorString(e));
  return 0;
}

int FluidSim::alloc_particles(int64_t n) {
  if (n <= cap_) return 0;
  void** bufs[] = {&px_, &py_, &pz_, &vx_, &vy_, &vz_, &spx_, &spy_, &spz_, &svx_, &svy_, &svz_};
  for (void** b : bufs) {
    if (*b) cudaFree(*b);
    if (cudaMalloc(b, rs_ * (size_t)n) != cudaSuccess) return ctx_->set_error(-3, "particle allocation failed");
  }
  for (int64_t** b : {&id_, &sid_}) {
    if (*b) cudaFree(*b);
    if (cudaMalloc(b, sizeof(int64_t) * (size_t)n) != cudaSuccess)
      return ctx_->set_error(-3, "particle allocation failed");
  }
  if (key_) cudaFree(key_);
  if (cudaMalloc(&key_, sizeof(int) * (size_t)n) != cudaSuccess)
    return ctx_->set_error(-3, "particle allocation failed");
  cap_ = n;
  return 0;
}

int FluidSim::set_particles(int64_t n, const double* pos, const double* vel, bool device) {
  if (n < 0) return ctx_->set_error(-1, "negative particle count");
  int e = alloc_particles(std::max<int64_t>(n, 1));
  if (e) return e;
  cudaStream_t st = ctx_->stream;
  const double *dp = pos, *dv = vel;
  double* stage = nullptr;
  if (!device && n > 0) {
    if (cudaMallocAsync(&stage, sizeof(double) * 6 * (size_t)n, st) != cudaSuccess)
      return ctx_->set_error(-3, "staging allocation failed");
    cudaMemcpyAsync(stage, pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, st);
    dp = stage;
    dv = nullptr;
    if (vel) {
      cudaMemcpyAsync(stage + 3 * n, vel, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, st);
      dv = stage + 3 * n;
    }
  }
  n_ = n;
  if (n > 0) {
    Parts p{px_, py_, pz_, vx_, vy_, vz_};
    if (c_.f32)
      k_aos_to_soa<float><<<nblk(n), kT, 0, st>>>(n, dp, dv, PartsT<float>::from(p), id_);
    else
      k_aos_to_soa<double><<<nblk(n), kT, 0, st>>>(n, dp, dv, PartsT<double>::from(p), id_);
  }
  if (stage) cudaFreeAsync(stage, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("set_particles");
  return err("set_particles");
}

int FluidSim::set_collider(const double* sdf, bool device) {
  const int64_t N = (int64_t)c_.nx * c_.ny * c_.nz;
  if (!sdf) {
    collider_ = nullptr;  // empty mesh: manifold2SDF leaves 1e9 everywhere
    return 0;
  }
  if (!collider_) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * N) != cudaSuccess) return ctx_->set_error(-3, "collider allocation failed");
    allocs_.push_back(p);
    collider_ = (double*)p;
  }
  cudaMemcpyAsync(collider_, sdf, sizeof(double) * N,
                  device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx_->stream);
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return err("set_collider");
  return err("set_collider");
}

double FluidSim::cfl() {
  cudaStream_t st = ctx_->stream;
  cudaMemsetAsync(redbuf_, 0, sizeof(double), st);
  // a few blocks per SM, each looping over the grid: one atomic per block (a
  // block per 256 nodes queued ~65k atomics on the one word at 256^3)
  for (int a = 0; a < 3; a++) {
    const int nb = std::min(nblk(fsz_[a]), 2048);
    if (c_.f32)
      k_maxabs<float><<<nb, kT, 0, st>>>(fsz_[a], (const float*)g_[a][gcur_[a]], redbuf_);
    else
      k_maxabs<double><<<nb, kT, 0, st>>>(fsz_[a], (const double*)g_[a][gcur_[a]], redbuf_);
  }
  launches_ += 3;
  cudaMemcpyAsync(host_red_, redbuf_, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  const double h = c_.h;
  double cfl = h / 1e-6;
  const double m = host_red_[0];
  if (m > 0.0) cfl = std::min(cfl, h / m);
  return c_.cfl_factor * std::max(1e-3, cfl);
}

template <class T>
int FluidSim::substep_t(double dt, StepStats* stt) {
  cudaStream_t st = ctx_->stream;
  const int nx = c_.nx, ny = c_.ny, nz = c_.nz;
  const double h = c_.h;
  const Geo G{nx, ny, nz};
  const int64_t N = (int64_t)nx * ny * nz;
  const int64_t n = n_;
  const int64_t l0 = launches_;
  PartsT<T> P{(T*)px_, (T*)py_, (T*)pz_, (T*)vx_, (T*)vy_, (T*)vz_};
  PartsT<T> S{(T*)spx_, (T*)spy_, (T*)spz_, (T*)svx_, (T*)svy_, (T*)svz_};
  auto G_ = [&](int a) { return (T*)g_[a][gcur_[a]]; };
  cudaEventRecord(ev_[0], st);
  // clear() (fluid-simulator.cc:20-37)
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 2; b++) {
      cudaMemsetAsync(g_[a][b], 0, rs_ * fsz_[a], st);
      cudaMemsetAsync(gv_[a][b], 0, fsz_[a], st);
    }
    cudaMemsetAsync(gw_[a], 0, rs_ * fsz_[a], st);
  }
  // advect on the just-cleared grids (fluid-simulator.cc:143)
  if (n > 0 && collider_)
    k_advect_still<T, true><<<nblk(n), kT, 0, st>>>(n, P, G, h, collider_, dt);
  else if (n > 0)
    k_advect_still<T, false><<<nblk(n), kT, 0, st>>>(n, P, G, h, nullptr, dt);
  launches_ += 1;
  cudaEventRecord(ev_[1], st);
  // sort by cell, then reconstruct (fluid-simulator.cc:146-148)
  if (n > 0) {
    SortBufs sb{key_, cnt_, start_, cursor_, bsum_};
    launches_ += sort_particles<T>(st, n, G, h, P, id_, S, sid_, sb);
    std::swap(px_, spx_);
    std::swap(py_, spy_);
    std::swap(pz_, spz_);
    std::swap(vx_, svx_);
    std::swap(vy_, svy_);
    std::swap(vz_, svz_);
    std::swap(id_, sid_);
    P = PartsT<T>{(T*)px_, (T*)py_, (T*)pz_, (T*)vx_, (T*)vy_, (T*)vz_};
  } else {
    cudaMemsetAsync(cnt_, 0, sizeof(int) * N, st);
    cudaMemsetAsync(start_, 0, sizeof(int) * N, st);
  }
  if (launch_reconstruct<T>(st, G, h, c_.recon_factor * h, start_, cnt_, P.px, P.py, P.pz, sdf_[scur_],
                            sdfv_[svcur_], clsS_[0]))
    return ctx_->set_error(-1, "reconstruct: radius reaches past 6 cells");
  launches_ += 1;
  // extrapolateFluidSdf(10), temporally blocked
  launches_ += launch_iter_cells<ITER_SDF>(st, G, c_.sdf_extrap_iters, sdf_, sdfv_, scur_, svcur_, clsS_);
  // smoothFluidSurface(5)
  launches_ += launch_smooth(st, G, c_.smooth_iters, sdf_, scur_);
  const double* fluid = sdf_[scur_];
  cudaEventRecord(ev_[2], st);
  // P2G + Dirichlet walls + extrapolation + gravity (fluid-simulator.cc:155-164)
  launches_ += launch_p2g<T>(st, G, h, start_, cnt_, P, p2g_scratch_at(p2g_scr_, G, rs_), G_(0), G_(1), G_(2),
                             (T*)gw_[0], (T*)gw_[1],
                             (T*)gw_[2], gv_[0][gcur_[0]], gv_[1][gcur_[1]], gv_[2][gcur_[2]],
                             c_.flip ? (T*)last_[0] : nullptr, c_.flip ? (T*)last_[1] : nullptr,
                             c_.flip ? (T*)last_[2] : nullptr);
  // Dirichlet walls, with the extrapolation tiles' classes
  {
    T* const gg[3] = {G_(0), G_(1), G_(2)};
    uint8_t* const ff[3] = {gv_[0][gcur_[0]], gv_[1][gcur_[1]], gv_[2][gcur_[2]]};
    launches_ += launch_dirichlet_tiles<T>(st, G, gg, ff, cls_[0]);
  }
  // extrapolate(.., 10) on the three face grids, temporally blocked
  {
    T* const fb[3][2] = {{(T*)g_[0][0], (T*)g_[0][1]}, {(T*)g_[1][0], (T*)g_[1][1]}, {(T*)g_[2][0], (T*)g_[2][1]}};
    launches_ += launch_extrap_faces<T>(st, G, c_.vel_extrap_iters, fb, gv_, nullptr, fsz_, gcur_, cls_);
  }
  k_force<T><<<nblk(fsz_[1]), kT, 0, st>>>(G, G_(1), gv_[1][gcur_[1]], c_.gravity * dt);
  launches_ += 1;
  cudaEventRecord(ev_[3], st);
  // buildSystem straight into the solver's tiled arrays (fluid-simulator.cc:166)
  SystemOut so;
  so.g = pcg_->geom();
  so.t_adiag = pcg_->adiag64();
  so.t_al = pcg_->al64();
  so.t_ad = pcg_->ad64();
  so.t_ab = pcg_->ab64();
  so.t_rhs = pcg_->rhs64();
  so.t_active = pcg_->active();
  int e = fvm_build_system<T>(st, nx, ny, nz, h, dt, G_(0), G_(1), G_(2), fluid, collider_, wt_[0],
                              wt_[1], wt_[2], so);
  if (e) return err("buildSystem");
  launches_ += 4;
  pcg_->mark_system_changed();
  cudaEventRecord(ev_[4], st);
  // solvePressure (fluid-simulator.cc:169)
  PcgStats ps;
  e = pcg_->solve(&ps);
  if (e) return e;
  launches_ += ps.kernel_launches;
  cudaEventRecord(ev_[5], st);
  // project + applyCollider + G2P (fluid-simulator.cc:175-180)
  const Tiled tg = pcg_->geom();
  e = fvm_project<T>(st, nx, ny, nz, h, dt, G_(0), G_(1), G_(2), pcg_->pressure64(), &tg, fluid,
                     wt_[0], wt_[1], wt_[2]);
  if (e) return err("project");
  launch_collider<T>(st, G, h, G_(0), G_(1), G_(2), collider_);
  // the particles are still in the order of this substep's sort
  if (n > 0)
    launch_g2p_tiles<T>(st, G, h, c_.flip ? c_.flip_alpha : -1.0, start_, cnt_, P, G_(0), G_(1), G_(2),
                        (T*)last_[0], (T*)last_[1], (T*)last_[2]);
  launches_ += 7;
  cudaEventRecord(ev_[6], st);
  cudaEventSynchronize(ev_[6]);
  if (stt) {
    float t[6];
    for (int k = 0; k < 6; k++) cudaEventElapsedTime(&t[k], ev_[k], ev_[k + 1]);
    stt->ms_advect += t[0];
    stt->ms_sort_sdf += t[1];
    stt->ms_p2g += t[2];
    stt->ms_build += t[3];
    stt->ms_solve += t[4];
    stt->ms_project_g2p += t[5];
    stt->ms_total += t[0] + t[1] + t[2] + t[3] + t[4] + t[5];
    stt->pcg_iterations = ps.iterations;
    stt->pcg_outer = ps.outer;
    stt->pcg_residual = ps.residual;
    stt->pcg_status = ps.status;
    stt->pcg_flags |= ps.device_flags;
    stt->substeps += 1;
    stt->kernel_launches += launches_ - l0;
  }
  return err("substep");
}

int FluidSim::substep(double dt, StepStats* st) {
  return c_.f32 ? substep_t<float>(dt, st) : substep_t<double>(dt, st);
}

// FluidSimulator::reconstruct (cpu/fluid-simulator.h:115-119): the surface of
// the particles as they are now into the current fluidSurface and sdfValid,
// sorted by cell first exactly as the substep sorts them (cell, then index), so
// later substeps see the same particle order.
template <class T>
int FluidSim::reconstruct_t(double radius) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  const double h = c_.h;
  const int64_t N = (int64_t)c_.nx * c_.ny * c_.nz;
  const int64_t n = n_;
  PartsT<T> P{(T*)px_, (T*)py_, (T*)pz_, (T*)vx_, (T*)vy_, (T*)vz_};
  PartsT<T> S{(T*)spx_, (T*)spy_, (T*)spz_, (T*)svx_, (T*)svy_, (T*)svz_};
  if (n > 0) {
    SortBufs sb{key_, cnt_, start_, cursor_, bsum_};
    launches_ += sort_particles<T>(st, n, G, h, P, id_, S, sid_, sb);
    std::swap(px_, spx_);
    std::swap(py_, spy_);
    std::swap(pz_, spz_);
    std::swap(vx_, svx_);
    std::swap(vy_, svy_);
    std::swap(vz_, svz_);
    std::swap(id_, sid_);
    P = PartsT<T>{(T*)px_, (T*)py_, (T*)pz_, (T*)vx_, (T*)vy_, (T*)vz_};
  } else {
    cudaMemsetAsync(cnt_, 0, sizeof(int) * N, st);
    cudaMemsetAsync(start_, 0, sizeof(int) * N, st);
  }
  if (launch_reconstruct<T>(st, G, h, radius, start_, cnt_, P.px, P.py, P.pz, sdf_[scur_], sdfv_[svcur_]))
    return ctx_->set_error(-1, "reconstruct: radius reaches past 6 cells");
  launches_ += 1;
  return err("reconstruct");
}

int FluidSim::reconstruct(double radius) {
  return c_.f32 ? reconstruct_t<float>(radius) : reconstruct_t<double>(radius);
}

// smoothFluidSurface (fluid-simulator.cc:39-74) on the simulator's surface
// buffers, flipping them once per pass as the substep does.
int FluidSim::smooth_fluid_surface(int iters) {
  cudaStream_t st = ctx_->stream;
  const Geo G{c_.nx, c_.ny, c_.nz};
  launches_ += launch_smooth(st, G, iters, sdf_, scur_);
  return err("smooth_fluid_surface");
}

int FluidSim::step(double frame_dt, StepStats* st) {  // fluid-simulator.cc:205-220
  double t = 0;
  while (t < frame_dt) {
    const double dt = std::min(cfl(), frame_dt - t);
    int e = substep(dt, st);
    if (e) return e;
    t += dt;
  }
  return 0;
}

int FluidSim::get_particles(double* pos, double* vel, bool device) {
  cudaStream_t st = ctx_->stream;
  const int64_t n = n_;
  if (n == 0) return 0;
  double* stage = nullptr;
  double *dp = pos, *dv = vel;
  if (!device) {
    if (cudaMallocAsync(&stage, sizeof(double) * 6 * (size_t)n, st) != cudaSuccess)
      return ctx_->set_error(-3, "staging allocation failed");
    dp = pos ? stage : nullptr;
    dv = vel ? stage + 3 * n : nullptr;
  }
  Parts p{px_, py_, pz_, vx_, vy_, vz_};
  if (c_.f32)
    k_soa_to_aos<float><<<nblk(n), kT, 0, st>>>(n, PartsT<float>::from(p), id_, dp, dv);
  else
    k_soa_to_aos<double><<<nblk(n), kT, 0, st>>>(n, PartsT<double>::from(p), id_, dp, dv);
  if (!device) {
    if (pos) cudaMemcpyAsync(pos, stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st);
    if (vel) cudaMemcpyAsync(vel, stage + 3 * n, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(stage, st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("get_particles");
  return err("get_particles");
}

int FluidSim::get_pressure(double* p, bool device) { return pcg_->download_pressure(p, device); }

int FluidSim::get_fluid_sdf(double* s, bool device) {
  const int64_t N = (int64_t)c_.nx * c_.ny * c_.nz;
  cudaMemcpyAsync(s, sdf_[scur_], sizeof(double) * N, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                  ctx_->stream);
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return err("get_fluid_sdf");
  return err("get_fluid_sdf");
}

// exportColliderSurface (cpu/fluid-simulator.h:191-193): the collider SDF; an
// empty collider is 1e9 everywhere, as manifold2SDF leaves it.
int FluidSim::get_collider_sdf(double* s, bool device) {
  const int64_t N = (int64_t)c_.nx * c_.ny * c_.nz;
  if (!collider_ && !device) {
    std::fill(s, s + N, 1e9);
    return 0;
  }
  std::vector<double> empty;
  if (collider_) {
    cudaMemcpyAsync(s, collider_, sizeof(double) * N, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                    ctx_->stream);
  } else {
    empty.assign((size_t)N, 1e9);
    cudaMemcpyAsync(s, empty.data(), sizeof(double) * N, cudaMemcpyHostToDevice, ctx_->stream);
  }
  if (cudaStreamSynchronize(ctx_->stream) != cudaSuccess) return err("get_collider_sdf");
  return err("get_collider_sdf");
}

int FluidSim::get_faces(double* u, double* v, double* w, bool device) {
  cudaStream_t st = ctx_->stream;
  double* outs[3] = {u, v, w};
  for (int a = 0; a < 3; a++) {
    if (!outs[a]) continue;
    if (!c_.f32) {
      cudaMemcpyAsync(outs[a], g_[a][gcur_[a]], sizeof(double) * fsz_[a],
                      device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
      continue;
    }
    double* dst = outs[a];
    double* stage = nullptr;
    if (!device) {
      if (cudaMallocAsync(&stage, sizeof(double) * fsz_[a], st) != cudaSuccess)
        return ctx_->set_error(-3, "staging allocation failed");
      dst = stage;
    }
    k_cast<float, double><<<nblk(fsz_[a]), kT, 0, st>>>(fsz_[a], (const float*)g_[a][gcur_[a]], dst);
    if (stage) {
      cudaMemcpyAsync(outs[a], stage, sizeof(double) * fsz_[a], cudaMemcpyDeviceToHost, st);
      cudaFreeAsync(stage, st);
    }
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return err("get_faces");
  return err("get_faces");
}

// =================================================================================
// Stage functions (device arrays, reference layout, AoS double particles).

namespace {
struct StageParticles {
  double* buf = nullptr;  // 6 SoA arrays
  int64_t* id = nullptr;
  cudaStream_t st;
  int64_t n;
  PartsT<double> P() const {
    return {buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, buf + 5 * n};
  }
  ~StageParticles() {
    if (buf) cudaFreeAsync(buf, st);
    if (id) cudaFreeAsync(id, st);
  }
};
}  // namespace

int flip_sample(cudaStream_t st, int64_t n, const double* pts, int nx, int ny, int nz, double h,
                const double* u, const double* v, const double* w, double* out) {
  // out = (sampleVelocity(p)) via the G2P kernel in PIC mode on a copy
  StageParticles sp;
  sp.st = st;
  sp.n = n;
  if (cudaMallocAsync(&sp.buf, sizeof(double) * 6 * (size_t)std::max<int64_t>(n, 1), st) != cudaSuccess) return -3;
  k_aos_to_soa<double><<<nblk(n), kT, 0, st>>>(n, pts, nullptr, sp.P(), nullptr);
  k_g2p<double><<<nblk(n), kT, 0, st>>>(n, sp.P(), u, v, w, nullptr, nullptr, nullptr, Geo{nx, ny, nz}, h,
                                        -1.0);
  k_soa_to_aos<double><<<nblk(n), kT, 0, st>>>(n, sp.P(), nullptr, nullptr, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int flip_advect(cudaStream_t st, int64_t n, double* pos, double* vel, int nx, int ny, int nz,
                double h, const double* u, const double* v, const double* w,
                const double* collider, double dt) {
  StageParticles sp;
  sp.st = st;
  sp.n = n;
  if (cudaMallocAsync(&sp.buf, sizeof(double) * 6 * (size_t)std::max<int64_t>(n, 1), st) != cudaSuccess) return -3;
  k_aos_to_soa<double><<<nblk(n), kT, 0, st>>>(n, pos, vel, sp.P(), nullptr);
  k_advect<double><<<nblk(n), kT, 0, st>>>(n, sp.P(), u, v, w, Geo{nx, ny, nz}, h, collider, dt);
  k_soa_to_aos<double><<<nblk(n), kT, 0, st>>>(n, sp.P(), nullptr, pos, vel);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

namespace {
// Sorted copy of AoS particles plus cell buckets, for the stage functions.
struct Sorted {
  StageParticles a, b;
  int *key = nullptr, *cnt = nullptr, *start = nullptr, *cursor = nullptr, *bsum = nullptr;
  cudaStream_t st;
  ~Sorted() {
    for (int* p : {key, cnt, start, cursor, bsum})
      if (p) cudaFreeAsync(p, st);
  }
};
int make_sorted(Sorted& s, cudaStream_t st, int64_t n, const double* pos, const double* vel,
                const Geo& G, double h) {
  const int64_t N = (int64_t)G.nx * G.ny * G.nz;
  const int64_t m = std::max<int64_t>(n, 1);
  s.st = st;
  s.a.st = s.b.st = st;
  s.a.n = s.b.n = n;
  if (cudaMallocAsync(&s.a.buf, sizeof(double) * 6 * m, st) != cudaSuccess ||
      cudaMallocAsync(&s.b.buf, sizeof(double) * 6 * m, st) != cudaSuccess ||
      cudaMallocAsync(&s.a.id, sizeof(int64_t) * m, st) != cudaSuccess ||
      cudaMallocAsync(&s.b.id, sizeof(int64_t) * m, st) != cudaSuccess ||
      cudaMallocAsync(&s.key, sizeof(int) * m, st) != cudaSuccess ||
      cudaMallocAsync(&s.cnt, sizeof(int) * N, st) != cudaSuccess ||
      cudaMallocAsync(&s.start, sizeof(int) * N, st) != cudaSuccess ||
      cudaMallocAsync(&s.cursor, sizeof(int) * N, st) != cudaSuccess ||
      cudaMallocAsync(&s.bsum, sizeof(int) * ((N + 1023) / 1024 + 1), st) != cudaSuccess)
    return -3;
  if (n == 0) {
    cudaMemsetAsync(s.cnt, 0, sizeof(int) * N, st);
    cudaMemsetAsync(s.start, 0, sizeof(int) * N, st);
    return 0;
  }
  k_aos_to_soa<double><<<nblk(n), kT, 0, st>>>(n, pos, vel, s.a.P(), s.a.id);
  SortBufs sb{s.key, s.cnt, s.start, s.cursor, s.bsum};
  sort_particles<double>(st, n, G, h, s.a.P(), s.a.id, s.b.P(), s.b.id, sb);
  return 0;
}
}  // namespace

int flip_p2g(cudaStream_t st, int64_t n, const double* pos, const double* vel, int nx, int ny,
             int nz, double h, double* u, double* v, double* w, double* uw, double* vw, double* ww,
             uint8_t* uvalid, uint8_t* vvalid, uint8_t* wvalid, double* ulast, double* vlast,
             double* wlast) {
  const Geo G{nx, ny, nz};
  Sorted s;
  int e = make_sorted(s, st, n, pos, vel, G, h);
  if (e) return e;
  const int64_t f0 = (int64_t)(nx + 1) * ny * nz, f1 = (int64_t)nx * (ny + 1) * nz,
                f2 = (int64_t)nx * ny * (nz + 1);
  cudaMemsetAsync(u, 0, sizeof(double) * f0, st);
  cudaMemsetAsync(v, 0, sizeof(double) * f1, st);
  cudaMemsetAsync(w, 0, sizeof(double) * f2, st);
  cudaMemsetAsync(uw, 0, sizeof(double) * f0, st);
  cudaMemsetAsync(vw, 0, sizeof(double) * f1, st);
  cudaMemsetAsync(ww, 0, sizeof(double) * f2, st);
  void* scr = nullptr;
  if (cudaMallocAsync(&scr, p2g_scratch_bytes(G, sizeof(double)), st) != cudaSuccess) return -3;
  launch_p2g<double>(st, G, h, s.start, s.cnt, s.b.P(), p2g_scratch_at(scr, G, sizeof(double)), u, v, w, uw, vw,
                     ww, uvalid, vvalid, wvalid, ulast, vlast, wlast);
  cudaFreeAsync(scr, st);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// solveG2P through the simulator's tile kernel: the particles are sorted by
// cell first, and each velocity is written back at its particle's index.
int flip_g2p(cudaStream_t st, int64_t n, const double* pos, double* vel, int nx, int ny, int nz,
             double h, const double* u, const double* v, const double* w, const double* ulast,
             const double* vlast, const double* wlast, double alpha) {
  const Geo G{nx, ny, nz};
  Sorted s;
  int e = make_sorted(s, st, n, pos, vel, G, h);
  if (e) return e;
  if (n > 0) {
    launch_g2p_tiles<double>(st, G, h, alpha, s.start, s.cnt, s.b.P(), u, v, w, ulast, vlast, wlast);
    k_soa_to_aos<double><<<nblk(n), kT, 0, st>>>(n, s.b.P(), s.b.id, nullptr, vel);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int flip_reconstruct(cudaStream_t st, int64_t n, const double* pos, int nx, int ny, int nz,
                     double h, double radius, double* sdf, uint8_t* valid) {
  const Geo G{nx, ny, nz};
  Sorted s;
  int e = make_sorted(s, st, n, pos, nullptr, G, h);
  if (e) return e;
  PartsT<double> P = s.b.P();
  if (launch_reconstruct<double>(st, G, h, radius, s.start, s.cnt, P.px, P.py, P.pz, sdf, valid)) return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace sc
