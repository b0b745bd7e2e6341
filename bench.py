"""Benchmark: SimCraft FluidSim pressure solve on B200.

Workload (N=1): standalone pressure solve on a 128^3 grid (fluid = seeded union
of 24 spheres at 50% fill, empty collider, solid walls, dt/h = 32/120), MIC(0)
preconditioned CG to 1e-8 relative residual; the mixed FP32-inner / FP64
defect-correction solve is the headline `value`, the plain FP64 solve is
reported beside it.  A step is one complete CgSolver3D::solve call: system
upload into the solver's layout, MIC(0) pivots, PCG iterations, pressure
download.  Multi-GPU runs are independent replicas (the MIC(0) sweep is one
global wavefront and does not shard).

A second leg times the FLIP step at scale: the 256^3 dam break (block x<0.5,
y<0.5, 8 jittered particles per cell = 33.5M particles, FP32 particles and
grids, CFL factor 1, FLIP blend 0.95, mixed MIC(0)-PCG to 1e-8 relative
residual), reported as FLIP substeps/s with the per-subsystem split.

A third leg times the differentiable step on the 64^3 control problem (fluid
y < 0.25, 524,288 particles, 20 substeps of dt = 1/120, checkpoints every 5):
forward and adjoint in FP32, and the FP64 adjoint against central finite
differences along 16 seeded directions.

`--impl reference` times the reference's own CgSolver3D::solve (its FluidSim
CPU sources compiled into oracle/_ref, oneTBB loops on OpenMP threads) on the
same system, for the iteration count that reaches the same tolerance.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per pressure solve to 1e-8 rel. residual (mixed vs FP64 PCG); FLIP steps/s"
N_GRID = 128
TOL = 1e-8
DT_OVER_H = 32.0 / 120.0
FLIP_N = 256
FRAME_DT = 1.0 / 120.0
DIFF_N = 64
DIFF_STEPS = 20
LARGE_N = 512
COLLIDER_N = 256


def build_scene(n, device=None):
    """Sphere-pool fluid: 24 seeded spheres at 50% fill (seed 2); the 512^3
    large-solve scene uses 60% fill (seed 9).  `device` evaluates the SDF there."""
    from simcraft_b200 import scenes

    fill, seed = (0.6, 9) if n >= 512 else (0.5, 2)
    sdf, info = scenes.sphere_pool(n, count=24, rmin=0.05, rmax=0.2, fill=fill, seed=seed, device=device)
    return np.ascontiguousarray(sdf), info


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic(key, n):
    """Per-launch DRAM traffic of a sweep at n^3 as measured by ncu
    (profiles/dram_traffic.json, written from the captures), or None."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
    except (OSError, ValueError):
        return None
    return float(d[key]) if d.get("grid") == n and key in d else None


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0}, "fallback"


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.build()
    return O


def reference_iterations(sysm, rhs, threads):
    """Iterations the reference's CG needs to reach TOL relative L2 residual on
    this system: the CPU restatement (equal to the reference bit for bit,
    tests/test_ref_pin_cpu.py) stops on that test; the reference's own solver
    only has its absolute L-inf test."""
    O = _oracle()
    O.set_threads(threads)
    O.set_parity_mode(False)
    _, _, it = O.pcg_solve(sysm["adiag"], sysm["an"], rhs, sysm["active"], tol=TOL, max_iter=5000,
                           criterion=O.CRIT_REL_L2)
    return it


def cpu_solve_ms(sysm, rhs, threads, iters):
    """One CgSolver3D::solve of the reference's own code (oracle/_ref timing
    build, oneTBB loops on `threads` OpenMP threads, serial MIC(0) and dot
    products as in the reference), run for `iters` iterations (tolerance 0,
    max_iterations = iters + 1).  Returns (ms, iterations, pressure, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref as R

    if R.available():
        st = {}
        pg, _ = R.cg_solve(sysm["adiag"], sysm["an"], rhs, sysm["active"], tol=0.0, max_iter=iters + 1,
                           parallel=True, threads=threads, stats=st)
        return st["ms"], st["iterations"], pg, "reference"
    # no reference library: the CPU restatement stands in (the "port")
    O = _oracle()
    O.set_threads(threads)
    O.set_parity_mode(False)
    t = time.perf_counter()
    pg, _, it = O.pcg_solve(sysm["adiag"], sysm["an"], rhs, sysm["active"], tol=0.0, max_iter=iters + 1,
                            criterion=O.CRIT_ABS_LINF)
    return (time.perf_counter() - t) * 1e3, it, pg, "port"


def solve_config(n, info, n_active, world):
    """The `config` of the headline workload, the same in both arms."""
    return {"workload": f"standalone pressure solve {n}^3 to {TOL:g} relative residual (sphere pool)",
            "grid": [n, n, n], "fill": info["fill"], "active_cells": n_active, "dt_over_h": DT_OVER_H,
            "tolerance": TOL, "criterion": "relative L2",
            "cache": "inputs larger than L2 (solver working set ~300 MB at 128^3)",
            "parallelism": f"replicas x{world}"}


def reference_arm(args, rank):
    """The reference's own CgSolver3D::solve (FluidSim/src/cpu/project-solver.cc:308-346,
    compiled into oracle/_ref) on the host cores, on the headline system, for
    the iteration count that reaches the headline tolerance."""
    if rank != 0:
        return
    O = _oracle()
    from simcraft_b200 import scenes

    threads = os.cpu_count() or 1
    n = args.solve_n
    sdf, info = build_scene(n)
    h = 1.0 / n
    z = np.zeros
    S = O.build_system((n, n, n), h, DT_OVER_H * h, z((n + 1, n, n)), z((n, n + 1, n)), z((n, n, n + 1)), sdf)
    rhs, _ = scenes.poisson_rhs(S["active"], sdf, seed=3)
    rhs = np.ascontiguousarray(rhs)
    iters = reference_iterations(S, rhs, threads)
    times = []
    kind, it = "port", iters
    for i in range(args.warmup + args.steps):
        ms, it, _, kind = cpu_solve_ms(S, rhs, threads, iters)
        if i >= args.warmup:
            times.append(ms)
    v = float(np.mean(times))
    what = ("the reference's own CgSolver3D::solve (oracle/_ref: FluidSim/src/cpu sources, oneTBB loops on "
            "OpenMP threads, serial MIC(0) and dot products)" if kind == "reference"
            else "the CPU restatement of CgSolver3D::solve (the reference library is absent)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms/solve", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sphere pool, no dataset)",
        "config": solve_config(n, info, int(S["active"].sum()), args.gpus),
        "solver": f"FP64 MIC(0)-PCG, {what}, {it} iterations",
        "cpu_baseline": {"value": v, "unit": "ms/solve", "cores": threads, "kind": kind,
                         "sample": f"one full FP64 solve of the {n}^3 system per step: {it} iterations, the count "
                                   f"at which the reference's recursion first has a relative L2 residual below "
                                   f"{TOL:g} (its own stopping test is absolute L-inf)"},
        "e2e": {"value": v, "unit": "ms/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def build_system_device(n, sdf, dev, ctx):
    """The standalone pressure system of an n^3 scene on the GPU
    (FvmSolver3D::buildSystem with zero velocity and the empty collider) and its
    seeded right-hand side: (Adiag, Aneighbour[6], active, active on the host,
    rhs on the host, rhs info)."""
    import torch

    from simcraft_b200 import _capi, scenes

    L = _capi.lib()
    h = 1.0 / n
    dt = DT_OVER_H * h
    f64 = dict(dtype=torch.float64, device=dev)
    sdf_d = torch.from_numpy(sdf).to(dev)
    u = torch.zeros((n + 1, n, n), **f64)
    v = torch.zeros((n, n + 1, n), **f64)
    w = torch.zeros((n, n, n + 1), **f64)
    adiag = torch.zeros((n, n, n), **f64)
    an = [torch.zeros((n, n, n), **f64) for _ in range(6)]
    rhs_b = torch.zeros((n, n, n), **f64)
    active = torch.zeros((n, n, n), dtype=torch.uint8, device=dev)
    uw, vw, ww = torch.zeros_like(u), torch.zeros_like(v), torch.zeros_like(w)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    ctx.set_stream(ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    rc = L.sc_fvm_build_system_device(ctx.handle, n, n, n, h, dt, _capi.SC_REAL_F64, ptr(u), ptr(v), ptr(w),
                                      ptr(sdf_d), None, ptr(adiag), _capi.ptr_array([ptr(a) for a in an]),
                                      ptr(rhs_b), ptr(active), ptr(uw), ptr(vw), ptr(ww))
    _capi.check("sc_fvm_build_system_device", rc, ctx.handle)
    ctx.use_own_stream()
    torch.cuda.synchronize()
    del u, v, w, uw, vw, ww, rhs_b, sdf_d
    act_h = active.cpu().numpy()
    rhs_h, rinfo = scenes.poisson_rhs(act_h, sdf, seed=3)
    return adiag, an, active, act_h, np.ascontiguousarray(rhs_h), rinfo


def tolerance_sweep(n, ctx, adiag, an, rhs_d, active, act_h):
    """The standalone system at the tolerances 1e-6, 1e-8 and 1e-10 (relative
    L2), FP64 against mixed: ms per solve (best of 2 after a warm-up, solver
    events), iterations, and each solution's relative L2 error over the active
    cells against an FP64 MIC(0)-PCG solve to 1e-12."""
    import torch

    from simcraft_b200 import _capi
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_FP64, PREC_MIXED

    L = _capi.lib()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    an_dev = _capi.ptr_array([ptr(a) for a in an])
    mask = torch.from_numpy(act_h.astype(bool)).to(rhs_d.device)

    def solve(s, out):
        st = _capi.sc_pcg_stats()
        rc = L.sc_pcg_solve_device(s.handle, ptr(adiag), an_dev, ptr(rhs_d), ptr(active), ptr(out),
                                   ctypes.byref(st))
        _capi.check("sc_pcg_solve_device", rc, ctx.handle)
        return st

    ref = torch.zeros((n, n, n), dtype=torch.float64, device=rhs_d.device)
    solve(CgSolver3D(n, n, n, context=ctx, tol=1e-12, max_iter=10000, criterion=CRIT_REL_L2, precision=PREC_FP64),
          ref)
    ref_norm = float(ref[mask].norm())
    pg = torch.zeros_like(ref)
    rows = []
    for tol in (1e-6, 1e-8, 1e-10):
        row = {"tolerance": tol}
        for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
            s = CgSolver3D(n, n, n, context=ctx, tol=tol, max_iter=10000, criterion=CRIT_REL_L2, precision=prec)
            sts = [solve(s, pg) for _ in range(3)]
            st = sts[-1]
            row[name] = {"ms_per_solve": min(x.ms for x in sts[1:]), "iterations": st.iterations,
                         "true_rel_l2": st.true_rel_l2,
                         "error_vs_fp64_1e-12": float((pg - ref)[mask].norm()) / ref_norm}
            del s
        rows.append(row)
    return {"reference": "FP64 MIC(0)-PCG to 1e-12 relative residual on the GPU", "rows": rows}


def large_solve_leg(args, dev, ctx, replicas, cpu=False):
    """FP64 against mixed on the 512^3 sphere pool (60% fill, seed 9), both to
    1e-8 relative residual, device-resident inputs; `--large-steps` timed solves
    after `--large-warmup` untimed ones, CUDA events on the solver stream."""
    import torch

    from simcraft_b200 import _capi
    from simcraft_b200.solver import CgSolver3D, CRIT_REL_L2, PREC_FP64, PREC_MIXED

    L = _capi.lib()
    n = LARGE_N
    sdf, info = build_scene(n, device=dev)
    adiag, an, active, act_h, rhs_h, _ = build_system_device(n, sdf, dev, ctx)
    del sdf
    rhs_d = torch.from_numpy(rhs_h).to(dev)
    pg = torch.zeros((n, n, n), dtype=torch.float64, device=dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    an_dev = _capi.ptr_array([ptr(a) for a in an])
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {"workload": f"standalone pressure solve {n}^3, sphere pool fill {info['fill']:.3f}, "
                       f"dt/h {DT_OVER_H:.4f}, to {TOL:g} rel. residual",
           "active_cells": int(act_h.sum()), "warmup": args.large_warmup, "steps": args.large_steps}
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        s = CgSolver3D(n, n, n, context=ctx, tol=TOL, max_iter=5000, criterion=CRIT_REL_L2, precision=prec)

        def solve():
            st = _capi.sc_pcg_stats()
            rc = L.sc_pcg_solve_device(s.handle, ptr(adiag), an_dev, ptr(rhs_d), ptr(active), ptr(pg),
                                       ctypes.byref(st))
            _capi.check("sc_pcg_solve_device", rc, ctx.handle)
            return st

        for _ in range(args.large_warmup):
            solve()
        torch.cuda.synchronize()
        replicas.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.large_steps):
            st = solve()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = replicas.max(e0.elapsed_time(e1)) / max(1, args.large_steps)
        out[name] = {"ms_per_solve": ms, "iterations": st.iterations, "iterations_per_s": st.iterations / (ms * 1e-3),
                     "outer": st.outer, "true_rel_l2": st.true_rel_l2, "kernel_launches": st.kernel_launches}
        # per-kernel device times on this system (sc_pcg_time_kernels) and the
        # algorithmic bandwidth of each: FP64 SpMV N(6s+1), axpy N(6s), scale-add
        # N(3s), sweeps N(6s+1) / N(7s+1); FP32 Eisenstat sweeps N*8*4 / N*9*4
        kt = (ctypes.c_double * 8)()
        _capi.check("sc_pcg_time_kernels", L.sc_pcg_time_kernels(s.handle, 5, kt), ctx.handle)
        km = list(kt)
        N = n * n * n
        gbs = lambda b, t: b / (t * 1e-3) / 1e9 if t > 0 else None
        if name == "fp64":
            out[name]["kernel_ms"] = {"forward_sweep": km[1], "backward_sweep": km[2], "spmv": km[3], "axpy": km[4],
                                      "scale_add": km[5]}
            out[name]["kernel_gbs"] = {"forward_sweep": gbs(N * 49, km[1]), "backward_sweep": gbs(N * 57, km[2]),
                                       "spmv": gbs(N * 49, km[3]), "axpy": gbs(N * 48, km[4]),
                                       "scale_add": gbs(N * 24, km[5])}
        else:
            out[name]["kernel_ms"] = {"eisenstat_backward_sweep": km[6], "eisenstat_forward_sweep": km[7], "axpy": km[4]}
            out[name]["kernel_gbs"] = {"eisenstat_backward_sweep": gbs(N * 32, km[6]),
                                       "eisenstat_forward_sweep": gbs(N * 36, km[7]), "axpy": gbs(N * 24, km[4])}
        if name == "fp64":
            pg64 = pg.clone()
        else:
            m = torch.from_numpy(act_h.astype(bool)).to(dev)
            out[name]["rel_l2_vs_fp64_solution"] = float((pg - pg64)[m].norm() / pg64[m].norm())
            del m, pg64
        del s
        torch.cuda.empty_cache()
    out["fp64_over_mixed"] = out["fp64"]["ms_per_solve"] / out["mixed"]["ms_per_solve"]
    if cpu:
        # the reference's own CgSolver3D on the host cores: a capped run of a few
        # iterations, its per-iteration time extrapolated to the FP64 count
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref as R

        if R.available():
            threads = os.cpu_count() or 1
            host = {"adiag": adiag.cpu().numpy(), "an": [a.cpu().numpy() for a in an], "active": act_h}
            capped = 3
            st = {}
            R.cg_solve(host["adiag"], host["an"], rhs_h, host["active"], tol=0.0, max_iter=capped + 1,
                       parallel=True, threads=threads, stats=st)
            # one preconditioner application precedes the loop: capped + 1 applications
            per_iter = st["ms"] / (capped + 1)
            iters = out["fp64"]["iterations"]
            out["cpu_baseline"] = {"value": per_iter * iters, "unit": "ms/solve", "cores": threads,
                                   "kind": "reference", "extrapolated": True,
                                   "ms_per_iteration": per_iter,
                                   "sample": f"the reference's CgSolver3D::solve on the same {n}^3 system, "
                                             f"capped at {capped} iterations ({st['ms']:.0f} ms); the total is "
                                             f"that per-iteration time x the FP64 solve's {iters} iterations "
                                             f"(extrapolated)"}
            del host
    del adiag, an, active, rhs_d, pg
    torch.cuda.empty_cache()
    return out


def flip32_leg(args, ctx, cpu):
    """The 32^3 FP64 dam break of the parity runs (block x<0.5, y<0.5, 8 particles
    per cell, FLIP 0.95, MIC(0)-PCG to 1e-6 relative, at most 200 iterations):
    frames/s on the GPU, wall clock around 10 frames of dt = 1/120 from the
    initial state (host round trips included; a separate simulator warms up
    first), and the CPU oracle (all host threads) on the same 10 frames, with
    pressure and positions compared after the last one."""
    import torch

    from simcraft_b200 import scenes
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2

    n, frames = 32, 10
    pos, vel, h = scenes.dam_break(n, seed=1)
    kw = dict(context=ctx, flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200, pcg_criterion=CRIT_REL_L2)
    warm = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), **kw)
    warm.set_initial_fluid(pos, vel)
    for _ in range(3):
        warm.step(FRAME_DT)
    del warm
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), **kw)
    sim.set_initial_fluid(pos, vel)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(frames):
        st = sim.step(FRAME_DT)
    torch.cuda.synchronize()
    gpu_ms = (time.perf_counter() - t0) * 1e3 / frames
    out = {"workload": "FLIP dam break 32^3 FP64, 65,536 particles, FLIP 0.95, PCG to 1e-6 relative (max 200)",
           "frames": frames, "ms_per_frame": gpu_ms, "frames_per_s": 1e3 / gpu_ms,
           "device_ms_last_frame": st["ms_total"], "pcg_iterations_last_frame": st["pcg_iterations"]}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        O.build()
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        O.set_parity_mode(False)
        ref = O.Sim(**O.default_config(n, n, n, h, flip_alpha=0.95, pcg_tol=1e-6, pcg_max_iter=200,
                                       pcg_criterion=CRIT_REL_L2))
        ref.set_particles(pos, vel)
        t0 = time.perf_counter()
        for _ in range(frames):
            ref.step(FRAME_DT)
        cpu_ms = (time.perf_counter() - t0) * 1e3 / frames
        p_ref, p = ref.pressure(), sim.pressure()
        x_ref, _ = ref.particles()
        x, _ = sim.particles()
        out["cpu_baseline"] = {"value": cpu_ms, "unit": "ms/frame", "cores": threads, "kind": "port",
                               "sample": f"the same {frames} frames (CPU oracle, OpenMP transfers)",
                               "pressure_rel_l2_vs_gpu": float(np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref)),
                               "positions_max_err_over_h": float(np.abs(x - x_ref).max() / h)}
    return out


def collider_leg(args, dev, ctx, cpu):
    """setCollider(mesh): manifold2SDF of a closed 20,480-triangle sphere (icosphere
    subdivided 5 times, radius 0.3) on the GPU at 128^3 and 256^3 (device-resident
    mesh, CUDA events on torch's stream around the call), and the CPU oracle
    (sequential, as the reference) on the 128^3 grid."""
    import torch

    from simcraft_b200 import scenes
    from simcraft_b200.mesh import manifold_to_sdf

    v, t = scenes.icosphere(5, 0.3)
    vd, td = torch.from_numpy(v).to(dev), torch.from_numpy(t).to(dev)
    out = {"workload": f"closed sphere mesh, {len(t)} triangles, exact band 3, reference distance arithmetic",
           "triangles": len(t)}
    stream = torch.cuda.current_stream(dev)
    for n in (128, args.collider_n):
        for _ in range(2):
            manifold_to_sdf(vd, td, (n, n, n), 1.0 / n, context=ctx)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record(stream)
        for _ in range(reps):
            sdf = manifold_to_sdf(vd, td, (n, n, n), 1.0 / n, context=ctx)
        e1.record(stream)
        torch.cuda.synchronize()
        out[f"gpu_ms_{n}"] = e0.elapsed_time(e1) / reps
        if n == 128:
            sdf128 = sdf.cpu().numpy()
        del sdf
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        O.build()
        t0 = time.perf_counter()
        ref, _, _ = O.manifold_to_sdf(v, t, (128, 128, 128), 1.0 / 128)
        out["cpu_baseline"] = {"value": 1e3 * (time.perf_counter() - t0), "unit": "ms", "cores": 1, "kind": "port",
                               "sample": "the same mesh on the 128^3 grid (the reference's sequential algorithm)",
                               "bit_exact_vs_gpu": bool(np.array_equal(ref, sdf128))}
    return out


def surface_leg(dev, ctx, sim, h, cpu):
    """rebuildSurface(mesh, exportFluidSurface()) of the FLIP dam break after its
    timed substeps, as the reference's app exports the fluid: the device call a
    user makes (count + fill, CUDA events on torch's stream), the same from host
    arrays (end to end), and one pass of the CPU oracle (sequential with a hash
    map, as the reference) on the same SDF, checked bit for bit."""
    import torch

    from simcraft_b200.surface import rebuild_surface

    sdf_h = sim.export_fluid_surface()
    n = sdf_h.shape[0]
    sdf_d = torch.from_numpy(sdf_h).to(dev)
    for _ in range(3):
        V, N, I = rebuild_surface(sdf_d, h, context=ctx)
    stream = torch.cuda.current_stream(dev)
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        V, N, I = rebuild_surface(sdf_d, h, context=ctx)
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_ms = e0.elapsed_time(e1) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        Vh, Nh, Ih = rebuild_surface(sdf_h, h, context=ctx)
    e2e_ms = 1e3 * (time.perf_counter() - t0) / reps
    nv, ni = V.shape[0], I.shape[0]
    alg = 8 * sdf_h.size + 48 * nv + 4 * ni
    out = {"workload": f"marching cubes of the {n}^3 dam-break fluid SDF after the timed substeps "
                       f"(FP64 mesh, reference vertex order)",
           "vertices": int(nv), "triangles": int(ni // 3), "gpu_ms": gpu_ms, "e2e_ms": e2e_ms,
           "algorithmic_bytes": int(alg), "algorithmic_gb_s": alg / (gpu_ms * 1e-3) / 1e9,
           "kernel_launches_per_call": 6,
           "host_equals_device": bool(np.array_equal(Vh, V.cpu().numpy()) and np.array_equal(Ih, I.cpu().numpy()))}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        O.build()
        t0 = time.perf_counter()
        Vr, Nr, Ir = O.rebuild_surface(sdf_h, h, counts=(nv, ni))
        out["cpu_baseline"] = {"value": 1e3 * (time.perf_counter() - t0), "unit": "ms", "cores": 1, "kind": "port",
                               "sample": f"one pass over the same {n}^3 SDF (the reference's sequential algorithm)",
                               "bit_exact_vs_gpu": bool(np.array_equal(Vr, Vh) and np.array_equal(Ir, Ih) and
                                                        np.array_equal(Nr, Nh, equal_nan=True))}
    return out


def flip_run(args, dev, ctx, dist, rank, world, steps, tau):
    """`steps` FLIP substeps timed after args.warmup untimed ones on the 256^3
    FP32 dam break (device-resident particles), MIC(0) tau = `tau`; returns
    the result dict and the simulator."""
    import torch

    from simcraft_b200 import scenes
    from simcraft_b200.fluid import FluidSimulator
    from simcraft_b200.solver import CRIT_REL_L2, PREC_MIXED

    n = args.flip_n
    pos, vel, h = scenes.dam_break(n, seed=4)
    sim = FluidSimulator(len(pos), (1.0, 1.0, 1.0), (n, n, n), context=ctx, precision="f32",
                         flip_alpha=0.95, cfl_factor=1.0, pcg_tol=TOL, pcg_max_iter=5000,
                         pcg_criterion=CRIT_REL_L2, pcg_precision=PREC_MIXED, pcg_mic_tau=tau)
    sim.set_initial_fluid(pos, vel)
    n_particles = len(pos)
    del pos, vel

    def one():
        # the reference's frame loop (fluid-simulator.cc:205-220): dt = min(CFL, frame)
        return sim.substep(min(sim.cfl(), FRAME_DT))

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    split = {}
    iters = []
    launches = 0
    unconverged, flags = 0, 0
    e0.record(stream)
    for _ in range(steps):
        st = one()
        for k, v in st.items():
            if k.startswith("ms_"):
                split[k[3:]] = split.get(k[3:], 0.0) + v
        iters.append(st["pcg_iterations"])
        launches += st["kernel_launches"]
        unconverged += st["pcg_status"] != 1
        flags |= st["pcg_flags"]
    e1.record(stream)
    torch.cuda.synchronize()
    from simcraft_b200.replicas import Replicas

    ms = Replicas(rank, world, dist, dev).max(e0.elapsed_time(e1))
    K = steps
    out = {"workload": f"FLIP dam break {n}^3, block x<0.5 y<0.5, 8 particles/cell, FP32 particles and grids, "
                       f"CFL factor 1, FLIP 0.95, mixed MIC(0)-PCG (tau {tau:g}, sigma 0.25) to {TOL:g}",
           "particles": n_particles, "steps": K, "warmup": args.warmup,
           "steps_per_s": world * K / (ms * 1e-3), "ms_per_step": ms / K,
           "split_ms_per_step": {k: v / K for k, v in split.items()},
           "pcg_inner_iterations_mean": float(np.mean(iters)), "gpu_launches": int(launches),
           "pcg_solves_not_converged": int(unconverged), "pcg_device_flags": int(flags)}
    return out, sim, h


def flip_leg(args, dev, ctx, dist, rank, world):
    """FLIP substeps/s on the 256^3 FP32 dam break with the reference's MIC(0)
    constants, and the configuration's 100 substeps with tau = 0."""
    import torch

    K = args.flip_steps
    out, sim, h = flip_run(args, dev, ctx, dist, rank, world, K, 0.97)
    out["steps_note"] = (
        f"{K} substeps timed after {args.warmup} warm-up ones (substeps {args.warmup}-{args.warmup + K - 1} from the "
        f"initial block). The configuration's 100 substeps are not reachable with the reference's MIC(0) constants "
        f"(tau 0.97, sigma 0.25): on this scene the preconditioner stalls from substep ~15 (5000 iterations short of "
        f"the tolerance, FP64 and mixed alike; its tau terms divide by E^2) and by substep ~18 the unprojected "
        f"velocities make the system non-finite. flip_100 is the same run over 100 substeps with tau = 0 (IC(0), "
        f"the same preconditioner code)")
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = flip_cpu_sample(sim, sim.dims[0], h)
    if args.surface:
        out["surface"] = surface_leg(dev, ctx, sim, h, rank == 0 and world == 1 and not args.no_cpu)
    del sim
    torch.cuda.empty_cache()
    if args.flip100 > 0:
        o100, sim, _ = flip_run(args, dev, ctx, dist, rank, world, args.flip100, 0.0)
        o100["steps_note"] = (f"the configuration's {args.flip100} substeps, timed after {args.warmup} warm-up "
                              f"ones, with MIC(0) tau = 0 (IC(0)): every solve reaches the tolerance")
        out["flip_100"] = o100
        del sim
        torch.cuda.empty_cache()
    return out


def diff_leg(args, ctx, replicas):
    """Differentiable step on the 64^3 control problem: FP32 forward + adjoint
    times (CUDA events around each call on the solver's stream), and the FP64
    adjoint against central differences (eps 1e-3) along seeded directions."""
    import torch

    from simcraft_b200.diff import DiffFlip, control_scene, faces_from_cells
    from simcraft_b200.replicas import fd_check

    n, steps = args.diff_n, DIFF_STEPS
    pos, param, target, h = control_scene(n)
    U = faces_from_cells(torch.from_numpy(param).cuda())
    out = {"workload": f"differentiable FLIP control {n}^3, fluid y<0.25, {len(pos)} particles, "
                       f"{steps} substeps dt=1/120, checkpoints every 5, FLIP 0.95, PCG tau=0 to 1e-10",
           "particles": len(pos), "steps": steps}
    sims = {}
    for prec in ("f32", "f64"):
        sim = DiffFlip((n, n, n), h, FRAME_DT, steps, context=ctx, precision=prec, checkpoint_every=5,
                       flip_alpha=0.95)
        sim.set_particles(pos)
        sim.set_target(target)
        sims[prec] = sim
    s32 = sims["f32"]
    for _ in range(2):
        s32.forward(U)
        s32.backward()
    fw, bw = [], []
    for _ in range(max(1, args.steps)):
        t = time.perf_counter()
        loss = s32.forward(U)
        fw.append(time.perf_counter() - t)
        t = time.perf_counter()
        g32 = s32.backward()
        bw.append(time.perf_counter() - t)
    out.update({"loss": loss, "forward_ms": 1e3 * float(np.median(fw)), "backward_ms": 1e3 * float(np.median(bw)),
                "precision": "f32 particles and grids, f64 pressure solves"})
    s64 = sims["f64"]
    s64.forward(U, tape="record")
    g64 = s64.backward()
    eps = 1e-3

    def loss_at(d, sign):
        D = faces_from_cells(torch.from_numpy(d).cuda())
        return s64.forward([u + sign * eps * x for u, x in zip(U, D)], tape="replay")

    def grad_dot(d):
        D = faces_from_cells(torch.from_numpy(d).cuda())
        return sum(float((g * x).sum()) for g, x in zip(g64, D))

    # the directions are split round-robin over the replicas and gathered
    errs = fd_check(loss_at, grad_dot, param.shape, args.diff_dirs, 8, eps, replicas)
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(g64, g32))
    den = sum(float((a ** 2).sum()) for a in g64)
    out.update({"fd_directions": args.diff_dirs, "fd_eps": eps, "fd_ranks": replicas.world,
                "fd_max_rel_err": max(errs) if errs else None,
                "fd_median_rel_err": float(np.median(errs)) if errs else None,
                "f32_vs_f64_grad_rel_l2": (num / den) ** 0.5,
                "cpu_baseline": {"value": None, "kind": "none",
                                 "note": "the reference has no differentiable step: there is no CPU adjoint to "
                                         "time (the FP64 reference gradient of the tests is central differences "
                                         "of the oracle's forward, tests/test_diff_gpu.py)"}})
    del sims, s32, s64
    torch.cuda.empty_cache()
    return out


def flip_cpu_sample(sim, n, h):
    """CPU oracle on a bounded sample of the same 256^3 state: advect + P2G + G2P
    of the first 1M particles scaled to all particles, plus the FP64 PCG's cost
    per iteration on the current 256^3 system times the iterations the GPU
    solve took.  Reconstruction, extrapolation, buildSystem and project are
    left out, so the CPU figure is a lower bound of the CPU substep."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    O.set_parity_mode(False)
    pos, vel = sim.particles()
    u, v, w = sim.faces()
    P = len(pos)
    m = min(P, 1 << 20)
    ps, vs = np.ascontiguousarray(pos[:m]), np.ascontiguousarray(vel[:m])
    dims = (n, n, n)
    t = time.perf_counter()
    O.advect(ps, vs, dims, h, u, v, w, None, FRAME_DT)
    O.g2p(ps, vs, dims, h, u, v, w, u, v, w, alpha=0.95)
    # the threaded P2G keeps one full set of face grids per thread: cap its threads
    O.set_threads(min(threads, 8))
    O.p2g(ps, vs, dims, h, flip=True)
    O.set_threads(threads)
    t_part = (time.perf_counter() - t) * P / m
    # PCG cost per iteration at full size on a system of the same shape
    sdf = sim.export_fluid_surface()
    S = O.build_system(dims, h, FRAME_DT, u, v, w, sdf)
    its = 10
    t = time.perf_counter()
    _, _, done = O.pcg_solve(S["adiag"], S["an"], S["rhs"], S["active"], tol=0.0, max_iter=its + 1,
                             criterion=O.CRIT_REL_L2)
    per_it = (time.perf_counter() - t) / max(done, 1)
    gpu_its = sim.last_stats["pcg_iterations"] if sim.last_stats else 0
    total = t_part + per_it * gpu_its
    return {"value": 1.0 / total, "unit": "FLIP substeps/s", "cores": threads, "kind": "port",
            "sample": f"advect+G2P ({threads} threads) and P2G ({min(threads, 8)} threads) on {m} of {P} "
                      f"particles scaled to all, plus FP64 PCG "
                      f"{per_it * 1e3:.1f} ms/iteration x {gpu_its} iterations at {n}^3; "
                      "other stages omitted (lower bound of the CPU substep)",
            "ms_per_step": total * 1e3}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--flip-steps", type=int, default=10, help="timed FLIP substeps (0 skips the FLIP leg)")
    ap.add_argument("--flip-n", type=int, default=FLIP_N, help="FLIP dam-break grid size (profiling runs)")
    ap.add_argument("--flip100", type=int, default=100,
                    help="substeps of the tau = 0 FLIP run (the configuration's 100; 0 skips it)")
    ap.add_argument("--skip-solve", action="store_true",
                    help="run only the FLIP leg (profiling runs; prints the FLIP object)")
    ap.add_argument("--solve-n", type=int, default=N_GRID, help="standalone solve grid size")
    ap.add_argument("--large-steps", type=int, default=1,
                    help="timed solves of the 512^3 FP64-vs-mixed leg (0 skips the leg)")
    ap.add_argument("--large-warmup", type=int, default=2, help="untimed solves of the 512^3 leg")
    ap.add_argument("--collider", type=int, default=1, help="mesh-to-SDF collider leg (0 skips)")
    ap.add_argument("--collider-n", type=int, default=COLLIDER_N, help="the collider leg's larger grid")
    ap.add_argument("--flip32", type=int, default=1, help="32^3 FP64 dam-break leg (0 skips)")
    ap.add_argument("--surface", type=int, default=1,
                    help="marching-cubes export of the FLIP leg's fluid (0 skips)")
    ap.add_argument("--diff-n", type=int, default=DIFF_N, help="grid of the differentiable leg (profiling runs)")
    ap.add_argument("--diff-dirs", type=int, default=16,
                    help="finite-difference directions of the differentiable leg (-1 skips the leg)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.impl == "reference":
        reference_arm(args, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    from simcraft_b200 import _capi, scenes
    from simcraft_b200.replicas import Replicas
    from simcraft_b200.solver import CgSolver3D, Context, CRIT_REL_L2, PREC_FP64, PREC_MIXED

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = Context(local)
    replicas = Replicas(rank, world, dist, dev)
    n = args.solve_n
    if args.skip_solve:
        fl = flip_leg(args, dev, ctx, dist, rank, world)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "flip": fl}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    L = _capi.lib()
    h = 1.0 / n
    dt = DT_OVER_H * h
    N = n * n * n
    sdf, info = build_scene(n)
    adiag, an, active, act_h, rhs_h, rinfo = build_system_device(n, sdf, dev, ctx)
    rhs_d = torch.from_numpy(rhs_h).to(dev)
    n_active = int(act_h.sum())
    f64 = dict(dtype=torch.float64, device=dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())

    # pinned host copies for the end-to-end arm (what a host caller passes)
    pin = lambda t: t.cpu().pin_memory()
    adiag_h, an_h, act_hp = pin(adiag), [pin(a) for a in an], pin(active)
    rhs_hp = torch.from_numpy(rhs_h).pin_memory()
    pg_h = torch.zeros((n, n, n), dtype=torch.float64).pin_memory()

    def hptr(t):
        return ctypes.c_void_p(t.data_ptr())

    solvers = {
        "mixed": CgSolver3D(n, n, n, context=ctx, tol=TOL, max_iter=5000, criterion=CRIT_REL_L2,
                            precision=PREC_MIXED),
        "fp64": CgSolver3D(n, n, n, context=ctx, tol=TOL, max_iter=5000, criterion=CRIT_REL_L2,
                           precision=PREC_FP64),
    }
    pg_d = torch.zeros((n, n, n), **f64)
    an_dev = _capi.ptr_array([ptr(a) for a in an])
    an_host = _capi.ptr_array([hptr(a) for a in an_h])

    def solve_device(s):
        st = _capi.sc_pcg_stats()
        rc = L.sc_pcg_solve_device(s.handle, ptr(adiag), an_dev, ptr(rhs_d), ptr(active), ptr(pg_d),
                                   ctypes.byref(st))
        _capi.check("sc_pcg_solve_device", rc, ctx.handle)
        return st

    def solve_host(s):
        st = _capi.sc_pcg_stats()
        rc = L.sc_pcg_solve_host(s.handle, hptr(adiag_h), an_host, hptr(rhs_hp), hptr(act_hp), hptr(pg_h),
                                 ctypes.byref(st))
        _capi.check("sc_pcg_solve_host", rc, ctx.handle)
        return st

    stream = torch.cuda.ExternalStream(ctx.stream)

    def timed(fn, s):
        """K steps between a barrier + synchronize; device time by CUDA events on the solver stream."""
        for _ in range(args.warmup):
            fn(s)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        last = None
        for _ in range(args.steps):
            last = fn(s)
        e1.record(stream)
        torch.cuda.synchronize()
        return replicas.max(e0.elapsed_time(e1)), last

    with Clocks(local) as clk:
        ms_mixed, st_mixed = timed(solve_device, solvers["mixed"])
        ms_fp64, st_fp64 = timed(solve_device, solvers["fp64"])
        e2e_ms, st_e2e = timed(solve_host, solvers["mixed"])
    clocks = clk.summary()

    # per-kernel device times on the resident FP64 system -> roofline of the sweeps
    kt = (ctypes.c_double * 8)()
    _capi.check("sc_pcg_time_kernels", L.sc_pcg_time_kernels(solvers["fp64"].handle, 20, kt), ctx.handle)
    kms = list(kt)
    kt32 = (ctypes.c_double * 8)()
    _capi.check("sc_pcg_time_kernels", L.sc_pcg_time_kernels(solvers["mixed"].handle, 20, kt32), ctx.handle)
    kms32 = list(kt32)
    pk, pk_src = peaks()
    # The headline (mixed) solve iterates Eisenstat's form in FP32; its top
    # kernel is the fused forward sweep: s, t, Pinv, Dt, cL, cD, cB, E read and
    # w written, 4 bytes each.  Its backward sweep reads rh, s, E, uR, uU, uF and
    # writes s and t.
    bytes_fwde32 = N * 9 * 4
    bytes_bwde32 = N * 8 * 4
    bytes_bwd = N * (7 * 8 + 1)
    bytes_fwd = N * (6 * 8 + 1)
    achieved = bytes_fwde32 / (kms32[7] * 1e-3) / 1e9
    traffic = read_traffic("fwd_eisenstat_fp32", n)
    roofline = {"bound": "hbm", "kernel": "fused Eisenstat forward sweep, FP32 (k_wave FwdEisenstatOp<float>), "
                                          "the top kernel of the mixed solve",
                "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src + " (burst copy)",
                "traffic": traffic, "algorithmic_bytes_per_launch": bytes_fwde32,
                "ms_per_launch": kms32[7],
                "eisenstat_backward_sweep_fp32": {"ms": kms32[6], "achieved_gbs": bytes_bwde32 / (kms32[6] * 1e-3) / 1e9},
                "fp64_backward_sweep": {"achieved_gbs": bytes_bwd / (kms[2] * 1e-3) / 1e9,
                                        "traffic": read_traffic("bwd_fp64", n)},
                "kernel_ms": {"pivot": kms[0], "forward_sweep": kms[1], "backward_sweep": kms[2],
                              "spmv": kms[3], "axpy": kms[4], "scale_add": kms[5]},
                "forward_sweep_gbs": bytes_fwd / (kms[1] * 1e-3) / 1e9,
                "kernel_ms_fp32_inner": {"eisenstat_backward_sweep": kms32[6], "eisenstat_forward_sweep": kms32[7],
                                         "axpy": kms32[4], "init_forward_sweep": kms32[1]},
                "kernel_ms_fp32_standard_step": {"forward_sweep": kms32[1], "backward_sweep": kms32[2],
                                                 "spmv": kms32[3]},
                "kernel_gbs_fp64": {"spmv": N * 49 / (kms[3] * 1e-3) / 1e9, "axpy": N * 48 / (kms[4] * 1e-3) / 1e9,
                                    "scale_add": N * 24 / (kms[5] * 1e-3) / 1e9}}

    ms_step = ms_mixed / args.steps
    value = ms_step / world  # replicas: whole-job ms per solve
    h2d = 5 * 8 * N + N  # Adiag, Left, Down, Back, rhs (doubles) + active (bytes)
    d2h = 8 * N
    out = {
        "metric": METRIC, "value": value, "unit": "ms/solve", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (FP32 Eisenstat-form MIC(0) CG, FP64 residual replacement)",
        "data": "synthetic (seeded sphere pool, no dataset)",
        "config": solve_config(n, info, n_active, world),
        "solver": "mixed MIC(0)-PCG: FP32 CG on the split system (Eisenstat) with FP64 residual replacement",
        "fp64": {"ms_per_solve": ms_fp64 / args.steps, "iterations": st_fp64.iterations,
                 "iterations_per_s": st_fp64.iterations / (ms_fp64 / args.steps * 1e-3),
                 "true_rel_l2": st_fp64.true_rel_l2},
        "mixed": {"ms_per_solve": ms_step, "inner_iterations": st_mixed.iterations,
                  "iterations_per_s": st_mixed.iterations / (ms_step * 1e-3),
                  "fp64_replacements": st_mixed.outer, "true_rel_l2": st_mixed.true_rel_l2},
        "mixed_speedup_vs_fp64": (ms_fp64 / ms_mixed),
        "e2e": {"value": e2e_ms / args.steps / world, "unit": "ms/solve", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "sc_pcg_solve_host (CgSolver3D::solve on pinned host arrays)"},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": None,
    }
    # kernels launched inside the timed region of the headline (mixed) arm,
    # counted by the solver itself (CUDA-graph nodes included)
    out["gpu_launches"] = int(st_mixed.kernel_launches) * args.steps
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sysm = {"adiag": adiag.cpu().numpy(), "an": [a.cpu().numpy() for a in an], "active": act_h}
        cit = reference_iterations(sysm, rhs_h, threads)
        cms, cit, pg_cpu, kind = cpu_solve_ms(sysm, rhs_h, threads, cit)
        a = act_h.astype(bool)
        pg_gpu = pg_d.cpu().numpy()
        out["cpu_baseline"] = {"value": cms, "unit": "ms/solve", "cores": threads, "kind": kind,
                               "sample": f"one full FP64 solve of the same {n}^3 system by the reference's "
                                         f"CgSolver3D::solve ({kind}), {cit} iterations (the count reaching "
                                         f"{TOL:g} relative L2)",
                               "rel_l2_vs_gpu_fp64": float(np.linalg.norm(pg_gpu[a] - pg_cpu[a]) /
                                                           np.linalg.norm(pg_cpu[a]))}
    del solvers
    torch.cuda.empty_cache()
    if rank == 0:
        out["tolerance_sweep"] = tolerance_sweep(n, ctx, adiag, an, rhs_d, active, act_h)
    if args.large_steps > 0:
        out["solve_512"] = large_solve_leg(args, dev, ctx, replicas,
                                           cpu=rank == 0 and world == 1 and not args.no_cpu)
    if args.flip_steps > 0:
        out["flip"] = flip_leg(args, dev, ctx, dist, rank, world)
        if "surface" in out["flip"]:
            out["surface"] = out["flip"].pop("surface")
    # CPU oracles on the host cores: one process only (as for the solve leg)
    cpu = rank == 0 and world == 1 and not args.no_cpu
    if args.collider:
        out["collider"] = collider_leg(args, dev, ctx, cpu)
    if args.flip32:
        out["flip_32"] = flip32_leg(args, ctx, cpu)
    if args.diff_dirs >= 0:
        out["diff"] = diff_leg(args, ctx, replicas)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
