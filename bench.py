"""Benchmark: periodic FP64 multigrid solves/s on one 256^3 grid, plus the 256^3 stencil roofline.

Workload (one "step"): -Lap u = f on a periodic cell-centred 256^3 grid (h = 1/256), f = 8 sine
modes (seed 1, mean removed), 7-point Laplacian, weighted Jacobi omega = 2/3, 2^3 averaging
restriction, piecewise-constant prolongation, coarsest grid 4^3, iterated from u = 0 to a 1e-10
relative max-norm residual, all in FP64 on the GPU. The cycle is V(4,4): V(2,2) with this
restriction/prolongation pair stalls at depth (reference CPU path: 0.48, 0.72, 0.95 per cycle at
32^3, 64^3, 128^3), so it never reaches 1e-10 at 256^3.

  value : solves/s with inputs resident in HBM (device-timed, max over ranks)
  e2e   : the same through the public API with host buffers: H2D of f, solve, D2H of u per step
          (copies on a second stream, overlapping the neighbouring steps' solves)
  stencil: Stencil::apply 7-point FP64 on a 256^3 box (src 258^3), GB/s and fraction of HBM
  roofline: the dominant kernel, the finest-level Jacobi sweep (k_star_tma<Lap7, EpiRelax>)
  mixed : the same problem with FP32 V-cycles inside FP64 residual/correction/norm
  mixed_384: FP64 vs mixed at 384^3, Poisson and Helmholtz with a per-cell alpha (exact coarsest solve)
  fas   : the reference's FAS LevelMultigridSolver (4th-order flux-form Laplacian) at 64^3..256^3
  amr_level: 100 steps of exchange + 13-point Euler update over a 512-patch uneven level
  serving: a stream of Poisson/Helmholtz requests (edges 32..192) served by the batching engine
          (mixed precision and FP64) vs plain multigrid one request at a time (saturated and at the
          200/s arrival rate)

Multi-GPU (torchrun): every rank solves its own grid (replicas; no data-path collective), value is
the whole-job rate. --impl reference times the reference's own CPU code (oracle/_ref) on host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
LEVELS = 6            # 256 -> 4
NU1 = NU2 = 4
NU_BOTTOM = 10
OMEGA = 2.0 / 3.0
TOL = 1e-10
MAX_ITER = 100
# V(4,4) cycles the GPU solver takes on this workload; the reference arm uses it only when it ran too
# few cycles for a solve of its own to converge (the two residual histories are bitwise identical)
GPU_CYCLES_PER_SOLVE = 16
STENCIL_BYTES = 8 * (258 ** 3 + 256 ** 3)          # algorithmic bytes of dst |= L(src), 256^3
RELAX_BYTES = 24 * 256 ** 3                        # read phi, read rho, write phi_new (one or two sweeps)
SERVE_MAX_ACTIVE = 128                             # serving: solves in one batched cycle at most


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def max_over_ranks_of(v, dist=None, device="cuda"):
    """The largest of every rank's v (a time: the whole job takes as long as its slowest rank)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, t_max):
    """Solves per second of the whole job: every rank solves `steps` grids of its own (replicas,
    weak scaling), and the job ends when the slowest rank does."""
    return world * steps / t_max


def workload_config():
    return {"workload": "periodic Poisson multigrid, 256^3 cell-centred FP64, 7-point, V(%d,%d) weighted Jacobi "
                        "omega=2/3, 2^3 average restriction, constant prolongation, coarsest 4^3, tol 1e-10 "
                        "(max-norm, relative), f = 8 sine modes seed 1" % (NU1, NU2),
            "n": N, "levels": LEVELS + 1, "nu1": NU1, "nu2": NU2, "nu_bottom": NU_BOTTOM, "omega": OMEGA,
            "tol": TOL, "l2_policy": "inputs larger than L2 (each 256^3 field is 134 MB; solver state ~0.9 GB)"}


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        for line in out.strip().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _host_procs(per_proc_gb=1.6, cap=32):
    """Independent single-threaded reference processes the host can run at once: one per CPU this
    process may use, bounded by available memory (about 1.6 GB per 256^3 reference solve)."""
    try:
        ncpu = len(os.sched_getaffinity(0))
    except AttributeError:
        ncpu = os.cpu_count() or 1
    procs = max(1, min(cap, ncpu))
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail_gb = int(line.split()[1]) / 2 ** 20
                    procs = max(1, min(procs, int(avail_gb * 0.8 / per_proc_gb)))
    except OSError:
        pass
    return procs, ncpu


def _ref_cycles_worker(ncycles):
    sys.path.insert(0, ROOT)
    from oracle.oracle import Ref
    from proto_b200 import workloads as W
    rho = W.poisson_rho(N, seed=1).reshape(-1).copy()
    first, done, t0, t_end = Ref().mg_cs_cycles(N, 64, LEVELS, NU1, NU2, NU_BOTTOM, OMEGA, TOL, rho, ncycles)
    return first, done, t0, [float(t) for t in t_end]


def cpu_reference_cycles(warmup, steps, gpu_cycles=None, procs=None):
    """The reference's own CPU solver (oracle/_ref: its LevelBoxData / Stencil / AvgDown /
    InterpStencil code, boxes of 64) on the host cores. `procs` independent single-threaded
    processes (the reference solver has no threading of its own) each run warmup + steps real
    V(4,4) cycles of the 256^3 solve, each cycle followed by the residual norm, from u = 0, starting a
    new solve whenever one converges. A step is one cycle in every process; the timed region is a
    process's last `steps` cycles, and the slowest process's region counts. Solves/s = procs * steps
    / (T * cycles per solve), the cycle count being the one the reference needed to converge, or, if
    no solve converged within the cycles run, the GPU solver's count for the same problem (the two
    residual histories are bitwise identical)."""
    import multiprocessing as mp
    from oracle.oracle import Ref
    if not Ref.available():
        raise RuntimeError("oracle/_ref/libproto_ref.so is not built")
    nproc, ncpu = _host_procs()
    if procs:
        nproc = procs
    ncyc = warmup + steps
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc) as pool:
        res = pool.map(_ref_cycles_worker, [ncyc] * nproc)
    spans = []
    for first, done, t0, t_end in res:
        t_a = t_end[warmup - 1] if warmup >= 1 else t0
        spans.append(t_end[ncyc - 1] - t_a)
    T = max(spans)
    firsts = [r[0] for r in res if r[0] > 0]
    if firsts:
        cps, src = firsts[0], "reference (converged within the run)"
    else:
        if not gpu_cycles:
            raise RuntimeError("no reference solve converged within %d cycles" % ncyc)
        cps, src = gpu_cycles, "GPU solver, same problem (bitwise-identical residual history)"
    rate = nproc * steps / (T * cps)
    return {"value": rate, "unit": "solves/s", "cores": nproc, "host_cpus": ncpu, "kind": "reference",
            "timed_s": T, "ms_per_cycle_step": 1000.0 * T / steps, "cycles_per_solve": cps,
            "cycles_per_solve_from": src, "solves_completed": int(sum(r[1] for r in res)),
            "sample": "%d processes x (%d warm-up + %d timed) real V(%d,%d) cycles + residual norm of the 256^3 "
                      "solve (reference code, boxes of 64, 1 thread each); %.2f s per cycle" %
                      (nproc, warmup, steps, NU1, NU2, T / steps)}


def profile_kernels(pb, torch):
    """One launch each of the bench's roofline kernels on 256^3 data: the FP64 Jacobi sweep, the
    FP32 sweep of the mixed-precision solver, the 7-point Stencil::apply, and the FP64 and FP32
    two-sweep passes."""
    offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    S = pb.Stencil([-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0], offs)
    src = torch.rand(258 ** 3, dtype=torch.float64, device="cuda")
    dst = torch.empty(256 ** 3, dtype=torch.float64, device="cuda")
    mg64 = pb.Multigrid(pb.MGParams(n=N, levels=LEVELS, nu1=NU1, nu2=NU2))
    mg32 = pb.Multigrid(pb.MGParams(n=N, levels=LEVELS, nu1=NU1, nu2=NU2, precision=pb.MG_MIXED))
    mg64.relax(1)
    mg32.relax(1)
    S.apply(src, pb.Box.cube(256).grow(1), dst, pb.Box.cube(256), scale=65536.0)
    mg64.relax(2)
    mg32.relax(2)
    torch.cuda.synchronize()
    pb.device_check()


def profile_solve(pb, torch, which):
    """Two solves (the second one is the one a launch list reads) of the bench's 256^3 problem
    ("f64", "mixed") or of the 384^3 Poisson configuration ("f64_384", "mixed_384": coarsest 3^3
    solved exactly)."""
    from proto_b200 import workloads as W
    prec = pb.MG_MIXED if which.startswith("mixed") else 0
    n, levels, bottom = (384, 7, pb.MG_BOTTOM_DIRECT) if which.endswith("384") else (N, LEVELS, 0)
    mg = pb.Multigrid(pb.MGParams(n=n, levels=levels, nu1=NU1, nu2=NU2, nu_bottom=NU_BOTTOM, omega=OMEGA,
                                  max_iter=MAX_ITER, tol=TOL, precision=prec, bottom=bottom))
    rho = torch.from_numpy(W.poisson_rho(n, seed=1).reshape(-1).copy()).cuda()
    phi = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    for _ in range(2):
        phi.zero_()
        it, _ = mg.solve(rho, phi)
    torch.cuda.synchronize()
    pb.device_check()
    print(json.dumps({"cycles": it, "launches_per_solve": 3 + it * mg.launches_per_cycle() + 1}))


LAP13_OFFS = [(1, 0, 0), (0, 0, 0), (-1, 0, 0), (2, 0, 0), (-2, 0, 0), (0, 1, 0), (0, -1, 0), (0, 2, 0), (0, -2, 0),
              (0, 0, 1), (0, 0, -1), (0, 0, 2), (0, 0, -2)]
LAP13_COEFS = [4.0 / 3, -7.5, 4.0 / 3, -1.0 / 12, -1.0 / 12] + [4.0 / 3, 4.0 / 3, -1.0 / 12, -1.0 / 12] * 2


def run_amr_level(pb, torch, steps=100, reps=5, cpu=True, tune=True):
    """Uneven AMR level: 512 patches (per-axis widths from {16,24,32,48,64}, seed 2) tiling a
    periodic domain, 2 ghost cells, u ~ U[-1,1]; a step = ghost exchange + u += dt*L13(u) (4th-order
    13-point Laplacian, dt = 0.1 h^2) over every patch; 100 steps as one captured graph, tiles
    autotuned per patch-size class. Algorithmic bytes: 16 B per interior cell per step."""
    from proto_b200 import workloads as W
    widths = W.amr_widths(seed=2)
    boxes, L = W.amr_patches(widths)
    lv = pb.Level([pb.Box(*b) for b in boxes], 2, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    S = pb.Stencil(LAP13_COEFS, LAP13_OFFS)
    interior = sum((b[1][0] - b[0][0] + 1) * (b[1][1] - b[0][1] + 1) * (b[1][2] - b[0][2] + 1) for b in boxes)
    a = torch.rand(lv.slab_elems, dtype=torch.float64, device="cuda") * 2 - 1
    b = torch.zeros_like(a)
    h = 1.0 / L[0]
    scale, dt = 1.0 / (h * h), 0.1 * h * h
    if tune:
        lv.autotune(S, a, b, scale=scale)
    lv.steps(S, pb.EPI_EULER, a, b, steps, scale=scale, a=dt)     # capture + warm
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        lv.steps(S, pb.EPI_EULER, a, b, steps, scale=scale, a=dt)
    e1.record(st)
    torch.cuda.synchronize()
    pb.device_check()
    t = e0.elapsed_time(e1) / 1000.0 / (reps * steps)
    peak, _ = measured_peaks()
    out = {"workload": "512 patches, domain %dx%dx%d, 2 ghosts, 13-point 4th-order, u += dt*L(u), %d steps per "
                       "graph launch" % (L[0], L[1], L[2], steps),
           "interior_cells": interior, "us_per_step": t * 1e6, "steps_per_s": 1.0 / t,
           "gpts_per_s": interior / t / 1e9, "gbs_algorithmic": 16.0 * interior / t / 1e9,
           "frac_of_hbm": 16.0 * interior / t / 1e9 / peak, "tiles": lv.tiles(),
           "gpu_launches_per_step": 1,   # fused step: the tensor-product tiling needs no exchange launch
           }
    try:   # the reference's own per-patch stepping on one host core, one step
        from oracle.oracle import Ref
        if cpu and Ref.available():
            import numpy as np
            data = np.zeros(lv.slab_elems)
            parts, off = [], 0
            for p, o in zip(lv.patches, lv.offsets):
                n = int(np.prod([p.size(d) + 4 for d in range(3)]))
                parts.append(data[o:o + n])
            cat = np.concatenate(parts)
            t0 = time.perf_counter()
            Ref().level13_steps(widths, 2, h, dt, 1, cat)
            tc = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": 1.0 / tc, "unit": "steps/s", "cores": 1, "kind": "reference",
                                   "sample": "1 step of the same level with the reference's BoxData/copyTo/Stencil "
                                             "code (oracle/_ref), single-threaded"}
    except Exception as e:   # the baseline never hides the GPU result
        out["cpu_baseline"] = {"error": str(e)}
    return out


def run_sharded_level(pb, torch, dist, rank, world, steps=20, warmup=3):
    """The uneven AMR level (512 patches, seed 2) sharded over the ranks: each rank owns a Morton
    run of 512/N patches in its own device level, a step = local ghost exchange + pack of the
    remote ghost regions + one grouped NCCL send/recv round with the neighbour ranks + unpack +
    u += dt*L13(u) on the rank's patches. Total work is fixed as N grows (strong scaling); the time
    is the slowest rank's, on CUDA events between barriers."""
    from proto_b200 import workloads as W
    from proto_b200 import sharding as SH
    boxes, L = W.amr_patches(W.amr_widths(seed=2))
    domain = ((0, 0, 0), tuple(v - 1 for v in L))
    sl = SH.ShardedLevel(boxes, 2, domain, (1, 1, 1), rank, world, SH.DistComm())
    S = pb.Stencil(LAP13_COEFS, LAP13_OFFS)
    u = torch.rand(sl.slab_elems, dtype=torch.float64, device="cuda") * 2 - 1
    tmp = torch.zeros_like(u)
    h = 1.0 / L[0]
    scale, dt = 1.0 / (h * h), 0.1 * h * h
    for _ in range(warmup):
        sl.step(S, u, tmp, scale, dt)
        u, tmp = tmp, u
    dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        sl.step(S, u, tmp, scale, dt)
        u, tmp = tmp, u
    e1.record(st)
    torch.cuda.synchronize()
    dist.barrier()
    t = max_over_ranks_of(e0.elapsed_time(e1) / 1000.0 / steps, dist, "cuda")
    m = sl.absmax(u)
    pb.device_check()
    interior = sum((b[1][0] - b[0][0] + 1) * (b[1][1] - b[0][1] + 1) * (b[1][2] - b[0][2] + 1) for b in boxes)
    halo = sum(b.numel() for b in sl.sbuf.values())
    return {"workload": "512 patches, domain %dx%dx%d, 2 ghosts, 13-point 4th-order, u += dt*L(u), sharded over "
                        "%d ranks (Morton runs), NCCL halo exchange every step" % (L[0], L[1], L[2], world),
            "scaling": "strong", "ranks": world, "patches_per_rank": len(sl.mine), "us_per_step": t * 1e6,
            "steps_per_s": 1.0 / t, "gpts_per_s": interior / t / 1e9, "halo_bytes_sent_per_step_rank0": 8 * halo,
            "peers_rank0": len(sl.sbuf), "absmax_after": m,
            "gpu_launches_per_step": 3 + (1 if sl.rbuf else 0)}


def run_precision(pb, torch, n=384, levels=7, reps=3):
    """Mixed precision at 384^3: the 8-mode Poisson problem (seed 1) and the Helmholtz variant
    alpha u - beta L u = f with alpha ~ U[0.1, 1] per cell (seed 3), beta = 1; V(4,4), omega = 2/3,
    coarsest 3^3 solved exactly, tol 1e-10. Each form: the FP64 solver and the mixed solver (FP32
    cycles, FP64 residual/correction/norms), iterations, solves/s (device events), final relative
    residual and the mixed solution's error against the FP64 one (the FP64 GPU solver performs the
    CPU oracle's arithmetic bit for bit)."""
    from proto_b200 import workloads as W
    rho = torch.from_numpy(W.poisson_rho(n, seed=1).reshape(-1).copy()).cuda()
    alpha = torch.from_numpy(W.helmholtz_alpha(n, seed=3).reshape(-1).copy()).cuda()
    st = torch.cuda.current_stream()
    out = {"workload": "%d^3 periodic, 7-point, V(%d,%d) omega=2/3, coarsest 3^3 exact, tol 1e-10; Poisson (8 sine "
                       "modes, seed 1) and Helmholtz alpha~U[0.1,1] per cell (seed 3), beta=1" % (n, NU1, NU2)}
    for form, name in ((pb.MG_POISSON, "poisson"), (pb.MG_HELMHOLTZ, "helmholtz")):
        f = rho if form == pb.MG_POISSON else -rho   # Poisson solves L u = -f in the reference's sign
        res = {}
        sol = {}
        for prec, pname in ((pb.MG_FP64, "fp64"), (pb.MG_MIXED, "mixed")):
            mg = pb.Multigrid(pb.MGParams(n=n, levels=levels, nu1=NU1, nu2=NU2, nu_bottom=NU_BOTTOM, omega=OMEGA,
                                          max_iter=MAX_ITER, tol=TOL, form=form, precision=prec,
                                          bottom=pb.MG_BOTTOM_DIRECT))
            if form == pb.MG_HELMHOLTZ:
                mg.set_alpha(alpha)
            phi = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
            it, hist = mg.solve(f, phi)   # warm-up (graph capture)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            for e0, e1 in ev:
                phi.zero_()
                e0.record(st)
                it, hist = mg.solve(f, phi)
                e1.record(st)
            torch.cuda.synchronize()
            ms = sorted(e0.elapsed_time(e1) for e0, e1 in ev)
            res[pname] = {"iters": it, "solves_per_s": 1000.0 / ms[len(ms) // 2], "ms_per_solve": ms[len(ms) // 2],
                          "final_rel_residual": hist[-1] / hist[0]}
            sol[pname] = phi
            del mg
        d = (sol["mixed"] - sol["fp64"]).abs().max().item()
        res["mixed"]["max_abs_err_vs_fp64"] = d
        res["mixed"]["max_rel_err_vs_fp64"] = d / sol["fp64"].abs().max().item()
        res["speedup_mixed_vs_fp64"] = res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"]
        out[name] = res
        del sol
    pb.device_check()
    return out


def run_fas(pb, torch, sizes=(64, 128, 256), reps=3, cpu=True):
    """LevelMultigridSolver<BoxOp_Laplace> (FAS V(6,6), 4th-order flux-form Laplacian, 10 bottom
    sweeps, lambda = 0.5/rho) on periodic n^3 boxes, coarsest 4^3, force = 8 sine modes (seed 1),
    tol 1e-10: solves/s (device events) and iterations per size; beside it the reference's own
    solver (oracle/_ref, one core) timed for one cycle at 64^3 (the reference example's size, boxes
    of 16) and scaled by the GPU's iteration count there."""
    import math
    from proto_b200 import workloads as W
    st = torch.cuda.current_stream()
    out = {"workload": "FAS V(6,6) 4th-order flux-form Laplace, periodic, coarsest 4^3, 8 sine modes (seed 1), "
                       "tol 1e-10"}
    for n in sizes:
        levels = int(round(math.log2(n))) - 1
        force = torch.from_numpy(-W.poisson_rho(n, seed=1).reshape(-1)).cuda()
        mg = pb.FAS(n, levels)
        phi = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
        it, hist = mg.solve(force, phi, max_iter=20, tol=1e-10)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for e0, e1 in ev:
            phi.zero_()
            e0.record(st)
            it, hist = mg.solve(force, phi, max_iter=20, tol=1e-10)
            e1.record(st)
        torch.cuda.synchronize()
        ms = sorted(e0.elapsed_time(e1) for e0, e1 in ev)[reps // 2]
        out["n%d" % n] = {"levels": levels, "iters": it, "ms_per_solve": ms, "solves_per_s": 1000.0 / ms,
                          "final_rel_residual": hist[-1] / hist[0]}
        del mg
    pb.device_check()
    if cpu:
        try:
            from oracle.oracle import Ref
            if Ref.available():
                R = Ref()
                f = -W.poisson_rho(64, seed=1).reshape(-1).copy()
                p = np.zeros(64 ** 3)
                t0 = time.perf_counter()
                it_ref, _ = R.mg_fas(64, 16, 5, 20, 1e-10, f, p)
                t = time.perf_counter() - t0
                out["cpu_baseline_64"] = {"value": 1.0 / t, "unit": "solves/s", "cores": 1, "kind": "reference",
                                          "iters": it_ref,
                                          "sample": "one whole FAS solve at 64^3 (boxes of 16, %d cycles to 1e-10) with "
                                                    "the reference's LevelMultigridSolver, one thread" % it_ref}
        except Exception as e:   # the baseline never hides the GPU result
            out["cpu_baseline_64"] = {"error": str(e)}
    return out


def profile_serving(pb, torch, count=16, n=96, steps=2):
    """A small in-flight batch for kernel captures: `count` Helmholtz solves of edge n submitted to
    one serving engine (public API, pinned host buffers), `steps` V-cycles for all of them."""
    from proto_b200 import serving as S
    from proto_b200 import workloads as W
    # max_active = 4 * count: up to count solves load at once, so all of them run from the first cycle
    eng = pb.Serve(8 << 30, max_active=4 * count, tol=1e-30, max_cycles=steps)
    f = S.pinned(n ** 3)
    f[:] = W.sine_modes_rhs(n, seed=5, modes=4).reshape(-1)
    outs = [S.pinned(n ** 3) for _ in range(count)]
    for k in range(count):
        eng.submit(n, f, outs[k], form=pb.MG_HELMHOLTZ, alpha=0.25 + 0.5 * k / count)
    eng.run_until_idle()
    eng.poll()
    torch.cuda.synchronize()
    pb.device_check()


def profile_serving_mix(pb, torch, count=150):
    """The first `count` requests of the serving trace, all available at once, through one engine
    (for launch lists of the batched phases on the real mix of edges and forms)."""
    from proto_b200 import serving as S
    trace = S.make_trace(count=count)
    data = S.TraceData(trace)
    S.serve_trace(pb, trace, data, realtime=False, max_active=128, tol=1e-8)
    torch.cuda.synchronize()
    pb.device_check()


def run_serving(pb, count):
    """Request stream of periodic Poisson/Helmholtz solves (Poisson arrivals at 200/s, seed 4; edge
    log-uniform in [32, 192] rounded to 16; alpha ~ U[0, 1]; a 4-mode right-hand side per request).
    Four arms, each with pinned host buffers and the copies inside the measured time: the batching
    engine in mixed precision and in FP64 (in-flight solves advanced together), plain mixed-precision
    multigrid one request at a time, and plain FP64 multigrid one request at a time; so the two
    served arms give what precision gains under batching, and each served arm against its
    one-at-a-time arm what batching gains. At tolerance 1e-8 (the configuration's) and 1e-10 (the
    precision target), saturated (every request available at once); at 1e-8 also open loop at the
    arrival rate for latency. Every served result is compared with the FP64 solver's solution of the
    same request (the FP64 engine's bitwise)."""
    from proto_b200 import serving as S
    trace = S.make_trace(count=count)
    t0 = time.perf_counter()
    data = S.TraceData(trace)
    out = {"workload": "%d requests, Poisson arrivals 200/s (seed 4), edge log-uniform [32,192] step 16, "
                       "Poisson/Helmholtz 50/50, alpha~U[0,1], one 4-sine-mode right-hand side per request" % count,
           "hbm_budget_gb": 150, "max_active": SERVE_MAX_ACTIVE, "rhs_bytes": data.nbytes,
           "setup_s": time.perf_counter() - t0}
    firsts = {}
    for r in trace:
        firsts.setdefault((r["n"], r["helm"]), r)
    for tol, name in ((1e-8, "tol_1e-8"), (1e-10, "tol_1e-10")):
        eng = pb.Serve(150 << 30, max_active=SERVE_MAX_ACTIVE, tol=tol)
        eng64 = pb.Serve(150 << 30, max_active=SERVE_MAX_ACTIVE, tol=tol, precision=pb.MG_FP64)
        fp64 = S.SingleSolvers(pb, trace, tol, pb.MG_FP64)
        mixed = S.SingleSolvers(pb, trace, tol, pb.MG_MIXED)
        # warm-up (untimed): each engine serves the trace once, as a running server would have (its
        # cache holds the hierarchies this traffic needs); every single solver solves once
        S.serve_trace(pb, trace, data, realtime=False, engine=eng)
        S.serve_trace(pb, trace, data, realtime=False, engine=eng64)
        for r in firsts.values():
            fp64.solve(r, data.rhs_of(r["i"]))
            mixed.solve(r, data.rhs_of(r["i"]))
        served64 = S.serve_trace(pb, trace, data, realtime=False, engine=eng64)
        err64 = S.verify(pb, trace, data, fp64)
        served = S.serve_trace(pb, trace, data, realtime=False, engine=eng)
        err = S.verify(pb, trace, data, fp64)
        m1 = S.single_trace(pb, trace, data, mixed, realtime=False)
        f1 = S.single_trace(pb, trace, data, fp64, realtime=False)
        sps = lambda a: a["solves_per_s"]
        res = {"saturated": {"served_mixed": served, "served_fp64_batched": served64, "mixed_one_at_a_time": m1,
                             "fp64_one_at_a_time": f1,
                             "served_vs_fp64": sps(served) / sps(f1),
                             "precision_gain_batched": sps(served) / sps(served64),
                             "batching_gain_fp64": sps(served64) / sps(f1),
                             "batching_gain": sps(served) / sps(m1),
                             "precision_gain": sps(m1) / sps(f1)},
               "served_rel_err_vs_fp64": err, "served_fp64_rel_err_vs_fp64": err64}
        if tol == 1e-8:
            a = S.serve_trace(pb, trace, data, realtime=True, engine=eng)
            b = S.single_trace(pb, trace, data, fp64, realtime=True)
            res["arrival_rate"] = {"served_mixed": a, "fp64_one_at_a_time": b}
        out[name] = res
        del eng, eng64, fp64, mixed
    return out


def run_reference(args, rank, world):
    """The reference's own CPU path, unmodified (oracle/_ref), on this host's cores, for the same
    workload and metric: every step is one real V(4,4) cycle (+ residual norm) of the 256^3 solve in
    each of the independent reference processes (cpu_reference_cycles). Rank 0 alone runs it."""
    if rank != 0:
        return
    t0 = time.perf_counter()
    cb = cpu_reference_cycles(args.warmup, args.steps, gpu_cycles=GPU_CYCLES_PER_SOLVE,
                              procs=args.ref_procs or None)
    wall = time.perf_counter() - t0
    line = {"impl": "reference", "metric": "MG solves/s", "value": cb["value"], "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["ms_per_cycle_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
            "step": "one V(%d,%d) cycle + residual norm in each of %d reference processes; solves/s = processes x "
                    "steps / (timed s x %d cycles per solve)" % (NU1, NU2, cb["cores"], cb["cycles_per_solve"]),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the 384^3 mixed-precision section")
    ap.add_argument("--no-fas", action="store_true", help="skip the FAS (LevelMultigridSolver) section")
    ap.add_argument("--no-amr", action="store_true", help="skip the AMR-level section (and its tile autotuning)")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="run one 256^3 FP64 sweep, one FP32 sweep and one Stencil::apply, then exit (for ncu)")
    ap.add_argument("--profile-solve", choices=["f64", "mixed", "f64_384", "mixed_384"], default=None,
                    help="two solves only (for launch lists)")
    ap.add_argument("--profile-level", action="store_true",
                    help="run the AMR-level setup and 2 graph steps with default tiles, then exit (for ncu)")
    ap.add_argument("--profile-serving-mix", action="store_true",
                    help="the first 150 requests of the serving trace through one engine, then exit")
    ap.add_argument("--profile-serving", action="store_true",
                    help="16 in-flight 96^3 Helmholtz solves, 2 V-cycles (small case for kernel captures)")
    ap.add_argument("--profile-fas", action="store_true",
                    help="FAS solves at 256^3 only (for kernel captures)")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="reference arm: independent reference processes (0 = one per usable host CPU)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import proto_b200 as pb
    from proto_b200 import workloads as W
    torch.cuda.set_device(local)
    if args.profile_kernels:
        return profile_kernels(pb, torch)
    if args.profile_solve:
        return profile_solve(pb, torch, args.profile_solve)
    if args.profile_level:
        return run_amr_level(pb, torch, steps=2, reps=1, cpu=False, tune=False)
    if args.profile_serving:
        return profile_serving(pb, torch)
    if args.profile_serving_mix:
        return profile_serving_mix(pb, torch)
    if args.profile_fas:
        return run_fas(pb, torch, sizes=(256,), reps=1, cpu=False)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return max_over_ranks_of(v, dist, "cuda")

    params = pb.MGParams(n=N, levels=LEVELS, nu1=NU1, nu2=NU2, nu_bottom=NU_BOTTOM, omega=OMEGA,
                         max_iter=MAX_ITER, tol=TOL)
    mg = pb.Multigrid(params)
    rho_host = W.poisson_rho(N, seed=1).reshape(-1).copy()
    rho = torch.from_numpy(rho_host).cuda()
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def one_solve():
        phi.zero_()
        return mg.solve(rho, phi)

    # clocks are sampled from before the first timed region to after the last multigrid one (the
    # timed regions are short; the sampler needs a moment to start)
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.5)
    for _ in range(max(args.warmup, 3)):
        it, hist = one_solve()
    iters = it
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_solve = []
    ev0.record(stream)
    for _ in range(args.steps):
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        it, hist = one_solve()
        e_b.record(stream)
        per_solve.append((e_a, e_b))
        assert it == iters
    ev1.record(stream)
    barrier()
    t_dev = ev0.elapsed_time(ev1) / 1000.0
    lat = sorted(a.elapsed_time(b) for a, b in per_solve)
    t_max = max_over_ranks(t_dev)
    value = whole_job_rate(world, args.steps, t_max)

    # end to end: host buffers, H2D of f and D2H of u of every step inside the timed region. The
    # copies run on a second stream, double-buffered: step k+1's f goes up and step k-1's u comes
    # down while step k solves.
    rho_pin = torch.from_numpy(rho_host).pin_memory()
    out_pin = [torch.empty(N ** 3, dtype=torch.float64).pin_memory() for _ in range(2)]
    rdev = [torch.empty_like(rho) for _ in range(2)]
    pdev = [torch.empty_like(phi) for _ in range(2)]
    cs = torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cs.wait_event(e0)
    with torch.cuda.stream(cs):
        rdev[0].copy_(rho_pin, non_blocking=True)
        ev_in[0].record(cs)
    for k in range(args.steps):
        b = k % 2
        if k + 1 < args.steps:
            with torch.cuda.stream(cs):
                rdev[1 - b].copy_(rho_pin, non_blocking=True)
                ev_in[1 - b].record(cs)
        stream.wait_event(ev_in[b])
        if k >= 2:
            stream.wait_event(ev_out[b])          # step k-2's result has left pdev[b]
        pdev[b].zero_()
        mg.solve(rdev[b], pdev[b])
        done = torch.cuda.Event()
        done.record(stream)
        cs.wait_event(done)
        with torch.cuda.stream(cs):
            out_pin[b].copy_(pdev[b], non_blocking=True)
            ev_out[b].record(cs)
    stream.wait_stream(cs)
    e1.record(stream)
    barrier()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    e2e = whole_job_rate(world, args.steps, t_e2e)

    # kernel-level figures (device events on the launching stream)
    coefs = [-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    S = pb.Stencil(coefs, offs)
    src = torch.rand(258 ** 3, dtype=torch.float64, device="cuda")
    dst = torch.empty(256 ** 3, dtype=torch.float64, device="cuda")
    sbox, dbox = pb.Box.cube(256).grow(1), pb.Box.cube(256)
    reps = 20
    for _ in range(3):
        S.apply(src, sbox, dst, dbox, scale=65536.0)
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        S.apply(src, sbox, dst, dbox, scale=65536.0)
    b.record(stream)
    barrier()
    t_st = a.elapsed_time(b) / 1000.0 / reps
    def time_relax(m, sweeps):
        for _ in range(3):
            m.relax(sweeps)
        barrier()
        a.record(stream)
        for _ in range(reps):
            m.relax(sweeps)
        b.record(stream)
        barrier()
        return a.elapsed_time(b) / 1000.0 / reps

    t_rx = time_relax(mg, 1)       # one sweep: k_star_tma<Lap7, EpiRelax>
    t_rx2 = time_relax(mg, 2)      # two sweeps in one pass: k_relax2 (the solve's dominant kernel)
    pb.device_check()
    phi64 = phi.clone()
    mg.solve(rho, phi64.zero_())

    # mixed precision: FP32 V-cycles inside FP64 residual and correction, same problem and tolerance
    mparams = pb.MGParams(n=N, levels=LEVELS, nu1=NU1, nu2=NU2, nu_bottom=NU_BOTTOM, omega=OMEGA,
                          max_iter=MAX_ITER, tol=TOL, precision=pb.MG_MIXED)
    mgm = pb.Multigrid(mparams)
    phim = torch.zeros_like(phi)

    def one_mixed():
        phim.zero_()
        return mgm.solve(rho, phim)

    for _ in range(max(args.warmup, 3)):
        itm, histm = one_mixed()
    barrier()
    lat_m = []
    a.record(stream)
    for _ in range(args.steps):
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        itm, histm = one_mixed()
        e_b.record(stream)
        lat_m.append((e_a, e_b))
    b.record(stream)
    barrier()
    t_mx = max_over_ranks(a.elapsed_time(b) / 1000.0)
    lat_m = sorted(x.elapsed_time(y) for x, y in lat_m)
    err_m = float((phim - phi64).abs().max() / phi64.abs().max())
    t_rx32 = time_relax(mgm, 1)
    t_rx32_2 = time_relax(mgm, 2)
    clk = clocks.stop()
    pb.device_check()
    value_m = whole_job_rate(world, args.steps, t_mx)
    amr = None if (world > 1 or args.no_amr) else run_amr_level(pb, torch)
    sharded = None if (world == 1 or args.no_amr) else run_sharded_level(pb, torch, dist, rank, world)
    precision = None if (world > 1 or args.no_precision) else run_precision(pb, torch)
    fas = None if (world > 1 or args.no_fas) else run_fas(pb, torch, cpu=not args.no_cpu_baseline)
    # the serving replay is a one-GPU measurement (replicas add nothing to it)
    serving = None if (args.no_serving or world > 1) else run_serving(pb, args.serve_requests)
    torch.cuda.synchronize()
    peak, peak_kind = measured_peaks()
    st_gbs = STENCIL_BYTES / t_st / 1e9
    rx_gbs = RELAX_BYTES / t_rx / 1e9
    rx2_gbs = RELAX_BYTES / t_rx2 / 1e9     # a two-sweep pass moves the bytes of one sweep

    traffic = {}
    tp = os.path.join(ROOT, "profiles", "relax_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp))
        except Exception:
            traffic = {}

    if rank == 0:
        launches = 3 + iters * mg.launches_per_cycle() + 1
        line = {
            "metric": "MG solves/s", "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(), "iters_per_solve": iters, "final_rel_residual": hist[-1] / hist[0],
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
        }
        if precision is not None:
            line["mixed_384"] = precision
        if fas is not None:
            line["fas"] = fas
        if amr is not None:
            line["amr_level"] = amr
        if sharded is not None:
            line["amr_level_sharded"] = sharded
        if serving is not None:
            line["serving"] = serving
        if iters != GPU_CYCLES_PER_SOLVE:
            line["note"] = "cycles per solve %d differ from the %d the reference arm assumes when it runs too few " \
                           "cycles to converge" % (iters, GPU_CYCLES_PER_SOLVE)
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_reference_cycles(1, 2, gpu_cycles=iters)
            except Exception as e:  # the baseline never hides the GPU result
                line["cpu_baseline"] = {"error": str(e)}
        # the short sections last (a log that keeps only the end of the line keeps them)
        line["stencil"] = {"metric": "Stencil::apply 7-point FP64 256^3 GB/s", "value": st_gbs, "unit": "GB/s",
                           "frac_of_hbm": st_gbs / peak, "us_per_apply": t_st * 1e6,
                           "gpts_per_s": 256 ** 3 / t_st / 1e9, "algorithmic_bytes": STENCIL_BYTES,
                           "traffic": traffic.get("k_star_tma_apply_f64_256")}
        line["mixed"] = {"metric": "MG solves/s, FP32 cycles with FP64 residual/correction", "value": value_m,
                         "unit": "solves/s", "speedup_vs_fp64": value_m / value, "iters_per_solve": itm,
                         "final_rel_residual": histm[-1] / histm[0], "max_rel_err_vs_fp64_solution": err_m,
                         "latency_ms": {"p50": lat_m[len(lat_m) // 2],
                                        "p99": lat_m[min(len(lat_m) - 1, int(0.99 * len(lat_m)))]},
                         "relax_fp32_us": t_rx32 * 1e6, "relax_fp32_frac": 12 * 256 ** 3 / t_rx32 / 1e9 / peak,
                         "relax2_fp32_us": t_rx32_2 * 1e6, "relax2_fp32_frac": 12 * 256 ** 3 / t_rx32_2 / 1e9 / peak,
                         "gpu_launches": (2 + itm * mgm.launches_per_cycle() + 1) * args.steps}
        line["relax_single_sweep"] = {"kernel": "k_star_tma<Lap7,double,EpiRelax> (one Jacobi sweep, 256^3)",
                                      "us_per_launch": t_rx * 1e6, "achieved_gbs": rx_gbs, "frac": rx_gbs / peak,
                                      "algorithmic_bytes_per_launch": RELAX_BYTES,
                                      "traffic": traffic.get("k_star_tma_relax_f64_256")}
        line["roofline"] = {"bound": "hbm", "kernel": "k_relax2<double,256> (two finest-level Jacobi sweeps per pass)",
                            "achieved": rx2_gbs, "peak": peak,
                            "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)", "unit": "GB/s",
                            "frac": rx2_gbs / peak, "traffic": traffic.get("k_relax2_f64_256"),
                            "algorithmic_bytes_per_launch": RELAX_BYTES, "us_per_launch": t_rx2 * 1e6,
                            "sweeps_per_launch": 2}
        line["e2e"] = {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": 8 * N ** 3,
                       "d2h_bytes_per_step": 8 * N ** 3}
        line["clocks"] = clk
        line["gpu_launches"] = launches * args.steps
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
