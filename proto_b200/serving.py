"""Serving workload: a seeded stream of periodic Poisson/Helmholtz requests and two ways to serve it.

  make_trace      arrivals of a Poisson process (rate per second), grid edge log-uniform in
                  [lo, hi] rounded to a multiple of 16, Poisson or Helmholtz form with equal odds,
                  alpha ~ U[0, 1] (Helmholtz, beta = 1), right-hand side = 4 sine modes (one of a
                  few seeded variants per edge), tolerance on the relative max-norm residual.
  serve_trace     the serving engine (pb_serve): requests join the in-flight batch as they arrive.
  fp64_trace      the plain FP64 multigrid (pb_mg), one request at a time in arrival order.

Both replay the trace open loop against the wall clock (realtime=True) or with every request
available at the start (realtime=False, saturated throughput). Latency is arrival -> result in host
memory. All inputs are synthetic and seeded; nothing is read from disk.
"""
import math
import time

import numpy as np

from . import workloads as W

VARIANTS = 2


def make_trace(count=2000, rate=200.0, seed=4, lo=32, hi=192, step=16, helm_share=0.5):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrive = np.concatenate([[0.0], np.cumsum(gaps[1:])])
    edge = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))
    edge = np.clip(np.round(edge / step) * step, lo, hi).astype(int)
    helm = rng.random(count) < helm_share
    alpha = rng.uniform(0.0, 1.0, size=count)
    variant = rng.integers(0, VARIANTS, size=count)
    return [dict(i=i, t=float(arrive[i]), n=int(edge[i]), helm=bool(helm[i]), alpha=float(alpha[i]) if helm[i] else 0.0,
                 variant=int(variant[i])) for i in range(count)]


def pinned(count):
    """A page-locked float64 host array (fast host<->device copies for both serving paths)."""
    import torch
    return torch.empty(count, dtype=torch.float64).pin_memory().numpy()


def rhs_pool(edges, seed=5):
    """Right-hand sides by (edge, variant, form): f = 4 sine modes, mean removed; the Poisson form
    solves L u = -f (the reference multigrid's sign), the Helmholtz form alpha u - L u = f."""
    pool = {}
    for n in sorted(set(edges)):
        for v in range(VARIANTS):
            f = W.sine_modes_rhs(n, seed=seed * 1000 + 7 * n + v, modes=4).reshape(-1)
            for helm, arr in ((True, f), (False, -f)):
                buf = pinned(n ** 3)
                buf[:] = arr
                pool[(n, v, helm)] = buf
    return pool


class _Ring:
    """A few reusable host result buffers per edge."""

    def __init__(self, edges, per_edge):
        self.free = {n: [pinned(n ** 3) for _ in range(per_edge)] for n in sorted(set(edges))}

    def take(self, n):
        return self.free[n].pop() if self.free[n] else None

    def give(self, n, buf):
        self.free[n].append(buf)


def _summary(lat, t_end, count, extra=None):
    lat = np.sort(np.asarray(lat))
    out = {"solves": count, "solves_per_s": count / t_end if t_end > 0 else float("nan"),
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "max_ms": float(lat[-1] * 1e3), "makespan_s": t_end}
    if extra:
        out.update(extra)
    return out


def serve_trace(pb, trace, pool, realtime=True, hbm_budget=150 << 30, max_active=64, tol=1e-8, keep=0,
                per_edge=12, engine=None, ring=None, **kw):
    """Replays the trace through pb_serve. keep: results of the first `keep` requests are returned.
    engine / ring: an existing engine (its hierarchies stay cached between replays) and result
    buffers to reuse."""
    sv = engine if engine is not None else pb.Serve(hbm_budget, max_active=max_active, tol=tol, **kw)
    max_active = sv.params.max_active
    ring = ring if ring is not None else _Ring([r["n"] for r in trace], per_edge)
    pending, lat, cycles, kept = {}, [], [], {}
    worst = 0.0
    i, n_req = 0, len(trace)
    t0 = time.perf_counter()
    while i < n_req or pending:
        now = time.perf_counter() - t0
        while i < n_req and (not realtime or trace[i]["t"] <= now):
            r = trace[i]
            buf = ring.take(r["n"])
            if buf is None:
                break
            rhs = pool[(r["n"], r["variant"], r["helm"])]
            tk = sv.submit(r["n"], rhs, buf, form=pb.MG_HELMHOLTZ if r["helm"] else pb.MG_POISSON, alpha=r["alpha"])
            pending[tk] = (r, buf)
            i += 1
        if not pending:
            if i < n_req:
                time.sleep(max(0.0, min(0.002, trace[i]["t"] - now)))
            continue
        sv.step()
        done_t = time.perf_counter() - t0
        for tk in sv.poll():
            r, buf = pending.pop(tk)
            st, cy, rr = sv.status(tk)
            if st != pb.SERVE_DONE:
                raise RuntimeError("serve: request %d ended in state %d" % (r["i"], st))
            lat.append(done_t - (r["t"] if realtime else 0.0))
            cycles.append(cy)
            worst = max(worst, rr)
            if r["i"] < keep:
                kept[r["i"]] = buf.copy()
            ring.give(r["n"], buf)
    t_end = time.perf_counter() - t0
    pb.device_check()
    return _summary(lat, t_end, n_req, {"mean_cycles": float(np.mean(cycles)), "max_rel_residual": worst,
                                        "max_active": max_active}), kept


def fp64_trace(pb, trace, pool, realtime=True, tol=1e-8, keep=0, nu=4, nu_bottom=10, omega=2.0 / 3.0):
    """Replays the trace through one FP64 pb_mg solver per (edge, form), one request at a time."""
    import torch

    def halvings(n):
        k = 0
        while n % 2 == 0 and n > 1:
            n //= 2
            k += 1
        return k

    solvers = {}
    for r in trace:
        key = (r["n"], r["helm"])
        if key not in solvers:
            p = pb.MGParams(n=r["n"], levels=halvings(r["n"]), nu1=nu, nu2=nu, nu_bottom=nu_bottom, omega=omega,
                            max_iter=100, tol=tol, form=pb.MG_HELMHOLTZ if r["helm"] else pb.MG_POISSON)
            solvers[key] = (pb.Multigrid(p), torch.empty(r["n"] ** 3, dtype=torch.float64, device="cuda"),
                            torch.empty(r["n"] ** 3, dtype=torch.float64, device="cuda"),
                            torch.empty(r["n"] ** 3, dtype=torch.float64, device="cuda"),
                            torch.from_numpy(pinned(r["n"] ** 3)))
    lat, cycles, kept = [], [], {}
    worst = 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in trace:
        if realtime:
            while time.perf_counter() - t0 < r["t"]:
                pass
        mg, rhs_d, phi_d, alpha_d, out_h = solvers[(r["n"], r["helm"])]
        rhs_d.copy_(torch.from_numpy(pool[(r["n"], r["variant"], r["helm"])]))
        if r["helm"]:
            alpha_d.fill_(r["alpha"])
            mg.set_alpha(alpha_d)
        phi_d.zero_()
        it, hist = mg.solve(rhs_d, phi_d)
        out_h.copy_(phi_d)
        out = out_h.numpy()
        lat.append(time.perf_counter() - t0 - (r["t"] if realtime else 0.0))
        cycles.append(it)
        worst = max(worst, hist[-1] / hist[0])
        if r["i"] < keep:
            kept[r["i"]] = out.copy()
    t_end = time.perf_counter() - t0
    return _summary(lat, t_end, len(trace), {"mean_cycles": float(np.mean(cycles)), "max_rel_residual": worst}), kept
