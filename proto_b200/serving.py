"""Serving workload: a seeded stream of periodic Poisson/Helmholtz requests and three ways to serve it.

  make_trace      arrivals of a Poisson process (rate per second), grid edge log-uniform in
                  [lo, hi] rounded to a multiple of 16, Poisson or Helmholtz form with equal odds,
                  alpha ~ U[0, 1] (Helmholtz, beta = 1), a right-hand side of 4 sine modes per request
                  (its own seed), tolerance on the relative max-norm residual.
  TraceData       every request's right-hand side and a result slot, in two page-locked host arrays.
  serve_trace     the serving engine (pb_serve, mixed precision or FP64): requests join the in-flight
                  batch as they arrive.
  single_trace    plain multigrid (pb_mg, FP64 or mixed precision), one request at a time in arrival
                  order: the FP64 arm is the baseline, the mixed arm separates what precision gains
                  from what batching gains.
  verify          every served (or single-solve) result against the FP64 solver's solution of the same
                  request at the same tolerance (the FP64 GPU solver performs the CPU oracle's
                  arithmetic bit for bit), one relative max-norm error per request.

Replays run open loop against the wall clock (realtime=True) or with every request available at the
start (realtime=False, saturated throughput). Latency is arrival -> result in host memory. All inputs
are synthetic and seeded; nothing is read from disk.
"""
import math
import time

import numpy as np

from . import workloads as W


def make_trace(count=2000, rate=200.0, seed=4, lo=32, hi=192, step=16, helm_share=0.5):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrive = np.concatenate([[0.0], np.cumsum(gaps[1:])])
    edge = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))
    edge = np.clip(np.round(edge / step) * step, lo, hi).astype(int)
    helm = rng.random(count) < helm_share
    alpha = rng.uniform(0.0, 1.0, size=count)
    return [dict(i=i, t=float(arrive[i]), n=int(edge[i]), helm=bool(helm[i]), alpha=float(alpha[i]) if helm[i] else 0.0,
                 seed=int(seed * 100000 + i)) for i in range(count)]


def pinned(count):
    """A page-locked float64 host array (fast host<->device copies for every serving path)."""
    import torch
    return torch.empty(count, dtype=torch.float64, pin_memory=True).numpy()


_REGISTERED = []


def pinned_large(count):
    """A large float64 host array, page-locked in place (cudaHostRegister) rather than through the
    caching host allocator, which may round a large request up. It stays registered until exit."""
    import torch
    a = np.empty(count, dtype=np.float64)
    rc = torch.cuda.cudart().cudaHostRegister(a.ctypes.data, a.nbytes, 0)
    if int(rc) != 0:
        raise RuntimeError("cudaHostRegister failed (%s)" % (rc,))
    _REGISTERED.append(a)
    return a


class TraceData:
    """Right-hand sides of every request of a trace (f = 4 sine modes from the request's seed, mean
    removed; the Poisson form solves L u = -f in the reference multigrid's sign, the Helmholtz form
    alpha u - L u = f) and one result slot per request, each in one page-locked host array. The
    right-hand sides are evaluated on the GPU and copied down once, before any timed region."""

    def __init__(self, trace):
        import torch
        sizes = [r["n"] ** 3 for r in trace]
        self.off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.rhs = pinned_large(int(self.off[-1]))
        self.out = pinned_large(int(self.off[-1]))
        host = torch.from_numpy(self.rhs)
        for r in trace:
            a, b = int(self.off[r["i"]]), int(self.off[r["i"] + 1])
            f = W.sine_modes_rhs_device(r["n"], r["seed"], modes=4).reshape(-1)
            host[a:b].copy_(f if r["helm"] else -f)
        torch.cuda.synchronize()

    def rhs_of(self, i):
        return self.rhs[self.off[i]:self.off[i + 1]]

    def out_of(self, i):
        return self.out[self.off[i]:self.off[i + 1]]

    @property
    def nbytes(self):
        return int(self.off[-1]) * 8


def _summary(lat, t_end, count, extra=None):
    lat = np.sort(np.asarray(lat))
    out = {"solves": count, "solves_per_s": count / t_end if t_end > 0 else float("nan"),
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "max_ms": float(lat[-1] * 1e3), "makespan_s": t_end}
    if extra:
        out.update(extra)
    return out


def serve_trace(pb, trace, data, realtime=True, engine=None, hbm_budget=150 << 30, max_active=64, tol=1e-8, **kw):
    """Replays the trace through pb_serve (an existing engine keeps its hierarchies cached between
    replays); each result lands in the request's slot of data.out."""
    sv = engine if engine is not None else pb.Serve(hbm_budget, max_active=max_active, tol=tol, **kw)
    pending, lat, cycles = {}, [], []
    worst = 0.0
    i, n_req = 0, len(trace)
    t0 = time.perf_counter()
    while i < n_req or pending:
        now = time.perf_counter() - t0
        while i < n_req and (not realtime or trace[i]["t"] <= now):
            r = trace[i]
            tk = sv.submit(r["n"], data.rhs_of(r["i"]), data.out_of(r["i"]),
                           form=pb.MG_HELMHOLTZ if r["helm"] else pb.MG_POISSON, alpha=r["alpha"])
            pending[tk] = r
            i += 1
        if not pending:
            if i < n_req:
                time.sleep(max(0.0, min(0.002, trace[i]["t"] - now)))
            continue
        sv.step()
        done_t = time.perf_counter() - t0
        for tk in sv.poll():
            r = pending.pop(tk)
            st, cy, rr = sv.status(tk)
            if st != pb.SERVE_DONE:
                raise RuntimeError("serve: request %d ended in state %d" % (r["i"], st))
            lat.append(done_t - (r["t"] if realtime else 0.0))
            cycles.append(cy)
            worst = max(worst, rr)
    t_end = time.perf_counter() - t0
    pb.device_check()
    return _summary(lat, t_end, n_req, {"mean_cycles": float(np.mean(cycles)), "max_rel_residual": worst,
                                        "max_active": sv.params.max_active})


def halvings(n):
    k = 0
    while n % 2 == 0 and n > 1:
        n //= 2
        k += 1
    return k


class SingleSolvers:
    """One pb_mg solver per (edge, form) of a trace, with device buffers for one request."""

    def __init__(self, pb, trace, tol, precision, nu=4, nu_bottom=10, omega=2.0 / 3.0):
        import torch
        self.s = {}
        for r in trace:
            key = (r["n"], r["helm"])
            if key not in self.s:
                p = pb.MGParams(n=r["n"], levels=halvings(r["n"]), nu1=nu, nu2=nu, nu_bottom=nu_bottom, omega=omega,
                                max_iter=100, tol=tol, form=pb.MG_HELMHOLTZ if r["helm"] else pb.MG_POISSON,
                                precision=precision)
                n3 = r["n"] ** 3
                self.s[key] = (pb.Multigrid(p), torch.empty(n3, dtype=torch.float64, device="cuda"),
                               torch.empty(n3, dtype=torch.float64, device="cuda"),
                               torch.empty(n3, dtype=torch.float64, device="cuda"))

    def solve(self, r, rhs_host, out_host=None):
        """H2D of the right-hand side, the solve, D2H of the solution (when out_host is given); the
        solution stays in the returned device buffer."""
        import torch
        mg, rhs_d, phi_d, alpha_d = self.s[(r["n"], r["helm"])]
        rhs_d.copy_(torch.from_numpy(rhs_host), non_blocking=True)
        if r["helm"]:
            alpha_d.fill_(r["alpha"])
            mg.set_alpha(alpha_d)
        phi_d.zero_()
        it, hist = mg.solve(rhs_d, phi_d)
        if out_host is not None:
            torch.from_numpy(out_host).copy_(phi_d)
        return it, hist, phi_d


def single_trace(pb, trace, data, solvers, realtime=True):
    """Replays the trace through plain multigrid solvers, one request at a time in arrival order."""
    import torch
    lat, cycles = [], []
    worst = 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in trace:
        if realtime:
            while time.perf_counter() - t0 < r["t"]:
                pass
        it, hist, _ = solvers.solve(r, data.rhs_of(r["i"]), data.out_of(r["i"]))
        lat.append(time.perf_counter() - t0 - (r["t"] if realtime else 0.0))
        cycles.append(it)
        worst = max(worst, hist[-1] / hist[0])
    t_end = time.perf_counter() - t0
    return _summary(lat, t_end, len(trace), {"mean_cycles": float(np.mean(cycles)), "max_rel_residual": worst})


def verify(pb, trace, data, fp64):
    """Relative max-norm error of every result in data.out against the FP64 solver's solution of the
    same request: max |out - ref| / max |ref| per request; and the same with each field's mean
    removed first, since a periodic Poisson solution is defined up to a constant (and a Helmholtz
    one with a small alpha only weakly fixes it). Returns max, p99 and median of both, and how many
    results are bitwise the FP64 solver's."""
    import torch
    errs = np.zeros(len(trace))
    errs0 = np.zeros(len(trace))
    same = 0
    for r in trace:
        _, _, ref = fp64.solve(r, data.rhs_of(r["i"]))
        got = torch.from_numpy(data.out_of(r["i"])).to("cuda", non_blocking=True)
        same += int(torch.equal(got, ref))
        errs[r["i"]] = float((got - ref).abs().max() / ref.abs().max())
        ref0 = ref - ref.mean()
        errs0[r["i"]] = float(((got - got.mean()) - ref0).abs().max() / ref0.abs().max())

    def stats(e):
        return {"max": float(e.max()), "p99": float(np.percentile(e, 99)), "median": float(np.median(e))}
    return {"requests": len(trace), "bitwise_equal": same, "rel_err": stats(errs), "rel_err_mean_removed": stats(errs0)}
