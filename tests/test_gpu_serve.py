"""Serving engine on the GPU: per-solve results bitwise equal to the single-solve mixed-precision
solver, the same alone and in a mix, under a memory budget, and close to the FP64 oracle."""
import numpy as np
import pytest

from proto_b200 import workloads as W

pytestmark = pytest.mark.gpu

BIG = 8 << 30


def halvings(n):
    k = 0
    while n % 2 == 0 and n > 1:
        n //= 2
        k += 1
    return k


def requests():
    """(n, form, alpha, rhs): Poisson and Helmholtz, edges whose hierarchies end on 1 and 5, and
    non-dyadic alphas (their coarse-level averages round)."""
    out = []
    for i, (n, helm, a) in enumerate([(32, 0, 0.0), (48, 1, 0.37), (64, 1, 0.9), (80, 0, 0.0), (40, 1, 0.05),
                                      (16, 1, 0.7)]):
        f = W.sine_modes_rhs(n, seed=10 + i, modes=4)
        rhs = (f if helm else -f).reshape(-1).copy()
        out.append((n, helm, a, rhs))
    return out


def serve(pb, reqs, **kw):
    sv = pb.Serve(kw.pop("budget", BIG), **kw)
    outs, tickets = [], []
    for n, helm, a, rhs in reqs:
        o = np.zeros(n ** 3)
        tickets.append(sv.submit(n, rhs, o, form=pb.MG_HELMHOLTZ if helm else pb.MG_POISSON, alpha=a))
        outs.append(o)
    peak = held = 0
    for _ in range(1000):
        act, wait = sv.step()
        peak = max(peak, act)
        held = max(held, sv.device_bytes())
        if act == 0 and wait == 0:
            break
    stats = [sv.status(t) for t in tickets]
    pb.device_check()
    serve.held = held
    return outs, stats, peak


def single_mixed(pb, n, helm, a, rhs):
    import torch
    p = pb.MGParams(n=n, levels=halvings(n), nu1=4, nu2=4, nu_bottom=10, omega=2.0 / 3.0, max_iter=100, tol=1e-8,
                    form=pb.MG_HELMHOLTZ if helm else pb.MG_POISSON, precision=pb.MG_MIXED)
    mg = pb.Multigrid(p)
    if helm:
        mg.set_alpha(torch.full((n ** 3,), a, dtype=torch.float64, device="cuda"))
    phi = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(torch.from_numpy(rhs).cuda(), phi)
    return it, hist, phi.cpu().numpy()


def test_served_equals_single_mixed_solver(pb):
    reqs = requests()
    outs, stats, _ = serve(pb, reqs)
    for (n, helm, a, rhs), o, (state, cycles, rel) in zip(reqs, outs, stats):
        assert state == pb.SERVE_DONE
        it, hist, phi = single_mixed(pb, n, helm, a, rhs)
        assert cycles == it
        assert rel == hist[-1] / hist[0]
        assert np.array_equal(o, phi), (n, helm)


def test_alone_and_in_the_mix_are_identical(pb):
    reqs = requests()
    mix, _, peak = serve(pb, reqs)
    assert peak == len(reqs)
    for r, m in zip(reqs, mix):
        alone, _, _ = serve(pb, [r])
        assert np.array_equal(alone[0], m)


def test_budget_limits_admission(pb):
    """Hierarchies held never exceed the budget; solves wait until memory frees up."""
    reqs = requests()
    sizes = [pb.Serve.request_bytes(n) for n, _, _, _ in reqs]
    budget = int(max(sizes) * 1.1)
    assert sum(sizes) > budget
    outs, stats, peak = serve(pb, reqs, budget=budget)
    assert serve.held <= budget
    assert 1 <= peak < len(reqs)
    ref, _, _ = serve(pb, reqs)
    for o, r, (state, _, _) in zip(outs, ref, stats):
        assert state == pb.SERVE_DONE
        assert np.array_equal(o, r)


def test_slot_limit_and_reuse(pb):
    reqs = requests() * 2
    outs, stats, peak = serve(pb, reqs, max_active=3)
    assert peak == 3
    for (state, _, _) in stats:
        assert state == pb.SERVE_DONE
    half = len(reqs) // 2
    for a, b in zip(outs[:half], outs[half:]):
        assert np.array_equal(a, b)


def test_error_against_fp64_oracle(pb, port):
    """Served (FP32 cycles, FP64 refinement) vs the FP64 CPU oracle run to the same tolerance."""
    reqs = requests()[:3]
    outs, stats, _ = serve(pb, reqs)
    for (n, helm, a, rhs), o in zip(reqs, outs):
        ref = np.zeros(n ** 3)
        alpha = np.full(n ** 3, a) if helm else None
        port.mg_cs(n, halvings(n), 4, 4, 10, 2.0 / 3.0, 1.0, alpha, 100, 1e-8, rhs.copy(), ref)
        err = np.max(np.abs(o - ref)) / np.max(np.abs(ref))
        assert err < 1e-6, (n, helm, err)


def test_failed_requests_leave_the_others_unchanged(pb):
    """Failure paths of the engine, made on the host: a right-hand side holding a NaN fails at its
    first residual pass (the norm reports a non-finite residual); a zero right-hand side never meets
    res < tol * res0 (res0 = 0) and fails after max_cycles. Every other solve in the same batch
    completes with bitwise the result it has alone."""
    reqs = requests()
    n = 32
    nan_rhs = reqs[0][3].copy()
    nan_rhs[n ** 3 // 2 + 7] = np.nan
    zero_rhs = np.zeros(n ** 3)
    mix = reqs[:3] + [(n, 0, 0.0, nan_rhs)] + reqs[3:] + [(n, 1, 0.5, zero_rhs)]
    outs, stats, _ = serve(pb, mix, max_cycles=40)
    nan_state, nan_cycles, _ = stats[3]
    assert nan_state == pb.SERVE_FAILED and nan_cycles == 1
    zero_state, zero_cycles, _ = stats[-1]
    assert zero_state == pb.SERVE_FAILED and zero_cycles == 40
    good = [i for i in range(len(mix)) if i not in (3, len(mix) - 1)]
    alone, astats, _ = serve(pb, [mix[i] for i in good], max_cycles=40)
    for k, i in enumerate(good):
        assert stats[i][0] == pb.SERVE_DONE and astats[k][0] == pb.SERVE_DONE
        assert stats[i][1] == astats[k][1]
        assert np.array_equal(outs[i], alone[k])
