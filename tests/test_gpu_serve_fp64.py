"""The serving engine with every level in FP64 (precision PB_MG_FP64): per-solve results bitwise
equal to the single-solve FP64 solver and to the C restatement of the reference's multigrid, the same
alone and in a mix, with failed requests isolated."""
import numpy as np
import pytest

from test_gpu_serve import halvings, requests, serve
from proto_b200 import workloads as W

pytestmark = pytest.mark.gpu


def requests_fp64():
    """The mixed engine's requests plus a 128^3 Helmholtz solve, whose single-solve counterpart runs
    its finest level through the two-sweep passes and the staged restriction."""
    f = W.sine_modes_rhs(128, seed=21, modes=4)
    return requests() + [(128, 1, 0.37, f.reshape(-1).copy())]


def serve64(pb, reqs, **kw):
    return serve(pb, reqs, precision=pb.MG_FP64, **kw)


def single_fp64(pb, n, helm, a, rhs, tol=1e-8):
    import torch
    p = pb.MGParams(n=n, levels=halvings(n), nu1=4, nu2=4, nu_bottom=10, omega=2.0 / 3.0, max_iter=100, tol=tol,
                    form=pb.MG_HELMHOLTZ if helm else pb.MG_POISSON, precision=pb.MG_FP64)
    mg = pb.Multigrid(p)
    if helm:
        mg.set_alpha(torch.full((n ** 3,), a, dtype=torch.float64, device="cuda"))
    phi = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(torch.from_numpy(rhs).cuda(), phi)
    return it, hist, phi.cpu().numpy()


def test_served_fp64_equals_single_fp64_solver(pb):
    reqs = requests_fp64()
    outs, stats, peak = serve64(pb, reqs)
    assert peak == len(reqs)
    for (n, helm, a, rhs), o, (state, cycles, rel) in zip(reqs, outs, stats):
        assert state == pb.SERVE_DONE
        it, hist, phi = single_fp64(pb, n, helm, a, rhs)
        assert cycles == it, (n, helm)
        assert rel == hist[-1] / hist[0], (n, helm)
        assert np.array_equal(o, phi), (n, helm)


def test_served_fp64_equals_the_oracle(pb, port):
    """Bitwise the C restatement's solve of the reference's multigrid (cycle count and solution)."""
    for n, helm, a, rhs in requests()[:3]:
        (o,), ((state, cycles, _),), _ = serve64(pb, [(n, helm, a, rhs)])
        assert state == pb.SERVE_DONE
        ref = np.zeros(n ** 3)
        alpha = np.full(n ** 3, a) if helm else None
        n2, _ = port.mg_cs(n, halvings(n), 4, 4, 10, 2.0 / 3.0, 1.0, alpha, 100, 1e-8, rhs.copy(), ref)
        assert cycles == n2, (n, helm)
        assert np.array_equal(o, ref), (n, helm)


def test_fp64_alone_and_in_the_mix_are_identical(pb):
    reqs = requests()
    mix, _, _ = serve64(pb, reqs, max_active=4)
    for r, m in zip(reqs, mix):
        alone, _, _ = serve64(pb, [r])
        assert np.array_equal(alone[0], m)


def test_fp64_tighter_tolerance(pb):
    """At 1e-10 the served FP64 solve still takes the single solver's cycles and solution."""
    n, helm, a, rhs = requests()[1]
    (o,), ((state, cycles, _),), _ = serve64(pb, [(n, helm, a, rhs)], tol=1e-10)
    it, _, phi = single_fp64(pb, n, helm, a, rhs, tol=1e-10)
    assert state == pb.SERVE_DONE and cycles == it
    assert np.array_equal(o, phi)


def test_fp64_failed_requests_leave_the_others_unchanged(pb):
    """A NaN in a right-hand side fails at the first norm pass; a zero right-hand side (res0 = 0)
    fails after max_cycles; the other solves of the batch keep the results they have alone."""
    reqs = requests()
    n = 32
    nan_rhs = reqs[0][3].copy()
    nan_rhs[n ** 3 // 3] = np.nan
    mix = reqs[:2] + [(n, 1, 0.5, nan_rhs), (n, 0, 0.0, np.zeros(n ** 3))] + reqs[2:]
    outs, stats, _ = serve64(pb, mix, max_cycles=30)
    assert stats[2][0] == pb.SERVE_FAILED and stats[2][1] == 1
    assert stats[3][0] == pb.SERVE_FAILED and stats[3][1] == 30
    good = [i for i in range(len(mix)) if i not in (2, 3)]
    alone, astats, _ = serve64(pb, [mix[i] for i in good], max_cycles=30)
    for k, i in enumerate(good):
        assert stats[i][0] == pb.SERVE_DONE and astats[k] == stats[i]
        assert np.array_equal(outs[i], alone[k])
