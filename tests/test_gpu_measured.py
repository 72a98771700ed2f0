"""The bench's measured configurations checked against the CPU oracle at their own sizes.

* The headline solve: 256^3 periodic Poisson, V(4,4), omega = 2/3, 10 bottom sweeps on 4^3, to a
  1e-10 relative max-norm residual: every cycle's residual and the final solution bitwise the C
  restatement's (which is pinned bitwise to the reference's own solver on smaller grids).
* Odd coarsest grids (3^3, the shape of the 384^3 mixed-precision configuration) with the exact
  bottom solve, Poisson and per-cell-alpha Helmholtz, at 48^3 and 96^3: bitwise.
* Mixed precision on a 3^3-coarsest hierarchy: the FP64 residual reaches 1e-10 and the solution
  stays within 1e-7 relative of the FP64 solver's.
* The 512-patch AMR level for the bench's full 100 graph steps with autotuned tiles: bitwise the
  C restatement's periodic stepping (the configuration's own bar is 1e-13 relative).
"""
import numpy as np
import pytest

from proto_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _gpu(pb, N, levels, nu, nub, max_iter, tol, precision=0, alpha=None, rhs=None, bottom=0):
    import torch
    p = pb.MGParams(n=N, levels=levels, nu1=nu, nu2=nu, nu_bottom=nub, omega=2.0 / 3.0, max_iter=max_iter, tol=tol,
                    form=pb.MG_HELMHOLTZ if alpha is not None else pb.MG_POISSON, precision=precision,
                    bottom=bottom)
    mg = pb.Multigrid(p)
    if alpha is not None:
        mg.set_alpha(torch.from_numpy(alpha.reshape(-1).copy()).cuda())
    r = torch.from_numpy(rhs.reshape(-1).copy()).cuda()
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(r, phi)
    pb.device_check()
    return it, hist, phi.cpu().numpy()


def test_headline_256_solve_bitwise(pb, port):
    N, lev = 256, 6
    rho = W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu(pb, N, lev, 4, 10, 100, 1e-10, rhs=rho)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None, 100, 1e-10, rho.reshape(-1).copy(), p2)
    assert it == n2 == 16
    assert hist == list(h2)
    assert hist[-1] < 1e-10 * hist[0]
    assert np.array_equal(phi, p2)


@pytest.mark.parametrize("N,lev", [(48, 4), (96, 5)])
@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_odd_coarsest_direct_bottom_bitwise(pb, port, N, lev, form):
    assert N >> lev == 3
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    rhs = -W.poisson_rho(N, seed=1) if alpha is not None else W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu(pb, N, lev, 4, 10, 30, 1e-10, alpha=alpha, rhs=rhs, bottom=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None if alpha is None else alpha.reshape(-1).copy(), 30,
                        1e-10, rhs.reshape(-1).copy(), p2, bottom=1)
    assert it == n2 and hist == list(h2)
    assert hist[-1] < 1e-10 * hist[0]
    assert np.array_equal(phi, p2)


@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_mixed_precision_odd_coarsest(pb, form):
    N, lev = 96, 5
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    rhs = -W.poisson_rho(N, seed=1) if alpha is not None else W.poisson_rho(N, seed=1)
    it64, h64, phi64 = _gpu(pb, N, lev, 4, 10, 30, 1e-10, alpha=alpha, rhs=rhs, bottom=1)
    itm, hm, phim = _gpu(pb, N, lev, 4, 10, 30, 1e-10, precision=pb.MG_MIXED, alpha=alpha, rhs=rhs, bottom=1)
    assert hm[0] == h64[0]
    assert hm[-1] < 1e-10 * hm[0]
    assert itm <= it64 + 2
    assert np.max(np.abs(phim - phi64)) / np.max(np.abs(phi64)) < 1e-7


def test_amr_level_100_steps_against_port(golden, pb, port):
    import torch
    from tests.test_gpu_level import _level13
    widths = W.amr_widths(seed=2)
    lv, S, (c, o), u, a, L = _level13(golden, pb, widths, 7)
    assert len(lv.patches) == 512
    h = 1.0 / L[0]
    b = torch.zeros_like(a)
    lv.autotune(S, a, b, scale=1.0 / (h * h))
    lv.steps(S, pb.EPI_EULER, a, b, 100, scale=1.0 / (h * h), a=0.1 * h * h)
    torch.cuda.synchronize()
    pb.device_check()
    got = a.cpu().numpy()
    gh = 2
    G = np.zeros((L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh))
    G[gh:-gh, gh:-gh, gh:-gh] = u
    G = G.reshape(-1).copy()
    port.periodic_steps(L, gh, c, o.reshape(-1), h, 0.1 * h * h, 100, G)
    ref = G.reshape(L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh)[gh:-gh, gh:-gh, gh:-gh]
    out = np.zeros_like(u)
    for p, off in zip(lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * gh for d in (2, 1, 0))
        blk = got[off:off + int(np.prod(shp))].reshape(shp)[gh:-gh, gh:-gh, gh:-gh]
        out[p.lo[2]:p.hi[2] + 1, p.lo[1]:p.hi[1] + 1, p.lo[0]:p.hi[0] + 1] = blk
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.array_equal(out, ref)
