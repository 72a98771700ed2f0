"""Multigrid on the GPU: residual histories bitwise equal to the reference CPU path."""
import numpy as np
import pytest

from proto_b200 import workloads as W
from tests.util import digest

pytestmark = pytest.mark.gpu


def _solve(pb, cfg, alpha=None, rhs=None):
    import torch
    N = cfg["N"]
    if cfg["kind"] == "archived":
        p = pb.MGParams(n=N, levels=cfg["numLevels"], nu1=6, nu2=6, nu_bottom=10, omega=0.5,
                        max_iter=cfg["maxIter"], tol=cfg["tol"])
    else:
        p = pb.MGParams(n=N, levels=cfg["levels"], nu1=cfg["nu1"], nu2=cfg["nu2"], nu_bottom=cfg["nub"],
                        omega=cfg["omega"], max_iter=cfg["maxIter"], tol=cfg["tol"],
                        form=pb.MG_HELMHOLTZ if alpha is not None else pb.MG_POISSON)
    mg = pb.Multigrid(p)
    rho = W.poisson_rho(N, seed=1) if rhs is None else rhs
    if alpha is not None:
        mg.set_alpha(torch.from_numpy(alpha.reshape(-1).copy()).cuda())
    r = torch.from_numpy(rho.reshape(-1).copy()).cuda()
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(r, phi)
    pb.device_check()
    return it, hist, phi.cpu().numpy()


@pytest.mark.parametrize("name", ["archived_32", "cs_v22_32", "cs_v22_64"])
def test_poisson_history_bitwise(golden, pb, name):
    cfg = golden[0]["mg"][name]
    it, hist, phi = _solve(pb, cfg)
    assert it == cfg["iters"]
    assert hist == cfg["hist"]
    assert digest(phi) == cfg["phi_sha256"]


def test_helmholtz_history_bitwise(golden, pb):
    cfg = golden[0]["mg"]["helm_v22_32"]
    alpha = W.helmholtz_alpha(cfg["N"], seed=3)
    it, hist, phi = _solve(pb, cfg, alpha=alpha, rhs=-W.poisson_rho(cfg["N"], seed=1))
    assert it == cfg["iters"]
    assert hist == cfg["hist"]
    assert digest(phi) == cfg["phi_sha256"]


def test_large_grid_against_port(pb, port):
    """128^3, V(4,4): the TMA relax kernel on the fine levels, history bitwise vs the C port."""
    N, lev = 128, 5
    rho = W.poisson_rho(N, seed=1)
    cfg = dict(kind="cs", N=N, levels=lev, nu1=4, nu2=4, nub=10, omega=2.0 / 3.0, maxIter=6, tol=1e-10)
    it, hist, phi = _solve(pb, cfg)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None, 6, 1e-10, rho.reshape(-1).copy(), p2)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi, p2)


def _gpu_solve(pb, N, levels, precision, nu=4, max_iter=60, tol=1e-10, alpha=None, rhs=None, nub=10, bottom=0):
    import torch
    p = pb.MGParams(n=N, levels=levels, nu1=nu, nu2=nu, nu_bottom=nub, omega=2.0 / 3.0, max_iter=max_iter, tol=tol,
                    form=pb.MG_HELMHOLTZ if alpha is not None else pb.MG_POISSON, precision=precision,
                    bottom=bottom)
    mg = pb.Multigrid(p)
    if alpha is not None:
        mg.set_alpha(torch.from_numpy(alpha.reshape(-1).copy()).cuda())
    rho = W.poisson_rho(N, seed=1) if rhs is None else rhs
    r = torch.from_numpy(rho.reshape(-1).copy()).cuda()
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(r, phi)
    pb.device_check()
    return it, hist, phi.cpu().numpy()


@pytest.mark.parametrize("N,levels", [(64, 4), (128, 5)])
def test_mixed_precision_reaches_tolerance(pb, N, levels):
    """FP32 V-cycles inside FP64 residual/correction: the FP64 residual reaches 1e-10 of its start
    and the solution agrees with the FP64 solver's to the discretisation's conditioning."""
    it64, h64, phi64 = _gpu_solve(pb, N, levels, pb.MG_FP64)
    itm, hm, phim = _gpu_solve(pb, N, levels, pb.MG_MIXED)
    assert hm[0] == h64[0]                      # same FP64 initial residual
    assert hm[-1] < 1e-10 * hm[0]
    assert itm <= it64 + 2
    err = np.max(np.abs(phim - phi64)) / np.max(np.abs(phi64))
    assert err < 1e-7


def test_direct_bottom_helmholtz_bitwise(pb, port):
    """Exact coarsest solve, Helmholtz form: history and solution bitwise vs the C port."""
    N, lev = 64, 3
    alpha = W.helmholtz_alpha(N, seed=3)
    rhs = -W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu_solve(pb, N, lev, pb.MG_FP64, max_iter=20, alpha=alpha, rhs=rhs, bottom=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, alpha.reshape(-1).copy(), 20, 1e-10,
                        rhs.reshape(-1).copy(), p2, bottom=1)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi, p2)
    assert hist[-1] < 1e-10 * hist[0]


def test_direct_bottom_poisson_bitwise(pb, port):
    """Exact coarsest solve of the (regularised) periodic Poisson operator, 4^3 coarsest cells."""
    N, lev = 32, 3
    rho = W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu_solve(pb, N, lev, pb.MG_FP64, max_iter=20, bottom=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None, 20, 1e-10, rho.reshape(-1).copy(), p2, bottom=1)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi, p2)


@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_odd_coarsest_direct_bottom_bitwise(pb, port, form):
    """An odd coarsest grid (96^3 over five halvings to 3^3, the shape of the 384^3 hierarchy) with
    the exact bottom solve, Poisson and per-cell-alpha Helmholtz: history and solution bitwise the C
    port's."""
    N, lev = 96, 5
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    rhs = -W.poisson_rho(N, seed=1) if alpha is not None else W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu_solve(pb, N, lev, pb.MG_FP64, max_iter=20, alpha=alpha, rhs=rhs, bottom=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None if alpha is None else alpha.reshape(-1).copy(), 20,
                        1e-10, rhs.reshape(-1).copy(), p2, bottom=1)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi, p2)
    assert hist[-1] < 1e-10 * hist[0]
    # mixed precision on the same hierarchy reaches the tolerance close to the FP64 solution
    itm, hm, phim = _gpu_solve(pb, N, lev, pb.MG_MIXED, max_iter=20, alpha=alpha, rhs=rhs, bottom=1)
    assert hm[-1] < 1e-10 * hm[0] and itm <= it + 2
    d = phim - phi
    ref = phi
    if alpha is None:   # a periodic Poisson solution is defined up to a constant
        d, ref = d - d.mean(), phi - phi.mean()
    assert np.max(np.abs(d)) / np.max(np.abs(ref)) < 1e-7


def test_mixed_helmholtz_direct_bottom(pb):
    N, lev = 64, 3
    alpha = W.helmholtz_alpha(N, seed=3)
    rhs = -W.poisson_rho(N, seed=1)
    it64, h64, phi64 = _gpu_solve(pb, N, lev, pb.MG_FP64, alpha=alpha, rhs=rhs, bottom=1)
    itm, hm, phim = _gpu_solve(pb, N, lev, pb.MG_MIXED, alpha=alpha, rhs=rhs, bottom=1)
    assert hm[-1] < 1e-10 * hm[0]
    assert itm <= it64 + 2
    err = np.max(np.abs(phim - phi64)) / np.max(np.abs(phi64))
    assert err < 1e-7


def test_levels_zero_direct_is_exact(pb, port):
    """A single grid with the exact bottom solve: one cycle, bitwise vs the C port."""
    N = 8
    rho = W.poisson_rho(N, seed=1)
    it, hist, phi = _gpu_solve(pb, N, 0, pb.MG_FP64, max_iter=3, bottom=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, 0, 4, 4, 10, 2.0 / 3.0, 1.0, None, 3, 1e-10, rho.reshape(-1).copy(), p2, bottom=1)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi, p2)


@pytest.mark.parametrize("edge,lev", [(0, 4), (16, 4), (32, 4), (8, 3), (16, 3)])
def test_coarse_levels_as_one_kernel_bitwise(pb, port, edge, lev):
    """Coarse levels run as one single-CTA kernel (edge 8..32; coarsest 4^3 or 8^3, exact or
    relaxed bottom) or one launch per step (0): the same arithmetic either way, so the history
    and solution are bitwise the C port's."""
    L = pb.lib()
    N = 64
    alpha = W.helmholtz_alpha(N, seed=3)
    rhs = -W.poisson_rho(N, seed=1)
    try:
        assert L.pb_mg_coarse_edge(edge) == 0
        it, hist, phi = _gpu_solve(pb, N, lev, pb.MG_FP64, max_iter=8, alpha=alpha, rhs=rhs, bottom=1)
        it2, hist2, phi2 = _gpu_solve(pb, N, lev, pb.MG_FP64, max_iter=8)
    finally:
        L.pb_mg_coarse_edge(8)
    p1 = np.zeros(N ** 3)
    n1, h1 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, alpha.reshape(-1).copy(), 8, 1e-10,
                        rhs.reshape(-1).copy(), p1, bottom=1)
    assert it == n1 and hist == list(h1) and np.array_equal(phi, p1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, lev, 4, 4, 10, 2.0 / 3.0, 1.0, None, 8, 1e-10,
                        W.poisson_rho(N, seed=1).reshape(-1).copy(), p2)
    assert it2 == n2 and hist2 == list(h2) and np.array_equal(phi2, p2)


def test_fas_history_bitwise(golden, pb):
    """LevelMultigridSolver<BoxOp_Laplace> (FAS, 4th-order flux form): the reference's own
    residual history and solution, bit for bit."""
    import torch
    cfg = golden[0]["mg"]["fas_32"]
    N = cfg["N"]
    rho = W.poisson_rho(N, seed=1).reshape(-1)
    mg = pb.FAS(N, cfg["numLevels"])
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(torch.from_numpy(-rho).cuda(), phi, max_iter=cfg["maxIter"], tol=cfg["tol"])
    pb.device_check()
    assert it == cfg["iters"]
    assert hist == cfg["hist"]
    assert digest(phi.cpu().numpy()) == cfg["phi_sha256"]


def test_fas_against_port_64(pb, port):
    import torch
    N, levels = 64, 5
    rho = W.poisson_rho(N, seed=1).reshape(-1).copy()
    mg = pb.FAS(N, levels)
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(torch.from_numpy(-rho).cuda(), phi, max_iter=6, tol=1e-10)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_fas(N, levels, 6, 1e-10, -rho, p2)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi.cpu().numpy(), p2)


def test_fas_against_port_80_partial_tiles(pb, port):
    """80^3 (staged two-cell sweeps with a partial x tile at the top level; 40^3 and below on the
    one-cell kernel): residual history and solution bitwise the C restatement's."""
    import torch
    N, levels = 80, 4
    rho = W.poisson_rho(N, seed=2).reshape(-1).copy()
    mg = pb.FAS(N, levels)
    phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
    it, hist = mg.solve(torch.from_numpy(-rho).cuda(), phi, max_iter=3, tol=1e-10)
    pb.device_check()
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_fas(N, levels, 3, 1e-10, -rho, p2)
    assert it == n2 and hist == list(h2)
    assert np.array_equal(phi.cpu().numpy(), p2)
