"""Two Jacobi sweeps per pass (k_relax2): the multigrid solves that use it are bitwise the ones that
run every sweep as its own launch, and bitwise the C restatement's, for FP64 and mixed precision,
Poisson and Helmholtz, on the edges the kernel is built for (128, 192 and 256 with one cell per
thread, 384 with two), with the fused residual norm, and with small z chunks (many chunk seams)."""
import numpy as np
import pytest

from proto_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solve(pb, N, levels, precision, alpha=None, max_iter=3, relax2=128, zc=0, bottom=0, pv=0, rg=0):
    import torch
    L = pb.lib()
    assert L.pb_mg_relax2_min_edge(relax2) == 0 and L.pb_mg_relax2_shape(zc, pv, rg) == 0
    try:
        p = pb.MGParams(n=N, levels=levels, nu1=4, nu2=4, nu_bottom=10, omega=2.0 / 3.0, max_iter=max_iter,
                        tol=1e-10, form=pb.MG_HELMHOLTZ if alpha is not None else pb.MG_POISSON,
                        precision=precision, bottom=bottom)
        mg = pb.Multigrid(p)
        if alpha is not None:
            mg.set_alpha(torch.from_numpy(alpha.reshape(-1).copy()).cuda())
        rhs = -W.poisson_rho(N, seed=1) if alpha is not None else W.poisson_rho(N, seed=1)
        phi = torch.zeros(N ** 3, dtype=torch.float64, device="cuda")
        it, hist = mg.solve(torch.from_numpy(rhs.reshape(-1).copy()).cuda(), phi)
        pb.device_check()
        return it, hist, phi.cpu().numpy()
    finally:
        L.pb_mg_relax2_min_edge(128)
        L.pb_mg_relax2_shape(0, 0, 0)


@pytest.mark.parametrize("N,levels", [(128, 5), (192, 6), (256, 6)])
@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_fp64_pairs_bitwise_single_sweeps_and_port(pb, port, N, levels, form):
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    a = _solve(pb, N, levels, pb.MG_FP64, alpha)
    b = _solve(pb, N, levels, pb.MG_FP64, alpha, relax2=0)
    assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
    rhs = -W.poisson_rho(N, seed=1) if alpha is not None else W.poisson_rho(N, seed=1)
    p2 = np.zeros(N ** 3)
    n2, h2 = port.mg_cs(N, levels, 4, 4, 10, 2.0 / 3.0, 1.0, None if alpha is None else alpha.reshape(-1).copy(), 3,
                        1e-10, rhs.reshape(-1).copy(), p2)
    assert a[0] == n2 and a[1] == list(h2) and np.array_equal(a[2], p2)


@pytest.mark.parametrize("zc", [8, 30])
def test_fp64_pairs_small_z_chunks(pb, zc):
    a = _solve(pb, 256, 6, pb.MG_FP64, max_iter=2, zc=zc)
    b = _solve(pb, 256, 6, pb.MG_FP64, max_iter=2, relax2=0)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_mixed_pairs_bitwise(pb, form):
    N = 256
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    a = _solve(pb, N, 6, pb.MG_MIXED, alpha)
    b = _solve(pb, N, 6, pb.MG_MIXED, alpha, relax2=0)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("form", ["poisson", "helmholtz"])
def test_384_two_cells_per_thread(pb, precision, form):
    N = 384
    alpha = W.helmholtz_alpha(N, seed=3) if form == "helmholtz" else None
    a = _solve(pb, N, 7, precision, alpha, max_iter=2, bottom=1)
    b = _solve(pb, N, 7, precision, alpha, max_iter=2, relax2=0, bottom=1)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("N,levels", [(128, 5), (256, 6)])
@pytest.mark.parametrize("precision", [0, 1])
def test_two_cells_per_thread_bitwise(pb, N, levels, precision):
    alpha = W.helmholtz_alpha(N, seed=3)
    a = _solve(pb, N, levels, precision, alpha, max_iter=2, pv=2)
    b = _solve(pb, N, levels, precision, alpha, max_iter=2, relax2=0)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])
    c = _solve(pb, N, levels, precision, None, max_iter=2, pv=2)
    d = _solve(pb, N, levels, precision, None, max_iter=2, relax2=0)
    assert c[1] == d[1] and np.array_equal(c[2], d[2])


@pytest.mark.parametrize("N,levels", [(256, 6), (384, 7)])
@pytest.mark.parametrize("precision", [0, 1])
def test_tall_tiles_bitwise(pb, N, levels, precision):
    a = _solve(pb, N, levels, precision, None, max_iter=2, rg=4, bottom=1)
    b = _solve(pb, N, levels, precision, None, max_iter=2, relax2=0, bottom=1)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


def test_launch_count_with_pairs(pb):
    """pb_mg_launches_per_cycle counts a two-sweep pass as one launch: 256^3 V(4,4) over 6 levels with
    the coarse levels (edge <= 8) as one kernel. FP64: 256 takes pairs (the norm pass does the first
    two sweeps, then one pair before and two after the coarse correction), 128 too (entered from
    zero: a pair from zero and a pair, then two pairs), 64..16 one launch per sweep. Mixed: the
    256^3 correction starts from zero (a pair from zero and a pair) and ends with a pair and the
    pair that adds it to the FP64 solution; then the FP64 residual pass."""
    import ctypes
    L = pb.lib()
    p = pb.MGParams(n=256, levels=6, nu1=4, nu2=4, nu_bottom=10)
    n = L.pb_mg_launches_per_cycle(ctypes.byref(p.c))
    # 64, 32, 16: 4 + 4 sweeps + restrict + prolong; the coarse kernel
    lower = 3 * 10 + 1
    # 128: zero pair + pair + restrict + prolong + 2 pairs
    l128 = 1 + 1 + 1 + 1 + 2
    # 256: 1 pair + restrict + prolong + 2 pairs; the norm pass
    assert n == (1 + 1 + 1 + 2) + l128 + lower + 1
    pm = pb.MGParams(n=256, levels=6, nu1=4, nu2=4, nu_bottom=10, precision=pb.MG_MIXED)
    nm = L.pb_mg_launches_per_cycle(ctypes.byref(pm.c))
    # 256: zero pair + pair + restrict + prolong + pair + update pair; the FP64 residual pass
    assert nm == (1 + 1 + 1 + 1 + 1 + 1) + l128 + lower + 1
