"""The synthetic workloads the bench and the GPU tests run, checked on CPU: the serving request
stream (2000 requests, Poisson arrivals at 200/s, edges log-uniform in [32, 192] rounded to 16,
Poisson/Helmholtz about half each, alpha in [0, 1], seeded), the right-hand sides (mean removed),
and the AMR-level widths (8 per axis from {16, 24, 32, 48, 64})."""
import numpy as np

from proto_b200 import serving as S
from proto_b200 import workloads as W


def test_serving_trace_shape_and_seed():
    t = S.make_trace()
    assert len(t) == 2000
    assert [r["i"] for r in t] == list(range(2000))
    edges = np.array([r["n"] for r in t])
    assert edges.min() >= 32 and edges.max() <= 192 and np.all(edges % 16 == 0)
    assert set(edges.tolist()) == set(range(32, 193, 16))
    arrive = np.array([r["t"] for r in t])
    assert arrive[0] == 0.0 and np.all(np.diff(arrive) >= 0)
    rate = (len(t) - 1) / arrive[-1]
    assert 180.0 < rate < 220.0                      # Poisson arrivals at 200/s
    helm = np.array([r["helm"] for r in t])
    assert 0.45 < helm.mean() < 0.55
    alpha = np.array([r["alpha"] for r in t])
    assert np.all(alpha[~helm] == 0.0) and np.all((alpha[helm] >= 0.0) & (alpha[helm] <= 1.0))
    # log-uniform edges: more small grids than large ones
    assert (edges <= 64).sum() > (edges >= 160).sum()
    assert S.make_trace() == t                      # seeded: the same stream every time
    assert S.make_trace(seed=5) != t


def test_every_served_edge_halves_down_to_the_coarse_cycle():
    """The engine takes edges m * 2^k with m <= 16 (its batched levels end where the single-CTA
    coarse cycle takes over); every edge of the stream qualifies."""
    for n in set(r["n"] for r in S.make_trace()):
        e = n
        while e > 16 and e % 2 == 0:
            e //= 2
        assert e <= 16, n


def test_right_hand_sides_have_zero_mean():
    for n in (32, 48):
        f = W.sine_modes_rhs(n, seed=7, modes=4)
        assert f.shape == (n, n, n)
        assert abs(float(f.mean())) < 1e-12 * max(1.0, float(np.abs(f).max()))
    rho = W.poisson_rho(32, seed=1)
    assert abs(float(rho.mean())) < 1e-12 * float(np.abs(rho).max())
    assert np.array_equal(rho, W.poisson_rho(32, seed=1))


def test_amr_level_widths():
    w = W.amr_widths()
    arr = np.asarray(w)
    assert arr.shape[0] == 3 and arr.shape[1] == 8
    assert set(arr.ravel().tolist()) <= {16, 24, 32, 48, 64}


def test_amr_level_tiles_the_periodic_domain():
    """512 patches that tile the domain exactly: no overlap, no gap (cell counts add up and every
    patch lies inside), as the level's ghost exchange assumes."""
    boxes, dom = W.amr_patches(W.amr_widths())
    assert len(boxes) == 512
    assert dom == [272, 344, 224]                    # the level the bench steps (21.0 M cells)
    cells = 0
    for lo, hi in boxes:
        assert all(0 <= lo[d] <= hi[d] < dom[d] for d in range(3))
        cells += (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1)
    assert cells == dom[0] * dom[1] * dom[2] == 20959232
    starts = {lo for lo, _ in boxes}
    assert len(starts) == 512


def test_one_right_hand_side_per_request():
    """Every request carries its own seed, and the device evaluation of its right-hand side (run here
    on the CPU through torch) agrees with the numpy evaluation to rounding."""
    import torch
    t = S.make_trace()
    seeds = [r["seed"] for r in t]
    assert len(set(seeds)) == len(t)
    for r in t[:3]:
        n = 32
        a = W.sine_modes_rhs(n, seed=r["seed"], modes=4)
        b = W.sine_modes_rhs_device(n, r["seed"], modes=4, device="cpu").numpy()
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
    x = W.sine_modes_rhs_device(32, t[0]["seed"], device="cpu")
    y = W.sine_modes_rhs_device(32, t[1]["seed"], device="cpu")
    assert not torch.equal(x, y)
