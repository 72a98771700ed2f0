"""LevelBoxData ghost exchange and batched level stepping on the GPU."""
import numpy as np
import pytest

from proto_b200 import workloads as W
from tests.util import digest, table

pytestmark = pytest.mark.gpu


def _slab_from_valid(level, valid_zyx, fill):
    slab = np.full(level.slab_elems, fill)
    g = level.ghost
    for p, off in zip(level.patches, level.offsets):
        shp = tuple(p.size(d) + 2 * g[d] for d in (2, 1, 0))
        a = np.full(shp, fill)
        a[g[2]:shp[0] - g[2], g[1]:shp[1] - g[1], g[0]:shp[2] - g[0]] = \
            valid_zyx[p.lo[2]:p.hi[2] + 1, p.lo[1]:p.hi[1] + 1, p.lo[0]:p.hi[0] + 1]
        slab[off:off + a.size] = a.reshape(-1)
    return slab


def _patch_arrays(level, slab):
    g = level.ghost
    out = []
    for p, off in zip(level.patches, level.offsets):
        n = int(np.prod([p.size(d) + 2 * g[d] for d in range(3)]))
        out.append(slab[off:off + n])
    return out


@pytest.mark.parametrize("k", range(4))
def test_uniform_exchange_golden(golden, pb, k):
    import torch
    case = golden[0]["exchange"][k]
    dom, per, bs, g = case["domain"], case["periodic"], case["box"], case["ghost"]
    npch = [dom[d] // bs[d] for d in range(3)]
    patches = []
    for pz in range(npch[2]):
        for py in range(npch[1]):
            for px in range(npch[0]):
                lo = (px * bs[0], py * bs[1], pz * bs[2])
                patches.append(pb.Box(lo, [lo[d] + bs[d] - 1 for d in range(3)]))
    lv = pb.Level(patches, g, pb.Box((0, 0, 0), [d - 1 for d in dom]), per)
    valid = np.random.default_rng(case["seed"]).uniform(-1, 1, int(np.prod(dom))).reshape(dom[2], dom[1], dom[0])
    slab = torch.from_numpy(_slab_from_valid(lv, valid, -777.0)).cuda()
    lv.exchange(slab)
    torch.cuda.synchronize()
    out = np.concatenate(_patch_arrays(lv, slab.cpu().numpy()))
    assert digest(out) == case["sha256"]


def test_uneven_exchange_against_oracle(pb, port):
    import torch
    widths = [[16, 24, 32], [24, 16], [48, 16, 32]]
    boxes, L = W.amr_patches(widths)
    g = (2, 2, 2)
    lv = pb.Level([pb.Box(*b) for b in boxes], g, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    valid = np.random.default_rng(4).uniform(-1, 1, (L[2], L[1], L[0]))
    host = _slab_from_valid(lv, valid, -777.0)
    slab = torch.from_numpy(host).cuda()
    lv.exchange(slab)
    torch.cuda.synchronize()
    datas = [a.copy() for a in _patch_arrays(lv, host)]
    port.exchange([b[0] + b[1] for b in boxes], g, ((0, 0, 0), [v - 1 for v in L]), (1, 1, 1), datas)
    assert np.array_equal(np.concatenate(_patch_arrays(lv, slab.cpu().numpy())), np.concatenate(datas))


def test_level13_steps_golden(golden, pb):
    import torch
    g = golden[0]["level13"]
    boxes, L = W.amr_patches(g["widths"])
    gh = g["ghost"]
    lv = pb.Level([pb.Box(*b) for b in boxes], gh, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    c, o, m = table(golden[1], "laplacian13")
    S = pb.Stencil(c, o)
    u = W.uniform_box((L[2], L[1], L[0]), g["seed"])
    a = torch.from_numpy(_slab_from_valid(lv, u, 0.0)).cuda()
    b = torch.zeros_like(a)
    for _ in range(g["steps"]):
        lv.exchange(a)
        lv.stencil(S, pb.EPI_EULER, a, b, scale=1.0 / (g["h"] * g["h"]), a=g["dt"])
        a, b = b, a
    torch.cuda.synchronize()
    host = a.cpu().numpy()
    parts = []
    for p, off in zip(lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * gh for d in (2, 1, 0))
        parts.append(host[off:off + int(np.prod(shp))].reshape(shp)[gh:-gh, gh:-gh, gh:-gh].reshape(-1))
    assert digest(np.concatenate(parts)) == g["sha256"]


def _level13(golden, pb, widths, seed):
    import torch
    boxes, L = W.amr_patches(widths)
    gh = 2
    lv = pb.Level([pb.Box(*b) for b in boxes], gh, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    c, o, m = table(golden[1], "laplacian13")
    u = W.uniform_box((L[2], L[1], L[0]), seed)
    a = torch.from_numpy(_slab_from_valid(lv, u, 0.0)).cuda()
    return lv, pb.Stencil(c, o), (c, o), u, a, L


def _valid(lv, slab):
    gh = lv.ghost[0]
    parts = []
    for p, off in zip(lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * gh for d in (2, 1, 0))
        parts.append(slab[off:off + int(np.prod(shp))].reshape(shp)[gh:-gh, gh:-gh, gh:-gh].reshape(-1))
    return np.concatenate(parts)


@pytest.mark.parametrize("tune", [False, True])
def test_level13_graph_steps_golden(golden, pb, tune):
    """The captured multi-step graph (with default or autotuned tiles) gives the golden digest."""
    import torch
    g = golden[0]["level13"]
    lv, S, _, _, a, _ = _level13(golden, pb, g["widths"], g["seed"])
    b = torch.zeros_like(a)
    if tune:
        lv.autotune(S, a, b, scale=1.0 / (g["h"] * g["h"]))
        assert all(tx in (8, 16, 32, 64) and zd in (4, 8, 16, 32) for _, tx, zd in lv.tiles())
    lv.steps(S, pb.EPI_EULER, a, b, g["steps"], scale=1.0 / (g["h"] * g["h"]), a=g["dt"])
    torch.cuda.synchronize()
    assert digest(_valid(lv, a.cpu().numpy())) == g["sha256"]
    lv.steps(S, pb.EPI_EULER, a, b, 2, scale=1.0 / (g["h"] * g["h"]), a=g["dt"])   # a new graph (step count)
    lv.steps(S, pb.EPI_EULER, a, b, 2, scale=1.0 / (g["h"] * g["h"]), a=g["dt"])   # replayed
    torch.cuda.synchronize()
    pb.device_check()


@pytest.mark.parametrize("steps", [4, 100])
def test_amr_level_full_size_against_port(golden, pb, port, steps):
    """The 512-patch uneven level (widths from seed 2), autotuned tiles, 4 graph steps and the
    measured workload's 100: bitwise the C port's periodic stepping on the whole domain."""
    import torch
    widths = W.amr_widths(seed=2)
    lv, S, (c, o), u, a, L = _level13(golden, pb, widths, 7)
    assert len(lv.patches) == 512
    h = 1.0 / L[0]
    b = torch.zeros_like(a)
    lv.autotune(S, a, b, scale=1.0 / (h * h))
    lv.steps(S, pb.EPI_EULER, a, b, steps, scale=1.0 / (h * h), a=0.1 * h * h)
    torch.cuda.synchronize()
    got = a.cpu().numpy()
    gh = 2
    G = np.zeros((L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh))
    G[gh:-gh, gh:-gh, gh:-gh] = u
    G = G.reshape(-1).copy()
    port.periodic_steps(L, gh, c, o.reshape(-1), h, 0.1 * h * h, steps, G)
    ref = G.reshape(L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh)[gh:-gh, gh:-gh, gh:-gh]
    out = np.zeros_like(u)
    for p, off in zip(lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * gh for d in (2, 1, 0))
        blk = got[off:off + int(np.prod(shp))].reshape(shp)[gh:-gh, gh:-gh, gh:-gh]
        out[p.lo[2]:p.hi[2] + 1, p.lo[1]:p.hi[1] + 1, p.lo[0]:p.hi[0] + 1] = blk
    assert np.array_equal(out, ref)


def test_steps_on_a_non_tensor_layout_use_the_exchange(golden, pb):
    """A tiling that is not a tensor product keeps exchange + ghost cells; graph steps equal the
    explicit loop bitwise."""
    import torch
    boxes = [((0, 0, 0), (15, 31, 31)), ((16, 0, 0), (31, 15, 31)), ((16, 16, 0), (31, 31, 31))]
    lv = pb.Level([pb.Box(*b) for b in boxes], 2, pb.Box((0, 0, 0), (31, 31, 31)), (1, 1, 1))
    c, o, m = table(golden[1], "laplacian13")
    S = pb.Stencil(c, o)
    u = W.uniform_box((32, 32, 32), 5)
    a = torch.from_numpy(_slab_from_valid(lv, u, 0.0)).cuda()
    b = torch.zeros_like(a)
    a2, b2 = a.clone(), b.clone()
    h = 1.0 / 32
    lv.steps(S, pb.EPI_EULER, a, b, 3, scale=1.0 / (h * h), a=0.1 * h * h)
    for _ in range(3):
        lv.exchange(a2)
        lv.stencil(S, pb.EPI_EULER, a2, b2, scale=1.0 / (h * h), a=0.1 * h * h)
        a2, b2 = b2, a2
    torch.cuda.synchronize()
    assert np.array_equal(_valid(lv, a.cpu().numpy()), _valid(lv, a2.cpu().numpy()))


@pytest.mark.parametrize("case", ["odd_x_extents_13pt", "even_7pt"])
def test_fused_steps_other_kernels_equal_the_exchange_loop(golden, pb, case):
    """Fused steps on tensor tilings that the two-cells-per-thread kernel does not take (odd x
    extents; a halo-1 stencil) run the one-cell ring kernel: bitwise the exchange + stencil loop."""
    import torch
    if case == "odd_x_extents_13pt":
        widths, name = [[15, 17, 16], [16, 24], [20, 12, 16]], "laplacian13"
    else:
        widths, name = [[16, 24, 32], [24, 16], [48, 16, 32]], "laplacian"
    boxes, L = W.amr_patches(widths)
    lv = pb.Level([pb.Box(*b) for b in boxes], 2, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    c, o, m = table(golden[1], name)
    S = pb.Stencil(c, o)
    u = W.uniform_box((L[2], L[1], L[0]), 11)
    a = torch.from_numpy(_slab_from_valid(lv, u, 0.0)).cuda()
    b = torch.zeros_like(a)
    a2, b2 = a.clone(), b.clone()
    h = 1.0 / L[0]
    lv.steps(S, pb.EPI_EULER, a, b, 3, scale=1.0 / (h * h), a=0.1 * h * h)
    for _ in range(3):
        lv.exchange(a2)
        lv.stencil(S, pb.EPI_EULER, a2, b2, scale=1.0 / (h * h), a=0.1 * h * h)
        a2, b2 = b2, a2
    torch.cuda.synchronize()
    pb.device_check()
    assert np.array_equal(_valid(lv, a.cpu().numpy()), _valid(lv, a2.cpu().numpy()))
