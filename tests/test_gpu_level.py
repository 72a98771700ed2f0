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
