"""A level sharded over ranks, on one GPU: every rank's patches in its own device level, the remote
ghost regions packed and unpacked by the library's halo plans, the buffers moved by LocalComm (all
ranks' sends posted before any rank receives, so no kernel waits on another rank). Exchange and
Euler steps are bitwise the oracle's single-process exchange and periodic stepping."""
import numpy as np
import pytest

from proto_b200 import sharding as S
from proto_b200 import workloads as W
from tests.util import table

# the 7-point Laplacian in Stencil<T>::Laplacian's insertion order (centre, then +e/-e per axis)
LAP7 = ([-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0],
        [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)])

pytestmark = pytest.mark.gpu


def _ranks(pb, boxes, ghost, L, world):
    domain = ((0, 0, 0), tuple(v - 1 for v in L))
    comm = S.LocalComm(world)
    return [S.ShardedLevel(boxes, ghost, domain, (1, 1, 1), r, world, comm.for_rank(r)) for r in range(world)]


def _fill(torch, sl, valid, fill):
    lv = sl.level
    slab = np.full(lv.slab_elems, fill)
    g = lv.ghost
    for p, off in zip(lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * g[d] for d in (2, 1, 0))
        a = np.full(shp, fill)
        a[g[2]:shp[0] - g[2], g[1]:shp[1] - g[1], g[0]:shp[2] - g[0]] = \
            valid[p.lo[2]:p.hi[2] + 1, p.lo[1]:p.hi[1] + 1, p.lo[0]:p.hi[0] + 1]
        slab[off:off + a.size] = a.reshape(-1)
    return torch.from_numpy(slab).cuda()


def _patches(sl, slab):
    """{global patch id: grown array} of one rank."""
    lv, g = sl.level, sl.level.ghost
    host = slab.cpu().numpy()
    out = {}
    for i, p, off in zip(sl.mine, lv.patches, lv.offsets):
        shp = tuple(p.size(d) + 2 * g[d] for d in (2, 1, 0))
        out[i] = host[off:off + int(np.prod(shp))].reshape(shp)
    return out


def _oracle_exchange(port, boxes, g, L, valid, fill):
    datas = []
    for lo, hi in boxes:
        a = np.full((hi[2] - lo[2] + 1 + 2 * g, hi[1] - lo[1] + 1 + 2 * g, hi[0] - lo[0] + 1 + 2 * g), fill)
        a[g:-g, g:-g, g:-g] = valid[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        datas.append(a.reshape(-1).copy())
    port.exchange([b[0] + b[1] for b in boxes], (g, g, g), ((0, 0, 0), [v - 1 for v in L]), (1, 1, 1), datas)
    return datas


@pytest.mark.parametrize("world,widths", [(2, [[8, 12, 4], [6, 10], [5, 7, 4]]), (3, [[16, 16], [16, 16], [16, 16]]),
                                          (4, [[24, 8, 16], [16, 16], [8, 24]])])
def test_exchange_bitwise_the_oracle(pb, port, world, widths):
    import torch
    g = 2
    boxes, L = W.amr_patches(widths)
    ranks = _ranks(pb, boxes, g, L, world)
    valid = np.random.default_rng(11).uniform(-1, 1, (L[2], L[1], L[0]))
    slabs = [_fill(torch, r, valid, -777.0) for r in ranks]
    S.exchange_all(ranks, slabs)
    torch.cuda.synchronize()
    want = _oracle_exchange(port, boxes, g, L, valid, -777.0)
    seen = set()
    for r, s in zip(ranks, slabs):
        for i, a in _patches(r, s).items():
            assert np.array_equal(a.reshape(-1), want[i]), i
            seen.add(i)
    assert seen == set(range(len(boxes)))
    pb.device_check()


def _steps(pb, ranks, slabs, nsteps, h, taps=LAP7):
    import torch
    c, o = taps
    st = pb.Stencil(c, o)
    tmps = [torch.zeros_like(s) for s in slabs]
    for _ in range(nsteps):
        S.exchange_all(ranks, slabs)
        for r, u, t in zip(ranks, slabs, tmps):
            r.level.stencil(st, pb.EPI_EULER, u, t, scale=1.0 / (h * h), a=0.1 * h * h)
        slabs, tmps = tmps, slabs
    return slabs, (c, o)


@pytest.mark.parametrize("world,widths", [(2, [[8, 12, 4], [6, 10], [5, 7, 4]]), (3, [[16, 16], [16, 16], [16, 16]])])
def test_steps_bitwise_the_oracle(pb, port, world, widths):
    import torch
    g, nsteps = 2, 3
    boxes, L = W.amr_patches(widths)
    ranks = _ranks(pb, boxes, g, L, world)
    valid = np.random.default_rng(12).uniform(-1, 1, (L[2], L[1], L[0]))
    slabs = [_fill(torch, r, valid, 0.0) for r in ranks]
    h = 1.0 / L[0]
    slabs, (c, o) = _steps(pb, ranks, slabs, nsteps, h)
    torch.cuda.synchronize()
    G = np.zeros((L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g))
    G[g:-g, g:-g, g:-g] = valid
    G = G.reshape(-1).copy()
    port.periodic_steps(L, g, c, np.asarray(o).reshape(-1), h, 0.1 * h * h, nsteps, G)
    ref = G.reshape(L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g)[g:-g, g:-g, g:-g]
    for r, s in zip(ranks, slabs):
        for i, a in _patches(r, s).items():
            lo, hi = boxes[i]
            assert np.array_equal(a[g:-g, g:-g, g:-g], ref[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]), i
    m = [r.backend.local_absmax(r.level, s) for r, s in zip(ranks, slabs)]
    assert max(m) == float(np.abs(ref).max())


def test_full_size_amr_level_on_two_ranks(golden, pb, port):
    """The 512-patch uneven level over two ranks, 4 Euler steps of the 13-point Laplacian (the
    reference's StencilLib table): bitwise the oracle's periodic stepping of the whole domain."""
    import torch
    g, nsteps = 2, 4
    boxes, L = W.amr_patches(W.amr_widths(seed=2))
    assert len(boxes) == 512
    ranks = _ranks(pb, boxes, g, L, 2)
    assert [len(r.mine) for r in ranks] == [256, 256]
    valid = np.random.default_rng(13).uniform(-1, 1, (L[2], L[1], L[0]))
    slabs = [_fill(torch, r, valid, 0.0) for r in ranks]
    h = 1.0 / L[0]
    c13, o13, _ = table(golden[1], "laplacian13")
    slabs, (c, o) = _steps(pb, ranks, slabs, nsteps, h, (c13, [tuple(v) for v in np.asarray(o13).reshape(-1, 3)]))
    torch.cuda.synchronize()
    G = np.zeros((L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g))
    G[g:-g, g:-g, g:-g] = valid
    G = G.reshape(-1).copy()
    port.periodic_steps(L, g, c, np.asarray(o).reshape(-1), h, 0.1 * h * h, nsteps, G)
    ref = G.reshape(L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g)[g:-g, g:-g, g:-g]
    for r, s in zip(ranks, slabs):
        for i, a in _patches(r, s).items():
            lo, hi = boxes[i]
            assert np.array_equal(a[g:-g, g:-g, g:-g], ref[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]), i


def test_halo_plan_rejects_regions_outside_the_grown_patch(pb):
    import ctypes
    boxes, L = W.amr_patches([[8, 8], [8], [8]])
    lv = pb.Level([pb.Box(*b) for b in boxes], 1, pb.Box((0, 0, 0), [v - 1 for v in L]), (1, 1, 1))
    with pytest.raises(pb.ProtoError):
        S._DevicePlan(lv, [(0, ((-2, 0, 0), (-1, 3, 3)), 0)])      # two cells out, ghost is one
    with pytest.raises(pb.ProtoError):
        S._DevicePlan(lv, [(2, ((0, 0, 0), (0, 0, 0)), 0)])        # no patch 2
    p = S._DevicePlan(lv, [(0, ((-1, 0, 0), (-1, 7, 7)), 0), (1, ((16, 0, 0), (16, 7, 7)), 64)])
    assert p.elems == 128
    L_ = pb.lib()
    assert L_.pb_halo_plan_elems(ctypes.c_void_p()) == -1
