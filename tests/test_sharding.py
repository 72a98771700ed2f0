"""A level sharded over processes on the CPU: the Morton partition against the reference's own
BoxPartition, the halo items' coverage, and two (and three) gloo ranks exchanging and stepping a
periodic level through ShardedLevel, bitwise the oracle's single-process exchange and stepping.

The ranks compute with HostBackend, a numpy restatement of the level (test infrastructure: the
library has no CPU compute path); the partition, the halo plans, the buffer layout and the
torch.distributed transport are the library's own."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from proto_b200 import sharding as S          # noqa: E402
from proto_b200 import workloads as W         # noqa: E402


# ---- numpy backend --------------------------------------------------------------------------------
class HostLevel:
    def __init__(self, boxes, ghost, domain, periodic, ncomp=1):
        self.boxes = boxes
        self.g = (ghost,) * 3 if isinstance(ghost, int) else tuple(ghost)
        self.shapes = [tuple(b[1][d] - b[0][d] + 1 + 2 * self.g[d] for d in (2, 1, 0)) for b in boxes]
        sizes = [int(np.prod(s)) for s in self.shapes]
        self.offsets = [int(v) for v in np.concatenate([[0], np.cumsum(sizes)[:-1]])] if boxes else []
        self.slab_elems = int(sum(sizes))
        self.items = S.halo_items(boxes, ghost, domain, periodic)

    def view(self, slab, k):
        a = slab.numpy() if isinstance(slab, torch.Tensor) else slab
        return a[self.offsets[k]:self.offsets[k] + int(np.prod(self.shapes[k]))].reshape(self.shapes[k])

    def sl(self, k, r):
        """numpy slices of region r (global coordinates) in patch k's grown array."""
        lo = self.boxes[k][0]
        return tuple(slice(r[0][d] - lo[d] + self.g[d], r[1][d] - lo[d] + self.g[d] + 1) for d in (2, 1, 0))

    def exchange(self, slab):
        for i, j, s, r in self.items:
            src = S._shift(r, tuple(-v for v in s))
            self.view(slab, i)[self.sl(i, r)] = self.view(slab, j)[self.sl(j, src)]

    def stencil(self, stencil, epilogue, u, out, scale=1.0, a=0.0):
        coefs, offs = stencil
        c = [cj * scale if scale != 1.0 else cj for cj in coefs]
        for k, b in enumerate(self.boxes):
            U, O = self.view(u, k), self.view(out, k)
            gz, gy, gx = self.g[2], self.g[1], self.g[0]
            nz, ny, nx = (b[1][d] - b[0][d] + 1 for d in (2, 1, 0))
            acc = np.zeros((nz, ny, nx))
            for cj, (ox, oy, oz) in zip(c, offs):
                acc = acc + cj * U[gz + oz:gz + oz + nz, gy + oy:gy + oy + ny, gx + ox:gx + ox + nx]
            O[gz:gz + nz, gy:gy + ny, gx:gx + nx] = U[gz:gz + nz, gy:gy + ny, gx:gx + nx] + a * acc


class HostPlan:
    def __init__(self, level, items):
        self.level, self.items = level, items

    def _each(self, slab, buf, unpack):
        b = buf.numpy()
        for k, region, off in self.items:
            v = self.level.view(slab, k)[self.level.sl(k, region)]
            if unpack:
                v[...] = b[off:off + v.size].reshape(v.shape)
            else:
                b[off:off + v.size] = v.reshape(-1)

    def pack(self, slab, buf):
        self._each(slab, buf, False)

    def unpack(self, slab, buf):
        self._each(slab, buf, True)


class HostBackend:
    device = "cpu"

    def level(self, boxes, ghost, domain, periodic, ncomp=1):
        return HostLevel(boxes, ghost, domain, periodic, ncomp)

    def plan(self, level, items):
        return HostPlan(level, items)

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def local_absmax(self, level, slab):
        m = 0.0
        for k in range(len(level.boxes)):
            v = level.view(slab, k)
            g = level.g
            m = max(m, float(np.abs(v[g[2]:v.shape[0] - g[2], g[1]:v.shape[1] - g[1], g[0]:v.shape[2] - g[0]]).max()))
        return m


def laplacian7():
    """Stencil<T>::Laplacian's taps in insertion order (centre, then +e/-e per axis)."""
    offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    return [-6.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0], offs


# ---- partition ------------------------------------------------------------------------------------
def test_morton_index_interleaves_bits():
    assert S.morton_index((1, 0, 0)) == 1
    assert S.morton_index((0, 1, 0)) == 2
    assert S.morton_index((0, 0, 1)) == 4
    assert S.morton_index((3, 0, 0)) == 0b001001
    assert S.morton_index((2, 3, 1)) == 0b011110


def test_balance_matches_the_reference_partition_golden(golden):
    meta, _ = golden
    assert len(meta["partition"]) >= 5
    for case in meta["partition"]:
        pts = [tuple(p) for p in case["points"]]
        assert S.balance(pts, case["nranks"]) == case["owner"]


def test_balance_matches_the_reference_partition_live(ref):
    rng = np.random.default_rng(7)
    for shape in [(2, 2, 2), (4, 2, 3), (5, 5, 5), (16, 1, 2)]:
        pts = [(x, y, z) for z in range(shape[2]) for y in range(shape[1]) for x in range(shape[0])]
        pts = [pts[k] for k in rng.permutation(len(pts))]
        for nr in (1, 2, 3, 4, 6, 9):
            assert S.balance(pts, nr) == ref.load_balance(pts, nr)


def test_balance_segments():
    pts = [(x, y, z) for z in range(2) for y in range(2) for x in range(2)]
    own = S.balance(pts, 3)
    assert [own.count(r) for r in range(3)] == [3, 3, 2]
    # Morton order (0,0,0) (1,0,0) (0,1,0) | (1,1,0) (0,0,1) (1,0,1) | (0,1,1) (1,1,1)
    assert own == [0, 0, 0, 1, 1, 1, 2, 2]


def test_index_points_of_an_uneven_tiling():
    boxes, _ = W.amr_patches([[16, 24, 8], [8, 8], [32]])
    assert S.index_points(boxes) == [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0)]


@pytest.mark.parametrize("ghost,periodic", [(1, (1, 1, 1)), (2, (1, 1, 1)), (2, (1, 0, 1)), ((3, 1, 2), (0, 1, 1))])
def test_halo_items_cover_every_ghost_cell_once(ghost, periodic):
    boxes, L = W.amr_patches([[8, 12, 4], [6, 10], [5, 7, 4]])
    domain = ((0, 0, 0), tuple(v - 1 for v in L))
    g = (ghost,) * 3 if isinstance(ghost, int) else ghost
    items = S.halo_items(boxes, ghost, domain, periodic)
    for i, b in enumerate(boxes):
        shp = tuple(b[1][d] - b[0][d] + 1 + 2 * g[d] for d in (2, 1, 0))
        cnt = np.zeros(shp, dtype=int)
        for ii, j, s, r in items:
            if ii == i:
                cnt[tuple(slice(r[0][d] - b[0][d] + g[d], r[1][d] - b[0][d] + g[d] + 1) for d in (2, 1, 0))] += 1
        # every ghost cell whose periodic image lies in the domain is covered exactly once
        want = np.zeros(shp, dtype=int)
        zz, yy, xx = np.meshgrid(*[np.arange(shp[k]) for k in range(3)], indexing="ij")
        coords = [xx - g[0] + b[0][0], yy - g[1] + b[0][1], zz - g[2] + b[0][2]]
        inside = np.ones(shp, dtype=bool)
        for d in range(3):
            if not periodic[d]:
                inside &= (coords[d] >= 0) & (coords[d] < L[d])
        valid = np.zeros(shp, dtype=bool)
        valid[g[2]:shp[0] - g[2], g[1]:shp[1] - g[1], g[0]:shp[2] - g[0]] = True
        want[inside & ~valid] = 1
        assert np.array_equal(cnt, want)


def test_halo_plan_buffers_pair_up():
    boxes, L = W.amr_patches([[8, 8, 8, 8], [8, 8], [8, 8]])
    domain = ((0, 0, 0), tuple(v - 1 for v in L))
    for world in (2, 3, 5):
        owner = S.balance(S.index_points(boxes), world)
        plans = [S.HaloPlan(boxes, 2, domain, (1, 1, 1), owner, r) for r in range(world)]
        for a in range(world):
            for b in range(world):
                assert plans[a].send_elems.get(b, 0) == plans[b].recv_elems.get(a, 0)
                if a != b:
                    assert len(plans[a].send.get(b, [])) == len(plans[b].recv.get(a, []))


# ---- gloo ranks -----------------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fill(level, boxes, mine, valid, fill):
    slab = torch.full((level.slab_elems,), fill, dtype=torch.float64)
    g = level.g
    for k, i in enumerate(mine):
        lo, hi = boxes[i]
        v = level.view(slab, k)
        v[g[2]:v.shape[0] - g[2], g[1]:v.shape[1] - g[1], g[0]:v.shape[2] - g[0]] = \
            valid[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
    return slab


def _rank(rank, world, port, widths, ghost, seed, steps, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        boxes, L = W.amr_patches(widths)
        domain = ((0, 0, 0), tuple(v - 1 for v in L))
        sl = S.ShardedLevel(boxes, ghost, domain, (1, 1, 1), rank, world, S.DistComm(), HostBackend())
        valid = np.random.default_rng(seed).uniform(-1, 1, (L[2], L[1], L[0]))
        u = _fill(sl.level, sl.boxes, sl.mine, valid, -777.0)
        sl.exchange(u)
        out[("x", rank)] = {i: sl.level.view(u, k).copy() for k, i in enumerate(sl.mine)}
        tmp = torch.zeros_like(u)
        h = 1.0 / L[0]
        for _ in range(steps):
            sl.step(laplacian7(), u, tmp, 1.0 / (h * h), 0.1 * h * h)
            u, tmp = tmp, u
        out[("s", rank)] = {i: sl.level.view(u, k).copy() for k, i in enumerate(sl.mine)}
        out[("m", rank)] = sl.absmax(u)
        out[("owner", rank)] = sl.owner
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,widths", [(2, [[8, 12, 4], [6, 10], [5, 7, 4]]), (3, [[8, 8], [8, 8], [8, 8]])])
def test_gloo_ranks_exchange_and_step_like_one_process(port, world, widths):
    ghost, seed, steps = 2, 5, 3
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), widths, ghost, seed, steps, out), nprocs=world, join=True)
        res = dict(out)
    boxes, L = W.amr_patches(widths)
    owner = res[("owner", 0)]
    assert all(res[("owner", r)] == owner for r in range(world))
    assert sorted(set(owner)) == list(range(world))
    valid = np.random.default_rng(seed).uniform(-1, 1, (L[2], L[1], L[0]))

    # exchange: the oracle's single-process exchange of every patch
    g = ghost
    datas = []
    for lo, hi in boxes:
        a = np.full((hi[2] - lo[2] + 1 + 2 * g, hi[1] - lo[1] + 1 + 2 * g, hi[0] - lo[0] + 1 + 2 * g), -777.0)
        a[g:-g, g:-g, g:-g] = valid[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        datas.append(a.reshape(-1).copy())
    port.exchange([b[0] + b[1] for b in boxes], (g, g, g), ((0, 0, 0), [v - 1 for v in L]), (1, 1, 1), datas)
    got = {}
    for r in range(world):
        got.update(res[("x", r)])
    assert sorted(got) == list(range(len(boxes)))
    for i in range(len(boxes)):
        assert np.array_equal(got[i].reshape(-1), datas[i]), i

    # steps: the oracle's periodic stepping of the whole domain
    c, o = laplacian7()
    h = 1.0 / L[0]
    G = np.zeros((L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g))
    G[g:-g, g:-g, g:-g] = valid
    G = G.reshape(-1).copy()
    port.periodic_steps(L, g, c, np.asarray(o).reshape(-1), h, 0.1 * h * h, steps, G)
    ref = G.reshape(L[2] + 2 * g, L[1] + 2 * g, L[0] + 2 * g)[g:-g, g:-g, g:-g]
    for r in range(world):
        for i, a in res[("s", r)].items():
            lo, hi = boxes[i]
            assert np.array_equal(a[g:-g, g:-g, g:-g], ref[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]), i
    for r in range(world):
        assert res[("m", r)] == float(np.abs(ref).max())
