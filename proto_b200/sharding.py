"""A level sharded over processes: patches in Morton order, a cross-process halo exchange and
distributed norms.

Reference (paths within the reference project):
  DisjointBoxLayout::loadBalance / BoxPartition::loadBalance .. include/base/implem/Proto_DisjointBoxLayoutImplem.H:114-125,
                                                                 include/base/implem/Proto_BoxPartitionImplem.H:43-54,196-222
  Morton::index ............................................... include/base/implem/Proto_MortonImplem.H
  Copier (local + remote motion items) ......................... include/base/implem/Proto_CopierImplem.H:172-181,307-460
  Reduction over ranks (MPI_Allreduce) ......................... include/base/implem/Proto_ReductionImplem.H:125-155

A process owns a contiguous run of patches in Morton order of their patch index points, the first
(npatch % nranks) processes one more than the rest, as the reference's load balance assigns them.
Each process holds its patches as one device level (pb_level: local ghost exchange and stencil steps
in single launches). A ghost region whose source patch lives on another process is a remote item:
the owner packs the source cells into one buffer per destination process (one launch for all of its
regions), the buffers move (NCCL point-to-point between GPUs, or any transport), and the receiver
unpacks them into its ghost cells (one launch). Both sides enumerate the items in one global order
(destination patch, source patch, periodic image), so a buffer's layout needs no header. Norms are
a local reduction followed by an all-reduce (max) of one double.

The compute backend and the transport are pluggable: DeviceBackend (the library's kernels on the
current GPU) with DistComm (torch.distributed over NCCL) is the product path; LocalComm moves
buffers between rank objects living in one process (one GPU can host every rank's data with no
kernel of one rank waiting on another's).
"""
import ctypes

import numpy as np

from . import Box, Level, lib, reduce, EPI_EULER, RED_ABS, _check, _c, _c_int, _ptr, _stream, pb_box


# ---- partition ------------------------------------------------------------------------------------
def morton_index(p):
    """Interleaved bits of a non-negative 3-D point: bit k of coordinate d at bit 3k + d."""
    r = 0
    for k in range(21):
        for d in range(3):
            r |= ((int(p[d]) >> k) & 1) << (3 * k + d)
    return r


def index_points(boxes):
    """Patch index points of a tiling: per axis, the rank of each patch's low corner among the
    distinct low corners (the patch grid coordinates of a tensor-product tiling)."""
    lows = [sorted(set(b[0][d] for b in boxes)) for d in range(3)]
    pos = [{v: k for k, v in enumerate(l)} for l in lows]
    return [tuple(pos[d][b[0][d]] for d in range(3)) for b in boxes]


def balance(points, nranks):
    """Owner of each patch: Morton order (ties kept in input order), then contiguous runs of
    len // nranks patches, the first len % nranks ranks taking one more."""
    order = sorted(range(len(points)), key=lambda i: (morton_index(points[i]), i))
    n = len(points)
    length, rem = n // nranks, n % nranks
    owner = [0] * n
    g = 0
    for r in range(nranks):
        seg = length + (1 if r < rem else 0)
        for i in order[g:g + seg]:
            owner[i] = r
        g += seg
    return owner


# ---- halo items -----------------------------------------------------------------------------------
def _isect(a, b):
    lo = tuple(max(a[0][d], b[0][d]) for d in range(3))
    hi = tuple(min(a[1][d], b[1][d]) for d in range(3))
    return (lo, hi) if all(lo[d] <= hi[d] for d in range(3)) else None


def _shift(b, s):
    return (tuple(b[0][d] + s[d] for d in range(3)), tuple(b[1][d] + s[d] for d in range(3)))


def halo_items(boxes, ghost, domain, periodic):
    """Every ghost region of the level: (dst patch, src patch, image shift, region in dst
    coordinates) for grown(dst) & (valid(src) + shift), over src patches and periodic images, in
    one global order. A region is filled from src cells region - shift."""
    g = (ghost,) * 3 if isinstance(ghost, int) else tuple(ghost)
    ext = [domain[1][d] - domain[0][d] + 1 for d in range(3)]
    axes = [(0, -ext[d], ext[d]) if periodic[d] else (0,) for d in range(3)]
    shifts = [(sx, sy, sz) for sz in axes[2] for sy in axes[1] for sx in axes[0]]
    out = []
    for i, bi in enumerate(boxes):
        grown = (tuple(bi[0][d] - g[d] for d in range(3)), tuple(bi[1][d] + g[d] for d in range(3)))
        for j, bj in enumerate(boxes):
            for s in shifts:
                if i == j and s == (0, 0, 0):
                    continue
                r = _isect(grown, _shift(bj, s))
                if r is not None:
                    out.append((i, j, s, r))
    return out


class HaloPlan:
    """This rank's remote items: for each peer, the regions it sends (source patch, source region)
    and receives (destination patch, region), with their offsets in the peer's buffer. Patch
    numbers are local (positions in this rank's patch list)."""

    def __init__(self, boxes, ghost, domain, periodic, owner, rank, ncomp=1):
        local = {i: k for k, i in enumerate(p for p in range(len(boxes)) if owner[p] == rank)}
        self.send, self.recv = {}, {}
        soff, roff = {}, {}
        for i, j, s, r in halo_items(boxes, ghost, domain, periodic):
            oi, oj = owner[i], owner[j]
            if oi == oj:
                continue
            vol = ncomp * int(np.prod([r[1][d] - r[0][d] + 1 for d in range(3)]))
            if oj == rank:       # j's cells travel to the owner of i
                o = soff.get(oi, 0)
                self.send.setdefault(oi, []).append((local[j], _shift(r, tuple(-v for v in s)), o))
                soff[oi] = o + vol
            elif oi == rank:     # i's ghost cells come from the owner of j
                o = roff.get(oj, 0)
                self.recv.setdefault(oj, []).append((local[i], r, o))
                roff[oj] = o + vol
        self.send_elems, self.recv_elems = soff, roff


# ---- transports -----------------------------------------------------------------------------------
class DistComm:
    """torch.distributed: one grouped point-to-point round per exchange (NCCL between GPUs, gloo on
    CPU) and all-reduce for norms."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def exchange(self, sends, recvs):
        """sends / recvs: {peer: tensor}; posts every transfer, then waits for all of them."""
        ops = []
        for peer in sorted(set(sends) | set(recvs)):
            if peer in sends:
                ops.append(self.dist.P2POp(self.dist.isend, sends[peer], peer, self.group))
            if peer in recvs:
                ops.append(self.dist.P2POp(self.dist.irecv, recvs[peer], peer, self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce_max(self, value, device):
        import torch
        t = torch.tensor([value], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(t.item())


class LocalComm:
    """Ranks living in one process: each rank posts its send buffers, then takes its receive
    buffers (copies between tensors; callers sequence the ranks' phases on the host)."""

    class _Mailbox:
        def __init__(self):
            self.box = {}
            self.values = {}

    def __init__(self, world, mailbox=None):
        self.world = world
        self.mb = mailbox if mailbox is not None else LocalComm._Mailbox()

    def for_rank(self, rank):
        c = LocalComm(self.world, self.mb)
        c.rank = rank
        return c

    def post(self, sends):
        for peer, t in sends.items():
            self.mb.box[(self.rank, peer)] = t

    def take(self, recvs):
        for peer, t in recvs.items():
            t.copy_(self.mb.box.pop((peer, self.rank)))

    def exchange(self, sends, recvs):
        raise RuntimeError("LocalComm ranks post all sends before any rank takes (see ShardedLevel.exchange_all)")

    def post_value(self, value):
        self.mb.values[self.rank] = value

    def max_value(self):
        return max(self.mb.values.values())


# ---- compute backend -----------------------------------------------------------------------------
class DeviceBackend:
    """The library on the current GPU: pb_level for the local patches, pb_halo plans for the remote
    regions, torch CUDA tensors as buffers."""

    def __init__(self):
        import torch
        self.torch = torch
        self.device = "cuda"

    def level(self, boxes, ghost, domain, periodic, ncomp=1):
        return Level([Box(*b) for b in boxes], ghost, Box(*domain), periodic, ncomp)

    def plan(self, level, items):
        return _DevicePlan(level, items)

    def zeros(self, n):
        return self.torch.zeros(n, dtype=self.torch.float64, device=self.device)

    def local_absmax(self, level, slab):
        """max |u| over this rank's valid cells (one reduction per patch)."""
        m = 0.0
        for p, off in zip(level.patches, level.offsets):
            g = p.grow(level.ghost)
            m = max(m, reduce(RED_ABS, slab[off:off + g.size()], g, region=p))
        return m


class _DevicePlan:
    def __init__(self, level, items):
        L = lib()
        n = len(items)
        arr = (pb_halo_item * max(n, 1))()
        for k, (patch, region, off) in enumerate(items):
            arr[k].patch = patch
            arr[k].region = _c(Box(*region))
            arr[k].offset = off
        h = ctypes.c_void_p()
        _check(L.pb_halo_plan_create(level._h, arr, _c_int(n), ctypes.byref(h)), "pb_halo_plan_create")
        self._lib = L        # kept for __del__, which may run while the interpreter shuts down
        self._h = h
        self.elems = L.pb_halo_plan_elems(h)

    def pack(self, slab, buf, stream=None):
        _check(lib().pb_halo_pack_f64(self._h, _ptr(slab), _ptr(buf), _stream(stream)), "pb_halo_pack_f64")

    def unpack(self, slab, buf, stream=None):
        _check(lib().pb_halo_unpack_f64(self._h, _ptr(slab), _ptr(buf), _stream(stream)), "pb_halo_unpack_f64")

    def __del__(self):
        if getattr(self, "_h", None) and getattr(self, "_lib", None) is not None:
            self._lib.pb_halo_plan_destroy(self._h)
            self._h = None


class pb_halo_item(ctypes.Structure):
    _fields_ = [("patch", ctypes.c_int), ("region", pb_box), ("offset", ctypes.c_longlong)]


# ---- the sharded level ----------------------------------------------------------------------------
class ShardedLevel:
    """This rank's share of a level (boxes: every patch of the level, ((lo), (hi)) tuples, the same
    list on every rank)."""

    def __init__(self, boxes, ghost, domain, periodic, rank, world, comm, backend=None, ncomp=1):
        self.backend = backend if backend is not None else DeviceBackend()
        self.boxes = [tuple(map(tuple, b)) for b in boxes]
        self.rank, self.world, self.comm = rank, world, comm
        self.owner = balance(index_points(self.boxes), world)
        self.mine = [i for i in range(len(self.boxes)) if self.owner[i] == rank]
        self.level = self.backend.level([self.boxes[i] for i in self.mine], ghost, domain, periodic, ncomp)
        hp = HaloPlan(self.boxes, ghost, domain, periodic, self.owner, rank, ncomp)
        self.send = {p: self.backend.plan(self.level, items) for p, items in hp.send.items()}
        self.recv = {p: self.backend.plan(self.level, items) for p, items in hp.recv.items()}
        self.sbuf = {p: self.backend.zeros(n) for p, n in hp.send_elems.items()}
        self.rbuf = {p: self.backend.zeros(n) for p, n in hp.recv_elems.items()}

    @property
    def slab_elems(self):
        return self.level.slab_elems

    @property
    def offsets(self):
        return self.level.offsets

    def pack(self, slab):
        """Local ghost exchange, then this rank's outgoing regions into the send buffers."""
        self.level.exchange(slab)
        for p, plan in self.send.items():
            plan.pack(slab, self.sbuf[p])

    def unpack(self, slab):
        for p, plan in self.recv.items():
            plan.unpack(slab, self.rbuf[p])

    def exchange(self, slab):
        """Every ghost cell of this rank's patches set to the valid cell at its periodic image."""
        self.pack(slab)
        if self.sbuf or self.rbuf:
            self.comm.exchange(self.sbuf, self.rbuf)   # NCCL orders itself after the pack on this stream
        self.unpack(slab)

    def step(self, stencil, u, tmp, scale, dt):
        """u + dt * S(u, scale) after an exchange, written to tmp (the caller swaps)."""
        self.exchange(u)
        self.level.stencil(stencil, EPI_EULER, u, tmp, scale=scale, a=dt)

    def absmax(self, slab):
        m = self.backend.local_absmax(self.level, slab)
        return self.comm.allreduce_max(m, getattr(self.backend, "device", "cpu"))


def exchange_all(ranks, slabs):
    """The exchange of every rank of one process (LocalComm): all ranks pack and post, then all take
    and unpack. Nothing on the device waits on another rank's work."""
    for r, s in zip(ranks, slabs):
        r.pack(s)
        r.comm.post(r.sbuf)
    for r, s in zip(ranks, slabs):
        r.comm.take(r.rbuf)
        r.unpack(s)
