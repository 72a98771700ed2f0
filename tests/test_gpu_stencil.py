"""Stencil::apply through the C ABI on the GPU against the reference's golden outputs, bitwise."""
import numpy as np
import pytest

from proto_b200 import workloads as W
from tests.util import apply_inputs, box_shape, digest, table

pytestmark = pytest.mark.gpu


def _dev(a, shape=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(-1)).cuda()
    return t


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("k", range(13))
def test_golden_apply_cases(golden, pb, k):
    meta, arrays = golden
    case = meta["apply"][k]
    c, o, m = table(arrays, case["stencil"])
    S = pb.Stencil(c, o, tuple(m[:3]), tuple(m[3:6]), tuple(m[6:9]))
    src, dst = apply_inputs(case)
    ds, dd = _dev(src), _dev(dst)
    S.apply(ds, pb.Box(*case["src"]), dd, pb.Box(*case["dst"]), init_to_zero=case["mode"] == 0,
            scale=case["scale"])
    pb.device_check()
    assert np.array_equal(_host(dd), arrays["apply_%d" % k])


def test_plain_method_fused_and_unfused(golden, pb):
    g = golden[0]["plain"]
    n = g["n"]
    c, o, m = table(golden[1], "laplacian")
    S = pb.Stencil(c, o)
    u = _dev(W.plain_input(n, g["seed"]))
    ub, ob = pb.Box.cube(n).grow(1), pb.Box.cube(n)
    import torch
    out = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    S.apply_fused(pb.EPI_AXPBY, u, ub, out, ob, scale=1.0 / (g["h"] * g["h"]), a=g["a"], b=g["b"])
    assert digest(_host(out)) == g["sha256"]
    # the reference's own two-pass form: Lu |= L(u, 1/h^2); out = a*Lu + b*u
    lu = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    S.apply(u, ub, lu, ob, scale=1.0 / (g["h"] * g["h"]))
    out2 = torch.zeros_like(out)
    pb.forall_axpby(out2, ob, lu, ob, u, ub, g["a"], g["b"])
    assert digest(_host(out2)) == g["sha256"]


@pytest.mark.parametrize("name,n,ghost,mode,scale", [
    ("laplacian", 256, 1, 0, 65536.0),     # the north-star box: TMA z-streaming kernel
    ("laplacian", 96, 1, 1, 0.25),         # accumulate form
    ("laplacian13", 128, 2, 0, 1.0),
    ("laplacian", 84, 3, 0, 3.0),          # odd halo offset inside the source box (TMA kernel)
])
def test_large_boxes_match_oracle(golden, pb, port, name, n, ghost, mode, scale):
    c, o, m = table(golden[1], name)
    S = pb.Stencil(c, o)
    sb = ((-ghost,) * 3, (n - 1 + ghost,) * 3)
    db = ((0, 0, 0), (n - 1, n - 1, n - 1))
    rng = np.random.default_rng(n + ghost)
    src = rng.uniform(-1, 1, (n + 2 * ghost) ** 3)
    dst = rng.uniform(-1, 1, n ** 3)
    ds, dd = _dev(src), _dev(dst)
    S.apply(ds, pb.Box(*sb), dd, pb.Box(*db), init_to_zero=mode == 0, scale=scale)
    pb.device_check()
    ib = port.infer_box(o.reshape(-1), m, sb, db)
    port.stencil_apply(c, o.reshape(-1), m, src, sb, dst, db, ib, mode == 0, scale)
    assert np.array_equal(_host(dd), dst)


def test_tma_and_simple_paths_agree(golden, pb, port):
    """Same input through the TMA kernel (large box) and, for a sub-box, the simple kernel."""
    c, o, m = table(golden[1], "laplacian")
    S = pb.Stencil(c, o)
    n = 130
    sb = ((-1, -1, -1), (n, n, n))
    rng = np.random.default_rng(7)
    src = rng.uniform(-1, 1, (n + 2) ** 3)
    ds = _dev(src)
    import torch
    d1 = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    S.apply(ds, pb.Box(*sb), d1, pb.Box.cube(n))
    small = pb.Box((3, 5, 7), (20, 9, 12))
    d2 = torch.zeros(small.size(), dtype=torch.float64, device="cuda")
    S.apply(ds, pb.Box(*sb), d2, small)
    a = _host(d1).reshape(n, n, n)[7:13, 5:10, 3:21]
    assert np.array_equal(a.reshape(-1), _host(d2))


def test_tiny_and_negative_boxes(golden, pb, port):
    c, o, m = table(golden[1], "laplacian27")
    S = pb.Stencil(c, o)
    for db in [((0, 0, 0), (0, 0, 0)), ((-3, -2, -5), (-2, -1, -5)), ((4, -1, 0), (4, 6, 1))]:
        sb = (tuple(v - 1 for v in db[0]), tuple(v + 1 for v in db[1]))
        rng = np.random.default_rng(3)
        src = rng.uniform(-1, 1, int(np.prod([sb[1][d] - sb[0][d] + 1 for d in range(3)])))
        dst = rng.uniform(-1, 1, int(np.prod([db[1][d] - db[0][d] + 1 for d in range(3)])))
        dd = _dev(dst)
        S.apply(_dev(src), pb.Box(*sb), dd, pb.Box(*db), scale=2.0)
        ib = port.infer_box(o.reshape(-1), m, sb, db)
        port.stencil_apply(c, o.reshape(-1), m, src, sb, dst, db, ib, True, 2.0)
        assert np.array_equal(_host(dd), dst)


def test_multicomponent(golden, pb, port):
    c, o, m = table(golden[1], "laplacian")
    S = pb.Stencil(c, o)
    sb, db = ((-1, -1, -1), (8, 9, 10)), ((0, 0, 0), (7, 8, 9))
    rng = np.random.default_rng(5)
    src = rng.uniform(-1, 1, 3 * 10 * 11 * 12)
    dst = rng.uniform(-1, 1, 3 * 8 * 9 * 10)
    dd = _dev(dst)
    S.apply(_dev(src), pb.Box(*sb), dd, pb.Box(*db), init_to_zero=False, scale=1.5, ncomp=3)
    ib = port.infer_box(o.reshape(-1), m, sb, db)
    port.stencil_apply(c, o.reshape(-1), m, src, sb, dst, db, ib, False, 1.5, ncomp=3)
    assert np.array_equal(_host(dd), dst)


def test_scale_zero_and_empty(golden, pb):
    import torch
    c, o, m = table(golden[1], "laplacian")
    S = pb.Stencil(c, o)
    src = torch.ones(10 ** 3, dtype=torch.float64, device="cuda")
    dst = torch.full((8 ** 3,), 5.0, dtype=torch.float64, device="cuda")
    S.apply(src, pb.Box.cube(10, -1), dst, pb.Box.cube(8), init_to_zero=False, scale=0.0)
    assert float(dst.min()) == 5.0 and float(dst.max()) == 5.0
    S.apply(src, pb.Box.cube(10, -1), dst, pb.Box.cube(8), init_to_zero=True, scale=0.0)
    assert float(dst.abs().max()) == 0.0


def test_insufficient_ghost_is_an_error(golden, pb):
    import torch
    c, o, m = table(golden[1], "laplacian")
    S = pb.Stencil(c, o)
    src = torch.ones(8 ** 3, dtype=torch.float64, device="cuda")
    dst = torch.zeros(8 ** 3, dtype=torch.float64, device="cuda")
    with pytest.raises(pb.ProtoError) as e:
        S.apply(src, pb.Box.cube(8), dst, pb.Box.cube(8), box=pb.Box.cube(8))
    assert e.value.status == -9


def test_fp32_against_torch_reference(golden, pb):
    """FP32 apply against a plain PyTorch fp32 evaluation of the same terms (same order)."""
    import torch
    c, o, m = table(golden[1], "laplacian13")
    S = pb.Stencil(c, o)
    n, g = 80, 2
    rng = np.random.default_rng(11)
    src = torch.from_numpy(rng.uniform(-1, 1, (n + 2 * g,) * 3).astype(np.float32)).cuda()
    dst = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    S.apply(src, pb.Box.cube(n + 2 * g, -g), dst, pb.Box.cube(n), scale=3.0)
    ref = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    for cj, (ox, oy, oz) in zip(c, o):
        ref = ref + (np.float32(cj) * np.float32(3.0)) * src[g + oz:g + oz + n, g + oy:g + oy + n, g + ox:g + ox + n]
    torch.cuda.synchronize()
    assert torch.equal(ref, dst) or float((ref - dst).abs().max() / ref.abs().max()) < 1e-6
