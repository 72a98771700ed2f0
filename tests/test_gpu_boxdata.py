"""BoxData algebra, copyTo, reductions and constant prolongation on the GPU."""
import numpy as np
import pytest

from tests.util import box_vol

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(-1)).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_binary_ops_on_box_intersection(pb):
    rng = np.random.default_rng(1)
    db, sb = ((-2, -1, 0), (5, 6, 4)), ((0, -3, 1), (8, 3, 7))
    for op in range(5):
        d = rng.uniform(1, 2, box_vol(db))
        s = rng.uniform(1, 2, box_vol(sb))
        dd = _dev(d)
        pb.boxdata_op(op, dd, pb.Box(*db), _dev(s), pb.Box(*sb))
        D = d.reshape(5, 8, 8).copy()
        S = s.reshape(7, 7, 9)
        lo = [max(db[0][k], sb[0][k]) for k in range(3)]
        hi = [min(db[1][k], sb[1][k]) for k in range(3)]
        dsl = tuple(slice(lo[k] - db[0][k], hi[k] - db[0][k] + 1) for k in (2, 1, 0))
        ssl = tuple(slice(lo[k] - sb[0][k], hi[k] - sb[0][k] + 1) for k in (2, 1, 0))
        if op == 0: D[dsl] = D[dsl] + S[ssl]
        if op == 1: D[dsl] = D[dsl] - S[ssl]
        if op == 2: D[dsl] = D[dsl] * S[ssl]
        if op == 3: D[dsl] = D[dsl] / S[ssl]
        if op == 4: D[dsl] = S[ssl]
        assert np.array_equal(_host(dd), D.reshape(-1))


def test_scalar_ops_and_setval(pb):
    rng = np.random.default_rng(2)
    b = ((0, 0, 0), (6, 5, 4))
    d = rng.uniform(-1, 1, box_vol(b))
    dd = _dev(d)
    pb.boxdata_scalar(pb.OP_MUL, dd, pb.Box(*b), 3.5)
    pb.boxdata_scalar(pb.OP_ADD, dd, pb.Box(*b), -0.25, region=pb.Box((1, 1, 1), (3, 3, 3)))
    D = d.reshape(5, 6, 7) * 3.5
    D[1:4, 1:4, 1:4] = D[1:4, 1:4, 1:4] + (-0.25)
    assert np.array_equal(_host(dd), D.reshape(-1))
    pb.boxdata_scalar(pb.OP_ASSIGN, dd, pb.Box(*b), 0.0)
    assert np.abs(_host(dd)).max() == 0.0


def test_copy_with_shift(pb):
    rng = np.random.default_rng(3)
    sb, db = ((0, 0, 0), (7, 7, 7)), ((-4, -4, -4), (11, 11, 11))
    s = rng.uniform(-1, 1, box_vol(sb))
    d = np.zeros(box_vol(db))
    dd = _dev(d)
    pb.boxdata_copy(_dev(s), pb.Box(*sb), dd, pb.Box(*db), pb.Box((1, 2, 3), (5, 6, 7)), shift=(-3, 2, 4))
    D = d.reshape(16, 16, 16)
    S = s.reshape(8, 8, 8)
    # dst(p + shift) = src(p) for p in region; p+shift must lie in dst box: z 3..7 -> 7..11
    for z in range(3, 8):
        for y in range(2, 7):
            for x in range(1, 6):
                D[z + 4 + 4, y + 2 + 4, x - 3 + 4] = S[z, y, x]
    assert np.array_equal(_host(dd), D.reshape(-1))


def test_reductions_match_reference(golden, pb):
    meta = golden[0]["reduce"]
    d = np.random.default_rng(41).uniform(-1, 1, 1001)
    b = pb.Box((0, 0, 0), (1000, 0, 0))
    for key, arr in [("mixed", d), ("negative", -np.abs(d))]:
        t = _dev(arr)
        got = [pb.reduce(op, t, b) for op in range(6)]
        exp = meta[key]
        assert got[0] == exp[0] and got[1] == exp[1] and got[2] == exp[2]     # exact
        for k in (3, 4, 5):                                                    # reassociated sums
            assert abs(got[k] - exp[k]) <= 1e-13 * max(1.0, abs(exp[k]))


def test_reduction_on_subregion_and_large(pb):
    import torch
    rng = np.random.default_rng(9)
    n = 200
    a = rng.uniform(-1, 1, n ** 3)
    t = _dev(a)
    b = pb.Box.cube(n)
    r = pb.Box((10, 20, 30), (150, 160, 170))
    A = a.reshape(n, n, n)[30:171, 20:161, 10:151]
    assert pb.reduce(pb.RED_ABS, t, b, region=r) == np.abs(A).max()
    assert pb.reduce(pb.RED_MAX, t, b) == a.max()
    s = pb.reduce(pb.RED_SUM, t, b)
    assert abs(s - a.sum()) < 1e-10
    # deterministic run to run
    assert all(pb.reduce(pb.RED_SUM, t, b) == s for _ in range(3))


@pytest.mark.parametrize("k", range(3))
def test_interp_constant_golden(golden, pb, k):
    meta, arrays = golden
    case = meta["interp"][k]
    rng = np.random.default_rng(case["seed"])
    src = rng.uniform(-1, 1, box_vol(case["src"]))
    dst = rng.uniform(-1, 1, box_vol(case["dst"]))
    dd = _dev(dst)
    pb.interp_constant(case["ratio"], _dev(src), pb.Box(*case["src"]), dd, pb.Box(*case["dst"]),
                       overwrite=case["overwrite"], scale=case["scale"])
    assert np.array_equal(_host(dd), arrays["interp_%d" % k])
