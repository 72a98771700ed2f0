"""The CPU oracle (C restatement) against the reference's golden fixtures, and against the
reference-built library where it exists. CPU only."""
import numpy as np
import pytest

from proto_b200 import workloads as W
from tests.util import apply_inputs, box_vol, digest, table


def test_stencil_tables_present(golden):
    meta, arrays = golden
    assert meta["stencils"]["laplacian"] == 7
    assert meta["stencils"]["laplacian13"] == 13
    c, o, m = table(arrays, "laplacian13")
    # sum_d Derivative(2,d,4): +x,0,-x,+2x,-2x,+y,-y,+2y,-2y,+z,-z,+2z,-2z, centre merged
    assert [tuple(v) for v in o[:5]] == [(1, 0, 0), (0, 0, 0), (-1, 0, 0), (2, 0, 0), (-2, 0, 0)]
    assert c[1] == -7.5


@pytest.mark.parametrize("k", range(13))
def test_port_stencil_apply_bitwise(golden, port, k):
    meta, arrays = golden
    case = meta["apply"][k]
    c, o, m = table(arrays, case["stencil"])
    src, dst = apply_inputs(case)
    ib = port.infer_box(o.reshape(-1), m, case["src"], case["dst"])
    port.stencil_apply(c, o.reshape(-1), m, src, case["src"], dst, case["dst"], ib, case["mode"] == 0, case["scale"])
    assert np.array_equal(dst, arrays["apply_%d" % k])


def test_port_plain_method(golden, port):
    g = golden[0]["plain"]
    u = W.plain_input(g["n"], g["seed"]).reshape(-1).copy()
    out = np.zeros(g["n"] ** 3)
    port.plain_apply(g["n"], u, out, g["h"], g["a"], g["b"])
    assert digest(out) == g["sha256"]


def test_port_reductions(golden, port):
    meta, _ = golden
    d = np.random.default_rng(41).uniform(-1, 1, 1001)
    assert [port.reduce(op, d) for op in range(6)] == meta["reduce"]["mixed"]
    assert [port.reduce(op, -np.abs(d)) for op in range(6)] == meta["reduce"]["negative"]
    # the reference's Max starts from numeric_limits<double>::min(), the smallest positive normal
    assert meta["reduce"]["negative"][0] == np.finfo(np.float64).tiny


@pytest.mark.parametrize("k", range(3))
def test_port_interp(golden, port, k):
    meta, arrays = golden
    case = meta["interp"][k]
    rng = np.random.default_rng(case["seed"])
    src = rng.uniform(-1, 1, box_vol(case["src"]))
    dst = rng.uniform(-1, 1, box_vol(case["dst"]))
    port.interp_constant(case["ratio"], src, case["src"], dst, case["dst"], case["overwrite"], case["scale"])
    assert np.array_equal(dst, arrays["interp_%d" % k])


def _exchange_port(port, dom, per, bs, g, valid):
    npch = [dom[d] // bs[d] for d in range(3)]
    V = valid.reshape(dom[2], dom[1], dom[0])
    boxes, datas = [], []
    for pz in range(npch[2]):
        for py in range(npch[1]):
            for px in range(npch[0]):
                lo = (px * bs[0], py * bs[1], pz * bs[2])
                hi = tuple(lo[d] + bs[d] - 1 for d in range(3))
                boxes.append(lo + hi)
                a = np.full((bs[2] + 2 * g[2], bs[1] + 2 * g[1], bs[0] + 2 * g[0]), -777.0)
                a[g[2]:g[2] + bs[2], g[1]:g[1] + bs[1], g[0]:g[0] + bs[0]] = \
                    V[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
                datas.append(a.reshape(-1).copy())
    port.exchange(boxes, g, ((0, 0, 0), tuple(d - 1 for d in dom)), per, datas)
    return np.concatenate(datas)


@pytest.mark.parametrize("k", range(4))
def test_port_exchange(golden, port, k):
    case = golden[0]["exchange"][k]
    valid = np.random.default_rng(case["seed"]).uniform(-1, 1, int(np.prod(case["domain"])))
    out = _exchange_port(port, case["domain"], case["periodic"], case["box"], case["ghost"], valid)
    assert digest(out) == case["sha256"]


@pytest.mark.parametrize("name", ["archived_32", "cs_v22_32", "cs_v22_64", "helm_v22_32"])
def test_port_multigrid_history_bitwise(golden, port, name):
    cfg = golden[0]["mg"][name]
    N = cfg["N"]
    rho = W.poisson_rho(N, seed=1).reshape(-1).copy()
    phi = np.zeros(N ** 3)
    if cfg["kind"] == "archived":
        # the archived driver's numLevels counts coarsenings: levels numLevels..0
        n, h = port.mg_cs(N, cfg["numLevels"], 6, 6, 10, 0.5, 1.0, None, cfg["maxIter"], cfg["tol"], rho, phi)
    elif cfg["kind"] == "cs":
        n, h = port.mg_cs(N, cfg["levels"], cfg["nu1"], cfg["nu2"], cfg["nub"], cfg["omega"], 1.0, None,
                          cfg["maxIter"], cfg["tol"], rho, phi)
    else:
        alpha = W.helmholtz_alpha(N, seed=3).reshape(-1).copy()
        n, h = port.mg_cs(N, cfg["levels"], cfg["nu1"], cfg["nu2"], cfg["nub"], cfg["omega"], 1.0, alpha,
                          cfg["maxIter"], cfg["tol"], -rho, phi)
    assert n == cfg["iters"]
    assert list(h) == cfg["hist"]
    assert digest(phi) == cfg["phi_sha256"]


def test_port_level13(golden, port):
    g = golden[0]["level13"]
    boxes, L = W.amr_patches(g["widths"])
    gh = g["ghost"]
    u = W.uniform_box((L[2], L[1], L[0]), g["seed"])
    G = np.zeros((L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh))
    G[gh:-gh, gh:-gh, gh:-gh] = u
    G = G.reshape(-1).copy()
    c, o, m = table(golden[1], "laplacian13")
    port.periodic_steps(L, gh, c, o.reshape(-1), g["h"], g["dt"], g["steps"], G)
    G = G.reshape(L[2] + 2 * gh, L[1] + 2 * gh, L[0] + 2 * gh)[gh:-gh, gh:-gh, gh:-gh]
    parts = [G[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1].reshape(-1) for lo, hi in boxes]
    assert digest(np.concatenate(parts)) == g["sha256"]


def test_port_box_ops(golden):
    from oracle.oracle import Port  # noqa: F401  (box math is restated in the library's own host code too)
    import ctypes
    import os
    lib = ctypes.CDLL(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "liboracle.so"))
    for case in golden[0]["box"]:
        lo = (ctypes.c_int * 3)(*case["lo"])
        hi = (ctypes.c_int * 3)(*case["hi"])
        r = (ctypes.c_int * 3)(*case["ratio"])
        olo, ohi = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        lib.or_box_coarsen(lo, hi, r, olo, ohi)
        assert [list(olo), list(ohi)] == case["coarsen"]
        lib.or_box_taper_coarsen(lo, hi, r, olo, ohi)
        assert [list(olo), list(ohi)] == case["taper"]


def test_port_matches_reference_live(ref, port):
    """Where the reference-built library exists, check a fresh seeded case directly."""
    rng = np.random.default_rng(99)
    c, o, m = ref.stencil_table(2)
    sb, db = ((-2, -1, -3), (9, 8, 7)), ((-1, 0, -2), (8, 7, 6))
    src = rng.uniform(-1, 1, box_vol(sb))
    d1 = rng.uniform(-1, 1, box_vol(db))
    d2 = d1.copy()
    ref.stencil_apply(c, o, m, src, sb, d1, db, 1, 0.7)
    ib = port.infer_box(o.reshape(-1), m, sb, db)
    port.stencil_apply(c, o.reshape(-1), m, src, sb, d2, db, ib, False, 0.7)
    assert np.array_equal(d1, d2)


def test_port_fas_bitwise(golden, port):
    """The C restatement of LevelMultigridSolver<BoxOp_Laplace> (FAS, 4th-order flux form) against
    the reference's own history and solution."""
    cfg = golden[0]["mg"]["fas_32"]
    N = cfg["N"]
    rho = W.poisson_rho(N, seed=1).reshape(-1).copy()
    phi = np.zeros(N ** 3)
    n, h = port.mg_fas(N, cfg["numLevels"], cfg["maxIter"], cfg["tol"], -rho, phi)
    assert n == cfg["iters"]
    assert list(h) == cfg["hist"]
    assert digest(phi) == cfg["phi_sha256"]


def test_boxop_laplace_port_matches_reference(port):
    """The C restatement of BoxOp_Laplace::operator() (flux form, flux scale, scale) against the
    reference's own operator on an offset box."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference-built oracle not present")
    R = Ref()
    rng = np.random.default_rng(3)
    sb, ob = ((-2, -1, -3), (13, 12, 10)), ((0, 1, -1), (11, 10, 8))
    u = rng.uniform(-1, 1, int(np.prod([sb[1][d] - sb[0][d] + 1 for d in range(3)])))
    nout = int(np.prod([ob[1][d] - ob[0][d] + 1 for d in range(3)]))
    for fs, sc in ((1.0, 1.0), (-1.0, 1.0), (-1.0, 0.37)):
        a, b = np.zeros(nout), np.zeros(nout)
        port.boxop_laplace(u, sb, a, ob, ob, 1.0 / 16, fs, sc)
        R.boxop_laplace(u, sb, b, ob, 1.0 / 16, fs, sc)
        assert np.array_equal(a, b)
