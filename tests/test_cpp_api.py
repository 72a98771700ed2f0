"""The C++ API (proto_b200/cpp/Proto_B200.H), compiled with g++ like a reference caller would:
host algebra against the reference's tables (CPU), and the device forms against the oracle (GPU)."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests.util import table

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compile(src, exe):
    cmd = ["g++", "-std=c++17", "-O1", "-I" + ROOT, "-I/usr/local/cuda/include", os.path.join(ROOT, src), "-o", exe,
           "-L" + os.path.join(ROOT, "proto_b200", "lib"), "-lproto_b200", "-L/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "proto_b200", "lib")]
    subprocess.run(cmd, check=True, capture_output=True)


def test_host_tables_and_boxes_match_reference(golden, tmp_path):
    meta, arrays = golden
    exe = str(tmp_path / "api_tables")
    _compile("tests/cpp/api_tables.cpp", exe)
    out = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
    for name, t in out["stencils"].items():
        c, o, m = table(arrays, name)
        assert np.array_equal(np.array(t["coefs"]), c), name
        assert np.array_equal(np.array(t["offs"]).reshape(-1, 3), o), name
        assert list(t["meta"]) == list(m), name
    for got, exp in zip(out["box"], meta["box"]):
        assert got["coarsen"] == exp["coarsen"] and got["taper"] == exp["taper"] and got["refine"] == exp["refine"]
    assert out["avg_range"] == [[-2, -2, -2], [5, 5, 5]]


@pytest.mark.gpu
def test_device_forms_match_oracle(golden, pb, port, tmp_path):
    n = 24
    exe = str(tmp_path / "api_device")
    _compile("tests/cpp/api_device.cpp", exe)
    u = np.random.default_rng(77).uniform(-1, 1, (n + 2) ** 3)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    u.tofile(fin)
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(fout)
    c, o, m = table(golden[1], "laplacian")
    ub, b = ((-1,) * 3, (n,) * 3), ((0,) * 3, (n - 1,) * 3)
    h = 1.0 / n
    lu = np.zeros(n ** 3)
    port.stencil_apply(c, o.reshape(-1), m, u, ub, lu, b, b, True, 1.0 / (h * h))
    k = 0
    assert np.array_equal(got[k:k + n ** 3], lu)
    k += n ** 3
    inner = ((1,) * 3, (n - 2,) * 3)
    port.stencil_apply(c, o.reshape(-1), m, u, ub, lu, b, inner, False, 2.0)
    lu = lu * 0.5
    lu = lu + u.reshape(n + 2, n + 2, n + 2)[1:-1, 1:-1, 1:-1].reshape(-1)
    assert np.array_equal(got[k:k + n ** 3], lu)
    k += n ** 3
    ca, oa, ma = table(golden[1], "avgdown2")
    nc = n // 2
    cc = np.zeros(nc ** 3)
    port.stencil_apply(ca, oa.reshape(-1), ma, lu, b, cc, ((0,) * 3, (nc - 1,) * 3), ((0,) * 3, (nc - 1,) * 3), True, 1.0)
    assert np.array_equal(got[k:k + nc ** 3], cc)
    k += nc ** 3
    fine = np.zeros(n ** 3)
    port.interp_constant(2, cc, ((0,) * 3, (nc - 1,) * 3), fine, b, False, 1.0)
    assert np.array_equal(got[k:k + n ** 3], fine)
    k += n ** 3
    # exchange: every patch's ghost cells hold the periodic image
    U = u.reshape(n + 2, n + 2, n + 2)[1:-1, 1:-1, 1:-1]
    for pz in range(2):
        for py in range(2):
            for px in range(2):
                a = got[k:k + 14 ** 3].reshape(14, 14, 14)
                k += 14 ** 3
                zz = (np.arange(-1, 13) + 12 * pz) % n
                yy = (np.arange(-1, 13) + 12 * py) % n
                xx = (np.arange(-1, 13) + 12 * px) % n
                assert np.array_equal(a, U[np.ix_(zz, yy, xx)])
    # multigrid with the archived solver's parameters on rho = interior of u, 8 cycles
    rho = U.reshape(-1).copy()
    p2 = np.zeros(n ** 3)
    it, hist = port.mg_cs(n, 3, 6, 6, 10, 0.5, 1.0, None, 8, 1e-10, rho, p2)
    assert np.array_equal(got[k:k + n ** 3], p2)
    assert ("mg %d %.17g %.17g" % (it + 1, hist[0], hist[-1])) in r.stdout


def _nvcc(src, exe):
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--extended-lambda",
           "-fmad=false", "-I" + ROOT, "-I/usr/local/cuda/include", os.path.join(ROOT, src), "-o", exe,
           "-L" + os.path.join(ROOT, "proto_b200", "lib"), "-lproto_b200",
           "-Xlinker", "-rpath=" + os.path.join(ROOT, "proto_b200", "lib")]
    subprocess.run(cmd, check=True, capture_output=True)


def _patches(n, bs):
    """Patch boxes of DisjointBoxLayout(Cube(n), bs), in the layout's order (x fastest)."""
    m = n // bs
    return [((px * bs, py * bs, pz * bs), (px * bs + bs - 1, py * bs + bs - 1, pz * bs + bs - 1))
            for pz in range(m) for py in range(m) for px in range(m)]


def _valid_of(block, bs, g):
    s = bs + 2 * g
    return block.reshape(s, s, s)[g:g + bs, g:g + bs, g:g + bs] if g else block.reshape(s, s, s)


def _assemble(blocks, n, bs, g):
    full = np.zeros((n, n, n))
    for (lo, hi), b in zip(_patches(n, bs), blocks):
        full[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = _valid_of(b, bs, g)
    return full


@pytest.mark.gpu
def test_forall_boxop_levelop_and_solvers_match_oracle(golden, pb, port, tmp_path):
    """The forall family (reference tests/ForallTests.cpp shapes), BoxOp_Laplace, LevelOp with the
    library's operator and with a user operator plugged in, the archived LevelMultigrid driven by
    vCycle/resnorm and LevelMultigridSolver<BoxOp_Laplace> with the reference's signatures."""
    exe, fout = str(tmp_path / "api_forall"), str(tmp_path / "out.bin")
    _nvcc("tests/cpp/api_forall.cu", exe)
    r = subprocess.run([exe, fout], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(fout)
    k = [0]

    def take(cnt):
        a = out[k[0]:k[0] + cnt]
        k[0] += cnt
        return a

    gamma, phase = 1.4, np.pi / 4
    z, y, x = np.meshgrid(np.arange(4), np.arange(4), np.arange(4), indexing="ij")
    U = take(5 * 64).reshape(5, 4, 4, 4)
    for c in range(5):
        assert np.array_equal(U[c], 1.0 + 0.25 * c + 0.01 * (x + 2 * y + 3 * z))

    def cons_to_prim(U):
        rho = U[0]
        W = np.empty_like(U)
        W[0] = rho
        v2 = np.zeros_like(rho)
        for i in range(1, 4):
            v = U[i] / rho
            W[i] = v
            v2 = v2 + v * v
        W[4] = (U[4] - 0.5 * rho * v2) * (gamma - 1.0)
        return W

    Wr = cons_to_prim(U)
    assert np.array_equal(take(5 * 64).reshape(5, 4, 4, 4), Wr)
    assert np.array_equal(take(5 * 27).reshape(5, 3, 3, 3), Wr[:, :3, :3, :3])
    assert np.array_equal(take(5 * 27).reshape(5, 3, 3, 3), Wr[:, :3, :3, :3])
    W4 = take(5 * 27).reshape(5, 3, 3, 3)
    assert np.array_equal(W4[:, :2, :2, :2], Wr[:, :2, :2, :2])
    m = np.ones((3, 3, 3), bool)
    m[:2, :2, :2] = False
    assert np.all(W4[:, m] == -7.0)
    X = take(3 * 64).reshape(3, 4, 4, 4)
    for d, p in enumerate((x, y, z)):
        assert np.array_equal(X[d], 0.1 * p + 0.05 * d)
    Yr = np.sin(X[0] + phase) + np.sin(X[1] + phase) + np.sin(X[2] + phase) + 0.001 * (x + 10 * y + 100 * z)
    assert np.max(np.abs(take(64).reshape(4, 4, 4) - Yr)) < 1e-15
    assert np.max(np.abs(take(27).reshape(3, 3, 3) - Yr[:3, :3, :3])) < 1e-15
    Y3 = take(27).reshape(3, 3, 3)
    assert np.max(np.abs(Y3[:2, :2, :2] - Yr[:2, :2, :2])) < 1e-15 and np.all(Y3[m] == 3.0)
    assert np.array_equal(take(64).reshape(4, 4, 4), (0.5 * x - 0.25 * z) + 0.125 * 2.0)
    # BoxOp_Laplace on a box (flux scale -1, scale 0.5) against the C restatement (pinned to the
    # reference's BoxOp_Laplace in tests/test_oracle.py)
    n, dx = 12, 1.0 / 12
    phi = take(16 ** 3)
    gb, vb = ((-2,) * 3, (13,) * 3), ((0,) * 3, (11,) * 3)
    ref = np.zeros(n ** 3)
    port.boxop_laplace(phi, gb, ref, vb, vb, dx, -1.0, 0.5)
    assert np.array_equal(take(n ** 3), ref)
    # LevelOp over the periodic 2x2x2 layout of 6^3 patches, ghost 2
    P = phi.reshape(16, 16, 16)[2:14, 2:14, 2:14]
    Pg = np.pad(P, 2, mode="wrap").reshape(-1).copy()
    lap = np.zeros(n ** 3)
    port.boxop_laplace(Pg, gb, lap, vb, vb, dx, 1.0, 1.0)
    got = _assemble([take(1000) for _ in range(8)], n, 6, 2)
    assert np.array_equal(got.reshape(-1), lap)
    c7, o7, m7 = table(golden[1], "laplacian")
    lap7 = np.zeros(n ** 3)
    port.stencil_apply(c7, o7.reshape(-1), m7, Pg, gb, lap7, vb, vb, True, 1.0 / (dx * dx))
    got7 = _assemble([take(1000) for _ in range(8)], n, 6, 2)
    assert np.array_equal(got7.reshape(-1), lap7)
    # the archived LevelMultigrid: resnorm, then vCycle + resnorm until 1e-10, at most 6 cycles
    N = 32
    rho = _assemble([take(16 ** 3) for _ in range(8)], N, 16, 0).reshape(-1).copy()
    psi = _assemble([take(18 ** 3) for _ in range(8)], N, 16, 1).reshape(-1)
    p2 = np.zeros(N ** 3)
    it, hist = port.mg_cs(N, 3, 6, 6, 10, 0.5, 1.0, None, 6, 1e-10, rho, p2)
    lines = [l.split() for l in r.stdout.splitlines() if l.startswith("mg res")]
    assert [float(l[3]) for l in lines] == list(hist)
    assert np.array_equal(psi, p2)
    # LevelMultigridSolver<BoxOp_Laplace, double>: FAS, 4 levels, force = rho
    st = _assemble([take(20 ** 3) for _ in range(8)], N, 16, 2).reshape(-1)
    p3 = np.zeros(N ** 3)
    it3, hist3 = port.mg_fas(N, 4, 8, 1e-10, rho, p3)
    lines = [l.split() for l in r.stdout.splitlines() if l.startswith("fas res")]
    assert [float(l[3]) for l in lines] == list(hist3)
    assert np.array_equal(st, p3)
    assert k[0] == out.size


@pytest.mark.gpu
def test_interp_stencils_match_reference_golden(golden, pb, tmp_path):
    """InterpStencil Constant (the fused kernel), Linear and Quadratic (the 1-D stages of the
    reference through the device stencil engine) against the reference's own outputs."""
    from tests.util import box_vol
    meta, arrays = golden
    exe = str(tmp_path / "api_interp")
    _compile("tests/cpp/api_interp.cpp", exe)
    kinds = set()
    for k, case in enumerate(meta["interp"]):
        rng = np.random.default_rng(case["seed"])
        src = rng.uniform(-1, 1, box_vol(case["src"]))
        dst = rng.uniform(-1, 1, box_vol(case["dst"]))
        fs, fd, fo = (str(tmp_path / ("%s%d.bin" % (t, k))) for t in ("s", "d", "o"))
        src.tofile(fs)
        dst.tofile(fd)
        args = [str(case.get("kind", 0)), str(case["ratio"])] + [str(v) for b in case["src"] for v in b] + \
               [str(v) for b in case["dst"] for v in b] + [str(int(case["overwrite"])), repr(case["scale"]), fs, fd, fo]
        r = subprocess.run([exe] + args, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert np.array_equal(np.fromfile(fo), arrays["interp_%d" % k]), k
        kinds.add(case.get("kind", 0))
    assert kinds == {0, 1, 2}
