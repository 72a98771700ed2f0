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
