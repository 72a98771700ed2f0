"""The C-ABI library loads, exports every symbol the header declares, and validates arguments on
the host (no GPU work). CPU only."""
import ctypes

import pytest

import proto_b200 as pb


def test_library_exports_header_symbols():
    L = pb.lib()
    names = pb.header_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def test_version_and_status_strings():
    assert b"sm_100a" in pb.lib().pb_version()
    assert pb.status_string(0) == "ok"
    assert "footprint" in pb.status_string(-9)


def test_stencil_create_and_shape_detection(golden):
    from tests.util import table
    _, arrays = golden
    for name, shape in [("laplacian", 1), ("laplacian13", 2), ("laplacian27", 0), ("avgdown2", 0)]:
        c, o, m = table(arrays, name)
        s = pb.Stencil(c, o, tuple(m[:3]), tuple(m[3:6]), tuple(m[6:9]))
        n, span, sh = s.info()
        assert n == len(c) and sh == shape
    c, o, m = table(arrays, "laplacian13")
    n, span, sh = pb.Stencil(c, o).info()
    assert span.lo == (-2, -2, -2) and span.hi == (2, 2, 2)


def test_stencil_reordered_is_not_specialised(golden):
    from tests.util import table
    c, o, m = table(golden[1], "laplacian")
    # same terms, different insertion order: a different summation order, so the table kernel
    s = pb.Stencil(c[::-1].copy(), o[::-1].copy())
    assert s.info()[2] == 0


def test_argument_errors():
    L = pb.lib()
    h = ctypes.c_void_p()
    c = (ctypes.c_double * 1)(1.0)
    o = (ctypes.c_int * 3)(0, 0, 0)
    bad_ratio = (ctypes.c_int * 3)(0, 1, 1)
    assert L.pb_stencil_create(c, o, 1, bad_ratio, None, None, ctypes.byref(h)) == -1
    assert L.pb_stencil_create(None, None, 1, None, None, None, ctypes.byref(h)) == -1
    with pytest.raises(pb.ProtoError):
        pb.Multigrid(pb.MGParams(n=48, levels=5))
    assert pb.MGParams(n=48, levels=5).device_bytes() == -1
    assert pb.MGParams(n=256, levels=6).device_bytes() > 256 ** 3 * 8 * 3


def test_launch_shape_knobs_validate():
    L = pb.lib()
    L.pb_star_tune_set.argtypes = [ctypes.c_int] * 5 + [ctypes.c_longlong]
    assert L.pb_star_tune_set(0, 0, 8, 3, 1, -1) == -1        # rows per thread must divide the tile
    assert L.pb_star_tune_set(0, 0, 12, 1, 1, -1) == -1
    assert L.pb_star_tune_set(0, 0, 8, 1, 2, -1) == -1
    assert L.pb_star_tune_set(0, 0, 8, 2, 3, -1) == -1
    assert L.pb_star_tune_set(3, 0, 8, 2, 2, -1) == -1
    assert L.pb_star_tune_ring(2, 1) == -1                    # fewer planes than a 7-point window
    assert L.pb_star_tune_ring(17, 1) == -1
    assert L.pb_star_tune_ring(0, 2) == -1
    for ty, yb, xv in ((8, 1, 1), (8, 2, 1), (4, 2, 2), (8, 2, 2)):
        assert L.pb_star_tune_set(0, 0, ty, yb, xv, -1) == 0
    assert L.pb_star_tune_ring(0, 1) == 0


def test_multigrid_parameter_rules():
    P = pb.MGParams
    # exact bottom: at most 512 coarsest cells
    assert P(n=256, levels=5, bottom=pb.MG_BOTTOM_DIRECT).device_bytes() > 0
    assert P(n=256, levels=4, bottom=pb.MG_BOTTOM_DIRECT).device_bytes() == -1
    assert P(n=64, levels=3, bottom=2).device_bytes() == -1
    # mixed precision fuses a pre- and a post-sweep of the finest grid and needs a coarse grid
    assert P(n=64, levels=3, precision=pb.MG_MIXED).device_bytes() > 0
    assert P(n=64, levels=3, nu1=0, precision=pb.MG_MIXED).device_bytes() == -1
    assert P(n=64, levels=3, nu2=0, precision=pb.MG_MIXED).device_bytes() == -1
    assert P(n=64, levels=0, precision=pb.MG_MIXED).device_bytes() == -1
    # mixed holds FP32 levels (two buffers + rhs: 12 B/cell) plus the FP64 solution and
    # right-hand side (16 B/cell) against FP64's 24 B/cell
    n = 256
    b64 = P(n=n, levels=6).device_bytes()
    bmx = P(n=n, levels=6, precision=pb.MG_MIXED).device_bytes()
    assert b64 > 24 * n ** 3 and bmx > 28 * n ** 3
    assert bmx - b64 < 6 * n ** 3
    L = pb.lib()
    lp = L.pb_mg_launches_per_cycle
    try:
        # one launch per step: (nu1 + nu2 + 2) per level above the coarsest, the bottom, the norm;
        # with nu1 >= 1 the FP64 norm rides on the next cycle's first sweep (two-sweep passes off;
        # where a GPU runs them, they are counted in test_gpu_relax2.py)
        assert L.pb_mg_relax2_min_edge(0) == 0
        assert L.pb_mg_coarse_edge(0) == 0
        assert lp(ctypes.byref(P(n=256, levels=6, nu1=4, nu2=4, nu_bottom=10).c)) == 6 * 10 + 10
        assert lp(ctypes.byref(P(n=256, levels=6, nu1=0, nu2=4, nu_bottom=10).c)) == 6 * 6 + 10 + 1
        assert lp(ctypes.byref(P(n=256, levels=5, nu1=4, nu2=4, bottom=1).c)) == 5 * 10 + 1
        assert lp(ctypes.byref(P(n=256, levels=6, nu1=4, nu2=4, nu_bottom=10, precision=pb.MG_MIXED).c)) == 6 * 10 + 10
        # levels of edge <= 16 (16, 8, 4 here) as one launch
        assert L.pb_mg_coarse_edge(16) == 0
        assert lp(ctypes.byref(P(n=256, levels=6, nu1=4, nu2=4, nu_bottom=10).c)) == 4 * 10 + 1
        assert lp(ctypes.byref(P(n=256, levels=6, nu1=4, nu2=4, precision=pb.MG_MIXED).c)) == 4 * 10 - 1 + 1 + 1
        # the finest grid always runs step by step, even when its edge is small
        assert lp(ctypes.byref(P(n=16, levels=2, nu1=4, nu2=4, nu_bottom=10).c)) == 1 * 10 + 1
        assert L.pb_mg_coarse_edge(-1) == -1
    finally:
        L.pb_mg_coarse_edge(8)
        L.pb_mg_relax2_min_edge(128)


def test_serve_host_rules():
    L = pb.lib()
    assert pb.Serve.request_bytes(33) == -1          # 33 does not halve down to <= 16
    assert pb.Serve.request_bytes(15) == -1          # the top level must coarsen once
    assert pb.Serve.request_bytes(16) > 0
    assert pb.Serve.request_bytes(16 * 12) > 8 * 192 ** 3 * 2
    assert pb.Serve.request_bytes(64) < pb.Serve.request_bytes(128)
    h = ctypes.c_void_p()
    bad = pb.pb_serve_params(1 << 30, 0, 4, 4, 10, 2.0 / 3.0, 1e-8, 100, pb.MG_MIXED)   # no slots
    assert L.pb_serve_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = pb.pb_serve_params(1 << 30, 4, 0, 4, 10, 2.0 / 3.0, 1e-8, 100, pb.MG_MIXED)   # nu1 = 0
    assert L.pb_serve_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = pb.pb_serve_params(0, 4, 4, 4, 10, 2.0 / 3.0, 1e-8, 100, pb.MG_MIXED)   # no budget
    assert L.pb_serve_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = pb.pb_serve_params(1 << 30, 4, 4, 4, 10, 2.0 / 3.0, 1e-8, 100, 7)  # no such precision
    assert L.pb_serve_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = pb.pb_serve_params(1 << 30, 4, 4, 3, 10, 2.0 / 3.0, 1e-8, 100, pb.MG_FP64)   # FP64: nu1 + nu2 odd
    assert L.pb_serve_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    # an FP64 hierarchy: every level in FP64 (the top level is the solution), no FP32 copies
    n = 64
    lv = sum(8 * (((e + 2 + 1) // 2 * 2) * (e + 2) ** 2 * 2 + e ** 3) for e in (64, 32))
    assert pb.Serve.request_bytes(n, pb.MG_FP64) > lv
    assert pb.Serve.request_bytes(33, pb.MG_FP64) == -1
    assert L.pb_serve_hierarchy_bytes(64, 7) == -1
    assert pb.Serve.request_bytes(64) == L.pb_serve_request_bytes(64)


def test_wait_expiry_hook_validates_arguments():
    L = pb.lib()
    e = ctypes.c_int()
    assert L.pb_debug_wait_expiry(ctypes.c_uint(0), ctypes.byref(e), None) == -1
    assert L.pb_debug_wait_expiry(ctypes.c_uint(1000), None, None) == -1
    assert L.pb_debug_wait_expiry(ctypes.c_uint((1 << 24) + 1), ctypes.byref(e), None) == -1
