"""The allocation-free reduction entry point, called through the C ABI.

pb_reduce_noalloc_f64 exists for callers that cannot let the library call cudaMalloc (for example
while a CUDA stream is being captured into a graph, or when device memory belongs to another
allocator). It keeps its scratch in a static device array, so it must agree with the ordinary
pb_reduce_f64 entry point on the same data, call after call (the shared scratch is reused).
This file is collected last so that a failure here comes after every other test has run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _box(lo, hi):
    import proto_b200 as pb
    return pb.Box(lo, hi).c()


def test_noalloc_reduction_matches_existing_entry_point(pb):
    import torch
    L = pb.lib()
    L.pb_reduce_noalloc_f64.restype = ctypes.c_int
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(2024)
    n = 150
    data = torch.from_numpy(rng.uniform(-1, 1, n ** 3)).cuda()
    box = _box((0, 0, 0), (n - 1, n - 1, n - 1))
    regions = [_box((0, 0, 0), (-1, -1, -1)), _box((5, 7, 9), (140, 120, 149))]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for region in regions:
        for op in range(6):
            ref = ctypes.c_double()
            assert L.pb_reduce_f64(op, ctypes.c_void_p(data.data_ptr()), box, region, ctypes.byref(ref), stream) == 0
            for _ in range(2):   # two calls in a row share (and must reset) the static scratch
                out.fill_(-12345.0)
                st = L.pb_reduce_noalloc_f64(op, ctypes.c_void_p(data.data_ptr()), box, region,
                                             ctypes.c_void_p(out.data_ptr()), stream)
                assert st == 0
                torch.cuda.synchronize()
                got = float(out.item())
                if op in (0, 1, 2):
                    assert got == ref.value
                else:
                    assert abs(got - ref.value) <= 1e-13 * max(1.0, abs(ref.value))
    # beyond the static scratch: rejected before any device work
    big = _box((0, 0, 0), (255, 255, 255))
    st = L.pb_reduce_noalloc_f64(2, ctypes.c_void_p(data.data_ptr()), big, big, ctypes.c_void_p(out.data_ptr()),
                                 stream)
    assert st == -7
