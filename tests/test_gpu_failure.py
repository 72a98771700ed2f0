"""Failure detection on the GPU without a fault: the bounded mbarrier wait that every pipelined
kernel uses is made to expire (a barrier nothing arrives on), the kernel returns, the device error
flag reports it through pb_device_check, and the context stays usable afterwards."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_and_is_reported(pb):
    import torch
    L = pb.lib()
    pb.device_check()                       # start from a clear flag
    expired = ctypes.c_int(-1)
    st = torch.cuda.current_stream().cuda_stream
    assert L.pb_debug_wait_expiry(ctypes.c_uint(1000), ctypes.byref(expired), ctypes.c_void_p(st)) == 0
    assert expired.value == 1
    assert L.pb_device_check(ctypes.c_void_p(st)) == -8          # PB_ERR_DEVICE: the flag was set
    # the flag was read and cleared: the next check is clean, and kernels still run
    assert L.pb_device_check(ctypes.c_void_p(st)) == 0
    x = torch.arange(1000, dtype=torch.float64, device="cuda")
    assert pb.reduce(pb.RED_SUM, x, pb.Box((0, 0, 0), (999, 0, 0))) == float(np.arange(1000).sum())
