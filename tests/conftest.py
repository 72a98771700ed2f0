"""Shared fixtures. GPU tests are marked 'gpu' and run only where a CUDA device exists."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        meta = json.load(f)
    arrays = dict(np.load(os.path.join(GOLDEN_DIR, "golden_arrays.npz")))
    return meta, arrays


@pytest.fixture(scope="session")
def port():
    from oracle.build_oracle import build_port
    build_port()
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference-built oracle not present")
    return Ref()


@pytest.fixture(scope="session")
def pb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import proto_b200
    proto_b200.lib()
    return proto_b200
