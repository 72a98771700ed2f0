"""Test helpers: golden stencil tables, box volumes and digests."""
import hashlib

import numpy as np


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def box_vol(b):
    return int(np.prod([b[1][d] - b[0][d] + 1 for d in range(3)]))


def box_shape(b):
    return tuple(b[1][d] - b[0][d] + 1 for d in (2, 1, 0))


def table(arrays, name):
    return (arrays["st_%s_coefs" % name], arrays["st_%s_offs" % name].reshape(-1, 3),
            arrays["st_%s_meta" % name])


def apply_inputs(case):
    rng = np.random.default_rng(case["seed"])
    src = rng.uniform(-1, 1, box_vol(case["src"]))
    dst = rng.uniform(-1, 1, box_vol(case["dst"]))
    return src, dst


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
