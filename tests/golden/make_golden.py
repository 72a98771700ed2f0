"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own code (oracle/_ref/libproto_ref.so, built from the reference headers by
oracle/build_oracle.py) on seeded inputs and stores its outputs: small arrays verbatim, large ones
as SHA-256 digests of their little-endian float64 bytes. Inputs are regenerated from the seeds by
the tests, so the fixtures hold outputs only.

    python tests/golden/make_golden.py        (needs the reference tree; run where it exists)
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Ref  # noqa: E402
from proto_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, which, a, b, c) for Ref.stencil_table
STENCILS = [
    ("laplacian", 0, 0, 0, 0),
    ("laplacian19", 1, 0, 0, 0),
    ("laplacian27", 2, 0, 0, 0),
    ("laplacian13", 6, 0, 0, 0),
    ("deriv_2_1_4", 3, 2, 1, 4),
    ("deriv_1_2_6", 3, 1, 2, 6),
    ("diffc2f_0_lo_4", 5, 0, 0, 4),
    ("diffc2f_2_hi_4", 5, 2, 1, 4),
    ("avgdown2", 4, 2, 0, 0),
    ("sum2", 9, 2, 0, 0),
    ("fluxdiv1", 8, 1, 0, 0),
    ("corners2cells4", 13, 4, 0, 0),
    ("identity", 12, 0, 0, 0),
]

# stencil-apply cases: (stencil, src box, dst box, mode, scale, seed)
APPLY_CASES = [
    ("laplacian", ((-1, -1, -1), (8, 9, 7)), ((0, 0, 0), (7, 8, 6)), 0, 1.0, 11),
    ("laplacian", ((-3, -2, -4), (12, 13, 11)), ((-2, -2, -2), (17, 17, 17)), 1, 0.37, 12),
    ("laplacian", ((5, -7, 2), (9, -3, 5)), ((5, -7, 2), (9, -3, 5)), 0, 4096.0, 13),
    ("laplacian13", ((-2, -2, -2), (13, 9, 11)), ((0, 0, 0), (11, 7, 9)), 0, 2.5, 14),
    ("laplacian13", ((-2, -2, -2), (13, 9, 11)), ((0, 0, 0), (11, 7, 9)), 1, 1.0, 15),
    ("laplacian19", ((-1, -1, -1), (10, 10, 10)), ((0, 0, 0), (9, 9, 9)), 0, 1.0, 16),
    ("laplacian27", ((-1, -1, -1), (10, 10, 10)), ((0, 0, 0), (9, 9, 9)), 1, -3.0, 17),
    ("deriv_1_2_6", ((-3, -3, -3), (8, 8, 8)), ((0, 0, 0), (5, 5, 5)), 0, 1.0, 18),
    ("diffc2f_0_lo_4", ((-2, -2, -2), (9, 9, 9)), ((0, 0, 0), (8, 7, 7)), 0, 64.0, 19),
    ("avgdown2", ((-4, -4, -4), (11, 11, 11)), ((-2, -2, -2), (5, 5, 5)), 0, 1.0, 20),
    ("avgdown2", ((0, 0, 0), (15, 15, 15)), ((0, 0, 0), (7, 7, 7)), 1, 0.5, 21),
    ("corners2cells4", ((-2, -2, -2), (9, 9, 9)), ((0, 0, 0), (7, 7, 7)), 0, 1.0, 22),
    ("fluxdiv1", ((0, 0, 0), (9, 9, 9)), ((0, 0, 0), (9, 9, 9)), 0, 1.0, 23),
]

EXCHANGE_CASES = [  # domain, periodic, box size, ghost, seed
    ((16, 16, 16), (1, 1, 1), (8, 8, 8), (1, 1, 1), 31),
    ((24, 16, 8), (1, 0, 1), (8, 8, 8), (2, 2, 2), 32),
    ((8, 8, 8), (1, 1, 1), (8, 8, 8), (2, 1, 3), 33),
    ((32, 16, 16), (1, 1, 1), (16, 8, 4), (2, 2, 2), 34),
]

BOX_CASES = [((-5, -4, -3), (6, 7, 9), (2, 2, 2)), ((-7, 0, 3), (-1, 5, 5), (2, 3, 4)),
             ((1, -9, -8), (15, -2, 8), (4, 4, 2)), ((0, 0, 0), (63, 63, 63), (2, 2, 2))]


PARTITION_CASES = [((2, 2, 2), 2), ((2, 2, 2), 3), ((4, 4, 4), 5), ((3, 5, 2), 4), ((8, 8, 8), 7), ((1, 1, 7), 3),
                   ((6, 3, 4), 8)]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def box_vol(b):
    return int(np.prod([b[1][d] - b[0][d] + 1 for d in range(3)]))


def main():
    R = Ref()
    tables = {}
    arrays = {}
    meta = {"stencils": {}, "apply": [], "exchange": [], "reduce": {}, "mg": {}, "plain": {}, "interp": [],
            "level13": {}, "box": []}
    for name, which, a, b, c in STENCILS:
        co, of, me = R.stencil_table(which, a, b, c)
        tables[name] = (co, of, me)
        arrays["st_%s_coefs" % name] = co
        arrays["st_%s_offs" % name] = of
        arrays["st_%s_meta" % name] = me
        meta["stencils"][name] = len(co)
    for k, (name, sb, db, mode, scale, seed) in enumerate(APPLY_CASES):
        co, of, me = tables[name]
        rng = np.random.default_rng(seed)
        src = rng.uniform(-1, 1, box_vol(sb))
        dst = rng.uniform(-1, 1, box_vol(db))
        R.stencil_apply(co, of, me, src, sb, dst, db, mode, scale)
        arrays["apply_%d" % k] = dst
        meta["apply"].append({"stencil": name, "src": sb, "dst": db, "mode": mode, "scale": scale, "seed": seed})
    for k, (dom, per, bs, g, seed) in enumerate(EXCHANGE_CASES):
        valid = np.random.default_rng(seed).uniform(-1, 1, int(np.prod(dom)))
        out = R.exchange(dom, per, bs, g, valid, -777.0)
        meta["exchange"].append({"domain": dom, "periodic": per, "box": bs, "ghost": g, "seed": seed,
                                 "sha256": digest(out)})
    d = np.random.default_rng(41).uniform(-1, 1, 1001)
    meta["reduce"]["mixed"] = [R.reduce(op, d) for op in range(6)]
    meta["reduce"]["negative"] = [R.reduce(op, -np.abs(d)) for op in range(6)]
    # plain method, small: out = 0.5*L(u, 1/h^2) + 2*u on 64^3, h = 1/64
    u = W.plain_input(64, 0).reshape(-1).copy()
    out = np.zeros(64 ** 3)
    R.plain_apply(64, u, out, 1.0 / 64, 0.5, 2.0)
    meta["plain"] = {"n": 64, "h": 1.0 / 64, "a": 0.5, "b": 2.0, "seed": 0, "sha256": digest(out),
                     "absmax": float(np.abs(out).max())}
    # interpolation
    for k, (kind, r, sb, db, overwrite, scale, seed) in enumerate([
            (0, 2, ((-1, -2, 0), (5, 6, 7)), ((-3, -4, -1), (12, 13, 15)), False, 1.0, 51),
            (0, 2, ((-1, -2, 0), (5, 6, 7)), ((-3, -4, -1), (12, 13, 15)), True, 0.3, 52),
            (0, 4, ((0, 0, 0), (3, 3, 3)), ((0, 0, 0), (15, 15, 15)), False, 1.0, 53),
            (1, 2, ((-1, -2, 0), (5, 6, 7)), ((-3, -4, -1), (12, 13, 15)), False, 1.0, 54),
            (1, 2, ((-1, -2, 0), (5, 6, 7)), ((-3, -4, -1), (12, 13, 15)), True, 0.3, 55),
            (1, 4, ((0, 0, 0), (3, 3, 3)), ((0, 0, 0), (15, 15, 15)), False, 1.0, 56),
            (2, 2, ((-1, -2, 0), (5, 6, 7)), ((-3, -4, -1), (12, 13, 15)), False, 1.0, 57),
            (2, 3, ((0, 0, 0), (4, 4, 4)), ((0, 0, 0), (14, 14, 14)), True, 2.0, 58)]):
        rng = np.random.default_rng(seed)
        src = rng.uniform(-1, 1, box_vol(sb))
        dst = rng.uniform(-1, 1, box_vol(db))
        R.interp_apply(kind, r, src, sb, dst, db, overwrite, scale)
        arrays["interp_%d" % k] = dst
        meta["interp"].append({"kind": kind, "ratio": r, "src": sb, "dst": db, "overwrite": overwrite,
                               "scale": scale, "seed": seed})
    # multigrid residual histories (inputs: the sine-mode right-hand side, seed 1)
    cases = {
        "archived_32": dict(kind="archived", N=32, box=16, numLevels=5, maxIter=20, tol=1e-10),
        "cs_v22_32": dict(kind="cs", N=32, box=16, levels=3, nu1=2, nu2=2, nub=10, omega=2.0 / 3.0, maxIter=60,
                          tol=1e-10),
        "cs_v22_64": dict(kind="cs", N=64, box=32, levels=4, nu1=2, nu2=2, nub=10, omega=2.0 / 3.0, maxIter=60,
                          tol=1e-10),
        "helm_v22_32": dict(kind="helm", N=32, box=16, levels=3, nu1=2, nu2=2, nub=10, omega=2.0 / 3.0,
                            maxIter=60, tol=1e-10),
        "fas_32": dict(kind="fas", N=32, box=16, numLevels=4, maxIter=20, tol=1e-10),
    }
    for name, cfg in cases.items():
        N = cfg["N"]
        rho = W.poisson_rho(N, seed=1).reshape(-1).copy()
        phi = np.zeros(N ** 3)
        if cfg["kind"] == "archived":
            n, h = R.mg_archived(N, cfg["box"], cfg["numLevels"], cfg["maxIter"], cfg["tol"], rho, phi)
        elif cfg["kind"] == "fas":
            n, h = R.mg_fas(N, cfg["box"], cfg["numLevels"], cfg["maxIter"], cfg["tol"], -rho, phi)
        elif cfg["kind"] == "cs":
            n, h = R.mg_cs(N, cfg["box"], cfg["levels"], cfg["nu1"], cfg["nu2"], cfg["nub"], cfg["omega"], 1.0,
                           None, cfg["maxIter"], cfg["tol"], rho, phi)
        else:
            alpha = W.helmholtz_alpha(N, seed=3).reshape(-1).copy()
            n, h = R.mg_cs(N, cfg["box"], cfg["levels"], cfg["nu1"], cfg["nu2"], cfg["nub"], cfg["omega"], 1.0,
                           alpha, cfg["maxIter"], cfg["tol"], -rho, phi)
        cfg = dict(cfg)
        cfg["iters"] = int(n)
        cfg["hist"] = [float(v) for v in h]
        cfg["phi_sha256"] = digest(phi)
        meta["mg"][name] = cfg
    # AMR-level stepping (small uneven tiling), 13-point, 5 steps
    widths = [[16, 24, 16], [24, 16], [16, 32]]
    boxes, L = W.amr_patches(widths)
    g = 2
    u = W.uniform_box((L[2], L[1], L[0]), 61)
    data = []
    for lo, hi in boxes:
        a = np.zeros((hi[2] - lo[2] + 1 + 2 * g, hi[1] - lo[1] + 1 + 2 * g, hi[0] - lo[0] + 1 + 2 * g))
        a[g:-g, g:-g, g:-g] = u[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        data.append(a.reshape(-1))
    data = np.concatenate(data)
    h = 1.0 / L[0]
    R.level13_steps(widths, g, h, 0.1 * h * h, 5, data)
    valid = []
    off = 0
    for lo, hi in boxes:
        shp = (hi[2] - lo[2] + 1 + 2 * g, hi[1] - lo[1] + 1 + 2 * g, hi[0] - lo[0] + 1 + 2 * g)
        n = int(np.prod(shp))
        valid.append(data[off:off + n].reshape(shp)[g:-g, g:-g, g:-g].reshape(-1))
        off += n
    meta["level13"] = {"widths": widths, "ghost": g, "seed": 61, "steps": 5, "h": h, "dt": 0.1 * h * h,
                       "sha256": digest(np.concatenate(valid))}
    for lo, hi, r in BOX_CASES:
        meta["box"].append({"lo": lo, "hi": hi, "ratio": r, "coarsen": R.box_op(0, lo, hi, r),
                            "taper": R.box_op(1, lo, hi, r), "refine": R.box_op(2, lo, hi, r)})
    # BoxPartition: process of each patch index point (points listed in a seeded shuffled order)
    meta["partition"] = []
    prng = np.random.default_rng(12)
    for shape, nranks in PARTITION_CASES:
        pts = [(x, y, z) for z in range(shape[2]) for y in range(shape[1]) for x in range(shape[0])]
        pts = [pts[k] for k in prng.permutation(len(pts))]
        meta["partition"].append({"points": pts, "nranks": nranks, "owner": R.load_balance(pts, nranks)})
    np.savez_compressed(os.path.join(OUT, "golden_arrays.npz"), **arrays)

    def conv(o):
        if isinstance(o, (np.integer,)):
            return int(o)
        if isinstance(o, (np.floating,)):
            return float(o)
        if isinstance(o, tuple):
            return [conv(v) for v in o]
        if isinstance(o, list):
            return [conv(v) for v in o]
        if isinstance(o, dict):
            return {k: conv(v) for k, v in o.items()}
        return o

    with open(os.path.join(OUT, "golden.json"), "w") as f:
        json.dump(conv(meta), f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
