"""ctypes bindings for the CPU oracle (test infrastructure only).

`Port` wraps oracle/liboracle.so (the plain-C restatement, pb_oracle.c); `Ref` wraps
oracle/_ref/libproto_ref.so (the reference's own code compiled from its headers), which exists
only where the reference tree was available at build time. Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference arm import this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_c_int, _c_dbl, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _i3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32).reshape(-1))


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


class Port:
    """The C restatement."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        self.lib = L = ctypes.CDLL(path)
        L.or_reduce.restype = _c_dbl
        L.or_reduce.argtypes = [_c_int, _vp, ctypes.c_long]
        for name in ("or_stencil_apply", "or_interp_constant", "or_exchange", "or_mg_cs", "or_mg_fas",
                     "or_plain_apply", "or_periodic_steps", "or_num_threads"):
            getattr(L, name).restype = _c_int

    def set_threads(self, n):
        self.lib.or_set_threads(_c_int(n))

    def num_threads(self):
        return self.lib.or_num_threads()

    def stencil_apply(self, coefs, offs, meta, src, src_box, dst, dst_box, box, init_to_zero,
                      scale, ncomp=1):
        coefs = _f64(coefs)
        offs, meta = _i3(offs), _i3(meta)
        return self.lib.or_stencil_apply(_p(coefs), _p(offs), _c_int(len(coefs)), _p(meta),
                                         _p(src), _p(_i3(src_box[0])), _p(_i3(src_box[1])),
                                         _p(dst), _p(_i3(dst_box[0])), _p(_i3(dst_box[1])),
                                         _p(_i3(box[0])), _p(_i3(box[1])), _c_int(int(init_to_zero)),
                                         _c_dbl(scale), _c_int(ncomp))

    def infer_box(self, offs, meta, src_box, dst_box):
        lo, hi = np.zeros(3, np.int32), np.zeros(3, np.int32)
        offs, meta = _i3(offs), _i3(meta)
        self.lib.or_stencil_infer_box(_p(offs), _c_int(len(offs) // 3), _p(meta),
                                      _p(_i3(src_box[0])), _p(_i3(src_box[1])),
                                      _p(_i3(dst_box[0])), _p(_i3(dst_box[1])), _p(lo), _p(hi))
        return tuple(lo), tuple(hi)

    def interp_constant(self, r, src, src_box, dst, dst_box, overwrite, scale=1.0):
        return self.lib.or_interp_constant(_c_int(r), _p(src), _p(_i3(src_box[0])), _p(_i3(src_box[1])),
                                           _p(dst), _p(_i3(dst_box[0])), _p(_i3(dst_box[1])),
                                           _c_int(int(overwrite)), _c_dbl(scale))

    def exchange(self, boxes, ghost, domain, periodic, datas, ncomp=1):
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int32).reshape(-1))
        ptrs = (_vp * len(datas))(*[d.ctypes.data for d in datas])
        return self.lib.or_exchange(_c_int(len(datas)), _p(b), _p(_i3(ghost)), _p(_i3(domain[0])),
                                    _p(_i3(domain[1])), _p(_i3(periodic)), ptrs, _c_int(ncomp))

    def reduce(self, op, data):
        data = _f64(data)
        return self.lib.or_reduce(_c_int(op), _p(data), ctypes.c_long(data.size))

    def mg_cs(self, N, levels, nu1, nu2, nu_bottom, omega, beta, alpha, max_iter, tol, rhs, phi, bottom=0):
        """bottom 0: nu_bottom coarsest sweeps (the reference's); 1: exact coarsest solve."""
        hist = np.zeros(max_iter + 1)
        rhs = _f64(rhs)
        alpha = None if alpha is None else _f64(alpha)
        n = self.lib.or_mg_cs(_c_int(N), _c_int(levels), _c_int(nu1), _c_int(nu2), _c_int(nu_bottom),
                              _c_dbl(omega), _c_dbl(beta), _p(alpha), _c_int(max_iter), _c_dbl(tol),
                              _p(rhs), _p(phi), _p(hist), _c_int(bottom))
        if n < 0:
            raise RuntimeError("or_mg_cs: singular coarsest operator")
        return n, hist[: n + 1]

    def mg_fas(self, N, num_levels, max_iter, tol, force, phi):
        """FAS V(6,6) with the 4th-order flux-form Laplacian (LevelMultigridSolver<BoxOp_Laplace>)."""
        hist = np.zeros(max_iter + 1)
        force = _f64(force)
        n = self.lib.or_mg_fas(_c_int(N), _c_int(num_levels), _c_int(max_iter), _c_dbl(tol), _p(force), _p(phi),
                               _p(hist))
        return n, hist[: n + 1]

    def plain_apply(self, n, u, out, h, a, b):
        return self.lib.or_plain_apply(_c_int(n), _p(u), _p(out), _c_dbl(h), _c_dbl(a), _c_dbl(b))

    def boxop_laplace(self, u, s_box, out, o_box, r_box, dx, flux_scale=1.0, scale=1.0):
        return self.lib.or_boxop_laplace(_p(u), _p(_i3(s_box[0])), _p(_i3(s_box[1])), _p(out), _p(_i3(o_box[0])),
                                         _p(_i3(o_box[1])), _p(_i3(r_box[0])), _p(_i3(r_box[1])), _c_dbl(dx),
                                         _c_dbl(flux_scale), _c_dbl(scale))

    def periodic_steps(self, L, g, coefs, offs, h, dt, steps, u):
        coefs = _f64(coefs)
        offs = _i3(offs)
        return self.lib.or_periodic_steps(_c_int(L[0]), _c_int(L[1]), _c_int(L[2]), _c_int(g), _p(coefs),
                                          _p(offs), _c_int(len(coefs)), _c_dbl(h), _c_dbl(dt),
                                          _c_int(steps), _p(u))


class Ref:
    """The reference compiled from its own sources (present only where it was built)."""

    PATH = os.path.join(HERE, "_ref", "libproto_ref.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self):
        self.lib = L = ctypes.CDLL(self.PATH)
        L.ref_reduce.restype = _c_dbl
        L.ref_mg_cs_time_cycles.restype = _c_dbl

    def stencil_table(self, which, a=0, b=0, c=0, cap=512):
        coefs = np.zeros(cap)
        offs = np.zeros(3 * cap, np.int32)
        meta = np.zeros(9, np.int32)
        n = self.lib.ref_stencil_table(_c_int(which), _c_int(a), _c_int(b), _c_int(c), _p(coefs), _p(offs),
                                       _p(meta), _c_int(cap))
        assert n >= 0
        return coefs[:n].copy(), offs[: 3 * n].reshape(n, 3).copy(), meta.copy()

    def stencil_apply(self, coefs, offs, meta, src, src_box, dst, dst_box, mode, scale, rng=None, ncomp=1):
        coefs = _f64(coefs)
        offs, meta = _i3(offs), _i3(meta)
        rlo, rhi = (rng if rng is not None else ((0, 0, 0), (-1, -1, -1)))
        return self.lib.ref_stencil_apply(_p(coefs), _p(offs), _c_int(len(coefs)), _p(meta), _p(src),
                                          _p(_i3(src_box[0])), _p(_i3(src_box[1])), _p(dst),
                                          _p(_i3(dst_box[0])), _p(_i3(dst_box[1])), _p(_i3(rlo)), _p(_i3(rhi)),
                                          _c_int(mode), _c_dbl(scale), _c_int(ncomp))

    def stencil_range(self, coefs, offs, meta, src_box):
        lo, hi = np.zeros(3, np.int32), np.zeros(3, np.int32)
        coefs = _f64(coefs)
        offs, meta = _i3(offs), _i3(meta)
        e = self.lib.ref_stencil_range(_p(coefs), _p(offs), _c_int(len(coefs)), _p(meta),
                                       _p(_i3(src_box[0])), _p(_i3(src_box[1])), _p(lo), _p(hi))
        return tuple(lo), tuple(hi), bool(e)

    def box_op(self, op, lo, hi, ratio):
        olo, ohi = np.zeros(3, np.int32), np.zeros(3, np.int32)
        self.lib.ref_box_op(_c_int(op), _p(_i3(lo)), _p(_i3(hi)), _p(_i3(ratio)), _p(olo), _p(ohi))
        return tuple(olo), tuple(ohi)

    def interp_apply(self, kind, r, src, src_box, dst, dst_box, overwrite, scale=1.0):
        return self.lib.ref_interp_apply(_c_int(kind), _c_int(r), _p(src), _p(_i3(src_box[0])),
                                         _p(_i3(src_box[1])), _p(dst), _p(_i3(dst_box[0])),
                                         _p(_i3(dst_box[1])), _c_int(int(overwrite)), _c_dbl(scale))

    def exchange(self, domain_size, periodic, box_size, ghost, valid, fill):
        np_ = [domain_size[d] // box_size[d] for d in range(3)]
        pv = int(np.prod([box_size[d] + 2 * ghost[d] for d in range(3)]))
        out = np.zeros(int(np.prod(np_)) * pv)
        valid = _f64(valid)
        self.lib.ref_exchange(_p(_i3(domain_size)), _p(_i3(periodic)), _p(_i3(box_size)), _p(_i3(ghost)),
                              _p(valid), _p(out), _c_dbl(fill))
        return out

    def reduce(self, op, data):
        data = _f64(data)
        return self.lib.ref_reduce(_c_int(op), _p(data), _c_int(data.size))

    def plain_apply(self, n, u, out, h, a, b):
        return self.lib.ref_plain_apply(_c_int(n), _p(u), _p(out), _c_dbl(h), _c_dbl(a), _c_dbl(b))

    def mg_archived(self, N, box_size, num_levels, max_iter, tol, rho, phi):
        hist = np.zeros(max_iter + 1)
        rho = _f64(rho)
        n = self.lib.ref_mg_archived(_c_int(N), _c_int(box_size), _c_int(num_levels), _c_int(max_iter),
                                     _c_dbl(tol), _p(rho), _p(phi), _p(hist))
        return n, hist[: n + 1]

    def mg_fas(self, N, box_size, num_levels, max_iter, tol, force, phi):
        hist = np.zeros(max_iter + 1)
        force = _f64(force)
        n = self.lib.ref_mg_fas(_c_int(N), _c_int(box_size), _c_int(num_levels), _c_int(max_iter),
                                _c_dbl(tol), _p(force), _p(phi), _p(hist))
        return n, hist[: n + 1]

    def mg_cs(self, N, box_size, levels, nu1, nu2, nu_bottom, omega, beta, alpha, max_iter, tol, rhs, phi):
        hist = np.zeros(max_iter + 1)
        rhs = _f64(rhs)
        alpha = None if alpha is None else _f64(alpha)
        n = self.lib.ref_mg_cs(_c_int(N), _c_int(box_size), _c_int(levels), _c_int(nu1), _c_int(nu2),
                               _c_int(nu_bottom), _c_dbl(omega), _c_dbl(beta), _p(alpha), _c_int(max_iter),
                               _c_dbl(tol), _p(rhs), _p(phi), _p(hist))
        return n, hist[: n + 1]

    def mg_cs_time_cycles(self, N, box_size, levels, nu1, nu2, nu_bottom, omega, rhs, reps):
        rhs = _f64(rhs)
        return self.lib.ref_mg_cs_time_cycles(_c_int(N), _c_int(box_size), _c_int(levels), _c_int(nu1),
                                              _c_int(nu2), _c_int(nu_bottom), _c_dbl(omega), _p(rhs),
                                              _c_int(reps))

    def mg_cs_cycles(self, N, box_size, levels, nu1, nu2, nu_bottom, omega, tol, rhs, ncycles):
        """Runs ncycles real V-cycles (+ norms) of the Poisson solve, restarting from zero after each
        converged solve. Returns (cycles of the first solve, solves completed, start time, end time of
        every cycle); times are steady-clock seconds."""
        rhs = _f64(rhs)
        t_end = np.zeros(ncycles)
        t0 = _c_dbl(0.0)
        done = _c_int(0)
        first = self.lib.ref_mg_cs_cycles(_c_int(N), _c_int(box_size), _c_int(levels), _c_int(nu1), _c_int(nu2),
                                          _c_int(nu_bottom), _c_dbl(omega), _c_dbl(tol), _p(rhs), _c_int(ncycles),
                                          ctypes.byref(t0), _p(t_end), ctypes.byref(done))
        return first, done.value, t0.value, t_end

    def boxop_laplace(self, u, s_box, out, o_box, dx, flux_scale=1.0, scale=1.0):
        """The reference's BoxOp_Laplace::operator()(out, state, scale) on out's box."""
        return self.lib.ref_boxop_laplace(_p(u), _p(_i3(s_box[0])), _p(_i3(s_box[1])), _p(out), _p(_i3(o_box[0])),
                                          _p(_i3(o_box[1])), _c_dbl(dx), _c_dbl(flux_scale), _c_dbl(scale))

    def load_balance(self, points, nranks):
        """The reference's BoxPartition assignment of patch index points to nranks processes."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.int32).reshape(-1))
        owner = np.zeros(len(points), dtype=np.int32)
        rc = self.lib.ref_load_balance(_p(pts), _c_int(len(points)), _c_int(nranks), _p(owner))
        if rc != 0:
            raise RuntimeError("ref_load_balance: %d" % rc)
        return owner.tolist()

    def level13_steps(self, widths, ghost, h, dt, steps, data):
        arrs = [_i3(w) for w in widths]
        counts = _i3([len(w) for w in widths])
        return self.lib.ref_level13_steps(_p(arrs[0]), _p(arrs[1]), _p(arrs[2]), _p(counts), _c_int(ghost),
                                          _c_dbl(h), _c_dbl(dt), _c_int(steps), _p(data))
