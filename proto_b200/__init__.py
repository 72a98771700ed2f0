"""Python binding of the proto_b200 C ABI (include/proto_b200.h).

Thin ctypes layer over proto_b200/lib/libproto_b200.so. Device memory is passed as torch CUDA
tensors (data_ptr) and work is enqueued on torch's current CUDA stream. There is no CPU fallback:
if the shared library is missing or was built without the sm_100a kernels, loading raises.

Names follow the reference's API (Proto's Box, Stencil, BoxData, LevelBoxData, Reduction,
LevelMultigridSolver); every call maps onto one C entry point.
"""
import ctypes
import os
import re

__all__ = ["ProtoError", "lib", "Box", "Stencil", "Level", "Multigrid", "MGParams", "status_string",
           "boxdata_op", "boxdata_scalar", "boxdata_copy", "forall_axpby", "reduce", "reduce_async",
           "interp_constant", "device_check", "OP_ADD", "OP_SUB", "OP_MUL", "OP_DIV", "OP_ASSIGN",
           "RED_MAX", "RED_MIN", "RED_ABS", "RED_SUM", "RED_SUMABS", "RED_SUMSQ", "EPI_AXPBY", "EPI_EULER",
           "MG_POISSON", "MG_HELMHOLTZ", "MG_FP64", "MG_MIXED", "MG_BOTTOM_RELAX", "MG_BOTTOM_DIRECT",
           "FAS", "Serve", "SERVE_WAITING", "SERVE_ACTIVE", "SERVE_DONE", "SERVE_FAILED",
           "header_functions"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libproto_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "proto_b200.h")

OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_ASSIGN = 0, 1, 2, 3, 4
RED_MAX, RED_MIN, RED_ABS, RED_SUM, RED_SUMABS, RED_SUMSQ = 0, 1, 2, 3, 4, 5
EPI_AXPBY, EPI_EULER = 1, 2
MG_POISSON, MG_HELMHOLTZ = 0, 1
MG_FP64, MG_MIXED = 0, 1
MG_BOTTOM_RELAX, MG_BOTTOM_DIRECT = 0, 1
SERVE_WAITING, SERVE_ACTIVE, SERVE_DONE, SERVE_FAILED = 0, 1, 2, 3

_c_int, _c_dbl, _c_flt, _vp, _c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_longlong


class pb_box(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3)]


class pb_mg_params(ctypes.Structure):
    _fields_ = [("n", _c_int), ("levels", _c_int), ("nu1", _c_int), ("nu2", _c_int), ("nu_bottom", _c_int),
                ("omega", _c_dbl), ("beta", _c_dbl), ("form", _c_int), ("precision", _c_int),
                ("max_iter", _c_int), ("tol", _c_dbl), ("bottom", _c_int)]


class pb_serve_params(ctypes.Structure):
    _fields_ = [("hbm_budget", _c_ll), ("max_active", _c_int), ("nu1", _c_int), ("nu2", _c_int),
                ("nu_bottom", _c_int), ("omega", _c_dbl), ("tol", _c_dbl), ("max_cycles", _c_int),
                ("precision", _c_int)]


class pb_serve_request(ctypes.Structure):
    _fields_ = [("n", _c_int), ("form", _c_int), ("alpha", _c_dbl), ("beta", _c_dbl), ("rhs", _vp), ("out", _vp)]


class ProtoError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = status_string(status) if _LIB is not None else str(status)
        if status == -3 and _LIB is not None:
            msg += " (cudaError %d)" % _LIB.pb_last_cuda_error()
        super().__init__("%s: %s [%d]" % (where, msg, status))


_LIB = None


def lib():
    """Load the shared library (once). Raises if it is absent: there is no fallback path."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("proto_b200: %s is missing; build it with proto_b200/build.py" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        L.pb_status_string.restype = ctypes.c_char_p
        L.pb_version.restype = ctypes.c_char_p
        L.pb_mg_device_bytes.restype = _c_ll
        L.pb_mg_device_bytes.argtypes = [ctypes.POINTER(pb_mg_params)]
        L.pb_mg_launches_per_cycle.argtypes = [ctypes.POINTER(pb_mg_params)]
        L.pb_serve_device_bytes.restype = _c_ll
        L.pb_serve_request_bytes.restype = _c_ll
        L.pb_serve_hierarchy_bytes.restype = _c_ll
        L.pb_halo_plan_elems.restype = _c_ll
        L.pb_halo_plan_elems.argtypes = [_vp]
        L.pb_serve_status.argtypes = [_vp, _c_ll, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int),
                                      ctypes.POINTER(_c_dbl)]
        for name in ("pb_stencil_apply_f64", "pb_stencil_apply_f32", "pb_stencil_apply_fused_f64",
                     "pb_boxdata_op_f64", "pb_boxdata_scalar_f64", "pb_boxdata_copy_f64", "pb_forall_axpby_f64",
                     "pb_reduce_f64", "pb_reduce_async_f64", "pb_interp_constant_f64"):
            getattr(L, name).restype = _c_int
        _LIB = L
    return _LIB


def status_string(s):
    return lib().pb_status_string(int(s)).decode()


def header_functions():
    """Names of every function include/proto_b200.h declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pb_[a-z0-9_]+)\s*\(", txt)))


def _check(status, where):
    if status != 0:
        raise ProtoError(status, where)


def _stream(stream=None):
    if stream is not None:
        return _vp(stream)
    import torch
    return _vp(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return _vp(t.data_ptr())


class Box:
    """Proto::Box: inclusive corners lo, hi (3-D)."""

    def __init__(self, lo, hi):
        self.lo = tuple(int(v) for v in lo)
        self.hi = tuple(int(v) for v in hi)

    @staticmethod
    def cube(n, lo=0):
        return Box((lo,) * 3, (lo + n - 1,) * 3)

    @staticmethod
    def empty():
        return Box((0, 0, 0), (-1, -1, -1))

    def grow(self, g):
        g = (g,) * 3 if isinstance(g, int) else tuple(g)
        return Box([self.lo[d] - g[d] for d in range(3)], [self.hi[d] + g[d] for d in range(3)])

    def shift(self, s):
        return Box([self.lo[d] + s[d] for d in range(3)], [self.hi[d] + s[d] for d in range(3)])

    def size(self, d=None):
        if d is not None:
            return max(0, self.hi[d] - self.lo[d] + 1)
        return self.size(0) * self.size(1) * self.size(2)

    def shape(self):
        """numpy/torch shape of a field on this box (z, y, x)."""
        return (self.size(2), self.size(1), self.size(0))

    def c(self):
        b = pb_box()
        for d in range(3):
            b.lo[d] = self.lo[d]
            b.hi[d] = self.hi[d]
        return b

    def __repr__(self):
        return "Box(%s, %s)" % (self.lo, self.hi)


def _c(box):
    return (box if isinstance(box, Box) else Box(*box)).c()


class Stencil:
    """A closed Stencil<T> (coefficients and offsets in insertion order, ratios, shift)."""

    def __init__(self, coefs, offsets, src_ratio=(1, 1, 1), dst_ratio=(1, 1, 1), dst_shift=(0, 0, 0)):
        L = lib()
        n = len(coefs)
        c = (ctypes.c_double * max(n, 1))(*[float(v) for v in coefs])
        flat = [int(v) for o in offsets for v in o]
        o = (ctypes.c_int * max(3 * n, 1))(*flat)
        sr = (ctypes.c_int * 3)(*src_ratio)
        dr = (ctypes.c_int * 3)(*dst_ratio)
        ds = (ctypes.c_int * 3)(*dst_shift)
        h = _vp()
        _check(L.pb_stencil_create(c, o, _c_int(n), sr, dr, ds, ctypes.byref(h)), "pb_stencil_create")
        self._h = h
        self.n = n

    def info(self):
        n, shape = _c_int(), _c_int()
        span = pb_box()
        _check(lib().pb_stencil_info(self._h, ctypes.byref(n), ctypes.byref(span), ctypes.byref(shape)),
               "pb_stencil_info")
        return n.value, Box(tuple(span.lo), tuple(span.hi)), shape.value

    def apply(self, src, src_box, dst, dst_box, box=None, init_to_zero=True, scale=1.0, ncomp=1, stream=None):
        """Stencil::apply: dst |= S(src, scale) (init_to_zero) or dst += S(src, scale)."""
        box = box if box is not None else Box.empty()
        if src.dtype.itemsize == 8:
            st = lib().pb_stencil_apply_f64(self._h, _ptr(src), _c(src_box), _ptr(dst), _c(dst_box), _c(box),
                                            _c_int(ncomp), _c_int(int(init_to_zero)), _c_dbl(scale), _stream(stream))
        else:
            st = lib().pb_stencil_apply_f32(self._h, _ptr(src), _c(src_box), _ptr(dst), _c(dst_box), _c(box),
                                            _c_int(ncomp), _c_int(int(init_to_zero)), _c_flt(scale), _stream(stream))
        _check(st, "pb_stencil_apply")

    def apply_fused(self, epilogue, u, u_box, out, out_box, box=None, scale=1.0, a=1.0, b=0.0, stream=None):
        box = box if box is not None else Box.empty()
        _check(lib().pb_stencil_apply_fused_f64(self._h, _c_int(epilogue), _ptr(u), _c(u_box), _ptr(out),
                                                _c(out_box), _c(box), _c_dbl(scale), _c_dbl(a), _c_dbl(b),
                                                _stream(stream)), "pb_stencil_apply_fused_f64")

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.pb_stencil_destroy(self._h)
            self._h = None


def boxdata_op(op, dst, dst_box, src, src_box, ncomp=1, stream=None):
    _check(lib().pb_boxdata_op_f64(_c_int(op), _ptr(dst), _c(dst_box), _ptr(src), _c(src_box), _c_int(ncomp),
                                   _stream(stream)), "pb_boxdata_op_f64")


def boxdata_scalar(op, dst, dst_box, scalar, region=None, ncomp=1, stream=None):
    region = region if region is not None else Box.empty()
    _check(lib().pb_boxdata_scalar_f64(_c_int(op), _ptr(dst), _c(dst_box), _c(region), _c_dbl(scalar),
                                       _c_int(ncomp), _stream(stream)), "pb_boxdata_scalar_f64")


def boxdata_copy(src, src_box, dst, dst_box, src_region=None, shift=(0, 0, 0), ncomp=1, stream=None):
    src_region = src_region if src_region is not None else Box.empty()
    sh = (ctypes.c_int * 3)(*shift)
    _check(lib().pb_boxdata_copy_f64(_ptr(src), _c(src_box), _ptr(dst), _c(dst_box), _c(src_region), sh,
                                     _c_int(ncomp), _stream(stream)), "pb_boxdata_copy_f64")


def forall_axpby(out, out_box, x, x_box, y, y_box, a, b, stream=None):
    _check(lib().pb_forall_axpby_f64(_ptr(out), _c(out_box), _ptr(x), _c(x_box), _ptr(y), _c(y_box), _c_dbl(a),
                                     _c_dbl(b), _stream(stream)), "pb_forall_axpby_f64")


def reduce(op, data, box, region=None, stream=None):
    region = region if region is not None else Box.empty()
    r = ctypes.c_double()
    _check(lib().pb_reduce_f64(_c_int(op), _ptr(data), _c(box), _c(region), ctypes.byref(r), _stream(stream)),
           "pb_reduce_f64")
    return r.value


def reduce_async(op, data, box, result_dev, region=None, stream=None):
    region = region if region is not None else Box.empty()
    _check(lib().pb_reduce_async_f64(_c_int(op), _ptr(data), _c(box), _c(region), _ptr(result_dev),
                                     _stream(stream)), "pb_reduce_async_f64")


def interp_constant(ratio, src, src_box, dst, dst_box, overwrite=False, scale=1.0, stream=None):
    _check(lib().pb_interp_constant_f64(_c_int(ratio), _ptr(src), _c(src_box), _ptr(dst), _c(dst_box),
                                        _c_int(int(overwrite)), _c_dbl(scale), _stream(stream)),
           "pb_interp_constant_f64")


def device_check(stream=None):
    _check(lib().pb_device_check(_stream(stream)), "pb_device_check")


class Level:
    """LevelBoxData layout: disjoint patches in one device slab, with ghost exchange."""

    def __init__(self, patches, ghost, domain, periodic=(1, 1, 1), ncomp=1):
        L = lib()
        n = len(patches)
        arr = (pb_box * n)(*[_c(p) for p in patches])
        g = (ctypes.c_int * 3)(*((ghost,) * 3 if isinstance(ghost, int) else ghost))
        per = (ctypes.c_int * 3)(*periodic)
        h = _vp()
        _check(L.pb_level_create(arr, _c_int(n), g, _c(domain), per, _c_int(ncomp), ctypes.byref(h)),
               "pb_level_create")
        self._h = h
        self.patches = [p if isinstance(p, Box) else Box(*p) for p in patches]
        self.ghost = tuple(g)
        offs = (ctypes.c_longlong * n)()
        slab = ctypes.c_longlong()
        nitems = _c_int()
        _check(L.pb_level_layout(h, offs, ctypes.byref(slab), ctypes.byref(nitems)), "pb_level_layout")
        self.offsets = list(offs)
        self.slab_elems = slab.value
        self.nitems = nitems.value

    def exchange(self, slab, stream=None):
        _check(lib().pb_level_exchange_f64(self._h, _ptr(slab), _stream(stream)), "pb_level_exchange_f64")

    def stencil(self, stencil, epilogue, u_slab, out_slab, scale=1.0, a=0.0, stream=None):
        _check(lib().pb_level_stencil_f64(self._h, stencil._h, _c_int(epilogue), _ptr(u_slab), _ptr(out_slab),
                                          _c_dbl(scale), _c_dbl(a), _stream(stream)), "pb_level_stencil_f64")

    def steps(self, stencil, epilogue, u_slab, tmp_slab, nsteps, scale=1.0, a=0.0, stream=None):
        """nsteps of exchange + stencil step as one captured graph; the result ends in u_slab."""
        _check(lib().pb_level_steps_f64(self._h, stencil._h, _c_int(epilogue), _ptr(u_slab), _ptr(tmp_slab),
                                        _c_dbl(scale), _c_dbl(a), _c_int(nsteps), _stream(stream)),
               "pb_level_steps_f64")

    def autotune(self, stencil, u_slab, out_slab, scale=1.0, stream=None):
        _check(lib().pb_level_autotune_f64(self._h, stencil._h, _ptr(u_slab), _ptr(out_slab), _c_dbl(scale),
                                           _stream(stream)), "pb_level_autotune_f64")

    def tiles(self):
        buf = (_c_int * 96)()
        n = _c_int()
        _check(lib().pb_level_tiles(self._h, buf, _c_int(32), ctypes.byref(n)), "pb_level_tiles")
        return [(buf[3 * k], buf[3 * k + 1], buf[3 * k + 2]) for k in range(n.value)]

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.pb_level_destroy(self._h)
            self._h = None


class MGParams:
    def __init__(self, n, levels, nu1=2, nu2=2, nu_bottom=10, omega=2.0 / 3.0, beta=1.0, form=MG_POISSON,
                 precision=MG_FP64, max_iter=100, tol=1e-10, bottom=0):
        self.c = pb_mg_params(n, levels, nu1, nu2, nu_bottom, omega, beta, form, precision, max_iter, tol, bottom)

    def device_bytes(self):
        return lib().pb_mg_device_bytes(ctypes.byref(self.c))


class Multigrid:
    """Periodic point-Jacobi multigrid solver (pb_mg_*)."""

    def __init__(self, params):
        self.params = params
        h = _vp()
        _check(lib().pb_mg_create(ctypes.byref(params.c), ctypes.byref(h)), "pb_mg_create")
        self._h = h

    def set_alpha(self, alpha, stream=None):
        _check(lib().pb_mg_set_alpha(self._h, _ptr(alpha), _stream(stream)), "pb_mg_set_alpha")

    def solve(self, rhs, phi, stream=None):
        it = _c_int()
        hist = (ctypes.c_double * (self.params.c.max_iter + 1))()
        _check(lib().pb_mg_solve(self._h, _ptr(rhs), _ptr(phi), ctypes.byref(it), hist, _stream(stream)),
               "pb_mg_solve")
        return it.value, [hist[k] for k in range(it.value + 1)]

    def relax(self, sweeps, stream=None):
        _check(lib().pb_mg_relax(self._h, _c_int(sweeps), _stream(stream)), "pb_mg_relax")

    def launches_per_cycle(self):
        return lib().pb_mg_launches_per_cycle(ctypes.byref(self.params.c))

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.pb_mg_destroy(self._h)
            self._h = None


class FAS:
    """FAS V(6,6) multigrid with the 4th-order flux-form Laplacian (pb_fas_*): the reference's
    LevelMultigridSolver<BoxOp_Laplace>, one periodic box per level."""

    def __init__(self, n, num_levels):
        self.n = n
        h = _vp()
        _check(lib().pb_fas_create(_c_int(n), _c_int(num_levels), ctypes.byref(h)), "pb_fas_create")
        self._h = h

    def solve(self, force, phi, max_iter=20, tol=1e-10, stream=None):
        it = _c_int()
        hist = (ctypes.c_double * (max_iter + 1))()
        _check(lib().pb_fas_solve(self._h, _ptr(force), _ptr(phi), _c_int(max_iter), _c_dbl(tol), ctypes.byref(it),
                                  hist, _stream(stream)), "pb_fas_solve")
        return it.value, [hist[k] for k in range(it.value + 1)]

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.pb_fas_destroy(self._h)
            self._h = None


class Serve:
    """Serving engine (pb_serve_*): in-flight solves advance together, one V-cycle per step.

    Requests carry host numpy float64 arrays (rhs read at admission, out written at completion);
    the engine keeps references until the request completes."""

    def __init__(self, hbm_budget, max_active=64, nu1=4, nu2=4, nu_bottom=10, omega=2.0 / 3.0, tol=1e-8,
                 max_cycles=100, precision=MG_MIXED):
        self.params = pb_serve_params(int(hbm_budget), max_active, nu1, nu2, nu_bottom, omega, tol, max_cycles,
                                      precision)
        h = _vp()
        _check(lib().pb_serve_create(ctypes.byref(self.params), ctypes.byref(h)), "pb_serve_create")
        self._h = h
        self._keep = {}

    @staticmethod
    def request_bytes(n, precision=MG_MIXED):
        return lib().pb_serve_hierarchy_bytes(_c_int(n), _c_int(precision))

    def submit(self, n, rhs, out, form=MG_POISSON, alpha=0.0, beta=1.0):
        import numpy as np
        assert rhs.dtype == np.float64 and out.dtype == np.float64 and rhs.size == n ** 3 and out.size == n ** 3
        assert rhs.flags["C_CONTIGUOUS"] and out.flags["C_CONTIGUOUS"]
        q = pb_serve_request(n, form, alpha, beta, rhs.ctypes.data, out.ctypes.data)
        t = _c_ll()
        _check(lib().pb_serve_submit(self._h, ctypes.byref(q), ctypes.byref(t)), "pb_serve_submit")
        self._keep[t.value] = (rhs, out)
        return t.value

    def step(self):
        a, w = _c_int(), _c_int()
        _check(lib().pb_serve_step(self._h, ctypes.byref(a), ctypes.byref(w)), "pb_serve_step")
        return a.value, w.value

    def poll(self, cap=4096):
        buf = (_c_ll * cap)()
        n = _c_int()
        _check(lib().pb_serve_poll(self._h, buf, _c_int(cap), ctypes.byref(n)), "pb_serve_poll")
        done = [buf[i] for i in range(n.value)]
        for t in done:
            self._keep.pop(t, None)
        return done

    def status(self, ticket):
        st, cy, rr = _c_int(), _c_int(), _c_dbl()
        _check(lib().pb_serve_status(self._h, _c_ll(ticket), ctypes.byref(st), ctypes.byref(cy), ctypes.byref(rr)),
               "pb_serve_status")
        return st.value, cy.value, rr.value

    def device_bytes(self):
        return lib().pb_serve_device_bytes(self._h)

    def timing(self):
        """Host seconds per step stage (admit, lists, first residual, cycle, retire) and steps."""
        t = (_c_dbl * 5)()
        n = _c_ll()
        _check(lib().pb_serve_timing(self._h, t, ctypes.byref(n)), "pb_serve_timing")
        return dict(zip(("admit", "lists", "first_residual", "cycle", "retire"), list(t)), steps=n.value)

    def run_until_idle(self, max_steps=100000):
        for _ in range(max_steps):
            a, w = self.step()
            if a == 0 and w == 0:
                return
        raise RuntimeError("serve: not idle after %d steps" % max_steps)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.pb_serve_destroy(self._h)
            self._h = None
