"""ctypes binding of the C ABI in include/fabipb_b200.h.

The CUDA library is required: if it is missing or cannot load, every call
raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libfabipb_b200.so")

FP64 = 0
MIXED = 1
NEAR = 1
FAR = 2
ALL = 3


class Params(C.Structure):
    _fields_ = [("order", C.c_int), ("order_mom", C.c_int), ("depth", C.c_int), ("height", C.c_int),
                ("quad_order", C.c_int), ("sep_ratio", C.c_double), ("kappa", C.c_double),
                ("eps1", C.c_double), ("eps2", C.c_double), ("rhs_theta", C.c_double),
                ("energy_theta", C.c_double), ("charge_order", C.c_int), ("precision", C.c_int),
                ("device", C.c_int)]


class Info(C.Structure):
    _fields_ = [("panels", C.c_int), ("leaves", C.c_int), ("near_pairs", C.c_int), ("m2l_pairs", C.c_int),
                ("cubes", C.c_int), ("max_order", C.c_int), ("leaf_order", C.c_int), ("max_leaf", C.c_int),
                ("near_panel_pairs", C.c_longlong), ("special_pairs", C.c_longlong),
                ("setup_seconds", C.c_double), ("device_bytes", C.c_double)]


_lib = None


def load():
    """Load libfabipb_b200.so (raises if it is absent: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libfabipb_b200.so is not built (run cuda-fabipb_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.fabipb_b200_default_params.argtypes = [C.POINTER(Params)]
    L.fabipb_b200_create.argtypes = [C.POINTER(Params), C.c_int, vp, vp, vp, C.POINTER(vp)]
    L.fabipb_b200_create_direct.argtypes = [C.POINTER(Params), C.c_int, vp, vp, vp, C.POINTER(vp)]
    L.fabipb_b200_set_charges.argtypes = [vp, C.c_int, vp, vp]
    L.fabipb_b200_destroy.argtypes = [vp]
    L.fabipb_b200_set_stream.argtypes = [vp, vp]
    L.fabipb_b200_launch_count.argtypes = [vp]
    L.fabipb_b200_launch_count.restype = C.c_longlong
    L.fabipb_b200_last_error.restype = C.c_char_p
    L.fabipb_b200_info_get.argtypes = [vp, C.POINTER(Info)]
    L.fabipb_b200_panel_order.argtypes = [vp, vp]
    L.fabipb_b200_leaf_layout.argtypes = [vp, vp, vp]
    L.fabipb_b200_near_pairs.argtypes = [vp, vp, vp]
    L.fabipb_b200_m2l_pairs.argtypes = [vp, vp, vp]
    L.fabipb_b200_cube_data.argtypes = [vp, vp, vp]
    L.fabipb_b200_apply.argtypes = [vp, C.c_int, C.c_double, vp, C.c_double, vp, C.c_int]
    L.fabipb_b200_matvec.argtypes = [vp, C.c_double, vp, C.c_double, vp, C.c_int]
    L.fabipb_b200_energy_weights.argtypes = [vp, vp, C.c_int]
    L.fabipb_b200_solve_refined.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, vp, vp,
                                            vp, vp, C.c_int]
    L.fabipb_b200_pass_times.argtypes = [vp, vp, C.c_int, vp, C.c_int]
    L.fabipb_b200_forward.argtypes = [vp, C.c_int, C.c_int, C.c_double, vp, vp, vp, vp]
    L.fabipb_b200_backward.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.c_double, vp, vp, vp, vp, vp, C.c_int]
    L.fabipb_b200_apply_adjoint.argtypes = [vp, C.c_int, C.c_double, vp, C.c_double, vp, C.c_int]
    L.fabipb_b200_matvec_adjoint.argtypes = [vp, C.c_double, vp, C.c_double, vp, C.c_int]
    for name, args in (("fabipb_b200_rhs", [vp, C.c_int, vp, C.c_int]),
                       ("fabipb_b200_energy", [vp, vp, vp, C.c_int]),
                       ("fabipb_b200_precond_setup", [vp, C.c_int]),
                       ("fabipb_b200_precond_apply", [vp, vp, vp, C.c_int]),
                       ("fabipb_b200_solve", [vp, vp, vp, C.c_int, C.c_int, C.c_double, vp, vp, vp, C.c_int])):
        if hasattr(L, name):
            getattr(L, name).argtypes = args
    _lib = L
    return L


def simt_peak_tflops(device=0, fp64=False) -> float:
    """Measured FMA rate of `device`'s FP32 (or FP64) pipe in TFLOP/s."""
    L = load()
    L.fabipb_b200_simt_peak.argtypes = [C.c_int, C.c_int, C.c_void_p]
    v = np.zeros(1)
    _check(L.fabipb_b200_simt_peak(int(device), int(bool(fp64)), _ptr(v)), "simt_peak")
    return float(v[0])


def last_error() -> str:
    return load().fabipb_b200_last_error().decode(errors="replace")


def _check(ok, what):
    if not ok:
        raise RuntimeError("%s failed: %s" % (what, last_error()))


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a)  # a device pointer (e.g. torch tensor .data_ptr())


def params(order=3, depth=5, height=2, sep_ratio=0.8, quad_order=1, kappa=0.1257, eps1=1.0, eps2=80.0,
           order_mom=0, rhs_theta=0.8, energy_theta=0.8, charge_order=0, precision=MIXED, device=0):
    p = Params()
    load().fabipb_b200_default_params(C.byref(p))
    p.order, p.order_mom, p.depth, p.height, p.quad_order = order, order_mom, depth, height, quad_order
    p.sep_ratio, p.kappa, p.eps1, p.eps2 = sep_ratio, kappa, eps1, eps2
    p.rhs_theta, p.energy_theta, p.charge_order = rhs_theta, energy_theta, charge_order
    p.precision, p.device = precision, device
    return p


class Surface:
    """One panel mesh resident on the GPU (see include/fabipb_b200.h)."""

    def __init__(self, panels, prm: Params, charges=None, direct=False):
        """direct=True: the dense direct operator (every panel pair, no FMM)."""
        L = load()
        self._vtx = np.ascontiguousarray(panels.vtx.reshape(-1), dtype=np.float64)
        self._nrm = np.ascontiguousarray(panels.normal.reshape(-1), dtype=np.float64)
        self._area = np.ascontiguousarray(panels.area, dtype=np.float64)
        h = C.c_void_p()
        make = L.fabipb_b200_create_direct if direct else L.fabipb_b200_create
        _check(make(C.byref(prm), int(panels.n), _ptr(self._vtx), _ptr(self._nrm), _ptr(self._area), C.byref(h)),
               "fabipb_b200_create")
        self.h = h
        self.params = prm
        self.n = int(panels.n)
        self.n_charges = 0
        if charges is not None:
            self.set_charges(charges)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            load().fabipb_b200_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_charges(self, charges):
        pos = np.ascontiguousarray(charges.pos.reshape(-1), dtype=np.float64)
        q = np.ascontiguousarray(charges.q, dtype=np.float64)
        _check(load().fabipb_b200_set_charges(self.h, int(q.shape[0]), _ptr(pos), _ptr(q)), "set_charges")
        self.n_charges = int(q.shape[0])

    def launch_count(self):
        return int(load().fabipb_b200_launch_count(self.h))

    def set_stream(self, stream_handle):
        _check(load().fabipb_b200_set_stream(self.h, stream_handle), "set_stream")

    def info(self):
        i = Info()
        _check(load().fabipb_b200_info_get(self.h, C.byref(i)), "info")
        return {k: getattr(i, k) for k, _ in Info._fields_}

    def panel_order(self):
        o = np.zeros(self.n, np.int32)
        _check(load().fabipb_b200_panel_order(self.h, _ptr(o)), "panel_order")
        return o

    def leaf_layout(self):
        nl = self.info()["leaves"]
        s = np.zeros(nl, np.int32)
        c = np.zeros(nl, np.int32)
        _check(load().fabipb_b200_leaf_layout(self.h, _ptr(s), _ptr(c)), "leaf_layout")
        return s, c

    def near_pairs(self):
        k = self.info()["near_pairs"]
        s = np.zeros(k, np.int32)
        d = np.zeros(k, np.int32)
        _check(load().fabipb_b200_near_pairs(self.h, _ptr(s), _ptr(d)), "near_pairs")
        return s, d

    def m2l_pairs(self):
        k = self.info()["m2l_pairs"]
        s = np.zeros(max(k, 1), np.int32)
        d = np.zeros(max(k, 1), np.int32)
        _check(load().fabipb_b200_m2l_pairs(self.h, _ptr(s), _ptr(d)), "m2l_pairs")
        return s[:k], d[:k]

    def cube_data(self):
        k = self.info()["cubes"]
        lev = np.zeros(k, np.int32)
        ctr = np.zeros(4 * k)
        _check(load().fabipb_b200_cube_data(self.h, _ptr(lev), _ptr(ctr)), "cube_data")
        return lev, ctr.reshape(k, 4)

    # operators (host numpy arrays, or device pointers with on_device=1)
    def apply(self, sgm, part=ALL, alpha=1.0, beta=0.0, pot=None, on_device=0):
        if on_device:
            _check(load().fabipb_b200_apply(self.h, part, alpha, _ptr(sgm), beta, _ptr(pot), 1), "apply")
            return pot
        sgm = np.ascontiguousarray(sgm, dtype=np.float64)
        pot = np.zeros(2 * self.n) if pot is None else np.array(pot, dtype=np.float64)
        _check(load().fabipb_b200_apply(self.h, part, alpha, _ptr(sgm), beta, _ptr(pot), 0), "apply")
        return pot

    def _host_out(self, y, out, beta):
        """The host array the library writes: `out` itself when it is a
        writeable C-contiguous float64 array of 2N (no copy: a pinned buffer
        stays pinned), else a fresh array; holds y on entry when beta != 0."""
        if (out is not None and isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                and out.flags.writeable and out.size == 2 * self.n):
            if beta != 0.0 and y is not None and y is not out:
                out[:] = y
            return out
        return np.zeros(2 * self.n) if y is None else np.array(y, dtype=np.float64)

    def matvec(self, x, alpha=1.0, beta=0.0, y=None, on_device=0, out=None):
        """y_new = alpha*(D - K)x + beta*y; host arrays are not modified
        unless `out` is given, which receives the result in place."""
        if on_device:
            _check(load().fabipb_b200_matvec(self.h, alpha, _ptr(x), beta, _ptr(y), 1), "matvec")
            return y
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = self._host_out(y, out, beta)
        _check(load().fabipb_b200_matvec(self.h, alpha, _ptr(x), beta, _ptr(y), 0), "matvec")
        return y

    def apply_adjoint(self, lam, part=ALL, alpha=1.0, beta=0.0, out=None, on_device=0):
        """out = beta*out + alpha*K_part^T lam (the transposed operator)."""
        if on_device:
            _check(load().fabipb_b200_apply_adjoint(self.h, part, alpha, _ptr(lam), beta, _ptr(out), 1),
                   "apply_adjoint")
            return out
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        out = np.zeros(2 * self.n) if out is None else np.array(out, dtype=np.float64)
        _check(load().fabipb_b200_apply_adjoint(self.h, part, alpha, _ptr(lam), beta, _ptr(out), 0), "apply_adjoint")
        return out

    def matvec_adjoint(self, x, alpha=1.0, beta=0.0, y=None, on_device=0):
        """y = alpha*(D - K)^T x + beta*y."""
        if on_device:
            _check(load().fabipb_b200_matvec_adjoint(self.h, alpha, _ptr(x), beta, _ptr(y), 1), "matvec_adjoint")
            return y
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(2 * self.n) if y is None else np.array(y, dtype=np.float64)
        _check(load().fabipb_b200_matvec_adjoint(self.h, alpha, _ptr(x), beta, _ptr(y), 0), "matvec_adjoint")
        return y

    PASSES = ("near", "q2m", "m2m", "m2l", "l2l", "l2p")

    def pass_times(self, x, reps=5, on_device=0):
        """Mean milliseconds per matvec pass (near, q2m, m2m, m2l, l2l, l2p)."""
        ms = np.zeros(6)
        if not on_device:
            x = np.ascontiguousarray(x, dtype=np.float64)
        _check(load().fabipb_b200_pass_times(self.h, _ptr(x), int(reps), _ptr(ms), int(on_device)), "pass_times")
        return dict(zip(self.PASSES, ms.tolist()))

    def solve_refined(self, b, x0, restart=10, maxit=200, tol_inner=1e-5, tol=1e-10, max_outer=20, on_device=0):
        """Iterative refinement (FP64 residuals, corrections by GMRES on this
        context's operator); returns (x, outer, iters, resid, info).
        on_device=1: b and x0 are device pointers, x0 is overwritten."""
        if on_device:
            x = x0
        else:
            b = np.ascontiguousarray(b, dtype=np.float64)
            x = np.array(x0, dtype=np.float64)
        ou = np.zeros(1, np.int32)
        it = np.zeros(1, np.int32)
        res = np.zeros(1)
        info = np.zeros(1, np.int32)
        _check(load().fabipb_b200_solve_refined(self.h, _ptr(b), _ptr(x), int(restart), int(maxit), float(tol_inner),
                                                float(tol), int(max_outer), _ptr(ou), _ptr(it), _ptr(res), _ptr(info),
                                                int(bool(on_device))), "solve_refined")
        return x, int(ou[0]), int(it[0]), float(res[0]), int(info[0])

    def energy_weights(self):
        """Direct energy weights e (2N, tree order): energy_raw = e . sigma."""
        e = np.zeros(2 * self.n)
        _check(load().fabipb_b200_energy_weights(self.h, _ptr(e), 0), "energy_weights")
        return e

    def forward(self, restart=10, maxit=100, tol=1e-6):
        """Direct RHS, GMRES, direct energy; returns (energy_raw, iters, resid, info)."""
        e = np.zeros(1)
        it = np.zeros(1, np.int32)
        res = np.zeros(1)
        info = np.zeros(1, np.int32)
        _check(load().fabipb_b200_forward(self.h, int(restart), int(maxit), float(tol), _ptr(e), _ptr(it), _ptr(res),
                                          _ptr(info)), "forward")
        return float(e[0]), int(it[0]), float(res[0]), int(info[0])

    def backward(self, grad_energy=1.0, restart=10, maxit=100, tol=1e-6):
        """Adjoint solve and charge gradients of grad_energy * energy_raw:
        returns (dE/dq (M,), dE/dx (M, 3), iters, resid, info)."""
        m = self.n_charges
        dq = np.zeros(m)
        dx = np.zeros(3 * m)
        it = np.zeros(1, np.int32)
        res = np.zeros(1)
        info = np.zeros(1, np.int32)
        _check(load().fabipb_b200_backward(self.h, float(grad_energy), int(restart), int(maxit), float(tol), _ptr(dq),
                                           _ptr(dx), _ptr(it), _ptr(res), _ptr(info), 0), "backward")
        return dq, dx.reshape(m, 3), int(it[0]), float(res[0]), int(info[0])

    def rhs(self, use_tree=False, out=None, on_device=0):
        if on_device:
            _check(load().fabipb_b200_rhs(self.h, int(use_tree), _ptr(out), 1), "rhs")
            return out
        r = np.zeros(2 * self.n)
        _check(load().fabipb_b200_rhs(self.h, int(use_tree), _ptr(r), 0), "rhs")
        return r

    def energy_raw(self, sgm, on_device=0):
        e = np.zeros(1)
        if not on_device:
            sgm = np.ascontiguousarray(sgm, dtype=np.float64)
        _check(load().fabipb_b200_energy(self.h, _ptr(sgm), _ptr(e), int(on_device)), "energy")
        return float(e[0])

    def precond_setup(self, mode):
        _check(load().fabipb_b200_precond_setup(self.h, int(mode)), "precond_setup")

    def precond_apply(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(2 * self.n)
        _check(load().fabipb_b200_precond_apply(self.h, _ptr(b), _ptr(x), 0), "precond_apply")
        return x

    def solve(self, b, x0, restart=10, maxit=100, tol=1e-4, on_device=0):
        """GMRES from x0; on_device=1: b and x0 are device pointers and x0 is
        overwritten with the solution (returned as is)."""
        it = np.zeros(1, np.int32)
        res = np.zeros(1)
        info = np.zeros(1, np.int32)
        if on_device:
            _check(load().fabipb_b200_solve(self.h, _ptr(b), _ptr(x0), int(restart), int(maxit), float(tol),
                                            _ptr(it), _ptr(res), _ptr(info), 1), "solve")
            return x0, int(it[0]), float(res[0]), int(info[0])
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64)
        it = np.zeros(1, np.int32)
        res = np.zeros(1)
        info = np.zeros(1, np.int32)
        _check(load().fabipb_b200_solve(self.h, _ptr(b), _ptr(x), int(restart), int(maxit), float(tol),
                                        _ptr(it), _ptr(res), _ptr(info), 0), "solve")
        return x, int(it[0]), float(res[0]), int(info[0])
