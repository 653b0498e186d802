"""ctypes binding of the CPU restatement oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this as the checker.  The product
(``cuda-fabipb_b200``) never imports it.

Also runs the reference CPU solver compiled from its own sources
(``oracle/_ref/ref_harness``) for the pin tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_HARNESS = os.path.join(REF_DIR, "ref_harness")
REF_BINARY = os.path.join(REF_DIR, "fabipb_ref")
# the reference's own CUDA backend built from its sources (make -C oracle refgpu)
REF_HARNESS_GPU = os.path.join(REF_DIR, "ref_harness_gpu")
REF_BINARY_GPU = os.path.join(REF_DIR, "fabipb_refgpu")


class Params(C.Structure):
    _fields_ = [("order", C.c_int), ("order_mom", C.c_int), ("depth", C.c_int),
                ("height", C.c_int), ("quad_order", C.c_int), ("sep_ratio", C.c_double),
                ("kappa", C.c_double), ("eps1", C.c_double), ("eps2", C.c_double),
                ("rhs_theta", C.c_double), ("energy_theta", C.c_double),
                ("charge_order", C.c_int), ("threads", C.c_int)]


def build(quiet=True):
    """Compile liboracle.so (and, when the reference sources are present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=out)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(Params), C.c_int, dp, dp, dp]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_set_charges.argtypes = [C.c_void_p, C.c_int, dp, dp]
        for name in ("or_num_panels", "or_num_leaves", "or_num_near_pairs", "or_num_m2l_pairs",
                     "or_num_cubes", "or_max_order"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_int
        L.or_panel_order.argtypes = [C.c_void_p, ip]
        L.or_leaf_layout.argtypes = [C.c_void_p, ip, ip]
        L.or_near_pairs.argtypes = [C.c_void_p, ip, ip]
        L.or_m2l_pairs.argtypes = [C.c_void_p, ip, ip]
        L.or_cube_data.argtypes = [C.c_void_p, ip, ip, dp]
        L.or_area_tree.argtypes = [C.c_void_p, dp]
        L.or_panel_ia0.argtypes = [C.c_void_p, C.c_int, C.c_int, dp]
        L.or_near_apply.argtypes = [C.c_void_p, C.c_double, dp, dp]
        L.or_fmm_apply.argtypes = [C.c_void_p, C.c_double, dp, C.c_double, dp]
        L.or_far_apply.argtypes = [C.c_void_p, C.c_double, dp, C.c_double, dp]
        L.or_matvec.argtypes = [C.c_void_p, C.c_double, dp, C.c_double, dp]
        L.or_rhs_direct.argtypes = [C.c_void_p, dp]
        L.or_rhs_tree.argtypes = [C.c_void_p, dp]
        L.or_energy_tree.argtypes = [C.c_void_p, dp]
        L.or_energy_tree.restype = C.c_double
        L.or_precond_setup.argtypes = [C.c_void_p, C.c_int]
        L.or_precond_setup.restype = C.c_int
        L.or_precond_apply.argtypes = [C.c_void_p, dp, dp]
        L.or_gmres.argtypes = [C.c_void_p, dp, dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.or_gmres.restype = C.c_int
        _lib = L
    return _lib


def make_params(order=3, depth=3, height=2, sep_ratio=0.8, quad_order=1, kappa=0.1257,
                eps1=1.0, eps2=80.0, order_mom=0, rhs_theta=0.8, energy_theta=0.8,
                charge_order=0, threads=0):
    return Params(order, order_mom, depth, height, quad_order, sep_ratio, kappa, eps1, eps2,
                  rhs_theta, energy_theta, charge_order, threads)


class Oracle:
    """FP64 restatement of the reference on one panel set (tree order inside)."""

    def __init__(self, panels, params: Params, charges=None):
        L = lib()
        vtx = np.ascontiguousarray(panels.vtx.reshape(-1), dtype=np.float64)
        nrm = np.ascontiguousarray(panels.normal.reshape(-1), dtype=np.float64)
        area = np.ascontiguousarray(panels.area, dtype=np.float64)
        self.params = params
        self.h = L.or_create(C.byref(params), int(panels.n), vtx, nrm, area)
        if not self.h:
            raise RuntimeError("oracle tree construction failed")
        self.n = L.or_num_panels(self.h)
        if charges is not None:
            L.or_set_charges(self.h, int(charges.q.shape[0]),
                             np.ascontiguousarray(charges.pos.reshape(-1)),
                             np.ascontiguousarray(charges.q))

    def set_charges(self, charges):
        lib().or_set_charges(self.h, int(charges.q.shape[0]), np.ascontiguousarray(charges.pos.reshape(-1)),
                             np.ascontiguousarray(charges.q))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    # tree
    def counts(self):
        L = lib()
        return dict(panels=self.n, leaves=L.or_num_leaves(self.h), near=L.or_num_near_pairs(self.h),
                    m2l=L.or_num_m2l_pairs(self.h), cubes=L.or_num_cubes(self.h),
                    max_order=L.or_max_order(self.h))

    def panel_order(self):
        o = np.zeros(self.n, np.int32)
        lib().or_panel_order(self.h, o)
        return o

    def leaf_layout(self):
        c = self.counts()
        s = np.zeros(c["leaves"], np.int32)
        k = np.zeros(c["leaves"], np.int32)
        lib().or_leaf_layout(self.h, s, k)
        return s, k

    def near_pairs(self):
        c = self.counts()
        s = np.zeros(c["near"], np.int32)
        d = np.zeros(c["near"], np.int32)
        lib().or_near_pairs(self.h, s, d)
        return s, d

    def m2l_pairs(self):
        c = self.counts()
        s = np.zeros(max(c["m2l"], 1), np.int32)
        d = np.zeros(max(c["m2l"], 1), np.int32)
        lib().or_m2l_pairs(self.h, s, d)
        return s[:c["m2l"]], d[:c["m2l"]]

    def cube_data(self):
        c = self.counts()["cubes"]
        lev = np.zeros(c, np.int32)
        cnt = np.zeros(c, np.int32)
        ctr = np.zeros(4 * c, np.float64)
        lib().or_cube_data(self.h, lev, cnt, ctr)
        return lev, cnt, ctr.reshape(c, 4)

    def area(self):
        a = np.zeros(self.n)
        lib().or_area_tree(self.h, a)
        return a

    def panel_ia0(self, x, y):
        out = np.zeros(4)
        lib().or_panel_ia0(self.h, int(x), int(y), out)
        return out

    # operators
    def near_apply(self, sgm, alpha=1.0, pot=None):
        pot = np.zeros(2 * self.n) if pot is None else np.array(pot, dtype=np.float64)
        lib().or_near_apply(self.h, alpha, np.ascontiguousarray(sgm, dtype=np.float64), pot)
        return pot

    def far_apply(self, sgm, alpha=1.0, beta=0.0, pot=None):
        pot = np.zeros(2 * self.n) if pot is None else np.array(pot, dtype=np.float64)
        lib().or_far_apply(self.h, alpha, np.ascontiguousarray(sgm, dtype=np.float64), beta, pot)
        return pot

    def fmm_apply(self, sgm, alpha=1.0, beta=0.0, pot=None):
        pot = np.zeros(2 * self.n) if pot is None else np.array(pot, dtype=np.float64)
        lib().or_fmm_apply(self.h, alpha, np.ascontiguousarray(sgm, dtype=np.float64), beta, pot)
        return pot

    def matvec(self, x, alpha=1.0, beta=0.0, y=None):
        y = np.zeros(2 * self.n) if y is None else np.array(y, dtype=np.float64)
        lib().or_matvec(self.h, alpha, np.ascontiguousarray(x, dtype=np.float64), beta, y)
        return y

    def rhs_direct(self):
        r = np.zeros(2 * self.n)
        lib().or_rhs_direct(self.h, r)
        return r

    def rhs_tree(self):
        r = np.zeros(2 * self.n)
        lib().or_rhs_tree(self.h, r)
        return r

    def energy_raw(self, sgm):
        return float(lib().or_energy_tree(self.h, np.ascontiguousarray(sgm, dtype=np.float64)))

    def precond_setup(self, mode):
        if not lib().or_precond_setup(self.h, int(mode)):
            raise RuntimeError("oracle preconditioner factorisation failed")

    def precond_apply(self, b):
        x = np.zeros(2 * self.n)
        lib().or_precond_apply(self.h, np.ascontiguousarray(b, dtype=np.float64), x)
        return x

    def gmres(self, b, x0, restart, maxit, tol):
        x = np.array(x0, dtype=np.float64)
        it = C.c_int(maxit)
        res = C.c_double(tol)
        info = lib().or_gmres(self.h, np.ascontiguousarray(b), x, int(restart), C.byref(it), C.byref(res))
        return x, it.value, res.value, info


def ref_available():
    return os.path.exists(REF_HARNESS) and os.path.exists(REF_BINARY)


def ref_env(threads=None):
    env = dict(os.environ)
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS",
              "VECLIB_MAXIMUM_THREADS", "BLIS_NUM_THREADS"):
        env[k] = "1"
    env["FABIPB_REUSE_MESH"] = "1"
    env["FABIPB_THREAD_ENV_REEXEC"] = "1"
    if threads is not None:
        for k in ("FABIPB_SETUP_THREADS", "FABIPB_NEARFIELD_APPLY_THREADS",
                  "FABIPB_PRECOND_APPLY_THREADS", "FABIPB_RHS_THREADS", "FABIPB_ENERGY_THREADS",
                  "FABIPB_GMRES_BASIS_THREADS"):
            env[k] = str(threads)
    return env


def run_ref_harness(mode, base, out_prefix, opts, sigma=None, threads=None, reps=None, warmup=None,
                    extra_env=None, budget=None, gpu=False, timeout=None):
    """Run oracle/_ref/ref_harness (gpu: ref_harness_gpu with -g=1, the
    reference's CUDA backend); return stdout.  Mesh files must sit at ``base``."""
    cmd = [REF_HARNESS_GPU if gpu else REF_HARNESS, mode, base, out_prefix] + list(opts)
    if gpu:
        cmd.append("-g=1")
    if sigma is not None:
        path = out_prefix + ".sigma.in"
        np.ascontiguousarray(sigma, dtype=np.float64).tofile(path)
        cmd.append("--sigma=" + path)
    if reps is not None:
        cmd.append("--reps=%d" % reps)
    if warmup is not None:
        cmd.append("--warmup=%d" % warmup)
    if budget is not None:
        cmd.append("--budget=%g" % budget)
    env = ref_env(threads)
    if extra_env:
        env.update(extra_env)
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, check=True, timeout=timeout)
    return r.stdout


def read_bin(out_prefix, name, dtype):
    return np.fromfile("%s.%s.bin" % (out_prefix, name), dtype=dtype)


def run_ref_solve(base, opts, threads=None, extra_env=None):
    """Run the reference CLI (CPU path); return (energy, iterations, residual, stdout)."""
    env = ref_env(threads)
    if extra_env:
        env.update(extra_env)
    r = subprocess.run([REF_BINARY, "-g=0", "-m=1"] + list(opts) + [base], env=env,
                       capture_output=True, text=True, check=True)
    energy = iters = resid = None
    for line in r.stdout.splitlines():
        if line.startswith("solvation energy:"):
            energy = float(line.split(":")[1])
        elif line.startswith("GMRES status:"):
            parts = dict(p.split("=") for p in line.split(":")[1].split())
            iters = int(parts["iterations"])
            resid = float(parts["final-residual"])
    return energy, iters, resid, r.stdout
