"""Parity at the benchmark configurations' sizes, through the C ABI.

* sphere20480 (the 20,480-panel Kirkwood sphere), star204800 (the
  204,800-panel star surface) and shell16384 (the two-shell geometry of the
  capsid-scale configuration, radii 200/230 A, at a coarse 16,384-panel
  resolution, diagonal preconditioner): the FP64 device solve against the
  reference CLI's own -g=0 run on the same mesh and options (goldens in
  tests/golden/solve_cases.json, written by make_golden.py --large): the same
  GMRES iteration count and the printed energy (%f) to its last digit; the
  mixed solve within 1e-4 of that energy, iterations within one.
* The library's direct context (every panel pair, no FMM) solved in FP64
  against the reference's dense direct mode -r=2 (cpuDirectApply,
  src/direct_backend.c:172): same iterations, energy to the last digit.
* The direct context's matvec against the FMM context's at FP64: the FMM's
  far-field truncation error only (relative L2 below 1e-3 at p=3..5).
"""
import os

import numpy as np
import pytest

from conftest import case_params, rel_l2
from fabipb_b200 import lib, meshio
import make_golden

pytestmark = pytest.mark.gpu
KCAL = 2 * np.pi * 332.0716


@pytest.fixture(scope="module")
def large_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("large")
    for name in make_golden.SOLVE_CASES:
        make_golden.generate_mesh(name, str(d))
    return str(d)


def _solve(pan, ch, opts, precision, direct=False):
    s = lib.Surface(pan, lib.params(precision=precision, **case_params(opts)), ch, direct=direct)
    b = s.rhs(use_tree=False)
    s.precond_setup(opts.get("P", 2))
    x, it, res, info = s.solve(b, b.copy(), restart=opts["a"], maxit=100, tol=opts["o"])
    e = s.energy_raw(x) * KCAL
    s.close()
    return e, it, res, info


@pytest.mark.parametrize("name", list(make_golden.SOLVE_CASES))
def test_large_solve_fp64_matches_reference(name, large_dir, solve_meta):
    meta = solve_meta[name]
    assert make_golden.mesh_digest(os.path.join(large_dir, name)) == meta["digest"]
    pan, ch = meshio.load_case(os.path.join(large_dir, name))
    e, it, res, info = _solve(pan, ch, meta["opts"], lib.FP64)
    assert info == 0
    assert it == meta["solve"]["iterations"]
    assert abs(res - meta["solve"]["residual"]) <= 1e-3 * meta["solve"]["residual"]
    assert abs(e - meta["solve"]["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.parametrize("name", list(make_golden.SOLVE_CASES))
def test_large_solve_mixed_energy(name, large_dir, solve_meta):
    meta = solve_meta[name]
    pan, ch = meshio.load_case(os.path.join(large_dir, name))
    e, it, res, info = _solve(pan, ch, meta["opts"], lib.MIXED)
    assert info == 0
    assert abs(it - meta["solve"]["iterations"]) <= 1
    assert abs(e - meta["solve"]["energy"]) <= 1e-4 * abs(meta["solve"]["energy"])


@pytest.mark.parametrize("name", list(make_golden.DIRECT_CASES))
def test_direct_context_matches_reference_direct(name, case_dir, golden_meta, solve_meta):
    opts = golden_meta[name]["opts"]
    ref = solve_meta["direct"][name]
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    e, it, res, info = _solve(pan, ch, opts, lib.FP64, direct=True)
    assert info == 0
    assert it == ref["iterations"]
    assert abs(e - ref["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.parametrize("name", list(make_golden.DIRECT_CASES))
def test_direct_context_matvec_vs_fmm(name, case_dir, golden_meta):
    opts = golden_meta[name]["opts"]
    pan, _ = meshio.load_case(os.path.join(case_dir, name))
    prm = lib.params(precision=lib.FP64, **case_params(opts))
    sd = lib.Surface(pan, prm, direct=True)
    sf = lib.Surface(pan, prm)
    x = make_golden.seeded_sigma(pan.n, 4)
    yd, yf = sd.matvec(x), sf.matvec(x)
    assert 0.0 < rel_l2(yf, yd) < 1e-3
    # the adjoint of the direct operator is its transpose: <u, A v> = <A^T u, v>
    u = make_golden.seeded_sigma(pan.n, 5)
    lhs = float(u @ sd.matvec(x))
    rhs = float(sd.matvec_adjoint(u) @ x)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
