"""Mixed-precision iterative refinement (fabipb_b200_solve_refined) through
the C ABI: FP32 near-field corrections with FP64 residuals reach the FP64
solution far below the FP32 floor of the plain mixed solve.

Checks against the FP64 context's own GMRES solution at the same tolerance:
solution relative L2 <= 1e-9 and raw energy relative 1e-10 at tol 1e-11.
"""
import os

import numpy as np
import pytest

from conftest import case_params, rel_l2
from fabipb_b200 import lib, meshio

pytestmark = pytest.mark.gpu


def surface(case_dir, meta, name, precision):
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    prm = lib.params(precision=precision, **case_params(meta[name]["opts"]))
    return lib.Surface(pan, prm, ch)


@pytest.mark.parametrize("name", ["sphere1280", "star2048"])
def test_refined_mixed_matches_fp64(name, case_dir, golden_meta):
    restart = golden_meta[name]["opts"]["a"]
    s64 = surface(case_dir, golden_meta, name, lib.FP64)
    b = s64.rhs()
    s64.precond_setup(2)
    x64, it64, res64, info64 = s64.solve(b, b.copy(), restart=restart, maxit=1000, tol=1e-11)
    assert info64 == 0
    s32 = surface(case_dir, golden_meta, name, lib.MIXED)
    s32.precond_setup(2)
    x, outer, its, res, info = s32.solve_refined(b, b.copy(), restart=restart, maxit=1000, tol_inner=1e-5,
                                                 tol=1e-11, max_outer=30)
    assert info == 0 and res <= 1e-11, (outer, its, res, info)
    assert outer >= 2
    assert rel_l2(x, x64) <= 1e-9
    # both energies through the FP64 walk: the solutions are compared, not the
    # mixed context's FP32 energy walk
    e, e64 = s64.energy_raw(x), s64.energy_raw(x64)
    assert abs(e - e64) <= 1e-10 * abs(e64)


def test_refined_fp64_is_plain_gmres_accuracy(case_dir, golden_meta):
    """In an FP64 context the corrections use the FP64 operator too."""
    name = "sphere1280"
    s = surface(case_dir, golden_meta, name, lib.FP64)
    b = s.rhs()
    s.precond_setup(2)
    x, outer, its, res, info = s.solve_refined(b, b.copy(), restart=10, maxit=500, tol_inner=1e-6, tol=1e-12)
    assert info == 0 and res <= 1e-12
    xr, _, _, _ = s.solve(b, b.copy(), restart=10, maxit=1000, tol=1e-12)
    assert rel_l2(x, xr) <= 1e-10
