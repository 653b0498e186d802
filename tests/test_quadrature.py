"""Panel quadrature order -q=2 against the reference CPU solver at -q=2
(tests/golden/quad_cases.json and <case>_q2.npz, written by
tests/golden/make_golden.py --quad from the reference binary).

At -q>1 the near field evaluates panelIA0 at order q for every near pair
(src/numQuad.c:629-697: q^4 kernel evaluations for a disjoint pair, the
Sauter rules at order q for touching ones) in FP64 (near_quad_kernel), in FP64
and mixed contexts alike; the right-hand side and the panel-tree energy take q^2
points per panel.

Tolerances: near field, FP64 matvec, direct RHS and energy 1e-12 relative (the
parity tolerances of the -q=1 goldens); the mixed matvec 5e-6 (its FMM passes
are FP32); the transposed near field by duality to 1e-12; the drop-in CLI
(-g=1 -q=2, the reference host's own preconditioner) with the reference's
iteration count and printed energy.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, case_params, rel_l2
from fabipb_b200 import lib, meshio
import make_golden

pytestmark = pytest.mark.gpu
Q = make_golden.QUAD_ORDER


@pytest.fixture(scope="module")
def quad_meta():
    with open(os.path.join(GOLDEN, "quad_cases.json")) as fp:
        return json.load(fp)


def surface(case_dir, quad_meta, name, precision, charges=False):
    opts = quad_meta[name]["opts"]
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    s = lib.Surface(pan, lib.params(precision=precision, quad_order=opts["q"], **case_params(opts)))
    if charges:
        s.set_charges(ch)
    return s


@pytest.mark.parametrize("name", make_golden.QUAD_CASES)
@pytest.mark.parametrize("precision,tol", [(lib.FP64, 1e-12), (lib.MIXED, 5e-6)])
def test_quad_near_field_and_matvec(name, precision, tol, case_dir, quad_meta):
    g = np.load(os.path.join(GOLDEN, "%s_q%d.npz" % (name, Q)))
    s = surface(case_dir, quad_meta, name, precision)
    sg = make_golden.seeded_sigma(s.n)
    assert rel_l2(s.apply(sg, part=lib.NEAR), g["near"]) < 1e-12
    assert rel_l2(s.matvec(sg), g["matvec"]) < tol


@pytest.mark.parametrize("name", make_golden.QUAD_CASES)
def test_quad_transposed_near_field(name, case_dir, quad_meta):
    """<lam, K_near sg> = <K_near^T lam, sg> for the order-q near field."""
    s = surface(case_dir, quad_meta, name, lib.FP64)
    sg = make_golden.seeded_sigma(s.n, 4)
    lam = make_golden.seeded_sigma(s.n, 5)
    ksg = s.apply(sg, part=lib.NEAR)
    ktl = s.apply_adjoint(lam, part=lib.NEAR)
    lhs, rhs = float(lam @ ksg), float(ktl @ sg)
    assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(lam) * np.linalg.norm(ksg)


@pytest.mark.parametrize("name", make_golden.QUAD_CASES)
def test_quad_rhs_and_energy(name, case_dir, quad_meta):
    g = np.load(os.path.join(GOLDEN, "%s_q%d.npz" % (name, Q)))
    s = surface(case_dir, quad_meta, name, lib.FP64, charges=True)
    assert rel_l2(s.rhs(use_tree=False), g["rhs"]) < 1e-12
    e = s.energy_raw(make_golden.seeded_sigma(s.n))
    ref = float(np.asarray(g["energy_raw"]).ravel()[0])
    assert abs(e - ref) <= 1e-12 * abs(ref)


@pytest.mark.parametrize("name", make_golden.QUAD_CASES)
def test_quad_dropin_solve_matches_cpu_reference(name, case_dir, quad_meta):
    import test_dropin as D
    if not os.path.exists(D.DROPIN):
        pytest.skip("drop-in binary not built (make -C oracle dropin)")
    meta = quad_meta[name]
    out = D.run_dropin(os.path.join(case_dir, name), meta["opts"], extra=["-q=%d" % Q])
    assert "CPU fallback" not in out and "unavailable" not in out, out
    e, it = D.parse(out)
    assert it == meta["solve"]["iterations"]
    assert abs(e - meta["solve"]["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.parametrize("name", make_golden.QUAD_CASES)
def test_quad_library_solve(name, case_dir, quad_meta):
    """The library's own device solve at -q=2 (FP64 operator; its block
    preconditioner assembled from one-point terms plus the order-q special
    pairs, where the reference's evaluates every block pair at order q):
    converged, the reference's energy within ten times the GMRES tolerance,
    its iteration count within two."""
    meta = quad_meta[name]
    opts = meta["opts"]
    s = surface(case_dir, quad_meta, name, lib.FP64, charges=True)
    b = s.rhs(use_tree=False)
    s.precond_setup(2)
    x, it, res, info = s.solve(b, b.copy(), restart=opts["a"], maxit=100, tol=opts["o"])
    e = s.energy_raw(x) * 2 * np.pi * 332.0716
    assert info == 0
    assert abs(it - meta["solve"]["iterations"]) <= 2
    assert abs(e - meta["solve"]["energy"]) <= 10 * opts["o"] * abs(meta["solve"]["energy"])
