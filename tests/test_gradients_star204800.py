"""Gradients of the solvation energy at the 204,800-panel star surface (the
adjoint configuration: 20,000 charges, p=4, MAC 0.7), and against the
reference's own finite differences.

* FP64 forward/backward (GMRES to 1e-12) against central finite differences
  of the library's FP64 energy on 64 seeded charges: step 1e-5 e for dE/dq
  and 1e-4 A for dE/dx (every finite-difference energy is a full solve of the
  perturbed charge set on the same surface context).
* The mixed-precision forward/backward (FP32 near field, tol 1e-6) against
  the FP64 gradients.
* The FMM gradients against those of the FP64 direct-summation oracle (the
  direct context: every panel pair, no FMM), which differ by the FMM's
  truncation only (p=4, MAC 0.7: energy 1.7e-4, dE/dq 1.7e-3 relative).
* On star2048, the library's gradients against central differences of the
  reference CLI's own energy (tests/golden/fd_star2048.json, written by
  make_golden.py --fd: direct energy, GMRES to 1e-14, raw energies at full
  precision).

The energy differentiated is the direct panel-charge sum E = e(q, r) . sigma
with (D - K) sigma = b(q, r) (fabipb_b200_forward / _backward).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, case_params, rel_l2
from fabipb_b200 import lib, meshio
import make_golden

pytestmark = pytest.mark.gpu
KCAL = 2 * np.pi * 332.0716
TIGHT = dict(restart=10, maxit=600, tol=1e-12)


@pytest.fixture(scope="module")
def star(tmp_path_factory):
    d = tmp_path_factory.mktemp("star204800")
    base = make_golden.generate_mesh("star204800", str(d))
    pan, ch = meshio.load_case(base)
    return pan, ch, make_golden.SOLVE_CASES["star204800"][2]


def _surface(pan, ch, opts, precision, direct=False):
    return lib.Surface(pan, lib.params(precision=precision, **case_params(opts)), ch, direct=direct)


def _shift(ch, k, dq=0.0, dx=None):
    q, pos = ch.q.copy(), ch.pos.copy()
    q[k] += dq
    if dx is not None:
        pos[k] += dx
    return meshio.ChargeSet(pos=pos, q=q, radius=ch.radius)


@pytest.fixture(scope="module")
def fp64_grad(star):
    pan, ch, opts = star
    s = _surface(pan, ch, opts, lib.FP64)
    s.precond_setup(2)
    e, it, res, info = s.forward(**TIGHT)
    assert info == 0
    dq, dx, it2, res2, info2 = s.backward(1.0, **TIGHT)
    assert info2 == 0
    return s, e, dq, dx


def test_fp64_gradients_match_finite_differences(star, fp64_grad):
    pan, ch, opts = star
    s, e0, dq, dx = fp64_grad
    ks = np.random.default_rng(31).choice(len(ch.q), size=64, replace=False)
    hq, hx = 1e-5, 1e-4

    def energy(c):
        s.set_charges(c)
        e, it, res, info = s.forward(**TIGHT)
        assert info == 0
        return e

    fdq, fdx = [], []
    for k in ks:
        fdq.append((energy(_shift(ch, k, dq=hq)) - energy(_shift(ch, k, dq=-hq))) / (2 * hq))
        row = []
        for a in range(3):
            step = np.zeros(3)
            step[a] = hx
            row.append((energy(_shift(ch, k, dx=step)) - energy(_shift(ch, k, dx=-step))) / (2 * hx))
        fdx.append(row)
    s.set_charges(ch)
    fdq, fdx = np.array(fdq), np.array(fdx)
    # E is quadratic in q: the charge differences are exact up to the solves' rounding
    assert rel_l2(dq[ks], fdq) < 1e-8
    # positions: O(h^2) truncation and solver noise / h
    assert rel_l2(dx[ks], fdx) < 1e-5
    assert np.max(np.abs(dx[ks] - fdx)) <= 1e-4 * np.max(np.abs(fdx))


def test_mixed_gradients_match_fp64(star, fp64_grad):
    pan, ch, opts = star
    _, e64, dq64, dx64 = fp64_grad
    s = _surface(pan, ch, opts, lib.MIXED)
    s.precond_setup(2)
    solver = dict(restart=10, maxit=400, tol=1e-6)
    e, it, res, info = s.forward(**solver)
    dq, dx, it2, res2, info2 = s.backward(1.0, **solver)
    assert info == 0 and info2 == 0
    assert abs(e - e64) <= 1e-5 * abs(e64)
    assert rel_l2(dq, dq64) < 1e-4
    assert rel_l2(dx, dx64) < 1e-3


def test_fmm_gradients_match_direct_oracle(star, fp64_grad):
    pan, ch, opts = star
    _, e64, dq64, dx64 = fp64_grad
    s = _surface(pan, ch, opts, lib.FP64, direct=True)
    s.precond_setup(2)
    solver = dict(restart=10, maxit=400, tol=1e-10)
    e, it, res, info = s.forward(**solver)
    dq, dx, it2, res2, info2 = s.backward(1.0, **solver)
    assert info == 0 and info2 == 0
    # the FMM (p=4, MAC 0.7) truncation: the energy to 1.7e-4 and dE/dq to
    # 1.7e-3 relative (measured on a B200); the forces, derivatives of the
    # same truncated field, to a few 1e-3 more
    assert abs(e64 - e) <= 1e-3 * abs(e)
    eq, ex = rel_l2(dq64, dq), rel_l2(dx64, dx)
    assert eq < 5e-3, eq
    assert ex < 5e-2, ex


def test_gradients_match_reference_finite_differences(case_dir, golden_meta):
    with open(os.path.join(GOLDEN, "fd_star2048.json")) as fp:
        fd = json.load(fp)
    name = fd["case"]
    opts = golden_meta[name]["opts"]
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    s = _surface(pan, ch, opts, lib.FP64)
    s.precond_setup(2)
    e, it, res, info = s.forward(**TIGHT)
    assert info == 0
    # both solves stop at a relative residual of 1e-12 (6e-9 apart in energy, measured)
    assert abs(e - fd["energy_raw"]) <= 1e-8 * abs(fd["energy_raw"])
    dq, dx, it2, res2, info2 = s.backward(1.0, **TIGHT)
    assert info2 == 0
    for k, rec in fd["charges"].items():
        k = int(k)
        # the reference's energies carry ~1e-9 of solver noise: over the steps
        # (1e-2 e, 1e-2 A) 5e-8 in the differences; positions also the O(h^2)
        # truncation (a few 1e-4 of the force)
        assert abs(dq[k] - rec["dq"]) <= 1e-5 * abs(rec["dq"]), (k, dq[k], rec["dq"])
        scale = max(abs(v) for v in rec["dx"])
        for a in range(3):
            assert abs(dx[k, a] - rec["dx"][a]) <= 1e-3 * scale + 2e-7, (k, a, dx[k, a], rec["dx"][a])
