"""The transposed operators (fabipb_b200_apply_adjoint / _matvec_adjoint)
through the C ABI.

* against the oracle: the dense near and far matrices of the FP64
  restatement, built column by column on the 320-panel sphere, transposed;
* on every golden case: the duality <u, K v> = <K^T u, v> with the forward
  operator of the same library, for the near field, the far field (both M2L
  kernels: orders 3-4 straight-line, order 5 list-driven) and the matvec.

Tolerances: FP64 relative 1e-12 (dense) and 1e-12 on the dualities; mixed
(FP32 near field) 5e-6.
"""
import os

import numpy as np
import pytest

from conftest import case_params, rel_l2
from fabipb_b200 import lib, meshio
import make_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CASES = list(make_golden.CASES)


def surface(case_dir, meta, name, precision):
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    prm = lib.params(precision=precision, **case_params(meta[name]["opts"]))
    return lib.Surface(pan, prm, ch), pan, ch


@pytest.fixture(scope="module")
def dense_sphere(case_dir, golden_meta):
    """Dense near and far matrices of the oracle on sphere320 (tree order)."""
    name = "sphere320"
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    orc = O.Oracle(pan, O.make_params(**case_params(golden_meta[name]["opts"])), ch)
    n2 = 2 * pan.n
    near = np.zeros((n2, n2))
    far = np.zeros((n2, n2))
    e = np.zeros(n2)
    for j in range(n2):
        e[:] = 0.0
        e[j] = 1.0
        near[:, j] = orc.near_apply(e)
        far[:, j] = orc.far_apply(e)
    return near, far, orc.area()


def test_adjoint_matches_oracle_dense_transpose(case_dir, golden_meta, dense_sphere):
    near, far = dense_sphere[:2]
    s, _, _ = surface(case_dir, golden_meta, "sphere320", lib.FP64)
    lam = make_golden.seeded_sigma(s.n, 5)
    assert rel_l2(s.apply_adjoint(lam, part=lib.NEAR), near.T @ lam) < 1e-12
    assert rel_l2(s.apply_adjoint(lam, part=lib.FAR), far.T @ lam) < 1e-12
    opts = golden_meta["sphere320"]["opts"]
    eps = opts.get("eps2", 80.0) / opts.get("eps1", 1.0)
    area = dense_sphere[2]
    d = np.concatenate([(1 + eps) / 2 * area, (1 + 1 / eps) / 2 * area])
    assert rel_l2(s.matvec_adjoint(lam), d * lam - (near + far).T @ lam) < 1e-12


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
@pytest.mark.parametrize("name", CASES)
def test_duality(name, precision, case_dir, golden_meta):
    s, _, _ = surface(case_dir, golden_meta, name, precision)
    tol = 1e-12 if precision == lib.FP64 else 5e-6
    rng = np.random.default_rng(11)
    for part in (lib.NEAR, lib.FAR, lib.ALL):
        u = rng.standard_normal(2 * s.n)
        v = rng.standard_normal(2 * s.n)
        kv = s.apply(v, part=part)
        ktu = s.apply_adjoint(u, part=part)
        lhs, rhs = u @ kv, ktu @ v
        scale = np.linalg.norm(u) * np.linalg.norm(kv)
        assert abs(lhs - rhs) <= tol * scale, (part, lhs, rhs)
    u = rng.standard_normal(2 * s.n)
    v = rng.standard_normal(2 * s.n)
    av = s.matvec(v)
    atu = s.matvec_adjoint(u)
    assert abs(u @ av - atu @ v) <= tol * np.linalg.norm(u) * np.linalg.norm(av)


# ---------------------------------------------------------------------------
# gradients: fabipb_b200_forward / _backward against central finite
# differences of the oracle's energy (reference restatement: direct RHS,
# block-LU GMRES, energy with every charge-tree cluster opened)
# ---------------------------------------------------------------------------
TIGHT = dict(restart=10, maxit=400, tol=1e-12)


def oracle_energy(pan, ch, opts):
    orc = O.Oracle(pan, O.make_params(energy_theta=0.0, **case_params(opts)), ch)
    b = orc.rhs_direct()
    orc.precond_setup(2)
    x, it, res, info = orc.gmres(b, b.copy(), TIGHT["restart"], TIGHT["maxit"], TIGHT["tol"])
    return orc.energy_raw(x)


def shifted(ch, k, dq=0.0, dx=None):
    q = ch.q.copy()
    pos = ch.pos.copy()
    q[k] += dq
    if dx is not None:
        pos[k] += dx
    return meshio.ChargeSet(pos=pos, q=q, radius=ch.radius)


@pytest.mark.parametrize("name", ["sphere320", "star2048"])
def test_forward_energy_matches_oracle(name, case_dir, golden_meta):
    opts = golden_meta[name]["opts"]
    s, pan, ch = surface(case_dir, golden_meta, name, lib.FP64)
    e, it, res, info = s.forward(**TIGHT)
    assert info == 0
    ref = oracle_energy(pan, ch, opts)
    assert abs(e - ref) <= 1e-9 * abs(ref)
    # the direct energy weights give the same energy through the tree entry point with theta 0
    orc = O.Oracle(pan, O.make_params(energy_theta=0.0, **case_params(opts)), ch)
    sig = make_golden.seeded_sigma(s.n, 2)
    assert abs(s.energy_weights() @ sig - orc.energy_raw(sig)) <= 1e-12 * abs(orc.energy_raw(sig))


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
def test_gradients_match_finite_differences(precision, case_dir, golden_meta):
    name = "sphere320"
    opts = golden_meta[name]["opts"]
    s, pan, ch = surface(case_dir, golden_meta, name, precision)
    # the FP32 near field puts a floor of ~1e-7 under the GMRES residual
    solver = TIGHT if precision == lib.FP64 else dict(restart=10, maxit=400, tol=1e-6)
    e, it, res, info = s.forward(**solver)
    assert info == 0
    dq, dx, it2, res2, info2 = s.backward(1.0, **solver)
    assert info2 == 0
    # FP64 at GMRES tol 1e-12: limited by the finite differences; mixed at
    # tol 1e-6: limited by the solver tolerance (~1e-4 relative)
    tol, tolx, floor = (1e-7, 1e-5, 1e-6) if precision == lib.FP64 else (1e-3, 1e-3, 1e-4)
    ks = np.random.default_rng(3).choice(len(ch.q), size=4, replace=False)
    hq, hx = 1e-5, 1e-4
    for k in ks:
        fd = (oracle_energy(pan, shifted(ch, k, dq=hq), opts) - oracle_energy(pan, shifted(ch, k, dq=-hq), opts)) / (2 * hq)
        assert abs(dq[k] - fd) <= tol * abs(fd) + 1e-9 * np.abs(dq).max(), (k, dq[k], fd)
        for a in range(3):
            step = np.zeros(3)
            step[a] = hx
            fd = (oracle_energy(pan, shifted(ch, k, dx=step), opts) -
                  oracle_energy(pan, shifted(ch, k, dx=-step), opts)) / (2 * hx)
            assert abs(dx[k, a] - fd) <= tolx * abs(fd) + floor * np.abs(dx).max(), (k, a, dx[k, a], fd)


def test_autograd_function(case_dir, golden_meta):
    import torch
    from fabipb_b200.autograd import SolvationEnergy, KCAL
    s, pan, ch = surface(case_dir, golden_meta, "sphere320", lib.FP64)
    q = torch.tensor(ch.q, requires_grad=True)
    pos = torch.tensor(ch.pos, requires_grad=True)
    E = SolvationEnergy.apply(q, pos, s, 10, 400, 1e-12)
    E.backward()
    dq, dx, _, _, _ = s.backward(1.0, **TIGHT)
    assert np.allclose(q.grad.numpy(), dq * KCAL, rtol=1e-10, atol=0)
    assert np.allclose(pos.grad.numpy(), dx * KCAL, rtol=1e-10, atol=1e-14)


def test_mixed_direct_sums_odd_counts(case_dir, golden_meta):
    """Odd panel and charge counts, a last charge tile of odd length: the
    packed FP32 kernels of a mixed context pad the last panel record pair and
    the last charge pair with zero weights.  Mixed direct RHS, energy weights
    and charge gradients against the FP64 context's, on the 320-panel sphere
    with its last panel removed (319 panels) and 1,101 seeded charges (one
    full tile of 1,024 and 77 more)."""
    name = "sphere320"
    pan, _ = meshio.load_case(os.path.join(case_dir, name))
    keep = pan.n - 1
    pan = meshio.PanelSet(vtx=pan.vtx[:keep], normal=pan.normal[:keep], area=pan.area[:keep],
                          face_index=pan.face_index[:keep])
    rng = np.random.default_rng(11)
    m = 1101
    d = rng.normal(size=(m, 3))
    pos = d / np.linalg.norm(d, axis=1)[:, None] * (15.0 * rng.random(m)[:, None] ** (1 / 3))
    ch = meshio.ChargeSet(pos=pos, q=rng.normal(0.0, 0.5, m), radius=np.full(m, 1.5))
    out = {}
    for prec, tol in ((lib.FP64, 1e-10), (lib.MIXED, 1e-6)):
        s = lib.Surface(pan, lib.params(precision=prec, **case_params(golden_meta[name]["opts"])), ch)
        rhs, ew = s.rhs(), s.energy_weights()
        e, it, res, info = s.forward(restart=10, maxit=400, tol=tol)
        assert info == 0
        dq, dx, it2, res2, info2 = s.backward(1.0, restart=10, maxit=400, tol=tol)
        assert info2 == 0
        out[prec] = (rhs, ew, dq, dx)
        s.close()
    a, b = out[lib.FP64], out[lib.MIXED]
    assert np.all(np.isfinite(np.concatenate([np.ravel(v) for v in b])))
    assert rel_l2(b[0], a[0]) < 2e-6   # FP32 pair terms, FP64 sums above 64 charges
    assert rel_l2(b[1], a[1]) < 2e-6
    assert rel_l2(b[2], a[2]) < 1e-3   # plus the mixed solves' tolerance
    assert rel_l2(b[3], a[3]) < 1e-3
