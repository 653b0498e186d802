"""GPU parity: the CUDA library against the FP64 restatement oracle and the
reference goldens, through the C ABI (include/fabipb_b200.h).

Tolerances:
  * tree layouts: identical integers and bit-identical box centres;
  * FP64 mode operators: relative L2 <= 1e-12 against the oracle;
  * mixed (FP32 near-field P2P) mode: relative L2 <= 5e-6 for the near field
    and the matvec, <= 1e-6 for the direct RHS (FP32 pair terms), 1e-5 for the
    energy walk (FP32 cluster and direct terms).
"""
import os

import numpy as np
import pytest

from conftest import case_params, load_golden, rel_l2
from fabipb_b200 import lib, meshio
import make_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CASES = list(make_golden.CASES)


def surface(case_dir, meta, name, precision):
    pan, ch = meshio.load_case(os.path.join(case_dir, name))
    prm = lib.params(precision=precision, **case_params(meta[name]["opts"]))
    return lib.Surface(pan, prm), pan, ch


@pytest.fixture(scope="module")
def oracles(case_dir, golden_meta):
    out = {}
    for name in CASES:
        pan, ch = meshio.load_case(os.path.join(case_dir, name))
        out[name] = O.Oracle(pan, O.make_params(**case_params(golden_meta[name]["opts"])), ch)
    return out


@pytest.mark.parametrize("name", CASES)
def test_tree_matches_reference(name, case_dir, golden_meta):
    g = load_golden(name)
    s, pan, _ = surface(case_dir, golden_meta, name, lib.FP64)
    info = s.info()
    assert (info["panels"], info["leaves"], info["near_pairs"], info["m2l_pairs"], info["cubes"]) == \
        tuple(int(v) for v in g["hdr"][:5])
    assert np.array_equal(pan.face_index[s.panel_order()], g["order"])
    st, ct = s.leaf_layout()
    assert np.array_equal(st, g["leafStart"]) and np.array_equal(ct, g["leafCount"])
    ns, nd = s.near_pairs()
    assert np.array_equal(ns, g["nearSrc"]) and np.array_equal(nd, g["nearDst"])
    ms, md = s.m2l_pairs()
    assert np.array_equal(ms, g["m2lSrc"]) and np.array_equal(md, g["m2lDst"])
    lev, ctr = s.cube_data()
    assert np.array_equal(lev, g["cubeLevel"]) and np.array_equal(ctr.reshape(-1), g["cubeCtr"])


def _tree_arrays(s):
    lev, ctr = s.cube_data()
    return [s.panel_order(), *s.leaf_layout(), *s.near_pairs(), *s.m2l_pairs(), lev, ctr]


@pytest.mark.parametrize("name", CASES + ["star204800", "shell16384"])
def test_device_tree_matches_host_tree(name, case_dir, golden_meta, tmp_path, monkeypatch):
    """The octree built on the device (cell keys, stable radix sort, key-prefix
    cubes, boxes, MAC lists) equals the host build bit for bit: panel order,
    leaves, near and M2L lists, box centres and radii -- on the golden cases
    and on two larger meshes (the 204,800-panel star, the 16,384-panel
    two-shell surface)."""
    if name in golden_meta:
        base, opts = os.path.join(case_dir, name), golden_meta[name]["opts"]
    else:
        base, opts = make_golden.generate_mesh(name, str(tmp_path)), make_golden.SOLVE_CASES[name][2]
    pan, _ = meshio.load_case(base)
    prm = lib.params(precision=lib.FP64, **case_params(opts))
    dev = _tree_arrays(lib.Surface(pan, prm))
    monkeypatch.setenv("FABIPB_B200_HOST_TREE", "1")
    host = _tree_arrays(lib.Surface(pan, prm))
    for a, b in zip(dev, host):
        assert a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision,tol", [(lib.FP64, 1e-12), (lib.MIXED, 5e-6)])
def test_near_field(name, precision, tol, case_dir, golden_meta):
    g = load_golden(name)
    s, _, _ = surface(case_dir, golden_meta, name, precision)
    sg = make_golden.seeded_sigma(s.n)
    got = s.apply(sg, part=lib.NEAR)
    assert rel_l2(got, g["near"]) < tol


@pytest.mark.parametrize("name", CASES)
def test_far_field_fp64(name, case_dir, golden_meta, oracles):
    s, _, _ = surface(case_dir, golden_meta, name, lib.FP64)
    sg = make_golden.seeded_sigma(s.n, 3)
    got = s.apply(sg, part=lib.FAR, alpha=0.5)
    ref = oracles[name].far_apply(sg, 0.5, 0.0)
    assert rel_l2(got, ref) < 1e-12


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision,tol", [(lib.FP64, 1e-12), (lib.MIXED, 5e-6)])
def test_matvec(name, precision, tol, case_dir, golden_meta):
    g = load_golden(name)
    s, _, _ = surface(case_dir, golden_meta, name, precision)
    sg = make_golden.seeded_sigma(s.n)
    got = s.matvec(sg)
    assert rel_l2(got, g["matvec"]) < tol


@pytest.mark.parametrize("name,depth,height", [("sphere1280", 1, 1), ("star2048", 2, 2), ("shell1152", 2, 2),
                                               ("star2048", 3, 2), ("sphere1280", 3, 2)])
def test_symmetric_near_field(name, depth, height, case_dir, golden_meta, monkeypatch):
    """The symmetric near field (each unordered pair of distinct near leaves
    evaluated once for both directions, sums through the scratch), FP32 packed
    (32-wide tiles, and half-warp tiles for leaves under 48 panels) and FP64,
    forward and transposed: shallow trees, so that the leaves are large enough
    for it, and depth 3, where many are small; against the ordered kernels alone
    (FABIPB_B200_NEAR_SYM=0): FP64 to 1e-13 (only the summation order
    differs), FP32 to 2e-6 of the ordered FP32 and 5e-6 of the FP64 near
    field, matvec and transposed near field; the duality of the symmetric
    FP64 near field."""
    opts = dict(golden_meta[name]["opts"], t=depth)
    pan, _ = meshio.load_case(os.path.join(case_dir, name))
    sg = make_golden.seeded_sigma(pan.n, 6)
    lam = make_golden.seeded_sigma(pan.n, 7)
    out = {}
    for sym in (True, False):
        monkeypatch.setenv("FABIPB_B200_NEAR_SYM", "1" if sym else "0")
        for prec in (lib.FP64, lib.MIXED):
            s = lib.Surface(pan, lib.params(precision=prec, height=height, **case_params(opts)))
            n0 = s.launch_count()
            near = s.apply(sg, part=lib.NEAR)
            out[sym, prec] = (near, s.launch_count() - n0, s.matvec(sg), s.apply_adjoint(lam, part=lib.NEAR))
    # the symmetric pack and kernel ran (mixed: the 32-wide and, with leaf pairs under 48 panels, the
    # half-warp kernel; FP64 keeps the pairs with a leaf under 48 panels in the ordered kernel)
    assert out[True, lib.FP64][1] - out[False, lib.FP64][1] in ((0, 2) if depth == 3 else (2,))
    assert out[True, lib.MIXED][1] - out[False, lib.MIXED][1] in (2, 3)
    ref_near, ref_mv, ref_adj = out[False, lib.FP64][0], out[False, lib.FP64][2], out[False, lib.FP64][3]
    assert rel_l2(out[True, lib.FP64][0], ref_near) < 1e-13
    assert rel_l2(out[True, lib.FP64][2], ref_mv) < 1e-13
    assert rel_l2(out[True, lib.FP64][3], ref_adj) < 1e-13      # the transposed operator
    assert rel_l2(out[True, lib.MIXED][0], ref_near) < 5e-6
    assert rel_l2(out[True, lib.MIXED][2], ref_mv) < 5e-6
    assert rel_l2(out[True, lib.MIXED][3], ref_adj) < 5e-6
    assert rel_l2(out[True, lib.MIXED][0], out[False, lib.MIXED][0]) < 2e-6
    # duality of the symmetric near field: <lam, K sg> = <K^T lam, sg>
    lhs, rhs = float(lam @ out[True, lib.FP64][0]), float(out[True, lib.FP64][3] @ sg)
    assert abs(lhs - rhs) <= 1e-12 * np.linalg.norm(lam) * np.linalg.norm(out[True, lib.FP64][0])


@pytest.mark.parametrize("name,order,depth", [("sphere1280", 3, 3), ("star2048", 4, 3), ("shell1152", 5, 3),
                                               ("star2048", 5, 4), ("sphere1280", 4, 4)])
def test_m2l_bulk_staging(name, order, depth, case_dir, golden_meta, monkeypatch):
    """The M2L of mixed contexts with its moments staged by bulk copies into
    shared memory (the default) against the plain-load staging
    (FABIPB_B200_M2L_BULK=0): the same FP32 tensors, moments and conv order, so
    the far fields agree to 1e-6 relative (FP32 rounding: the compiler pairs and
    contracts the FP32 operations of the two kernels differently), forward and
    transposed; both within
    2e-5 of the FP64 far field (FP32 tensors, moments and leaf matrices); the bulk path launches one kernel more (the FP32
    row pack).  The depth-4 trees give destinations with more than 64 pairs, so
    the copies of the next batch are in flight while a batch is summed."""
    opts = dict(golden_meta[name]["opts"], p=order, t=depth)
    pan, _ = meshio.load_case(os.path.join(case_dir, name))
    sg = make_golden.seeded_sigma(pan.n, 8)
    lam = make_golden.seeded_sigma(pan.n, 9)
    out = {}
    for mode, prec, env in (("bulk", lib.MIXED, "1"), ("plain", lib.MIXED, "0"), ("fp64", lib.FP64, "1")):
        monkeypatch.setenv("FABIPB_B200_M2L_BULK", env)
        s = lib.Surface(pan, lib.params(precision=prec, **case_params(opts)))
        n0 = s.launch_count()
        far = s.apply(sg, part=lib.FAR)
        out[mode] = (far, s.launch_count() - n0, s.apply_adjoint(lam, part=lib.FAR))
        if mode == "bulk":
            _, dst = s.m2l_pairs()
            most = int(np.bincount(dst).max()) if dst.size else 0
    if depth == 4:
        assert most > 64
    assert out["bulk"][1] == out["plain"][1] + 1
    assert rel_l2(out["bulk"][0], out["plain"][0]) < 1e-6
    assert rel_l2(out["bulk"][2], out["plain"][2]) < 1e-6
    assert rel_l2(out["bulk"][0], out["fp64"][0]) < 2e-5
    assert rel_l2(out["bulk"][2], out["fp64"][2]) < 2e-5


def test_apply_alpha_beta_semantics(case_dir, golden_meta, oracles):
    name = "star2048"
    s, _, _ = surface(case_dir, golden_meta, name, lib.FP64)
    rng = np.random.default_rng(5)
    sg, y0 = rng.standard_normal(2 * s.n), rng.standard_normal(2 * s.n)
    got = s.matvec(sg, alpha=-1.0, beta=1.0, y=y0)
    ref = oracles[name].matvec(sg, -1.0, 1.0, y0)
    assert rel_l2(got, ref) < 1e-12
    got = s.apply(sg, part=lib.ALL, alpha=0.3, beta=-2.0, pot=y0)
    ref = oracles[name].fmm_apply(sg, 0.3, -2.0, y0)
    assert rel_l2(got, ref) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_special_pairs_device_matches_host(name, case_dir, golden_meta, monkeypatch):
    """The device special-pair search (sorted corner hashes) builds the same
    CSR table as the host search (hash map of exact coordinates): same count,
    and the FP64 near field is bit-identical."""
    sg = make_golden.seeded_sigma(surface(case_dir, golden_meta, name, lib.FP64)[0].n, 3)
    s_dev, _, _ = surface(case_dir, golden_meta, name, lib.FP64)
    monkeypatch.setenv("FABIPB_B200_HOST_SPECIAL", "1")
    s_host, _, _ = surface(case_dir, golden_meta, name, lib.FP64)
    assert s_dev.info()["special_pairs"] == s_host.info()["special_pairs"] > 0
    assert np.array_equal(s_dev.apply(sg, part=lib.NEAR), s_host.apply(sg, part=lib.NEAR))


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
@pytest.mark.parametrize("name", CASES)
def test_rhs_direct(name, precision, case_dir, golden_meta):
    """FP64 contexts sum in FP64 (1e-13); mixed contexts in FP32 pair terms
    with FP64 tile sums (1e-6)."""
    g = load_golden(name)
    s, _, ch = surface(case_dir, golden_meta, name, precision)
    s.set_charges(ch)
    tol = 1e-13 if precision == lib.FP64 else 1e-6
    assert rel_l2(s.rhs(use_tree=False), g["rhs"]) < tol


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
@pytest.mark.parametrize("name", CASES)
def test_rhs_tree(name, precision, case_dir, golden_meta):
    """The charge-tree RHS walk: FP64 contexts in FP64 (1e-12); mixed contexts
    with FP32 cluster and direct terms, FP64 sums (1e-6)."""
    g = load_golden(name)
    s, _, ch = surface(case_dir, golden_meta, name, precision)
    s.set_charges(ch)
    tol = 1e-12 if precision == lib.FP64 else 1e-6
    assert rel_l2(s.rhs(use_tree=True), g["rhs_tree"]) < tol


@pytest.mark.parametrize("precision", [lib.FP64, lib.MIXED])
@pytest.mark.parametrize("name", CASES)
def test_energy(name, precision, case_dir, golden_meta):
    """The charge-tree energy walk: FP64 contexts walk in FP64 (1e-12); mixed
    contexts evaluate the clusters and direct terms in FP32 with FP64 sums
    (1e-5)."""
    g = load_golden(name)
    s, _, ch = surface(case_dir, golden_meta, name, precision)
    s.set_charges(ch)
    e = s.energy_raw(make_golden.seeded_sigma(s.n))
    ref = float(g["energy_raw"][0])
    tol = 1e-12 if precision == lib.FP64 else 1e-5
    assert abs(e - ref) <= tol * abs(ref)


@pytest.mark.parametrize("name", CASES)
def test_solve_fp64_matches_reference(name, case_dir, golden_meta):
    """Device GMRES + block-LU preconditioner with the FP64 operator: same
    iteration count as the reference CLI, energy equal to its %f print."""
    meta = golden_meta[name]
    s, _, ch = surface(case_dir, golden_meta, name, lib.FP64)
    s.set_charges(ch)
    b = s.rhs(use_tree=False)
    s.precond_setup(2)
    x, it, res, info = s.solve(b, b.copy(), restart=meta["opts"]["a"], maxit=100, tol=meta["opts"]["o"])
    e = s.energy_raw(x) * 2 * np.pi * 332.0716
    assert info == 0
    assert it == meta["solve"]["iterations"]
    assert abs(res - meta["solve"]["residual"]) <= 1e-3 * meta["solve"]["residual"]
    assert abs(e - meta["solve"]["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.parametrize("name", CASES)
def test_solve_mixed_energy(name, case_dir, golden_meta):
    """FP32 near-field operator inside GMRES: energy within 1e-4 relative of
    the reference, iteration count within one."""
    meta = golden_meta[name]
    s, _, ch = surface(case_dir, golden_meta, name, lib.MIXED)
    s.set_charges(ch)
    b = s.rhs(use_tree=False)
    s.precond_setup(2)
    x, it, res, info = s.solve(b, b.copy(), restart=meta["opts"]["a"], maxit=100, tol=meta["opts"]["o"])
    e = s.energy_raw(x) * 2 * np.pi * 332.0716
    assert info == 0
    assert abs(it - meta["solve"]["iterations"]) <= 1
    assert abs(e - meta["solve"]["energy"]) <= 1e-4 * abs(meta["solve"]["energy"])


@pytest.mark.parametrize("name", ["star2048", "shell1152"])
@pytest.mark.parametrize("mode", [2, 3])
@pytest.mark.parametrize("precision,tol", [(lib.FP64, 1e-11), (lib.MIXED, 1e-4)])
def test_precond_apply_matches_oracle(name, mode, precision, tol, case_dir, golden_meta, oracles):
    """Block-LU (mode 2) and diagonal (mode 3) preconditioners against the
    FP64 oracle: FP64 contexts to 1e-11; mixed contexts, whose block inverses
    are computed and stored in FP32 (applied with FP64 sums), to 1e-4 (the
    diagonal is FP64 in both)."""
    s, _, _ = surface(case_dir, golden_meta, name, precision)
    s.precond_setup(mode)
    orc = oracles[name]
    orc.precond_setup(mode)
    b = make_golden.seeded_sigma(s.n, 9)
    got, ref = s.precond_apply(b), orc.precond_apply(b)
    assert rel_l2(got, ref) < (1e-13 if mode == 3 else tol)
