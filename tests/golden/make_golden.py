"""Generate the golden fixtures under tests/golden/ from the reference itself.

    python tests/golden/make_golden.py            # the small cases (cases.json, *.npz)
    python tests/golden/make_golden.py --large    # solve-only goldens (solve_cases.json)
    python tests/golden/make_golden.py --fd       # the reference's energy gradient by FD (fd_star2048.json)
    python tests/golden/make_golden.py --quad     # panel quadrature order -q=2 (quad_cases.json, *_q2.npz)

Needs the reference CPU solver compiled from its own sources
(``make -C oracle ref``, which reads the read-only reference mount).  For each
small seeded case it writes ``<case>.npz`` holding what the reference
computes on that mesh:

* tree layout: panel order (mesh-face index per tree slot), leaf start/count,
  near and M2L pair lists, FMM cube levels/centres/radii, panel areas;
* one near-field apply and one full matvec (MtVmain) of a seeded density;
* the direct and the charge-tree right-hand side (setupRHS);
* the panel-tree energy of the seeded density;
* the full CLI solve: solvation energy, GMRES iterations, final residual.

The meshes themselves are regenerated by ``fabipb_b200.meshgen`` from the
seeds recorded in ``cases.json``; a SHA-256 of the generated files is stored so
a test can tell a generator change from a solver change.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cuda-fabipb_b200"))
sys.path.insert(0, ROOT)

from fabipb_b200 import meshgen  # noqa: E402

# name -> (generator, generator kwargs, reference options)
CASES = {
    "sphere320": ("sphere", dict(nsub=2, radius=20.0, n_charges=50, seed=3),
                  dict(p=3, t=2, S=0.8, a=10, o=1e-4, eps1=1.0, eps2=80.0)),
    "sphere1280": ("sphere", dict(nsub=3, radius=20.0, n_charges=100, seed=4),
                   dict(p=3, t=3, S=0.8, a=10, o=1e-4, eps1=1.0, eps2=80.0)),
    "star2048": ("star", dict(freq=16, radius=25.0, n_charges=300, seed=5),
                 dict(p=4, t=3, S=0.7, a=10, o=1e-5, eps1=2.0, eps2=80.0)),
    "shell1152": ("shell", dict(freq=12, r_in=20.0, r_out=26.0, n_charges=200, seed=6),
                  dict(p=5, t=3, S=0.6, a=10, o=1e-6, eps1=2.0, eps2=80.0)),
}


# Larger seeded cases (the benchmark configurations' meshes, and the
# two-shell geometry at a coarse resolution) for which only the full CLI solve
# is recorded: solvation energy, GMRES iterations, final residual.  "P" selects
# the reference's preconditioner (-P=3 diagonal); without it the reference's
# auto policy picks block LU for eps1 <= 2 and eps2/eps1 >= 40.
SOLVE_CASES = {
    "sphere20480": ("sphere", dict(nsub=5, radius=20.0, n_charges=500, seed=0),
                    dict(p=3, t=3, S=0.8, a=10, o=1e-4, eps1=1.0, eps2=80.0)),
    "shell16384": ("shell", dict(freq=32, r_in=200.0, r_out=230.0, n_charges=5000, seed=2),
                   dict(p=5, t=4, S=0.6, a=10, o=1e-6, eps1=2.0, eps2=80.0, P=3)),
    "star204800": ("star", dict(freq=160, radius=25.0, n_charges=20000, seed=1),
                   dict(p=4, t=5, S=0.7, a=10, o=1e-5, eps1=2.0, eps2=80.0)),
}
# Golden cases also solved with the reference's dense direct operator (-r=2:
# every panel pair by panelIA0 on the CPU, no FMM), the counterpart of the
# library's dense context (-r=1 through the plugin ABI).
DIRECT_CASES = ("sphere320", "sphere1280", "star2048")


def generate_mesh(name, directory):
    kind, kw, _ = CASES[name] if name in CASES else SOLVE_CASES[name]
    base = os.path.join(directory, name)
    fn = {"sphere": meshgen.sphere_case, "star": meshgen.star_case, "shell": meshgen.shell_case}[kind]
    fn(base, **kw)
    return base


def mesh_digest(base):
    h = hashlib.sha256()
    for ext in (".vert", ".face", ".pqr"):
        with open(base + ext, "rb") as fp:
            h.update(fp.read())
    return h.hexdigest()


def ref_opts(opts, with_solver=False):
    out = ["-p=%d" % opts["p"], "-t=%d" % opts["t"], "-S=%g" % opts["S"], "-eps1=%g" % opts["eps1"],
           "-eps2=%g" % opts["eps2"]]
    if with_solver:
        out += ["-a=%d" % opts["a"], "-o=%g" % opts["o"]]
        if "P" in opts:
            out.append("-P=%d" % opts["P"])
    return out


def seeded_sigma(n, seed=0):
    return np.random.default_rng(seed).standard_normal(2 * n)


def main_large():
    """Solve-only goldens of SOLVE_CASES (minutes of reference CPU time) and the
    dense direct solves of DIRECT_CASES, into solve_cases.json."""
    from oracle import oracle as O
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    out = {}
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as tmp:
        for name, (_, _, opts) in SOLVE_CASES.items():
            base = generate_mesh(name, tmp)
            e, it, res, _ = O.run_ref_solve(base, ref_opts(opts, True), threads=threads)
            out[name] = {"opts": opts, "digest": mesh_digest(base),
                         "solve": {"energy": e, "iterations": it, "residual": res}}
            print(name, "energy", e, "its", it, "resid", res, flush=True)
        direct = {}
        for name in DIRECT_CASES:
            opts = CASES[name][2]
            base = generate_mesh(name, tmp)
            e, it, res, _ = O.run_ref_solve(base, ref_opts(opts, True) + ["-r=2"], threads=threads)
            direct[name] = {"energy": e, "iterations": it, "residual": res}
            print(name, "direct (-r=2) energy", e, "its", it, "resid", res, flush=True)
        out["direct"] = direct
    with open(os.path.join(HERE, "solve_cases.json"), "w") as fp:
        json.dump(out, fp, indent=1, sort_keys=True)


# Golden cases recomputed at panel quadrature order -q=2 (panelIA0 with q^4
# kernel evaluations for every disjoint near pair): one near-field apply and
# one matvec of the seeded density, the direct right-hand side and the
# panel-tree energy (q^2 points per panel), and the full CLI solve.
QUAD_CASES = ("sphere320", "star2048")
QUAD_ORDER = 2


def main_quad():
    from oracle import oracle as O
    meta = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name in QUAD_CASES:
            opts = CASES[name][2]
            base = generate_mesh(name, tmp)
            pre = os.path.join(tmp, name + "_out")
            o = ref_opts(opts) + ["-q=%d" % QUAD_ORDER]
            O.run_ref_harness("tree", base, pre, o)
            n = int(O.read_bin(pre, "hdr", np.int32)[0])
            sg = seeded_sigma(n)
            data = {}
            O.run_ref_harness("near", base, pre, o, sigma=sg)
            data["near"] = O.read_bin(pre, "pot", np.float64)
            O.run_ref_harness("matvec", base, pre, o, sigma=sg)
            data["matvec"] = O.read_bin(pre, "pot", np.float64)
            O.run_ref_harness("rhs", base, pre, o)
            data["rhs"] = O.read_bin(pre, "rhs", np.float64)
            O.run_ref_harness("energy", base, pre, o, sigma=sg)
            data["energy_raw"] = O.read_bin(pre, "energy", np.float64)
            e, it, res, _ = O.run_ref_solve(base, ref_opts(opts, True) + ["-q=%d" % QUAD_ORDER], threads=4)
            np.savez_compressed(os.path.join(HERE, "%s_q%d.npz" % (name, QUAD_ORDER)), **data)
            meta[name] = {"panels": n, "opts": dict(opts, q=QUAD_ORDER), "digest": mesh_digest(base),
                          "solve": {"energy": e, "iterations": it, "residual": res}}
            print(name, "q=%d" % QUAD_ORDER, n, "energy", e, "its", it, "resid", res, flush=True)
    with open(os.path.join(HERE, "quad_cases.json"), "w") as fp:
        json.dump(meta, fp, indent=1, sort_keys=True)


# Central finite differences of the reference CLI's own energy on star2048:
# every charge-tree cluster opened (FABIPB_ENERGY_TREE_THETA=1e-9, so the
# panel-tree energy is the direct panel-charge sum), GMRES to 1e-14, the
# charges written with ten decimals, the raw energy read at full precision
# from the CLI's energy-compare line (FABIPB_ENERGY_MODE=compare,
# src/fabipb.c:1172-1181).  The reference's energies carry ~1e-9 (raw) of
# solver noise from run to run, which steps of 1e-5 e and 1e-4 A turn into
# errors of 5e-5 and 5e-6 in the differences, so the steps are 1e-2 e for a
# charge (the energy is quadratic in the charges: the central difference is
# exact at any step) and 1e-2 A for a position (noise 5e-8, truncation a few
# 1e-4 of the force for a charge 1.4 A from the surface).  Values in raw energy
# units (kcal/mol over 2 pi 332.0716).
FD_CASE = "star2048"
FD_CHARGES = 4
FD_SEED = 21
FD_HQ, FD_HX = 1e-2, 1e-2


def write_pqr(path, ch):
    with open(path, "w") as fp:
        for i, (p, c, r) in enumerate(zip(ch.pos, ch.q, ch.radius)):
            fp.write("ATOM %d C ALA A 1 %.10f %.10f %.10f %.10f %.4f\n" % (i + 1, p[0], p[1], p[2], c, r))


def fd_charges(n_charges):
    return sorted(int(k) for k in np.random.default_rng(FD_SEED).choice(n_charges, size=FD_CHARGES, replace=False))


def main_fd():
    """fd_star2048.json: the reference's central differences of its energy."""
    from fabipb_b200 import meshio
    from oracle import oracle as O
    opts = dict(CASES[FD_CASE][2], o=1e-14)
    env = {"FABIPB_ENERGY_TREE_THETA": "1e-9", "FABIPB_ENERGY_MODE": "compare"}
    out = {"case": FD_CASE, "hq": FD_HQ, "hx": FD_HX, "units": "raw energy", "charges": {}}
    with tempfile.TemporaryDirectory() as tmp:
        base = generate_mesh(FD_CASE, tmp)
        pan, ch = meshio.load_case(base)
        write_pqr(base + ".pqr", ch)   # ten decimals: the perturbed files below differ only in one value

        def energy(c):
            write_pqr(base + ".pqr", c)
            _, it, res, out = O.run_ref_solve(base, ref_opts(opts, True) + ["-i=1000"], threads=os.cpu_count(),
                                              extra_env=env)
            assert res <= opts["o"], (it, res)   # converged: the differences see no solver noise above 1e-14
            line = [l for l in out.splitlines() if l.startswith("Energy compare:")][0]
            return float(line.split("panel-tree raw=")[1].split()[0])

        out["energy_raw"] = energy(ch)
        for k in fd_charges(len(ch.q)):
            rec = {}
            q = ch.q.copy()
            q[k] += FD_HQ
            ep = energy(meshio.ChargeSet(ch.pos, q, ch.radius))
            q[k] -= 2 * FD_HQ
            em = energy(meshio.ChargeSet(ch.pos, q, ch.radius))
            rec["dq"] = (ep - em) / (2 * FD_HQ)
            rec["dx"] = []
            for a in range(3):
                pos = ch.pos.copy()
                pos[k, a] += FD_HX
                ep = energy(meshio.ChargeSet(pos, ch.q, ch.radius))
                pos[k, a] -= 2 * FD_HX
                em = energy(meshio.ChargeSet(pos, ch.q, ch.radius))
                rec["dx"].append((ep - em) / (2 * FD_HX))
            out["charges"][str(k)] = rec
            print(k, rec, flush=True)
    with open(os.path.join(HERE, "fd_star2048.json"), "w") as fp:
        json.dump(out, fp, indent=1, sort_keys=True)


def main():
    from oracle import oracle as O
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    if "--large" in sys.argv:
        return main_large()
    if "--fd" in sys.argv:
        return main_fd()
    if "--quad" in sys.argv:
        return main_quad()
    meta = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (_, _, opts) in CASES.items():
            base = generate_mesh(name, tmp)
            pre = os.path.join(tmp, name + "_out")
            o = ref_opts(opts)
            O.run_ref_harness("tree", base, pre, o)
            hdr = O.read_bin(pre, "hdr", np.int32)
            n = int(hdr[0])
            data = {"hdr": hdr}
            for key, dt in (("order", np.int32), ("leafStart", np.int32), ("leafCount", np.int32),
                            ("nearSrc", np.int32), ("nearDst", np.int32), ("m2lSrc", np.int32),
                            ("m2lDst", np.int32), ("cubeLevel", np.int32), ("cubeCtr", np.float64),
                            ("area", np.float64)):
                data[key] = O.read_bin(pre, key, dt)
            sg = seeded_sigma(n)
            O.run_ref_harness("near", base, pre, o, sigma=sg)
            data["near"] = O.read_bin(pre, "pot", np.float64)
            O.run_ref_harness("matvec", base, pre, o, sigma=sg)
            data["matvec"] = O.read_bin(pre, "pot", np.float64)
            O.run_ref_harness("rhs", base, pre, o)
            data["rhs"] = O.read_bin(pre, "rhs", np.float64)
            O.run_ref_harness("rhs", base, pre, o, extra_env={"FABIPB_FORCE_TREE_RHS": "1"})
            data["rhs_tree"] = O.read_bin(pre, "rhs", np.float64)
            O.run_ref_harness("energy", base, pre, o, sigma=sg)
            data["energy_raw"] = O.read_bin(pre, "energy", np.float64)
            e, it, res, _ = O.run_ref_solve(base, ref_opts(opts, True), threads=4)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
            meta[name] = {"panels": n, "opts": opts, "digest": mesh_digest(base),
                          "solve": {"energy": e, "iterations": it, "residual": res}}
            print(name, n, "energy", e, "its", it, "resid", res)
    with open(os.path.join(HERE, "cases.json"), "w") as fp:
        json.dump(meta, fp, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
