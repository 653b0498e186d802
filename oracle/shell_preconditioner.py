"""TEST INFRASTRUCTURE ONLY: the reference CPU solver's GMRES on the two-shell
geometry with its block-LU and its diagonal preconditioner.

    python oracle/shell_preconditioner.py [--maxit 60]

Generates the seeded two-shell surface of the capsid-scale configuration
(radii 200/230 A, inward inner normals, l <= 12 harmonics of 2%) at a coarse
16,384-panel resolution with 5,000 charges, and runs the reference CLI
(oracle/_ref/fabipb_ref, -g=0, compiled from the reference's own sources)
with p=5, MAC 0.6, depth 4, restart 10, tol 1e-6, eps 2/80:

* -P=2, the block-LU preconditioner the reference's auto policy picks for
  eps1 <= 2 and eps2/eps1 >= 40 (src/fabipb_options.c:85-88, 231-237);
* -P=2 from a zero initial guess (FABIPB_GMRES_INITIAL=zero);
* -P=3, the diagonal preconditioner.

and prints the residual history of each (FABIPB_GMRES_LOG_RESID=1,
src/gmres.c:296-299).  Measured here: -P=2 stagnates near 2.9 from x0 = b and
near 1.7e-3 from x0 = 0, -P=3 converges in 29 iterations.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this directory comes first on the path and would shadow the package
sys.path = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
sys.path.insert(0, os.path.join(ROOT, "cuda-fabipb_b200"))
sys.path.insert(0, ROOT)


def main():
    from fabipb_b200 import meshgen
    from oracle import oracle as O
    ap = argparse.ArgumentParser()
    ap.add_argument("--maxit", type=int, default=60)
    args = ap.parse_args()
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    opts = ["-p=5", "-t=4", "-S=0.6", "-a=10", "-o=1e-6", "-eps1=2", "-eps2=80", "-i=%d" % args.maxit]
    with tempfile.TemporaryDirectory() as tmp:
        base = os.path.join(tmp, "shell16384")
        meshgen.shell_case(base, freq=32, r_in=200.0, r_out=230.0, n_charges=5000, seed=2)
        for label, extra, env_extra in (("-P=2 (block LU), x0 = b", ["-P=2"], {}),
                                        ("-P=2 (block LU), x0 = 0", ["-P=2"], {"FABIPB_GMRES_INITIAL": "zero"}),
                                        ("-P=3 (diagonal), x0 = b", ["-P=3"], {})):
            env = O.ref_env(os.cpu_count() or 1)
            env["FABIPB_GMRES_LOG_RESID"] = "1"
            env.update(env_extra)
            r = subprocess.run([O.REF_BINARY, "-g=0", "-m=1"] + opts + extra + [base], env=env,
                               capture_output=True, text=True, check=True)
            hist = [l.split("resid=")[1] for l in r.stdout.splitlines() if l.startswith("GMRES residual:")]
            status = [l for l in r.stdout.splitlines() if l.startswith("GMRES status:")]
            print(label)
            print("  residuals:", " ".join(hist))
            print(" ", status[0] if status else "no status line")


if __name__ == "__main__":
    main()
