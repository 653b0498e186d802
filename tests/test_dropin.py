"""Drop-in check: the reference host, compiled from its own sources, linked
against libfabipb_b200.so in place of its CUDA backend (oracle/_ref/
fabipb_dropin), run through its own CLI with -g=1 exactly as a user would,
compared with the reference's CPU path (-g=0) goldens.

FABIPB_GPU_PRECOND_BUILD_DISJOINT=0 keeps the block preconditioner on the
host as with -g=0 (the reference's GPU block builder evaluates the transposed
disjoint pair, src/gpu/gpu_preconditioner_cuda.inc:240-325, so -g=1 and -g=0
runs of the reference itself use slightly different preconditioners)."""
import os
import subprocess

import pytest

from conftest import ROOT
import make_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DROPIN = os.path.join(ROOT, "oracle", "_ref", "fabipb_dropin")


def run_dropin(base, opts, extra=None, env_extra=None):
    env = O.ref_env(threads=4)
    env["FABIPB_GPU_PRECOND_BUILD_DISJOINT"] = "0"
    if env_extra:
        env.update(env_extra)
    cmd = [DROPIN, "-g=1", "-m=1", "-B=1"] + make_golden.ref_opts(opts, True) + (extra or []) + [base]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def parse(out):
    e = it = None
    for line in out.splitlines():
        if line.startswith("solvation energy:"):
            e = float(line.split(":")[1])
        elif line.startswith("GMRES status:"):
            it = int(dict(p.split("=") for p in line.split(":")[1].split())["iterations"])
    return e, it


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in binary not built (make -C oracle dropin)")
@pytest.mark.parametrize("name", list(make_golden.CASES))
def test_dropin_solve_matches_cpu_reference(name, case_dir, golden_meta):
    meta = golden_meta[name]
    out = run_dropin(os.path.join(case_dir, name), meta["opts"])
    assert "GPU mode=1" in out
    assert "CPU fallback" not in out and "unavailable" not in out, out
    e, it = parse(out)
    assert it == meta["solve"]["iterations"]
    assert abs(e - meta["solve"]["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in binary not built (make -C oracle dropin)")
def test_dropin_debug_compare(case_dir, golden_meta):
    """-c=1: the reference compares one CPU applyFMM with the GPU one."""
    name = "star2048"
    out = run_dropin(os.path.join(case_dir, name), golden_meta[name]["opts"], extra=["-c=1"])
    line = [l for l in out.splitlines() if l.startswith("applyFMM debug compare")][0]
    rel = float(line.split("rel_l2=")[1].split()[0])
    assert rel < 1e-12, line


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in binary not built (make -C oracle dropin)")
@pytest.mark.parametrize("name", list(make_golden.DIRECT_CASES))
def test_dropin_direct_mode_matches_reference_direct(name, case_dir, golden_meta, solve_meta):
    """-r=1 (the dense direct matvec through gpuDirectApply) against the
    reference's own CPU direct mode -r=2 (cpuDirectApply,
    src/direct_backend.c:172) on the same mesh: the same GMRES iteration count
    and the printed energy to its last digit."""
    meta = golden_meta[name]
    ref = solve_meta["direct"][name]
    out = run_dropin(os.path.join(case_dir, name), meta["opts"], extra=["-r=1"])
    assert "unavailable" not in out and "CPU fallback" not in out, out
    e, it = parse(out)
    assert it == ref["iterations"]
    assert abs(e - ref["energy"]) <= 2e-6 + 1e-8 * abs(e)


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in binary not built (make -C oracle dropin)")
def test_dropin_direct_mode_with_gpu_precond(case_dir, golden_meta, solve_meta):
    """-r=1 with the reference's GPU preconditioner block builder
    (gpuBuildPrecondDisjointBlock, which evaluates the transposed disjoint
    pairs, so the preconditioner differs slightly from the host's): no CPU
    fallback, and the energy of the direct solve within the solver tolerance
    of the reference's -r=2 energy."""
    name = "sphere320"
    meta = golden_meta[name]
    out = run_dropin(os.path.join(case_dir, name), meta["opts"], extra=["-r=1"],
                     env_extra={"FABIPB_GPU_PRECOND_BUILD_DISJOINT": "1"})
    assert "unavailable" not in out and "CPU fallback" not in out, out
    e, it = parse(out)
    ref = solve_meta["direct"][name]["energy"]
    assert e is not None and abs(e - ref) <= 1e-4 * abs(ref)
