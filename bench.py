"""Benchmark of the FABIPB GMRES matvec and solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--case shell2097152|star204800|...]

Default workload, the capsid-scale two-shell configuration: a spherical shell
of inner radius 200 A and outer radius 230 A as two closed octahedral
geodesic spheres of frequency 362 (2,096,704 flat triangles; inner normals
into the cavity), both perturbed by seeded l <= 12 harmonics of amplitude 2%,
500,000 charges uniform in the shell at least 1.4 A from both surfaces
(q ~ N(0, 0.4^2) e, net 0), eps 2/80, kappa 0.1257, Taylor order p=5, MAC
0.6, octree depth 5 (mean leaf 254 panels, the depth nearest a 200-panel
leaf), GMRES restart 10, tol 1e-6, diagonal preconditioner (the reference's
-P=3: its block-LU policy stagnates on the two-shell surface, see the
design notes).  One "step" = one operator application y = (D - K)x, the GMRES
matvec of src/fabipb.c:1237.  Inputs are synthetic and seeded.
--case star204800 runs the 204,800-panel star surface (p=4, MAC 0.7, depth 5,
20,000 charges), where the FP64 direct-summation oracle (every panel pair,
no FMM) is also solved; sphere20480 the 20,480-panel Kirkwood sphere.

Reported:
  value      matvec/s of the FP32-mixed operator with x, y resident in HBM
             (CUDA events on the library's stream), L2 flushed between steps
             outside the timed intervals;
  e2e        matvec/s through the C ABI with host buffers (H2D of x and D2H
             of y inside the timed region, pinned host memory); e2e_dropin
             the same through the reference host's MtVmain on this library's
             plugin ABI (src/gpu_backend.h), host wall time;
  roofline   the near-field P2P kernel (the dominant kernel): algorithmic
             FLOPs (60 per panel pair) per launch / its event-timed duration,
             against the FP32 FMA rate measured on this GPU;
  fp64       matvec/s of the FP64 operator (the plain FP64 GPU path);
  solve      GMRES, refined and FP64 solves (every run), energies and their
             errors, the adjoint's backward/forward cost;
  cpu_baseline  the reference CPU solver compiled from its own sources
             (oracle/_ref), on this host's cores: whole matvecs, or on the
             large meshes the FMM passes whole plus the near field on a leaf
             sample scaled by panel pairs;
  ref_gpu_baseline  the reference's own CUDA backend compiled from its
             sources for sm_100a (oracle/_ref/ref_harness_gpu), -g=1 on this
             GPU.
With --impl reference the line times that reference CPU matvec itself.
N>1 GPUs run independent replicas (the path does not shard: replicas only);
value is the sum over replicas, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-fabipb_b200"))
sys.path.insert(0, ROOT)

CASES = {
    # name: (generator, kwargs, solver options); precond 2 = block LU, 3 = diagonal (the reference's -P)
    # the capsid-scale two-shell surface: 2,096,704 triangles, 500,000 charges
    "shell2097152": ("shell", dict(freq=362, r_in=200.0, r_out=230.0, n_charges=500000, seed=2),
                     dict(order=5, depth=5, sep_ratio=0.6, eps1=2.0, eps2=80.0, tol=1e-6, restart=10, maxit=100,
                          precond=3)),
    "star204800": ("star", dict(freq=160, radius=25.0, n_charges=20000, seed=1),
                   dict(order=4, depth=5, sep_ratio=0.7, eps1=2.0, eps2=80.0, tol=1e-5, restart=10, maxit=100,
                        precond=2)),
    # a 2.1M-panel star (octahedral freq 512, radius 50 A), 100,000 charges
    "star2097152": ("star", dict(freq=512, radius=50.0, n_charges=100000, seed=7),
                    dict(order=4, depth=7, sep_ratio=0.7, eps1=2.0, eps2=80.0, tol=1e-6, restart=10, maxit=100,
                         precond=2)),
    # the scale-stress shell: radii 400/440 A, 8,386,816 triangles, 2,000,000 charges
    "shell8388608": ("shell", dict(freq=724, r_in=400.0, r_out=440.0, n_charges=2000000, seed=4),
                     dict(order=5, depth=6, sep_ratio=0.6, eps1=2.0, eps2=80.0, tol=1e-6, restart=10, maxit=100,
                          precond=3)),
    # the two-shell configuration's leaf structure at a quarter of its size (radii 100/115 A,
    # 524,176 triangles, depth 4: mean leaf 300, max 1219), for kernel profiles
    "shell524176": ("shell", dict(freq=181, r_in=100.0, r_out=115.0, n_charges=125000, seed=13),
                    dict(order=5, depth=4, sep_ratio=0.6, eps1=2.0, eps2=80.0, tol=1e-6, restart=10, maxit=100,
                         precond=3)),
    "sphere20480": ("sphere", dict(nsub=5, radius=20.0, n_charges=500, seed=0),
                    dict(order=3, depth=3, sep_ratio=0.8, eps1=1.0, eps2=80.0, tol=1e-4, restart=10, maxit=100,
                         precond=2)),
}
PANELS = {"shell2097152": 2096704, "star204800": 204800, "star2097152": 2097152, "shell8388608": 8386816,
          "shell524176": 524176, "sphere20480": 20480}
DEFAULT_CASE = "shell2097152"
METRIC = "matvec/s"
FLOP_PER_PAIR = 60.0   # algorithmic count per near panel pair (KER4 + apply)
# a workload too large for a full ncu capture -> (the captured case, panel ratio)
PROFILE_PROXY = {"shell2097152": (("shell524176", 2096704 / 524176),)}
DIRECT_ORACLE_MAX = 300000   # panels up to which the FP64 direct-summation oracle is solved
SAMPLE_ABOVE = 500000        # panels above which the CPU reference matvec is sampled
REF_GPU_DEFAULT_MAX = 2200000  # panels up to which the reference's CUDA backend is timed by default


def case_base(name):
    d = os.path.join(tempfile.gettempdir(), "fabipb_b200_cases")
    os.makedirs(d, exist_ok=True)
    base = os.path.join(d, name)
    if not all(os.path.exists(base + e) for e in (".vert", ".face", ".pqr")):
        from fabipb_b200 import meshgen
        kind, kw, _ = CASES[name]
        tmp = base + ".tmp%d" % os.getpid()
        {"sphere": meshgen.sphere_case, "star": meshgen.star_case, "shell": meshgen.shell_case}[kind](tmp, **kw)
        for e in (".vert", ".face", ".pqr"):
            os.replace(tmp + e, base + e)
    return base


def ref_opts(opts):
    return ["-p=%d" % opts["order"], "-t=%d" % opts["depth"], "-S=%g" % opts["sep_ratio"],
            "-eps1=%g" % opts["eps1"], "-eps2=%g" % opts["eps2"]]


def case_config(name, opts, extra=None):
    """The `config` object both arms report (same keys for the same case)."""
    cfg = {"workload": name, "panels": PANELS[name], "charges": CASES[name][1]["n_charges"],
           "order": opts["order"], "depth": opts["depth"], "sep_ratio": opts["sep_ratio"],
           "eps1": opts["eps1"], "eps2": opts["eps2"], "kappa": 0.1257, "tol": opts["tol"],
           "restart": opts["restart"], "precond": {2: "block LU (-P=2)", 3: "diagonal (-P=3)"}[opts["precond"]],
           "l2": "256 MiB buffer written between steps, outside the timed intervals"}
    if extra:
        cfg.update(extra)
    return cfg


def cpu_reference_rate(base, name, opts, reps, warmup=1, budget=60.0):
    """matvec/s of the reference CPU solver (oracle/_ref) on every host core,
    or of the FP64 restatement oracle when that build is absent; returns
    (value, kind, cores, sample, steps_timed).  Meshes up to SAMPLE_ABOVE
    panels: whole MtVmain calls, at most `reps`, fewer when the warm-up shows
    they would exceed `budget` seconds.  Larger meshes: `reps` estimated
    steps, each the FMM passes timed whole plus the near field timed on a
    leaf sample of about budget/reps seconds and scaled by panel pairs."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    if O.ref_available():
        pre = os.path.join(tempfile.gettempdir(), "fabipb_ref_time")
        if PANELS[name] > SAMPLE_ABOVE:
            out = O.run_ref_harness("sample", base, pre, ref_opts(opts), threads=cores, reps=reps, warmup=warmup,
                                    budget=max(budget / max(reps + warmup, 1) * 0.5, 1.0))
            r = json.loads(out.strip().splitlines()[-1])
            sample = ("%d estimated matvecs (MtVmain) after %d warm-up: the FMM passes and diagonal timed whole "
                      "(%.2f s each), the near field timed on the first %d of %d leaves (%.3g of %.3g panel pairs, "
                      "%.2f s) and scaled by panel pairs" %
                      (r["reps"], warmup, r["far_s"], r["sample_leaves"], r["leaves"], r["sample_pairs"],
                       r["near_pairs"], r["near_sample_s"]))
            cpu_reference_rate.sampled_step_s = r["seconds"] / max(r["reps"], 1)
            return r["matvec_per_s"], "reference", cores, sample, r["reps"]
        out = O.run_ref_harness("time", base, pre, ref_opts(opts), threads=cores, reps=reps,
                                warmup=max(warmup, 1), budget=budget)
        r = json.loads(out.strip().splitlines()[-1])
        return (r["matvec_per_s"], "reference", cores,
                "%d timed matvecs (MtVmain) of the full mesh after %d warm-up" % (r["reps"], max(warmup, 1)),
                r["reps"])
    from fabipb_b200 import meshio
    pan, _ = meshio.load_case(base)
    orc = O.Oracle(pan, O.make_params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"],
                                      eps1=opts["eps1"], eps2=opts["eps2"], threads=cores))
    x = np.random.default_rng(0).standard_normal(2 * pan.n)
    w0 = time.perf_counter()
    for _ in range(max(warmup, 1)):
        orc.matvec(x)
    reps = max(1, min(reps, int(budget / max(time.perf_counter() - w0, 1e-9))))
    t0 = time.perf_counter()
    for _ in range(reps):
        orc.matvec(x)
    dt = time.perf_counter() - t0
    return reps / dt, "port", cores, "%d timed matvecs of the full mesh (FP64 restatement)" % reps, reps


def ref_gpu_rate(base, name, opts, reps=10, timeout=900, budget=60.0):
    """matvec/s of the reference's own CUDA backend (src/gpu_backend_cuda.cu,
    compiled from its sources into oracle/_ref by `make -C oracle refgpu`):
    MtVmain with -g=1 on this GPU, host wall time of `reps` calls after two
    warm-up calls.  None when that build is absent."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_HARNESS_GPU):
        return None
    try:
        pre = os.path.join(tempfile.gettempdir(), "fabipb_refgpu_time")
        out = O.run_ref_harness("time", base, pre, ref_opts(opts), threads=os.cpu_count() or 1, reps=reps,
                                warmup=2, gpu=True, timeout=timeout, budget=budget)
        r = json.loads(out.strip().splitlines()[-1])
    except Exception as e:   # a baseline, not the product: report the failure, keep the line
        return {"value": None, "error": str(e)[-300:]}
    return {"value": r["matvec_per_s"], "unit": "matvec/s", "kind": "reference CUDA backend (-g=1, FP64)",
            "sample": "%d timed MtVmain calls after 2 warm-up, host wall time" % r["reps"]}


def dropin_rate(base, opts, reps=10, timeout=900):
    """matvec/s end to end through the plugin ABI: the reference host's
    MtVmain (its host M2M/L2L, host vectors) with this library behind
    gpu_backend.h (oracle/_ref/ref_harness_dropin, -g=1), host wall time."""
    from oracle import oracle as O
    exe = os.path.join(os.path.dirname(O.REF_HARNESS), "ref_harness_dropin")
    if not os.path.exists(exe):
        return None
    try:
        pre = os.path.join(tempfile.gettempdir(), "fabipb_dropin_time")
        cmd = [exe, "time", base, pre] + ref_opts(opts) + ["-g=1", "--reps=%d" % reps, "--warmup=2",
                                                         "--budget=60"]
        r = subprocess.run(cmd, env=O.ref_env(os.cpu_count() or 1), capture_output=True, text=True,
                           timeout=timeout, check=True)
        v = json.loads(r.stdout.strip().splitlines()[-1])
    except Exception as e:
        return {"value": None, "error": str(e)[-300:]}
    n2 = 2 * v["panels"]
    return {"value": v["matvec_per_s"], "unit": "matvec/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
            "path": "reference host MtVmain on gpu_backend.h (host M2M/L2L, per-stage copies of the %d-vector)" % n2,
            "sample": "%d timed MtVmain calls after 2 warm-up, host wall time" % v["reps"]}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.path = os.path.join(tempfile.gettempdir(), "fabipb_clocks_%d.csv" % os.getpid())
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.fp = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fp.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fp:
            for line in fp:
                p = [v.strip() for v in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        load = [v for v in sm if smax and v > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": smax,
                "sm_mhz_p10": float(np.percentile(sm, 10)) if sm else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args, backend="nccl"):
    """One process per GPU under torchrun (RANK/WORLD_SIZE/LOCAL_RANK from the
    environment); the path does not shard, so the ranks are independent
    replicas and the process group only carries barriers and the timing
    reduction."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def replica_times(pg, total_s, e2e_s, device="cuda"):
    """The slowest replica's device and end-to-end times (max over ranks)."""
    if not pg:
        return total_s, e2e_s
    import torch
    t = torch.tensor([total_s, e2e_s], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t[0]), float(t[1])


def replica_value(world, steps, total_s):
    """Whole-job matvec/s: every replica did `steps` matvecs in at most total_s."""
    return world * steps / total_s


def run_reference(args):
    """The reference arm: the reference's own CPU implementation of the
    matvec (oracle/_ref, compiled from its sources), every host core, on this
    arm's case, metric and config; rank 0 alone under torchrun."""
    rank, world, local, pg = dist_setup(args)
    name = args.case
    opts = CASES[name][2]
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    base = case_base(name)
    t0 = time.perf_counter()
    cpu_reference_rate.sampled_step_s = None
    value, kind, cores, sample, timed = cpu_reference_rate(base, name, opts, args.steps, args.warmup,
                                                           budget=args.ref_budget)
    wall = time.perf_counter() - t0
    # a sampled step (large meshes) takes far less than the matvec it stands for: ms_per_step is
    # the wall time of the steps actually timed, value the whole-matvec rate they estimate
    step_s = cpu_reference_rate.sampled_step_s or 1.0 / value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world,
            "steps": timed, "warmup": args.warmup, "ms_per_step": 1000.0 * step_s,
            "ms_per_matvec_estimated": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded %s surface, %d panels, %d charges)" %
                    (CASES[name][0], PANELS[name], CASES[name][1]["n_charges"]),
            "config": case_config(name, opts, {"precision": "fp64 (reference CPU)",
                                               "parallelism": "host threads"}),
            "cpu_baseline": {"value": value, "unit": "matvec/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "steps_requested": args.steps, "wall_s": wall}
    if pg:
        pg.destroy_process_group()
    print(json.dumps(line))


def measured_hbm_gbs():
    """Copy bandwidth measured on this pool (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            return float(json.load(fp)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pass_report(surf, info, x_ptr, flush, reps, prec_is_mixed, fp32, fp64):
    """Per-pass device times (CUDA events between the passes of one matvec,
    L2 flushed before every matvec) against each pass's bound: algorithmic
    FLOPs for the near field and M2L, algorithmic bytes for the rest."""
    import torch
    acc = None
    for _ in range(reps):
        flush.zero_()
        t = surf.pass_times(x_ptr, reps=1, on_device=1)
        acc = t if acc is None else {k: acc[k] + t[k] for k in acc}
    ms = {k: v / reps for k, v in acc.items()}
    n, leaves, cubes = info["panels"], info["leaves"], info["cubes"]
    p, pl = info["max_order"], info["leaf_order"]
    nmom = lambda q: (q + 1) * (q + 2) * (q + 3) // 6
    from math import comb
    hbm, hbm_src = measured_hbm_gbs()
    near_peak = fp32 if prec_is_mixed else fp64
    qb = 4.0 if prec_is_mixed else 8.0   # bytes per leaf-matrix entry (FP32 copies in a mixed context)
    work = {
        "near": ("flop", FLOP_PER_PAIR * info["near_panel_pairs"], near_peak),
        "q2m": ("bytes", qb * 2 * nmom(pl) * n + 8.0 * (2 * n + 2 * nmom(p) * leaves), hbm),
        "m2m": ("bytes", 8.0 * 2 * nmom(p) * 2 * cubes, hbm),
        "m2l": ("flop", 8.0 * comb(p + 6, 6) * info["m2l_pairs"], fp32 if prec_is_mixed and p <= 5 else fp64),
        "l2l": ("bytes", 8.0 * 4 * nmom(p) * 2 * cubes, hbm),
        "l2p": ("bytes", qb * 2 * nmom(pl) * n + 8.0 * (4 * nmom(p) * leaves + 6 * n), hbm),
    }
    out = {}
    for k, (kind, amount, peak) in work.items():
        t = ms[k] / 1000.0
        if kind == "flop":
            ach = amount / t / 1e12
            out[k] = {"ms": ms[k], "bound": ("fp32" if peak == fp32 else "fp64"),
                      "achieved": ach, "unit": "TFLOP/s", "peak": peak, "frac": ach / peak,
                      "algorithmic": amount, "peak_source": "measured FMA rate of this GPU"}
        else:
            ach = amount / t / 1e9
            out[k] = {"ms": ms[k], "bound": "hbm", "achieved": ach, "unit": "GB/s", "peak": peak,
                      "frac": ach / peak, "algorithmic": amount, "peak_source": hbm_src}
    return out


def _ev():
    import torch
    return torch.cuda.Event(enable_timing=True)


def solve_report(pan, ch, name, opts, device, st, reps=3, adjoint=True, fp64_adjoint=True):
    """Full solves of the case in both precisions, every vector on the device:
    RHS (direct, or the charge-tree treecode above 2e11 panel-charge pairs as
    the reference's GPU policy), the case's preconditioner, GMRES from x0 = b
    (as the reference CLI), the panel-tree energy; the mixed context also
    solves by iterative refinement (FP64 residuals) to the same tolerance.
    Each precision runs 1 + reps times on a fresh context; the first run is
    not reported (it pays the one-time module loading).  Every timed interval
    is CUDA events on the library's stream around library calls only: setup
    = context (tree, near field, FMM lists) + RHS + preconditioner."""
    import torch
    from fabipb_b200 import lib
    kcal = 2.0 * np.pi * 332.0716
    use_tree = pan.n * len(ch.q) > 2e11
    n2 = 2 * pan.n
    runs = {"mixed": [], "fp64": []}
    mem_peak = {"mixed": 0.0, "fp64": 0.0}
    seq = [("mixed", lib.MIXED)] * (1 + reps) + [("fp64", lib.FP64)] * (1 + reps)
    b = torch.empty(n2, dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    for tag, prec in seq:
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        ev = [_ev() for _ in range(4)]
        ev[0].record(st)
        prm = lib.params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"], eps1=opts["eps1"],
                         eps2=opts["eps2"], precision=prec, device=device)
        s = lib.Surface(pan, prm, ch)
        s.set_stream(st.cuda_stream)
        s.rhs(use_tree=use_tree, out=b.data_ptr(), on_device=1)
        s.precond_setup(opts["precond"])
        ev[1].record(st)
        torch.cuda.synchronize()
        free, total = torch.cuda.mem_get_info()
        mem_peak[tag] = max(mem_peak[tag], (total - free) / 2**30)
        x.copy_(b)
        ev[2].record(st)
        _, it, res, info = s.solve(b.data_ptr(), x.data_ptr(), restart=opts["restart"], maxit=opts["maxit"],
                                   tol=opts["tol"], on_device=1)
        ev[3].record(st)
        ee = [_ev(), _ev()]
        ee[0].record(st)
        e = s.energy_raw(x.data_ptr(), on_device=1) * kcal
        ee[1].record(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        r = {"setup_s": ev[0].elapsed_time(ev[1]) / 1000.0, "gmres_s": ev[2].elapsed_time(ev[3]) / 1000.0,
             "energy_s": ee[0].elapsed_time(ee[1]) / 1000.0, "iterations": it, "residual": res, "info": info,
             "energy_kcal_mol": e, "wall_s": wall}
        r["solve_s"] = r["setup_s"] + r["gmres_s"] + r["energy_s"]
        if tag == "mixed":
            # FP32-FMM corrections with FP64 residuals, to the same tolerance
            x.copy_(b)
            rf = [_ev(), _ev()]
            rf[0].record(st)
            _, outer, itr, resr, infr = s.solve_refined(b.data_ptr(), x.data_ptr(), restart=opts["restart"],
                                                        maxit=2 * opts["maxit"], tol_inner=opts["tol"],
                                                        tol=opts["tol"], max_outer=10, on_device=1)
            rf[1].record(st)
            torch.cuda.synchronize()
            er = s.energy_raw(x.data_ptr(), on_device=1) * kcal
            r["refined"] = {"gmres_s": rf[0].elapsed_time(rf[1]) / 1000.0, "outer": outer, "iterations": itr,
                            "residual_fp64": resr, "info": infr, "energy_kcal_mol": er}
            r["refined"]["solve_s"] = r["setup_s"] + r["refined"]["gmres_s"] + r["energy_s"]
        if adjoint and (fp64_adjoint or tag == "mixed"):
            # gradients of the (direct) energy: forward = direct RHS + GMRES +
            # direct energy, backward = adjoint GMRES + dE/dq, dE/dx of every charge
            ag = [_ev() for _ in range(3)]
            torch.cuda.synchronize()
            ag[0].record(st)
            ef, itf, resf, inff = s.forward(restart=opts["restart"], maxit=opts["maxit"], tol=opts["tol"])
            ag[1].record(st)
            dq, dx, itb, resb, infb = s.backward(1.0, restart=opts["restart"], maxit=opts["maxit"], tol=opts["tol"])
            ag[2].record(st)
            torch.cuda.synchronize()
            fs, bs = ag[0].elapsed_time(ag[1]) / 1000.0, ag[1].elapsed_time(ag[2]) / 1000.0
            r["adjoint"] = {"forward_s": fs, "backward_s": bs, "backward_over_forward": bs / fs,
                            "forward_iterations": itf, "backward_iterations": itb, "info": [inff, infb],
                            "charges": int(len(ch.q)), "energy_direct_kcal_mol": ef * kcal}
        # the pool keeps freed blocks (release threshold at its maximum), so memory in use
        # at the end of the run is the high-water mark of the run's allocations
        torch.cuda.synchronize()
        free, total = torch.cuda.mem_get_info()
        r["device_mem_high_water_gib"] = (total - free) / 2**30
        s.close()
        runs[tag].append(r)
    med = lambda v: float(np.median(v))
    out = {}
    for tag, rs in runs.items():
        rs = rs[1:]
        r = dict(rs[-1])
        for k in ("setup_s", "gmres_s", "energy_s", "solve_s", "wall_s"):
            r[k] = med([q[k] for q in rs])
            r[k + "_runs"] = [q[k] for q in rs]
        if "refined" in r:
            r["refined"] = dict(rs[-1]["refined"])
            for k in ("gmres_s", "solve_s"):
                r["refined"][k] = med([q["refined"][k] for q in rs])
                r["refined"][k + "_runs"] = [q["refined"][k] for q in rs]
        if "adjoint" in rs[-1]:
            a = dict(rs[-1]["adjoint"])
            for k in ("forward_s", "backward_s"):
                a[k] = med([q["adjoint"][k] for q in rs])
                a[k + "_runs"] = [q["adjoint"][k] for q in rs]
            a["backward_over_forward"] = a["backward_s"] / a["forward_s"]
            r["adjoint"] = a
        r["runs"] = len(rs)
        r["device_mem_gib"] = mem_peak[tag]
        r["device_mem_high_water_gib"] = max(q["device_mem_high_water_gib"] for q in rs)
        out[tag] = r
    m, f = out["mixed"], out["fp64"]
    rel = lambda a, b: abs(a - b) / abs(b)
    out["energy_rel_err_mixed_vs_fp64"] = rel(m["energy_kcal_mol"], f["energy_kcal_mol"])
    out["energy_rel_err_refined_vs_fp64"] = rel(m["refined"]["energy_kcal_mol"], f["energy_kcal_mol"])
    out["gmres_speedup_mixed_vs_fp64"] = f["gmres_s"] / m["gmres_s"]
    out["gmres_speedup_refined_vs_fp64"] = f["gmres_s"] / m["refined"]["gmres_s"]
    out["solve_speedup_refined_vs_fp64"] = f["solve_s"] / m["refined"]["solve_s"]
    out["rhs"] = "charge tree" if use_tree else "direct"
    out["tol"] = opts["tol"]
    out["restart"] = opts["restart"]
    out["precond"] = opts["precond"]
    return out


def direct_oracle_report(pan, ch, opts, device, st, energies):
    """The FP64 direct-summation oracle: the dense direct operator (every
    panel pair through the near-field rules, no FMM), solved in FP64 with the
    case's preconditioner to 1e-8, its panel-tree energy; the relative error
    of each FMM energy in `energies` (tag -> kcal/mol) against it."""
    import torch
    from fabipb_b200 import lib
    kcal = 2.0 * np.pi * 332.0716
    prm = lib.params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"], eps1=opts["eps1"],
                     eps2=opts["eps2"], precision=lib.FP64, device=device)
    ev = [_ev() for _ in range(3)]
    ev[0].record(st)
    s = lib.Surface(pan, prm, ch, direct=True)
    s.set_stream(st.cuda_stream)
    n2 = 2 * pan.n
    b = torch.empty(n2, dtype=torch.float64, device="cuda")
    s.rhs(use_tree=False, out=b.data_ptr(), on_device=1)
    s.precond_setup(opts["precond"])
    ev[1].record(st)
    x = b.clone()
    _, it, res, info = s.solve(b.data_ptr(), x.data_ptr(), restart=opts["restart"], maxit=300, tol=1e-8,
                               on_device=1)
    ev[2].record(st)
    e = s.energy_raw(x.data_ptr(), on_device=1) * kcal
    torch.cuda.synchronize()
    pairs = s.info()["near_panel_pairs"]
    s.close()
    out = {"energy_kcal_mol": e, "iterations": it, "residual": res, "info": info, "tol": 1e-8,
           "panel_pairs_per_matvec": pairs, "setup_s": ev[0].elapsed_time(ev[1]) / 1000.0,
           "gmres_s": ev[1].elapsed_time(ev[2]) / 1000.0}
    for tag, v in energies.items():
        out["energy_rel_err_" + tag] = abs(v - e) / abs(e)
    return out


def run_ours(args):
    import torch
    from fabipb_b200 import lib, meshio

    rank, world, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    name = args.case
    opts = CASES[name][2]
    base = case_base(name)
    pan, ch = meshio.load_case(base)
    # the reference's CUDA backend first, in its own process, while this
    # process holds no device memory yet
    ref_gpu = None
    if rank == 0 and not args.no_ref_gpu:
        if PANELS[name] <= DIRECT_ORACLE_MAX:
            ref_gpu = ref_gpu_rate(base, name, opts)
        elif PANELS[name] <= REF_GPU_DEFAULT_MAX or args.ref_gpu:
            # a few seconds per reference matvec here: 3 timed calls, about 30 s of timing
            ref_gpu = ref_gpu_rate(base, name, opts, reps=3, budget=30.0)
        else:
            ref_gpu = {"value": None, "skipped": "not run by default above %d panels (--ref-gpu runs it)" %
                       REF_GPU_DEFAULT_MAX}
    fp32_peak = lib.simt_peak_tflops(local, fp64=False)
    fp64_peak = lib.simt_peak_tflops(local, fp64=True)
    prec = lib.MIXED if args.precision == "mixed" else lib.FP64
    prm = lib.params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"], eps1=opts["eps1"],
                     eps2=opts["eps2"], precision=prec, device=local)
    surf = lib.Surface(pan, prm, ch)
    info = surf.info()
    n2 = 2 * surf.n
    stream = torch.cuda.current_stream()
    surf.set_stream(stream.cuda_stream)
    x = torch.from_numpy(np.random.default_rng(rank).standard_normal(n2)).cuda()
    y = torch.zeros(n2, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_steps(fn, k):
        st_, en_ = [_ev() for _ in range(k)], [_ev() for _ in range(k)]
        for i in range(k):
            flush.zero_()
            st_[i].record(stream)
            fn()
            en_[i].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in zip(st_, en_)]

    def step():
        surf.matvec(x.data_ptr(), 1.0, 0.0, y.data_ptr(), on_device=1)

    def near_only():
        surf.apply(x.data_ptr(), part=lib.NEAR, alpha=1.0, beta=1.0, pot=y.data_ptr(), on_device=1)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = surf.launch_count()
    with ClockSampler(local) as clk:
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        step_ms = timed_steps(step, args.steps)
        if pg:
            pg.barrier()
        launches = surf.launch_count() - launches0
        # the dominant kernel alone, same stream, for the roofline
        near_ms = timed_steps(near_only, args.steps)
        # e2e: host buffers through the C ABI (pinned), copies inside the region
        xh = torch.from_numpy(np.random.default_rng(rank + 7).standard_normal(n2)).pin_memory()
        yh = torch.zeros(n2, dtype=torch.float64).pin_memory()
        xh_np, yh_np = xh.numpy(), yh.numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            surf.matvec(xh_np, 1.0, 0.0, out=yh_np)
        e2e_s = time.perf_counter() - t0
    total_s = sum(step_ms) / 1000.0
    if pg:
        total_s, e2e_s = replica_times(pg, total_s, e2e_s)
    e2e_rate = args.steps / e2e_s
    value = replica_value(world, args.steps, total_s)
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    clocks = clk.summary()
    near_s = float(np.mean(near_ms)) / 1000.0
    pairs = float(info["near_panel_pairs"])
    achieved = FLOP_PER_PAIR * pairs / near_s / 1e12
    if prec == lib.MIXED:
        peak, bound = fp32_peak, "fp32"
        peak_src = "measured FP32 FMA rate of this GPU (packed f32x2 FMA chains, fabipb_b200_simt_peak)"
    else:
        peak, bound = fp64_peak, "fp64"
        peak_src = "measured FP64 FMA rate of this GPU (DFMA chains, fabipb_b200_simt_peak)"
    # DRAM bytes per launch from the committed ncu summary of this kernel and
    # workload, or of the smaller capture that stands in for it, scaled by panels
    # the near-field pass: the symmetric kernel (unordered leaf pairs) and the ordered kernel (self
    # pairs, scratch sums, FP64 special pairs), timed together as one apply
    kname = ("near_sym_f2_kernel<0> + near_apply_f2_kernel<0>" if prec == lib.MIXED
             else "near_sym_kernel<double,0> + near_apply_kernel<double,0>")
    kfiles = (("near_sym_f2_kernel", "near_apply_f2_kernel") if prec == lib.MIXED
              else ("near_sym_kernel_double", "near_apply_kernel_double"))
    traffic, traffic_src = None, None
    for kfile in kfiles:
        for case, scale in ((args.case, 1.0),) + tuple(PROFILE_PROXY.get(args.case, ())):
            prof = os.path.join(ROOT, "profiles", "%s_%s.md" % (kfile, case))
            if traffic is None and os.path.exists(prof):
                with open(prof) as fp:
                    m = re.search(r"dram_bytes_per_launch[^|]*\| (\d+)", fp.read())
                if m:
                    traffic = int(int(m.group(1)) * scale)
                    traffic_src = "ncu capture %s of %s%s" % (os.path.basename(prof), case, "" if scale == 1.0 else
                                                              ", scaled by panels (x%.2f)" % scale)
    passes = pass_report(surf, info, x.data_ptr(), flush, args.steps, prec == lib.MIXED, fp32_peak, fp64_peak)
    free, total = torch.cuda.mem_get_info()
    mem_ctx = (total - free) / 2**30
    surf.close()
    # the plain FP64 operator on the same case (a second context)
    fp64_rate = None
    if prec == lib.MIXED and not args.no_fp64:
        s64 = lib.Surface(pan, lib.params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"],
                                          eps1=opts["eps1"], eps2=opts["eps2"], precision=lib.FP64, device=local), ch)
        s64.set_stream(stream.cuda_stream)
        for _ in range(2):
            s64.matvec(x.data_ptr(), 1.0, 0.0, y.data_ptr(), on_device=1)
        k64 = max(3, args.steps // 2)
        ms64 = timed_steps(lambda: s64.matvec(x.data_ptr(), 1.0, 0.0, y.data_ptr(), on_device=1), k64)
        fp64_rate = {"value": 1000.0 * k64 / sum(ms64), "unit": "matvec/s", "steps": k64,
                     "ms_per_step": sum(ms64) / k64}
        s64.close()
    del flush
    torch.cuda.empty_cache()
    solve = None
    if not args.no_solve:
        with ClockSampler(local) as clk2:   # the clocks during the solves too
            # the FP64 context's gradients by default only up to DIRECT_ORACLE_MAX panels (at 2.1M panels
            # and 500,000 charges its direct sums take 20 s a run; --fp64-adjoint times them anyway)
            fp64_adj = args.fp64_adjoint or (PANELS[name] <= DIRECT_ORACLE_MAX and not args.no_fp64_adjoint)
            solve = solve_report(pan, ch, name, opts, local, stream, reps=args.solve_reps,
                                 adjoint=not args.no_adjoint, fp64_adjoint=fp64_adj)
            if PANELS[name] <= DIRECT_ORACLE_MAX and not args.no_direct_oracle:
                en = {"mixed": solve["mixed"]["energy_kcal_mol"], "refined": solve["mixed"]["refined"]["energy_kcal_mol"],
                      "fp64": solve["fp64"]["energy_kcal_mol"]}
                solve["direct_oracle"] = direct_oracle_report(pan, ch, opts, local, stream, en)
        solve["clocks"] = clk2.summary()
    dropin = None if args.no_dropin else dropin_rate(base, opts)
    cpu = None
    if not args.no_cpu_baseline:
        v, kind, cores, sample, _ = cpu_reference_rate(base, name, opts, args.cpu_reps, 1, budget=30.0)
        cpu = {"value": v, "unit": "matvec/s", "cores": cores, "kind": kind, "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == lib.MIXED else "f64",
        "data": "synthetic (seeded %s surface, %d panels, %d charges)" %
                (CASES[name][0], surf.n, CASES[name][1]["n_charges"]),
        "config": case_config(name, opts, {"precision": args.precision,
                                           "parallelism": "replicas" if world > 1 else "single"}),
        "tree": {"leaves": info["leaves"], "max_leaf": info["max_leaf"], "mean_leaf": surf.n / info["leaves"],
                 "near_panel_pairs": info["near_panel_pairs"], "m2l_pairs": info["m2l_pairs"],
                 "special_pairs": info["special_pairs"]},
        "e2e": {"value": e2e_rate * world, "unit": "matvec/s", "h2d_bytes_per_step": n2 * 8,
                "d2h_bytes_per_step": n2 * 8, "path": "fabipb_b200_matvec, pinned host x and y"},
        "e2e_dropin": dropin,
        "roofline": {"kernel": kname, "bound": bound, "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_src, "flop_per_pair": FLOP_PER_PAIR,
                     "pairs_per_launch": pairs, "launch_ms": near_s * 1000.0},
        "peaks": {"fp32_tflops": fp32_peak, "fp64_tflops": fp64_peak, "hbm_gbs": measured_hbm_gbs()[0]},
        "fp64": fp64_rate,
        "cpu_baseline": cpu,
        "ref_gpu_baseline": ref_gpu,
        "gpu_launches": launches,
        "clocks": clocks,
        "setup_s": info["setup_seconds"],
        "passes": passes,
        "solve": solve,
        "device_mem_gib_matvec_context": mem_ctx,
    }
    if pg:
        pg.destroy_process_group()
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--case", default=DEFAULT_CASE, choices=sorted(CASES))
    ap.add_argument("--cpu-reps", type=int, default=2)
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of timed reference work at most (--impl reference)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="time the reference's own CUDA backend also on meshes above %d panels" % REF_GPU_DEFAULT_MAX)
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's CUDA backend")
    ap.add_argument("--no-dropin", action="store_true", help="skip the plugin-ABI end-to-end timing")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 operator's matvec rate")
    ap.add_argument("--no-direct-oracle", action="store_true", help="skip the FP64 direct-summation oracle solve")
    ap.add_argument("--no-solve", action="store_true", help="skip the mixed/FP64 solve report")
    ap.add_argument("--solve-reps", type=int, default=3, help="reported runs per precision (after one warm-up run)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward/backward gradient timing")
    ap.add_argument("--no-fp64-adjoint", action="store_true", help="time the gradients of the mixed context only")
    ap.add_argument("--fp64-adjoint", action="store_true",
                    help="time the FP64 context's gradients also above %d panels" % DIRECT_ORACLE_MAX)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
