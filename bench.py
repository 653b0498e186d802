"""Benchmark of the FABIPB GMRES matvec on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--case star204800|star2097152|sphere20480]

Workload (one "step" = one operator application y = (D - K)x, the GMRES
matvec of src/fabipb.c:1237): the star-shaped globular surface of 204,800
flat triangles (octahedral geodesic, frequency 160, radius 25 A perturbed by
l=2..6 harmonics), Taylor order p=4, MAC ratio 0.7, octree depth 5 (mean
leaf 46 panels), eps 2/80, kappa 0.1257, synthetic seeded inputs.
--case star2097152 runs the same measurement on the 2,097,152-panel star
(frequency 512, radius 50 A, depth 7: mean leaf 31 panels, 100,000 charges),
--case star8388608 on the 8,388,608-panel star (frequency 1024, radius 100 A,
depth 8, 2,000,000 charges; with --solve-reps 1 --no-adjoint for a short run).

Reported:
  value      matvec/s with x, y resident in HBM (device time, CUDA events on
             the library's stream), L2 flushed between steps outside the
             timed intervals;
  e2e        matvec/s through the C ABI with host buffers (H2D of x and D2H
             of y inside the timed region, pinned host memory);
  roofline   the near-field P2P kernel (the dominant kernel): algorithmic
             FLOPs (60 per panel pair) per launch / its event-timed duration,
             against the FP32 SIMT peak of the measured SM clock;
  cpu_baseline  the reference CPU solver compiled from its own sources
             (oracle/_ref), timed on a bounded sample of matvecs on this
             host's cores;
  ref_gpu_baseline  (--ref-gpu) the reference's own CUDA backend compiled
             from its sources for sm_100a (oracle/_ref/ref_harness_gpu), the
             same matvec with -g=1 on this GPU.
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
    # name: (generator, kwargs, solver options)
    "star204800": ("star", dict(freq=160, radius=25.0, n_charges=20000, seed=1),
                   dict(order=4, depth=5, sep_ratio=0.7, eps1=2.0, eps2=80.0, tol=1e-5, restart=10)),
    # the 2.1M-panel size: 2,097,152 triangles (octahedral freq 512, radius 50 A), 100,000 charges
    "star2097152": ("star", dict(freq=512, radius=50.0, n_charges=100000, seed=7),
                    dict(order=4, depth=7, sep_ratio=0.7, eps1=2.0, eps2=80.0, tol=1e-6, restart=10)),
    # the scale-stress size: 8,388,608 triangles (freq 1024, radius 100 A), 2,000,000 charges
    "star8388608": ("star", dict(freq=1024, radius=100.0, n_charges=2000000, seed=11),
                    dict(order=4, depth=8, sep_ratio=0.7, eps1=2.0, eps2=80.0, tol=1e-6, restart=10)),
    "sphere20480": ("sphere", dict(nsub=5, radius=20.0, n_charges=500, seed=0),
                    dict(order=3, depth=3, sep_ratio=0.8, eps1=1.0, eps2=80.0, tol=1e-4, restart=10)),
}
PANELS = {"star204800": 204800, "star2097152": 2097152, "star8388608": 8388608, "sphere20480": 20480}
METRIC = "matvec/s"
FLOP_PER_PAIR = 60.0   # algorithmic count per near panel pair (KER4 + apply)


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


def cpu_reference_rate(base, opts, reps, warmup=1, budget=60.0):
    """matvec/s of the reference CPU solver (oracle/_ref) or, if it is absent,
    of the FP64 restatement oracle; returns (value, kind, cores, sample).
    At most `reps` timed matvecs, fewer if the warm-up matvec shows they would
    exceed `budget` seconds (at least one is always timed)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    if O.ref_available():
        pre = os.path.join(tempfile.gettempdir(), "fabipb_ref_time")
        out = O.run_ref_harness("time", base, pre, ref_opts(opts), threads=cores, reps=reps,
                                warmup=max(warmup, 1), budget=budget)
        r = json.loads(out.strip().splitlines()[-1])
        return (r["matvec_per_s"], "reference", cores,
                "%d timed matvecs (MtVmain) of the full mesh after %d warm-up" % (r["reps"], max(warmup, 1)))
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
    return reps / dt, "port", cores, "%d timed matvecs of the full mesh (FP64 restatement)" % reps


def ref_gpu_rate(base, opts, reps=10):
    """matvec/s of the reference's own CUDA backend (src/gpu_backend_cuda.cu,
    compiled from its sources into oracle/_ref by `make -C oracle refgpu`):
    MtVmain with -g=1 on this GPU, host wall time of `reps` calls after two
    warm-up calls.  None when that build is absent or the run fails."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_HARNESS_GPU):
        return None
    try:
        pre = os.path.join(tempfile.gettempdir(), "fabipb_refgpu_time")
        out = O.run_ref_harness("time", base, pre, ref_opts(opts), threads=os.cpu_count() or 1, reps=reps,
                                warmup=2, gpu=True, timeout=900)
        r = json.loads(out.strip().splitlines()[-1])
    except Exception as e:   # a baseline, not the product: report the failure, keep the line
        return {"value": None, "error": str(e)[:200]}
    return {"value": r["matvec_per_s"], "unit": "matvec/s", "kind": "reference CUDA backend (-g=1, FP64)",
            "sample": "%d timed MtVmain calls after 2 warm-up, host wall time" % r["reps"]}


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
    rank, world, local, pg = dist_setup(args)
    name = args.case
    opts = CASES[name][2]
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    base = case_base(name)
    t0 = time.perf_counter()
    # one process: setup once, `warmup` untimed matvecs, then `steps` timed ones
    value, kind, cores, sample = cpu_reference_rate(base, opts, args.steps, 1, budget=args.ref_budget)
    wall = time.perf_counter() - t0
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded %s surface, %d panels)" % (CASES[name][0], PANELS[name]),
            "config": {"workload": name, "panels": PANELS[name],
                       "order": opts["order"], "depth": opts["depth"], "sep_ratio": opts["sep_ratio"]},
            "cpu_baseline": {"value": value, "unit": "matvec/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
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


def pass_report(surf, info, x_ptr, flush, reps, prec_is_mixed, sm_mhz, n_sm):
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
    fp32 = n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
    fp64 = n_sm * 64 * 2 * sm_mhz * 1e6 / 1e12
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
                      "algorithmic": amount}
        else:
            ach = amount / t / 1e9
            out[k] = {"ms": ms[k], "bound": "hbm", "achieved": ach, "unit": "GB/s", "peak": peak,
                      "frac": ach / peak, "algorithmic": amount, "peak_source": hbm_src}
    m2l_bytes = 16.0 * nmom(p) * info["m2l_pairs"]   # the (D G0, D Gk) tensors read per launch
    out["m2l"]["tensor_gbs"] = m2l_bytes / (ms["m2l"] / 1000.0) / 1e9
    return out


def solve_report(pan, ch, opts, device, st, reps=3, adjoint=True):
    """Full solves of the same case in both precisions: RHS (direct, or the
    charge-tree treecode above 2e11 panel-charge pairs as the reference), block-LU
    preconditioner, device GMRES from x0 = b (as the reference CLI), energy.
    Times are CUDA-event times on the library's stream (the calls are
    synchronous); setup = context (tree, near field, FMM lists) + RHS +
    preconditioner."""
    import torch
    from fabipb_b200 import lib
    out = {}
    runs = {"mixed": [], "fp64": []}
    mem_peak = {"mixed": 0.0, "fp64": 0.0}   # device memory in use after the solver set-up, GiB
    kcal = 2.0 * np.pi * 332.0716
    # each precision runs 1 + reps times: the first pays the one-time loading
    # of the kernels it is the first to use and is not reported; every time
    # reported is the median over the other reps runs
    seq = [("mixed", lib.MIXED)] * (1 + reps) + [("fp64", lib.FP64)] * (1 + reps)
    # the reference's RHS policy on the GPU path: direct sums up to 2e11
    # panel-charge pairs, the charge-tree treecode above (src/fabipb_options.c:15-16)
    use_tree = pan.n * len(ch.q) > 2e11
    for tag, prec in seq:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        ev[0].record(st)
        prm = lib.params(order=opts["order"], depth=opts["depth"], sep_ratio=opts["sep_ratio"], eps1=opts["eps1"],
                         eps2=opts["eps2"], precision=prec, device=device)
        s = lib.Surface(pan, prm, ch)
        s.set_stream(st.cuda_stream)
        b = s.rhs(use_tree=use_tree)
        s.precond_setup(2)
        ev[1].record(st)
        torch.cuda.synchronize()
        free, total = torch.cuda.mem_get_info()
        mem_peak[tag] = max(mem_peak[tag], (total - free) / 2**30)
        x, it, res, info = s.solve(b, b.copy(), restart=opts["restart"], maxit=100, tol=opts["tol"])
        ev[2].record(st)
        e = s.energy_raw(x) * kcal
        ev[3].record(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        # iterative refinement to the same tolerance (FP64 residuals; in the
        # mixed context the corrections use the FP32 near field)
        rf = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        rf[0].record(st)
        xr, outer, itr, resr, infr = s.solve_refined(b, b.copy(), restart=opts["restart"], maxit=200,
                                                     tol_inner=opts["tol"], tol=opts["tol"], max_outer=10)
        rf[1].record(st)
        torch.cuda.synchronize()
        refined = {"gmres_s": rf[0].elapsed_time(rf[1]) / 1000.0, "outer": outer, "iterations": itr,
                   "residual_fp64": resr, "info": infr, "energy_kcal_mol": s.energy_raw(xr) * kcal}
        out[tag] = {"gmres_s": ev[1].elapsed_time(ev[2]) / 1000.0, "setup_s": ev[0].elapsed_time(ev[1]) / 1000.0,
                    "energy_s": ev[2].elapsed_time(ev[3]) / 1000.0, "wall_s": wall, "iterations": it,
                    "residual": res, "info": info, "energy_kcal_mol": e, "refined": refined}
        if not adjoint:
            s.close()
            runs[tag].append(out.pop(tag))
            continue
        # gradients of the (direct) energy: forward = RHS + GMRES + energy,
        # backward = adjoint GMRES + dE/dq, dE/dx of every charge
        ag = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ag[0].record(st)
        ef, itf, resf, inff = s.forward(restart=opts["restart"], maxit=100, tol=opts["tol"])
        ag[1].record(st)
        dq, dx, itb, resb, infb = s.backward(1.0, restart=opts["restart"], maxit=100, tol=opts["tol"])
        ag[2].record(st)
        torch.cuda.synchronize()
        fs, bs = ag[0].elapsed_time(ag[1]) / 1000.0, ag[1].elapsed_time(ag[2]) / 1000.0
        out[tag]["adjoint"] = {"forward_s": fs, "backward_s": bs, "backward_over_forward": bs / fs,
                               "forward_iterations": itf, "backward_iterations": itb, "info": [inff, infb],
                               "charges": int(len(ch.q)), "energy_direct_kcal_mol": ef * kcal}
        s.close()
        runs[tag].append(out.pop(tag))
    med = lambda v: float(np.median(v))
    for tag, rs in runs.items():
        rs = rs[1:]
        r = dict(rs[-1])
        for k in ("gmres_s", "setup_s", "energy_s", "wall_s"):
            r[k] = med([q[k] for q in rs])
        r["wall_s_runs"] = [q["wall_s"] for q in rs]
        r["refined"] = dict(rs[-1]["refined"], gmres_s=med([q["refined"]["gmres_s"] for q in rs]))
        if adjoint:
            a = dict(rs[-1]["adjoint"])
            a["forward_s"] = med([q["adjoint"]["forward_s"] for q in rs])
            a["backward_s"] = med([q["adjoint"]["backward_s"] for q in rs])
            a["backward_over_forward"] = a["backward_s"] / a["forward_s"]
            r["adjoint"] = a
        r["runs"] = len(rs)
        r["device_mem_gib"] = mem_peak[tag]
        out[tag] = r
    m, f = out["mixed"], out["fp64"]
    out["energy_rel_err_mixed_vs_fp64"] = abs(m["energy_kcal_mol"] - f["energy_kcal_mol"]) / abs(f["energy_kcal_mol"])
    out["gmres_speedup_mixed_vs_fp64"] = f["gmres_s"] / m["gmres_s"]
    out["rhs"] = "charge tree" if use_tree else "direct"
    out["tol"] = opts["tol"]
    out["restart"] = opts["restart"]
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
    ref_gpu = ref_gpu_rate(base, opts) if (args.ref_gpu and rank == 0) else None
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

    def step():
        surf.matvec(x.data_ptr(), 1.0, 0.0, y.data_ptr(), on_device=1)

    def near_only():
        surf.apply(x.data_ptr(), part=lib.NEAR, alpha=1.0, beta=1.0, pot=y.data_ptr(), on_device=1)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = surf.launch_count()
    with ClockSampler(local) as clk:
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        launches = surf.launch_count() - launches0
        # the dominant kernel alone, same stream, for the roofline
        nstarts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        nends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for i in range(args.steps):
            flush.zero_()
            nstarts[i].record(stream)
            near_only()
            nends[i].record(stream)
        torch.cuda.synchronize()
        # e2e: host buffers through the C ABI (pinned), copies inside the region
        xh = torch.from_numpy(np.random.default_rng(rank + 7).standard_normal(n2)).pin_memory()
        yh = torch.zeros(n2, dtype=torch.float64).pin_memory()
        xh_np, yh_np = xh.numpy(), yh.numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            surf.matvec(xh_np, 1.0, 0.0, out=yh_np)
        e2e_s = time.perf_counter() - t0
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    near_ms = [s.elapsed_time(e) for s, e in zip(nstarts, nends)]
    total_s = sum(step_ms) / 1000.0
    e2e_rate = args.steps / e2e_s
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
    sm_mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    props = torch.cuda.get_device_properties(local)
    n_sm = props.multi_processor_count
    if prec == lib.MIXED:
        peak = n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12
        peak_src = "FP32 SIMT FMA pipe: %d SMs x 128 lanes x 2 flop x %.0f MHz (median SM clock sampled)" % (n_sm, sm_mhz)
    else:
        peak = n_sm * 64 * 2 * sm_mhz * 1e6 / 1e12
        peak_src = "FP64 SIMT FMA pipe: %d SMs x 64 lanes x 2 flop x %.0f MHz (median SM clock sampled)" % (n_sm, sm_mhz)
    traffic = None
    # DRAM bytes per launch from the committed ncu summary of this kernel and workload
    kname = "near_apply_f2_kernel<0>" if prec == lib.MIXED else "near_apply_kernel<double,0>"
    tname = "%s_%s.md" % ("near_apply_f2_kernel" if prec == lib.MIXED else "near_apply_kernel_double", args.case)
    prof = os.path.join(ROOT, "profiles", tname)
    if os.path.exists(prof):
        with open(prof) as fp:
            m = re.search(r"dram_bytes_per_launch \| (\d+)", fp.read())
        traffic = int(m.group(1)) if m else None
    passes = pass_report(surf, info, x.data_ptr(), flush, args.steps, prec == lib.MIXED, sm_mhz, n_sm)
    mem_ctx = None
    if not args.no_solve:   # the matvec context is not needed any more: free it before the solves
        free, total = torch.cuda.mem_get_info()
        mem_ctx = (total - free) / 2**30
        surf.close()
    solve = None
    if not args.no_solve:
        with ClockSampler(local) as clk2:   # the clocks during the solves too
            solve = solve_report(pan, ch, opts, local, stream, reps=args.solve_reps, adjoint=not args.no_adjoint)
        solve["clocks"] = clk2.summary()
    cpu = None
    if not args.no_cpu_baseline:
        v, kind, cores, sample = cpu_reference_rate(base, opts, args.cpu_reps, 1, budget=30.0)
        cpu = {"value": v, "unit": "matvec/s", "cores": cores, "kind": kind, "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == lib.MIXED else "f64",
        "data": "synthetic (seeded %s surface, %d seeded charges)" % (CASES[name][0], CASES[name][1]["n_charges"]),
        "config": {"workload": name, "panels": surf.n, "order": opts["order"], "depth": opts["depth"],
                   "sep_ratio": opts["sep_ratio"], "eps1": opts["eps1"], "eps2": opts["eps2"],
                   "precision": args.precision, "parallelism": "replicas" if world > 1 else "single",
                   "leaves": info["leaves"], "near_panel_pairs": info["near_panel_pairs"],
                   "m2l_pairs": info["m2l_pairs"], "special_pairs": info["special_pairs"],
                   "l2": "256 MiB buffer written between steps, outside the timed intervals"},
        "e2e": {"value": e2e_rate * world, "unit": "matvec/s", "h2d_bytes_per_step": n2 * 8,
                "d2h_bytes_per_step": n2 * 8},
        "roofline": {"kernel": kname,
                     "bound": "fp32" if prec == lib.MIXED else "fp64", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src, "flop_per_pair": FLOP_PER_PAIR,
                     "pairs_per_launch": pairs, "launch_ms": near_s * 1000.0},
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
    ap.add_argument("--case", default="star204800", choices=sorted(CASES))
    ap.add_argument("--cpu-reps", type=int, default=2)
    ap.add_argument("--ref-budget", type=float, default=90.0,
                    help="seconds of timed reference matvecs at most (--impl reference)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="also time the reference's own CUDA backend (oracle/_ref/ref_harness_gpu, -g=1)")
    ap.add_argument("--no-solve", action="store_true", help="skip the mixed/FP64 solve report")
    ap.add_argument("--solve-reps", type=int, default=3, help="reported runs per precision (after one warm-up run)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward/backward gradient timing")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
