#!/usr/bin/env python
"""Throughput benchmark: shell-pair x RPP-centre tasks per second.

Workload (config 1): 64 atoms uniform in a 40-bohr cube (min separation 3 bohr,
seed 1), each with U_L (4 terms) + semilocal projectors l = 0..4 (3 terms) and
s..g shells of 8 primitives (exponents log-uniform [0.02, 5e3]). The full task
list is 320^2 ordered shell pairs x 64 centres = 6.55M tasks. A step is one
block of it: 32 bra shells x 32 ket shells x all 64 centres = 65536 tasks,
ordered by (la, lb); step s of rank r takes block pair (r + s*N) mod 100, so
ranks never repeat each other's work (weak scaling, no collective on the data
path; NCCL/gloo only for the start barrier and the max-over-ranks time).

Reported: value = tasks / device time of the engine's kernels with inputs
resident in HBM (CUDA events on the engine's stream, L2 flushed between
steps) for the learned batched form (the walk scheduled by the level model);
"plain" = the same steps with the plain level-by-level schedule, and
learned_over_plain their ratio (results are bit-identical); e2e = the same
tasks through the public batched C-ABI call with host inputs and outputs
(packing, host->device and device->host copies included; the outputs go to
page-locked host arrays allocated once through libgrpp_b200_host_alloc).
cpu_baseline and --impl reference time libgrpp itself (oracle/_ref, compiled
from its sources) on this host's cores: a class-stratified seeded sample of a
step's tasks, serially per (la, lb, lpot) class and on all cores, extrapolated to
the whole step by class counts. The default line also carries the gradient
workload (config3: d tr(D V)/dR of the config-2 system) and the uneven
multi-molecule batch (config4), each with learned vs plain, CUDA-event kernel
times and its roofline.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BLOCK = 32
WORKLOAD = ("config1: 64 atoms in a 40-bohr cube, s..g shells x 8 primitives, U_L + projectors l=0..4; "
            "step = 32 x 32 shell block x 64 centres = 65536 tasks")
METRIC = "shell-pair x RPP-centre tasks/s (full GRPP blocks, FP64)"


def get_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


_SYSTEM = None


def system():
    global _SYSTEM
    if _SYSTEM is None:
        from libgrpp_b200 import synthetic
        _SYSTEM = synthetic.config1()
    return _SYSTEM


def step_tasks(idx: int):
    """Tasks of block pair idx (of 100): 32 x 32 shells x 64 centres, ordered by (la, lb)."""
    S = system()
    nb = len(S.shells) // BLOCK
    ia, ib = (idx // nb) % nb, idx % nb
    sa = np.arange(ia * BLOCK, (ia + 1) * BLOCK)
    sb = np.arange(ib * BLOCK, (ib + 1) * BLOCK)
    a, b, c = np.meshgrid(sa, sb, np.arange(len(S.centres)), indexing="ij")
    a, b, c = a.ravel().astype(np.int32), b.ravel().astype(np.int32), c.ravel().astype(np.int32)
    La = np.array([s.L for s in S.shells])
    o = np.lexsort((c, b, a, La[b], La[a]))
    return a[o], b[o], c[o]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_rate(batch_fn, n_sample: int, threads: int, seed: int = 0):
    """libgrpp (oracle/_ref) on a seeded sample of a step's tasks: (tasks/s, sample description)."""
    from libgrpp_b200.capi import LibGRPP
    ref = LibGRPP(os.path.join(ROOT, "oracle", "_ref", "libgrpp_ref.so"))
    a, b, c = batch_fn()
    sel = np.sort(np.random.default_rng(seed).choice(len(a), n_sample, replace=False))
    batch = system().batch(a[sel], b[sel], c[sel])
    t0 = time.perf_counter()
    ref.driver_full_batch(batch, nthreads=threads)
    dt = time.perf_counter() - t0
    return n_sample / dt, dt


def task_classes(S, a, b, c):
    """(la, lb, lpot) class of every task: shell angular momenta and the centre's largest projector L."""
    La = np.array([s.L for s in S.shells])
    lpot = np.array([max([p.L for p in g.arep + g.so] + [0]) for g in S.grpps])
    cg = np.array([cc[1] for cc in S.centres])
    return (La[a] * 16 + La[b]) * 16 + lpot[cg[c]]


def cpu_reference_stratified(S, a, b, c, per_class: int, threads: int, seed: int = 0):
    """libgrpp (oracle/_ref, compiled from its sources) on a class-stratified sample of a task list:
    per_class seeded tasks of every (la, lb, lpot) class, run serially class by class (mean
    seconds per task of each class) and then all together on `threads` threads (parallel
    efficiency of the sample). The list's serial time is extrapolated as sum over classes of
    (tasks in the class) x (mean seconds per task of the class); the all-cores time as that
    over threads x efficiency. Returns the serial and all-cores tasks/s and a description."""
    from libgrpp_b200.capi import LibGRPP
    ref = LibGRPP(os.path.join(ROOT, "oracle", "_ref", "libgrpp_ref.so"))
    cls = task_classes(S, a, b, c)
    rng = np.random.default_rng(seed)
    keys, counts = np.unique(cls, return_counts=True)
    sel_all, serial_work, t_ser_sample = [], 0.0, 0.0
    for key, n in zip(keys, counts):
        idx = np.where(cls == key)[0]
        sel = np.sort(rng.choice(idx, min(per_class, len(idx)), replace=False))
        sel_all.append(sel)
        t0 = time.perf_counter()
        ref.driver_full_batch(S.batch(a[sel], b[sel], c[sel]), nthreads=1)
        dt = time.perf_counter() - t0
        t_ser_sample += dt
        serial_work += n * dt / len(sel)
    sel = np.sort(np.concatenate(sel_all))
    # parallel efficiency on the sample repeated to at least 8 tasks per thread (a step has
    # 65536: the all-cores run of a short sample would measure its load imbalance instead)
    reps = max(1, -(-8 * threads // len(sel)))
    rep = np.tile(sel, reps)
    t0 = time.perf_counter()
    ref.driver_full_batch(S.batch(a[rep], b[rep], c[rep]), nthreads=threads)
    t_par = time.perf_counter() - t0
    eff = reps * t_ser_sample / (threads * t_par)
    n = len(a)
    return {"serial": n / serial_work, "all_cores": n * threads * eff / serial_work, "efficiency": eff,
            "sample_tasks": int(len(sel)), "classes": int(len(keys)), "seconds": t_ser_sample + t_par,
            "parallel_copies": reps,
            "sample": f"{len(sel)} seeded tasks, {min(per_class, int(counts.min()))}..{per_class} of each of the "
                      f"{len(keys)} (la, lb, lpot) classes of the {n}-task step, serially per class, then "
                      f"{reps} copies of the sample on {threads} threads (efficiency {eff:.2f}); rates extrapolated "
                      f"by class counts"}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = host_threads()
    S = system()
    for w in range(args.warmup):
        cpu_reference_rate(lambda: step_tasks(w), max(8, threads), threads, seed=100 + w)
    serial, allc, secs, desc = [], [], [], ""
    for st in range(args.steps):
        a, b, c = step_tasks(st)
        r = cpu_reference_stratified(S, a, b, c, args.ref_per_class, threads, seed=st)
        serial.append(r["serial"])
        allc.append(r["all_cores"])
        secs.append(r["seconds"])
        desc = r["sample"]
    rate = len(allc) / sum(1.0 / x for x in allc)  # tasks/s over the steps' extrapolated times
    rate_serial = len(serial) / sum(1.0 / x for x in serial)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "tasks/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * 65536 / rate, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": rate, "unit": "tasks/s", "cores": threads, "kind": "reference", "sample": desc,
                         "serial": rate_serial, "measured_seconds": sum(secs)},
        "e2e": {"value": rate, "unit": "tasks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def rank_blocks(rank: int, world: int, steps: int, n_blocks: int = 100):
    """Block pairs (of the config-1 task list) that rank `rank` of `world` runs in its
    `steps` steps: r, r + N, r + 2N, ... mod n_blocks; ranks never share a block while
    steps * world <= n_blocks."""
    return [(rank + world * s) % n_blocks for s in range(steps)]


def reduce_time_and_work(dist, elapsed, work, device):
    """(max over ranks of elapsed, sum over ranks of work): the job's time is the slowest
    rank's, its work everyone's. dist is torch.distributed (None on one rank)."""
    if dist is None:
        return float(elapsed), float(work)
    import torch
    t = torch.tensor([elapsed, work], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(t[1])


def time_plans(plans, flush, local):
    """Execute each plan once (L2 flushed before each); per-kernel ms summed, counters summed."""
    import torch
    ms, kms = [], {"ms_type1": 0.0, "ms_screen": 0.0, "ms_walk": 0.0, "ms_predict": 0.0, "ms_assembly": 0.0}
    cnt, fallbacks = None, 0
    with ClockSampler(local) as clk:
        for p in plans:
            flush.fill_(1.0)
            torch.cuda.synchronize()
            p.execute()
            st = p.stats()
            ls = p.learned_stats()
            ms.append(st["ms_total"])
            kms["ms_type1"] += st["ms_type1"]
            kms["ms_screen"] += st["ms_screen"]
            kms["ms_predict"] += ls["ms_predict"]
            kms["ms_walk"] += st["ms_radial"] - st["ms_screen"] - ls["ms_predict"]
            kms["ms_assembly"] += st["ms_assembly"]
            fallbacks += ls["fallbacks"]
            c = p.counters()
            cnt = c if cnt is None else {k: cnt[k] + c[k] for k in c}
    torch.cuda.synchronize()
    return float(sum(ms)), kms, cnt, fallbacks, clk.summary()


def count_type1(plans, cnt, scale=1.0):
    """The type 1 kernel's operation counts, from one more, untimed execution of each plan (its
    counting build is slower); the radial counters of the timed runs are kept."""
    if not cnt:
        return
    for k in ("mmd_triples", "mmd_flops"):
        cnt[k] = 0
    for p in plans:
        p.set_counting(True)
        p.execute()
        mc = p.counters()
        p.set_counting(False)
        for k in ("mmd_triples", "mmd_flops"):
            cnt[k] += mc[k] * scale


def autotune_leg(lib, batches, mode, flush, local):
    """Per-class block size of the assembly kernel: one pass over the batches with 128 threads
    for every task (fixed), with the default rule, and with the autotuner's table (built on the
    same batches beforehand, its time reported); the table stays in force afterwards."""
    import torch
    res = {}

    def one_pass(threads):
        plans = [lib.plan(b, mode, assembly_threads=threads) for b in batches]
        plans[0].execute()
        torch.cuda.synchronize()
        tot, kms, _, _, _ = time_plans(plans, flush, local)
        for p in plans:
            p.close()
        return {"ms_per_step": tot, "ms_assembly": kms["ms_assembly"]}

    lib.autotune_reset()
    res["fixed_128"] = one_pass(128)
    res["default_rule"] = one_pass(0)
    t0 = time.perf_counter()
    table = {}
    for b in batches:
        table.update(lib.autotune_assembly(b, mode))
    res["tuning_seconds"] = time.perf_counter() - t0
    res["autotuned"] = one_pass(0)
    res["classes"] = len(table)
    res["choices"] = {str(s): sum(1 for v in table.values() if v[4] == s) for s in (128, 256, 512)}
    res["autotuned_over_fixed"] = res["fixed_128"]["ms_per_step"] / res["autotuned"]["ms_per_step"]
    res["assembly_autotuned_over_fixed"] = res["fixed_128"]["ms_assembly"] / res["autotuned"]["ms_assembly"]
    return res


def run_ours(args, rank, world, local):
    import torch
    from libgrpp_b200 import engine

    dist = None
    torch.cuda.set_device(local)  # before the process group, so NCCL binds this rank's GPU
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    lib = engine.load()
    lib.set_device(local)
    modes = {"plain": 0, "learned": 1}

    idxs = rank_blocks(rank, world, args.steps)
    S = system()
    batches = []
    for i in idxs:
        a, b, c = step_tasks(i)
        if args.tasks_per_step and args.tasks_per_step < len(a):
            sel = np.linspace(0, len(a) - 1, args.tasks_per_step).astype(np.int64)
            a, b, c = a[sel], b[sel], c[sel]
        batches.append(S.batch(a, b, c))
    n_tasks = [len(b.task_a) for b in batches]
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # the assembly kernel's block size per class: autotuned on this rank's batches (untimed
    # setup, like building the plans); fixed-size and default-rule passes are reported beside it
    tune = autotune_leg(lib, batches, {"plain": 0, "learned": 1}[args.mode], flush, local) if not args.no_autotune else None
    res = {}
    for name in ("plain", args.mode) if args.mode == "learned" else ("plain",):
        plans = [lib.plan(b, modes[name]) for b in batches]
        for w in range(args.warmup):
            plans[w % len(plans)].execute()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        total_ms, kms, cnt, fallbacks, clocks = time_plans(plans, flush, local)
        total_ms, tasks = reduce_time_and_work(dist, total_ms, float(sum(n_tasks)), "cuda")
        st0 = plans[0].stats()
        count_type1(plans, cnt)
        res[name] = {"value": tasks / (total_ms / 1e3), "ms_per_step": total_ms / len(plans),
                     "kernel_ms_per_step": {k: v / len(plans) for k, v in kms.items()},
                     "counters": {k: v / len(plans) for k, v in cnt.items()} if cnt else None,
                     "fallbacks_per_step": fallbacks / len(plans), "clocks": clocks,
                     "launches_per_step": (1 if st0["n_type1_items"] else 0) + 1
                                          + (2 if st0["n_radial"] else 0) + (2 if name == "learned" else 0),
                     "h2d": st0["h2d_bytes"]}
        for p in plans:
            p.close()
    main_mode = args.mode
    R = res[main_mode]

    # end to end through the public batched call (host in, host out): outputs land in
    # page-locked host arrays the caller allocated once (libgrpp_b200_host_alloc)
    e2e_batches = batches[: max(1, min(len(batches), args.e2e_steps))] if args.e2e_steps > 0 else batches
    n_out = max(int(b.block_offsets()[-1]) for b in e2e_batches)
    outs = [lib.pinned_empty(n_out) for _ in range(4)]
    lib.full_grpp_batch(e2e_batches[0], modes[main_mode], out=outs)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for b in e2e_batches:
        lib.full_grpp_batch(b, modes[main_mode], out=outs)
    e2e_s = time.perf_counter() - t0
    e2e_s, e2e_tasks = reduce_time_and_work(dist, e2e_s, float(sum(len(b.task_a) for b in e2e_batches)), "cuda")
    d2h = 4 * 8 * int(batches[0].block_offsets()[-1])

    line = {
        "metric": METRIC, "value": R["value"], "unit": "tasks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": R["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded config 1)",
        "config": {"workload": WORKLOAD, "tasks_per_step": n_tasks[0], "radial_mode": main_mode,
                   "l2": "flushed between steps (512 MiB write)", "parallelism": f"task blocks over {world} GPU(s)"},
        "kernel_ms_per_step": R["kernel_ms_per_step"],
        "gpu_launches": args.steps * R["launches_per_step"],
        "e2e": {"value": e2e_tasks / e2e_s, "unit": "tasks/s", "h2d_bytes_per_step": R["h2d"],
                "d2h_bytes_per_step": d2h},
        "clocks": R["clocks"],
    }
    if tune is not None:
        line["autotune"] = tune
    if main_mode == "learned":
        P = res["plain"]
        line["plain"] = {"value": P["value"], "ms_per_step": P["ms_per_step"],
                         "kernel_ms_per_step": P["kernel_ms_per_step"], "clocks": P["clocks"]}
        line["learned_over_plain"] = R["value"] / P["value"]
        line["learned_fallbacks_per_step"] = R["fallbacks_per_step"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        r = cpu_reference_stratified(S, *step_tasks(idxs[0]), args.ref_per_class, threads)
        line["cpu_baseline"] = {"value": r["all_cores"], "unit": "tasks/s", "cores": threads, "kind": "reference",
                                "sample": r["sample"], "serial": r["serial"], "serial_cores": 1,
                                "measured_seconds": r["seconds"]}
    peak = lib.fp64_peak()
    line["roofline"] = roofline(R["kernel_ms_per_step"], R["counters"], peak)
    line["roofline"]["traffic"] = TRAFFIC_PER_TASK.get(line["roofline"]["kernel"], 0.0) * n_tasks[0] or None
    if line["roofline"]["traffic"]:
        line["roofline"]["traffic_source"] = TRAFFIC_SOURCE
    if rank == 0 and world == 1 and not args.no_extra:
        # north_star's other workloads in the same run: the gradient (config 3) and the uneven batch (config 4)
        line["config3"], _ = gradient_leg(args, lib, local, flush, max(1, min(args.steps, 3)))
        line["config4"], _ = config4_leg(args, lib, local, flush, 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# DRAM bytes per task of the dominant kernel, from one ncu capture of it (dram__bytes_read.sum +
# dram__bytes_write.sum over the captured launch / its tasks); see profiles/
TRAFFIC_PER_TASK = {"ms_screen": (15.772672e6 + 14.599936e6) / 4096}
TRAFFIC_SOURCE = ("ncu --set full of radial_screen_unit_kernel (the screening of the long runs, about 85% of the "
                  "screening time) on 4096 tasks of the first config-1 step: 30.37 MB DRAM read+write, scaled to "
                  "the step's tasks (profiles/screen_unit_kernel_full_4096tasks.md)")

# FLOP model of the radial path (count of FP64 add/mul, FMA = 2, each exp/pow/sqrt/log/erf = 1,
# per operation of libgrpp's algorithm, libgrpp/radial_type2_integral.c and screening.c):
RADIAL_FLOPS = {
    "points": 15,      # Log3 abscissa and weight of one grid point
    "term_pts": 6,     # c r^(n-2) exp(-zeta r^2) for one potential term at one point
    "prim_pts": 6,     # c exp(-a (r-CA)^2) and k r for one primitive at one point
    "bessel": 18,      # 4th-order Taylor M_l(x) (16) and F += e M (2)
    "pow_pts": 1,      # r^N
    "accum": 5,        # S += w U F1 F2 r^N
    "scr_combos": 12,  # setup and contribution of one primitive screening estimate
    "scr_iters": 80,   # one fixed-point step: 4 M_l evaluations, 2 ratios, sqrt
    "scr_final": 57,   # the envelope: 2 M_l, exp, erf, pow, sqrt
}


SCREEN_KEYS = ("scr_combos", "scr_iters", "scr_final")


def kernel_flops(kernel, counters):
    """Algorithmic FP64 operations of one launch of a kernel, from its counters."""
    if kernel == "ms_type1":
        return float(counters.get("mmd_flops", 0))
    keys = SCREEN_KEYS if kernel == "ms_screen" else [k for k in RADIAL_FLOPS if k not in SCREEN_KEYS]
    return float(sum(RADIAL_FLOPS[k] * counters[k] for k in keys))


def roofline(kernel_ms, counters, peak_tflops):
    """FP64 roofline of the dominant kernel (and of the other counted kernels beside it).
    bound is "fp64": the GRPP path has no dense contraction and a task reads a few kB,
    so the FP64 pipe, not HBM or the tensor cores, bounds it."""
    dominant = max(("ms_type1", "ms_screen", "ms_walk", "ms_assembly"), key=kernel_ms.get)
    out = {"bound": "fp64", "kernel": dominant, "unit": "TFLOP/s", "peak": peak_tflops,
           "peak_source": "measured in this run (FP64 FMA microkernel, all SMs)", "traffic": None,
           "achieved": None, "frac": None}
    if counters is None:
        return out
    per = {}
    for k in ("ms_type1", "ms_screen", "ms_walk"):
        fl = kernel_flops(k, counters)
        ach = fl / (kernel_ms[k] * 1e-3) / 1e12 if kernel_ms[k] > 0 and fl > 0 else None
        per[k] = {"flops_per_launch": fl, "achieved": ach, "frac": ach / peak_tflops if ach and peak_tflops else None}
    if dominant in per:
        out.update(per[dominant])
    out["kernels"] = per
    out["counters"] = counters
    return out


def config4_tasks(n_mol):
    from libgrpp_b200 import synthetic
    M, (a, b, c) = synthetic.merge_systems(synthetic.config4()[:n_mol])
    return M, a, b, c


def config4_leg(args, lib, local, flush, steps):
    """Uneven batch: the first --molecules molecules of config 4 (2..24 atoms each, full GRPP,
    basis l <= 6, projectors l <= 5) as one class-sorted task list in chunks of 65536 tasks; a
    step is one pass over all chunks (CUDA events per kernel), learned and plain alike."""
    M, a, b, c = config4_tasks(args.molecules)
    chunks = [M.batch(a[i:i + 65536], b[i:i + 65536], c[i:i + 65536]) for i in range(0, len(a), 65536)]
    res, outs = {}, {}
    tune = autotune_leg(lib, chunks, 1, flush, local) if not args.no_autotune else None
    peak = lib.fp64_peak()
    for name, mode in (("plain", 0), ("learned", 1)):
        plans = [lib.plan(ch, mode) for ch in chunks]
        for p in plans[: max(1, args.warmup)]:
            p.execute()
        tot, kms, cnt, fb, clk = 0.0, None, None, 0, None
        for _ in range(steps):
            t, k, cn, f, clk = time_plans(plans, flush, local)
            tot += t
            fb += f
            kms = k if kms is None else {q: kms[q] + k[q] for q in k}
            cnt = cn if cnt is None else {q: cnt[q] + cn[q] for q in cn}
        outs[name] = [np.concatenate([p.outputs()[m] for p in plans]) for m in range(4)]
        kms = {q: v / steps for q, v in kms.items()}
        cnt = {q: v / steps for q, v in cnt.items()}
        count_type1(plans, cnt)
        res[name] = {"value": steps * len(a) / (tot / 1e3), "ms_per_step": tot / steps, "kernel_ms_per_step": kms,
                     "fallbacks_per_step": fb / steps, "clocks": clk,
                     "roofline": {k: v for k, v in roofline(kms, cnt, peak).items() if k not in ("counters",)}}
        for p in plans:
            p.close()
    max_err = max(float(np.max(np.abs(x - y))) for x, y in zip(outs["learned"], outs["plain"]))
    out = {"workload": f"config4: first {args.molecules} of 512 molecules (2..24 atoms, full GRPP, l <= 6), {len(a)} "
                       f"tasks sorted by (la, lb, lpot), {len(chunks)} chunks of 65536, L2 flushed before every chunk",
           "value": res["learned"]["value"], "unit": "tasks/s", "steps": steps, "learned": res["learned"],
           "plain": res["plain"], "learned_over_plain": res["learned"]["value"] / res["plain"]["value"],
           "learned_fallback_rate": res["learned"]["fallbacks_per_step"] / len(a),
           "max_abs_diff_learned_vs_plain": max_err}
    if tune is not None:
        out["autotune"] = tune
    return out, (M, a, b, c)


def gradient_leg(args, lib, local, flush, steps):
    """Density-contracted gradient d tr(D V)/dR (four matrices, all atoms) of the config-2 system
    (16 heavy atoms + 32 H, basis up to h, random symmetric D) over its first --tasks
    class-sorted tasks: wall clock of the host-in/host-out call (libgrpp_b200_grpp_gradient_contract,
    and its symmetric-density form with the shell pairs folded), and CUDA-event kernel times of
    the derivative blocks the call evaluates, for one chunk of 16384 tasks."""
    from libgrpp_b200 import gradient, synthetic
    S = synthetic.config2()
    D = synthetic.config3_density(S)
    a, b, c = synthetic.sort_tasks(S, *S.all_tasks())
    n = min(args.tasks, len(a))
    batch = S.batch(a[:n], b[:n], c[:n])
    e2e = {}
    for name, mode, sym in (("plain", 0, False), ("learned", 1, False), ("learned_folded", 1, True)):
        for _ in range(max(args.warmup, 1)):
            lib.grad_contract(S, batch, D, radial_mode=mode, symmetric=sym)
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            lib.grad_contract(S, batch, D, radial_mode=mode, symmetric=sym)
            times.append(time.perf_counter() - t0)
        e2e[name] = {"value": n / float(np.median(times)), "seconds_per_step": float(np.median(times))}
    nk = min(16384, n)
    dbatch, _ = gradient.derivative_batch(S.batch(a[:nk], b[:nk], c[:nk]), S.cart_order)
    kern = {}
    peak = lib.fp64_peak()
    for name, mode in (("plain", 0), ("learned", 1)):
        plan = lib.plan(dbatch, mode)
        for _ in range(max(args.warmup, 1)):
            plan.execute()
        tot, kms, cnt, clk = 0.0, None, None, None
        for _ in range(steps):
            t, k, cn, _, clk = time_plans([plan], flush, local)
            tot += t
            kms = k if kms is None else {q: kms[q] + k[q] for q in k}
            cnt = cn if cnt is None else {q: cnt[q] + cn[q] for q in cn}
        kms = {q: v / steps for q, v in kms.items()}
        cnt = {q: v / steps for q, v in cnt.items()}
        count_type1([plan], cnt)
        plan.close()
        kern[name] = {"tasks_per_s": nk / (tot / steps / 1e3), "derivative_blocks": len(dbatch.task_a),
                      "ms_per_chunk": tot / steps, "kernel_ms_per_chunk": kms, "clocks": clk,
                      "roofline": {k: v for k, v in roofline(kms, cnt, peak).items() if k not in ("counters",)}}
    return {"workload": f"config3: first {n} of {len(a)} class-sorted tasks of config 2 (d tr(D V)/dR, 4 matrices); "
                        f"e2e = host in / host out wall clock, kernels = CUDA events on {nk} tasks' derivative blocks",
            "value": e2e["learned"]["value"], "unit": "tasks/s", "steps": steps, "e2e": e2e,
            "folded_over_full": e2e["learned_folded"]["value"] / e2e["learned"]["value"],
            "kernels": kern, "learned_over_plain": kern["learned"]["tasks_per_s"] / kern["plain"]["tasks_per_s"]}, \
        (S, D, a[:n], b[:n], c[:n])


def run_config4(args, rank, world, local):
    import torch
    from libgrpp_b200 import engine
    if rank != 0:
        return
    torch.cuda.set_device(local)
    lib = engine.load()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    leg, (M, a, b, c) = config4_leg(args, lib, local, flush, args.steps)
    line = {"metric": METRIC, "value": leg["value"], "unit": "tasks/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": leg["learned"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded config 4)",
            "config": {"workload": leg["workload"]}, "clocks": leg["learned"]["clocks"], "config4": leg}
    if not args.no_cpu_baseline:
        r = cpu_reference_stratified(M, a, b, c, args.ref_per_class, host_threads())
        line["cpu_baseline"] = {"value": r["all_cores"], "unit": "tasks/s", "cores": host_threads(), "kind": "reference",
                                "sample": r["sample"], "serial": r["serial"]}
    print(json.dumps(line), flush=True)


def run_config3(args, rank, world, local):
    import torch
    from libgrpp_b200 import engine
    if rank != 0:
        return
    torch.cuda.set_device(local)
    lib = engine.load()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    leg, (S, D, a, b, c) = gradient_leg(args, lib, local, flush, args.steps)
    line = {"metric": "shell-pair x RPP-centre gradient tasks/s (d tr(D V)/dR, 4 matrices, FP64)",
            "value": leg["value"], "unit": "tasks/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1),
            "ms_per_step": 1e3 * leg["e2e"]["learned"]["seconds_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded config 2 system, D seed 3)",
            "config": {"workload": leg["workload"]}, "config3": leg}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = gradient_cpu_baseline(args, S, D, a, b, c)
    print(json.dumps(line), flush=True)


def gradient_cpu_baseline(args, S, D, a, b, c):
    """The oracle's restated libgrpp_full_grpp_integrals_gradient contracted with D (libgrpp's own
    gradient reads outside its L-1 block and can return NaN), all cores, on a seeded sample."""
    from libgrpp_b200.capi import LibGRPP
    ref = LibGRPP(os.path.join(ROOT, "oracle", "_build", "libgrpp_oracle.so"))
    ns = min(args.ref_sample, len(a))
    sel = np.sort(np.random.default_rng(0).choice(len(a), ns, replace=False))
    threads = host_threads()
    t0 = time.perf_counter()
    ref.driver_grad_contract(S, S.batch(a[sel], b[sel], c[sel]), D, nthreads=threads)
    dt = time.perf_counter() - t0
    return {"value": ns / dt, "unit": "tasks/s", "cores": threads, "kind": "port",
            "sample": f"{ns} seeded random tasks, the oracle's restated gradient per atom ({dt:.1f} s)"}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["plain", "learned"], default="learned",
                    help="headline radial mode; learned also times plain on the same steps")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps timed end to end; 0 = every timed step")
    ap.add_argument("--ref-sample", type=int, default=256, help="config3 CPU baseline: sampled tasks")
    ap.add_argument("--ref-per-class", type=int, default=6,
                    help="CPU baseline: seeded tasks per (la, lb, lpot) class of the stratified sample")
    ap.add_argument("--no-autotune", action="store_true", help="skip the assembly autotuner (default rule only)")
    ap.add_argument("--no-extra", action="store_true", help="leave the config3 / config4 legs out of the default line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tasks-per-step", type=int, default=0,
                    help="evenly spaced subset of each step's tasks (profiling runs); 0 = the full block")
    ap.add_argument("--workload", choices=["config1", "config3", "config4"], default="config1",
                    help="config1 (default, the headline), config3 (density-contracted gradient), "
                         "config4 (uneven multi-molecule batch)")
    ap.add_argument("--molecules", type=int, default=16, help="config4: molecules in the batch")
    ap.add_argument("--tasks", type=int, default=65536, help="config3: tasks differentiated")
    args = ap.parse_args()
    rank, world, local = get_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "config4":
        run_config4(args, rank, world, local)
    elif args.workload == "config3":
        run_config3(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
