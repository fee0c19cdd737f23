#!/usr/bin/env python
"""Benchmark of the radix-partitioned inner equi-join on B200.

Workload (one "step"): the 2^27 x 2^27 int32 join -- build keys a seeded
permutation of 0..2^27-1, probe keys 90 % uniform from the build keys and
10 % above them, generated on the device -- run once through the C ABI
(pj_inner_join), inputs resident in HBM.  Inputs (1 GiB of keys) are larger than L2, so no flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU join (inner_join_cpu,
compiled from the reference sources into oracle/_ref) on a bounded sample of
the same workload with every host thread.  Under torchrun only rank 0 runs it.

One JSON line on rank 0.  value = input tuples / s over all ranks (each rank
joins its own replica of the workload: weak scaling, no data-path
collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tuples/s & HBM-roofline %, 2^27x2^27 int32 join"
# kernels of one pj_inner_join: per side histogram, scan, scatter; then
# join_items, scan, items_expand, join, fix-up plan, fix-up move
LAUNCHES_PER_JOIN = 12
UNIT = "tuples/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["cfg2", "cfg3", "cfg4", "cfg5"], default="cfg2",
                    help="cfg2: 2^27 x 2^27 int32 uniform (the headline); cfg3: 2^26 x 2^28 int64, Zipf probe "
                         "keys; cfg4: learned against exact plans on a held-out sweep; cfg5: 512 int32 joins of "
                         "uneven sizes, batched against one after another")
    ap.add_argument("--sweep", type=int, default=60, help="cfg4: held-out workloads")
    ap.add_argument("--cfg4-max-log2-build", type=int, default=28)
    ap.add_argument("--cfg4-max-log2-probe", type=int, default=29)
    ap.add_argument("--batch", type=int, default=512, help="cfg5: joins in the batch")
    ap.add_argument("--batch-only", action="store_true",
                    help="cfg5: only the batch in its default configuration (for launch lists)")
    ap.add_argument("--zipf", type=float, default=1.0, help="cfg3: Zipf exponent of the probe keys")
    ap.add_argument("--log2-build", type=int, default=None)
    ap.add_argument("--log2-probe", type=int, default=None)
    ap.add_argument("--match-rate", type=float, default=0.9)
    ap.add_argument("--cpu-sample-log2", type=int, default=24,
                    help="build and probe rows of the bounded CPU sample (log2)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="cfg2: skip the cfg3/cfg4/cfg5 measurements added to the line (other_configs)")
    ap.add_argument("--no-ref-gpu", action="store_true", help="--impl reference: skip the reference's GPU path")
    ap.add_argument("--plan", type=str, default="", help="JSON overrides of pj_plan fields")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--default-plan", action="store_true", help="plan from sizes only (no histogram)")
    a = ap.parse_args()
    if a.log2_build is None:
        a.log2_build = 27 if a.workload == "cfg2" else 26
    if a.log2_probe is None:
        a.log2_probe = 27 if a.workload == "cfg2" else 28
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# inputs

def gen_config2_device(n_b, n_p, match_rate, seed, device):
    """Seeded cfg2-shaped inputs generated on the device by the library's
    own generator (pj_generate_tables): build = a seeded permutation of
    0..n_b-1, probe = a uniform build key with probability match_rate, else a
    key above n_b-1.  Returns (build, probe, matching probe rows)."""
    import torch
    from partitioned_join_b200 import api
    return api.generate_tables(n_b, n_p, torch.int32, n_b - 1, match_rate, True, 0.0, seed, device)


def cpu_sample(log2n, match_rate, seed):
    from partitioned_join_b200 import datagen
    n = 1 << log2n
    return datagen.config2(seed=seed, n_build=n, n_probe=n, match_rate=match_rate)


def workload_config(args, world):
    """The workload's description, shared by both arms' JSON lines."""
    if args.workload == "cfg2":
        w = (f"2^{args.log2_build}x2^{args.log2_probe} int32 inner join (cfg2): build = seeded permutation of "
             f"0..2^{args.log2_build}-1, probe {args.match_rate:.0%} uniform hits, the rest above the build keys")
    else:
        w = (f"2^{args.log2_build}x2^{args.log2_probe} int64 inner join (cfg3): unique random build keys, probe keys "
             f"Zipf({args.zipf}) over a seeded rank order")
    return {"workload": w, "build_rows": 1 << args.log2_build, "probe_rows": 1 << args.log2_probe,
            "unique_build_keys": True, "match_rate": args.match_rate if args.workload == "cfg2" else 1.0,
            "l2": "inputs (1 GiB or more) larger than L2, no flush", "parallelism": f"replicas x{world}"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def verify_pairs_device(build, probe, build_row, probe_row, n, expected):
    """Pair-level check of a unique-build-key join on the device: every
    output pair joins equal keys, both row ids are in range, no probe row
    appears twice, and the pair count equals the number of probe rows the
    generator made to match.  With unique build keys each matching probe row
    has exactly one partner, so these together make the output the same
    multiset as inner_join_cpu's (inner_join_cpu.hpp:24-107)."""
    import torch
    br = build_row[:n].long()
    pr = probe_row[:n].long()
    in_range = bool(((br >= 0) & (br < build.numel()) & (pr >= 0) & (pr < probe.numel())).all().item())
    keys_equal = in_range and bool((build[br] == probe[pr]).all().item())
    seen = torch.zeros(probe.numel(), dtype=torch.int32, device=probe.device)
    if in_range:
        seen.index_add_(0, pr, torch.ones_like(pr, dtype=torch.int32))
    distinct = in_range and int(seen.max().item() if n else 0) <= 1
    del seen, br, pr
    res = {"pairs_checked": int(n), "rows_in_range": in_range, "keys_equal": keys_equal,
           "probe_rows_distinct": distinct, "count_equals_generator": int(n) == int(expected)}
    res["ok"] = all(v for k, v in res.items() if k != "pairs_checked")
    return res


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi's start-up (driver queries) must not overlap the timed
        # region: wait for its first sample
        t_end = time.time() + 10
        while time.time() < t_end and self.proc.poll() is None and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# roofline helpers

def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel_tag):
    """DRAM bytes per launch of a kernel from a committed ncu summary
    (profiles/*.md line 'dram_bytes_per_launch[<tag>]: <bytes>'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    pat = re.compile(r"dram_bytes_per_launch\[" + re.escape(kernel_tag) + r"\]:\s*([0-9.eE+]+)")
    for name in sorted(os.listdir(pdir)):
        if not name.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, name)):
            m = pat.search(line)
            if m:
                return float(m.group(1))
    return None


# ---------------------------------------------------------------------------

def run_reference(args, rank, world):
    """The reference's own CPU join on a bounded sample of the workload."""
    if rank != 0:
        return
    from oracle import oracle
    b, p = cpu_sample(args.cpu_sample_log2, args.match_rate, args.seed)
    if oracle.ref_cpu_available():
        kind = "reference"
        threads = oracle.ref_cpu().ref_omp_max_threads()
        run = lambda: oracle.ref_inner_join_cpu(b, p, True)[1]  # noqa: E731
    else:
        kind = "port"
        threads = 1

        def run():
            t0 = time.perf_counter()
            oracle.inner_join(b, p, True)
            return time.perf_counter() - t0
    for _ in range(args.warmup):
        run()
    secs = [run() for _ in range(args.steps)]
    total = sum(secs)
    tuples = (b.shape[0] + p.shape[0]) * args.steps
    value = tuples / total
    sample = (f"2^{args.cpu_sample_log2} x 2^{args.cpu_sample_log2} rows of the same generator "
              f"(match rate {args.match_rate}); time = inner_join_cpu's own omp_get_wtime interval "
              f"(build + probe), unique-key path")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "ms_per_step_median": 1e3 * statistics.median(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": workload_config(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "cpu_model": cpu_model(),
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu(args)
    print(json.dumps(line), flush=True)


def reference_gpu(args):
    """The reference's own GPU path (main.cu:762-892), compiled unchanged for
    sm_100a into oracle/_ref, on the full workload: -R -n 256 -N 512 -u -V
    (two radix passes, the largest partition counts its 96 000-byte table
    cap admits at 2^27 rows, partitioned_join.cuh:198-206,324).  Its inputs
    are host columns from the numpy generator with the same recipe; the
    stage times are the reference's own cudaEvent timers around each stage
    (main.cu:769-896), copies and allocations excluded."""
    import numpy as np

    from oracle import oracle
    from partitioned_join_b200 import datagen
    if args.workload != "cfg2" or not oracle.ref_gpu_available(4):
        return {"unavailable": "reference GPU library not built (oracle/build_ref.sh) or workload not cfg2"}
    n_b, n_p = 1 << args.log2_build, 1 << args.log2_probe
    b, p = datagen.config2(seed=args.seed, n_build=n_b, n_probe=n_p, match_rate=args.match_rate)
    expected = int(np.count_nonzero(p <= n_b))
    p1, p2, factor = 256, 512, 3.0
    runs = []
    count_ok = True
    for k in range(4):
        keys, rows, ms = oracle.ref_gpu_partitioned_join(b, p, True, True, True, p1, p2, factor, False, capacity=n_p)
        count_ok &= keys.shape[0] == expected
        if k > 0:  # the first run is a warm-up
            runs.append([float(x) for x in ms])
    names = ["combined_histogram", "partition_pass1", "partition_pass2", "skew_handler", "join", "total"]
    med = {n: statistics.median(r[i] for r in runs) for i, n in enumerate(names)}
    return {"flags": f"-R -n {p1} -N {p2} -f {factor} -u -V", "build_rows": n_b, "probe_rows": n_p,
            "runs": len(runs), "stages_ms_median": med, "ms_per_join": med["total"],
            "tuples_per_s": (n_b + n_p) / (med["total"] / 1e3), "count_equals_generator": bool(count_ok),
            "timer": "the reference's own stage events (main.cu:769-896), median of 3 runs after 1 warm-up"}


def run_ours(args, rank, world, local, emit=True):
    import torch
    import torch.distributed as dist

    from partitioned_join_b200 import _lib, api, replicas

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1 and emit:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)

    n_b, n_p = 1 << args.log2_build, 1 << args.log2_probe
    seed = replicas.replica_seed(args.seed, rank)
    if args.workload == "cfg2":
        build, probe, expected = gen_config2_device(n_b, n_p, args.match_rate, seed, device)
    else:
        # unique random int64 build keys, every probe key a build key drawn by Zipf(args.zipf)
        build, probe, expected = api.generate_tables(n_b, n_p, torch.int64, (1 << 62) - 1, 1.0, True, args.zipf, seed,
                                                     device)
    kb = build.element_size()
    # Planning belongs to the timed step.  The size-only planner runs inside
    # every pj_inner_join call (a null plan); where the exact-histogram
    # planner (which reads the keys) would choose differently, its plan is
    # made once before the timed region and the line says so.
    plan_sizes = api.plan_default(n_b, n_p, kb, True)
    plan_hist = api.plan_exact(build, probe, True)
    same = plan_sizes.as_dict() == plan_hist.as_dict()
    plan = plan_sizes if (same or args.default_plan) else plan_hist
    if args.plan:
        for k, v in json.loads(args.plan).items():
            setattr(plan, k, v)
    per_call = (same or args.default_plan) and not args.plan
    j = api.Joiner(build, probe, True, plan, capacity=n_p, plan_per_call=per_call)
    plan_note = ("pj_plan_default inside every timed pj_inner_join call (a null plan); it equals "
                 "pj_plan_exact's plan for these inputs" if per_call and same else
                 "pj_plan_default inside every timed pj_inner_join call (a null plan)" if per_call else
                 "plan made once before the timed region (pj_plan_exact or --plan)")
    stream = torch.cuda.current_stream()

    # warm-up, then a pair-level check of the warm-up join's output
    for _ in range(max(args.warmup, 1)):
        j.launch()
    st = j.status()
    _lib.check(st, "warm-up join")
    got = int(j.count.item())
    verified = verify_pairs_device(build, probe, j.build_row, j.probe_row, got, expected)
    if not verified["ok"]:
        raise SystemExit(f"bench: join output failed the pair check: {verified} (expected {expected} pairs)")

    # timed region: K steps with per-stage events
    n_st = len(_lib.STAGES)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(n_st)] for _ in range(args.steps)]
    for row in ev:
        for e in row:
            e.record(stream)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    replicas.barrier()
    torch.cuda.synchronize()
    t0.record(stream)
    for k in range(args.steps):
        j.launch_with_events(ev[k])
    t1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier()
    clk = clocks.stop()
    _lib.check(j.status(), "timed joins")
    ms = replicas.max_over_ranks(t0.elapsed_time(t1), device)
    stage_ms = {name: 0.0 for name in _lib.STAGES[:-1]}
    for row in ev:
        for i, name in enumerate(_lib.STAGES[:-1]):
            stage_ms[name] += row[i].elapsed_time(row[i + 1]) / args.steps
    step_ms = ms / args.steps
    step_median = replicas.max_over_ranks(statistics.median(row[0].elapsed_time(row[-1]) for row in ev), device)
    # the last timed join's output, checked pair by pair like the warm-up's
    verified_last = verify_pairs_device(build, probe, j.build_row, j.probe_row, int(j.count.item()), expected)
    if not verified_last["ok"]:
        raise SystemExit(f"bench: timed join output failed the pair check: {verified_last}")
    tuples_all = replicas.sum_over_ranks((n_b + n_p) * args.steps, device)
    value = replicas.whole_job_rate(tuples_all, ms)

    # roofline: the dominant kernel and the whole join
    peak, peak_kind = measured_peak_gbs()
    tb = 8 if kb == 4 else 16  # partitioned tuple bytes: {hash, row} or {key_lo, key_hi, hash, row}
    alg = {
        "build_hist": n_b * kb, "probe_hist": n_p * kb,
        "build_scatter": n_b * (kb + tb), "probe_scatter": n_p * (kb + tb),
        "join": (n_b + n_p) * tb + expected * 8,
    }
    dom = max(alg, key=lambda k: stage_ms[k])
    achieved = alg[dom] / (stage_ms[dom] / 1e3) / 1e9
    kernel_of = {"build_hist": "hist_keys_kernel", "probe_hist": "hist_keys_kernel",
                 "build_scatter": "scatter_keys_kernel", "probe_scatter": "scatter_keys_kernel",
                 "join": "join_kernel"}
    traffic = ncu_traffic(f"{kernel_of[dom]}:{dom}")
    b_alg = (n_b + n_p) * (kb + kb) + expected * 8        # (k+v) per input tuple + 8 per output pair
    b_keys = (n_b + n_p) * kb + expected * 8              # what the path must move at least
    join_gbs = b_alg / (step_ms / 1e3) / 1e9

    line = {
        "metric": METRIC if args.workload == "cfg2" else "tuples/s, 2^26x2^28 int64 Zipf join",
        "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32" if kb == 4 else "int64", "data": "synthetic",
        "config": workload_config(args, world),
        "inputs": "generated on the device by pj_generate_tables (seeded)",
        "output_pairs": expected,
        "plan": plan.as_dict(), "planning": plan_note,
        "ms_per_step_median": step_median,
        "clocks": clk,
        "gpu_launches": LAUNCHES_PER_JOIN * args.steps,
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "kernel": f"{kernel_of[dom]} ({dom})", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes_per_launch": alg[dom]},
        "roofline_join": {"algorithmic_bytes": b_alg, "achieved": join_gbs, "peak": peak, "unit": "GB/s",
                          "frac": join_gbs / peak, "frac_keys_only": (b_keys / (step_ms / 1e3) / 1e9) / peak},
        "verified": {"warmup_join": verified, "last_timed_join": verified_last},
    }

    if not args.no_e2e:
        line["e2e"] = e2e_measure(args, j, build, probe, stream)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args)
    if args.workload == "cfg2" and world == 1 and not args.no_extra:
        del j, build, probe
        torch.cuda.empty_cache()
        line["other_configs"] = other_configs(args, local)
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    if world > 1 and emit:
        dist.destroy_process_group()
    return line


def other_configs(args, local):
    """The other configurations, measured in the same run after the
    headline (outside its timed region) so that one bench line records
    them: cfg3 (2^26 x 2^28 int64, Zipf 0 and 1.5), cfg5 (the 512-join
    batch against the same joins one after another with default and with
    per-join autotuned plans) and a short cfg4 sweep (16 held-out joins of
    2^18..2^26 build rows, learned against exact plans)."""
    import argparse as _ap
    import torch

    out = {}
    for zipf in (0.0, 1.5):
        a = _ap.Namespace(**vars(args))
        a.workload, a.log2_build, a.log2_probe, a.zipf = "cfg3", 26, 28, zipf
        a.steps, a.warmup, a.no_e2e, a.no_cpu, a.no_extra, a.plan = min(args.steps, 10), max(args.warmup, 3), True, True, True, ""
        ln = run_ours(a, 0, 1, local, emit=False)
        out[f"cfg3_zipf{zipf}"] = {"value": ln["value"], "unit": UNIT, "ms_per_step": ln["ms_per_step"],
                                   "ms_per_step_median": ln["ms_per_step_median"], "stages_ms": ln["stages_ms"],
                                   "plan": {k: ln["plan"][k] for k in ("passes", "bits1", "digit_mode", "table_mode",
                                                                         "n_heavy")},
                                   "roofline_join_frac": ln["roofline_join"]["frac"],
                                   "verified": ln["verified"]["last_timed_join"]["ok"] and
                                   ln["verified"]["warmup_join"]["ok"]}
        torch.cuda.empty_cache()
    a = _ap.Namespace(**vars(args))
    a.workload, a.steps, a.warmup = "cfg5", 5, 3
    ln = run_batch(a, 0, 1, local, emit=False)
    out["cfg5"] = {"value": ln["value"], "unit": UNIT, "makespan_ms": ln["makespan_ms"],
                   "speedup_vs_plain": ln["speedup_vs_plain"], "speedup_vs_plain_autotuned": ln["speedup_vs_plain_autotuned"],
                   "joins_by_path": ln["joins_by_path"],
                   "verified": all(v["ok"] for v in ln["verified"].values())}
    torch.cuda.empty_cache()
    a = _ap.Namespace(**vars(args))
    a.workload, a.sweep, a.cfg4_max_log2_build, a.cfg4_max_log2_probe = "cfg4", 16, 26, 27
    ln = run_learned(a, 0, 1, local, emit=False)
    out["cfg4_short"] = {"value": ln["value"], "unit": "x", "workload": ln["config"]["workload"],
                         "fallback_rate": ln["fallback_rate"], "join_ms_total": ln["join_ms_total"]}
    return out


def e2e_measure(args, j, build, probe, stream):
    """Host buffers in, host pairs out, through the C ABI: every step copies
    its two key columns from pinned host memory to the device, joins them
    and copies the count and the pairs back.  Steps are pipelined over two
    sets of device buffers: step k+1's inputs go up while step k's pairs
    come down (PCIe is full duplex), and a step's join waits only for its
    own inputs and for its output buffer's previous copy-out."""
    import torch

    from partitioned_join_b200 import api

    cap = j.capacity
    js = [j, api.Joiner(build.clone(), probe.clone(), True, j.plan, capacity=cap, plan_per_call=j.plan_per_call)]
    hb = build.cpu().pin_memory()
    hp = probe.cpu().pin_memory()
    ob = [torch.empty(cap, dtype=torch.int32).pin_memory() for _ in range(2)]
    op = [torch.empty(cap, dtype=torch.int32).pin_memory() for _ in range(2)]
    cnt = [torch.empty(1, dtype=torch.int64).pin_memory() for _ in range(2)]
    s_in, s_out, s_comp = torch.cuda.Stream(), torch.cuda.Stream(), stream
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_join = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    h2d = hb.numel() * hb.element_size() + hp.numel() * hp.element_size()
    steps = max(2, min(args.steps, 8))

    def copy_in(k):
        b = k % 2
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_join[b])  # join k-2 has read these inputs
            js[b].build_keys.copy_(hb, non_blocking=True)
            js[b].probe_keys.copy_(hp, non_blocking=True)
            ev_in[b].record(s_in)

    def join(k):
        b = k % 2
        with torch.cuda.stream(s_comp):
            s_comp.wait_event(ev_in[b])
            s_comp.wait_event(ev_out[b])  # step k-2's pairs have been copied out
            js[b].launch(s_comp)
            cnt[b].copy_(js[b].count, non_blocking=True)
            ev_join[b].record(s_comp)

    def copy_out(k):
        b = k % 2
        ev_join[b].synchronize()
        n = min(int(cnt[b].item()), cap)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_join[b])
            ob[b][:n].copy_(js[b].build_row[:n], non_blocking=True)
            op[b][:n].copy_(js[b].probe_row[:n], non_blocking=True)
            ev_out[b].record(s_out)
        return 8 + 8 * n

    def run(n_steps):
        d2h = []
        copy_in(0)
        join(0)
        for k in range(n_steps):
            if k + 1 < n_steps:
                copy_in(k + 1)
            d2h.append(copy_out(k))
            if k + 1 < n_steps:
                join(k + 1)
        torch.cuda.synchronize()
        return d2h

    run(2)  # warm-up
    t0 = time.perf_counter()
    d2h = run(steps)
    secs = time.perf_counter() - t0
    for b in range(2):
        _lib_check_status(js[b])
    n_tuples = (j.desc.n_build + j.desc.n_probe) * steps
    return {"value": n_tuples / secs, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": int(sum(d2h) / len(d2h)), "steps": steps,
            "ms_per_step": 1e3 * secs / steps,
            "timer": "host wall clock from the first copy-in to the last copy-out, steps pipelined over two "
                     "buffer sets"}


def _lib_check_status(joiner):
    from partitioned_join_b200 import _lib
    _lib.check(joiner.status(), "end-to-end join")


def cpu_baseline(args):
    from oracle import oracle
    b, p = cpu_sample(args.cpu_sample_log2, args.match_rate, args.seed)
    if oracle.ref_cpu_available():
        _, secs = oracle.ref_inner_join_cpu(b, p, True)
        kind, cores = "reference", oracle.ref_cpu().ref_omp_max_threads()
    else:
        t0 = time.perf_counter()
        oracle.inner_join(b, p, True)
        secs, kind, cores = time.perf_counter() - t0, "port", 1
    return {"value": (b.shape[0] + p.shape[0]) / secs, "unit": UNIT, "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": f"2^{args.cpu_sample_log2} x 2^{args.cpu_sample_log2} rows of the cfg2 generator, "
                      f"inner_join_cpu's own timer (build + probe)"}


def run_batch(args, rank, world, local, emit=True):
    """cfg5: a batch of int32 joins, build sizes log-uniform in 2^10..2^20
    (unique keys), probe sizes 4x, 70 % uniform matches, every fourth join
    with Zipf(1.0) probe keys -- run one after another with the plain
    method (default plans, and per-join autotuned plans: the fastest of the
    default, the exact-histogram plan and one radix bit less or more), then
    as one batch (default, autotuned, autotuned in a CUDA graph).  value =
    batch input tuples/s of the fastest batched form."""
    import ctypes

    import numpy as np
    import torch

    from partitioned_join_b200 import _lib, api

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    rng = np.random.default_rng(args.seed + 1000003 * rank)
    pairs, expected = [], []
    for i in range(args.batch):
        nb = int(2 ** rng.uniform(10, 20))
        b, p, hits = api.generate_tables(nb, 4 * nb, torch.int32, nb - 1, 0.7, True, 1.0 if i % 4 == 3 else 0.0,
                                         args.seed * 7919 + i, device)
        pairs.append((b, p))
        expected.append(hits)
    tuples = sum(b.numel() + p.numel() for b, p in pairs)
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    # plain: pj_inner_join per join, default plan, one reused workspace
    descs = [api.make_desc(b, p, True) for b, p in pairs]
    plans = [api.plan_default(d.n_build, d.n_probe, 4, True) for d in descs]
    ws_bytes = max(api.workspace_size(d, pl) for d, pl in zip(descs, plans))
    ws = api.alloc_workspace(ws_bytes, device)
    outs, keep = [], []
    counts = torch.zeros(len(pairs), dtype=torch.int64, device=device)
    for i, (b, p) in enumerate(pairs):
        br = torch.empty(max(p.numel(), 1), dtype=torch.int32, device=device)
        pr = torch.empty_like(br)
        keep += [br, pr]
        o = _lib.Output()
        o.build_row, o.probe_row, o.capacity, o.count = br.data_ptr(), pr.data_ptr(), p.numel(), counts.data_ptr() + 8 * i
        outs.append(o)
    L = _lib.lib()

    def plain():
        for d, pl, o in zip(descs, plans, outs):
            _lib.check(L.pj_inner_join(ctypes.byref(d), ctypes.byref(pl), ctypes.byref(o),
                                       ctypes.c_void_p(ws.data_ptr()), ws_bytes, api._stream_ptr(None)))

    def verify_all(brs, prs, cnts):
        """Pair-level check of every join of the batch (verify_pairs_device)."""
        cnts = cnts.cpu().tolist()
        bad = [i for i, (b, p) in enumerate(pairs)
               if not verify_pairs_device(b, p, brs[i], prs[i], cnts[i], expected[i])["ok"]]
        return {"joins_checked": len(pairs), "pairs_checked": int(sum(cnts)), "failed_joins": bad[:8],
                "ok": not bad}

    if args.batch_only:
        bj = api.BatchJoiner(pairs)
        ms = timed(bj.launch, max(1, args.steps))
        bj.check()
        ok = verify_all(bj.build_row, bj.probe_row, bj.count)
        line = {"metric": "batch ms, default configuration (cfg5, batch only)", "value": ms, "unit": "ms",
                "higher_is_better": False, "config": {"workload": f"{args.batch} int32 joins (cfg5)"},
                "verified": ok}
        if emit and rank == 0:
            print(json.dumps(line), flush=True)
        return line

    steps = max(1, min(args.steps, 5))
    plain_ms = timed(plain, steps)
    _lib.check(L.pj_check(ctypes.c_void_p(ws.data_ptr()), None))
    plain_ok = verify_all(keep[0::2], keep[1::2], counts)

    # plain autotuned: every join alone with the fastest of its default plan,
    # the exact-histogram plan and the default radix width -1 / +1 bit
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def one_ms(d, pl, o, wsb, wsz):
        _lib.check(L.pj_inner_join(ctypes.byref(d), ctypes.byref(pl), ctypes.byref(o), ctypes.c_void_p(wsb), wsz,
                                   api._stream_ptr(None)))
        best = float("inf")
        for _ in range(2):
            e0.record(stream)
            L.pj_inner_join(ctypes.byref(d), ctypes.byref(pl), ctypes.byref(o), ctypes.c_void_p(wsb), wsz,
                            api._stream_ptr(None))
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    tuned_plans = []
    for (b, p), d, pl, o in zip(pairs, descs, plans, outs):
        cands = [pl, api.plan_exact(b, p, True)]
        for dlt in (-1, 1):
            q = _lib.Plan.from_buffer_copy(pl)
            q.bits1 = max(0, pl.bits1 + dlt)
            n = ctypes.c_size_t()
            if L.pj_workspace_size(ctypes.byref(d), ctypes.byref(q), ctypes.byref(n)) == _lib.OK:
                cands.append(q)
        sized = [(c, api.workspace_size(d, c)) for c in cands]
        tws = api.alloc_workspace(max(z for _, z in sized), device)
        times = [one_ms(d, c, o, tws.data_ptr(), tws.numel()) for c, _ in sized]
        tuned_plans.append(cands[int(np.argmin(times))])
        del tws
    tws_bytes = max(api.workspace_size(d, pl) for d, pl in zip(descs, tuned_plans))
    tws = api.alloc_workspace(tws_bytes, device)

    def plain_tuned():
        for d, pl, o in zip(descs, tuned_plans, outs):
            _lib.check(L.pj_inner_join(ctypes.byref(d), ctypes.byref(pl), ctypes.byref(o),
                                       ctypes.c_void_p(tws.data_ptr()), tws_bytes, api._stream_ptr(None)))

    plain_tuned_ms = timed(plain_tuned, steps)
    _lib.check(L.pj_check(ctypes.c_void_p(tws.data_ptr()), None))
    plain_tuned_ok = verify_all(keep[0::2], keep[1::2], counts)

    bj = api.BatchJoiner(pairs)
    default_cfg = bj.config.as_dict()
    batch_ms = timed(bj.launch, steps)
    bj.check()
    batch_ok = verify_all(bj.build_row, bj.probe_row, bj.count)
    tuned_ms_est = bj.autotune()
    tuned_ms = timed(bj.launch, steps)
    g = bj.graph()
    graph_ms = timed(g.replay, steps)
    bj.check()
    graph_ok = verify_all(bj.build_row, bj.probe_row, bj.count)
    best_ms = min(batch_ms, tuned_ms, graph_ms)
    line = {
        "metric": "tuples/s, 512-join uneven batch (cfg5)", "value": tuples / (best_ms / 1e3), "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": best_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"{args.batch} int32 joins, build log-uniform 2^10..2^20 unique, probe 4x, 70% "
                               f"matches, every fourth Zipf(1.0) (generated on the device)",
                   "input_tuples": tuples, "batch_default_config": default_cfg, "batch_tuned_config": bj.config.as_dict()},
        "makespan_ms": {"one_after_another_plain": plain_ms, "one_after_another_plain_autotuned": plain_tuned_ms,
                        "batch_default": batch_ms, "batch_autotuned": tuned_ms,
                        "batch_autotuned_graph": graph_ms, "autotuner_estimate": tuned_ms_est},
        "speedup_vs_plain": plain_ms / best_ms,
        "speedup_vs_plain_autotuned": plain_tuned_ms / best_ms,
        "joins_by_path": {"direct": int(sum(1 for b, _ in pairs if 0 < b.numel() <= bj.config.direct_max_build)),
                          "partitioned_together": int(sum(1 for b, _ in pairs if b.numel() > bj.config.direct_max_build))
                          if bj.config.large_batched else 0},
        "verified": {"plain": plain_ok, "plain_autotuned": plain_tuned_ok, "batch": batch_ok, "graph": graph_ok},
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def run_learned(args, rank, world, local, emit=True):
    """cfg4: the shipped planner weights against the exact-histogram planner
    on a held-out seeded sweep (build 2^18..2^28 log-uniform, probe/build 1,
    4 or 16 with the probe side capped at 2^29 rows, int32 or int64, Zipf
    0..1.5, match rate 0.1..1).  Per workload
    both plans are made and timed (join time, and planning time apart);
    value = geometric-mean speedup of the learned plans' joins, fallbacks
    (a learned plan that overflows, rerun with the exact plan) counted at
    their full cost."""
    import numpy as np
    import torch

    from partitioned_join_b200 import _lib, api, planner

    torch.cuda.set_device(local)
    params = planner.load_weights(device=torch.device("cuda", local))
    if params is None:
        raise SystemExit("no planner weights (partitioned_join_b200/planner_weights.npz)")
    rng = np.random.default_rng(args.seed + 424242)
    rows = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_join(b, p, plan):
        j = api.Joiner(b, p, True, plan)
        j.launch()
        st = j.status()
        best = float("inf")
        for _ in range(2):
            e0.record()
            j.launch()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best, st

    for i in range(args.sweep):
        b, p, meta = planner.sweep_workload(rng, args.cfg4_max_log2_build, args.cfg4_max_log2_probe)
        # planning times on a workspace allocated beforehand (the planners
        # themselves allocate nothing; the allocation is the caller's)
        pws = api.alloc_workspace(api.workspace_size(api.make_desc(b, p, True)), b.device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        exact = api.plan_exact(b, p, True, ws=pws)
        plan_exact_ms = 1e3 * (time.perf_counter() - t0)
        t0 = time.perf_counter()
        learned, _ = planner.plan_learned(b, p, True, params, ws=pws)
        plan_learned_ms = 1e3 * (time.perf_counter() - t0)
        del pws
        t_exact, st = time_join(b, p, exact)
        _lib.check(st, "exact plan")
        t_learned, st = time_join(b, p, learned)
        fallback = st != _lib.OK
        if fallback:
            t_learned += t_exact
        rows.append(dict(meta, t_exact=t_exact, t_learned=t_learned, fallback=fallback, plan_exact_ms=plan_exact_ms,
                         plan_learned_ms=plan_learned_ms))
        del b, p
    sp = np.array([r["t_exact"] / r["t_learned"] for r in rows])
    z = np.array([r["zipf"] for r in rows])
    geo = float(np.exp(np.log(sp).mean()))

    def geo_of(mask):
        return float(np.exp(np.log(sp[mask]).mean())) if mask.any() else None

    line = {
        "metric": "geomean speedup of learned over exact plans (cfg4 held-out sweep)", "value": geo, "unit": "x",
        "n_gpus": world, "steps": 2, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/int64", "data": "synthetic",
        "config": {"workload": f"{args.sweep} held-out joins: build 2^18..2^{args.cfg4_max_log2_build} log-uniform, "
                               f"probe/build 1/4/16 (at most 2^{args.cfg4_max_log2_probe}), int32 or int64, Zipf 0..1.5, "
                               "match 0.1..1 (generated on the device)"},
        "fallback_rate": float(np.mean([r["fallback"] for r in rows])),
        "speedup_by_zipf": {"uniform(<0.2)": geo_of(z < 0.2), "0.2-1.0": geo_of((z >= 0.2) & (z < 1.0)),
                            ">=1.0": geo_of(z >= 1.0)},
        "join_ms_total": {"exact": float(sum(r["t_exact"] for r in rows)),
                          "learned": float(sum(r["t_learned"] for r in rows))},
        "planning_ms_median": {"exact": float(np.median([r["plan_exact_ms"] for r in rows])),
                               "learned": float(np.median([r["plan_learned_ms"] for r in rows]))},
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "cfg5":
        run_batch(args, rank, world, local)
    elif args.workload == "cfg4":
        run_learned(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
