#!/usr/bin/env python3
"""Benchmark of the B200 extreme-point decoder (decodes/sec at bit-exact parity).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload multi_restart|batched|stress|single_pass]

A step is one batched solve of the workload: every restart decoded on the
device (persistent decoder kernel + per-instance best-of selection). The
default workload is the lockstep multi-restart case: one seeded synthetic
instance (587 x 233 x 220 cm container, 10 box types, edges U[25,115], flags
p=0.8, fill [1.0, 1.1]) with 1024 restarts (seeds 0..1023), eps 0.3,
theta 0.9, one pass each.

Reported: `value` = decodes/s with the instance tables resident on the device
(CUDA events on the library's stream, max over ranks); `e2e` = the same
through plp_solve from host objects (tables copied in, every restart's result
copied out, each step); `roofline` for the decoder kernel against INT32 issue;
`cpu_baseline` = the reference's own g++ decoder (oracle/_ref/ref_harness,
compiled from the reference sources) on the host cores; `plain_path` = this
library's one-launch-per-step path on the same GPU.

Multi-GPU (torchrun): each rank decodes its own restarts (seeds offset by
rank), no data-path collective; scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "plp-gpu_b200")
sys.path.insert(0, PKG)

import plpb200 as P  # noqa: E402
from plpb200 import synth  # noqa: E402

REF_HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")
REF_GPU = os.path.join(REPO, "oracle", "_ref", "plp_gpu_cuda")
GOLDEN = os.path.join(REPO, "tests", "golden", "decoder.jsonl")
PROFILE_INPUTS = os.path.join(REPO, "profiles", "roofline_inputs.txt")
INT_OPS_PER_AABB = 6   # x, y, z interval tests of one AABB comparison


def workload(name: str, rank: int):
    """(instances, opts, description). Seeds of rank r start at r * restarts."""
    if name == "multi_restart":
        insts = [synth.multi_restart(2)]
        R = 1024
        desc = "multi_restart: 1 instance, 10 types, 1024 restarts, eps 0.3, theta 0.9, 1 pass"
    elif name == "batched":
        insts = synth.batched_set(4096)
        R = 256
        desc = "batched: 4096 instances (3-100 types), 256 restarts each, eps 0.3, theta 0.9, 1 pass"
    elif name == "stress":
        insts = synth.stress_set(512)
        R = 4096
        desc = "stress: 512 instances x 100 types, 4096 restarts each, eps 0.3, theta 0.9, 1 pass"
    elif name == "block":
        insts = synth.batched_set(512)
        R = 64
        desc = ("block: block-building engine, 512 batched instances, 64 restarts each, amax 4 bmax 4 "
                "kmax 6 eps 0.5 topk 64 pick first, theta 0.9, 1 pass")
    elif name == "single_pass":
        insts = [synth.single_pass(1)]
        R = 1
        desc = "single_pass: 1 instance, 3 types, eps 0, no theta, seed 1"
    else:
        raise SystemExit(f"unknown workload {name}")
    kw = dict(eps=0.0, theta=None) if name == "single_pass" else dict(eps=0.3, theta=0.9)
    if name == "block":
        kw = dict(eps=0.5, theta=0.9, engine="block", amax=4, bmax=4, kmax=6, topk=64)
    seed = (1 if name == "single_pass" else 0) + rank * R
    opts = P.make_opts(seed=seed, restarts=R, **kw)
    return insts, opts, desc, R


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [v.strip() for v in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx.append(float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def read_profile_inputs() -> dict:
    out = {}
    if os.path.exists(PROFILE_INPUTS):
        for line in open(PROFILE_INPUTS):
            line = line.strip()
            if line and not line.startswith("#") and "=" in line:
                k, v = line.split("=", 1)
                out[k.strip()] = v.strip()
    return out


def measured_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def golden_parity(results, opts_seed: int, name: str):
    """Checks the bench's own restarts against the reference g++ goldens:
    multi_restart restarts 0..63, and restart 0 of a seeded 1 % sample of the
    batched / stress instances."""
    if opts_seed != 0 or not os.path.exists(GOLDEN):
        return None
    rows = [json.loads(l) for l in open(GOLDEN)]
    if name == "multi_restart":
        case = next((r for r in rows if r["case"] == "multi_restart"), None)
        pairs = [(results[0], k, exp) for k, exp in enumerate(case["expected"])
                 if k < results[0].restarts] if case else []
        what = "restarts"
    elif name in ("batched", "stress"):
        pairs = [(results[r["set_index"]], 0, r["expected"][0]) for r in rows
                 if r["case"] == f"{name}_1pct" and r["set_index"] < len(results)]
        what = "sampled instances (1 %, restart 0)"
    else:
        return None
    if not pairs:
        return None
    ok = 0
    for res, k, exp in pairs:
        got = json.loads(res.json(k))
        got.pop("time_s")
        ok += got == exp
    return f"{ok}/{len(pairs)} {what} bit-identical to the reference g++ build"


def cpu_baseline(insts, opts, R, threads):
    """The reference's own g++ decoder on the host cores (bounded sample)."""
    if not os.path.exists(REF_HARNESS):
        return None
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(insts[0].to_thpack())
        path = f.name
    sample = min(R, 1024)
    flags = ["--eps", str(opts.eps)] + (["--no-theta"] if math.isnan(opts.theta) else ["--theta", str(opts.theta)])
    cmd = [REF_HARNESS, path, "--seed", str(opts.seed), "--restarts", str(sample), "--threads", str(threads),
           "--repeat", "4"] + flags
    out = json.loads(subprocess.run(cmd, capture_output=True, text=True, check=True).stdout)
    os.unlink(path)
    return out["decodes"] / out["seconds"], out, sample


def reference_gpu(inst_py, opts):
    """The reference's own CUDA build (gpu/plp_gpu.cu for sm_100a, built
    under oracle/_ref) on the same instance: its --device K persistent kernel
    at its K = 16 cap (time_s of the run, context set-up excluded), and its
    plain one-launch-per-step path, as the rate difference of a 3 s and a
    one-pass run, which cancels the CUDA context start-up."""
    if not os.path.exists(REF_GPU):
        return None
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(inst_py.to_thpack())
        path = f.name
    flags = ["--eps", str(opts.eps)] + (["--no-theta"] if math.isnan(opts.theta) else ["--theta", str(opts.theta)])
    run = lambda extra: json.loads(subprocess.run([REF_GPU, path, "--json", "--seed", str(opts.seed)] + flags + extra,
                                                  capture_output=True, text=True, check=True, timeout=120).stdout)
    try:
        dev = run(["--single-pass", "--device", "16"])
        one = run(["--single-pass"])
        many = run(["--time", "3"])
    finally:
        os.unlink(path)
    plain = (many["n_passes"] - one["n_passes"]) / max(1e-9, many["time_s"] - one["time_s"])
    return {"device_k16_decodes_per_s": 16 / dev["time_s"], "device_k16_ms_per_launch": 1000 * dev["time_s"],
            "plain_decodes_per_s": plain,
            "binary": "oracle/_ref/plp_gpu_cuda: the reference's gpu/plp_gpu.cu built for sm_100a"}


def run_reference(args):
    """--impl reference: the reference's g++ decoder, all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    insts, opts, desc, R = workload(args.workload, 0)
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_HARNESS):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
        return 0
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(insts[0].to_thpack())
        path = f.name
    sample = min(R, 1024)
    flags = ["--eps", str(opts.eps)] + (["--no-theta"] if math.isnan(opts.theta) else ["--theta", str(opts.theta)])
    cmd = [REF_HARNESS, path, "--seed", str(opts.seed), "--restarts", str(sample), "--threads", str(threads)] + flags
    for _ in range(args.warmup):
        subprocess.run(cmd, capture_output=True, check=True)
    secs = []
    for _ in range(args.steps):
        out = json.loads(subprocess.run(cmd, capture_output=True, text=True, check=True).stdout)
        secs.append(out["seconds"])
    os.unlink(path)
    total = sum(secs)
    value = sample * args.steps / total
    line = {
        "impl": "reference", "metric": "decodes/sec", "value": value, "unit": "decodes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32+f64", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "sample_restarts_per_step": sample},
        "cpu_baseline": {"value": value, "unit": "decodes/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} restarts of the workload per step, reference g++ "
                                   f"(gpu/plp_common.hpp) on {threads} threads"},
        "e2e": {"value": value, "unit": "decodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def serving_report(device: int, rates=(100, 1000, 10000), window_s=2.0, max_requests=600):
    """Poisson streams of pallet-solve requests (batched-workload sizes,
    restarts drawn from {64, 256, 1024}) through the serving loop; p50/p99
    latency from submit to result, and the sustained solve rate. The plain
    comparison solves the same requests one at a time (one plp_solve each,
    no batching), back to back."""
    out = []
    for rate in rates:
        n = int(min(max_requests, max(20, rate * window_s)))
        stream = synth.serving_stream(n, float(rate), seed=50000 + rate)
        insts = [P.Instance.parse(i.to_thpack()) for _, i, _ in stream]
        opts = [P.make_opts(seed=k, restarts=r) for k, (_, _, r) in enumerate(stream)]
        with P.Handle(device=device) as h:
            h.solve([insts[0]], opts[0])                 # warm the pool and kernels
            t0 = time.perf_counter()
            ids = []
            for (arrive, _, _), inst, o in zip(stream, insts, opts):
                delay = arrive - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids.append(h.submit(inst, o))
            lat = []
            for rid in ids:
                if h.wait(rid, 600000) != P.OK:
                    raise SystemExit(f"serving request failed: {P.last_error()}")
                lat.append(h.times(rid)[1])
                h.take(rid)
            span = time.perf_counter() - t0
            # plain: the same requests solved one by one
            t1 = time.perf_counter()
            for inst, o in zip(insts[:min(n, 100)], opts[:min(n, 100)]):
                h.solve([inst], o)
            plain_per = (time.perf_counter() - t1) / min(n, 100)
        lat.sort()
        q = lambda p: 1000 * lat[min(len(lat) - 1, int(p * len(lat)))]
        out.append({"rate_per_s": rate, "requests": n, "p50_ms": q(0.50), "p99_ms": q(0.99),
                    "solves_per_s": n / span,
                    "decodes_per_s": sum(o.restarts for o in opts) / span,
                    "plain_solve_ms": 1000 * plain_per})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="multi_restart",
                    choices=["multi_restart", "batched", "stress", "single_pass", "block"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--instances", type=int, default=0,
                    help="profiling runs: only the workload's first N instances")
    ap.add_argument("--restarts", type=int, default=0,
                    help="profiling runs: R restarts per instance instead of the workload's")
    ap.add_argument("--tile", default=None,
                    help="P,C,G,D,M decoder tile instead of the autotuner's choice (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    insts_py, opts, desc, R = workload(args.workload, rank)
    if args.instances > 0 or args.restarts > 0:   # a smaller case of the same workload
        if args.instances > 0:
            insts_py = insts_py[:args.instances]
        if args.restarts > 0:
            R = args.restarts
            opts.restarts = R
            opts.seed = rank * R
        desc += f" [profiling case: {len(insts_py)} instances x {R} restarts]"
    insts = [P.Instance.parse(i.to_thpack()) for i in insts_py]
    n_items = [i.n_items for i in insts_py]
    h = P.Handle(device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    # ---- tile: the project's autotuner, on a sample of this workload ----
    if args.tile:
        tile = tuple(int(v) for v in args.tile.split(","))
        h.set_tile(*tile)
    else:
        tile = h.autotune(insts, opts)

    # ---- device-resident timing (value) ----
    batch = h.prepare(insts, opts)
    for _ in range(args.warmup):
        batch.run()
    graph = batch.graph          # later runs replay one captured CUDA graph
    warm_results = batch.fetch()
    parity = golden_parity(warm_results, opts.seed, args.workload)
    # algorithmic work of the reference per decode, replayed on the host from
    # the results of an evenly spaced sample of at most 512 restarts
    slots = [(r, k) for r in warm_results for k in range(r.restarts)]
    stride = max(1, len(slots) // 512)
    # (the block engine has no reference work replay: its roofline reports time only)
    sample = slots[::stride]
    work = [r.work(k) for r, k in sample] if args.workload != "block" else [(0, 0)]
    T = [w[0] for w in work]
    t_mean = sum(T) / len(T)
    placed = [r.summary(k).n_boxes for r, k in sample]
    pairs = [w[1] for w in work]
    dist = {"placed_per_decode": [min(placed), sum(placed) / len(placed), max(placed)],
            "pairs_per_decode": [min(pairs), sum(pairs) / len(pairs), max(pairs)],
            "sampled_decodes": len(sample)}
    del sample
    del slots, warm_results   # their pinned result block goes back to the handle's pool
    clocks = Clocks(local)

    def hold(seconds):
        """The same step, untimed, so that the 200 ms clock sampler sees the
        load of a timed region shorter than its period."""
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end:
            batch.run()

    barrier()
    clocks.start()
    hold(0.6)
    dev_ms, dec_ms, launches = [], [], 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        d, k, n = batch.run()
        dev_ms.append(d)
        dec_ms.append(k)
        launches += n
    barrier()
    hold(0.4)
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(dev_ms))
    decodes_per_step = R * len(insts) * world
    value = decodes_per_step * args.steps / (total_ms / 1000.0)
    h2d, d2h = batch.io_bytes()
    batch.close()

    # ---- end to end through plp_solve (host objects in, results out) ----
    res = None
    for _ in range(2):     # as the timed loop: the previous results stay alive during a solve
        res = h.solve(insts, opts)
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(e2e_steps):
        res = h.solve(insts, opts)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = decodes_per_step * e2e_steps / e2e_s

    out = None
    if rank == 0:
        peaks = measured_peaks()
        props = torch.cuda.get_device_properties(local)
        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        int_peak = props.multi_processor_count * 128 * sm_max * 1e6 / 1e12   # T int-op/s
        dec_mean_ms = sum(dec_ms) / len(dec_ms)
        achieved = t_mean * R * len(insts) * INT_OPS_PER_AABB / (dec_mean_ms / 1000.0) / 1e12
        prof = read_profile_inputs()
        traffic = prof.get(f"traffic_bytes_per_launch.{args.workload}")
        if args.workload == "block":   # no reference work replay for the block engine
            achieved = None
        roofline = {
            "bound": "int32", "achieved": achieved, "peak": int_peak, "unit": "Tint-op/s",
            "frac": achieved / int_peak if achieved is not None else None,
            "traffic": float(traffic) if traffic else None,
            "peak_source": f"{props.multi_processor_count} SMs x 128 INT32 lanes x {sm_max:.0f} MHz "
                           "(sm_max_mhz of MEASURED_PEAKS.json)",
            "work_unit": f"reference AABB tests per decode T = {t_mean:.0f} (mean over {len(T)} of the "
                         f"step's restarts, evenly spaced) x {INT_OPS_PER_AABB} int ops",
            "issue_active_pct_ncu": float(prof[f"issue_active_pct.{args.workload}"])
            if f"issue_active_pct.{args.workload}" in prof else None,
            "fp64_pipe_pct_ncu": float(prof[f"fp64_pipe_pct.{args.workload}"])
            if f"fp64_pipe_pct.{args.workload}" in prof else None,
            "note": "T counts the reference's full C1/C3 scans; the incremental decoder skips most of "
                    "them, so frac can exceed 1. issue_active_pct_ncu is the hardware's own measure.",
            "kernel": ("block_kernel" if args.workload == "block"
                       else "decoder1_kernel" if tile[2] == 1 else "decoder_kernel"),
            "kernel_ms_per_launch": dec_mean_ms,
        }
        cpu = None
        if not args.no_cpu_baseline:
            cb = cpu_baseline(insts_py, opts, R, os.cpu_count() or 1)
            if cb:
                v, raw, sample = cb
                cpu = {"value": v, "unit": "decodes/s", "cores": raw["threads"], "kind": "reference",
                       "sample": f"{sample} restarts x 4 repeats of the workload's first instance, reference "
                                 f"g++ build of gpu/plp_common.hpp, {raw['threads']} threads"}
                one = cpu_baseline(insts_py, opts, min(R, 128), 1)
                if one:
                    cpu["single_core"] = {"value": one[0], "unit": "decodes/s",
                                          "sample": f"{one[2]} restarts x 4 repeats, 1 thread"}
        plain = None
        if not args.no_plain:
            n_pl = 8
            o_pl = P.make_opts(seed=opts.seed, restarts=n_pl, eps=opts.eps,
                               theta=None if math.isnan(opts.theta) else opts.theta)
            P.run_plain(insts[0], **{"seed": opts.seed, "restarts": 1, "eps": opts.eps,
                                     "theta": None if math.isnan(opts.theta) else opts.theta})
            t1 = time.perf_counter()
            P.run_plain(insts[0], **{"seed": opts.seed, "restarts": n_pl, "eps": opts.eps,
                                     "theta": None if math.isnan(opts.theta) else opts.theta})
            pv = n_pl / (time.perf_counter() - t1)
            plain = {"value": pv, "unit": "decodes/s", "sample": f"{n_pl} restarts, one device "
                     "feasibility launch per item step (plp_run_plain)", "speedup_of_persistent": value / world / pv}
            del o_pl
        serving = None if args.no_serving else serving_report(local)
        ref_gpu = None
        if not args.no_reference_gpu and args.workload == "multi_restart":
            ref_gpu = reference_gpu(insts_py[0], opts)
        out = {
            "metric": "decodes/sec", "value": value, "unit": "decodes/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64",
            "data": "synthetic (seeded generator, 587x233x220 container)",
            "config": {"workload": desc, "instances": len(insts), "restarts": R,
                       "items_per_instance": [min(n_items), max(n_items)],
                       "distributions": {**dist, "note": "min, mean, max over the sampled decodes; pairs = "
                                                         "(extreme point, orientation) pairs the reference "
                                                         "evaluates per decode"},
                       "parallelism": f"dp{world} (restarts sharded by rank)",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "tile": dict(zip(("P", "C", "G", "D", "M"), tile)), "tile_source": "--tile" if args.tile else "plp_autotune",
                       "cuda_graph": graph},
            "parity": parity,
            "e2e": {"value": e2e_value, "unit": "decodes/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "plain_path": plain,
            "reference_gpu": ref_gpu,
            "serving": serving,
            "clocks": {**clk, "window": "nvidia-smi every 200 ms over the timed steps, plus 0.6 s before "
                                        "and 0.4 s after them of the same step, untimed"},
        }
        print(json.dumps(out))
    h.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
