#!/usr/bin/env python3
"""Benchmark of the B200 extreme-point decoder (decodes/sec at bit-exact parity).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|stress|multi_restart|single_pass|block]
    python bench.py --workload feas|feas_plain|fsr|item_order     (kernel timings)

A step is one batched solve of the workload: every restart decoded on the
device (persistent decoder kernel + per-instance best-of selection). The
default workload is the batched one, the largest that fits one launch:
4096 seeded synthetic instances (587 x 233 x 220 cm container, 3-100 box
types, 30-370 items) with 256 restarts each (1.05 M decodes per step),
eps 0.3, theta 0.9, one pass each.

Reported: `value` = decodes/s with the instance tables resident on the device
(CUDA events on the library's stream, max over ranks); `e2e` = the same
through plp_solve from host objects (tables copied in, every restart's result
copied out, each step); `roofline` for the decoder kernel against INT32 issue
(the reference's full-scan work, and the instructions the kernel executes);
`cpu_baseline` = the reference's own g++ decoder (oracle/_ref/ref_harness,
compiled from the reference sources) on the host cores, over a seeded 1 % of
the workload's instances, with the reference CPython solver's recorded rate
on the same sample beside it; `plain_path` = this library's
one-launch-per-step path on the same GPU; `serving` = Poisson request streams
through the serving loop.

The kernel workloads (feas, feas_plain, fsr, item_order) time the standalone
kernel entry points on seeded inputs and print one JSON line each; they are
the commands the ncu summaries of those kernels were taken with.

Multi-GPU (torchrun): each rank decodes its own restarts (seeds offset by
rank), no data-path collective; scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import random
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
CPYTHON_RECORD = os.path.join(REPO, "profiles", "cpython_reference_{}_sample.txt")
KERNEL_WORKLOADS = ("feas", "feas_plain", "fsr", "item_order")
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


def read_profile_inputs(path: str = PROFILE_INPUTS) -> dict:
    """key = value lines of a committed profile summary (# starts a comment)."""
    out = {}
    if os.path.exists(path):
        for line in open(path):
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


class CpuSample:
    """The workload's CPU sample (plpb200.synth.cpu_sample: a seeded 1 % of
    its instances, the first restarts of each) written to instance files for
    the reference's g++ harness."""

    def __init__(self, name: str, insts_py, opts):
        idx, restarts = synth.cpu_sample(name)
        self.idx = [i for i in idx if i < len(insts_py)] or [0]
        self.restarts = restarts
        self.dir = tempfile.TemporaryDirectory()
        self.paths = []
        self.items = []
        for i in self.idx:
            p = os.path.join(self.dir.name, f"inst_{i}.txt")
            with open(p, "w") as f:
                f.write(insts_py[i].to_thpack())
            self.paths.append(p)
            self.items.append(insts_py[i].n_items)
        self.flags = ["--seed", str(opts.seed), "--eps", str(opts.eps)] + (
            ["--no-theta"] if math.isnan(opts.theta) else ["--theta", str(opts.theta)])

    def describe(self, restarts=None, n_inst=None) -> str:
        n = len(self.idx) if n_inst is None else n_inst
        r = self.restarts if restarts is None else restarts
        items = self.items[:n]
        return (f"{n} instances (a seeded 1 % of the workload's, {min(items)}-{max(items)} items) x restarts "
                f"0..{r - 1} = {n * r} decodes")

    def harness(self, threads: int, restarts=None, n_inst=None, repeat=1) -> dict:
        r = self.restarts if restarts is None else restarts
        paths = self.paths if n_inst is None else self.paths[:n_inst]
        cmd = [REF_HARNESS] + paths + ["--restarts", str(r), "--threads", str(threads),
                                       "--repeat", str(repeat)] + self.flags
        return json.loads(subprocess.run(cmd, capture_output=True, text=True, check=True).stdout)

    def close(self):
        self.dir.cleanup()


def cpu_baseline(sample: CpuSample, name: str, threads: int):
    """The reference's own g++ decoder on the host cores over the workload's
    CPU sample (all threads, and one thread on the first instances), with the
    reference CPython solver's recorded rate on the same sample beside it."""
    if not os.path.exists(REF_HARNESS):
        return None
    out = sample.harness(threads)
    cpu = {"value": out["decodes"] / out["seconds"], "unit": "decodes/s", "cores": out["threads"],
           "kind": "reference",
           "sample": sample.describe() + f", reference g++ build of gpu/plp_common.hpp on {out['threads']} "
                                         f"threads ({out['seconds']:.2f} s)"}
    n1 = min(len(sample.idx), 8)
    r1 = max(1, min(sample.restarts, 4))
    one = sample.harness(1, restarts=r1, n_inst=n1)
    cpu["single_core"] = {"value": one["decodes"] / one["seconds"], "unit": "decodes/s",
                          "sample": sample.describe(r1, n1) + ", 1 thread"}
    py = read_profile_inputs(CPYTHON_RECORD.format(name))
    if py:
        cpu["python"] = {
            "value": float(py["cpython_allcores_decodes_per_s"]), "unit": "decodes/s",
            "cores": int(py["cpython_allcores_cores"]), "kind": "reference",
            "single_core": float(py["cpython_1core_decodes_per_s"]),
            "sample": py["cpython_allcores_sample"] + "; 1 core: " + py["cpython_1core_sample"],
            "where": f"recorded in the build container ({py['host']}) by oracle/time_cpython.py: the "
                     "reference's CPython solver does not travel to the GPU host; the g++ build timed there "
                     f"ran at {py['gpp_allcores_decodes_per_s']} decodes/s on the same sample and cores",
            "source": os.path.relpath(CPYTHON_RECORD.format(name), REPO)}
    return cpu


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
    """--impl reference: the reference's g++ decoder (its gpu/plp_common.hpp,
    built from its sources as oracle/_ref/ref_harness) on all host threads,
    each step one pass over the workload's CPU sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in KERNEL_WORKLOADS or args.workload == "block":
        print(json.dumps({"impl": "reference", "unavailable": f"no reference decoder arm for {args.workload}"}))
        return 0
    insts, opts, desc, R = workload(args.workload, 0)
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_HARNESS):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
        return 0
    sample = CpuSample(args.workload, insts, opts)
    for _ in range(args.warmup):
        sample.harness(threads)
    secs, decodes = [], 0
    for _ in range(args.steps):
        out = sample.harness(threads)
        secs.append(out["seconds"])
        decodes += out["decodes"]
    total = sum(secs)
    value = decodes / total
    line = {
        "impl": "reference", "metric": "decodes/sec", "value": value, "unit": "decodes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32+f64", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "sample_decodes_per_step": decodes // args.steps},
        "cpu_baseline": {"value": value, "unit": "decodes/s", "cores": threads, "kind": "reference",
                         "sample": sample.describe() + f" per step, reference g++ (gpu/plp_common.hpp) on "
                                                       f"{threads} threads"},
        "e2e": {"value": value, "unit": "decodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    sample.close()
    print(json.dumps(line))
    return 0


def _serve_stream(device: int, rate: float, duration_s: float, max_requests: int, seed: int, keep=0):
    """One Poisson stream of pallet-solve requests through the handle's
    serving loop: arrivals at `rate`, batched-workload sizes, restarts drawn
    from {64, 256, 1024}. Latency runs from submit to the result's arrival on
    the host. Returns the figures and the first `keep` (instance, opts,
    result) triples."""
    n = int(min(max_requests, max(20, rate * duration_s)))
    stream = synth.serving_stream(n, float(rate), seed=seed)
    insts = [P.Instance.parse(i.to_thpack()) for _, i, _ in stream]
    opts = [P.make_opts(seed=k, restarts=r) for k, (_, _, r) in enumerate(stream)]
    kept = []
    with P.Handle(device=device) as h:
        h.solve([insts[0]], opts[0])                 # warm the pool and kernels
        warm = h.submit(insts[0], opts[0])           # and the serving launch
        h.wait(warm, 600000)
        h.take(warm)
        time.sleep(0.02)
        t0 = time.perf_counter()
        ids = []
        for (arrive, _, _), inst, o in zip(stream, insts, opts):
            delay = arrive - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(h.submit(inst, o))
        lat = []
        for k, rid in enumerate(ids):
            if h.wait(rid, 600000) != P.OK:
                raise SystemExit(f"serving request failed: {P.last_error()}")
            lat.append(h.times(rid)[1])
            res = h.take(rid)
            if k < keep:
                kept.append((stream[k][1], opts[k], res))
        span = time.perf_counter() - t0
        counters = h.serve_counters()
    lat.sort()
    q = lambda p: 1000 * lat[min(len(lat) - 1, int(p * len(lat)))]
    return {"rate_per_s": rate, "requests": n, "p50_ms": q(0.50), "p99_ms": q(0.99),
            "solves_per_s": n / span, "decodes_per_s": sum(o.restarts for o in opts) / span,
            "serving_launches": counters["launches"], "served_by_persistent_launch": counters["served"],
            "tile_overflow_reruns": counters["fallbacks"]}, kept


def _serve_parity(kept):
    """Served restarts against the reference g++ build (restarts 0 and the
    last of each kept request)."""
    if not os.path.exists(REF_HARNESS):
        return None
    ok = total = 0
    with tempfile.TemporaryDirectory() as td:
        for i, (inst, o, res) in enumerate(kept):
            path = os.path.join(td, f"r{i}.txt")
            with open(path, "w") as f:
                f.write(inst.to_thpack())
            for k in (0, o.restarts - 1):
                out = subprocess.run([REF_HARNESS, path, "--seed", str(o.seed + k), "--restarts", "1", "--json",
                                      "--eps", str(o.eps), "--theta", str(o.theta)],
                                     capture_output=True, text=True, check=True).stdout
                exp = json.loads(out.splitlines()[0])
                exp.pop("time_s")
                got = json.loads(res.json(k))
                got.pop("time_s")
                ok += got == exp
                total += 1
    return f"{ok}/{total} served restarts bit-identical to the reference g++ build"


def serving_report(device: int, rates=(100, 1000, 10000), sweep=(2000, 3000, 4000, 5000, 6000, 8000),
                   duration_s=1.5, max_requests=3000):
    """The serving workload: Poisson streams at 100, 1000 and 10000 requests/s
    through the persistent serving launch, then a sweep of rates for the
    highest one whose p99 stays under 50 ms while the solve rate keeps up with
    the arrivals; the same three streams on the wave path (PLP_SERVE=0)
    beside them; the plain one-launch-per-placement path's time per request;
    and served restarts against the reference g++ build."""
    out = {"persistent": [], "waves": [], "sweep": []}
    kept = []
    for rate in rates:
        r, k = _serve_stream(device, rate, duration_s, max_requests, seed=50000 + int(rate),
                             keep=4 if not kept else 0)
        kept += k
        out["persistent"].append(r)
    best = None
    for rate in sweep:
        r, _ = _serve_stream(device, rate, duration_s, max_requests, seed=51000 + int(rate))
        out["sweep"].append(r)
        if r["p99_ms"] < 50.0 and r["solves_per_s"] >= 0.95 * rate:
            best = rate
    out["sustained_rate_at_p99_50ms"] = best
    os.environ["PLP_SERVE"] = "0"
    try:
        for rate in rates:
            r, _ = _serve_stream(device, rate, duration_s, min(max_requests, 1000), seed=50000 + int(rate))
            out["waves"].append(r)
    finally:
        os.environ.pop("PLP_SERVE", None)
    # the plain path: one feasibility launch per placement; a request of R
    # restarts takes R decodes at the measured time per decode
    stream = synth.serving_stream(3, 100.0, seed=50100)
    per = []
    for _, inst_py, _ in stream:
        inst = P.Instance.parse(inst_py.to_thpack())
        P.run_plain(inst, seed=0, restarts=1)
        t = time.perf_counter()
        P.run_plain(inst, seed=0, restarts=2)
        per.append((time.perf_counter() - t) / 2)
    mean_r = (64 + 256 + 1024) / 3
    out["plain_path"] = {"ms_per_decode": 1000 * sum(per) / len(per),
                         "ms_per_request_mean_budget": 1000 * sum(per) / len(per) * mean_r,
                         "sample": "3 requests of the stream x 2 restarts each, plp_run_plain; a request's time "
                                   "is its restarts x the time per decode (mean budget 448 restarts)"}
    out["parity"] = _serve_parity(kept)
    return out


# ---------------------------------------------------------------------------
# kernel timings (--workload feas|feas_plain|fsr|item_order): the standalone
# kernel entry points on seeded inputs, best wall time of a few calls
# ---------------------------------------------------------------------------
def _best(fn, reps=5):
    fn()
    best = float("inf")
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t)
    return best


def feas_bench(n_cand=4096, n_boxes=512, seed=3):
    """One feasibility step of stress size: n_cand extreme points x 6
    orientations against n_boxes placed boxes stacked in a 587x233x220
    container (non-overlapping boxes on a grid of columns)."""
    rng = random.Random(seed)
    L, W, H = 587, 233, 220
    boxes = []
    cols = [(x, y) for x in range(0, L - 40, 41) for y in range(0, W - 40, 41)]
    rng.shuffle(cols)
    for i in range(n_boxes):
        x, y = cols[i % len(cols)]
        z = 11 * (i // len(cols))
        boxes.append((x, y, z, x + rng.randint(10, 40), y + rng.randint(10, 40), z + rng.randint(5, 11)))
    cand = sorted({(rng.randrange(L), rng.randrange(W), rng.randrange(H)) for _ in range(n_cand)},
                  key=lambda p: (p[2], p[1], p[0]))
    ors = [(37, 21, 15), (21, 37, 15), (37, 15, 21), (15, 37, 21), (21, 15, 37), (15, 21, 37)]
    t = _best(lambda: P.feas_check_all(cand, ors, boxes, L, W, H))
    return {"kernel": "feas_kernel", "entry": "plp_feas_check_all", "candidates": len(cand),
            "orientations": 6, "boxes": n_boxes, "ms_per_call": t * 1e3}


def feas_plain_bench(restarts=2):
    """The plain path on the multi_restart instance: one launch per item step."""
    inst = P.Instance.parse(synth.multi_restart(2).to_thpack())
    t = _best(lambda: P.run_plain(inst, seed=0, restarts=restarts), reps=2)
    return {"kernel": "feas_kernel", "entry": "plp_run_plain", "restarts": restarts,
            "ms_per_decode": t * 1e3 / restarts}


def fsr_bench(n_inst=64, restarts=64):
    """FSR of n_inst x restarts packings decoded from the batched workload."""
    insts = [P.Instance.parse(i.to_thpack()) for i in synth.batched_set(n_inst)]
    with P.Handle() as h:
        res = h.solve(insts, P.make_opts(seed=0, restarts=restarts))
    packs = [r.placements(k) for r in res for k in range(r.restarts)]
    t = _best(lambda: P.fsr_score(packs))
    return {"kernel": "fsr_kernel", "entry": "plp_fsr_score", "packings": len(packs),
            "boxes": int(sum(len(p) for p in packs)), "ms_per_call": t * 1e3}


def item_order_bench(n_inst=4096):
    """Item order (kernel d) of the batched workload's instances."""
    insts = [P.Instance.parse(i.to_thpack()) for i in synth.batched_set(n_inst)]
    t = _best(lambda: P.item_order(insts))
    return {"kernel": "item_order_kernel", "entry": "plp_item_order", "instances": n_inst,
            "items": int(sum(i.info()[2] for i in insts)), "ms_per_call": t * 1e3}


def kernel_bench(name: str) -> int:
    fn = {"feas": feas_bench, "feas_plain": feas_plain_bench, "fsr": fsr_bench,
          "item_order": item_order_bench}[name]
    print(json.dumps(fn()))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "stress", "multi_restart", "single_pass", "block"] + list(KERNEL_WORKLOADS))
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
    if args.workload in KERNEL_WORKLOADS:
        return kernel_bench(args.workload)
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
        # a sample of up to 1/8 of the workload (at least the tuner's default
        # 32768 decodes) keeps the estimates' spread below the tiles' gaps
        tile = h.autotune(insts, opts, max_decodes=max(32768, R * len(insts) // 8))

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
    distributions = {"placed_per_decode": [min(placed), sum(placed) / len(placed), max(placed)],
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
        if "sm_max_mhz" in peaks:
            sm_max, sm_src = float(peaks["sm_max_mhz"]), "sm_max_mhz of MEASURED_PEAKS.json"
        elif clk.get("sm_max_mhz"):
            sm_max, sm_src = float(clk["sm_max_mhz"]), "clocks.max.sm sampled by nvidia-smi in this run"
        else:
            sm_max, sm_src = 1965.0, "the B200's nominal clocks.max.sm (no clock record)"
        int_peak = props.multi_processor_count * 128 * sm_max * 1e6 / 1e12   # T int-op/s
        dec_mean_ms = sum(dec_ms) / len(dec_ms)
        decodes_per_launch = R * len(insts)
        achieved = t_mean * decodes_per_launch * INT_OPS_PER_AABB / (dec_mean_ms / 1000.0) / 1e12
        prof = read_profile_inputs()
        traffic = prof.get(f"traffic_bytes_per_launch.{args.workload}")
        if args.workload == "block":   # no reference work replay for the block engine
            achieved = None
        # the instructions the kernel really executes: thread instructions per
        # decode from the committed ncu capture of a smaller case of the same
        # workload, times this launch's decodes, over the decoder's own time
        executed = None
        tin = prof.get(f"thread_inst_per_decode.{args.workload}")
        if tin:
            ex = float(tin) * decodes_per_launch / (dec_mean_ms / 1000.0) / 1e12
            executed = {"achieved": ex, "peak": int_peak, "unit": "T thread-inst/s", "frac": ex / int_peak,
                        "thread_inst_per_decode": float(tin),
                        "source": prof.get(f"thread_inst_source.{args.workload}"),
                        "note": "every executed thread instruction (integer, FP64, memory, control) counted "
                                "against one instruction per INT32 lane per clock: the hardware's own "
                                "occupancy of the issue peak"}
        roofline = {
            "bound": "int32", "achieved": achieved, "peak": int_peak, "unit": "Tint-op/s",
            "frac": achieved / int_peak if achieved is not None else None,
            "frac_kind": "reference-work equivalent: the reference's full-scan AABB work per decode "
                         "delivered per second, over the INT32 issue peak (executed: the hardware's own "
                         "fraction)",
            "executed": executed,
            "traffic": float(traffic) if traffic else None,
            "peak_source": f"{props.multi_processor_count} SMs x 128 INT32 lanes x {sm_max:.0f} MHz ({sm_src})",
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
        if not args.no_cpu_baseline and args.workload != "block":
            sample = CpuSample(args.workload, insts_py, opts)
            cpu = cpu_baseline(sample, args.workload, os.cpu_count() or 1)
            sample.close()
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
                       "distributions": {**distributions, "note": "min, mean, max over the sampled decodes; pairs = "
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
