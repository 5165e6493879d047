#!/usr/bin/env python3
"""Times the reference's CPython solver (plp/solver.py) on the CPU sample of a
bench workload -- measurement infrastructure, run where the reference tree is
mounted (it cannot travel to the GPU host, so the figures are recorded).

    python oracle/time_cpython.py [batched|stress|multi_restart] [--out FILE]

Reference tree: $PLP_REFERENCE (default /root/reference). One decode is
`plp.solver.run(inst, seed=k, time_limit_s=0, single_pass=True, eps=0.3,
theta=0.9)` (plp/solver.py:243-271), called in-process in a loop so no
process start-up is timed. Two figures, on the CPU sample of the workload
(plpb200.synth.cpu_sample: a seeded 1 % of its instances):

  * 1 core: restart 0 of every sampled instance, in this process;
  * all cores: restarts 0 .. 8 x cores - 1 of every sampled instance, spread
    over one spawned worker process per core, timed from the release of the
    workers to the last result.

Beside them it times the reference's g++ build (oracle/_ref/ref_harness) on
the same sample in the same container, so the CPython-to-g++ ratio is
measured on one machine. The output is key = value lines (bench.py reads the
`cpython_*` keys and prints them as cpu_baseline.python).
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import platform
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "plp-gpu_b200"))
from plpb200 import synth  # noqa: E402

REF = os.environ.get("PLP_REFERENCE", "/root/reference")
HARNESS = os.path.join(HERE, "_ref", "ref_harness")


def _instances(workload):
    idx, restarts = synth.cpu_sample(workload)
    if workload == "batched":
        return [synth.batched(30000 + i).to_thpack() for i in idx], restarts
    if workload == "stress":
        return [synth.stress(40000 + i).to_thpack() for i in idx], restarts
    return [synth.multi_restart(2).to_thpack()], restarts


def _decode_all(texts, seeds):
    sys.path.insert(0, REF)
    from plp.parser import parse
    from plp.solver import run
    insts = [parse(t)[0] for t in texts]
    n = 0
    for inst in insts:
        for k in seeds:
            run(inst, seed=k, time_limit_s=0, single_pass=True, eps=0.3, theta=0.9)
            n += 1
    return n


def _worker(texts, seeds, start, q):
    start.wait()
    t0 = time.perf_counter()
    n = _decode_all(texts, seeds)
    q.put((n, t0, time.perf_counter()))


def time_one_core(texts):
    _decode_all(texts[:1], [0])                      # imports and warm-up
    t0 = time.perf_counter()
    n = _decode_all(texts, [0])
    return n, time.perf_counter() - t0


def time_all_cores(texts, per_proc_restarts, procs):
    """Every process decodes all sampled instances at its own restart seeds."""
    ctx = mp.get_context("spawn")
    start, q = ctx.Event(), ctx.Queue()
    seeds = [list(range(p, per_proc_restarts * procs, procs)) for p in range(procs)]
    ws = [ctx.Process(target=_worker, args=(texts, s, start, q)) for s in seeds]
    for w in ws:
        w.start()
    time.sleep(2.0)                                   # let every worker import
    t_rel = time.perf_counter()
    start.set()
    outs = [q.get() for _ in ws]
    for w in ws:
        w.join()
    return sum(o[0] for o in outs), max(o[2] for o in outs) - t_rel


def time_gpp(texts, restarts, threads):
    paths = []
    with tempfile.TemporaryDirectory() as td:
        for i, t in enumerate(texts):
            p = os.path.join(td, f"i{i}.txt")
            open(p, "w").write(t)
            paths.append(p)
        out = subprocess.run([HARNESS] + paths + ["--restarts", str(restarts), "--threads", str(threads)],
                             capture_output=True, text=True, check=True).stdout
    d = json.loads(out)
    return d["decodes"], d["seconds"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="batched")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    texts, restarts = _instances(args.workload)
    procs = os.cpu_count() or 1
    per_proc = max(1, min(restarts, 8))
    n1, s1 = time_one_core(texts)
    nn, sn = time_all_cores(texts, per_proc, procs)
    g1 = time_gpp(texts, 1, 1)
    gn = time_gpp(texts, per_proc * procs, procs)
    lines = [
        "# reference CPython solver (plp/solver.py run, single pass, eps 0.3, theta 0.9) on the CPU",
        f"# sample of the {args.workload} workload: {len(texts)} instances; recorded by oracle/time_cpython.py",
        f"workload = {args.workload}",
        f"host = {platform.processor() or platform.machine()}, {procs} cores, Python {platform.python_version()}",
        f"cpython_1core_decodes_per_s = {n1 / s1:.3f}",
        f"cpython_1core_sample = restart 0 of each of the {len(texts)} sampled instances ({n1} decodes, {s1:.2f} s)",
        f"cpython_allcores_decodes_per_s = {nn / sn:.3f}",
        f"cpython_allcores_cores = {procs}",
        f"cpython_allcores_sample = restarts 0..{per_proc * procs - 1} of each sampled instance over {procs} "
        f"spawned processes ({nn} decodes, {sn:.2f} s)",
        f"gpp_1core_decodes_per_s = {g1[0] / g1[1]:.3f}",
        f"gpp_allcores_decodes_per_s = {gn[0] / gn[1]:.3f}",
        f"gpp_sample = the same instances and restarts, oracle/_ref/ref_harness (reference gpu/plp_common.hpp), "
        f"1 and {procs} threads",
    ]
    text = "\n".join(lines) + "\n"
    if args.out:
        open(args.out, "w").write(text)
    print(text, end="")


if __name__ == "__main__":
    main()
