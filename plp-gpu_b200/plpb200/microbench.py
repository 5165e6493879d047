"""Micro-benchmarks of the standalone kernel entry points.

    python -m plpb200.microbench feas        # check_all contract, one large step
    python -m plpb200.microbench feas_plain  # one launch per item step (plain path)
    python -m plpb200.microbench fsr         # FSR of 4096 packings
    python -m plpb200.microbench item_order  # item order of 4096 instances

Each prints one JSON line: the calls made, the best wall time per call and
the problem size. Inputs are the seeded synthetic workloads of plpb200.synth.
"""
from __future__ import annotations

import json
import random
import sys
import time

import numpy as np

from . import Handle, Instance, feas_check_all, fsr_score, item_order, make_opts, run_plain, synth


def _best(fn, reps=5):
    fn()
    best = float("inf")
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t)
    return best


def feas(n_cand=4096, n_boxes=512, seed=3):
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
    t = _best(lambda: feas_check_all(cand, ors, boxes, L, W, H))
    return {"kernel": "feas_kernel", "entry": "plp_feas_check_all", "candidates": len(cand),
            "orientations": 6, "boxes": n_boxes, "ms_per_call": t * 1e3}


def feas_plain(restarts=2):
    """The plain path on the multi_restart instance: one launch per item step."""
    inst = Instance.parse(synth.multi_restart(2).to_thpack())
    t = _best(lambda: run_plain(inst, seed=0, restarts=restarts), reps=2)
    return {"kernel": "feas_kernel", "entry": "plp_run_plain", "restarts": restarts,
            "ms_per_decode": t * 1e3 / restarts}


def fsr(n_inst=64, restarts=64):
    """FSR of n_inst x restarts packings decoded from the batched workload."""
    insts = [Instance.parse(i.to_thpack()) for i in synth.batched_set(n_inst)]
    with Handle() as h:
        res = h.solve(insts, make_opts(seed=0, restarts=restarts))
    packs = [r.placements(k) for r in res for k in range(r.restarts)]
    t = _best(lambda: fsr_score(packs))
    return {"kernel": "fsr_kernel", "entry": "plp_fsr_score", "packings": len(packs),
            "boxes": int(sum(len(p) for p in packs)), "ms_per_call": t * 1e3}


def item_order_bench(n_inst=4096):
    insts = [Instance.parse(i.to_thpack()) for i in synth.batched_set(n_inst)]
    t = _best(lambda: item_order(insts))
    return {"kernel": "item_order_kernel", "entry": "plp_item_order", "instances": n_inst,
            "items": int(sum(i.info()[2] for i in insts)), "ms_per_call": t * 1e3}


def main(argv):
    which = argv[1] if len(argv) > 1 else "feas"
    fn = {"feas": feas, "feas_plain": feas_plain, "fsr": fsr, "item_order": item_order_bench}.get(which)
    if fn is None:
        raise SystemExit(f"unknown benchmark {which}")
    print(json.dumps(fn()))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
