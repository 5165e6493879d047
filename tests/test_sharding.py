"""Multi-rank sharding of restarts (CPU, gloo, world size 2).

Each rank decodes its block of restarts (here with the CPU oracle standing in
for the device solve, since this container has no GPU) and the gathered
summaries must equal a single-process run, with the same global best.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from plpb200 import synth
from plpb200.shard import best_restart, restart_range, solve_sharded


def test_restart_range_partitions_exactly():
    for total in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            blocks = [restart_range(total, world, r) for r in range(world)]
            assert sum(c for _, c in blocks) == total
            pos = 0
            for first, count in blocks:
                assert first == pos
                pos += count


def test_best_restart_rule():
    s = [dict(fallback=True, volume=10, n_boxes=1), dict(fallback=False, volume=5, n_boxes=1),
         dict(fallback=False, volume=5, n_boxes=2), dict(fallback=False, volume=5, n_boxes=2)]
    assert best_restart(s) == 2


def _oracle_solve(text):
    import oracle_py as O
    inst = O.OInstance(text)

    def solve(first, count):
        return [O.run(inst, seed=first + k)[1] for k in range(count)]
    return solve


def _worker(rank, world, port, text, total, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "plp-gpu_b200"))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    summ, best = solve_sharded(_oracle_solve(text), total, seed=100)
    out[rank] = (summ, best)
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gather_equals_single_process():
    text = synth.multi_restart(2).to_thpack()
    total = 9
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, _free_port(), text, total, out), nprocs=2, join=True)
    single = [dict(volume=s["volume"], n_boxes=s["n_boxes"], fallback=s["fallback"], score=s["score"])
              for s in _oracle_solve(text)(100, total)]
    for rank in (0, 1):
        summ, best = out[rank]
        assert summ == single
        assert best == best_restart(single)
