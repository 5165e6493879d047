"""Seeded synthetic thpack instances for the five benchmark workloads.

The reference ships no generator, so the workloads are defined here:
every instance uses the 587 x 233 x 220 cm container of the BR family, box
edges are integers drawn uniformly, orientation flags are 0/1 draws, and
quantities grow from 1 per type until the total box volume reaches the
lower fill bound (the draw is repeated if it overshoots the upper bound).
All randomness comes from ``random.Random(seed)`` so every path (GPU,
oracle, reference CPU builds) sees byte-identical files.

Workloads (name -> what one unit of work is):
  single_pass   3 types, edges U[30,120], all flags 1, fill [0.95,1.10]
  multi_restart 10 types, edges U[25,115], flags p=0.8 (>=1 set), fill [1.0,1.1]
  batched       types round(exp U[ln 3, ln 100]), edges U[20,120], all flags 1,
                fill [1.0,1.1]
  stress        100 types, qty U{1..3}, edges U[15,120], flags p=0.7 (>=1 set)
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass

CONTAINER = (587, 233, 220)


@dataclass(frozen=True)
class BoxType:
    l: int
    lf: int
    w: int
    wf: int
    h: int
    hf: int
    qty: int

    @property
    def volume(self) -> int:
        return self.l * self.w * self.h


@dataclass(frozen=True)
class SynthInstance:
    L: int
    W: int
    H: int
    types: tuple
    seed: int

    @property
    def n_items(self) -> int:
        return sum(t.qty for t in self.types)

    def to_thpack(self) -> str:
        lines = ["1", f"1 {self.seed}", f"{self.L} {self.W} {self.H}", str(len(self.types))]
        for i, t in enumerate(self.types, 1):
            lines.append(f"{i} {t.l} {t.lf} {t.w} {t.wf} {t.h} {t.hf} {t.qty}")
        return "\n".join(lines) + "\n"


def _flags(rng: random.Random, p: float) -> tuple:
    if p >= 1.0:
        return (1, 1, 1)
    while True:
        f = tuple(1 if rng.random() < p else 0 for _ in range(3))
        if any(f):
            return f


def _fill(rng, n_types, lo, hi, p_flag, fill_lo, fill_hi, L, W, H, seed):
    cvol = L * W * H
    while True:
        dims = [(rng.randint(lo, hi), rng.randint(lo, hi), rng.randint(lo, hi))
                for _ in range(n_types)]
        flags = [_flags(rng, p_flag) for _ in range(n_types)]
        qty = [1] * n_types
        vol = sum(a * b * c for a, b, c in dims)
        while vol < fill_lo * cvol:
            t = rng.randrange(n_types)
            qty[t] += 1
            a, b, c = dims[t]
            vol += a * b * c
        if vol <= fill_hi * cvol:
            break
    types = tuple(BoxType(d[0], f[0], d[1], f[1], d[2], f[2], q)
                  for d, f, q in zip(dims, flags, qty))
    return SynthInstance(L, W, H, types, seed)


def single_pass(seed: int = 1) -> SynthInstance:
    rng = random.Random(seed)
    return _fill(rng, 3, 30, 120, 1.0, 0.95, 1.10, *CONTAINER, seed)


def multi_restart(seed: int = 2) -> SynthInstance:
    rng = random.Random(seed)
    return _fill(rng, 10, 25, 115, 0.8, 1.0, 1.1, *CONTAINER, seed)


def batched(seed: int) -> SynthInstance:
    rng = random.Random(seed)
    n = int(round(math.exp(rng.uniform(math.log(3), math.log(100)))))
    return _fill(rng, n, 20, 120, 1.0, 1.0, 1.1, *CONTAINER, seed)


def stress(seed: int) -> SynthInstance:
    rng = random.Random(seed)
    types = []
    for _ in range(100):
        l, w, h = rng.randint(15, 120), rng.randint(15, 120), rng.randint(15, 120)
        f = _flags(rng, 0.7)
        types.append(BoxType(l, f[0], w, f[1], h, f[2], rng.randint(1, 3)))
    return SynthInstance(*CONTAINER, tuple(types), seed)


def batched_set(n: int, base_seed: int = 30000) -> list:
    return [batched(base_seed + i) for i in range(n)]


def stress_set(n: int, base_seed: int = 40000) -> list:
    return [stress(base_seed + i) for i in range(n)]


def serving_stream(n_requests: int, rate_per_s: float, seed: int = 50000):
    """Poisson arrivals of batched-size requests: (arrival_s, instance, restarts)."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.expovariate(rate_per_s)
        out.append((t, batched(seed + 1 + i), rng.choice((64, 256, 1024))))
    return out


def cpu_sample(workload: str):
    """The bounded sample of a workload that the CPU baselines time: a seeded
    1 % of its instances (at least one) with the first restarts of each, so
    the sample keeps the workload's mix of sizes. Returns (indices into the
    workload's instance list, restarts per instance); restart seeds start at 0
    as in the workload. The same indices are the 1 % parity sample of the
    batched and stress workloads."""
    if workload == "batched":
        return sorted(random.Random(7).sample(range(4096), 41)), 32
    if workload == "stress":
        return sorted(random.Random(8).sample(range(512), 5)), 128
    if workload == "multi_restart":
        return [0], 1024
    if workload == "single_pass":
        return [0], 1
    raise ValueError(f"no CPU sample for workload {workload}")
