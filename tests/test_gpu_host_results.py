"""Host side of synchronous solves: the results of one plp_solve share a
pinned block from the handle's pool and read it in place. They must stay
valid after later solves and after the handle is gone, and the pageable
path (pool off) must give the same results.
"""
import os

import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth

pytestmark = pytest.mark.gpu


def _jsons(res):
    return [[O.strip_time(r.json(k)) for k in range(r.restarts)] for r in res]


def _insts(n, base):
    texts = [i.to_thpack() for i in synth.batched_set(n, base)]
    return texts, [P.Instance.parse(t) for t in texts]


def test_results_outlive_later_solves_and_the_handle():
    texts, insts = _insts(3, 37000)
    h = P.Handle()
    first = h.solve(insts, P.make_opts(seed=4, restarts=6))
    kept = [h.solve(insts, P.make_opts(seed=100 + s, restarts=6)) for s in range(12)]   # 12 live blocks
    h.close()
    for t, r in zip(texts, first):
        oi = O.OInstance(t)
        for k in range(6):
            js, _, _ = O.run(oi, seed=4 + k)
            assert O.strip_time(r.json(k)) == O.strip_time(js)
    for s, res in enumerate(kept):
        oi = O.OInstance(texts[s % 3])
        js, _, _ = O.run(oi, seed=100 + s + 2)
        assert O.strip_time(res[s % 3].json(2)) == O.strip_time(js)
    del first, kept   # blocks of a closed handle are freed with their last result


def test_pageable_results_match_pooled(monkeypatch):
    _, insts = _insts(4, 37100)
    opts = P.make_opts(seed=9, restarts=40)
    with P.Handle() as h:
        pooled = _jsons(h.solve(insts, opts))
    monkeypatch.setenv("PLP_PINNED_POOL_MB", "0")
    with P.Handle() as h:
        paged = _jsons(h.solve(insts, opts))
        again = _jsons(h.solve(insts, opts))
    assert paged == pooled == again


def test_batch_fetch_results_survive_rerun_and_close():
    """plp_batch_fetch results are a snapshot: a later run of the batch and
    its release leave them unchanged."""
    texts, insts = _insts(2, 37200)
    with P.Handle() as h:
        b = h.prepare(insts, P.make_opts(seed=1, restarts=16))
        b.run()
        snap = b.fetch()
        before = _jsons(snap)
        b.run()
        b.close()
    assert _jsons(snap) == before
    oi = O.OInstance(texts[0])
    js, _, _ = O.run(oi, seed=1 + 5)
    assert before[0][5] == O.strip_time(js)


def test_large_batch_build_matches_oracle():
    """300 instances take the threaded item-sequence build; per-instance
    options (volume or input order) stay with their instance."""
    texts = [i.to_thpack() for i in synth.batched_set(300, 38000)]
    insts = [P.Instance.parse(t) for t in texts]
    orders = ["volume" if n % 3 else "input" for n in range(300)]
    opts = [P.make_opts(seed=n, restarts=2, order=orders[n]) for n in range(300)]
    with P.Handle() as h:
        res = h.solve(insts, opts)
    for n in range(0, 300, 13):
        oi = O.OInstance(texts[n])
        for k in range(2):
            js, _, _ = O.run(oi, seed=n + k, order=orders[n])
            assert O.strip_time(res[n].json(k)) == O.strip_time(js), (n, k)
