"""GPU parity of the persistent decoder (plp_solve) and the plain path
(plp_run_plain) against the reference g++ goldens and the CPU oracle.

Every restart's JSON (time_s excluded, as parity/compare_parity.py:30-31
does) must be identical.
"""
import hashlib
import json
import os

import pytest

import oracle_py as O
import plpb200 as P
from conftest import GOLDEN
from plpb200 import synth
from test_oracle_pins import _golden_cases, _instance_for, flags_to_kw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    h = P.Handle()
    yield h
    h.close()


def _opts(seed, restarts, passes, kw, best_only=False):
    return P.make_opts(seed=seed, restarts=restarts, passes=passes, eps=kw["eps"], theta=kw["theta"],
                       order=kw["order"], first_fit=kw["first_fit"], mu=kw["mu"], best_only=best_only)


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: f"{c['case']}-{c['instance']}")
def test_solve_matches_reference_goldens(handle, case):
    inst = P.Instance.parse(_instance_for(case))
    kw = flags_to_kw(case["flags"])
    res = handle.solve([inst], _opts(case["seeds"][0], len(case["seeds"]), case["passes"], kw))[0]
    for k, exp in enumerate(case["expected"]):
        assert O.strip_time(res.json(k)) == exp, (case["case"], k)


def test_solve_batched_uneven_matches_oracle(handle):
    insts = synth.batched_set(24, base_seed=31000) + synth.stress_set(2, base_seed=41000)
    ps = [P.Instance.parse(i.to_thpack()) for i in insts]
    res = handle.solve(ps, P.make_opts(seed=100, restarts=3))
    for i, r in zip(insts, res):
        oi = O.OInstance(i.to_thpack())
        for k in range(3):
            js, _, _ = O.run(oi, seed=100 + k)
            assert O.strip_time(r.json(k)) == O.strip_time(js)


def test_solve_many_restarts_and_best(handle):
    text = synth.multi_restart(2).to_thpack()
    inst = P.Instance.parse(text)
    r = handle.solve([inst], P.make_opts(seed=0, restarts=256))[0]
    oi = O.OInstance(text)
    summ = []
    for k in range(0, 256, 5):
        js, s, _ = O.run(oi, seed=k)
        assert O.strip_time(r.json(k)) == O.strip_time(js)
    for k in range(256):
        summ.append(r.summary(k))
    # best: accepted first, then (volume, n_boxes), earliest on ties
    key = lambda k: (not summ[k].fallback, summ[k].volume, summ[k].n_boxes, -k)
    best = max(range(256), key=key)
    assert r.best() == (best, summ[best].fallback)


def test_solve_tiny_tile_retries_give_same_results(handle):
    text = synth.stress(40003).to_thpack()
    inst = P.Instance.parse(text)
    h2 = P.Handle()
    h2.set_tile(P=16, C=32, G=1, D=4)
    r_small = h2.solve([inst], P.make_opts(seed=7, restarts=8))[0]
    h2.close()
    r_ref = handle.solve([inst], P.make_opts(seed=7, restarts=8))[0]
    oi = O.OInstance(text)
    for k in range(8):
        js, _, _ = O.run(oi, seed=7 + k)
        assert O.strip_time(r_small.json(k)) == O.strip_time(js) == O.strip_time(r_ref.json(k))


def test_solve_best_only(handle):
    text = synth.batched(30005).to_thpack()
    inst = P.Instance.parse(text)
    full = handle.solve([inst], P.make_opts(seed=3, restarts=16))[0]
    bo = handle.solve([inst], P.make_opts(seed=3, restarts=16, best_only=True))[0]
    b, _ = full.best()
    assert bo.best() == full.best()
    assert bo.json(b) == full.json(b).replace(str(full.summary(b).time_s), str(bo.summary(b).time_s)) or \
        O.strip_time(bo.json(b)) == O.strip_time(full.json(b))
    other = (b + 1) % 16
    with pytest.raises(P.PlpError):
        bo.json(other)


@pytest.mark.parametrize("kw", [dict(eps=0.0, theta=None), dict(eps=0.3, theta=0.9, order="input"),
                                dict(eps=0.7, theta=0.5, passes=2), dict(first_fit=True)])
def test_plain_path_matches_oracle(kw):
    text = synth.single_pass(1).to_thpack()
    inst = P.Instance.parse(text)
    passes = kw.pop("passes", 1)
    r = P.run_plain(inst, seed=4, restarts=2, passes=passes, **kw)
    oi = O.OInstance(text)
    for k in range(2):
        js, _, _ = O.run(oi, seed=4 + k, passes=passes, **kw)
        assert O.strip_time(r.json(k)) == O.strip_time(js)


CONFIGS = [(1, 1, 1), (1, 1, 12), (1, 1, 16), (1, 2, 1), (1, 4, 1), (1, 4, 4), (1, 8, 1), (1, 8, 2), (2, 1, 1), (2, 2, 1), (2, 2, 5), (2, 4, 1),
           (2, 4, 3), (4, 1, 1), (4, 1, 5), (4, 1, 6), (4, 2, 1), (4, 2, 3), (4, 4, 1), (8, 1, 1), (8, 1, 3),
           (8, 2, 1)]


@pytest.mark.parametrize("G,D,M", CONFIGS)
def test_every_tile_config_matches_oracle(G, D, M):
    """Warps per decoder and decoders per CTA change speed only."""
    texts = [synth.single_pass(1).to_thpack(), synth.stress(40002).to_thpack(),
             synth.batched(30009).to_thpack()]
    insts = [P.Instance.parse(t) for t in texts]
    with P.Handle() as h:
        h.set_tile(P=64, C=128, G=G, D=D, M=M)   # shallow: some restarts also take the retry path
        res = h.solve(insts, [P.make_opts(seed=0, restarts=4, eps=0.0, theta=None),
                              P.make_opts(seed=5, restarts=4), P.make_opts(seed=9, restarts=4, passes=2)])
    for t, r, (seed, kw) in zip(texts, res, [(0, dict(eps=0.0, theta=None)), (5, {}), (9, dict(passes=2))]):
        oi = O.OInstance(t)
        for k in range(4):
            js, _, _ = O.run(oi, seed=seed + k, **kw)
            assert O.strip_time(r.json(k)) == O.strip_time(js), (G, D, M, seed + k)


def test_reference_work_accounting_matches_oracle_counter(handle):
    """plp_result_work replays the reference candidate list: T equals the
    oracle's instrumented count of AABB tests (the roofline's unit)."""
    for make, seeds in ((lambda: synth.multi_restart(2), 6), (lambda: synth.stress(40006), 3),
                        (lambda: synth.single_pass(1), 2)):
        text = make().to_thpack()
        inst = P.Instance.parse(text)
        r = handle.solve([inst], P.make_opts(seed=11, restarts=seeds))[0]
        oi = O.OInstance(text)
        for k in range(seeds):
            _, _, _, st = O.run(oi, seed=11 + k, stats=True)
            assert r.work(k) == (st["aabb_full"], st["pairs"])


def test_graph_replay_gives_identical_results():
    inst = P.Instance.parse(synth.multi_restart(2).to_thpack())
    with P.Handle() as h:
        b = h.prepare([inst], P.make_opts(seed=3, restarts=96))
        assert not b.graph
        b.run()
        first = [O.strip_time(b.fetch()[0].json(k)) for k in range(96)]
        assert b.graph                      # the clean run was captured
        for _ in range(2):
            dm, km, nl = b.run()            # graph replays
            assert nl == 2 and dm >= km > 0
            again = [O.strip_time(b.fetch()[0].json(k)) for k in range(96)]
            assert again == first
        b.close()


def test_graph_replay_best_only_gather():
    insts = [P.Instance.parse(i.to_thpack()) for i in synth.batched_set(6, 31000)]
    with P.Handle() as h:
        direct = [r.json(r.best()[0]) for r in h.solve(insts, P.make_opts(seed=1, restarts=24))]
        b = h.prepare(insts, P.make_opts(seed=1, restarts=24, best_only=True))
        b.run()
        b.run()
        assert b.graph
        res = b.fetch()
        assert [O.strip_time(r.json(r.best()[0])) for r in res] == [O.strip_time(j) for j in direct]
        b.close()


def test_autotune_picks_a_supported_tile_and_keeps_results():
    insts = [P.Instance.parse(i.to_thpack()) for i in synth.batched_set(8, 32000)]
    opts = P.make_opts(seed=2, restarts=32)
    with P.Handle() as h:
        before = [[O.strip_time(r.json(k)) for k in range(r.restarts)] for r in h.solve(insts, opts)]
        tile = h.autotune(insts, opts, max_decodes=128)
        Pd, Cd, G, D, M = tile
        assert G == 1 and (G, D, M) in CONFIGS and Pd >= 32 and Cd % 32 == 0
        after = [[O.strip_time(r.json(k)) for k in range(r.restarts)] for r in h.solve(insts, opts)]
        assert after == before


def _jsons(res):
    return [O.strip_time(res.json(k)) for k in range(res.restarts)]


def test_time_budget_zero_runs_exactly_one_pass():
    inst = P.Instance.parse(synth.multi_restart(2).to_thpack())
    with P.Handle() as h:
        r = h.solve([inst], P.make_opts(seed=5, restarts=16, passes=0, time_limit_s=0.0))[0]
        one = h.solve([inst], P.make_opts(seed=5, restarts=16, passes=1))[0]
    assert all(r.summary(k).n_passes == 1 for k in range(16))
    assert _jsons(r) == _jsons(one)


def test_time_budget_matches_fixed_pass_count_and_oracle():
    text = synth.single_pass(1).to_thpack()
    inst = P.Instance.parse(text)
    with P.Handle() as h:
        r = h.solve([inst], P.make_opts(seed=7, restarts=6, passes=0, time_limit_s=0.01))[0]
        counts = [r.summary(k).n_passes for k in range(6)]
        assert min(counts) >= 2
        for k in range(6):
            f = h.solve([inst], P.make_opts(seed=7 + k, restarts=1, passes=counts[k]))[0]
            assert O.strip_time(r.json(k)) == O.strip_time(f.json(0))
    js, _, _ = O.run(O.OInstance(text), seed=7, passes=counts[0])
    assert O.strip_time(r.json(0)) == O.strip_time(js)


def test_time_budget_pass_cap_binds():
    inst = P.Instance.parse(synth.single_pass(1).to_thpack())
    with P.Handle() as h:
        r = h.solve([inst], P.make_opts(seed=1, restarts=8, passes=3, time_limit_s=30.0))[0]
        f = h.solve([inst], P.make_opts(seed=1, restarts=8, passes=3))[0]
    assert [r.summary(k).n_passes for k in range(8)] == [3] * 8
    assert _jsons(r) == _jsons(f)


def test_retry_stage_small_tile_matches_oracle():
    """A multi-wave batch (6400 restarts) at a tile too small for its larger
    restarts: the restarts that overflow run again on the device at a deeper
    tile in the same stream pass (and on the host beyond that). Results match
    the oracle on every run."""
    texts = [i.to_thpack() for i in synth.batched_set(40, 36000)]
    insts = [P.Instance.parse(t) for t in texts]
    with P.Handle() as h:
        h.set_tile(64, 128, 1, 1, 1)
        b = h.prepare(insts, P.make_opts(seed=5, restarts=160))
        runs = [b.run() for _ in range(3)]
        res = b.fetch()
        b.close()
    # decoder, retry list, retry decoder and selection at least
    assert runs[0][2] >= 4, runs
    for n, (t, r) in enumerate(zip(texts, res)):
        oi = O.OInstance(t)
        for k in range(n % 11, 160, 37):
            js, _, _ = O.run(oi, seed=5 + k)
            assert O.strip_time(r.json(k)) == O.strip_time(js), (n, k)


def test_multi_wave_batch_matches_oracle():
    """A batch larger than one wave of resident decoders (3000 restarts) runs
    with the contact areas in 16 bits; a stride sample against the oracle."""
    texts = [i.to_thpack() for i in synth.batched_set(60, 35000)]
    insts = [P.Instance.parse(t) for t in texts]
    with P.Handle() as h:
        res = h.solve(insts, P.make_opts(seed=20, restarts=50))
    for n, (t, r) in enumerate(zip(texts, res)):
        oi = O.OInstance(t)
        for k in range((n * 7) % 13, 50, 13):
            js, _, _ = O.run(oi, seed=20 + k)
            assert O.strip_time(r.json(k)) == O.strip_time(js), (n, k)


def test_multi_restart_every_one_of_1024_restarts_and_best_match_reference_host(handle):
    """The lockstep multi-restart workload in full (10 types, seeds 0..1023,
    eps 0.3, theta 0.9, one pass): every restart's JSON against the
    reference g++ build by digest, and the best packing over the 1024
    restarts under the reference's selection rule (gpu/plp_common.hpp:493-511)
    in full (tests/golden/multi_restart_1024.json)."""
    from parity_gate import row_digest
    g = json.load(open(os.path.join(GOLDEN, "multi_restart_1024.json")))
    text = synth.multi_restart(2).to_thpack()
    assert hashlib.sha256(text.encode()).hexdigest() == g["sha256"]
    r = handle.solve([P.Instance.parse(text)], P.make_opts(seed=0, restarts=1024))[0]
    got = [json.loads(r.json(k)) for k in range(1024)]
    bad = [k for k in range(1024) if row_digest(got[k]) != g["restarts"][k][0]]
    assert not bad, f"{len(bad)} restarts differ, first {bad[:8]}"
    best, fallback = r.best()
    assert (best, fallback) == (g["best"]["index"], g["best"]["fallback_over_restarts"])
    row = got[best]
    row.pop("time_s")
    assert row == g["best"]["row"]
    accepted = [e for e in g["restarts"] if e[3] >= 0.9] or g["restarts"]
    assert row["volume_cm3"] == max(e[1] for e in accepted)


# A 12-cube that fits once and a 9-cube that never fits in a 20-cube
# container: their items fail step after step with nothing placed in
# between, which the decoder skips (a repeat of a failed type meets the same
# states and draws no random number). The 4-cubes and bars after them must
# come out as the oracle places them.
REPEATED_FAILURES = ("1\n1 7\n20 20 20\n4\n1 12 1 12 1 12 1 6\n2 9 1 9 1 9 1 10\n"
                     "3 4 1 4 1 4 1 40\n4 13 1 2 1 2 1 3\n")


@pytest.mark.parametrize("passes", [1, 2])
def test_repeated_failures_of_a_type_match_oracle(handle, passes):
    inst = P.Instance.parse(REPEATED_FAILURES)
    oi = O.OInstance(REPEATED_FAILURES)
    res = handle.solve([inst], P.make_opts(seed=3, restarts=8, passes=passes, eps=0.5))[0]
    for k in range(8):
        js, _, _ = O.run(oi, seed=3 + k, passes=passes, eps=0.5)
        assert O.strip_time(res.json(k)) == O.strip_time(js), k


def test_repeated_failures_of_a_type_served_match_oracle():
    """The same instance through the serving launch (its main decoders share
    the decoder body)."""
    inst = P.Instance.parse(REPEATED_FAILURES)
    oi = O.OInstance(REPEATED_FAILURES)
    with P.Handle() as h:
        rid = h.submit(inst, P.make_opts(seed=11, restarts=16, eps=0.5))
        assert h.wait(rid, 600000) == P.OK
        res = h.take(rid)
    for k in range(16):
        js, _, _ = O.run(oi, seed=11 + k, eps=0.5)
        assert O.strip_time(res.json(k)) == O.strip_time(js), k
