"""Serving loop: continuous batching of requests admitted by a device-memory
budget. Each request's result must be identical alone and in the mix (bit
for bit: every restart's JSON without time_s)."""
import random
import time

import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth

pytestmark = pytest.mark.gpu


def _requests(n, seed=5):
    rng = random.Random(seed)
    out = []
    for i in range(n):
        inst = synth.batched(60000 + i)
        out.append((inst.to_thpack(), P.make_opts(seed=rng.randrange(1000), restarts=rng.choice((4, 16, 64)),
                                                   eps=rng.choice((0.0, 0.3)))))
    return out


def _jsons(res):
    return [O.strip_time(res.json(k)) for k in range(res.restarts)]


def test_results_identical_alone_and_in_the_mix():
    reqs = _requests(24)
    insts = [P.Instance.parse(t) for t, _ in reqs]
    with P.Handle() as h:
        alone = [_jsons(h.solve([i], o)[0]) for i, (_, o) in zip(insts, reqs)]
        ids = []
        for i, (_, o) in zip(insts, reqs):
            ids.append(h.submit(i, o))
            time.sleep(0.0005)                      # staggered arrivals join running waves
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK, P.last_error()
        mixed = [_jsons(h.take(rid)) for rid in ids]
    assert mixed == alone


def test_small_budget_serialises_but_stays_exact():
    reqs = _requests(6, seed=9)
    insts = [P.Instance.parse(t) for t, _ in reqs]
    with P.Handle() as h:
        alone = [_jsons(h.solve([i], o)[0]) for i, (_, o) in zip(insts, reqs)]
    with P.Handle(budget_bytes=4 << 20) as h:      # about one request at a time
        ids = [h.submit(i, o) for i, (_, o) in zip(insts, reqs)]
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK
        assert [_jsons(h.take(rid)) for rid in ids] == alone


def test_over_budget_request_is_refused():
    inst = P.Instance.parse(synth.multi_restart(2).to_thpack())
    with P.Handle(budget_bytes=64 << 10) as h:
        with pytest.raises(P.PlpError) as e:
            h.submit(inst, P.make_opts(restarts=1024))
        assert e.value.status == P.E_BUDGET


def test_cancel_and_timeouts():
    reqs = _requests(12, seed=3)
    insts = [P.Instance.parse(t) for t, _ in reqs]
    with P.Handle(budget_bytes=2 << 20) as h:      # forces a queue
        ids = [h.submit(i, P.make_opts(seed=1, restarts=64)) for i in insts]
        h.cancel(ids[-1])
        statuses = [h.wait(rid, 120000) for rid in ids]
        assert statuses[-1] in (P.E_CANCELLED, P.OK)   # it may already have been running
        assert all(s == P.OK for s in statuses[:-1])
        q, t = h.times(ids[0])
        assert t >= q >= 0
        with pytest.raises(P.PlpError) as e:
            h.take(10 ** 9)
        assert e.value.status == P.E_NOT_FOUND
        assert h.poll(10 ** 9) == P.E_NOT_FOUND


def test_served_results_match_the_oracle_with_restart_budgets_64_256_1024():
    """Serving-loop requests of the batched workload's sizes with the
    serving workload's restart budgets {64, 256, 1024}, submitted while
    others run: sampled restarts of every request against the CPU oracle,
    and each request's best restart against the selection rule applied to
    its own restarts."""
    rng = random.Random(21)
    reqs = []
    for i, R in enumerate((64, 256, 1024, 256, 64, 1024)):
        text = synth.batched(61000 + 37 * i).to_thpack()
        reqs.append((text, P.Instance.parse(text), P.make_opts(seed=rng.randrange(100000), restarts=R)))
    with P.Handle() as h:
        ids = []
        for _, inst, o in reqs:
            ids.append(h.submit(inst, o))
            time.sleep(0.001)
        for rid in ids:
            assert h.wait(rid, 300000) == P.OK, P.last_error()
        results = [h.take(rid) for rid in ids]
    for (text, _, o), res in zip(reqs, results):
        oi = O.OInstance(text)
        R = o.restarts
        for k in sorted(set(range(0, R, max(1, R // 24))) | {R - 1}):
            js, _, _ = O.run(oi, seed=o.seed + k)
            assert O.strip_time(res.json(k)) == O.strip_time(js), (R, k)
        summ = res.summaries()
        key = lambda k: (not summ[k].fallback, summ[k].volume, summ[k].n_boxes, -k)
        assert res.best()[0] == max(range(R), key=key)


def _thpack(L, W, H, types):
    lines = ["1", "1 1", f"{L} {W} {H}", str(len(types))]
    for i, (l, lf, w, wf, h, hf, q) in enumerate(types, 1):
        lines.append(f"{i} {l} {lf} {w} {wf} {h} {hf} {q}")
    return "\n".join(lines) + "\n"


def _check_oracle(text, opts, res, stride=1):
    oi = O.OInstance(text)
    theta = None if opts.theta != opts.theta else opts.theta
    for k in range(0, opts.restarts, stride):
        js, _, _ = O.run(oi, seed=opts.seed + k, eps=opts.eps, theta=theta)
        assert O.strip_time(res.json(k)) == O.strip_time(js), k


def test_requests_join_one_persistent_launch():
    """Staggered requests are served by the persistent serving launch (not
    one launch each), and each result equals the synchronous solve's."""
    reqs = _requests(32, seed=12)
    insts = [P.Instance.parse(t) for t, _ in reqs]
    with P.Handle() as h:
        alone = [_jsons(h.solve([i], o)[0]) for i, (_, o) in zip(insts, reqs)]
        ids = []
        for i, (_, o) in zip(insts, reqs):
            ids.append(h.submit(i, o))
            time.sleep(0.0003)
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK, P.last_error()
        mixed = [_jsons(h.take(rid)) for rid in ids]
        c = h.serve_counters()
    assert mixed == alone
    assert c["served"] == 32 and c["fallbacks"] == 0 and c["waved"] == 0
    assert 1 <= c["launches"] <= 8


def test_launch_configuration_changes_drain_and_relaunch():
    """A container too tall for the running launch's top-z index, and
    footprints too large for its 16-bit contact areas, wait for the launch to
    drain and run in a relaunch with the merged configuration; every result
    equals the oracle's."""
    rng = random.Random(8)
    tall = _thpack(50, 40, 5000, [(rng.randint(8, 25), 1, rng.randint(8, 20), 1, rng.randint(20, 90), 1,
                                   rng.randint(20, 60)) for _ in range(4)])
    wide = _thpack(1000, 1000, 100, [(300, 1, 300, 1, 40, 1, 9), (250, 1, 180, 1, 30, 1, 14),
                                     (90, 1, 70, 1, 20, 1, 30)])
    texts = [synth.batched(62000).to_thpack(), tall, synth.batched(62001).to_thpack(), wide,
             synth.batched(62002).to_thpack()]
    opts = [P.make_opts(seed=10 * i, restarts=6) for i in range(len(texts))]
    with P.Handle() as h:
        ids = [h.submit(P.Instance.parse(t), o) for t, o in zip(texts, opts)]
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK, P.last_error()
        res = [h.take(rid) for rid in ids]
        c = h.serve_counters()
    for t, o, r in zip(texts, opts, res):
        _check_oracle(t, o, r)
    assert c["served"] == 5 and c["launches"] >= 2


def test_restarts_outgrowing_the_serving_tile_go_to_the_overflow_decoders():
    """300 small boxes all fit, so a decode places more boxes than the serving
    tile holds (256): its decoder hands the restart to the launch's overflow
    decoders (a 512-box tile in global memory) inside the same launch. The
    results equal the oracle's, and a normal request served beside it too."""
    text = _thpack(587, 233, 220, [(20, 1, 20, 1, 20, 1, 300)])
    normal = synth.batched(62010).to_thpack()
    o, on = P.make_opts(seed=3, restarts=3), P.make_opts(seed=9, restarts=16)
    with P.Handle() as h:
        rid = h.submit(P.Instance.parse(text), o)
        rn = h.submit(P.Instance.parse(normal), on)
        assert h.wait(rid, 300000) == P.OK, P.last_error()
        assert h.wait(rn, 300000) == P.OK, P.last_error()
        res, resn = h.take(rid), h.take(rn)
        c = h.serve_counters()
    assert c["fallbacks"] == 0 and c["served"] == 2
    assert res.summary(0).n_boxes > 256
    _check_oracle(text, o, res)
    _check_oracle(normal, on, resn, stride=3)


def test_restarts_outgrowing_the_overflow_tile_rerun_on_the_wave_path():
    """600 boxes outgrow the overflow decoders' 512-box tile as well: the
    request runs again through the wave path's code, with deeper tiles, and
    its results equal the oracle's."""
    text = _thpack(587, 233, 220, [(10, 1, 10, 1, 10, 1, 600)])
    o = P.make_opts(seed=5, restarts=2)
    with P.Handle() as h:
        rid = h.submit(P.Instance.parse(text), o)
        assert h.wait(rid, 300000) == P.OK, P.last_error()
        res = h.take(rid)
        c = h.serve_counters()
    assert c["fallbacks"] == 1
    assert res.summary(0).n_boxes > 512
    _check_oracle(text, o, res)


def test_wave_path_when_serving_is_off(monkeypatch):
    monkeypatch.setenv("PLP_SERVE", "0")
    reqs = _requests(6, seed=14)
    with P.Handle() as h:
        ids = [h.submit(P.Instance.parse(t), o) for t, o in reqs]
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK
        res = [h.take(rid) for rid in ids]
        assert h.serve_counters() == {"launches": 0, "served": 0, "fallbacks": 0, "waved": 0}
    for (t, o), r in zip(reqs, res):
        _check_oracle(t, o, r, stride=max(1, o.restarts // 4))


def test_solve_after_serving_on_the_same_handle():
    """The serving launch stops once idle, so a synchronous solve that
    follows on the same handle runs and is exact."""
    reqs = _requests(4, seed=15)
    with P.Handle() as h:
        ids = [h.submit(P.Instance.parse(t), o) for t, o in reqs]
        for rid in ids:
            assert h.wait(rid, 120000) == P.OK
        t, o = reqs[0]
        t0 = time.perf_counter()
        r = h.solve([P.Instance.parse(t)], o)[0]
        assert time.perf_counter() - t0 < 30
        _check_oracle(t, o, r, stride=max(1, o.restarts // 4))
