"""Block-building engine on the device (engine 1; blockproof/plp_block.cpp)
against the reference's own block engine build (golden fixtures) and the C
oracle: every restart's JSON, time_s removed, must be identical."""
import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth
from test_oracle_pins import block_cases, block_instance_text

pytestmark = pytest.mark.gpu


def _opts(seed, restarts=1, passes=1, **kw):
    kw = dict(kw)
    theta = kw.pop("theta", 0.9)
    return P.make_opts(seed=seed, restarts=restarts, passes=passes, theta=theta, engine="block", **kw)


@pytest.fixture(scope="module")
def handle():
    with P.Handle() as h:
        yield h


@pytest.mark.parametrize("case", block_cases(), ids=lambda c: f"{c['instance']}-{c['config']}-{c['seed']}")
def test_block_engine_matches_reference_goldens(handle, case):
    inst = P.Instance.parse(block_instance_text(case))
    r = handle.solve([inst], _opts(case["seed"], **O.block_flags_to_kw(case["flags"])))[0]
    assert O.strip_time(r.json(0)) == case["expected"]


@pytest.mark.parametrize("cfg", [dict(), dict(amax=4, bmax=4, kmax=6, eps=0.5, topk=64),
                                 dict(pick="support", eps=0.3), dict(pick="contact", eps=0.2, kmax=2)])
def test_block_engine_uneven_batch_matches_oracle(handle, cfg):
    texts = [i.to_thpack() for i in synth.batched_set(5, 33000)] + [synth.stress(40003).to_thpack()]
    insts = [P.Instance.parse(t) for t in texts]
    res = handle.solve(insts, _opts(11, restarts=6, **cfg))
    for t, r in zip(texts, res):
        oi = O.OInstance(t)
        for k in range(6):
            assert O.strip_time(r.json(k)) == O.strip_time(O.run_block(oi, seed=11 + k, **cfg)), k


def test_block_engine_multi_pass_matches_oracle(handle):
    text = synth.multi_restart(2).to_thpack()
    r = handle.solve([P.Instance.parse(text)], _opts(3, restarts=4, passes=3, eps=0.5))[0]
    oi = O.OInstance(text)
    for k in range(4):
        assert r.summary(k).n_passes == 3
        assert O.strip_time(r.json(k)) == O.strip_time(O.run_block(oi, seed=3 + k, passes=3, eps=0.5))


def test_block_engine_tiny_tile_retries_keep_results():
    texts = [i.to_thpack() for i in synth.batched_set(4, 34000)]
    insts = [P.Instance.parse(t) for t in texts]
    opts = _opts(1, restarts=8)
    with P.Handle() as h:
        ref = [[O.strip_time(r.json(k)) for k in range(8)] for r in h.solve(insts, opts)]
    with P.Handle() as h:
        h.set_tile(P=16, C=64, G=1, D=4, M=1)
        got = [[O.strip_time(r.json(k)) for k in range(8)] for r in h.solve(insts, opts)]
    assert got == ref


def test_block_engine_retry_stage_multi_wave_matches_oracle():
    """6400 restarts at a tiny tile: more than one wave, so the restarts that
    overflow re-run on the device at a deeper tile in the same pass."""
    texts = [i.to_thpack() for i in synth.batched_set(40, 34100)]
    insts = [P.Instance.parse(t) for t in texts]
    with P.Handle() as h:
        h.set_tile(P=16, C=64, G=1, D=1, M=1)
        b = h.prepare(insts, _opts(2, restarts=160))
        runs = [b.run() for _ in range(2)]
        res = b.fetch()
        b.close()
    assert runs[0][2] >= 4, runs   # decoder, retry list, retry decoder, selection
    for n, (t, r) in enumerate(zip(texts, res)):
        oi = O.OInstance(t)
        for k in range(n % 7, 160, 53):
            assert O.strip_time(r.json(k)) == O.strip_time(O.run_block(oi, seed=2 + k)), (n, k)


def test_block_engine_batch_rejects_mixed_engines(handle):
    inst = P.Instance.parse(synth.single_pass(1).to_thpack())
    with pytest.raises(P.PlpError):
        handle.solve([inst, inst], [P.make_opts(seed=0), _opts(0)])


def test_block_tables_cached_across_solves_stay_exact(handle):
    """The per-instance block tables are built once per (container, types,
    amax, bmax, kmax) and appended on later solves, at any position of a
    batch; the second solve (reordered, another configuration in between)
    equals the oracle."""
    texts = [i.to_thpack() for i in synth.batched_set(4, 35000)]
    insts = [P.Instance.parse(t) for t in texts]
    first = handle.solve(insts, _opts(2, restarts=3))
    handle.solve(insts[:2], _opts(2, restarts=3, amax=2, bmax=2, kmax=2))
    again = handle.solve(list(reversed(insts)), _opts(2, restarts=3))
    for t, a, b in zip(texts, first, reversed(again)):
        oi = O.OInstance(t)
        for k in range(3):
            exp = O.strip_time(O.run_block(oi, seed=2 + k))
            assert O.strip_time(a.json(k)) == exp
            assert O.strip_time(b.json(k)) == exp
