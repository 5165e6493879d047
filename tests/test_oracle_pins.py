"""Pins the CPU oracle to the reference before it is trusted as the checker.

Sources of truth (reference file:line):
  * parity/ref_cpu/{BR1,BR2,BR3,SYN1}.json -- CPython outputs checked in by
    the reference (read from the reference tree when it is mounted);
  * the --selftest protocol (gpu/plp_gpu.cpp:43-66, gpu/make_selftest_ref.py)
    regenerated from CPython into tests/golden/selftest_ref.txt;
  * CPython random.Random streams and repr() (tests/golden/*.json);
  * known answers of tests/test_solver.py:107-231 and tests/test_geometry.py
    (FSR hand calculations, C1/C2/C3 edge cases, decode rules);
  * the reference g++ build's per-restart JSON on synthetic workloads
    (tests/golden/decoder.jsonl).
"""
import glob
import hashlib
import json
import os
import struct
import sys

import pytest

import oracle_py as O
from conftest import GOLDEN, REFERENCE, has_reference
from plpb200 import synth

BR = ["BR1", "BR2", "BR3"]


def inst_text(L, W, H, types):
    lines = ["1", "1 1", f"{L} {W} {H}", str(len(types))]
    for i, t in enumerate(types, 1):
        l, w, h, q = t
        lines.append(f"{i} {l} 1 {w} 1 {h} 1 {q}")
    return "\n".join(lines) + "\n"


# ---------------------------------------------------------------- reference JSONs
@pytest.mark.skipif(not has_reference(), reason="reference tree not mounted")
@pytest.mark.parametrize("name", BR + ["SYN1"])
def test_oracle_matches_reference_cpu_json(name):
    src = (os.path.join(REFERENCE, "data", "synthetic", "SYN1.txt") if name == "SYN1"
           else os.path.join(REFERENCE, "data", "instances", f"{name}_050.txt"))
    inst = O.OInstance(open(src).read())
    js, _, _ = O.run(inst, seed=0, passes=1, eps=0.0, theta=None)
    ref = json.load(open(os.path.join(REFERENCE, "parity", "ref_cpu", f"{name}.json")))
    ref.pop("time_s")
    assert O.strip_time(js) == ref


# ---------------------------------------------------------------- RNG / repr
def test_oracle_selftest_matches_cpython():
    out = __import__("subprocess").run([O.CLI, "--selftest"], capture_output=True, text=True,
                                       check=True).stdout
    assert out == open(os.path.join(GOLDEN, "selftest_ref.txt")).read()


def _bits(x):
    return format(struct.unpack("<Q", struct.pack("<d", x))[0], "016x")


def test_oracle_rng_matches_cpython_streams():
    vec = json.load(open(os.path.join(GOLDEN, "rng_vectors.json")))["vectors"]
    for v in vec:
        r, _ = O.rng_stream(v["seed"], n_random=len(v["random_bits"]), n_bits=0)
        assert [_bits(x) for x in r] == v["random_bits"], v["seed"]


def test_oracle_repr_matches_cpython():
    vals = json.load(open(os.path.join(GOLDEN, "repr_vectors.json")))["values"]
    for hexbits, rep in vals:
        x = struct.unpack("<d", struct.pack("<Q", int(hexbits, 16)))[0]
        assert O.py_repr(x) == rep


# ---------------------------------------------------------------- FSR known answers
def test_fsr_single_box_on_floor():
    f, s = O.fsr([(0, 0, 0, 0, 10, 10, 10)])
    assert f[0] == pytest.approx(2 / 3) and s == 0.0


def test_fsr_two_box_stack():
    f, s = O.fsr([(0, 0, 0, 0, 10, 10, 10), (0, 0, 0, 10, 10, 10, 10)])
    assert f == pytest.approx([4 / 3, 2 / 3]) and s == 0.5


def test_fsr_partial_support_split():
    f, s = O.fsr([(0, 0, 0, 0, 14, 10, 10), (0, 14, 0, 0, 14, 10, 10), (0, 5, 0, 10, 14, 10, 10)])
    assert f == pytest.approx([23 / 21, 19 / 21, 2 / 3]) and s == pytest.approx(1 / 3)


def test_fsr_three_tower():
    f, s = O.fsr([(0, 0, 0, 10 * i, 10, 10, 10) for i in range(3)])
    assert f == pytest.approx([2.0, 4 / 3, 2 / 3]) and s == pytest.approx(2 / 3)


def test_fsr_empty_packing_scores_zero():
    assert O.fsr([])[1] == 0.0


# ---------------------------------------------------------------- C1 / C2 / C3
def feas(x, y, z, w, d, h, boxes, L=100, W=100, H=100):
    import numpy as np
    fast = np.asarray([[b[0], b[1], b[2], b[0] + b[3], b[1] + b[4], b[2] + b[5]] for b in boxes] or
                      np.zeros((0, 6)), np.int32)
    return bool(O.check_all([[x, y, z]], [[w, d, h]], fast, L, W, H)[0])


def test_c1_touching_faces_is_not_overlap():
    assert feas(10, 0, 0, 10, 10, 10, [(0, 0, 0, 10, 10, 10)])
    assert not feas(5, 0, 0, 10, 10, 10, [(0, 0, 0, 10, 10, 10)])


def test_c1_stacked_different_heights_regression():
    # tests/test_geometry.py:33-36: lower top 98+56=154 touches upper bottom 154
    assert feas(243, 95, 154, 59, 39, 60, [(243, 95, 98, 81, 40, 56)], 587, 233, 220)


def test_c2_boundary():
    assert feas(0, 0, 0, 100, 50, 10, [], 100, 50, 10)
    assert not feas(0, 0, 0, 101, 50, 10, [], 100, 50, 10)
    assert not feas(0, 0, 0, 100, 50, 11, [], 100, 50, 10)


def test_c3_exact_half_is_supported_and_below_half_is_not():
    lower = [(0, 0, 0, 10, 10, 10)]
    assert feas(0, 0, 10, 20, 10, 10, lower)        # 0.5 -> ok (>= tau)
    assert not feas(7, 0, 10, 10, 10, 10, lower)    # 0.3 -> rejected
    assert not feas(0, 0, 10, 10, 10, 10, [(0, 0, 0, 10, 10, 5)])   # other level


def test_c3_sums_over_boxes():
    two = [(0, 0, 0, 10, 10, 10), (10, 0, 0, 10, 10, 10)]
    assert feas(5, 0, 10, 14, 10, 10, two)


# ---------------------------------------------------------------- decode rules
def test_decode_two_boxes_side_by_side():
    inst = O.OInstance(inst_text(100, 100, 100, [(60, 50, 50, 2)]))
    _, s, pl = O.run(inst, eps=0.0, theta=None)
    assert pl[0][1:] == (0, 0, 0, 50, 50, 60) and pl[1][1:4] == (50, 0, 0)


def test_decode_stacks_when_floor_full():
    inst = O.OInstance(inst_text(10, 10, 30, [(10, 10, 10, 3)]))
    _, s, pl = O.run(inst, eps=0.0, theta=None)
    assert [p[3] for p in pl] == [0, 10, 20]


def test_decode_skips_unplaceable_and_continues():
    inst = O.OInstance(inst_text(20, 20, 20, [(15, 15, 15, 1), (25, 10, 10, 1)]))
    _, s, pl = O.run(inst, eps=0.0, theta=None)
    assert len(pl) == 1 and pl[0][0] == 0


def test_decode_volume_vs_input_order():
    inst = O.OInstance(inst_text(100, 100, 100, [(10, 10, 10, 1), (50, 50, 50, 1)]))
    assert O.run(inst, eps=0.0, theta=None, order="volume")[2][0][0] == 1
    assert O.run(inst, eps=0.0, theta=None, order="input")[2][0][0] == 0


def test_first_fit_equals_eps_zero():
    inst = O.OInstance(inst_text(100, 100, 100, [(60, 50, 50, 2), (30, 30, 30, 4)]))
    assert O.run(inst, first_fit=True)[2] == O.run(inst, eps=0.0)[2]


def test_tower10_accepted_tower9_fallback():
    t10 = O.OInstance(inst_text(10, 10, 100, [(10, 10, 10, 10)]))
    _, s, _ = O.run(t10, seed=0)
    assert s["score"] == pytest.approx(0.9) and not s["fallback"]
    t9 = O.OInstance(inst_text(10, 10, 90, [(10, 10, 10, 9)]))
    _, s, _ = O.run(t9, seed=0)
    assert s["score"] == pytest.approx(8 / 9) and s["fallback"]


# ---------------------------------------------------------------- parser errors
def one_instance(body):
    return "\n".join(["1", "1 1001", *body])


BAD = [
    one_instance(["587 233 220", "1", "1 10 1 20 1 30 1"]),
    one_instance(["587 233 220", "1", "1 10 2 20 1 30 1 5"]),
    one_instance(["587 0 220", "1", "1 10 1 20 1 30 1 5"]),
    one_instance(["587 233 220", "1", "1 0 1 20 1 30 1 5"]),
    one_instance(["587 233 220", "1", "1 10 1 20 1 30 1 -5"]),
    one_instance(["587 233 220", "1", "1 10.5 1 20 1 30 1 5"]),
    one_instance(["587 233 220", "2", "1 10 1 20 1 30 1 5", "3 5 1 6 1 7 1 2"]),
    "\n".join(["2", "1 1001", "587 233 220", "1", "1 10 1 20 1 30 1 5"]),
    "0",
    "",
]


@pytest.mark.parametrize("text", BAD)
def test_oracle_parser_rejects(text):
    with pytest.raises(O.OracleFormatError):
        O.OInstance(text)


# ---------------------------------------------------------------- reference g++ goldens
def _golden_cases():
    return [json.loads(l) for l in open(os.path.join(GOLDEN, "decoder.jsonl"))]


def _instance_for(case):
    if "set_index" in case:   # 1 % samples of the bench's batched / stress sets
        i = case["set_index"]
        inst = synth.batched(30000 + i) if case["case"].startswith("batched") else synth.stress(40000 + i)
        text = inst.to_thpack()
        assert hashlib.sha256(text.encode()).hexdigest() == case["sha256"], "generator drifted"
        return text
    gen = {"single_pass": lambda: [synth.single_pass(1)],
           "multi_restart": lambda: [synth.multi_restart(2)],
           "batched": lambda: synth.batched_set(8),
           "stress": lambda: synth.stress_set(2)}
    key = next(k for k in gen if case["case"].startswith(k))
    inst = gen[key]()[case["instance"]]
    text = inst.to_thpack()
    assert hashlib.sha256(text.encode()).hexdigest() == case["sha256"], "generator drifted"
    return text


def flags_to_kw(flags):
    kw = dict(eps=0.3, theta=0.9, order="volume", first_fit=False, mu=0.2)
    i = 0
    while i < len(flags):
        f = flags[i]
        if f == "--eps":
            kw["eps"] = float(flags[i + 1]); i += 2
        elif f == "--no-theta":
            kw["theta"] = None; i += 1
        elif f == "--theta":
            kw["theta"] = float(flags[i + 1]); i += 2
        elif f == "--order":
            kw["order"] = flags[i + 1]; i += 2
        elif f == "--first-fit":
            kw["first_fit"] = True; i += 1
        elif f == "--mu":
            kw["mu"] = float(flags[i + 1]); i += 2
        else:
            raise ValueError(f)
    return kw


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: f"{c['case']}-{c['instance']}")
def test_oracle_matches_reference_gpp_goldens(case):
    inst = O.OInstance(_instance_for(case))
    kw = flags_to_kw(case["flags"])
    for s, exp in zip(case["seeds"], case["expected"]):
        js, _, _ = O.run(inst, seed=s, passes=case["passes"], **kw)
        assert O.strip_time(js) == exp, (case["case"], s)


@pytest.mark.skipif(not has_reference(), reason="reference tree not mounted")
def test_oracle_matches_reference_cpython_eps():
    sys.path.insert(0, REFERENCE)
    from plp.parser import parse
    from plp.solver import run
    for inst_s in (synth.single_pass(1), synth.multi_restart(2)):
        text = inst_s.to_thpack()
        ref_inst = parse(text)[0]
        oi = O.OInstance(text)
        for seed in (11, 12):
            r = run(ref_inst, seed=seed, time_limit_s=0, eps=0.3, theta=0.9, single_pass=True)
            _, s, pl = O.run(oi, seed=seed)
            assert pl == [tuple(p) for p in r.placements]
            assert (s["n_boxes"], s["volume"], s["score"], s["fallback"]) == \
                (r.n_boxes, r.volume, r.score, r.fallback)


# ---------------------------------------------------------------- block engine
def block_cases():
    return [json.loads(l) for l in open(os.path.join(GOLDEN, "block.jsonl"))]


def block_instance_text(case):
    gen = {"single_pass": lambda: synth.single_pass(1), "multi_restart": lambda: synth.multi_restart(2),
           "batched_30001": lambda: synth.batched(30001), "stress_40000": lambda: synth.stress(40000)}
    text = gen[case["instance"]]().to_thpack()
    assert hashlib.sha256(text.encode()).hexdigest() == case["sha256"], "generator drifted"
    return text


@pytest.mark.parametrize("case", block_cases(), ids=lambda c: f"{c['instance']}-{c['config']}-{c['seed']}")
def test_oracle_block_matches_reference_block_engine(case):
    """The C restatement of blockproof/plp_block.cpp against the reference's
    own build (golden fixtures), --single-pass."""
    js = O.run_block(O.OInstance(block_instance_text(case)), seed=case["seed"],
                     **O.block_flags_to_kw(case["flags"]))
    assert O.strip_time(js) == case["expected"]
