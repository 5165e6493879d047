"""Host side of the C ABI (no GPU): the library loads and exports every
symbol include/plp_capi.h declares; parser, orientation table, item order,
host MT19937 and float formatting match the oracle / CPython vectors."""
import json
import os
import random
import re
import struct

import numpy as np
import pytest

import oracle_py as O
import plpb200 as P
from conftest import GOLDEN
from plpb200 import synth
from test_oracle_pins import BAD


def declared_symbols():
    text = open(P.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(plp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = P.lib()
    names = declared_symbols()
    assert len(names) > 30
    for n in names:
        assert hasattr(lib, n), n


def test_selftest_matches_cpython():
    assert P.selftest() == open(os.path.join(GOLDEN, "selftest_ref.txt")).read()


def test_py_repr_matches_cpython():
    vals = json.load(open(os.path.join(GOLDEN, "repr_vectors.json")))["values"]
    for hexbits, rep in vals:
        x = struct.unpack("<d", struct.pack("<Q", int(hexbits, 16)))[0]
        assert P.py_repr(x) == rep


def test_host_rng_matches_cpython():
    vec = json.load(open(os.path.join(GOLDEN, "rng_vectors.json")))["vectors"]
    seeds = [v["seed"] for v in vec]
    r, _ = P.rng_dump(seeds, n_random=700, n_bits=0, device=False)
    for i, v in enumerate(vec):
        got = [format(struct.unpack("<Q", struct.pack("<d", x))[0], "016x") for x in r[i]]
        assert got == v["random_bits"], v["seed"]
    for s in (0, 3, 2**40 + 7):
        rr = random.Random(s)
        _, b = P.rng_dump([s], n_random=0, n_bits=30, k_bits=7, device=False)
        assert b[0].tolist() == [rr.getrandbits(7) for _ in range(30)]


@pytest.mark.parametrize("text", BAD)
def test_parser_rejects_like_the_oracle(text):
    with pytest.raises(P.InstanceFormatError):
        P.Instance.parse(text)


def test_parser_messages_match_reference_cpp_parser():
    # messages of gpu/plp_common.hpp:68-141 (printed after "instance error: ")
    cases = {
        "": "empty file",
        "x": "not an integer: x (instance count)",
        "0": "instance count must be >= 1",
        "1\n1 2 3\n": "malformed problem line",
        "1\n1\n587 233\n": "container line must have 3 dimensions",
        "1\n1\n587 0 220\n1\n": "container dimensions must be positive",
        "1\n1\n587 233 220\n1 2\n": "type-count line must be a single integer",
        "1\n1\n587 233 220\n2\n1 10 1 20 1 30 1 5\n": "instance truncated",
        "1\n1\n587 233 220\n1\n1 10 1 20 1 30 1\n": "item line must have 8 tokens",
        "1\n1\n587 233 220\n1\n2 10 1 20 1 30 1 5\n": "item index must be sequential",
        "1\n1\n587 233 220\n1\n1 10 1 20 1 0 1 5\n": "item dimensions must be positive",
        "1\n1\n587 233 220\n1\n1 10 1 20 3 30 1 5\n": "orientation flags must be 0/1",
        "1\n1\n587 233 220\n1\n1 10 1 20 1 30 1 -1\n": "item qty must be >= 0",
        "1\n1\n587 233 220\n1\n1 10 1 20 1 30 1 5\n7\n": "trailing data after last instance",
    }
    for text, msg in cases.items():
        with pytest.raises(P.InstanceFormatError) as e:
            P.Instance.parse_multi(text)
        assert e.value.message == msg, text


def test_parse_multi_and_info():
    a, b = synth.single_pass(1), synth.multi_restart(2)
    ta, tb = a.to_thpack().splitlines(), b.to_thpack().splitlines()
    text = "\n".join(["2"] + ta[1:] + tb[1:]) + "\n"
    insts = P.Instance.parse_multi(text)
    assert len(insts) == 2
    assert insts[0].info() == ((587, 233, 220), 3, a.n_items)
    assert insts[1].info() == ((587, 233, 220), 10, b.n_items)


def test_orientations_and_item_order_match_oracle():
    for inst in [synth.single_pass(1), synth.multi_restart(2)] + synth.stress_set(3) + synth.batched_set(5):
        text = inst.to_thpack()
        p, o = P.Instance.parse(text), O.OInstance(text)
        n_types = p.info()[1]
        for t in range(n_types):
            assert p.orientations(t) == o.orientations(t)
        for order in ("volume", "input"):
            assert p.item_sequence(order) == o.item_sequence(0 if order == "volume" else 1)


def test_orientation_dedup_and_parser_order():
    cube = P.Instance.from_types(100, 100, 100, [[10, 1, 10, 1, 10, 1, 1]])
    assert cube.orientations(0) == [(10, 10, 10)]
    box = P.Instance.from_types(100, 100, 100, [[2, 1, 3, 1, 4, 1, 1]])
    assert box.orientations(0) == [(3, 4, 2), (4, 3, 2), (2, 4, 3), (4, 2, 3), (2, 3, 4), (3, 2, 4)]
    flat = P.Instance.from_types(100, 100, 100, [[2, 0, 3, 0, 4, 0, 1]])
    assert flat.orientations(0) == []


def test_bad_arguments_return_status_not_crash():
    lib = P.lib()
    assert lib.plp_feas_check_all(None, -1, None, 0, None, 0, 1, 1, 1, None) == P.E_INVALID
    assert lib.plp_result_restarts(None) == 0
    assert lib.plp_solve(None, None, 0, None, 0, None) == P.E_INVALID
    assert "null" in P.last_error() or "bad" in P.last_error()
