"""GPU parity of the individual kernels against the oracle / CPython vectors.

  kernel (a) one-step feasibility   plp_feas_check_all  vs  orc_check_all
  kernel (c) device MT19937         plp_rng_dump        vs  CPython streams
  kernel (d) device item order      plp_item_order      vs  host item sequence
  kernel (e) device FSR             plp_fsr_score       vs  orc_compute_fsr
All comparisons are bit-exact (integers, bytes, and FP64 bit patterns).
"""
import json
import os
import random
import struct

import numpy as np
import pytest

import oracle_py as O
import plpb200 as P
from conftest import GOLDEN
from plpb200 import synth

pytestmark = pytest.mark.gpu


def _states(text, seed, eps=0.3, limit=40):
    """Decode states (placed prefix, type of the next box) from an oracle run."""
    inst = O.OInstance(text)
    _, _, pl = O.run(inst, seed=seed, eps=eps)
    L, W, H = inst.dims()
    out = []
    for k in range(0, len(pl), max(1, len(pl) // limit)):
        prefix = pl[:k]
        cand = O.candidate_points(prefix)
        fast = [(x, y, z, x + w, y + d, z + h) for (_t, x, y, z, w, d, h) in prefix]
        t = pl[k][0]
        ors = inst.orientations(t)
        out.append((cand, ors, fast, (L, W, H)))
    return out


@pytest.mark.parametrize("gen,seed", [(lambda: synth.single_pass(1), 1),
                                      (lambda: synth.multi_restart(2), 3),
                                      (lambda: synth.batched(30001), 4),
                                      (lambda: synth.stress(40001), 5)])
def test_feas_check_all_matches_oracle(gen, seed):
    text = gen().to_thpack()
    for cand, ors, fast, (L, W, H) in _states(text, seed):
        got = P.feas_check_all(cand, ors, fast or np.zeros((0, 6)), L, W, H)
        exp = O.check_all(cand, ors, fast or np.zeros((0, 6)), L, W, H)
        assert np.array_equal(got, exp)


def test_feas_edge_cases():
    L, W, H = 100, 80, 60
    rng = random.Random(7)
    # no placed boxes, more than 6 orientations, unsorted / covered points
    cand = [(rng.randint(0, L), rng.randint(0, W), rng.randint(0, H)) for _ in range(700)]
    ors = [(rng.randint(1, 50), rng.randint(1, 50), rng.randint(1, 50)) for _ in range(9)]
    boxes = []
    for _ in range(60):
        x, y, z = rng.randint(0, L - 1), rng.randint(0, W - 1), rng.choice([0, 10, 20, 30])
        boxes.append((x, y, z, x + rng.randint(1, 30), y + rng.randint(1, 30), z + rng.choice([10, 20])))
    for fast in ([], boxes[:1], boxes):
        f = np.asarray(fast, np.int32).reshape(-1, 6)
        assert np.array_equal(P.feas_check_all(cand, ors, f, L, W, H), O.check_all(cand, ors, f, L, W, H))
    assert P.feas_check_all(np.zeros((0, 3)), ors, boxes, L, W, H).size == 0


def _bits(x):
    return format(struct.unpack("<Q", struct.pack("<d", x))[0], "016x")


def test_device_rng_matches_cpython():
    vec = json.load(open(os.path.join(GOLDEN, "rng_vectors.json")))["vectors"]
    seeds = [v["seed"] for v in vec]
    r, _ = P.rng_dump(seeds, n_random=700, n_bits=0)
    for i, v in enumerate(vec):
        assert [_bits(x) for x in r[i]] == v["random_bits"], v["seed"]
    # getrandbits(k) right after seeding, many seeds, host stream as reference
    many = list(range(0, 3000, 7)) + [2**32 + 3, 2**45 + 1]
    for k in (1, 13, 32):
        rd, bd = P.rng_dump(many, n_random=3, n_bits=650, k_bits=k)
        rh, bh = P.rng_dump(many, n_random=3, n_bits=650, k_bits=k, device=False)
        assert np.array_equal(bd, bh) and np.array_equal(rd.view(np.uint64), rh.view(np.uint64))
    # the host stream itself is CPython's
    for s in (0, 5, 2**33 + 9):
        rr = random.Random(s)
        _, bh = P.rng_dump([s], n_random=0, n_bits=20, k_bits=13, device=False)
        assert bh[0].tolist() == [rr.getrandbits(13) for _ in range(20)]


def _oracle_packings():
    packs = []
    for gen, seeds in ((lambda: synth.multi_restart(2), range(6)), (lambda: synth.stress(40000), range(3)),
                       (lambda: synth.batched(30002), range(3))):
        inst = O.OInstance(gen().to_thpack())
        for s in seeds:
            packs.append(O.run(inst, seed=s)[2])
    packs.append([(0, 0, 0, 0, 10, 10, 10)])
    packs.append([(0, 0, 0, 10 * i, 10, 10, 10) for i in range(3)])
    packs.append([(0, 0, 0, 0, 14, 10, 10), (0, 14, 0, 0, 14, 10, 10), (0, 5, 0, 10, 14, 10, 10)])
    packs.append([])
    return packs


@pytest.mark.parametrize("mu", [0.2, 0.45])
def test_device_fsr_matches_oracle(mu):
    packs = _oracle_packings()
    scores, fsrs = P.fsr_score(packs, mu=mu)
    for p, s, f in zip(packs, scores, fsrs):
        of, os_ = O.fsr(p, mu=mu)
        assert _bits(s) == _bits(os_)
        assert [_bits(v) for v in f] == [_bits(v) for v in of]


def test_device_item_order_matches_host():
    insts = [P.Instance.parse(synth.batched(30000 + i).to_thpack()) for i in range(12)]
    insts.append(P.Instance.parse(synth.stress(40000).to_thpack()))
    for order in ("volume", "input"):
        dev = P.item_order(insts, order)
        for inst, d in zip(insts, dev):
            assert d == [t for t, _ in inst.item_sequence(order)]


def test_device_item_order_matches_oracle():
    """Kernel (d) against the oracle's item_sequence (gpu/plp_common.hpp:335-351):
    the bench's batched and stress instances and the reference's BR instances."""
    texts = [synth.batched(30000 + i).to_thpack() for i in range(0, 4096, 97)]
    texts += [synth.stress(40000 + i).to_thpack() for i in range(0, 512, 101)]
    man = json.load(open(os.path.join(GOLDEN, "reference", "data", "manifest.json")))["instances"]
    texts += [open(os.path.join(GOLDEN, "reference", "data", e["file"])).read() for e in man]
    insts = [P.Instance.parse(t) for t in texts]
    for order, code in (("volume", 0), ("input", 1)):
        dev = P.item_order(insts, order)
        for t, d in zip(texts, dev):
            assert d == [ti for ti, _ in O.OInstance(t).item_sequence(order=code)]
