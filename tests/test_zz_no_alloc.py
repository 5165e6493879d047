"""Allocation-free decode (plp_decode_noalloc) against plp_solve and the oracle.

Some callers cannot allocate device memory: a process whose device memory is
owned by another framework's caching allocator, or a plugin hosted by a
runtime that forbids allocation on its request path. They call
plp_decode_noalloc with output buffers they already own; the decoder's
scratch is a fixed array inside the library. Its results must equal
plp_solve's bit for bit, on two calls in a row (the second call finds the
scratch as the first call left it), and the CPU oracle's on sampled
restarts. The refusals are part of its contract too: bad arguments, the
block engine, tables larger than the fixed scratch, and a call made while
its stream is being captured.

The test owns its device buffers (allocated through torch); the entry point
itself allocates none.
"""
import ctypes
import struct

import numpy as np
import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth

pytestmark = pytest.mark.gpu


def _call(inst, opts, heads, places, stream=None):
    import torch
    stream = torch.cuda.current_stream().cuda_stream if stream is None else stream
    hp = ctypes.c_void_p(heads.data_ptr() if heads is not None else None)
    pp = ctypes.c_void_p(places.data_ptr() if places is not None else None)
    return P.lib().plp_decode_noalloc(inst._p, ctypes.byref(opts), hp, pp, ctypes.c_void_p(stream))


def _buffers(restarts, stride):
    import torch
    return (torch.zeros(restarts * 32, dtype=torch.uint8, device="cuda"),
            torch.zeros(restarts * stride * 8, dtype=torch.uint8, device="cuda"))


def _noalloc(inst, opts, restarts, stride):
    import torch
    heads, places = _buffers(restarts, stride)
    status = _call(inst, opts, heads, places)
    assert status == 0, P.last_error()
    torch.cuda.synchronize()
    return heads.cpu().numpy().tobytes(), places.cpu().numpy().view(np.uint64)


def _rows(places, k, stride, n, ors):
    rows = []
    for i in range(n):
        v = int(places[k * stride + i])
        t, oi = v >> 51, (v >> 48) & 7
        w, d, hh = ors[t][oi]
        rows.append((t, v & 0xFFFF, (v >> 16) & 0xFFFF, (v >> 32) & 0xFFFF, w, d, hh))
    return rows


@pytest.mark.parametrize("make,kw", [
    (lambda: synth.multi_restart(2), dict(seed=0, restarts=64)),
    (lambda: synth.single_pass(1), dict(seed=1, restarts=4, eps=0.0, theta=None)),
    (lambda: synth.stress(40004), dict(seed=3, restarts=8, passes=2)),
])
def test_noalloc_equals_solve_on_two_calls(make, kw):
    inst = P.Instance.parse(make().to_thpack())
    _, n_types, n_items = inst.info()
    stride = max(n_items, 1)
    opts = P.make_opts(**kw)
    R = kw["restarts"]
    with P.Handle() as h:
        ref = h.solve([inst], opts)[0]
    ors = [inst.orientations(t) for t in range(n_types)]
    for call in range(2):
        heads, places = _noalloc(inst, opts, R, stride)
        for k in range(R):
            n, err, vol, score, n_passes, fallback = struct.unpack_from("<iiqdii", heads, 32 * k)
            s = ref.summary(k)
            assert err == 0, (call, k)
            assert (n, vol, n_passes, bool(fallback)) == (s.n_boxes, s.volume, s.n_passes, s.fallback), (call, k)
            assert struct.pack("<d", score) == struct.pack("<d", s.score), (call, k)
            assert _rows(places, k, stride, n, ors) == ref.placements(k), (call, k)


def test_noalloc_matches_the_oracle_on_sampled_restarts():
    text = synth.batched(30007).to_thpack()
    inst = P.Instance.parse(text)
    _, n_types, n_items = inst.info()
    stride = max(n_items, 1)
    R = 48
    heads, places = _noalloc(inst, P.make_opts(seed=11, restarts=R), R, stride)
    ors = [inst.orientations(t) for t in range(n_types)]
    oi = O.OInstance(text)
    for k in range(0, R, 7):
        n, err, vol, score, n_passes, fallback = struct.unpack_from("<iiqdii", heads, 32 * k)
        assert err == 0
        js, _, _ = O.run(oi, seed=11 + k)
        exp = O.strip_time(js)
        assert (n, vol, bool(fallback)) == (exp["n_boxes"], exp["volume_cm3"], exp["fallback"])
        assert struct.pack("<d", score) == struct.pack("<d", exp["stability_score"])
        assert [list(r) for r in _rows(places, k, stride, n, ors)] == exp["placements"]


def test_noalloc_refusals():
    import torch
    inst = P.Instance.parse(synth.single_pass(1).to_thpack())
    _, _, n_items = inst.info()
    heads, places = _buffers(4, n_items)
    assert _call(inst, P.make_opts(restarts=4), None, places) == P.E_INVALID
    assert _call(inst, P.make_opts(restarts=4), heads, None) == P.E_INVALID
    block = P.make_opts(restarts=4)
    block.engine = 1
    assert _call(inst, block, heads, places) == P.E_INVALID
    # a work list of 2^20 restarts (8 bytes each) alone exceeds the 8 MiB scratch
    R = 1 << 20
    big_heads, big_places = _buffers(R, n_items)
    assert _call(inst, P.make_opts(restarts=R), big_heads, big_places) == P.E_CAPACITY
    assert "8 MiB" in P.last_error()
    del big_heads, big_places
    # refused while its stream is being captured: nothing is enqueued
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        status = _call(inst, P.make_opts(restarts=4), heads, places, stream=s.cuda_stream)
        torch.zeros(1, device="cuda")
    assert status == P.E_INVALID
    assert "capture" in P.last_error()
    # and still usable afterwards
    assert _call(inst, P.make_opts(restarts=4), heads, places) == P.OK
    torch.cuda.synchronize()
