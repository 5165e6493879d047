"""Allocation-free decode (plp_decode_noalloc) against plp_solve.

Some callers cannot allocate device memory: a process whose device memory is
owned by another framework's caching allocator, or a plugin hosted by a
runtime that forbids allocation on its request path. They call
plp_decode_noalloc with output buffers they already own; the decoder's
scratch is a fixed array inside the library. Its results must equal
plp_solve's bit for bit, on two calls in a row (the second call finds the
scratch as the first call left it).

The test owns its device buffers (allocated through torch); the entry point
itself allocates none.
"""
import ctypes
import struct

import numpy as np
import pytest

import plpb200 as P
from plpb200 import synth

pytestmark = pytest.mark.gpu


def _noalloc(inst, opts, restarts, stride):
    import torch
    heads = torch.zeros(restarts * 32, dtype=torch.uint8, device="cuda")
    places = torch.zeros(restarts * stride * 8, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    status = P.lib().plp_decode_noalloc(inst._p, ctypes.byref(opts), ctypes.c_void_p(heads.data_ptr()),
                                        ctypes.c_void_p(places.data_ptr()), ctypes.c_void_p(stream))
    assert status == 0, P.last_error()
    torch.cuda.synchronize()
    return heads.cpu().numpy().tobytes(), places.cpu().numpy().view(np.uint64)


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
            rows = []
            for i in range(n):
                v = int(places[k * stride + i])
                t, oi = v >> 51, (v >> 48) & 7
                w, d, hh = ors[t][oi]
                rows.append((t, v & 0xFFFF, (v >> 16) & 0xFFFF, (v >> 32) & 0xFFFF, w, d, hh))
            assert rows == ref.placements(k), (call, k)
