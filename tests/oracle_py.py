"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE.

Used only by the tests, the smoke check and bench.py's CPU-baseline leg as
the checker of the CUDA path.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
LIB = os.path.join(ORACLE_DIR, "liboracle.so")
CLI = os.path.join(ORACLE_DIR, "plp_oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")


class Item(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("l", "w", "h", "lf", "wf", "hf", "qty")]


class Inst(ctypes.Structure):
    _fields_ = [("L", ctypes.c_int), ("W", ctypes.c_int), ("H", ctypes.c_int),
                ("n_types", ctypes.c_int), ("items", ctypes.POINTER(Item))]


class Rng(ctypes.Structure):
    _fields_ = [("mt", ctypes.c_uint32 * 624), ("pos", ctypes.c_int)]


class Place(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("type", "x", "y", "z", "w", "d", "h")]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("steps", "pairs", "c2_pairs", "aabb_full",
                                              "max_cand", "pairs_to_first", "random_steps")]


class BlockCfg(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("amax", "bmax", "kmax", "topk", "pick")]


class Res(ctypes.Structure):
    _fields_ = [("n_boxes", ctypes.c_int), ("volume", ctypes.c_int64), ("score", ctypes.c_double),
                ("fallback", ctypes.c_int), ("n_passes", ctypes.c_int), ("time_s", ctypes.c_double),
                ("seed", ctypes.c_int64), ("placements", ctypes.POINTER(Place))]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.orc_parse.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(Inst)), ctypes.c_char_p,
                                ctypes.c_int]
        L.orc_free_instances.argtypes = [ctypes.POINTER(Inst), ctypes.c_int]
        L.orc_rng_seed.argtypes = [ctypes.POINTER(Rng), ctypes.c_uint64]
        L.orc_rng_random.argtypes = [ctypes.POINTER(Rng)]
        L.orc_rng_random.restype = ctypes.c_double
        L.orc_rng_getrandbits.argtypes = [ctypes.POINTER(Rng), ctypes.c_int]
        L.orc_rng_getrandbits.restype = ctypes.c_uint32
        L.orc_rng_randrange.argtypes = [ctypes.POINTER(Rng), ctypes.c_int]
        L.orc_check_all.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, P]
        L.orc_feasible_one.argtypes = [ctypes.c_int] * 6 + [P] + [ctypes.c_int] * 4
        L.orc_compute_fsr.argtypes = [ctypes.POINTER(Place), ctypes.c_int, ctypes.c_double, P]
        L.orc_stability_score.argtypes = [ctypes.POINTER(Place), ctypes.c_int, ctypes.c_double]
        L.orc_stability_score.restype = ctypes.c_double
        L.orc_run.argtypes = [ctypes.POINTER(Inst), ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                              ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                              ctypes.c_double, ctypes.POINTER(Res), ctypes.POINTER(Stats)]
        L.orc_free_result.argtypes = [ctypes.POINTER(Res)]
        L.orc_block_run.argtypes = [ctypes.POINTER(Inst), ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(BlockCfg), ctypes.POINTER(Res)]
        L.orc_to_json.argtypes = [ctypes.POINTER(Res), ctypes.c_char_p, ctypes.c_int]
        L.orc_py_repr.argtypes = [ctypes.c_double, ctypes.c_char_p]
        L.orc_orientations.argtypes = [ctypes.POINTER(Item), ctypes.POINTER(ctypes.c_int * 3 * 6)]
        L.orc_item_sequence.argtypes = [ctypes.POINTER(Inst), ctypes.c_int, P, P]
        _lib = L
    return _lib


class OracleFormatError(ValueError):
    pass


class OInstance:
    def __init__(self, text: str):
        out = ctypes.POINTER(Inst)()
        err = ctypes.create_string_buffer(256)
        n = lib().orc_parse(text.encode(), ctypes.byref(out), err, 256)
        if n < 0:
            raise OracleFormatError(err.value.decode())
        self._p, self._n = out, n

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_free_instances(self._p, self._n)
            self._p = None

    @property
    def n(self):
        return self._n

    def at(self, i=0):
        return ctypes.pointer(self._p[i])

    def items(self, i=0):
        I = self._p[i]
        return [(I.items[t].l, I.items[t].lf, I.items[t].w, I.items[t].wf, I.items[t].h, I.items[t].hf,
                 I.items[t].qty) for t in range(I.n_types)]

    def dims(self, i=0):
        I = self._p[i]
        return I.L, I.W, I.H

    def orientations(self, t, i=0):
        out = (ctypes.c_int * 3 * 6)()
        n = lib().orc_orientations(ctypes.pointer(self._p[i].items[t]), ctypes.byref(out))
        return [tuple(out[k]) for k in range(n)]

    def item_sequence(self, order=0, i=0):
        I = self._p[i]
        n = sum(I.items[t].qty for t in range(I.n_types))
        ti = np.zeros(max(n, 1), np.int32)
        cp = np.zeros(max(n, 1), np.int32)
        lib().orc_item_sequence(ctypes.pointer(I), order, ti.ctypes.data_as(ctypes.c_void_p),
                                cp.ctypes.data_as(ctypes.c_void_p))
        return list(zip(ti[:n].tolist(), cp[:n].tolist()))


def run(inst: OInstance, seed=0, passes=1, eps=0.3, theta=0.9, order="volume", first_fit=False,
        mu=0.2, stats=False, i=0):
    """One run with a fixed pass count. Returns (json_without_time, summary, placements[, stats])."""
    r = Res()
    st = Stats()
    has_theta = theta is not None
    lib().orc_run(inst.at(i), int(seed), int(passes), -1.0, float(eps), 1 if has_theta else 0,
                  float(theta) if has_theta else 0.0, 0 if order == "volume" else 1,
                  1 if first_fit else 0, float(mu), ctypes.byref(r), ctypes.byref(st) if stats else None)
    pl = [(r.placements[k].type, r.placements[k].x, r.placements[k].y, r.placements[k].z,
           r.placements[k].w, r.placements[k].d, r.placements[k].h) for k in range(r.n_boxes)]
    summ = dict(n_boxes=r.n_boxes, volume=r.volume, score=r.score, fallback=bool(r.fallback),
                n_passes=r.n_passes, seed=r.seed)
    need = lib().orc_to_json(ctypes.byref(r), None, 0)
    buf = ctypes.create_string_buffer(need + 1)
    lib().orc_to_json(ctypes.byref(r), buf, need + 1)
    lib().orc_free_result(ctypes.byref(r))
    js = buf.value.decode()
    if stats:
        return js, summ, pl, {f: getattr(st, f) for f, _ in Stats._fields_}
    return js, summ, pl


def check_all(cand, ors, fast, L, W, H) -> np.ndarray:
    c = np.ascontiguousarray(np.asarray(cand, np.int32).reshape(-1, 3))
    o = np.ascontiguousarray(np.asarray(ors, np.int32).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(fast, np.int32).reshape(-1, 6))
    bits = np.zeros(max(len(c) * len(o), 1), np.uint8)
    V = ctypes.c_void_p
    lib().orc_check_all(c.ctypes.data_as(V), len(c), o.ctypes.data_as(V), len(o), f.ctypes.data_as(V),
                        len(f), L, W, H, bits.ctypes.data_as(V))
    return bits[:len(c) * len(o)]


def rng_stream(seed, n_random=16, n_bits=16, k_bits=13):
    r = Rng()
    lib().orc_rng_seed(ctypes.byref(r), abs(int(seed)))
    a = [lib().orc_rng_random(ctypes.byref(r)) for _ in range(n_random)]
    b = [lib().orc_rng_getrandbits(ctypes.byref(r), k_bits) for _ in range(n_bits)]
    return a, b


def fsr(placed, mu=0.2):
    n = len(placed)
    arr = (Place * max(n, 1))(*[Place(*p) for p in placed])
    out = np.zeros(max(n, 1), np.float64)
    lib().orc_compute_fsr(arr, n, mu, out.ctypes.data_as(ctypes.c_void_p))
    return out[:n].tolist(), lib().orc_stability_score(arr, n, mu)


def py_repr(x):
    buf = ctypes.create_string_buffer(48)
    lib().orc_py_repr(float(x), buf)
    return buf.value.decode()


def strip_time(js: str) -> dict:
    import json
    d = json.loads(js)
    d.pop("time_s", None)
    return d


def candidate_points(placed):
    """Extreme points of a placement prefix (plp/solver.py:86-96 rule), sorted (z, y, x)."""
    pts = {(0, 0, 0)}
    for (_t, x, y, z, w, d, h) in placed:
        for cx in (x, x + w):
            for cy in (y, y + d):
                for cz in (z, z + h):
                    pts.add((cx, cy, cz))
    if placed:
        pts = {p for p in pts if not any(x < p[0] < x + w and y < p[1] < y + d and z < p[2] < z + h
                                         for (_t, x, y, z, w, d, h) in placed)}
    return sorted(pts, key=lambda p: (p[2], p[1], p[0]))


def nan_or(theta):
    return math.nan if theta is None else theta


PICKS = {"first": 0, "support": 1, "contact": 2}


def run_block(inst: "OInstance", seed=0, passes=1, eps=0.3, theta=0.9, mu=0.2, amax=3, bmax=3, kmax=4,
              topk=8, pick="first", i=0):
    """Block-building engine (blockproof/plp_block.cpp), fixed pass count.
    Returns the JSON line (time_s included)."""
    r = Res()
    cfg = BlockCfg(max(1, amax), max(1, bmax), max(1, kmax), max(1, topk), PICKS[pick])
    has_theta = theta is not None
    lib().orc_block_run(inst.at(i), int(seed), int(passes), -1.0, float(eps), 1 if has_theta else 0,
                        float(theta) if has_theta else 0.0, float(mu), ctypes.byref(cfg), ctypes.byref(r))
    need = lib().orc_to_json(ctypes.byref(r), None, 0)
    buf = ctypes.create_string_buffer(need + 1)
    lib().orc_to_json(ctypes.byref(r), buf, need + 1)
    lib().orc_free_result(ctypes.byref(r))
    return buf.value.decode()


def block_flags_to_kw(flags):
    """plp_block CLI flags -> run_block keyword arguments (reference defaults)."""
    kw = dict(eps=0.3, theta=0.9, amax=3, bmax=3, kmax=4, topk=8, pick="first")
    i = 0
    while i < len(flags):
        f = flags[i]
        if f == "--no-theta":
            kw["theta"] = None
            i += 1
            continue
        v = flags[i + 1]
        key = f[2:]
        kw[key] = v if key == "pick" else (float(v) if key in ("eps", "theta") else int(v))
        i += 2
    return kw
