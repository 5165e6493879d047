"""Python binding of libplp_b200.so (the B200 extreme-point decoder).

Thin ctypes layer over include/plp_capi.h. The names follow the reference's
Python API where one exists (plp/solver.py: ``run``, results with
``n_boxes``, ``volume``, ``score``, ``fallback``, ``placements``), and every
call goes through the C ABI; there is no Python or CPU fallback: if the
library is missing or a CUDA call fails, a PlpError is raised.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_DIR, "libplp_b200.so")
CLI_PATH = os.path.join(PKG_DIR, "plp_gpu")
BLOCK_CLI_PATH = os.path.join(os.path.dirname(CLI_PATH), "plp_block")
HEADER_PATH = os.path.join(os.path.dirname(PKG_DIR), "include", "plp_capi.h")

OK, E_INVALID, E_FORMAT, E_CUDA, E_CAPACITY, E_BUDGET, E_TIMEOUT, E_NOT_FOUND, E_CANCELLED, \
    E_PENDING, E_DEVICE = range(11)


class PlpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


class InstanceFormatError(PlpError, ValueError):
    """The thpack text violates the format (reference InstanceFormatError)."""


class RunOpts(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_int64),
        ("restarts", ctypes.c_int32),
        ("passes", ctypes.c_int32),
        ("eps", ctypes.c_double),
        ("theta", ctypes.c_double),
        ("order", ctypes.c_int32),
        ("first_fit", ctypes.c_int32),
        ("mu", ctypes.c_double),
        ("time_limit_s", ctypes.c_double),
        ("best_only", ctypes.c_int32),
        ("engine", ctypes.c_int32),
        ("blk_amax", ctypes.c_int32),
        ("blk_bmax", ctypes.c_int32),
        ("blk_kmax", ctypes.c_int32),
        ("blk_topk", ctypes.c_int32),
        ("blk_pick", ctypes.c_int32),
    ]


class Summary(ctypes.Structure):
    _fields_ = [
        ("n_boxes", ctypes.c_int32),
        ("fallback", ctypes.c_int32),
        ("volume", ctypes.c_int64),
        ("score", ctypes.c_double),
        ("n_passes", ctypes.c_int32),
        ("err", ctypes.c_int32),
        ("seed", ctypes.c_int64),
        ("time_s", ctypes.c_double),
    ]


_lib = None


def lib():
    """Load libplp_b200.so (raises PlpError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PlpError(E_INVALID, f"{LIB_PATH} is missing: build it with `make -C plp-gpu_b200`")
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64, D, SZ = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t
    sig = {
        "plp_last_error": (ctypes.c_char_p, [P]),
        "plp_feas_check_all": (ctypes.c_int, [P, I32, P, I32, P, I32, I32, I32, I32, P]),
        "plp_feas_check_all_dev": (ctypes.c_int, [P, I32, P, I32, P, I32, I32, I32, I32, P, P]),
        "plp_instance_parse": (ctypes.c_int, [ctypes.c_char_p, SZ, P]),
        "plp_instance_parse_multi": (ctypes.c_int, [ctypes.c_char_p, SZ, P, P]),
        "plp_instance_load": (ctypes.c_int, [ctypes.c_char_p, P]),
        "plp_instance_from_types": (ctypes.c_int, [I32, I32, I32, I32, P, P]),
        "plp_instance_free": (None, [P]),
        "plp_instance_info": (ctypes.c_int, [P, P, P, P]),
        "plp_orientations": (ctypes.c_int, [P, I32, P, P]),
        "plp_item_sequence": (ctypes.c_int, [P, I32, P, P]),
        "plp_free": (None, [P]),
        "plp_default_opts": (None, [P]),
        "plp_result_restarts": (I32, [P]),
        "plp_result_summary": (ctypes.c_int, [P, I32, P]),
        "plp_result_placements": (ctypes.c_int, [P, I32, P, I32, P]),
        "plp_result_best": (ctypes.c_int, [P, P, P]),
        "plp_result_json": (ctypes.c_int, [P, I32, P, SZ, P]),
        "plp_result_free": (None, [P]),
        "plp_run_plain": (ctypes.c_int, [P, P, P]),
        "plp_create": (ctypes.c_int, [SZ, I32, P]),
        "plp_destroy": (None, [P]),
        "plp_set_tile": (ctypes.c_int, [P, I32, I32, I32, I32, I32]),
        "plp_debug_sync_bound": (ctypes.c_int, [P, I32, I32]),
        "plp_serve_counters": (ctypes.c_int, [P, P, P, P, P]),
        "plp_autotune": (ctypes.c_int, [P, P, I32, P, I32, I32, P]),
        "plp_batch_graph": (ctypes.c_int, [P]),
        "plp_solve": (ctypes.c_int, [P, P, I32, P, I32, P]),
        "plp_submit": (ctypes.c_int, [P, P, P, P]),
        "plp_poll": (ctypes.c_int, [P, I64]),
        "plp_wait": (ctypes.c_int, [P, I64, I64]),
        "plp_take_result": (ctypes.c_int, [P, I64, P]),
        "plp_cancel": (ctypes.c_int, [P, I64]),
        "plp_request_times": (ctypes.c_int, [P, I64, P, P]),
        "plp_batch_prepare": (ctypes.c_int, [P, P, I32, P, I32, P]),
        "plp_batch_run": (ctypes.c_int, [P, P, P, P]),
        "plp_batch_fetch": (ctypes.c_int, [P, P]),
        "plp_batch_io_bytes": (ctypes.c_int, [P, P, P]),
        "plp_batch_free": (None, [P]),
        "plp_result_work": (ctypes.c_int, [P, I32, P, P]),
        "plp_decode_noalloc": (ctypes.c_int, [P, P, P, P, P]),
        "plp_rng_dump": (ctypes.c_int, [P, I32, I32, I32, I32, P, P]),
        "plp_rng_dump_host": (ctypes.c_int, [P, I32, I32, I32, I32, P, P]),
        "plp_fsr_score": (ctypes.c_int, [P, P, I32, D, P, P]),
        "plp_item_order": (ctypes.c_int, [P, I32, I32, P, P]),
        "plp_py_repr": (ctypes.c_int, [D, P, SZ]),
        "plp_selftest": (ctypes.c_int, [P, SZ, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error(handle=None) -> str:
    m = lib().plp_last_error(handle)
    return m.decode() if m else ""


def _check(status: int, handle=None):
    if status != OK:
        msg = last_error(handle)
        if status == E_FORMAT:
            raise InstanceFormatError(status, msg)
        raise PlpError(status, msg)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def make_opts(seed=0, restarts=1, passes=1, eps=0.3, theta=0.9, order="volume", first_fit=False,
              mu=0.2, time_limit_s=-1.0, best_only=False, engine="ep", amax=3, bmax=3, kmax=4, topk=8,
              pick="first") -> RunOpts:
    o = RunOpts()
    o.seed = int(seed)
    o.restarts = int(restarts)
    o.passes = int(passes)
    o.eps = float(eps)
    o.theta = math.nan if theta is None else float(theta)
    o.order = {"volume": 0, "input": 1}[order] if isinstance(order, str) else int(order)
    o.first_fit = 1 if first_fit else 0
    o.mu = float(mu)
    o.time_limit_s = float(time_limit_s)
    o.best_only = 1 if best_only else 0
    o.engine = {"ep": 0, "block": 1}[engine] if isinstance(engine, str) else int(engine)
    o.blk_amax, o.blk_bmax, o.blk_kmax, o.blk_topk = int(amax), int(bmax), int(kmax), int(topk)
    o.blk_pick = {"first": 0, "support": 1, "contact": 2}[pick] if isinstance(pick, str) else int(pick)
    return o


# ---------------------------------------------------------------------------
# instances
# ---------------------------------------------------------------------------
class Instance:
    """One thpack instance (reference plp.parser.Instance)."""

    def __init__(self, ptr):
        self._p = ctypes.c_void_p(ptr)

    def __del__(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.plp_instance_free(self._p)
            self._p = None

    @classmethod
    def parse(cls, text: str) -> "Instance":
        out = ctypes.c_void_p()
        b = text.encode()
        _check(lib().plp_instance_parse(b, len(b), ctypes.byref(out)))
        return cls(out.value)

    @classmethod
    def parse_multi(cls, text: str) -> list:
        arr = ctypes.c_void_p()
        n = ctypes.c_int32()
        b = text.encode()
        _check(lib().plp_instance_parse_multi(b, len(b), ctypes.byref(arr), ctypes.byref(n)))
        ptrs = ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))
        out = [cls(ptrs[i]) for i in range(n.value)]
        lib().plp_free(arr)
        return out

    @classmethod
    def load(cls, path: str) -> "Instance":
        out = ctypes.c_void_p()
        _check(lib().plp_instance_load(path.encode(), ctypes.byref(out)))
        return cls(out.value)

    @classmethod
    def from_types(cls, L, W, H, types7) -> "Instance":
        t = np.ascontiguousarray(np.asarray(types7, dtype=np.int32).reshape(-1, 7))
        out = ctypes.c_void_p()
        _check(lib().plp_instance_from_types(L, W, H, len(t), _ptr(t), ctypes.byref(out)))
        return cls(out.value)

    def info(self):
        lwh = np.zeros(3, np.int32)
        nt, ni = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().plp_instance_info(self._p, _ptr(lwh), ctypes.byref(nt), ctypes.byref(ni)))
        return tuple(int(v) for v in lwh), nt.value, ni.value

    def orientations(self, t: int) -> list:
        buf = np.zeros(18, np.int32)
        n = ctypes.c_int32()
        _check(lib().plp_orientations(self._p, t, _ptr(buf), ctypes.byref(n)))
        return [tuple(int(v) for v in buf[3 * i:3 * i + 3]) for i in range(n.value)]

    def item_sequence(self, order="volume") -> list:
        n = self.info()[2]
        ti = np.zeros(max(n, 1), np.int32)
        cp = np.zeros(max(n, 1), np.int32)
        _check(lib().plp_item_sequence(self._p, 0 if order == "volume" else 1, _ptr(ti), _ptr(cp)))
        return list(zip(ti[:n].tolist(), cp[:n].tolist()))


# ---------------------------------------------------------------------------
# results
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class RestartResult:
    n_boxes: int
    volume: int
    score: float
    fallback: bool
    n_passes: int
    seed: int
    err: int
    time_s: float


class Result:
    """All restarts of one instance."""

    def __init__(self, ptr):
        self._p = ctypes.c_void_p(ptr)

    def __del__(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.plp_result_free(self._p)
            self._p = None

    @property
    def restarts(self) -> int:
        return lib().plp_result_restarts(self._p)

    def summary(self, k: int) -> RestartResult:
        s = Summary()
        _check(lib().plp_result_summary(self._p, k, ctypes.byref(s)))
        return RestartResult(s.n_boxes, s.volume, s.score, bool(s.fallback), s.n_passes, s.seed,
                             s.err, s.time_s)

    def summaries(self) -> list:
        return [self.summary(k) for k in range(self.restarts)]

    def placements(self, k: int) -> list:
        n = ctypes.c_int32()
        _check(lib().plp_result_placements(self._p, k, None, 0, ctypes.byref(n)))
        buf = np.zeros(max(7 * n.value, 7), np.int32)
        _check(lib().plp_result_placements(self._p, k, _ptr(buf), n.value, ctypes.byref(n)))
        return [tuple(int(v) for v in buf[7 * i:7 * i + 7]) for i in range(n.value)]

    def best(self):
        r, f = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().plp_result_best(self._p, ctypes.byref(r), ctypes.byref(f)))
        return r.value, bool(f.value)

    def work(self, k: int):
        """(aabb_tests, pairs) of the reference algorithm for restart k."""
        t, p = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().plp_result_work(self._p, k, ctypes.byref(t), ctypes.byref(p)))
        return t.value, p.value

    def json(self, k: int) -> str:
        need = ctypes.c_size_t()
        _check(lib().plp_result_json(self._p, k, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value + 1)
        _check(lib().plp_result_json(self._p, k, buf, need.value + 1, ctypes.byref(need)))
        return buf.value.decode()


def run_plain(inst: Instance, **kw) -> Result:
    """Plain path: host decode loop, one device feasibility launch per step."""
    o = make_opts(**kw)
    out = ctypes.c_void_p()
    _check(lib().plp_run_plain(inst._p, ctypes.byref(o), ctypes.byref(out)))
    return Result(out.value)


# ---------------------------------------------------------------------------
# handle: batched persistent solver + serving loop
# ---------------------------------------------------------------------------
class Handle:
    def __init__(self, budget_bytes: int = 0, device: int = 0):
        out = ctypes.c_void_p()
        _check(lib().plp_create(budget_bytes, device, ctypes.byref(out)))
        self._p = ctypes.c_void_p(out.value)

    def close(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.plp_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_tile(self, P: int = 0, C: int = 0, G: int = 0, D: int = 0, M: int = 0):
        _check(lib().plp_set_tile(self._p, P, C, G, D, M), self._p)

    def serve_counters(self) -> dict:
        """Serving launches, requests they served, re-runs on the wave path's
        code, and eligible requests sent to the waves."""
        v = [ctypes.c_int64() for _ in range(4)]
        _check(lib().plp_serve_counters(self._p, *[ctypes.byref(x) for x in v]), self._p)
        return dict(zip(("launches", "served", "fallbacks", "waved"), (x.value for x in v)))

    def debug_sync_bound(self, wait_limit: int = 0, skip_warp: int = -1):
        """Test hook of the multi-warp decoders' bounded barrier wait."""
        _check(lib().plp_debug_sync_bound(self._p, wait_limit, skip_warp), self._p)

    def autotune(self, instances, opts, max_decodes: int = 0) -> tuple:
        """Times candidate tiles on a sample of the workload and keeps the
        fastest for later solves; returns (P, C, G, D, M)."""
        insts = (ctypes.c_void_p * len(instances))(*[i._p.value for i in instances])
        oarr = (RunOpts * 1)(opts) if isinstance(opts, RunOpts) else (RunOpts * len(opts))(*opts)
        out = (ctypes.c_int32 * 5)()
        _check(lib().plp_autotune(self._p, insts, len(instances), oarr, len(oarr), max_decodes, out), self._p)
        return tuple(out)

    def solve(self, instances, opts) -> list:
        """opts: one RunOpts for all instances or a list with one per instance."""
        insts = (ctypes.c_void_p * len(instances))(*[i._p.value for i in instances])
        if isinstance(opts, RunOpts):
            oarr = (RunOpts * 1)(opts)
        else:
            oarr = (RunOpts * len(opts))(*opts)
        res = (ctypes.c_void_p * len(instances))()
        _check(lib().plp_solve(self._p, insts, len(instances), oarr, len(oarr), res), self._p)
        return [Result(res[i]) for i in range(len(instances))]

    def prepare(self, instances, opts) -> "Batch":
        return Batch(self, instances, opts)

    def submit(self, inst: Instance, opts: RunOpts) -> int:
        rid = ctypes.c_int64()
        _check(lib().plp_submit(self._p, inst._p, ctypes.byref(opts), ctypes.byref(rid)), self._p)
        return rid.value

    def poll(self, rid: int) -> int:
        return lib().plp_poll(self._p, rid)

    def wait(self, rid: int, timeout_ms: int = -1) -> int:
        return lib().plp_wait(self._p, rid, timeout_ms)

    def take(self, rid: int) -> Result:
        out = ctypes.c_void_p()
        _check(lib().plp_take_result(self._p, rid, ctypes.byref(out)), self._p)
        return Result(out.value)

    def cancel(self, rid: int):
        _check(lib().plp_cancel(self._p, rid), self._p)

    def times(self, rid: int):
        q, t = ctypes.c_double(), ctypes.c_double()
        _check(lib().plp_request_times(self._p, rid, ctypes.byref(q), ctypes.byref(t)), self._p)
        return q.value, t.value


class Batch:
    """Tables of a solve resident on the device; run() times the device work."""

    def __init__(self, handle: Handle, instances, opts):
        self._h = handle
        self._n = len(instances)
        insts = (ctypes.c_void_p * len(instances))(*[i._p.value for i in instances])
        oarr = (RunOpts * 1)(opts) if isinstance(opts, RunOpts) else (RunOpts * len(opts))(*opts)
        out = ctypes.c_void_p()
        _check(lib().plp_batch_prepare(handle._p, insts, len(instances), oarr, len(oarr), ctypes.byref(out)),
               handle._p)
        self._p = ctypes.c_void_p(out.value)

    def run(self):
        """Returns (device_ms, decoder_ms, launches) of one execution."""
        dm, km, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32()
        _check(lib().plp_batch_run(self._p, ctypes.byref(dm), ctypes.byref(km), ctypes.byref(nl)), self._h._p)
        return dm.value, km.value, nl.value

    @property
    def graph(self) -> bool:
        """True when the next run replays the batch's captured CUDA graph."""
        return bool(lib().plp_batch_graph(self._p))

    def fetch(self) -> list:
        res = (ctypes.c_void_p * self._n)()
        _check(lib().plp_batch_fetch(self._p, res), self._h._p)
        return [Result(res[i]) for i in range(self._n)]

    def io_bytes(self):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().plp_batch_io_bytes(self._p, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.plp_batch_free(self._p)
            self._p = None

    def __del__(self):
        self.close()


# ---------------------------------------------------------------------------
# one-step feasibility and kernel hooks
# ---------------------------------------------------------------------------
def feas_check_all(cand, ors, fast, L, W, H) -> np.ndarray:
    c = np.ascontiguousarray(np.asarray(cand, np.int32).reshape(-1, 3))
    o = np.ascontiguousarray(np.asarray(ors, np.int32).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(fast, np.int32).reshape(-1, 6))
    bits = np.zeros(max(len(c) * len(o), 1), np.uint8)
    _check(lib().plp_feas_check_all(_ptr(c), len(c), _ptr(o), len(o), _ptr(f), len(f), L, W, H,
                                    _ptr(bits)))
    return bits[:len(c) * len(o)]


def rng_dump(seeds, n_random=16, n_bits=16, k_bits=13, device=True):
    s = np.ascontiguousarray(np.asarray(seeds, np.int64))
    r = np.zeros(max(len(s) * n_random, 1), np.float64)
    b = np.zeros(max(len(s) * n_bits, 1), np.uint32)
    fn = lib().plp_rng_dump if device else lib().plp_rng_dump_host
    _check(fn(_ptr(s), len(s), n_random, n_bits, k_bits, _ptr(r), _ptr(b)))
    return r[:len(s) * n_random].reshape(len(s), n_random), b[:len(s) * n_bits].reshape(len(s), n_bits)


def fsr_score(packings, mu=0.2):
    """packings: list of lists of (type, x, y, z, w, d, h). Returns (scores, fsr lists)."""
    offs = np.zeros(len(packings) + 1, np.int32)
    for i, p in enumerate(packings):
        offs[i + 1] = offs[i] + len(p)
    rows = np.ascontiguousarray(np.asarray([r for p in packings for r in p] or [[0] * 7],
                                           np.int32).reshape(-1, 7))
    sc = np.zeros(max(len(packings), 1), np.float64)
    fs = np.zeros(max(int(offs[-1]), 1), np.float64)
    _check(lib().plp_fsr_score(_ptr(rows), _ptr(offs), len(packings), mu, _ptr(sc), _ptr(fs)))
    return sc[:len(packings)], [fs[offs[i]:offs[i + 1]].tolist() for i in range(len(packings))]


def item_order(instances, order="volume") -> list:
    arr = (ctypes.c_void_p * len(instances))(*[i._p.value for i in instances])
    offs = np.zeros(len(instances) + 1, np.int64)
    total = sum(i.info()[2] for i in instances)
    out = np.zeros(max(total, 1), np.int32)
    _check(lib().plp_item_order(arr, len(instances), 0 if order == "volume" else 1, _ptr(out), _ptr(offs)))
    return [out[offs[i]:offs[i + 1]].tolist() for i in range(len(instances))]


def py_repr(x: float) -> str:
    buf = ctypes.create_string_buffer(64)
    _check(lib().plp_py_repr(float(x), buf, 64))
    return buf.value.decode()


def selftest() -> str:
    need = ctypes.c_size_t()
    lib().plp_selftest(None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(need.value + 1)
    lib().plp_selftest(buf, need.value + 1, ctypes.byref(need))
    return buf.value.decode()
