"""ctypes wrapper of the CPU oracle (oracle/ltl_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU-baseline
leg of bench.py as the checker, never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libltloracle.so")

KEY_EXACT, KEY_REF1, KEY_REF2, KEY_REF3, KEY_HASH64 = range(5)
FOUND, NOT_FOUND, INPUT_LIMITS, TIMEOUT, NO_MEMORY, BAD_ARGS, CHUNK_TOO_SMALL = range(7)
OPS = "~&|XFGU"


class Traces(C.Structure):
    _fields_ = [("num_pos", C.c_int32), ("num_neg", C.c_int32), ("alphabet", C.c_char_p),
                ("steps", C.POINTER(C.c_uint32)), ("offsets", C.POINTER(C.c_int32))]


class Options(C.Structure):
    _fields_ = [("cost_fun", C.c_int32 * 8), ("max_cost", C.c_int32), ("key_mode", C.c_int32),
                ("neg_type", C.c_int32), ("stop_at_found", C.c_int32), ("threads", C.c_int32),
                ("limit_traces", C.c_int32), ("pad_", C.c_int32), ("cache_rows", C.c_int64),
                ("temp_rows", C.c_int64), ("time_limit_s", C.c_double)]


class Progress(C.Structure):
    _fields_ = [("cost", C.c_int32), ("op", C.c_int32), ("all_ltls", C.c_uint64), ("stored", C.c_int64),
                ("to_check", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("cost", C.c_int32), ("all_ltls", C.c_uint64), ("formula", C.c_void_p),
                ("n", C.c_int32), ("alphabet_size", C.c_int32), ("num_rows", C.c_int64),
                ("rows", C.POINTER(C.c_uint64)), ("row_op", C.POINTER(C.c_int8)),
                ("row_left", C.POINTER(C.c_int32)), ("row_right", C.POINTER(C.c_int32)),
                ("num_costs", C.c_int32), ("pad_", C.c_int32), ("level_start", C.POINTER(C.c_int64)),
                ("level_candidates", C.POINTER(C.c_uint64)), ("num_progress", C.c_int32),
                ("found_op", C.c_int32), ("progress", C.POINTER(Progress)), ("seconds", C.c_double),
                ("evaluated", C.c_uint64), ("on_the_fly", C.c_int32), ("threads_used", C.c_int32),
                ("internal_", C.c_void_p)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.lo_learn.argtypes = [C.POINTER(Traces), C.POINTER(Options), C.POINTER(Result)]
        L.lo_result_free.argtypes = [C.POINTER(Result)]
        L.lo_default_options.argtypes = [C.POINTER(Options)]
        L.lo_eval.argtypes = [C.c_char_p, C.POINTER(Traces), C.POINTER(C.c_uint8)]
        L.lo_formula_cost.argtypes = [C.c_char_p, C.POINTER(C.c_int32)]
        L.lo_formula_cost.restype = C.c_int64
        L.lo_fp64.argtypes = [C.POINTER(C.c_uint64), C.c_int32]
        L.lo_fp64.restype = C.c_uint64
        L.lo_ref_key.argtypes = [C.POINTER(C.c_uint64), C.c_int32, C.POINTER(C.c_uint8), C.c_int32, C.c_int32,
                                 C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.lo_apply_op.argtypes = [C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64), C.c_int32, C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def _traces(inst):
    steps = np.ascontiguousarray(inst.steps, dtype=np.uint32)
    offs = np.ascontiguousarray(inst.offsets, dtype=np.int32)
    alpha = inst.alphabet.encode()
    t = Traces(inst.num_pos, inst.num_neg, alpha, steps.ctypes.data_as(C.POINTER(C.c_uint32)),
               offs.ctypes.data_as(C.POINTER(C.c_int32)))
    return t, (steps, offs, alpha)


def _u64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


class OracleRun:
    """Outcome of one oracle enumeration, with copies of the language cache."""

    def __init__(self, res: Result, keep_rows: bool):
        self.status = res.status
        self.cost = res.cost
        self.all_ltls = res.all_ltls
        self.formula = C.string_at(res.formula).decode() if res.formula else ""
        self.n = res.n
        self.num_rows = res.num_rows
        self.seconds = res.seconds
        self.evaluated = res.evaluated
        self.on_the_fly = bool(res.on_the_fly)
        self.threads = res.threads_used
        self.found_op = res.found_op
        self.level_start = ([res.level_start[i] for i in range(res.num_costs + 1)] if res.level_start else [])
        self.level_candidates = ([res.level_candidates[i] for i in range(res.num_costs + 1)]
                                 if res.level_candidates else [])
        self.progress = [(p.cost, chr(p.op), p.all_ltls, p.stored, p.to_check)
                         for p in (res.progress[i] for i in range(res.num_progress))] if res.progress else []
        if keep_rows and res.num_rows > 0:
            w = res.num_rows * max(res.n, 1)
            self.rows = np.ctypeslib.as_array(res.rows, shape=(w,)).copy().reshape(res.num_rows, max(res.n, 1))
            self.row_op = np.ctypeslib.as_array(res.row_op, shape=(res.num_rows,)).copy()
            self.row_left = np.ctypeslib.as_array(res.row_left, shape=(res.num_rows,)).copy()
            self.row_right = np.ctypeslib.as_array(res.row_right, shape=(res.num_rows,)).copy()
        else:
            self.rows = None

    def level_rows(self, cost: int) -> np.ndarray:
        a, b = self.level_start[cost], self.level_start[cost + 1]
        return self.rows[a:b]

    def level_set(self, cost: int) -> set:
        return {r.tobytes() for r in self.level_rows(cost)}


def learn(inst, costs=(1,) * 8, max_cost=500, key_mode=KEY_EXACT, neg_type=1, stop_at_found=True,
          threads=1, limit_traces=False, cache_rows=1 << 20, temp_rows=0, time_limit_s=0.0,
          keep_rows=True) -> OracleRun:
    L = lib()
    t, keep = _traces(inst)
    o = Options()
    L.lo_default_options(C.byref(o))
    for i, c in enumerate(costs):
        o.cost_fun[i] = int(c)
    o.max_cost = int(max_cost)
    o.key_mode = int(key_mode)
    o.neg_type = int(neg_type)
    o.stop_at_found = int(bool(stop_at_found))
    o.threads = int(threads)
    o.limit_traces = int(bool(limit_traces))
    o.cache_rows = int(cache_rows)
    o.temp_rows = int(temp_rows)
    o.time_limit_s = float(time_limit_s)
    r = Result()
    L.lo_learn(C.byref(t), C.byref(o), C.byref(r))
    try:
        return OracleRun(r, keep_rows)
    finally:
        L.lo_result_free(C.byref(r))


def evaluate(formula: str, inst) -> np.ndarray:
    """Per trace: does the formula hold at position 0 (independent positional evaluator)."""
    L = lib()
    t, keep = _traces(inst)
    out = np.zeros(inst.n, dtype=np.uint8)
    rc = L.lo_eval(formula.encode(), C.byref(t), out.ctypes.data_as(C.POINTER(C.c_uint8)))
    if rc != 0:
        raise ValueError(f"malformed formula: {formula!r}")
    return out.astype(bool)


def separates(formula: str, inst) -> bool:
    h = evaluate(formula, inst)
    return bool(h[:inst.num_pos].all() and not h[inst.num_pos:].any())


def formula_cost(formula: str, costs=(1,) * 8) -> int:
    cf = (C.c_int32 * 8)(*costs)
    return int(lib().lo_formula_cost(formula.encode(), cf))


def fp64(cs: np.ndarray) -> int:
    cs = np.ascontiguousarray(cs, dtype=np.uint64)
    return int(lib().lo_fp64(_u64p(cs), len(cs)))


def ref_key(cs: np.ndarray, lens: np.ndarray, rtype: int):
    cs = np.ascontiguousarray(cs, dtype=np.uint64)
    ln = np.ascontiguousarray(lens, dtype=np.uint8)
    h, l = C.c_uint64(), C.c_uint64()
    lib().lo_ref_key(_u64p(cs), len(cs), ln.ctypes.data_as(C.POINTER(C.c_uint8)), int(ln.astype(np.int64).sum()),
                     rtype, C.byref(h), C.byref(l))
    return h.value, l.value


def apply_op(op: int, a: np.ndarray, b: np.ndarray | None, mask: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    bb = np.ascontiguousarray(b if b is not None else a, dtype=np.uint64)
    m = np.ascontiguousarray(mask, dtype=np.uint64)
    out = np.zeros_like(a)
    out2 = np.zeros_like(a)
    lib().lo_apply_op(op, _u64p(a), _u64p(bb), _u64p(m), len(a), _u64p(out), _u64p(out2))
    return out, out2
