"""ctypes binding of include/ltlgpu.h (libltlgpu.so, built in-tree for sm_100a).

The library is the product path: there is no CPU fallback.  If the shared
library is missing, ``lib()`` raises instead of degrading.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from .gen import Instance

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libltlgpu.so")
CLI_PATH = os.path.join(HERE, "_build", "ltli6463")

ABI_VERSION = 2  # LTLG_ABI_VERSION of include/ltlgpu.h
KEY_EXACT, KEY_REF, KEY_HASH64 = 0, 1, 2
SCHEDULE_FUSED, SCHEDULE_PER_BLOCK = 0, 1
ORDER_PLAIN, ORDER_LEARNED = 0, 1
(FOUND, NOT_FOUND, INPUT_LIMITS, TIMEOUT, NO_MEMORY, BAD_ARGS, CUDA_ERROR, DEVICE_WAIT, TABLE_FULL,
 NO_DEVICE, FORMULA_TOO_LONG) = range(11)
FORMULA_MAX_BYTES = 1280
OPS = "~&|XFGU"

EXPORTED = [
    "ltlg_abi_version", "ltlg_status_string", "ltlg_default_engine_config", "ltlg_default_options",
    "ltlg_engine_create", "ltlg_engine_destroy", "ltlg_engine_learn", "ltlg_learn", "ltlg_result_free",
    "ltlg_engine_read_rows", "ltlg_engine_level_starts", "ltlg_device_apply_op", "ltlg_read_scarlet",
    "ltlg_traces_free", "ltlg_engine_stream", "ltlg_batch_create", "ltlg_batch_destroy", "ltlg_batch_learn",
    "ltlg_batch_stream", "ltlg_learn_noalloc", "ltlg_block_features", "ltlg_engine_set_scorer",
    "ltlg_batch_set_scorer", "ltlg_engine_label_blocks", "ltlg_scorer_forward", "ltlg_scorer_grad",
    "ltlg_scorer_train", "ltlg_evaluate", "ltlg_engine_hold_slot",
]
SCORER_FEATURES = 32
SCORER_PARAMS = 6337


class Traces(C.Structure):
    _fields_ = [("num_pos", C.c_int32), ("num_neg", C.c_int32), ("alphabet", C.c_char_p),
                ("steps", C.POINTER(C.c_uint32)), ("offsets", C.POINTER(C.c_int32))]


class EngineConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots_log2", C.c_int32), ("cache_bytes", C.c_int64),
                ("max_rows", C.c_int64), ("max_traces", C.c_int32), ("block_threads", C.c_int32),
                ("left_tile", C.c_int32), ("right_chunk", C.c_int32), ("unary_rows", C.c_int32),
                ("small_rows", C.c_int32), ("wait_spins", C.c_int32), ("pad_", C.c_int32),
                ("small_level", C.c_int64)]


class Options(C.Structure):
    _fields_ = [("cost_fun", C.c_int32 * 8), ("max_cost", C.c_int32), ("rlx_unq_chk_type", C.c_int32),
                ("neg_type", C.c_int32), ("key_mode", C.c_int32), ("schedule", C.c_int32), ("order", C.c_int32),
                ("stop_at_found", C.c_int32), ("limit_traces", C.c_int32), ("record_levels", C.c_int32),
                ("pad_", C.c_int32), ("time_limit_s", C.c_double)]


class LevelStat(C.Structure):
    _fields_ = [("cost", C.c_int32), ("blocks", C.c_int32), ("candidates", C.c_uint64), ("uniques", C.c_uint64),
                ("ms", C.c_double), ("plan_us", C.c_double), ("claim_us", C.c_double), ("start_us", C.c_double)]


class BlockStat(C.Structure):
    _fields_ = [("cost", C.c_int32), ("op", C.c_int32), ("left_cost", C.c_int32), ("right_cost", C.c_int32),
                ("stored_before", C.c_int64), ("all_before", C.c_uint64), ("to_check", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("cost", C.c_int32), ("all_ltls", C.c_uint64), ("evaluated", C.c_uint64),
                ("rows", C.c_int64), ("formula", C.c_void_p), ("seconds", C.c_double), ("device_ms", C.c_double),
                ("num_levels", C.c_int32), ("num_blocks", C.c_int32), ("levels", C.POINTER(LevelStat)),
                ("blocks", C.POINTER(BlockStat)), ("found_op", C.c_int32), ("device_flags", C.c_uint32),
                ("on_the_fly", C.c_int32), ("launches", C.c_int32)]


class BlockInfo(C.Structure):
    _fields_ = [("op", C.c_int32), ("cost", C.c_int32), ("c1", C.c_int32), ("lcost", C.c_int32),
                ("rcost", C.c_int32), ("position", C.c_int32), ("nblocks", C.c_int32), ("pad_", C.c_int32),
                ("lrows", C.c_int64), ("rrows", C.c_int64), ("candidates", C.c_int64), ("level_cands", C.c_int64),
                ("lstat", C.c_int64 * 2), ("rstat", C.c_int64 * 2), ("npos", C.c_int32), ("nneg", C.c_int32),
                ("nalpha", C.c_int32), ("pad2_", C.c_int32)]


class BlockRecord(C.Structure):
    _fields_ = [("cost", C.c_int32), ("op", C.c_int32), ("lcost", C.c_int32), ("rcost", C.c_int32),
                ("position", C.c_int32), ("won", C.c_int32), ("candidates", C.c_int64),
                ("features", C.c_float * SCORER_FEATURES)]


class TrainConfig(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("pos_weight", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_uint64)]


_lib = None


def lib():
    """Load libltlgpu.so; raises if it was not built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        L.ltlg_status_string.restype = C.c_char_p
        L.ltlg_default_engine_config.argtypes = [C.POINTER(EngineConfig)]
        L.ltlg_default_options.argtypes = [C.POINTER(Options)]
        L.ltlg_engine_create.argtypes = [C.POINTER(EngineConfig), C.POINTER(C.c_void_p)]
        L.ltlg_engine_destroy.argtypes = [C.c_void_p]
        L.ltlg_engine_learn.argtypes = [C.c_void_p, C.POINTER(Traces), C.POINTER(Options), C.POINTER(Result)]
        L.ltlg_learn.argtypes = [C.POINTER(Traces), C.POINTER(Options), C.POINTER(Result)]
        L.ltlg_result_free.argtypes = [C.POINTER(Result)]
        L.ltlg_engine_read_rows.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(C.c_uint64),
                                            C.POINTER(C.c_uint64)]
        L.ltlg_engine_level_starts.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.c_int32]
        L.ltlg_device_apply_op.argtypes = [C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint64), C.c_int32, C.c_int32, C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.ltlg_read_scarlet.argtypes = [C.c_char_p, C.POINTER(Traces)]
        L.ltlg_traces_free.argtypes = [C.POINTER(Traces)]
        L.ltlg_engine_stream.argtypes = [C.c_void_p]
        L.ltlg_engine_stream.restype = C.c_void_p
        L.ltlg_batch_create.argtypes = [C.POINTER(EngineConfig), C.c_int32, C.POINTER(C.c_void_p)]
        L.ltlg_batch_destroy.argtypes = [C.c_void_p]
        L.ltlg_batch_learn.argtypes = [C.c_void_p, C.POINTER(Traces), C.c_int32, C.POINTER(Options),
                                       C.POINTER(Result)]
        L.ltlg_batch_stream.argtypes = [C.c_void_p, C.c_int32]
        L.ltlg_batch_stream.restype = C.c_void_p
        fp = C.POINTER(C.c_float)
        L.ltlg_block_features.argtypes = [C.POINTER(BlockInfo), fp]
        L.ltlg_block_features.restype = None
        L.ltlg_engine_set_scorer.argtypes = [C.c_void_p, fp, C.c_int32]
        L.ltlg_batch_set_scorer.argtypes = [C.c_void_p, fp, C.c_int32]
        L.ltlg_engine_label_blocks.argtypes = [C.c_void_p, C.POINTER(Traces), C.POINTER(Options),
                                               C.POINTER(BlockRecord), C.c_int32, C.POINTER(C.c_int32),
                                               C.POINTER(Result)]
        L.ltlg_scorer_forward.argtypes = [fp, fp, C.c_int32, fp]
        L.ltlg_scorer_grad.argtypes = [fp, fp, fp, C.c_int32, C.c_float, fp, fp]
        L.ltlg_scorer_train.argtypes = [fp, fp, fp, C.c_int32, C.POINTER(TrainConfig), fp]
        L.ltlg_evaluate.argtypes = [C.POINTER(Traces), C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint8)]
        L.ltlg_engine_hold_slot.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_int32]
        _lib = L
    return _lib


def status_string(code: int) -> str:
    return lib().ltlg_status_string(int(code)).decode()


def _u64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _traces(inst: Instance):
    steps = np.ascontiguousarray(inst.steps, dtype=np.uint32)
    offs = np.ascontiguousarray(inst.offsets, dtype=np.int32)
    alpha = inst.alphabet.encode()
    t = Traces(inst.num_pos, inst.num_neg, alpha, steps.ctypes.data_as(C.POINTER(C.c_uint32)),
               offs.ctypes.data_as(C.POINTER(C.c_int32)))
    return t, (steps, offs, alpha)


@dataclasses.dataclass
class LearnResult:
    status: int
    cost: int
    all_ltls: int
    evaluated: int
    rows: int
    formula: str
    seconds: float
    device_ms: float
    levels: list
    blocks: list
    found_op: int
    device_flags: int
    on_the_fly: bool
    launches: int

    @property
    def found(self) -> bool:
        return self.status == FOUND


def _result(r: Result) -> LearnResult:
    levels = [dict(cost=r.levels[i].cost, blocks=r.levels[i].blocks, candidates=r.levels[i].candidates,
                   uniques=r.levels[i].uniques, ms=r.levels[i].ms, plan_us=r.levels[i].plan_us,
                   claim_us=r.levels[i].claim_us, start_us=r.levels[i].start_us) for i in range(r.num_levels)]
    blocks = [dict(cost=b.cost, op=OPS[b.op], left_cost=b.left_cost, right_cost=b.right_cost,
                   stored_before=b.stored_before, all_before=b.all_before, to_check=b.to_check)
              for b in (r.blocks[i] for i in range(r.num_blocks))]
    return LearnResult(r.status, r.cost, r.all_ltls, r.evaluated, r.rows,
                       C.string_at(r.formula).decode() if r.formula else "", r.seconds, r.device_ms, levels, blocks,
                       r.found_op, r.device_flags, bool(r.on_the_fly), r.launches)


def make_options(costs=(1,) * 8, max_cost=500, rlx_type=3, neg_type=2, key_mode=KEY_EXACT,
                 schedule=SCHEDULE_FUSED, order=ORDER_PLAIN, stop_at_found=True, limit_traces=False,
                 record_levels=False, time_limit_s=0.0) -> Options:
    o = Options()
    lib().ltlg_default_options(C.byref(o))
    for i, c in enumerate(costs):
        o.cost_fun[i] = int(c)
    o.max_cost = int(max_cost)
    o.rlx_unq_chk_type = int(rlx_type)
    o.neg_type = int(neg_type)
    o.key_mode = int(key_mode)
    o.schedule = int(schedule)
    o.order = int(order)
    o.stop_at_found = int(bool(stop_at_found))
    o.limit_traces = int(bool(limit_traces))
    o.record_levels = int(bool(record_levels))
    o.time_limit_s = float(time_limit_s)
    return o


class Engine:
    """Device state for repeated learns: language cache, hash set, stream."""

    def __init__(self, device=0, slots_log2=27, cache_bytes=16 << 30, max_rows=64 << 20, max_traces=8192,
                 block_threads=1024, left_tile=4, right_chunk=16, unary_rows=32, small_rows=1, wait_spins=0,
                 small_level=0):
        L = lib()
        cfg = _engine_config(device, slots_log2, cache_bytes, max_rows, max_traces, block_threads, left_tile,
                             right_chunk, unary_rows, small_rows, wait_spins, small_level)
        h = C.c_void_p()
        rc = L.ltlg_engine_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"ltlg_engine_create failed: {status_string(rc)}")
        self._h = h
        self.config = cfg
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().ltlg_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def learn(self, inst: Instance, **kw) -> LearnResult:
        o = make_options(**kw)
        t, keep = _traces(inst)
        r = Result()
        lib().ltlg_engine_learn(self._h, C.byref(t), C.byref(o), C.byref(r))
        try:
            out = _result(r)
        finally:
            lib().ltlg_result_free(C.byref(r))
        self.n = inst.n
        return out

    @property
    def stream(self) -> int:
        """The engine's cudaStream_t as an integer handle."""
        return lib().ltlg_engine_stream(self._h) or 0

    def set_scorer(self, params: np.ndarray):
        """Load the block-order scorer (SCORER_PARAMS floats) for order=ORDER_LEARNED."""
        p = _f32(params, SCORER_PARAMS)
        rc = lib().ltlg_engine_set_scorer(self._h, _fp(p), SCORER_PARAMS)
        if rc != 0:
            raise RuntimeError(f"set_scorer failed: {status_string(rc)}")

    def label_blocks(self, inst: Instance, cap: int = 4096, **kw):
        """Learn in plain order, then label every block of the level of the find (holds an
        accepting candidate or not).  Returns (LearnResult, records: list of dicts,
        features: float32 [k, 32], won: int32 [k])."""
        o = make_options(**kw)
        t, keep = _traces(inst)
        recs = (BlockRecord * cap)()
        cnt = C.c_int32(0)
        r = Result()
        lib().ltlg_engine_label_blocks(self._h, C.byref(t), C.byref(o), recs, cap, C.byref(cnt), C.byref(r))
        try:
            out = _result(r)
        finally:
            lib().ltlg_result_free(C.byref(r))
        self.n = inst.n
        k = cnt.value
        feats = np.zeros((k, SCORER_FEATURES), dtype=np.float32)
        won = np.zeros(k, dtype=np.int32)
        meta = []
        for i in range(k):
            x = recs[i]
            feats[i] = np.frombuffer(x.features, dtype=np.float32, count=SCORER_FEATURES)
            won[i] = x.won
            meta.append(dict(cost=x.cost, op=OPS[x.op], lcost=x.lcost, rcost=x.rcost, position=x.position,
                             candidates=x.candidates, won=x.won))
        return out, meta, feats, won

    def hold_slot(self, cs: np.ndarray):
        """Fault injection for tests: the next learn finds the hash slot of this CS (exact keys)
        held by a publication that never comes, so its wait runs out (DEVICE_WAIT)."""
        a = np.ascontiguousarray(cs, dtype=np.uint64)
        rc = lib().ltlg_engine_hold_slot(self._h, _u64p(a), a.size)
        if rc != 0:
            raise RuntimeError(f"hold_slot failed: {status_string(rc)}")

    def level_starts(self, count: int) -> list:
        a = (C.c_int64 * count)()
        lib().ltlg_engine_level_starts(self._h, a, count)
        return list(a)

    def read_rows(self, first: int, count: int):
        rows = np.zeros((count, max(self.n, 1)), dtype=np.uint64)
        par = np.zeros(count, dtype=np.uint64)
        rc = lib().ltlg_engine_read_rows(self._h, first, count, _u64p(rows), _u64p(par))
        if rc != 0:
            raise RuntimeError(f"read_rows failed: {status_string(rc)}")
        return rows, par


def _engine_config(device=0, slots_log2=27, cache_bytes=16 << 30, max_rows=64 << 20, max_traces=8192,
                   block_threads=1024, left_tile=4, right_chunk=16, unary_rows=32, small_rows=1, wait_spins=0,
                   small_level=0) -> EngineConfig:
    cfg = EngineConfig()
    lib().ltlg_default_engine_config(C.byref(cfg))
    cfg.device, cfg.slots_log2, cfg.cache_bytes, cfg.max_rows = device, slots_log2, cache_bytes, max_rows
    cfg.max_traces, cfg.block_threads, cfg.left_tile = max_traces, block_threads, left_tile
    cfg.right_chunk, cfg.unary_rows, cfg.small_rows = right_chunk, unary_rows, small_rows
    cfg.wait_spins, cfg.small_level = wait_spins, small_level
    return cfg


class Batch:
    """Independent instances learned concurrently by `workers` engines (native threads)."""

    def __init__(self, workers=8, **engine_kw):
        cfg = _engine_config(**engine_kw)
        h = C.c_void_p()
        rc = lib().ltlg_batch_create(C.byref(cfg), int(workers), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"ltlg_batch_create failed: {status_string(rc)}")
        self._h = h
        self.workers = workers

    def close(self):
        if getattr(self, "_h", None):
            lib().ltlg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def stream(self, worker: int = 0) -> int:
        return lib().ltlg_batch_stream(self._h, worker) or 0

    def set_scorer(self, params: np.ndarray):
        p = _f32(params, SCORER_PARAMS)
        rc = lib().ltlg_batch_set_scorer(self._h, _fp(p), SCORER_PARAMS)
        if rc != 0:
            raise RuntimeError(f"set_scorer failed: {status_string(rc)}")

    def learn(self, instances, **kw) -> list:
        o = make_options(**kw)
        n = len(instances)
        arr = (Traces * n)()
        keep = []
        for i, inst in enumerate(instances):
            t, k = _traces(inst)
            arr[i] = t
            keep.append(k)
        res = (Result * n)()
        lib().ltlg_batch_learn(self._h, arr, n, C.byref(o), res)
        out = []
        for i in range(n):
            try:
                out.append(_result(res[i]))
            finally:
                lib().ltlg_result_free(C.byref(res[i]))
        return out


def learn(inst: Instance, **kw) -> LearnResult:
    """One-shot learn (the reference's LTLI): allocates, learns, frees."""
    o = make_options(**kw)
    t, keep = _traces(inst)
    r = Result()
    lib().ltlg_learn(C.byref(t), C.byref(o), C.byref(r))
    try:
        return _result(r)
    finally:
        lib().ltlg_result_free(C.byref(r))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a, size=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if size is not None and a.size != size:
        raise ValueError(f"expected {size} floats, got {a.size}")
    return a


def block_features(**info) -> np.ndarray:
    """The 32 features of a block (the library's host-side copy of the planner's function)."""
    b = BlockInfo()
    for k, v in info.items():
        if k in ("lstat", "rstat"):
            getattr(b, k)[:] = [int(x) for x in v]
        else:
            setattr(b, k, int(v))
    out = np.zeros(SCORER_FEATURES, dtype=np.float32)
    lib().ltlg_block_features(C.byref(b), _fp(out))
    return out


def scorer_forward(params: np.ndarray, features: np.ndarray) -> np.ndarray:
    """Logits of the scorer on the device (BF16 operands, FP32 sums)."""
    p = _f32(params, SCORER_PARAMS)
    x = _f32(features).reshape(-1, SCORER_FEATURES)
    out = np.zeros(x.shape[0], dtype=np.float32)
    rc = lib().ltlg_scorer_forward(_fp(p), _fp(x), x.shape[0], _fp(out))
    if rc != 0:
        raise RuntimeError(f"scorer_forward failed: {status_string(rc)}")
    return out


def scorer_grad(params: np.ndarray, features: np.ndarray, labels: np.ndarray, pos_weight: float = 1.0):
    """Gradient (and loss) of the mean weighted binary cross-entropy, computed on the device."""
    p = _f32(params, SCORER_PARAMS)
    x = _f32(features).reshape(-1, SCORER_FEATURES)
    y = _f32(labels)
    g = np.zeros(SCORER_PARAMS, dtype=np.float32)
    loss = C.c_float(0.0)
    rc = lib().ltlg_scorer_grad(_fp(p), _fp(x), _fp(y), x.shape[0], float(pos_weight), _fp(g), C.byref(loss))
    if rc != 0:
        raise RuntimeError(f"scorer_grad failed: {status_string(rc)}")
    return g, loss.value


def scorer_train(params: np.ndarray, features: np.ndarray, labels: np.ndarray, epochs=30, batch=1024, lr=2e-3,
                 pos_weight=1.0, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, seed=0):
    """Adam training on the device; returns (new params, per-epoch mean loss)."""
    p = _f32(params, SCORER_PARAMS).copy()
    x = _f32(features).reshape(-1, SCORER_FEATURES)
    y = _f32(labels)
    cfg = TrainConfig(int(epochs), int(batch), float(lr), float(pos_weight), float(beta1), float(beta2), float(eps),
                      float(weight_decay), int(seed))
    curve = np.zeros(max(int(epochs), 1), dtype=np.float32)
    rc = lib().ltlg_scorer_train(_fp(p), _fp(x), _fp(y), x.shape[0], C.byref(cfg), _fp(curve))
    if rc != 0:
        raise RuntimeError(f"scorer_train failed: {status_string(rc)}")
    return p, curve[:int(epochs)]


def evaluate(inst: Instance, formula: str):
    """The formula's CS on every trace (uint64, bit k = holds at position k) and whether it
    holds at position 0 (bool), computed on the device."""
    t, keep = _traces(inst)
    cs = np.zeros(max(inst.n, 1), dtype=np.uint64)
    holds = np.zeros(max(inst.n, 1), dtype=np.uint8)
    rc = lib().ltlg_evaluate(C.byref(t), formula.encode(), _u64p(cs), holds.ctypes.data_as(C.POINTER(C.c_uint8)))
    if rc != 0:
        raise ValueError(f"evaluate failed ({status_string(rc)}): {formula!r}")
    return cs[:inst.n], holds[:inst.n].astype(bool)


def separates(inst: Instance, formula: str) -> bool:
    """Holds at position 0 on every positive trace and on no negative one (device)."""
    _, h = evaluate(inst, formula)
    return bool(h[:inst.num_pos].all() and not h[inst.num_pos:].any())


def device_apply_op(op: int, a: np.ndarray, b: np.ndarray | None, lenmask: np.ndarray):
    """Apply one operator to rows of a (and b) on the device; returns (out, out2, fingerprints)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    count, n = a.shape
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.uint64)
    m = np.ascontiguousarray(lenmask, dtype=np.uint64)
    out = np.zeros_like(a)
    out2 = np.zeros_like(a)
    fp = np.zeros(2 * count, dtype=np.uint64)
    rc = lib().ltlg_device_apply_op(op, _u64p(a), None if bb is None else _u64p(bb), _u64p(m), n, count,
                                    _u64p(out), _u64p(out2), _u64p(fp))
    if rc != 0:
        raise RuntimeError(f"device_apply_op failed: {status_string(rc)}")
    return out, out2, fp


def read_scarlet(path: str) -> Instance:
    """Read a Scarlet file with the reference's rules (through the library's C++ reader)."""
    t = Traces()
    rc = lib().ltlg_read_scarlet(path.encode(), C.byref(t))
    if rc != 0:
        raise OSError(f"cannot read {path}")
    try:
        n = t.num_pos + t.num_neg
        offs = np.ctypeslib.as_array(t.offsets, shape=(n + 1,)).copy()
        total = int(offs[-1])
        steps = (np.ctypeslib.as_array(t.steps, shape=(total,)).copy() if total
                 else np.zeros(0, dtype=np.uint32))
        return Instance(t.num_pos, t.num_neg, t.alphabet.decode(), steps, offs)
    finally:
        lib().ltlg_traces_free(C.byref(t))
