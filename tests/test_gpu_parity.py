"""GPU path vs the CPU oracle: per-level unique-CS sets, counts, minimal cost, formulas.

All calls go through the C ABI (libltlgpu.so).  Integer work: comparisons are exact.
"""
import numpy as np
import pytest

import oracle as O
from ltlb200 import api, gen
from helpers import last_round_gap, lensum, load_fixture, on_the_fly_cases, row_set

pytestmark = pytest.mark.gpu

OPCODES = {"~": 0, "&": 1, "|": 2, "X": 3, "F": 4, "G": 5, "U": 6}


@pytest.fixture(scope="module")
def engine():
    e = api.Engine(slots_log2=24, cache_bytes=4 << 30, max_rows=8 << 20)
    yield e
    e.close()


def gpu_levels(engine, inst, max_cost, **kw):
    res = engine.learn(inst, max_cost=max_cost, stop_at_found=False, **kw)
    starts = engine.level_starts(max_cost + 2)
    rows, par = engine.read_rows(0, starts[max_cost + 1])
    return res, starts, rows, par


def assert_levels_equal(inst, engine, costs, max_cost, neg_type, schedule=api.SCHEDULE_FUSED, oracle_key=O.KEY_EXACT,
                        key_mode=api.KEY_EXACT, rlx_type=3):
    res, starts, rows, par = gpu_levels(engine, inst, max_cost, costs=costs, neg_type=neg_type, schedule=schedule,
                                        key_mode=key_mode, rlx_type=rlx_type)
    assert res.device_flags & ~1 == 0, res.device_flags
    ref = O.learn(inst, costs=costs, max_cost=max_cost, neg_type=neg_type, stop_at_found=False, key_mode=oracle_key,
                  cache_rows=8 << 20)
    for c in range(costs[0], max_cost + 1):
        mine = rows[starts[c]:starts[c + 1]]
        theirs = ref.level_rows(c)
        assert len(mine) == len(theirs), (c, len(mine), len(theirs))
        if key_mode == api.KEY_EXACT:
            assert row_set(mine) == row_set(theirs), c
    return res, ref, rows, par, starts


def check_parents(inst, rows, par, starts, max_cost):
    """Every stored row equals its operator applied to its parent rows."""
    n = inst.n
    mask = (np.uint64(1) << inst.lengths.astype(np.uint64)) - np.uint64(1)
    nal = len(inst.alphabet)
    for r in range(nal, starts[max_cost + 1]):
        p = int(par[r])
        op, l, rr = (p >> 60) & 7, (p >> 30) & 0x3FFFFFFF, p & 0x3FFFFFFF
        out, out2 = O.apply_op(op, rows[l], rows[rr] if op in (1, 2, 6) else None, mask)
        assert np.array_equal(out, rows[r]), (r, op, l, rr)
    assert n == rows.shape[1]


@pytest.mark.parametrize("name,max_cost,neg", [("ham1_len3.trace", 7, 1), ("ham1_len4.trace", 7, 2),
                                               ("ham2_len3.trace", 7, 1), ("f10x10_p3_s0.trace", 5, 2),
                                               ("deep8x8_p3_s508.trace", 6, 1), ("e10x2_p3_s1.trace", 6, 1)])
def test_level_sets_fixtures(engine, name, max_cost, neg):
    inst = load_fixture(name)
    res, ref, rows, par, starts = assert_levels_equal(inst, engine, [1] * 8, max_cost, neg)
    check_parents(inst, rows, par, starts, max_cost)


@pytest.mark.parametrize("costs", [[1, 2, 1, 1, 2, 3, 3, 2], [2, 1, 3, 2, 1, 1, 2, 3]])
def test_level_sets_skewed_costs(engine, costs):
    inst = load_fixture("deep8x8_p3_s512.trace")
    assert_levels_equal(inst, engine, costs, 9, 2)


def test_level_sets_cfg1_shape(engine):
    inst = gen.generate(450, 2, 20, 20, 8, 16, 0.5, 8)
    assert_levels_equal(inst, engine, [1] * 8, 7, 1)


def test_level_sets_thousand_traces(engine):
    inst = gen.generate(2, 3, 500, 500, 16, 32, 0.5, 9)
    assert_levels_equal(inst, engine, [1] * 8, 6, 1)


def test_per_block_schedule_matches_oracle_progress(engine):
    inst = load_fixture("deep8x8_p3_s530.trace")
    res = engine.learn(inst, max_cost=7, stop_at_found=False, neg_type=1, schedule=api.SCHEDULE_PER_BLOCK)
    ref = O.learn(inst, max_cost=7, stop_at_found=False, neg_type=1)
    mine = [(b["cost"], b["op"], b["all_before"], b["stored_before"], b["to_check"]) for b in res.blocks]
    theirs = [p for p in ref.progress if p[1] != "A"]
    assert mine == theirs


@pytest.mark.parametrize("seed", range(8))
def test_found_cost_equals_oracle(engine, seed):
    inst = gen.generate(seed, 2, 20, 20, 8, 16, 0.5, 5)
    res = engine.learn(inst, neg_type=1)
    ref = O.learn(inst, neg_type=1)
    assert res.status == api.FOUND and ref.status == O.FOUND
    assert res.cost == ref.cost
    assert O.separates(res.formula, inst), res.formula
    assert O.formula_cost(res.formula) == res.cost


@pytest.mark.parametrize("seed", [2, 3, 8, 19])
def test_found_cost_thousand_traces(engine, seed):
    inst = gen.generate(seed, 3, 500, 500, 16, 32, 0.5, 9)
    res = engine.learn(inst, neg_type=1)
    ref = O.learn(inst, neg_type=1, threads=0, cache_rows=2 << 20, keep_rows=False)
    assert res.cost == ref.cost
    assert O.separates(res.formula, inst)
    assert O.formula_cost(res.formula) == res.cost


def test_hash64_mode_equals_exact_sets_here(engine):
    inst = gen.generate(450, 2, 20, 20, 8, 16, 0.5, 8)
    a = engine.learn(inst, max_cost=6, stop_at_found=False, neg_type=1, key_mode=api.KEY_HASH64)
    ref = O.learn(inst, max_cost=6, stop_at_found=False, neg_type=1, key_mode=O.KEY_HASH64)
    assert a.rows == ref.num_rows


@pytest.mark.parametrize("rtype", [1, 2, 3])
def test_reference_keys_level_counts(engine, rtype):
    inst = gen.generate(450, 2, 20, 20, 8, 16, 0.5, 8)
    assert lensum(inst) > 126
    # level 2 is built only from letters, so its relaxed key set is representative-independent
    res = engine.learn(inst, max_cost=2, stop_at_found=False, neg_type=1, key_mode=api.KEY_REF, rlx_type=rtype)
    ref = O.learn(inst, max_cost=2, stop_at_found=False, neg_type=1, key_mode=rtype)
    assert res.rows == ref.num_rows


def test_device_operators_and_fingerprint_bit_exact():
    rng = np.random.default_rng(3)
    count, n = 50, 101
    lens = rng.integers(1, 64, size=n)
    mask = np.array([(1 << int(l)) - 1 for l in lens], dtype=np.uint64)
    a = rng.integers(0, 2 ** 63, size=(count, n), dtype=np.uint64) & mask
    b = rng.integers(0, 2 ** 63, size=(count, n), dtype=np.uint64) & mask
    for op in range(7):
        out, out2, fp = api.device_apply_op(op, a, b if op in (1, 2, 6) else None, mask)
        for r in range(count):
            o1, o2 = O.apply_op(op, a[r], b[r], mask)
            assert np.array_equal(out[r], o1), (op, r)
            assert int(fp[r]) == O.fp64(o1)
            if op == 6:
                assert np.array_equal(out2[r], o2)
                assert int(fp[count + r]) == O.fp64(o2)


def test_letter_hit_and_limits(engine):
    inst = gen.generate(400, 2, 20, 20, 8, 16, 0.5, 5)  # 'p' separates
    res = engine.learn(inst)
    assert res.status == api.FOUND and res.cost == 1 and res.formula == "p"
    big = load_fixture("len64.trace")
    res = engine.learn(big)
    assert res.status == api.INPUT_LIMITS and res.formula == "see_the_error"
    over = load_fixture("over64.trace")
    res = engine.learn(over, limit_traces=True)
    assert res.status == api.INPUT_LIMITS
    res = engine.learn(over)
    ref = O.learn(over)
    assert res.cost == ref.cost



@pytest.mark.parametrize("costs", [(1,) * 8, (1, 2, 1, 1, 2, 2, 2, 2)])
def test_on_the_fly_regime_matches_oracle(costs):
    """Caches that hold exactly the rows through level k: level k + 1 overflows, the engine
    switches to the reference's on-the-fly regime (ltli6463.cu:1021-1027, 1202-1206,
    1442-1443) and checks the following levels without storing; status, cost, candidate
    count and the switch equal the oracle's, and a find separates the traces."""
    inst = gen.generate(3, 3, 30, 30, 6, 14, 0.5, 7)
    ex, cases = on_the_fly_cases(inst, costs)
    assert len(cases) >= 3
    for k, cap in cases:
        ref = O.learn(inst, costs=costs, neg_type=1, max_cost=14, cache_rows=cap, keep_rows=False)
        with api.Engine(slots_log2=20, cache_bytes=64 << 20, max_rows=cap) as e:
            res = e.learn(inst, costs=costs, neg_type=1, max_cost=14)
        assert res.device_flags & ~1 == 0, (k, res.device_flags)
        assert res.on_the_fly and ref.on_the_fly and res.rows == cap, k
        assert (res.status, res.cost) == ((api.FOUND if ref.status == O.FOUND else api.NOT_FOUND), ref.cost), k
        if res.status == api.FOUND:
            assert O.separates(res.formula, inst) and O.formula_cost(res.formula, costs) == res.cost
        else:
            assert res.cost == k + 1 + last_round_gap(costs)
            assert res.all_ltls == ref.all_ltls, k

def test_engine_reuse_many_instances(engine):
    # hash-set generations: later instances must not see earlier instances' slots
    for seed in range(12):
        inst = gen.generate(1000 + seed, 3, 30, 30, 5, 20, 0.5, 6)
        res = engine.learn(inst, neg_type=1)
        ref = O.learn(inst, neg_type=1)
        assert res.cost == ref.cost, seed
        assert O.separates(res.formula, inst)


def _golden_exact_runs():
    from helpers import reference_runs
    runs = reference_runs()
    if not runs:
        return []
    out = []
    for r in runs["runs"]:
        inst = load_fixture(r["file"])
        if r["final"]["limits_error"] or lensum(inst) > 126:
            continue
        out.append(r)
    return out


@pytest.mark.parametrize("run", _golden_exact_runs(), ids=lambda r: r["id"])
def test_gpu_matches_reference_outputs(engine, run):
    """Per-block schedule vs the reference binary's own progress lines (exact regime)."""
    inst = load_fixture(run["file"])
    res = engine.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"],
                       schedule=api.SCHEDULE_PER_BLOCK, limit_traces=True)
    mine = [[b["cost"], b["op"], b["all_before"], b["stored_before"], b["to_check"]] for b in res.blocks]
    ref = [p for p in run["progress"] if p[1] != "A"]
    assert mine == ref
    fin = run["final"]
    assert res.cost == fin["cost"] and res.all_ltls == fin["all_ltls"]
    if fin["formula"] == "not_found":
        assert res.status == api.NOT_FOUND and res.formula == "not_found"
    else:
        assert res.status == api.FOUND
        assert O.separates(res.formula, inst)
        assert O.formula_cost(res.formula, run["costs"]) == fin["cost"]


@pytest.mark.parametrize("run", _golden_exact_runs(), ids=lambda r: r["id"])
def test_fused_count_matches_reference_outputs(engine, run):
    """The default (fused) schedule against the reference binary's final lines: the same cost
    and the same "Number of All LTLs", which counts a found level through the first block of
    the reference's order that holds an accepting candidate (ltli6463.cu:1232-1234), whichever
    warp finds first on the device."""
    inst = load_fixture(run["file"])
    fin = run["final"]
    for _ in range(3):
        res = engine.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"],
                           limit_traces=True)
        assert (res.cost, res.all_ltls) == (fin["cost"], fin["all_ltls"])


def test_batch_learn_matches_single_engine():
    insts = [gen.generate(2000 + s, 3, 40, 40, 5, 20, 0.5, 6) for s in range(16)]
    with api.Batch(workers=4, slots_log2=22, cache_bytes=1 << 30, max_rows=1 << 20) as pool:
        res = pool.learn(insts, neg_type=1)
    for inst, r in zip(insts, res):
        ref = O.learn(inst, neg_type=1)
        assert r.status == api.FOUND and r.cost == ref.cost
        assert O.separates(r.formula, inst)
