"""The device paths the benchmark and the workloads run, against the CPU oracle.

Each engine knob below selects a different code path of the level kernel: work items of many
right rows per warp (large levels), left tiles of 2 and 8 rows (long rows and the autotuned
batch), the reference's relaxed keys, and the failure statuses a search can end with.  All
calls go through the C ABI; the work is integer, so sets and counts compare exactly.
"""
import numpy as np
import pytest

import oracle as O
from ltlb200 import api, gen
from helpers import edge_cases, lensum, load_fixture, reference_runs, row_set

pytestmark = pytest.mark.gpu

UNIT = [1] * 8
CFG3_COSTS = [1, 1, 1, 1, 1, 2, 2, 3]  # p ~ & | X F G U of the 5-proposition, 4000-trace shape


def assert_level_sets(eng, inst, max_cost, costs=UNIT, neg_type=1, **kw):
    """Every level's sorted set of unique CS rows (and its size) equals the oracle's."""
    res = eng.learn(inst, costs=costs, max_cost=max_cost, stop_at_found=False, neg_type=neg_type, **kw)
    assert res.device_flags & ~1 == 0, res.device_flags
    ref = O.learn(inst, costs=costs, max_cost=max_cost, neg_type=neg_type, stop_at_found=False, threads=0,
                  cache_rows=8 << 20)
    starts = eng.level_starts(max_cost + 2)
    for c in range(costs[0], max_cost + 1):
        theirs = ref.level_rows(c)
        assert starts[c + 1] - starts[c] == len(theirs), (c, starts[c + 1] - starts[c], len(theirs))
        if len(theirs):
            mine, _ = eng.read_rows(starts[c], starts[c + 1] - starts[c])
            assert row_set(mine) == row_set(theirs), c
    return res, ref


@pytest.fixture(scope="module")
def engine():
    e = api.Engine(slots_log2=24, cache_bytes=4 << 30, max_rows=8 << 20)
    yield e
    e.close()


@pytest.mark.parametrize("right_chunk,unary_rows", [(16, 32), (7, 5)])
def test_large_level_items_thousand_traces(right_chunk, unary_rows):
    """The 500 + 500-trace shape with every level cut into the large items (right_chunk right
    rows per tile, unary_rows source rows), through cost 7, where the default sizing gives
    these levels smaller items.  Odd sizes leave ragged item ends."""
    inst = gen.generate(2, 3, 500, 500, 16, 32, 0.5, 9)
    with api.Engine(slots_log2=24, cache_bytes=4 << 30, max_rows=8 << 20, small_level=1, right_chunk=right_chunk,
                    unary_rows=unary_rows) as e:
        assert_level_sets(e, inst, 7)


@pytest.mark.parametrize("tile", [2, 8])
@pytest.mark.parametrize("small_level", [0, 1])
def test_left_tiles_two_and_eight(tile, small_level):
    """Left tiles of 2 rows (the engine's choice for rows of 32 KB; U pairs one left row with
    each right row) and of 8 rows (the autotuner's pick for the batch), on small-level and
    large-level items, on the 1000-trace shape and on a 40-trace instance."""
    with api.Engine(slots_log2=24, cache_bytes=4 << 30, max_rows=8 << 20, left_tile=tile,
                    small_level=small_level) as e:
        assert_level_sets(e, gen.generate(2, 3, 500, 500, 16, 32, 0.5, 9), 6)
        assert_level_sets(e, load_fixture("cfg1_deep.trace"), 7)


def test_scale_shape_four_thousand_traces():
    """The 5-proposition shape with 2000 + 2000 traces of length 32-63 (rows of 32 KB, so a
    2-row left tile) under costs ~ = X = & = | = 1, F = G = 2, U = 3, through cost 7."""
    inst = gen.generate(1, 5, 2000, 2000, 32, 63, 0.3, 12)
    with api.Engine(slots_log2=24, cache_bytes=8 << 30, max_rows=1 << 20, max_traces=4000) as e:
        res, ref = assert_level_sets(e, inst, 7, costs=CFG3_COSTS)
        found = e.learn(inst, costs=CFG3_COSTS, neg_type=1)
    want = O.learn(inst, costs=CFG3_COSTS, neg_type=1, threads=0, cache_rows=1 << 20, keep_rows=False)
    assert found.status == api.FOUND and found.cost == want.cost
    assert O.separates(found.formula, inst) and O.formula_cost(found.formula, CFG3_COSTS) == found.cost


def _relaxed_golden_runs():
    runs = reference_runs()
    if not runs:
        return []
    return [r for r in runs["runs"] if not r["final"]["limits_error"] and lensum(load_fixture(r["file"])) > 126]


@pytest.mark.parametrize("run", _relaxed_golden_runs(), ids=lambda r: r["id"])
def test_reference_keys_match_reference_runs(engine, run):
    """The reference's relaxed keys (types 1/2/3, lenSum > 126) on the device.  Of the CSs that
    share a key in a level, the device keeps the candidate first in the reference's order
    (blocks in order, then thread index inside a block).  The per-block progress lines equal the
    oracle's exactly.  Against the reference binary's own progress lines the rule of the
    oracle's pinning applies: cost 2 is built from letters only and matches exactly, later
    stored counts within 1% (the reference keeps whichever thread wins its atomic race).  The
    final cost is the reference's.

    Enumerated to max_cost, every stored row is its parents' operator applied to them, and each
    level holds the oracle's number of rows with the oracle's set of keys while the levels below
    hold the oracle's rows.  Which CS represents a shared key can differ: a thread index counts
    rows of the operand levels in the order they were stored, and the device (like the
    reference) stores a level's rows in the order its warps reach the hash set, while the oracle
    stores them sequentially.  After the first level whose representatives differ, counts are
    held to the 1% rule."""
    inst = load_fixture(run["file"])
    res = engine.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"],
                       key_mode=api.KEY_REF, rlx_type=run["rlx"], schedule=api.SCHEDULE_PER_BLOCK, limit_traces=True)
    assert res.device_flags & ~1 == 0
    mine = [[b["cost"], b["op"], b["all_before"], b["stored_before"], b["to_check"]] for b in res.blocks]
    oracle = O.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"], key_mode=run["rlx"],
                     limit_traces=True)
    assert mine == [list(p) for p in oracle.progress if p[1] != "A"]
    ref = [p for p in run["progress"] if p[1] != "A"]
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a[:2] == b[:2]
        if a[0] <= 2:
            assert a == b
        else:
            assert abs(a[3] - b[3]) <= max(2, 0.01 * b[3]), (a, b)
    fin = run["final"]
    assert res.cost == fin["cost"]
    if fin["formula"] == "not_found":
        assert res.status == api.NOT_FOUND
    else:
        assert res.status == api.FOUND and O.separates(res.formula, inst)
        assert O.formula_cost(res.formula, run["costs"]) == fin["cost"]
    fused = engine.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"],
                         key_mode=api.KEY_REF, rlx_type=run["rlx"], limit_traces=True)
    assert (fused.status, fused.cost, fused.all_ltls) == (res.status, res.cost, res.all_ltls)
    # every level to max_cost
    full = engine.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"],
                        key_mode=api.KEY_REF, rlx_type=run["rlx"], limit_traces=True, stop_at_found=False)
    assert full.device_flags & ~1 == 0
    want = O.learn(inst, costs=run["costs"], max_cost=run["max_cost"], neg_type=run["neg"], key_mode=run["rlx"],
                   limit_traces=True, stop_at_found=False)
    starts = engine.level_starts(run["max_cost"] + 2)
    c1 = run["costs"][0]
    rows, parents = engine.read_rows(0, starts[run["max_cost"] + 1])
    mask = np.array([(1 << int(x)) - 1 for x in inst.lengths], dtype=np.uint64)
    for i in range(starts[c1 + 1], len(rows)):  # each row is its parents' operator
        p = int(parents[i])
        op, left, right = (p >> 60) & 7, (p >> 30) & 0x3FFFFFFF, p & 0x3FFFFFFF
        cs, _ = O.apply_op(op, rows[left], rows[right] if op in (1, 2, 6) else None, mask)
        assert np.array_equal(cs, rows[i]), (i, op, left, right)
    keys = lambda rs: {O.ref_key(np.ascontiguousarray(r), np.asarray(inst.lengths), run["rlx"]) for r in rs}
    same_below = True
    for c in range(c1, run["max_cost"] + 1):
        theirs = want.level_rows(c)
        mine = rows[starts[c]:starts[c + 1]]
        if same_below:
            assert len(mine) == len(theirs) and keys(mine) == keys(theirs), c
            same_below = row_set(mine) == row_set(theirs)
        else:
            assert abs(len(mine) - len(theirs)) <= max(2, 0.01 * len(theirs)), (c, len(mine), len(theirs))


@pytest.mark.parametrize("name", sorted(edge_cases()))
@pytest.mark.parametrize("schedule", [api.SCHEDULE_FUSED, api.SCHEDULE_PER_BLOCK])
def test_edge_cases_match_oracle(engine, name, schedule):
    """Inputs at the domain's edges on the device: an empty side, a trace of no steps,
    one-step traces, a 63-step trace, duplicate traces, one trace on both sides."""
    inst = edge_cases()[name]
    assert_level_sets(engine, inst, 4, schedule=schedule)
    found = engine.learn(inst, max_cost=4, neg_type=1, schedule=schedule)
    want = O.learn(inst, max_cost=4, neg_type=1)
    assert (found.status, found.cost) == ((api.FOUND if want.status == O.FOUND else api.NOT_FOUND), want.cost)
    if found.status == api.FOUND:
        assert O.separates(found.formula, inst) and O.formula_cost(found.formula) == found.cost
    else:
        assert found.formula == "not_found"


def test_hash_set_full_status():
    """A hash set of 2^10 slots cannot hold the 1,637 unique CSs of costs up to 6: the learn ends
    with LTLG_TABLE_FULL instead of a wrong answer, and the engine's next learn (within the
    set's size) is right."""
    inst = load_fixture("cfg1_deep.trace")
    small = gen.generate(3, 2, 20, 20, 8, 16, 0.5, 5)
    with api.Engine(slots_log2=10, cache_bytes=1 << 30, max_rows=1 << 20) as e:
        res = e.learn(inst, max_cost=7, stop_at_found=False, neg_type=1)
        assert res.status == api.TABLE_FULL and res.formula == "hash_set_full"
        again = e.learn(small, neg_type=1)
    want = O.learn(small, neg_type=1)
    assert again.status == api.FOUND and again.cost == want.cost and O.separates(again.formula, small)


def test_publication_wait_runs_out():
    """A candidate whose hash slot is held by a publication that never comes waits a bounded
    number of polls and the learn returns LTLG_DEVICE_WAIT (no hang); the engine's next learn
    starts from a clean set and equals the oracle."""
    inst = gen.generate(3, 2, 20, 20, 8, 16, 0.5, 5)
    x_first = inst.atom_cs()[0] >> np.uint64(1)  # X of the first letter: a cost-2 candidate
    with api.Engine(slots_log2=16, cache_bytes=256 << 20, max_rows=1 << 18, wait_spins=64) as e:
        e.hold_slot(x_first)
        res = e.learn(inst, max_cost=3, stop_at_found=False, neg_type=1)
        assert res.status == api.DEVICE_WAIT and res.device_flags & 2
        assert_level_sets(e, inst, 4)


def test_costs_and_splits_beyond_old_caps():
    """Expensive operators (costs of 100, maxCost 5000) find at cost 900, past the 511 level
    starts the device once kept; cheap letters with uneven operator costs give levels with more
    than 64 splits per operator (the reference has no split cap, ltli6463.cu:1245).  Cost and
    candidate count equal the oracle's, and every level's set of CSs up to cost 600."""
    inst = load_fixture("ham1_len3.trace")
    with api.Engine(slots_log2=22, cache_bytes=1 << 30, max_rows=1 << 20) as e:
        for costs in ([100] * 8, [100, 100, 150, 150, 100, 200, 200, 300]):
            res = e.learn(inst, costs=costs, max_cost=5000, neg_type=1)
            ref = O.learn(inst, costs=costs, max_cost=5000, neg_type=1, keep_rows=False)
            assert res.status == api.FOUND and ref.status == O.FOUND and res.cost > 511
            assert (res.cost, res.all_ltls) == (ref.cost, ref.all_ltls)
            assert O.separates(res.formula, inst) and O.formula_cost(res.formula, costs) == res.cost
        costs = [1, 37, 41, 43, 29, 53, 59, 61]
        res, ref = assert_level_sets(e, inst, 600, costs=costs)
    ls = [ref.level_start[k] for k in range(602)]
    nonempty = {k for k in range(601) if ls[k + 1] > ls[k]}
    splits = max(sum(1 for i in nonempty if 2 * i <= c - cop and (c - i - cop) in nonempty)
                 for c in range(601) for cop in (costs[2], costs[3], costs[7]))
    assert splits > 64, splits


def test_level_stamps_are_ordered(engine):
    """record_levels: every level with candidates reports when its plan was published, its first
    item claimed and its first row begun, in that order and within the level's time."""
    inst = gen.generate(2, 3, 500, 500, 16, 32, 0.5, 9)
    res = engine.learn(inst, neg_type=1, max_cost=7, stop_at_found=False, record_levels=True)
    levels = [lv for lv in res.levels if lv["candidates"] > 0]
    assert len(levels) >= 5
    for lv in levels:
        assert 0 < lv["plan_us"] <= lv["claim_us"] <= lv["start_us"] <= lv["ms"] * 1e3, lv
