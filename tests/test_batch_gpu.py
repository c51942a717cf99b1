"""The batch call: one persistent launch learns many instances through a few instance slots.

Every instance's result must equal what one engine gives it alone: status, minimal cost and
the reference's candidate count (the count follows the reference's block order, so it does
not depend on which warp finds first), and the formula separates the traces at that cost.
The slots take instances of different sizes one after another (device-side set-up: letters,
hash-set generation, first plan), instances that end at set-up (a separating letter, no
traces) never reach a level, and the ones the device batch does not take (over-long traces,
the reference's relaxed keys, a slot whose cache overflows) come back from the host path.
"""
import numpy as np
import pytest

import oracle as O
from ltlb200 import api, gen
from helpers import edge_instance, load_fixture

pytestmark = pytest.mark.gpu


def mixed_instances(count=24, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        out.append(gen.generate(5000 + i, int(rng.integers(2, 5)), int(rng.integers(8, 120)),
                                int(rng.integers(8, 120)), 4, 30, 0.5, int(rng.integers(3, 7))))
    out.insert(3, gen.generate(400, 2, 20, 20, 8, 16, 0.5, 5))  # a letter separates
    out.insert(9, edge_instance([], []))                       # no traces
    return out


def assert_same(r, want, inst, costs=(1,) * 8):
    assert (r.status, r.cost, r.all_ltls) == (want.status, want.cost, want.all_ltls), (r.formula, want.formula)
    if r.status == api.FOUND:
        assert O.separates(r.formula, inst) and O.formula_cost(r.formula, costs) == r.cost


def test_batch_recycles_slots_and_matches_one_engine():
    insts = mixed_instances()
    with api.Batch(workers=3, slots_log2=20, cache_bytes=512 << 20, max_traces=512) as pool:
        res = pool.learn(insts, neg_type=1)
        again = pool.learn(insts[::-1], neg_type=1)  # generations go on in the same slots
    with api.Engine(slots_log2=20, cache_bytes=512 << 20, max_traces=512) as e:
        for inst, r, r2 in zip(insts, res, again[::-1]):
            want = e.learn(inst, neg_type=1)
            assert_same(r, want, inst)
            assert_same(r2, want, inst)


def test_batch_enumerates_to_max_cost_like_one_engine():
    insts = mixed_instances(8, seed=11)
    with api.Batch(workers=4, slots_log2=20, cache_bytes=512 << 20, max_traces=512) as pool:
        res = pool.learn(insts, neg_type=1, max_cost=4, stop_at_found=False)
    with api.Engine(slots_log2=20, cache_bytes=512 << 20, max_traces=512) as e:
        for inst, r in zip(insts, res):
            want = e.learn(inst, neg_type=1, max_cost=4, stop_at_found=False)
            assert (r.status, r.cost, r.all_ltls, r.rows) == (want.status, want.cost, want.all_ltls, want.rows)


def test_batch_host_paths():
    """Over-long traces are refused on the host; relaxed reference keys and a slot whose cache
    overflows are learned by the fallback engine, with the results one engine of the same
    configuration gives."""
    deep = load_fixture("cfg1_deep.trace")     # 1,637 rows up to cost 6, 6,281 up to cost 7
    long_ = load_fixture("len64.trace")
    small = gen.generate(3, 2, 20, 20, 8, 16, 0.5, 5)
    # a cache of exactly the rows up to cost 6: level 7 overflows with nothing of it stored, so
    # the on-the-fly regime that follows is the same in every run
    kw = dict(slots_log2=16, cache_bytes=1 << 20, max_rows=1637, max_traces=512)
    with api.Batch(workers=2, **kw) as pool:
        res = pool.learn([small, long_, deep], neg_type=1)
        rel = pool.learn([small, deep], neg_type=1, key_mode=api.KEY_REF, rlx_type=3, max_cost=6)
    assert res[1].status == api.INPUT_LIMITS and res[1].formula == "see_the_error"
    with api.Engine(**kw) as e:
        assert_same(res[0], e.learn(small, neg_type=1), small)
        want = e.learn(deep, neg_type=1)
        assert want.on_the_fly and (res[2].status, res[2].cost) == (want.status, want.cost)
        for inst, r in zip([small, deep], rel):
            w = e.learn(inst, neg_type=1, key_mode=api.KEY_REF, rlx_type=3, max_cost=6)
            assert (r.status, r.cost) == (w.status, w.cost)


def test_cfg4_sample_matches_oracle():
    """The first 256 instances of the cfg4 batch (2-4 propositions, 8-256 positive and negative
    traces of length 4-40, hidden formula size 3-8, unit costs) in one batch launch with the
    autotuner's kind of configuration: every minimal cost and candidate count is the oracle's,
    and every formula separates its traces at that cost."""
    from ltlb200 import workloads
    insts = [gen.generate(*s) for s in workloads.cfg4_specs(4096, 0)[:256]]
    with api.Batch(workers=16, slots_log2=22, cache_bytes=1 << 30, max_traces=512, left_tile=4, right_chunk=32,
                   unary_rows=16) as pool:
        res = pool.learn(insts, neg_type=1)
    for inst, r in zip(insts, res):
        want = O.learn(inst, neg_type=1, threads=0, keep_rows=False, cache_rows=1 << 21)
        assert r.status == api.FOUND and want.status == O.FOUND
        assert (r.cost, r.all_ltls) == (want.cost, want.all_ltls)
        assert O.separates(r.formula, inst) and O.formula_cost(r.formula) == r.cost
