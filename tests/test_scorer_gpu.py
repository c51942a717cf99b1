"""The learned block order on the GPU: the scorer's forward and backward kernels against the
CPU oracle, training, labels, and the learned order itself (same minimal cost as the plain
order; fewer candidates before the find with the trained scorer)."""
import os

import numpy as np
import pytest

import scorer_oracle as SO
from ltlb200 import api, learned

pytestmark = pytest.mark.gpu


def _data(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.random((n, SO.NF)).astype(np.float32)
    X[:, :7] = (rng.random((n, 7)) < 0.2)
    Y = (rng.random(n) < 0.25).astype(np.float32)
    return X, Y


def test_forward_matches_oracle():
    X, _ = _data(1, 1000)
    p = SO.init_params(2)
    got = api.scorer_forward(p, X)
    want = SO.forward(p, X)
    scale = 1.0 + np.max(np.abs(want))
    # BF16 activations: a rounding flip inside a unit moves a logit by about 1e-2 of its size
    assert np.max(np.abs(got - want)) <= 2e-2 * scale
    assert np.median(np.abs(got - want)) <= 1e-4 * scale


@pytest.mark.parametrize("n,pw", [(64, 1.0), (1000, 3.0), (4097, 1.5)])
def test_gradient_matches_oracle(n, pw):
    X, Y = _data(n, n)
    p = SO.init_params(n + 1)
    g, loss = api.scorer_grad(p, X, Y, pw)
    gw, lw = SO.grad(p, X, Y, pw)
    assert abs(loss - lw) <= 1e-4 * (1.0 + abs(lw))
    assert np.linalg.norm(g - gw) <= 1e-2 * np.linalg.norm(gw)
    ge = SO.grad_exact(p, X, Y, pw)  # the unrounded gradient points the same way
    assert float(np.dot(g, ge)) / (np.linalg.norm(g) * np.linalg.norm(ge)) > 0.99


def test_training_fits_a_rule():
    rng = np.random.default_rng(5)
    X = rng.random((8192, SO.NF)).astype(np.float32)
    Y = ((X[:, 3] > 0.6) & (X[:, 10] < 0.5)).astype(np.float32)
    p, curve = api.scorer_train(SO.init_params(0), X, Y, epochs=25, batch=512, lr=3e-3, pos_weight=1.0, seed=1)
    assert curve[-1] < 0.5 * curve[0]
    acc = ((api.scorer_forward(p, X) > 0) == (Y > 0.5)).mean()
    assert acc > 0.95


def test_labels_and_learned_order_keep_the_cost():
    p = learned.init_params(9)  # an untrained scorer: any order gives the same cost
    with api.Engine(slots_log2=22, cache_bytes=2 << 30) as eng:
        eng.set_scorer(p)
        for seed in range(6):
            inst = learned.hamming_instance(seed, 60, 60)
            r0, meta, X, Y = eng.label_blocks(inst, neg_type=1)
            assert r0.status == api.FOUND
            if meta:
                assert all(m["cost"] == r0.cost for m in meta)
                assert Y.sum() >= 1  # the block of the find holds an accepting candidate
                assert X.shape == (len(meta), SO.NF)
            r1 = eng.learn(inst, neg_type=1, order=api.ORDER_LEARNED)
            r2 = eng.learn(inst, neg_type=1, order=api.ORDER_PLAIN)
            assert r1.status == r2.status == api.FOUND
            assert r1.cost == r2.cost == r0.cost


def test_learned_order_requires_a_scorer():
    inst = learned.hamming_instance(1, 30, 30)
    with api.Engine(slots_log2=20, cache_bytes=1 << 30) as eng:
        r = eng.learn(inst, neg_type=1, order=api.ORDER_LEARNED)
        assert r.status == api.BAD_ARGS


def test_label_features_match_host_function():
    """The label writer's features are the host feature function's (same code as the planner)."""
    with api.Engine(slots_log2=22, cache_bytes=2 << 30) as eng:
        inst = learned.hamming_instance(3, 80, 80)
        _, meta, X, Y = eng.label_blocks(inst, neg_type=1)
    for m, x in zip(meta, X):
        assert x[ "~&|XFGU".index(m["op"])] == 1.0
        assert x[31] == 1.0
        assert abs(x[7] - m["cost"] / 16.0) < 1e-7


@pytest.mark.skipif(not os.path.exists(learned.DEFAULT_SCORER), reason="no trained scorer in the package")
def test_trained_scorer_gains_over_plain_order():
    """Held-out Hamming-style instances (1000 + 1000 traces, hidden formula of size 9; seeds
    never used for training): the learned order finds the same minimal cost on every one and
    evaluates fewer candidates before the find over the set."""
    p = learned.load_scorer()
    insts = [learned.hamming_instance(s, 1000, 1000, 9) for s in learned.HELD_OUT_SEEDS]
    with api.Engine(slots_log2=26, cache_bytes=16 << 30) as eng:
        rows = learned.compare(eng, insts, p)
    s = learned.summarize(rows)
    assert s["same_cost"], rows
    assert sum(r["evaluated_learned"] for r in rows) < sum(r["evaluated_plain"] for r in rows), s


def test_learned_order_with_per_block_schedule():
    """Per-block launches under a learned order (windows of the sorted item table) find the
    same minimal cost and the same level counts as the fused plain schedule."""
    p = learned.init_params(11)
    with api.Engine(slots_log2=22, cache_bytes=2 << 30) as eng:
        eng.set_scorer(p)
        for seed in range(3):
            inst = learned.hamming_instance(seed + 20, 80, 80)
            a = eng.learn(inst, neg_type=1, order=api.ORDER_LEARNED, schedule=api.SCHEDULE_PER_BLOCK,
                          max_cost=6, stop_at_found=False, record_levels=True)
            b = eng.learn(inst, neg_type=1, max_cost=6, stop_at_found=False, record_levels=True)
            assert a.status == b.status and a.cost == b.cost
            assert [(l["cost"], l["candidates"], l["uniques"]) for l in a.levels] == \
                   [(l["cost"], l["candidates"], l["uniques"]) for l in b.levels]
