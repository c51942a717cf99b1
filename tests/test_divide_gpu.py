"""Formula evaluation on the device (against the oracle's independent evaluator) and the
divide-and-conquer driver on the engine."""
import numpy as np
import pytest

import oracle as O
from ltlb200 import api, divide, gen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(4))
def test_evaluate_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    inst = gen.generate(seed, 3, 60, 60, 4, 63, 0.5, 5)
    atoms, mask = inst.atom_cs(), (np.uint64(1) << inst.lengths.astype(np.uint64)) - np.uint64(1)
    for size in (1, 2, 4, 8, 16, 40):
        f = gen.random_formula(rng, size, 3)
        s = gen.formula_str(f, inst.alphabet)
        cs, holds = api.evaluate(inst, s)
        assert holds.tolist() == O.evaluate(s, inst).tolist(), s
        assert cs.tolist() == gen.eval_cs(f, atoms, mask).tolist(), s


def test_learned_formula_separates_by_both_evaluators():
    inst = gen.generate(11, 2, 20, 20, 8, 16, 0.5, 5)
    r = api.learn(inst, neg_type=1)
    assert api.separates(inst, r.formula) and O.separates(r.formula, inst)


def test_evaluate_rejects_malformed():
    inst = gen.generate(1, 2, 5, 5, 4, 8, 0.5, 3)
    for bad in ("(p)&q", "X(p", "~p", "(p)&(z)", "", "pq"):
        with pytest.raises(ValueError):
            api.evaluate(inst, bad)


@pytest.mark.parametrize("algo", ["det", "rand"])
def test_dc_on_engine_separates(algo):
    inst = gen.generate(21, 3, 200, 200, 8, 24, 0.5, 7)
    out = divide.run_dc(inst, algo=algo, window=64, key_mode=api.KEY_EXACT, neg_type=1, timeout_s=300)
    assert out["formula"] not in ("not_found", "Function timed out."), out
    assert O.separates(out["formula"], inst), out
    assert out["subproblems"] >= 1  # a first leaf's formula may already separate everything


def test_dc_splits_when_needed():
    """Near-miss negatives (Hamming style): small windows rarely generalise, so the driver
    has to combine several sub-results; the combination still separates every trace."""
    inst = gen.generate_hamming(5, 3, 120, 120, 10, 20, 0.5, 6)
    out = divide.run_dc(inst, algo="rand", window=16, key_mode=api.KEY_EXACT, neg_type=1, timeout_s=300)
    assert out["formula"] not in ("not_found", "Function timed out."), out
    assert O.separates(out["formula"], inst), out


def test_dc_window_covering_everything_matches_direct_learn():
    inst = gen.generate(22, 2, 30, 30, 6, 14, 0.5, 5)
    out = divide.run_dc(inst, algo="det", window=64, key_mode=api.KEY_EXACT, neg_type=1)
    direct = api.learn(inst, neg_type=1)
    assert out["subproblems"] == 1
    assert O.formula_cost(out["formula"]) == direct.cost
