"""The divide-and-conquer driver's control flow on the CPU, with the oracle as the solver and
as the checker (the product runs both on the device): results separate every trace, and a
window covering the whole instance gives the direct result."""
import numpy as np
import pytest

import oracle as O
from ltlb200 import divide, gen


def _driver(inst, **kw):
    def solve(pos, neg):
        sub = divide.sub_instance(inst, pos, neg)
        r = O.learn(sub, costs=(1,) * 8, neg_type=1, max_cost=12, keep_rows=False)
        return r.formula if r.status == O.FOUND else None

    return divide.Driver(inst, solve=solve, holds=lambda f: O.evaluate(f, inst), **kw)


def test_sub_instance_slices_traces():
    inst = gen.generate(3, 2, 10, 10, 4, 12, 0.5, 4)
    sub = divide.sub_instance(inst, [1, 4], [0, 9])
    lines = inst.trace_lines()
    assert sub.num_pos == 2 and sub.num_neg == 2
    assert sub.trace_lines() == [lines[1], lines[4], lines[10], lines[19]]


@pytest.mark.parametrize("algo", ["det", "rand"])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_dc_result_separates(algo, seed):
    inst = gen.generate(seed, 3, 40, 40, 6, 14, 0.5, 6)
    d = _driver(inst)
    pos, neg = list(range(inst.num_pos)), list(range(inst.num_neg))
    f = (d.rand_split if algo == "rand" else d.det_split)(16, pos, neg)
    assert O.separates(f, inst), f
    assert d.calls >= 1


def test_window_covering_everything_is_one_call():
    inst = gen.generate(5, 2, 12, 12, 4, 10, 0.5, 4)
    d = _driver(inst)
    f = d.det_split(64, list(range(12)), list(range(12)))
    assert d.calls == 1 and O.separates(f, inst)
    assert O.formula_cost(f) == O.learn(inst, neg_type=1, keep_rows=False).cost


def test_formula_size_counts_symbols():
    assert divide.formula_size("(p)&(q)") == 3
    assert divide.formula_size("G(((p)&(q))|(~((p)|(q))))") == 9
    assert divide.formula_size("p, q ") == 2


def test_over_fitted_string():
    assert divide.over_fitted("pq", ["1,0;0,1"]) == "p&~q&X(~p&q&~X(p|~p))"
    assert divide.over_fitted("pq", ["1,1", "0,0"]) == "(p&q&~X(p|~p))|(~p&~q&~X(p|~p))"


def _parenthesise(s):
    """The reference's infix form (~ binds tightest, then &, then |) as the enumerator's fully
    parenthesised form, so the oracle's evaluator can read it."""
    pos = 0

    def expr():
        nonlocal pos
        f = term()
        while pos < len(s) and s[pos] == "|":
            pos += 1
            f = f"({f})|({term()})"
        return f

    def term():
        nonlocal pos
        f = factor()
        while pos < len(s) and s[pos] == "&":
            pos += 1
            f = f"({f})&({factor()})"
        return f

    def factor():
        nonlocal pos
        c = s[pos]
        if c == "~":
            pos += 1
            return f"~({factor()})"
        if c in "XFG" and pos + 1 < len(s) and s[pos + 1] == "(":
            pos += 2
            f = expr()
            assert s[pos] == ")"
            pos += 1
            return f"{c}({f})"
        if c == "(":
            pos += 1
            f = expr()
            assert s[pos] == ")"
            pos += 1
            return f
        pos += 1
        return c

    out = expr()
    assert pos == len(s)
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_over_fitted_holds_exactly_on_the_positive_traces(seed):
    inst = gen.generate(seed, 3, 12, 12, 2, 6, 0.5, 4)
    lines = inst.trace_lines()
    f = _parenthesise(divide.over_fitted(inst.alphabet, lines[:inst.num_pos]))
    h = O.evaluate(f, inst)
    expect = np.array([ln in set(lines[:inst.num_pos]) for ln in lines], dtype=bool)
    assert np.array_equal(h.astype(bool), expect)


@pytest.mark.parametrize("algo", ["det", "rand"])
def test_contradictory_traces_end_as_unsolvable(algo):
    """One trace both positive and negative: the recursion comes back to a sub-problem it is
    still solving (the reference recurses until its timeout); the driver raises Unsolvable,
    which run_dc reports as not_found."""
    text = "1,0;0,1\n0,1\n---\n1,0;0,1\n---\nAll operators\n---\np,q"
    inst = gen.from_scarlet_text(text)
    d = _driver(inst)
    with pytest.raises(divide.Unsolvable):
        (d.rand_split if algo == "rand" else d.det_split)(4, [0, 1], [0])
