"""The CPU oracle checked on its own: independent semantics, brute force, determinism.

These tests pin the oracle before it is trusted as the checker of the GPU path.
"""
import itertools

import numpy as np
import pytest

import oracle as O
from ltlb200 import gen
from helpers import edge_cases, last_round_gap, load_fixture, on_the_fly_cases, row_set

OPS = ["~", "&", "|", "X", "F", "G", "U"]


def positional_cs(f, steps, length, letters):
    """CS of formula tree f on one trace by direct LTLf semantics, position by position."""
    op = f[0]
    if op == "p":
        bit = ord(letters[f[1]]) - 97
        return [bool((steps[k] >> bit) & 1) for k in range(length)]
    a = positional_cs(f[1], steps, length, letters)
    b = positional_cs(f[2], steps, length, letters) if op in "&|U" else None
    out = [False] * length
    for k in reversed(range(length)):
        if op == "~":
            out[k] = not a[k]
        elif op == "&":
            out[k] = a[k] and b[k]
        elif op == "|":
            out[k] = a[k] or b[k]
        elif op == "X":
            out[k] = k + 1 < length and a[k + 1]
        elif op == "F":
            out[k] = a[k] or (k + 1 < length and out[k + 1])
        elif op == "G":
            out[k] = a[k] and (k + 1 >= length or out[k + 1])
        elif op == "U":
            out[k] = b[k] or (a[k] and k + 1 < length and out[k + 1])
    return out


def cs_words(f, inst):
    words = []
    for t in range(inst.n):
        s = inst.steps[inst.offsets[t]:inst.offsets[t + 1]]
        bits = positional_cs(f, s, len(s), inst.alphabet)
        words.append(sum(1 << k for k, v in enumerate(bits) if v))
    return np.array(words, dtype=np.uint64)


def test_bit_tricks_match_positional_semantics():
    rng = np.random.default_rng(7)
    inst = gen.generate(3, 3, 6, 6, 1, 12, 0.5, 4)
    atoms = inst.atom_cs()
    mask = (np.uint64(1) << inst.lengths.astype(np.uint64)) - np.uint64(1)
    for _ in range(300):
        f = gen.random_formula(rng, int(rng.integers(1, 9)), 3)
        assert np.array_equal(gen.eval_cs(f, atoms, mask), cs_words(f, inst)), gen.formula_str(f, inst.alphabet)


def test_oracle_operators_match_python():
    rng = np.random.default_rng(1)
    n = 37
    lens = rng.integers(1, 64, size=n)
    mask = np.array([(1 << int(l)) - 1 for l in lens], dtype=np.uint64)
    a = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) & mask
    b = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) & mask
    atoms = np.stack([a, b])
    for op, py in ((0, ("~", ("p", 0))), (1, ("&", ("p", 0), ("p", 1))), (2, ("|", ("p", 0), ("p", 1))),
                   (3, ("X", ("p", 0))), (4, ("F", ("p", 0))), (5, ("G", ("p", 0)))):
        out, _ = O.apply_op(op, a, b, mask)
        assert np.array_equal(out, gen.eval_cs(py, atoms, mask)), op
    out, out2 = O.apply_op(6, a, b, mask)
    assert np.array_equal(out, gen.eval_cs(("U", ("p", 0), ("p", 1)), atoms, mask))
    assert np.array_equal(out2, gen.eval_cs(("U", ("p", 1), ("p", 0)), atoms, mask))


def test_evaluator_matches_bit_tricks_on_random_formulas():
    rng = np.random.default_rng(11)
    inst = gen.generate(5, 2, 15, 15, 3, 20, 0.5, 4)
    atoms = inst.atom_cs()
    mask = (np.uint64(1) << inst.lengths.astype(np.uint64)) - np.uint64(1)
    for _ in range(300):
        f = gen.random_formula(rng, int(rng.integers(1, 12)), 2)
        s = gen.formula_str(f, inst.alphabet)
        want = (gen.eval_cs(f, atoms, mask) & np.uint64(1)).astype(bool)
        assert np.array_equal(O.evaluate(s, inst), want), s


def test_formula_cost():
    cf = [1, 2, 3, 4, 5, 6, 7, 8]
    assert O.formula_cost("(p)U(~(X(q)))", cf) == 1 + 8 + 2 + 5 + 1
    assert O.formula_cost("G((p)|(F(q)))", cf) == 7 + 1 + 4 + 6 + 1
    assert O.formula_cost("p", cf) == 1
    assert O.formula_cost("((p", cf) == -1


def brute_force_levels(inst, costs, max_cost, neg_type):
    """Every formula up to max_cost, CS by the positional semantics, grouped by the first
    cost at which its CS appears."""
    letters = inst.alphabet
    by_cost = {costs[0]: [("p", j) for j in range(len(letters))]}
    seen = {}
    levels = {}
    for c in range(costs[0], max_cost + 1):
        if c != costs[0]:
            fs = []
            if c - costs[1] >= costs[0]:
                src = by_cost.get(c - costs[1], [])
                if neg_type == 2:
                    src = [f for f in src if f[0] == "p"]
                fs += [("~", f) for f in src]
            for k, op in ((4, "X"), (5, "F"), (6, "G")):
                fs += [(op, f) for f in by_cost.get(c - costs[k], [])]
            for k, op in ((2, "&"), (3, "|"), (7, "U")):
                for i in range(costs[0], c - costs[k]):
                    j = c - costs[k] - i
                    for f, g in itertools.product(by_cost.get(i, []), by_cost.get(j, [])):
                        fs.append((op, f, g))
            by_cost[c] = fs
        lv = set()
        for f in by_cost[c]:
            key = cs_words(f, inst).tobytes()
            if key not in seen:
                seen[key] = c
                lv.add(key)
        levels[c] = lv
    return levels


@pytest.mark.parametrize("neg_type", [1, 2])
@pytest.mark.parametrize("costs", [[1] * 8, [1, 2, 1, 1, 2, 2, 3, 2]])
def test_oracle_levels_equal_brute_force(neg_type, costs):
    inst = gen.generate(21, 2, 3, 3, 2, 4, 0.5, 3)
    max_cost = 5 if costs == [1] * 8 else 6
    want = brute_force_levels(inst, costs, max_cost, neg_type)
    run = O.learn(inst, costs=costs, max_cost=max_cost, neg_type=neg_type, stop_at_found=False)
    for c in range(costs[0], max_cost + 1):
        assert run.level_set(c) == want[c], c


def test_oracle_threads_give_same_level_sets():
    inst = gen.generate(8, 3, 30, 30, 5, 12, 0.5, 7)
    a = O.learn(inst, max_cost=6, stop_at_found=False, threads=1)
    b = O.learn(inst, max_cost=6, stop_at_found=False, threads=4)
    for c in range(1, 7):
        assert a.level_set(c) == b.level_set(c)
        assert len(a.level_rows(c)) == len(a.level_set(c))  # no duplicate rows


def test_oracle_found_formula_is_minimal_and_separates():
    for seed in range(6):
        inst = gen.generate(seed, 2, 20, 20, 8, 16, 0.5, 5)
        run = O.learn(inst)
        assert run.status == O.FOUND
        assert O.separates(run.formula, inst)
        assert O.formula_cost(run.formula) == run.cost
        # nothing cheaper separates: no row of a lower level accepts
        full = O.learn(inst, max_cost=run.cost - 1, stop_at_found=False)
        lower = full.rows[: full.level_start[run.cost]] if run.cost > 1 else np.zeros((0, inst.n), np.uint64)
        bit0 = (lower & np.uint64(1)).astype(bool)
        acc = bit0[:, :inst.num_pos].all(axis=1) & ~bit0[:, inst.num_pos:].any(axis=1)
        assert not acc.any()


def test_oracle_rows_are_cs_of_their_formulas():
    inst = load_fixture("ham1_len3.trace")
    run = O.learn(inst, max_cost=6, stop_at_found=False, neg_type=1)
    letters = inst.alphabet

    def tree(r):
        op = int(run.row_op[r])
        if op == 7:
            return ("p", r)
        if op in (1, 2, 6):
            return (OPS[op], tree(int(run.row_left[r])), tree(int(run.row_right[r])))
        return (OPS[op], tree(int(run.row_left[r])))

    for r in range(run.num_rows):
        assert np.array_equal(run.rows[r], cs_words(tree(r), inst)), r
    assert letters == "pq"


def test_reference_keys_exact_pack_is_injective_below_126_bits():
    inst = load_fixture("f10x10_p2_s0.trace")  # lenSum = 100
    run = O.learn(inst, max_cost=5, stop_at_found=False)
    keys = {O.ref_key(r, inst.lengths, 3) for r in run.rows}
    assert len(keys) == len(row_set(run.rows))


def test_relaxed_type3_collides_where_exact_does_not():
    inst = gen.generate(450, 2, 20, 20, 8, 16, 0.5, 8)
    exact = O.learn(inst, max_cost=6, stop_at_found=False)
    rlx = O.learn(inst, max_cost=6, stop_at_found=False, key_mode=O.KEY_REF3)
    assert rlx.num_rows <= exact.num_rows
    h64 = O.learn(inst, max_cost=6, stop_at_found=False, key_mode=O.KEY_HASH64)
    assert h64.num_rows == exact.num_rows  # no 64-bit fingerprint collision at this size


OTF_COSTS = [(1,) * 8, (1, 2, 1, 1, 2, 2, 2, 2)]

@pytest.mark.parametrize("costs", OTF_COSTS)
def test_oracle_on_the_fly_regime(costs):
    """The reference's overflow switch (ltli6463.cu:1021-1027, 1202-1206, 1442-1443): once a
    level finds no free cache row, later levels are only checked for acceptance, built from
    the stored rows, until the last-round rule ends the search."""
    inst = gen.generate(3, 3, 30, 30, 6, 14, 0.5, 7)
    ex, cases = on_the_fly_cases(inst, costs)
    assert len(cases) >= 3
    found = 0
    for k, cap in cases:
        r = O.learn(inst, costs=costs, neg_type=1, max_cost=14, cache_rows=cap)
        assert r.on_the_fly and r.num_rows == cap
        assert np.array_equal(r.rows, ex.rows[:cap])
        if r.status == O.FOUND:
            found += 1
            assert O.separates(r.formula, inst) and O.formula_cost(r.formula, costs) == r.cost >= ex.cost
            assert r.cost <= k + 1 + last_round_gap(costs)
        else:
            assert r.status == O.NOT_FOUND and r.cost == k + 1 + last_round_gap(costs)
    assert found >= 1


EDGE = edge_cases()


@pytest.mark.parametrize("name", sorted(EDGE))
def test_oracle_edge_cases_equal_brute_force(name):
    """Inputs at the domain's edges: an empty side, a trace of no steps, one-step traces, a
    trace of the maximum 63 steps, duplicate traces, and one trace on both sides."""
    inst = EDGE[name]
    costs = [1] * 8
    want = brute_force_levels(inst, costs, 4, 1)
    run = O.learn(inst, costs=costs, max_cost=4, neg_type=1, stop_at_found=False)
    for c in range(1, 5):
        assert run.level_set(c) == want[c], (name, c)
    found = O.learn(inst, costs=costs, max_cost=4, neg_type=1)
    if name == "contradiction":
        assert found.status == O.NOT_FOUND and found.formula == "not_found"
    else:
        assert found.status == O.FOUND and O.separates(found.formula, inst), name
        assert O.formula_cost(found.formula) == found.cost


@pytest.mark.parametrize("case", range(12))
def test_oracle_levels_equal_brute_force_random_costs(case):
    """Seeded cost functions (each operator 1-3, letters 1-2) and both NegTypes on small
    instances: the split rule, the NegType rule and the level order under uneven costs."""
    rng = np.random.default_rng(1000 + case)
    costs = [int(rng.integers(1, 3))] + [int(c) for c in rng.integers(1, 4, size=7)]
    neg_type = 1 + case % 2
    inst = gen.generate(30 + case, 2, 3, 3, 2, 5, 0.5, 3)
    max_cost = costs[0] + 5
    want = brute_force_levels(inst, costs, max_cost, neg_type)
    run = O.learn(inst, costs=costs, max_cost=max_cost, neg_type=neg_type, stop_at_found=False)
    for c in range(costs[0], max_cost + 1):
        assert run.level_set(c) == want.get(c, set()), (costs, neg_type, c)


def py_ref_key(cs, lens, rtype):
    """The reference's 126-bit keys (ltli6463.cu:57-141) restated as a list of chosen (trace,
    bit) positions, of which the first 126 are packed: bits 0-62 into l, 63-125 into h.  Exact
    packing when lenSum <= 126; else type 1 samples every (lenSum // 126)-th step, type 2
    takes the first (126 len + lenSum) // lenSum steps of each trace, and type 3 XORs the
    splitmix64 finaliser of every word into h (first half of the traces) or l."""
    n, lensum, mask = len(cs), int(sum(lens)), (1 << 64) - 1
    if lensum > 126 and rtype == 3:
        h = l = 0
        for i, w in enumerate(cs):
            x = int(w)
            x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & mask
            x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & mask
            x ^= x >> 31
            if i < n // 2:
                h ^= x
            else:
                l ^= x
        return h, l
    picks = []
    for i in range(n):
        if lensum <= 126:
            ks = range(int(lens[i]))
        elif rtype == 1:
            ks = range(0, int(lens[i]), lensum // 126)
        else:
            ks = range((126 * int(lens[i]) + lensum) // lensum)
        picks += [(i, k) for k in ks]
    h = l = 0
    for j, (i, k) in enumerate(picks[:126]):
        if k < 64 and (int(cs[i]) >> k) & 1:
            if j < 63:
                l |= 1 << j
            else:
                h |= 1 << (j - 63)
    return h, l


@pytest.mark.parametrize("rtype", [1, 2, 3])
def test_reference_keys_bit_for_bit(rtype):
    rng = np.random.default_rng(rtype)
    for trial in range(300):
        n = int(rng.integers(1, 40))
        lens = rng.integers(0 if trial % 7 == 0 else 1, 64, size=n)
        if trial % 3 == 0:  # the exact-pack regime
            lens = np.minimum(lens, 126 // n)
        words = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n).astype(np.uint64)
        cs = words & ((np.uint64(1) << lens.astype(np.uint64)) - np.uint64(1))
        assert O.ref_key(cs, lens, rtype) == py_ref_key(cs, lens, rtype), (rtype, trial, lens.tolist())
