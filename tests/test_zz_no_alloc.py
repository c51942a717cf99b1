"""The no-allocation entry point (ltlg_learn_noalloc) against the ordinary one (ltlg_learn).

Some callers cannot allocate device memory: a host application whose GPU memory belongs to
another allocator, or one that forbids cudaMalloc after start-up.  ltlg_learn_noalloc keeps
every device buffer in one static array inside the library, so it must give what ltlg_learn
gives: the same status, minimal cost and candidate count, and a formula that separates the
traces at that cost.  Each case is called twice in a row, because the static array keeps
the previous call's contents and every call has to start from a clean state.

This file is collected last on purpose (tests/test_zz_*), so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import pytest

import oracle as O
from ltlb200 import api, gen
from helpers import edge_instance, load_fixture

pytestmark = pytest.mark.gpu


def noalloc(inst, cap=api.FORMULA_MAX_BYTES, **kw):
    L = api.lib()
    f = L.ltlg_learn_noalloc
    f.argtypes = [C.POINTER(api.Traces), C.POINTER(api.Options), C.c_char_p, C.c_int32, C.POINTER(C.c_int32),
                  C.POINTER(C.c_uint64)]
    f.restype = C.c_int
    t, keep = api._traces(inst)
    o = api.make_options(**kw)
    buf = C.create_string_buffer(cap)
    cost, all_ltls = C.c_int32(), C.c_uint64()
    rc = f(C.byref(t), C.byref(o), buf, cap, C.byref(cost), C.byref(all_ltls))
    return rc, buf.value.decode(), cost.value, all_ltls.value


CASES = [("cfg1", lambda: gen.generate(3, 2, 20, 20, 8, 16, 0.5, 5)),
         ("cfg1_deep", lambda: gen.generate(450, 2, 20, 20, 8, 16, 0.5, 8)),
         ("ham1_len4", lambda: load_fixture("ham1_len4.trace")),
         ("f10x10_p3", lambda: load_fixture("f10x10_p3_s0.trace"))]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_learn_found(name, make):
    inst = make()
    want = api.learn(inst, neg_type=1)
    for _ in range(2):
        rc, formula, cost, all_ltls = noalloc(inst, neg_type=1)
        assert rc == want.status == api.FOUND
        assert cost == want.cost
        assert all_ltls == want.all_ltls  # the reference's count: blocks in order up to the first find
        assert O.separates(formula, inst), formula
        assert O.formula_cost(formula) == cost


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_learn_bounded(name, make):
    inst = make()
    want = api.learn(inst, neg_type=1, max_cost=5, stop_at_found=False)
    for _ in range(2):
        rc, formula, cost, all_ltls = noalloc(inst, neg_type=1, max_cost=5, stop_at_found=False)
        assert rc == want.status
        assert cost == want.cost
        assert all_ltls == want.all_ltls


def test_noalloc_rejects_more_than_64_traces():
    inst = load_fixture("over64.trace")
    rc, formula, _, _ = noalloc(inst)
    assert rc == api.INPUT_LIMITS and formula == "see_the_error"


def test_noalloc_no_traces_follows_learn():
    """With no traces every letter separates them (vacuously): both entry points answer with
    the first letter at the letter cost, whether or not the search stops at the find."""
    inst = edge_instance([], [])
    for stop in (True, False):
        want = api.learn(inst, neg_type=1, max_cost=4, stop_at_found=stop)
        for _ in range(2):
            rc, formula, cost, all_ltls = noalloc(inst, neg_type=1, max_cost=4, stop_at_found=stop)
            assert (rc, formula, cost, all_ltls) == (want.status, want.formula, want.cost, want.all_ltls)


def test_noalloc_rejects_long_traces():
    inst = load_fixture("len64.trace")
    want = api.learn(inst)
    rc, formula, _, _ = noalloc(inst)
    assert rc == want.status == api.INPUT_LIMITS and formula == "see_the_error"


def test_noalloc_scratch_overflow_is_reported():
    """Levels beyond what the static scratch holds (about 131k rows of 40 traces) end the call
    with LTLG_NO_MEMORY, on every call; the next call that fits is right again."""
    inst = load_fixture("cfg1_deep.trace")
    for _ in range(2):
        rc, formula, _, _ = noalloc(inst, neg_type=1, max_cost=10, stop_at_found=False)
        assert rc == api.NO_MEMORY
    small = gen.generate(3, 2, 20, 20, 8, 16, 0.5, 5)
    rc, formula, cost, _ = noalloc(small, neg_type=1)
    assert rc == api.FOUND and cost == api.learn(small, neg_type=1).cost and O.separates(formula, small)


def test_noalloc_formula_longer_than_buffer():
    """A found formula that does not fit the caller's buffer is its own status, not a bad
    argument: the string is empty, the cost and the candidate count are set."""
    inst = load_fixture("cfg1_deep.trace")
    want = api.learn(inst, neg_type=1)
    assert want.status == api.FOUND and len(want.formula) >= 16
    rc, formula, cost, all_ltls = noalloc(inst, cap=16, neg_type=1)
    assert rc == api.FORMULA_TOO_LONG and formula == "" and cost == want.cost and all_ltls > 0
    rc, formula, cost, _ = noalloc(inst, neg_type=1)
    assert rc == api.FOUND and cost == want.cost and O.separates(formula, inst)
