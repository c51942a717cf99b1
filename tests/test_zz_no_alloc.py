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
from helpers import load_fixture

pytestmark = pytest.mark.gpu


def noalloc(inst, **kw):
    L = api.lib()
    f = L.ltlg_learn_noalloc
    f.argtypes = [C.POINTER(api.Traces), C.POINTER(api.Options), C.c_char_p, C.c_int32, C.POINTER(C.c_int32),
                  C.POINTER(C.c_uint64)]
    f.restype = C.c_int
    t, keep = api._traces(inst)
    o = api.make_options(**kw)
    buf = C.create_string_buffer(4096)
    cost, all_ltls = C.c_int32(), C.c_uint64()
    rc = f(C.byref(t), C.byref(o), buf, 4096, C.byref(cost), C.byref(all_ltls))
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
