"""The reference's dc.py names (ltlb200.dc) on the CPU: the oracle stands in for the device
backend, so the calls, their arguments, return values and printed output are checked against
the reference's contract (code/dc.py) without a GPU."""
import os
import time
from types import SimpleNamespace

import numpy as np
import pytest

import oracle as O
from ltlb200 import api, dc, gen


class OracleBackend:
    def __init__(self):
        self.learns = 0

    def learn(self, inst, costs, max_cost, rlx_type, neg_type, key_mode):
        self.learns += 1
        r = O.learn(inst, costs=costs, max_cost=min(max_cost, 12), neg_type=neg_type, keep_rows=False)
        return SimpleNamespace(status=api.FOUND if r.status == O.FOUND else api.NOT_FOUND, formula=r.formula,
                               cost=r.cost, all_ltls=r.all_ltls)

    def evaluate(self, inst, formula):
        return None, O.evaluate(formula, inst).astype(bool)


@pytest.fixture
def oracle_backend(monkeypatch):
    b = OracleBackend()
    monkeypatch.setattr(dc, "backend", b)
    return b


def lines_of(inst):
    ls = inst.trace_lines()
    return ls[:inst.num_pos], ls[inst.num_pos:], ",".join(inst.alphabet)


def test_star_import_exports_the_reference_names():
    ns = {}
    exec("from ltlb200.dc import *", ns)
    for name in ("makeInputFile", "runGPU", "get_all_file_paths_in_folder", "bitVec", "LTLmatch", "DetSplit",
                 "RandSplit", "c", "LTLOfSingleTrace", "overFittedCase", "runWithTimeout", "runDC"):
        assert callable(ns[name]), name


def test_run_gpu_output_is_parsed_as_the_reference_parses_it(oracle_backend):
    inst = gen.generate(5, 2, 12, 12, 4, 10, 0.5, 4)
    pos, neg, alphabet = lines_of(inst)
    out = dc.runGPU(pos, neg, alphabet, [1] * 8, 500, 3, 1)
    f = out.split("\n")[-2].split()[-1][1:-1]  # code/dc.py:194
    assert "not_found" not in out and O.separates(f, inst)
    small = dc.runGPU(["1,0;0,1"], ["0,0"], "p,q", [1, 2, 1, 1, 1, 1, 1, 3], 500, 3, 2)
    assert small.startswith("\nPositive: \n\t{p}\t{q}\t\n\nNegative: \n\t{}\t\n")
    assert "\nCost Function: p:1, ~:2, &:1, |:1, X:1, F:1, G:1, U:3\nNumber of Traces: 2\n" in small


def test_run_gpu_reports_not_found(oracle_backend):
    # the same trace as positive and negative: no formula separates them
    out = dc.runGPU(["1,0;0,1"], ["1,0;0,1"], "p,q", [1] * 8, 3, 3, 1)
    assert "not_found" in out and out.split("\n")[-2] == 'LTL: "not_found"'


def test_ltlmatch_and_bitvec(oracle_backend, monkeypatch):
    inst = gen.generate(6, 3, 10, 10, 3, 9, 0.5, 5)
    pos, neg, alphabet = lines_of(inst)
    f = "(p)U(X(q))"
    assert dc.LTLmatch(pos + neg, alphabet, f) == O.evaluate(f, inst).astype(bool).tolist()
    assert dc.LTLmatch([], alphabet, f) == []

    class Words:
        def evaluate(self, inst, formula):
            return np.array([0b0101, 0b1], dtype=np.uint64), None

    monkeypatch.setattr(dc, "backend", Words())
    # bitarray order of the reference: last position first, element -1 is position 0
    assert dc.bitVec(["1;0;1;0", "1,0"], "p", "p") == [[0, 1, 0, 1], [1]]


@pytest.mark.parametrize("algo", ["DetSplit", "RandSplit"])
@pytest.mark.parametrize("seed", [1, 2])
def test_splits_separate(oracle_backend, algo, seed):
    inst = gen.generate(seed, 3, 40, 40, 6, 14, 0.5, 6)
    pos, neg, alphabet = lines_of(inst)
    f = getattr(dc, algo)(16, pos, neg, alphabet, [1] * 8, 500, 3, 1)
    assert O.separates(f, inst), f
    assert oracle_backend.learns >= 1


def test_unsolvable_leaf_is_not_found(oracle_backend):
    f = dc.DetSplit(4, ["1,0;0,1"], ["1,0;0,1"], "p,q", [1] * 8, 3, 3, 1)
    assert f == "not_found"


def test_run_dc_prints_the_reference_lines(oracle_backend, tmp_path, capsys):
    inst = gen.generate(3, 2, 20, 20, 4, 10, 0.5, 5)
    p = tmp_path / "in.trace"
    p.write_text(inst.to_scarlet())  # the layout code/dc.py:8-21 writes, no final newline
    dc.runDC(str(p), dc.DetSplit, 16, [1] * 8, 500, 3, 1, 60)
    out = capsys.readouterr().out.split("\n")
    assert out[0] == "Size(P, N): (20, 20)"
    assert out[1].startswith("Time: ") and out[1].endswith("s")
    assert out[2].startswith("LTL: ") and O.separates(out[2][len("LTL: "):], inst)


def test_run_with_timeout():
    assert dc.runWithTimeout(lambda a, b: a + b, [2, 3], 5) == 5
    assert dc.runWithTimeout(time.sleep, [3], 1) == "Function timed out."


def test_make_input_file_and_paths(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    dc.makeInputFile(["1,0;0,1", "0,1"], ["1,1"], "p,q")
    text = (tmp_path / "subInput").read_text()
    assert text == "1,0;0,1\n0,1\n---\n1,1\n---\nAll operators\n---\np,q"
    inst = gen.from_scarlet_text(text)
    assert (inst.num_pos, inst.num_neg, inst.alphabet) == (2, 1, "pq")
    (tmp_path / "d").mkdir()
    (tmp_path / "d" / "a.trace").write_text("")
    (tmp_path / "d" / "b.txt").write_text("")
    found = dc.get_all_file_paths_in_folder(str(tmp_path))
    assert found == [os.path.join(str(tmp_path), "d", "a.trace")]


def test_size_and_over_fitted_names():
    assert dc.c("(p)&(q)") == 3
    assert dc.LTLOfSingleTrace(["p", "q"], [["p", "~q"], ["~p", "q"]]) == "p&~q&X(~p&q&~X(p|~p))"
    assert dc.overFittedCase(["p", "q"], ["1,0;0,1", "1,1"]) == \
        "(p&~q&X(~p&q&~X(p|~p)))|(p&q&~X(p|~p))"
