"""Divide-and-conquer learning over large trace sets: the reference's dc.py driver
(code/dc.py:189-327) on this library, in process.

The reference writes every sub-problem to a file and runs the enumerator binary on it
(code/dc.py:8-43), and re-checks sub-formulas on the host with bitarray (code/dc.py:136-187).
Here a sub-problem is a pair of index lists into one base instance; it is learned by one
long-lived engine (`Engine.learn`), and formulas are checked on the device
(`api.evaluate`, once per distinct formula on all traces of the base instance).

DetSplit halves the positives and negatives, learns the halves, and patches the result with
conjunctions / disjunctions of further sub-results (code/dc.py:190-252).  RandSplit learns a
random window (halved until the enumerator succeeds) and recurses on the traces the result
gets wrong (code/dc.py:255-327).  Both return a formula string in the enumerator's format,
composed with "(f)&(g)" and "(f)|(g)".

Difference from the reference: set differences of trace lists (`set(neg) - set(...)`) keep
the traces in input order here; the reference iterates a Python set of trace strings, whose
order depends on the interpreter's string hashing.
"""
from __future__ import annotations

import random
import time

import numpy as np

from . import api
from .gen import Instance


def sub_instance(base: Instance, pos: list, neg: list) -> Instance:
    """The traces base.pos[pos] + base.neg[neg] as an instance (indices are per side)."""
    idx = list(pos) + [base.num_pos + j for j in neg]
    offs = np.zeros(len(idx) + 1, dtype=np.int32)
    parts = []
    for k, t in enumerate(idx):
        a, b = int(base.offsets[t]), int(base.offsets[t + 1])
        parts.append(base.steps[a:b])
        offs[k + 1] = offs[k] + (b - a)
    steps = np.concatenate(parts).astype(np.uint32) if parts else np.zeros(0, np.uint32)
    return Instance(len(pos), len(neg), base.alphabet, steps, offs, base.hidden)


class Timeout(Exception):
    pass


class Unsolvable(Exception):
    """A sub-problem of at most one trace has no formula within the cost bound, or the
    recursion came back to a sub-problem it is still solving (e.g. one trace both positive
    and negative).  The reference recurses on both forever."""


class Driver:
    """One divide-and-conquer run over `base`.  `solve(pos, neg)` returns a formula for the
    sub-problem or None; `holds(formula)` returns, for every trace of `base`, whether the
    formula holds at position 0 (positives first).  By default both run on the device."""

    def __init__(self, base: Instance, engine: api.Engine | None = None, solve=None, holds=None,
                 costs=(1,) * 8, max_cost=500, rlx_type=3, neg_type=2, key_mode=api.KEY_EXACT, deadline=None):
        self.base = base
        self.engine = engine
        self.opts = dict(costs=costs, max_cost=max_cost, rlx_type=rlx_type, neg_type=neg_type, key_mode=key_mode)
        self._solve = solve or self._engine_solve
        self._holds = holds or (lambda f: api.evaluate(base, f)[1])
        self._cache = {}
        self.deadline = deadline
        self.calls = 0
        self._open = set()  # sub-problems on the recursion stack

    def _engine_solve(self, pos, neg):
        r = self.engine.learn(sub_instance(self.base, pos, neg), **self.opts)
        return r.formula if r.status == api.FOUND else None

    def solve(self, pos, neg):
        if self.deadline is not None and time.monotonic() > self.deadline:
            raise Timeout()
        self.calls += 1
        return self._solve(list(pos), list(neg))

    def _h(self, f):
        h = self._cache.get(f)
        if h is None:
            h = np.asarray(self._holds(f), dtype=bool)
            self._cache[f] = h
        return h

    def match_pos(self, f, pos):
        h = self._h(f)
        return [bool(h[i]) for i in pos]

    def match_neg(self, f, neg):
        h = self._h(f)
        return [bool(h[self.base.num_pos + j]) for j in neg]

    def _guarded(self, tag, step, window, pos, neg):
        key = (tag, tuple(pos), tuple(neg))
        if key in self._open:
            raise Unsolvable()
        self._open.add(key)
        try:
            return step(window, pos, neg)
        finally:
            self._open.discard(key)

    # ------------------------------------------------------------ DetSplit (dc.py:190-252)
    def det_split(self, window, pos, neg):
        return self._guarded("det", self._det_split, window, pos, neg)

    def _det_split(self, window, pos, neg):
        if len(pos) + len(neg) <= window:
            f = self.solve(pos, neg)
            if f is not None:
                return f
            if len(pos) + len(neg) <= 1:
                raise Unsolvable()
        p1, p2 = pos[:len(pos) // 2], pos[len(pos) // 2:]
        n1, n2 = neg[:len(neg) // 2], neg[len(neg) // 2:]
        phi11 = self.det_split(window, p1, n1)
        on_p2, on_n2 = self.match_pos(phi11, p2), self.match_neg(phi11, n2)
        if all(on_p2) and not any(on_n2):
            return phi11
        if not any(on_n2):
            left = phi11
        else:
            n2_and = [x for x, m in zip(n2, on_n2) if m]
            phi12 = self.det_split(window, p1, n2_and)
            drop = set(n2_and)
            rest = [x for x in neg if x not in drop]
            left = phi12 if not any(self.match_neg(phi12, rest)) else f"({phi11})&({phi12})"
            if all(self.match_pos(left, p2)):
                return left
        p2_left = [x for x, m in zip(p2, self.match_pos(left, p2)) if not m]
        phi21 = self.det_split(window, p2_left, n1)
        drop = set(p2_left)
        others = [x for x in pos if x not in drop]
        on_p1, on_n2 = self.match_pos(phi21, others), self.match_neg(phi21, n2)
        if all(on_p1) and not any(on_n2):
            return phi21
        if not any(on_n2):
            right = phi21
        else:
            n2_and = [x for x, m in zip(n2, on_n2) if m]
            phi22 = self.det_split(window, p2_left, n2_and)
            drop = set(n2_and)
            rest = [x for x in neg if x not in drop]
            right = phi22 if not any(self.match_neg(phi22, rest)) else f"({phi21})&({phi22})"
            if all(self.match_pos(right, others)):
                return right
        return f"({left})|({right})"

    # ------------------------------------------------------------ RandSplit (dc.py:255-327)
    def rand_split(self, window, pos, neg):
        return self._guarded("rand", self._rand_split, window, pos, neg)

    def _rand_split(self, window, pos, neg):
        rnd = random.Random(0)  # the reference reseeds at every call (dc.py:257)
        win = window
        while True:
            if len(pos) + len(neg) <= win:
                p1, n1 = pos, neg
            elif len(pos) <= win / 2:
                p1 = pos
                n1 = rnd.sample(neg, win - len(p1))
            elif len(neg) <= win / 2:
                n1 = neg
                p1 = rnd.sample(pos, win - len(n1))
            else:
                p1 = rnd.sample(pos, int(win / 2))
                n1 = rnd.sample(neg, win - len(p1))
            phi11 = self.solve(p1, n1)
            if phi11 is not None:
                break
            if win <= 1:
                raise Unsolvable()
            win = int(win / 2)
        on_p, on_n = self.match_pos(phi11, pos), self.match_neg(phi11, neg)
        p2 = [x for x, m in zip(pos, on_p) if not m]
        n2 = [x for x, m in zip(neg, on_n) if m]
        p1 = [x for x, m in zip(pos, on_p) if m]
        n1 = [x for x, m in zip(neg, on_n) if not m]
        if not p2 and not n2:
            return phi11
        if not n2:
            left = phi11
        else:
            phi12 = self.rand_split(window, p1, n2)
            left = phi12 if not any(self.match_neg(phi12, n1)) else f"({phi11})&({phi12})"
            if all(self.match_pos(left, p2)):
                return left
        phi21 = self.rand_split(window, p2, n1)
        if all(self.match_pos(phi21, p1)) and not any(self.match_neg(phi21, n2)):
            return phi21
        if not any(self.match_neg(phi21, n2)):
            right = phi21
        else:
            phi22 = self.rand_split(window, p2, n2)
            right = phi22 if not any(self.match_neg(phi22, n1)) else f"({phi21})&({phi22})"
            if all(self.match_pos(right, p1)):
                return right
        return f"({left})|({right})"


def formula_size(ltl: str) -> int:
    """The reference's formula size measure (code/dc.py:329-330, `c`): the characters of the
    string other than ',', ' ', '(' and ')'."""
    return sum(ch not in ",() " for ch in ltl)


def over_fitted(alphabet, pos_lines) -> str:
    """The reference's over-fitted formula for a set of positive traces (code/dc.py:332-356,
    `LTLOfSingleTrace` and `overFittedCase`).  `alphabet` is the letters in the file's value
    order; each line is a Scarlet trace ("1,0;0,1").  A trace becomes the chain
    "l0&X(l1&X(... ln&~X(a|~a)))", li the conjunction of every letter or its negation at step
    i and a the first letter (so the chain also says the trace ends there); several traces
    are joined as "(f1)|(f2)|...".  The result is in the reference's infix form, not the
    enumerator's fully parenthesised one."""
    a0 = alphabet[0]
    chains = []
    for line in pos_lines:
        steps = ["&".join(a if v == "1" else "~" + a for a, v in zip(alphabet, tok.split(",")))
                 for tok in line.split(";")]
        f = f"{steps[-1]}&~X({a0}|~{a0})"
        for lit in reversed(steps[:-1]):
            f = f"{lit}&X({f})"
        chains.append(f)
    return chains[0] if len(chains) == 1 else "|".join(f"({f})" for f in chains)


def run_dc(base: Instance, algo: str = "rand", window: int = 64, timeout_s: float = 2000.0, engine=None,
           **opts) -> dict:
    """The reference's runDC (code/dc.py:368-387) on an instance: the formula (or 'Function
    timed out.'), wall time, sub-problems learned."""
    own = engine is None
    eng = engine or api.Engine(slots_log2=24, cache_bytes=4 << 30, max_traces=max(window, 64))
    try:
        d = Driver(base, eng, deadline=time.monotonic() + timeout_s, **opts)
        pos, neg = list(range(base.num_pos)), list(range(base.num_neg))
        t0 = time.perf_counter()
        try:
            f = (d.rand_split if algo == "rand" else d.det_split)(window, pos, neg)
        except Timeout:
            f = "Function timed out."
        except Unsolvable:
            f = "not_found"
        el = time.perf_counter() - t0
    finally:
        if own:
            eng.close()
    return {"formula": f, "seconds": el, "subproblems": d.calls, "size": (base.num_pos, base.num_neg)}
