"""The reference's divide-and-conquer module under its own names (code/dc.py), on this library.

A notebook or script written for the reference keeps working after

    from ltlb200.dc import *
    runDC(input_path, RandSplit, 64, [1, 1, 1, 1, 1, 1, 1, 1], 500, 3, 2, 2000)

Every function keeps the reference's name, argument order and meaning, and return value:
trace lists are lists of Scarlet lines ("1,0;0,1"), `alphabet` is the file's last line
("p,q"), formulas are strings in the enumerator's format.  What runs underneath differs:

  * runGPU learns in process on one long-lived engine (the reference writes "subInput" and
    starts the enumerator binary per call, code/dc.py:23-43) and returns the text the
    command line prints, so `output.split("\\n")[-2]` is still the LTL line;
  * LTLmatch and bitVec evaluate on the device (`ltlg_evaluate`) instead of with bitarray
    (code/dc.py:54-187);
  * DetSplit and RandSplit run divide.Driver over index lists of one instance built from the
    given traces.  Set differences keep input order (the reference's follow Python's string
    hashing), so RandSplit's samples, and with them its sub-problems, can differ from the
    reference's.

Uniqueness is exact by default, as this library's `ltli6463` is; `set_key_mode(api.KEY_REF)`
selects the reference's relaxed keys of type AprUnqChkTyp.  There is no CPU fallback: without
a CUDA device the calls raise.
"""
from __future__ import annotations

import os
import signal
import time

import numpy as np

from . import api, divide
from .gen import from_scarlet_text

__all__ = ["makeInputFile", "runGPU", "get_all_file_paths_in_folder", "bitVec", "LTLmatch", "DetSplit",
           "RandSplit", "c", "LTLOfSingleTrace", "overFittedCase", "runWithTimeout", "runDC"]

_key_mode = api.KEY_EXACT
_engine = None


def set_key_mode(mode: int) -> None:
    """api.KEY_EXACT (default) or api.KEY_REF (the reference's keys of type AprUnqChkTyp)."""
    global _key_mode
    _key_mode = mode


def _get_engine():
    global _engine
    if _engine is None:
        _engine = api.Engine(slots_log2=24, cache_bytes=4 << 30, max_traces=8192)
    return _engine


def close() -> None:
    """Release the module's engine (it is created on first use)."""
    global _engine
    if _engine is not None:
        _engine.close()
        _engine = None


class _DeviceBackend:
    """learn(instance, **opts) -> LearnResult; evaluate(instance, formula) -> (CS words,
    holds at position 0), one entry per trace."""

    @staticmethod
    def learn(inst, **opts):
        return _get_engine().learn(inst, **opts)

    @staticmethod
    def evaluate(inst, formula):
        return api.evaluate(inst, formula)


backend = _DeviceBackend()


def _instance(pos, neg, alphabet):
    """The traces as one instance, read with the enumerator's rules from the file
    makeInputFile would write."""
    return from_scarlet_text(_input_text(pos, neg, alphabet))


def _input_text(pos, neg, alphabet):
    return "".join(f"{p}\n" for p in pos) + "---\n" + "".join(f"{n}\n" for n in neg) + \
        "---\nAll operators\n---\n" + alphabet


def _opts(costfun, maxCost, AprUnqChkTyp, NegType):
    return dict(costs=tuple(int(c) for c in costfun), max_cost=int(maxCost), rlx_type=int(AprUnqChkTyp),
                neg_type=int(NegType), key_mode=_key_mode)


# ---------------------------------------------------------------- code/dc.py:8-43
def makeInputFile(pos, neg, alphabet):
    """Writes the sub-problem file "subInput" in the working directory (code/dc.py:8-21)."""
    with open("subInput", "w") as f:
        f.write(_input_text([str(p) for p in pos], [str(n) for n in neg], alphabet))


def _listing(lines, letters):
    out = []
    for ln in lines:
        steps = []
        for tok in ln.split(";"):
            vals = [c for c in tok if c != ","]
            steps.append("{" + ", ".join(letters[j] for j, c in enumerate(vals) if c == "1" and j < len(letters)) + "}")
        out.append("\t" + "".join(s + "\t" for s in steps) + "\n")
    return "".join(out)


def runGPU(pos, neg, alphabet, costfun, maxCost, AprUnqChkTyp, NegType):
    """Learns the sub-problem and returns the enumerator's printed output (ltli6463.cu:1642-1677):
    the traces, the cost function, the counts, the running time and, second to last, the line
    LTL: "<formula>" (or "not_found")."""
    inst = _instance(pos, neg, alphabet)
    t0 = time.perf_counter()
    r = backend.learn(inst, **_opts(costfun, maxCost, AprUnqChkTyp, NegType))
    el = time.perf_counter() - t0
    letters = [c for c in alphabet if "a" <= c <= "z"]
    cf = [int(c) for c in costfun]
    return ("\nPositive: \n" + _listing(pos, letters) + "\nNegative: \n" + _listing(neg, letters) +
            f"\nCost Function: p:{cf[0]}, ~:{cf[1]}, &:{cf[2]}, |:{cf[3]}, X:{cf[4]}, F:{cf[5]}, G:{cf[6]}, U:{cf[7]}"
            f"\nNumber of Traces: {len(pos) + len(neg)}"
            f"\nNumber of All LTLs: {r.all_ltls}"
            f"\nCost of Final LTL: {r.cost}"
            f"\nRunning Time: {el:f} s"
            f"\n\nLTL: \"{r.formula}\"\n")


def get_all_file_paths_in_folder(path):
    """Every file under `path` whose path contains ".trace" (code/dc.py:45-52)."""
    return [os.path.join(root, f) for root, _, files in os.walk(path) for f in files
            if ".trace" in os.path.join(root, f)]


# ---------------------------------------------------------------- code/dc.py:136-187
def bitVec(traceList, alphabet, formula):
    """Per trace, the positions where the formula holds, last position first (the reference's
    bitarray order: element -1 is position 0).  Lists of 0/1 instead of bitarrays."""
    inst = _instance(list(traceList), [], alphabet)
    cs, _ = backend.evaluate(inst, formula)
    lengths = np.asarray(inst.lengths)
    return [[int((int(w) >> k) & 1) for k in reversed(range(int(n)))] for w, n in zip(cs, lengths)]


def LTLmatch(traceList, alphabet, formula):
    """Per trace, whether the formula holds at position 0 (code/dc.py:185-187)."""
    if not traceList:
        return []
    return [bool(h) for h in backend.evaluate(_instance(list(traceList), [], alphabet), formula)[1]]


# ---------------------------------------------------------------- code/dc.py:189-327
def _driver(pos, neg, alphabet, costfun, maxCost, AprUnqChkTyp, NegType):
    base = _instance(pos, neg, alphabet)
    opts = _opts(costfun, maxCost, AprUnqChkTyp, NegType)

    def solve(p, n):
        r = backend.learn(divide.sub_instance(base, p, n), **opts)
        return r.formula if r.status == api.FOUND else None

    d = divide.Driver(base, solve=solve, holds=lambda f: backend.evaluate(base, f)[1], **opts)
    return d, list(range(len(pos))), list(range(len(neg)))


def DetSplit(window, pos, neg, alphabet, costfun, maxCost, AprUnqChkTyp, NegType):
    """Deterministic splitting (code/dc.py:189-251): a formula separating pos from neg, or
    "not_found" when a single trace has no formula within maxCost (the reference recurses on
    it until its timeout)."""
    d, p, n = _driver(list(pos), list(neg), alphabet, costfun, maxCost, AprUnqChkTyp, NegType)
    try:
        return d.det_split(window, p, n)
    except divide.Unsolvable:
        return "not_found"


def RandSplit(window, pos, neg, alphabet, costfun, maxCost, AprUnqChkTyp, NegType):
    """Random splitting (code/dc.py:253-327): as DetSplit, with the reference's seeded samples."""
    d, p, n = _driver(list(pos), list(neg), alphabet, costfun, maxCost, AprUnqChkTyp, NegType)
    try:
        return d.rand_split(window, p, n)
    except divide.Unsolvable:
        return "not_found"


# ---------------------------------------------------------------- code/dc.py:329-387
c = divide.formula_size


def LTLOfSingleTrace(alphabet, trace, LTL=""):
    """The chain formula of one trace given as steps of literals (code/dc.py:332-339)."""
    a0 = alphabet[0]
    for i, step in enumerate(reversed(trace)):
        lits = "&".join(step)
        LTL = f"{lits}&~X({a0}|~{a0})" if i == 0 and LTL == "" else f"{lits}&X({LTL})"
    return LTL


def overFittedCase(alphabet, pos):
    """(code/dc.py:341-356)"""
    return divide.over_fitted(alphabet, pos)


def runWithTimeout(func, args, timeout):
    """func(*args), or 'Function timed out.' after `timeout` seconds (code/dc.py:358-371)."""

    class _Expired(Exception):
        pass

    def on_alarm(signum, frame):
        raise _Expired()

    old = signal.signal(signal.SIGALRM, on_alarm)
    signal.alarm(int(timeout))
    try:
        return func(*args)
    except _Expired:
        return "Function timed out."
    finally:
        signal.alarm(0)
        signal.signal(signal.SIGALRM, old)


def runDC(filePath, dcAlgo=RandSplit, window=64, costfun=[1, 1, 1, 1, 1, 1, 1, 1], maxCost=500, RlxUnqChkTyp=3,
          NegTyp=2, timeout=2000):
    """Reads a Scarlet file the way the reference's runDC does (positives up to the first
    "---", negatives up to the fourth line from the end, the alphabet on the last line),
    runs dcAlgo under the timeout and prints Size(P, N), Time and LTL (code/dc.py:373-387)."""
    with open(filePath, "r") as f:
        lines = f.read().split("\n")
    k = lines.index("---")
    pos, neg, alphabet = lines[:k], lines[k + 1:-4], lines[-1]
    t0 = time.time()
    res = runWithTimeout(dcAlgo, [window, pos, neg, alphabet, costfun, maxCost, RlxUnqChkTyp, NegTyp], timeout)
    t1 = time.time()
    print(f"Size(P, N): ({len(pos)}, {len(neg)})")
    print(f"Time: {round(t1 - t0, 3)}s")
    print(f"LTL: {res}")
