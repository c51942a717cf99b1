"""The reference enumerator and this library side by side on the same GPU.

oracle/_ref/ltli6463_measure is code/ltli6463.cu built from its own sources with
-D MEASUREMENT_MODE (oracle/Makefile, target ref).  Both command lines get the same input
file and the same twelve arguments; where the reference is exact (lenSum <= 126) both must
report the same minimal cost and the same candidate count ("Number of All LTLs"), in the
default schedule and under --per-block: a found level is counted through the first block of
the reference's order that holds an accepting candidate, as the reference stops after that
block (code/ltli6463.cu:1232-1234).  The running times each prints (the
reference: around LTLI, ltli6463.cu:1626-1636; here: around ltlg_learn, both including the
CUDA context and the device allocations of a fresh process), and the time of the same learn
on a warm in-process engine, are printed as one JSON line per case (run with -s to see them).
"""
import json
import os
import subprocess

import pytest

from ltlb200 import api
from helpers import fixture_path, lensum, load_fixture

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ltli6463_measure")

# (file, max cost, RlxUnqChkTyp, NegType): inputs of the reference's benchmark shapes
CASES = [
    ("ham1_len3.trace", 500, 3, 1),
    ("ham1_len4.trace", 500, 3, 1),
    ("ham1_len5.trace", 14, 3, 1),
    ("ham2_len3.trace", 500, 3, 1),
    ("e10x2_p3_s1.trace", 500, 3, 1),
    ("deep8x8_p3_s508.trace", 7, 3, 1),
    ("cfg1_s2.trace", 6, 3, 1),
    ("cfg1_deep.trace", 6, 3, 1),
]


def parse(out):
    lines = out.split("\n")
    get = lambda key: next((ln.split(": ", 1)[1] for ln in lines if ln.startswith(key + ": ")), None)
    t = get("Running Time")
    return {"all_ltls": int(get("Number of All LTLs")), "cost": int(get("Cost of Final LTL")),
            "seconds": float(t.split()[0]) if t else None, "formula": lines[-2][len('LTL: "'):-1]}


def run(binary, path, max_cost, rlx, neg, *flags):
    p = subprocess.run([binary, path, *["1"] * 8, str(max_cost), str(rlx), str(neg), *flags],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    return parse(p.stdout)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built (oracle/Makefile target ref)")
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_reference_binary_side_by_side(case):
    name, max_cost, rlx, neg = case
    path = fixture_path(name)
    inst = load_fixture(name)
    ref = run(REF, path, max_cost, rlx, neg)
    mine = run(api.CLI_PATH, path, max_cost, rlx, neg)
    with api.Engine(slots_log2=24, cache_bytes=4 << 30, max_rows=8 << 20) as e:
        e.learn(inst, max_cost=max_cost, neg_type=neg)  # warm-up
        warm = e.learn(inst, max_cost=max_cost, neg_type=neg)
    exact = lensum(inst) <= 126
    if exact:
        per_block = run(api.CLI_PATH, path, max_cost, rlx, neg, "--per-block")
        assert mine["cost"] == ref["cost"] and per_block["cost"] == ref["cost"]
        assert per_block["all_ltls"] == ref["all_ltls"]
        assert mine["all_ltls"] == ref["all_ltls"]
        assert (mine["formula"] == "not_found") == (ref["formula"] == "not_found")
    assert warm.cost == mine["cost"]
    print(json.dumps({"case": name, "max_cost": max_cost, "rlx": rlx, "neg": neg, "n": inst.n,
                      "reference_exact": exact, "cost": mine["cost"], "all_ltls": mine["all_ltls"],
                      "reference_s": ref["seconds"], "cli_s": mine["seconds"], "warm_engine_s": warm.seconds,
                      "warm_engine_device_ms": warm.device_ms}))
