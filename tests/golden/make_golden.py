"""Golden vectors from the reference enumerator itself.

The reference (MojtabaValizadeh/ltl-learning-on-gpus) ships no expected outputs,
so they are made here:

  1. ``python tests/golden/make_golden.py inputs``
        writes the seeded fixture files to tests/golden/inputs/ and the run list to
        tests/golden/manifest.json (shapes of the reference's own benchmark families:
        Hamming neighbourhoods, 10+10 traces of length 5, cfg1-like 20+20 traces);
  2. ``make -C oracle ref``  (in a checkout that has the reference sources)
        compiles code/ltli6463.cu twice into oracle/_ref/: with and without
        -D MEASUREMENT_MODE;
  3. ``python tests/golden/make_golden.py run --out <raw dir>``  (on a B200)
        runs both binaries on every manifest entry and keeps their stdout;
  4. ``python tests/golden/make_golden.py collect --raw <raw dir>``
        parses the outputs into tests/golden/reference_runs.json.

Only step 3 needs a GPU; steps 1 and 4 and the tests that read the JSON do not.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
INPUTS = os.path.join(HERE, "inputs")
MANIFEST = os.path.join(HERE, "manifest.json")
RUNS = os.path.join(HERE, "reference_runs.json")
REF_PROGRESS = os.path.join(ROOT, "oracle", "_ref", "ltli6463_progress")
REF_MEASURE = os.path.join(ROOT, "oracle", "_ref", "ltli6463_measure")

UNIT = [1] * 8
SKEW = [1, 2, 1, 1, 2, 3, 3, 2]   # a non-unit cost function: p ~ & | X F G U


def _gen():
    sys.path.insert(0, ROOT)
    from __graft_entry__ import load_package
    load_package()
    from ltlb200 import gen
    return gen


def fixtures():
    """(name, instance) pairs; every instance is fully determined by its seed."""
    g = _gen()
    out = []
    for length in (3, 4, 5):
        out.append((f"ham1_len{length}", g.hamming_neighbourhood(length, 2, length, 1)))
    out.append(("ham2_len3", g.hamming_neighbourhood(3, 2, 3, 2)))
    for s in range(4):
        out.append((f"f10x10_p2_s{s}", g.generate(100 + s, 2, 10, 10, 5, 5, 0.5, 4)))
        out.append((f"f10x10_p3_s{s}", g.generate(200 + s, 3, 10, 10, 5, 5, 0.5, 5)))
    for s in (508, 512, 530):   # seeds whose minimal cost is 8 or 9
        out.append((f"deep8x8_p3_s{s}", g.generate(s, 3, 8, 8, 7, 7, 0.5, 9)))
    for s in range(3):
        out.append((f"e10x2_p3_s{s}", g.generate(300 + s, 3, 10, 2, 4, 8, 0.5, 6)))
    for s in range(4):
        out.append((f"cfg1_s{s}", g.generate(400 + s, 2, 20, 20, 8, 16, 0.5, 5)))
    out.append(("cfg1_deep", g.generate(450, 2, 20, 20, 8, 16, 0.5, 8)))
    out.append(("over64", g.generate(600, 2, 40, 40, 4, 6, 0.5, 4)))
    base = g.generate(601, 2, 3, 3, 60, 63, 0.5, 3)
    long_steps = list(base.steps[:base.offsets[1]]) + [1] * (64 - int(base.offsets[1]))
    rest = list(base.steps[base.offsets[1]:])
    import numpy as np
    offs = np.concatenate([[0], np.cumsum([64] + list(np.diff(base.offsets)[1:]))]).astype(np.int32)
    out.append(("len64", g.Instance(base.num_pos, base.num_neg, base.alphabet,
                                    np.array(long_steps + rest, dtype=np.uint32), offs)))
    return out


def manifest_runs(insts):
    """Run list: exact-regime fixtures with both NegTypes (and a skewed cost function on
    some), bounded enumerations (maxCost below the minimal cost) for full per-level
    progress, and the relaxed regime (lenSum > 126) with each RlxUnqChkTyp."""
    runs = []

    def add(name, costs, max_cost, r, neg):
        runs.append(dict(id=f"{name}__c{''.join(map(str, costs))}_m{max_cost}_r{r}_n{neg}", file=f"{name}.trace",
                         costs=costs, max_cost=max_cost, rlx=r, neg=neg))

    for name, inst in insts:
        lensum = int(inst.lengths.sum())
        if name.startswith("ham"):
            add(name, UNIT, 500 if name != "ham1_len5" else 14, 3, 1)
            add(name, UNIT, 500 if name != "ham1_len5" else 14, 3, 2)
        elif name.startswith("f10x10") or name.startswith("e10x2"):
            add(name, UNIT, 500, 3, 1)
            add(name, UNIT, 500, 3, 2)
            add(name, SKEW, 500, 3, 2)
        elif name.startswith("deep8x8"):
            add(name, UNIT, 7, 3, 1)
            add(name, SKEW, 9, 3, 2)
        elif name.startswith("cfg1"):
            assert lensum > 126
            for r in (1, 2, 3):
                add(name, UNIT, 6, r, 1)
                add(name, UNIT, 6, r, 2)
        elif name in ("over64", "len64"):
            add(name, UNIT, 5, 3, 2)
    return runs


def cmd_inputs(_a):
    os.makedirs(INPUTS, exist_ok=True)
    insts = fixtures()
    for name, inst in insts:
        with open(os.path.join(INPUTS, name + ".trace"), "w") as f:
            f.write(inst.to_scarlet())
    runs = manifest_runs(insts)
    with open(MANIFEST, "w") as f:
        json.dump(dict(runs=runs), f, indent=1)
    print(f"{len(insts)} inputs, {len(runs)} runs")


def _argv(binary, run):
    return [binary, os.path.join(INPUTS, run["file"])] + [str(c) for c in run["costs"]] + [
        str(run["max_cost"]), str(run["rlx"]), str(run["neg"])]


def cmd_run(a):
    os.makedirs(a.out, exist_ok=True)
    runs = json.load(open(MANIFEST))["runs"]
    for run in runs:
        for tag, binary in (("progress", REF_PROGRESS), ("measure", REF_MEASURE)):
            path = os.path.join(a.out, f"{run['id']}.{tag}.txt")
            p = subprocess.run(["timeout", "-k", "10", str(a.timeout)] + _argv(binary, run), capture_output=True,
                               text=True)
            with open(path, "w") as f:
                f.write(p.stdout)
            with open(path + ".rc", "w") as f:
                f.write(f"{p.returncode}\n{p.stderr[-2000:]}")
            print(run["id"], tag, p.returncode, flush=True)
            if p.returncode != 0:
                print(p.stderr[-500:], flush=True)
    # the device's pitch limit sets the reference's cache capacity (ltli6463.cu:1152-1156)
    try:
        from cuda.bindings import runtime as rt
        err, v = rt.cudaDeviceGetAttribute(rt.cudaDeviceAttr.cudaDevAttrMaxPitch, 0)
        with open(os.path.join(a.out, "max_pitch.txt"), "w") as f:
            f.write(str(int(v)))
    except Exception as e:  # pragma: no cover - informational only
        print("max pitch unavailable:", e)


PROG = re.compile(r"^Cost (\d+)\s*\| \((.)\) \| AllLTLs: (\d+)\s*\| StoredLTLs: (\d+)\s*\| ToBeChecked: (\d+)")


def parse_progress(text):
    return [[int(m.group(1)), m.group(2), int(m.group(3)), int(m.group(4)), int(m.group(5))]
            for m in (PROG.match(line) for line in text.splitlines()) if m]


def parse_final(text):
    out = {}
    m = re.search(r'LTL: "(.*)"', text)
    out["formula"] = m.group(1) if m else None
    for key, pat in (("all_ltls", r"Number of All LTLs: (\d+)"), ("cost", r"Cost of Final LTL: (-?\d+)"),
                     ("seconds", r"Running Time: ([0-9.]+) s")):
        m = re.search(pat, text)
        out[key] = (float(m.group(1)) if key == "seconds" else int(m.group(1))) if m else None
    out["limits_error"] = "In this version, The input can have" in text
    return out


def cmd_collect(a):
    runs = json.load(open(MANIFEST))["runs"]
    out = []
    for run in runs:
        rec = dict(run)
        for tag in ("progress", "measure"):
            path = os.path.join(a.raw, f"{run['id']}.{tag}.txt")
            text = open(path).read() if os.path.exists(path) else ""
            rc = open(path + ".rc").read().split("\n")[0] if os.path.exists(path + ".rc") else "missing"
            rec[f"{tag}_rc"] = rc
            if tag == "progress":
                rec["progress"] = parse_progress(text)
                rec["progress_final"] = parse_final(text)
            else:
                rec["final"] = parse_final(text)
        out.append(rec)
    mp = os.path.join(a.raw, "max_pitch.txt")
    doc = dict(source="reference code/ltli6463.cu built by oracle/Makefile (target ref) for sm_100a, run on a B200",
               max_pitch=int(open(mp).read()) if os.path.exists(mp) else None, runs=out)
    with open(RUNS, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"{len(out)} runs collected")


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    sub.add_parser("inputs")
    r = sub.add_parser("run")
    r.add_argument("--out", required=True)
    r.add_argument("--timeout", type=int, default=120)
    c = sub.add_parser("collect")
    c.add_argument("--raw", required=True)
    a = ap.parse_args()
    {"inputs": cmd_inputs, "run": cmd_run, "collect": cmd_collect}[a.cmd](a)


if __name__ == "__main__":
    main()
