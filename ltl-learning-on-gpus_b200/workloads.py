"""The measured workloads besides the default bench line, and the engine autotuner.

* cfg3 — scale and relaxed mode: 5 propositions, 2000 + 2000 traces of length 32-63,
  Bernoulli(0.3) bits, hidden formula of size 12, costs ~ = X = 1, F = G = 2, & = | = 1,
  U = 3 (letters 1).  The same instance is learned with exact uniqueness and with the
  relaxed 64-bit-fingerprint uniqueness; the per-level unique counts side by side give the
  relaxed mode's completeness loss.
* cfg4 — batched learning: 4096 independent instances (2-4 propositions, 8-256 positive and
  8-256 negative traces of length 4-40, Bernoulli(0.5), hidden formula of size 3-8, unit
  costs) through the batch call (one persistent launch), with the configuration picked by
  `autotune`.
* cfg1 — the reference's own binary side by side: 2 propositions, 20 + 20 traces of length
  8-16 (the committed cfg1 fixtures), this library's ltli6463 and the reference's ltli6463
  built from its sources, same files and arguments, each one's printed Running Time, and the
  same learn on a warm engine.

Instances are seeded synthetic data of the shapes above (the reference ships none), made by
the generator in child interpreters when `workers` > 1 (the generator is plain Python).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pickle
import subprocess
import sys
import time

import numpy as np

from . import api, gen

HERE = os.path.dirname(os.path.abspath(__file__))

_CHUNK_CODE = (
    "import pickle, sys\n"
    "sys.path.insert(0, sys.argv[1])\n"
    "from __graft_entry__ import load_package\n"
    "load_package()\n"
    "from ltlb200 import gen\n"
    "kind, specs = pickle.load(sys.stdin.buffer)\n"
    "fn = getattr(gen, kind)\n"
    "sys.stdout.buffer.write(pickle.dumps([fn(*s) for s in specs]))\n")


def _run_chunk(kind, specs):
    out = subprocess.run([sys.executable, "-c", _CHUNK_CODE, os.path.dirname(HERE)],
                         input=pickle.dumps((kind, list(specs))), capture_output=True, check=True)
    return pickle.loads(out.stdout)


def generate_many(kind: str, specs, workers: int = 0, chunk: int = 64):
    """gen.<kind>(*spec) for every spec, in order; with workers > 1 in that many child
    interpreters, `chunk` specs each."""
    specs = list(specs)
    fn = getattr(gen, kind)
    if workers <= 1:
        yield from (fn(*s) for s in specs)
        return
    with cf.ThreadPoolExecutor(workers) as ex:
        futs = [ex.submit(_run_chunk, kind, specs[i:i + chunk]) for i in range(0, len(specs), chunk)]
        for f in futs:
            yield from f.result()


# ---------------------------------------------------------------- cfg3
CFG3_COSTS = (1, 1, 1, 1, 1, 2, 2, 3)  # letter, ~, &, |, X, F, G, U


def cfg3_instance(seed: int = 0, npos: int = 2000, nneg: int = 2000) -> gen.Instance:
    return gen.generate(seed, 5, npos, nneg, 32, 63, 0.3, 12)


def pick_cfg3_seed(npos=2000, nneg=2000, min_cost=5, first=0, tries=64, device=0) -> int:
    """The first seed from `first` whose instance has no separating formula below `min_cost`
    (many cfg3 draws are separated by one letter, which measures nothing)."""
    with api.Engine(device=device, slots_log2=24, cache_bytes=8 << 30, max_traces=npos + nneg) as eng:
        for seed in range(first, first + tries):
            r = eng.learn(cfg3_instance(seed, npos, nneg), costs=CFG3_COSTS, neg_type=1, max_cost=min_cost - 1)
            if r.status == api.NOT_FOUND:
                return seed
    raise RuntimeError("no cfg3 seed without a cheap separating formula")


def run_cfg3(seed=None, npos=2000, nneg=2000, time_limit_s=120.0, max_cost=10, stop_at_found=False,
             cache_gb=120.0, slots_log2=28, device=0) -> dict:
    """Enumerate one cfg3 instance with exact and with relaxed (64-bit fingerprint) uniqueness,
    every level up to max_cost in full (stop_at_found False: a level cut short by a find is
    not comparable); per-level candidates, uniques and time side by side.  seed None:
    pick_cfg3_seed()."""
    if seed is None:
        seed = pick_cfg3_seed(npos, nneg, device=device)
    inst = cfg3_instance(seed, npos, nneg)
    out = {"workload": f"cfg3: 5 props, {npos}+{nneg} traces, len U[32,63], Bernoulli(0.3), hidden formula "
                       f"size 12, costs ~=X=1 F=G=2 &=|=1 U=3, seed {seed}",
           "hidden": inst.hidden}
    runs = {}
    for name, key in (("exact", api.KEY_EXACT), ("relaxed_hash64", api.KEY_HASH64)):
        with api.Engine(device=device, slots_log2=slots_log2, cache_bytes=int(cache_gb * (1 << 30)),
                        max_rows=(1 << 30) - 1, max_traces=npos + nneg) as eng:
            t0 = time.perf_counter()
            r = eng.learn(inst, costs=CFG3_COSTS, neg_type=1, key_mode=key, max_cost=max_cost,
                          stop_at_found=stop_at_found, time_limit_s=time_limit_s, record_levels=True)
            el = time.perf_counter() - t0
        runs[name] = r
        out[name] = {"status": api.status_string(r.status), "cost": r.cost, "formula": r.formula, "seconds": el,
                     "on_the_fly": r.on_the_fly,
                     "rows": r.rows, "evaluated": r.evaluated, "device_ms": r.device_ms,
                     "cache_gb_used": r.rows * ((inst.n + 3) // 4 * 4) * 8 / 2 ** 30,
                     "unique_cs_per_s": max(0, r.rows - len(inst.alphabet)) / (r.device_ms / 1e3) if r.device_ms > 0
                     else None}
    ex, rl = runs["exact"], runs["relaxed_hash64"]

    def complete(r):  # levels that ran to their end
        lv = {l["cost"]: l for l in r.levels}
        if (stop_at_found and r.status == api.FOUND) or r.status == api.TIMEOUT or r.on_the_fly:
            lv.pop(max(lv), None) if lv else None
        return lv
    lv_e, lv_r = complete(ex), complete(rl)
    table = []
    for c in sorted(set(lv_e) & set(lv_r)):
        a, b = lv_e[c], lv_r[c]
        table.append({"cost": c, "candidates_exact": a["candidates"], "uniques_exact": a["uniques"],
                      "uniques_relaxed": b["uniques"], "lost": a["uniques"] - b["uniques"],
                      "ms_exact": round(a["ms"], 3), "ms_relaxed": round(b["ms"], 3)})
    out["levels"] = table
    lost = sum(t["lost"] for t in table)
    tot = sum(t["uniques_exact"] for t in table)
    out["completeness_loss"] = {"uniques_lost": lost, "of_uniques": tot, "fraction": lost / tot if tot else 0.0,
                                "same_cost": ex.cost == rl.cost and ex.status == rl.status}
    return out


# ---------------------------------------------------------------- cfg4
def cfg4_specs(count: int = 4096, seed: int = 0):
    """(seed, nprops, npos, nneg, lmin, lmax, p_bit, fsize) of the cfg4 instances."""
    rng = np.random.default_rng(seed)
    return [(int(seed * 1000003 + i), int(rng.integers(2, 5)), int(rng.integers(8, 257)), int(rng.integers(8, 257)),
             4, 40, 0.5, int(rng.integers(3, 9))) for i in range(count)]


AUTOTUNE_SPACE = [dict(left_tile=lt, right_chunk=rc, unary_rows=ur, slots_log2=sl, workers=w)
                  for lt in (4, 8) for rc in (8, 32) for ur in (16, 64) for sl in (20, 22) for w in (48, 96)]


def autotune(sample, space=AUTOTUNE_SPACE, cache_bytes=1 << 30, repeats=3, device=0, **opts):
    """Time the batch call on `sample` under every configuration of `space` (tile shapes,
    item sizes, hash-set size = load factor, instance slots) and return (best, table)."""
    table = []
    for cfg in space:
        c = dict(cfg)
        w = c.pop("workers")
        with api.Batch(workers=w, device=device, cache_bytes=cache_bytes, max_traces=512, **c) as b:
            b.learn(sample, **opts)  # warm-up
            best = float("inf")
            for _ in range(repeats):
                t0 = time.perf_counter()
                res = b.learn(sample, **opts)
                best = min(best, time.perf_counter() - t0)
        ok = all(r.status in (api.FOUND, api.NOT_FOUND) for r in res)
        table.append(dict(cfg, seconds=best, ok=ok))
    good = [t for t in table if t["ok"]]
    return min(good, key=lambda t: t["seconds"]), table


def run_cfg4(count=4096, seed=0, tune_sample=1024, gen_workers=16, device=0) -> dict:
    """Generate the cfg4 batch, autotune the engine configuration on a sample, learn the whole
    batch with the best one; instances/s, unique CS/s, time to minimal formula."""
    t0 = time.perf_counter()
    insts = list(generate_many("generate", cfg4_specs(count, seed), workers=gen_workers, chunk=64))
    t_gen = time.perf_counter() - t0
    opts = dict(neg_type=1)
    best, table = autotune(insts[:tune_sample], device=device, **opts)
    cfg = {k: v for k, v in best.items() if k not in ("seconds", "ok")}
    w = cfg.pop("workers")
    with api.Batch(workers=w, device=device, cache_bytes=1 << 30, max_traces=512, **cfg) as b:
        b.learn(insts[:tune_sample], **opts)
        t1 = time.perf_counter()
        res = b.learn(insts, **opts)
        el = time.perf_counter() - t1
    found = sum(r.status == api.FOUND for r in res)
    uniq = sum(r.rows - len(i.alphabet) for r, i in zip(res, insts))
    costs = [r.cost for r in res if r.status == api.FOUND]
    return {"workload": f"cfg4: {count} instances, props U[2,4], pos/neg U[8,256], len U[4,40], Bernoulli(0.5), "
                        f"hidden formula size U[3,8], unit costs",
            "instances": count, "found": found, "seconds": el, "instances_per_s": count / el,
            "unique_cs_per_s": uniq / el, "min_cost": min(costs) if costs else None,
            "max_cost": max(costs) if costs else None,
            "time_to_minimal_ms": {"mean": float(np.mean([r.device_ms for r in res])),
                                   "max": float(np.max([r.device_ms for r in res])),
                                   "note": "device time of each instance from its slot's set-up to its result"},
            "launches": "one batch-start launch and one level-kernel launch for the whole batch",
            "autotune": {"best": best, "sample": tune_sample, "configs": len(table),
                         "worst_seconds": max(t["seconds"] for t in table)},
            "generation_s": t_gen}


# ---------------------------------------------------------------- cfg1
CFG1_FILES = ("cfg1_s0.trace", "cfg1_s1.trace", "cfg1_s2.trace", "cfg1_s3.trace", "cfg1_deep.trace")


def _parse_cli(out: str) -> dict:
    lines = out.split("\n")
    get = lambda key: next((ln.split(": ", 1)[1] for ln in lines if ln.startswith(key + ": ")), None)
    t = get("Running Time")
    formula = lines[-2][len('LTL: "'):-1] if len(lines) >= 2 and lines[-2].startswith("LTL: ") else None
    return {"all_ltls": int(get("Number of All LTLs") or -1), "cost": int(get("Cost of Final LTL") or -1),
            "seconds": float(t.split()[0]) if t else None, "formula": formula}


def run_cfg1(reference_binary: str, fixtures_dir: str, max_cost: int = 6, rlx: int = 3, neg: int = 1,
             timeout_s: float = 60.0) -> dict:
    """This library's ltli6463 and the reference's, on the same cfg1 files and arguments (unit
    costs); each one's printed Running Time (both include their process's CUDA context and
    device allocations) and the time of the same learn on a warm in-process engine."""
    rows = []
    have_ref = os.path.exists(reference_binary)
    with api.Engine(slots_log2=22, cache_bytes=2 << 30, max_rows=4 << 20) as eng:
        for name in CFG1_FILES:
            path = os.path.join(fixtures_dir, name)
            args = [path] + ["1"] * 8 + [str(max_cost), str(rlx), str(neg)]
            mine = _parse_cli(subprocess.run([api.CLI_PATH] + args, capture_output=True, text=True,
                                             timeout=timeout_s).stdout)
            ref = None
            if have_ref:
                ref = _parse_cli(subprocess.run([reference_binary] + args, capture_output=True, text=True,
                                                timeout=timeout_s).stdout)
            inst = gen.from_scarlet_text(open(path).read())
            eng.learn(inst, max_cost=max_cost, neg_type=neg)
            warm = eng.learn(inst, max_cost=max_cost, neg_type=neg)
            rows.append({"file": name, "cost": mine["cost"], "reference_cost": ref["cost"] if ref else None,
                         "all_ltls": mine["all_ltls"], "reference_all_ltls": ref["all_ltls"] if ref else None,
                         "cli_s": mine["seconds"], "reference_s": ref["seconds"] if ref else None,
                         "warm_engine_ms": warm.seconds * 1e3, "warm_engine_device_ms": warm.device_ms})
    out = {"workload": f"cfg1: 2 props, 20+20 traces, len U[8,16] (the committed cfg1 fixtures), unit costs, "
                       f"maxCost {max_cost}, RlxUnqChkTyp {rlx}, NegType {neg}",
           "files": rows}
    if not have_ref:
        out["reference"] = "unavailable: the reference binary is not built (oracle/Makefile, target ref)"
    return out
