#!/usr/bin/env python
"""Benchmark of the characteristic-set (CS) enumeration on B200.

Workload (one "step"): a fixed batch of seeded instances of the cfg2 shape — 3
propositions, 500 positive + 500 negative traces of length uniform 16-32,
Bernoulli(0.5) bits, labels from a hidden formula of size 9, unit costs, exact
uniqueness in a 2^27-slot hash set — each solved to its minimal formula.

Metric: unique CS per second (time-to-minimal-formula and candidate CS/s are
reported beside it).  Each timed step runs the batch twice:
  - through the public batch call (ltlg_batch_learn: host traces in, formula strings
    out; one persistent launch whose instance slots take the instances from a device
    queue) — CUDA-event time around the call gives ``e2e``;
  - one instance at a time on one engine (one persistent launch per learn, inputs
    already in HBM) — the summed device time of the launches gives ``value`` and the
    roofline.
After the timed steps the line also carries, each time-capped: the learned block order
against the plain one (cfg5 shape), cfg1 against the reference's own binary, cfg3 exact
against relaxed uniqueness, and cfg4's batched instances.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun) every rank solves its own batch (weak scaling, no data-path
collective); rank 0 prints the JSON line with the max step time over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-minimal-formula & unique CS/s; learned vs plain order, same cost"
UNIT = "unique CS/s"
WORKLOAD = ("cfg2: 3 props, 500+500 traces, len U[16,32], Bernoulli(0.5), hidden formula size 9, unit costs, "
            "exact uniqueness, 2^27-slot hash set; a batch of seeded instances solved to the minimal formula")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seeds", type=str, default="0-39", help="seed range a-b of the batch (per rank)")
    ap.add_argument("--max-cost", type=int, default=500)
    ap.add_argument("--no-stop", action="store_true", help="enumerate every level up to --max-cost")
    ap.add_argument("--cache-gb", type=float, default=6.0, help="language cache per engine")
    ap.add_argument("--slots", type=int, default=20,
                    help="instance slots of the batch call; 0 times the single engine only (profiling runs)")
    ap.add_argument("--slot-cache-gb", type=float, default=5.0,
                    help="language cache per batch slot (the largest instance of the batch must fit: 3.9 GB)")
    ap.add_argument("--slot-slots-log2", type=int, default=24, help="hash slots per batch slot")
    ap.add_argument("--slots-log2", type=int, default=27)
    ap.add_argument("--small-rows", type=int, default=1, help="small levels: right rows per warp and item")
    ap.add_argument("--right-chunk", type=int, default=16, help="large levels: right rows per binary item")
    ap.add_argument("--unary-rows", type=int, default=32, help="large levels: source rows per unary item")
    ap.add_argument("--left-tile", type=int, default=4, help="left rows staged in shared memory per binary item")
    ap.add_argument("--block-threads", type=int, default=1024, help="kept for the engine config layout (the level kernel runs 1024 threads per CTA)")
    ap.add_argument("--cpu-sample-s", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--quiet-extra", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain block order comparison")
    ap.add_argument("--no-extras", action="store_true", help="skip the cfg1 / cfg3 / cfg4 objects of the line")
    ap.add_argument("--workload", choices=["cfg2", "cfg3", "cfg4"], default="cfg2",
                    help="cfg3: exact vs relaxed uniqueness on one large instance; cfg4: 4096 batched instances")
    ap.add_argument("--time-limit", type=float, default=120.0, help="cfg3: seconds per uniqueness mode")
    return ap.parse_args()


def seeds_of(spec: str, rank: int):
    a, b = (int(x) for x in spec.split("-"))
    width = b - a + 1
    return list(range(a + rank * width, b + 1 + rank * width))


def reduce_over_ranks(step_t: float, kern_t: float, totals, device: str):
    """Whole-job figures: the slowest rank's step and kernel times (max) and the units all
    ranks processed (sum).  Every rank calls it; works on NCCL (cuda) and gloo (cpu)."""
    import torch
    import torch.distributed as D
    t = torch.tensor([step_t, kern_t], dtype=torch.float64, device=device)
    D.all_reduce(t, op=D.ReduceOp.MAX)
    u = torch.tensor(list(totals), dtype=torch.float64, device=device)
    D.all_reduce(u, op=D.ReduceOp.SUM)
    return float(t[0]), float(t[1]), [float(x) for x in u]


def make_batch(seeds):
    from __graft_entry__ import load_package
    load_package()
    from ltlb200 import gen
    return [gen.generate(s, 3, 500, 500, 16, 32, 0.5, 9) for s in seeds]


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, enabled: bool):
        self.enabled = enabled
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if self.enabled:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                     "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.path or not os.path.exists(self.path):
            return None
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sms:
            return None
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxes), "samples": len(sms),
                "reasons": sorted(reasons)}


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_per_candidate():
    """Bytes of DRAM traffic per evaluated candidate of the level kernel, from the ncu
    summary committed under profiles/ (None when no summary exists yet)."""
    p = os.path.join(ROOT, "profiles", "level_kernel_cfg2.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_candidate:"):
            return float(line.split(":")[1])
    return None


def cpu_baseline(batch, sample_s: float, threads: int = 0, costs=(1,) * 8):
    """The CPU port of the same enumeration (oracle/, OpenMP) on the host cores, on the
    batch in order until sample_s seconds are spent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    t0 = time.perf_counter()
    uniques = cands = solved = 0
    used = 0
    for inst in batch:
        left = sample_s - (time.perf_counter() - t0)
        if left <= 0:
            break
        r = O.learn(inst, costs=costs, neg_type=1, threads=threads, cache_rows=4 << 20, time_limit_s=left,
                    keep_rows=False)
        uniques += r.num_rows - len(inst.alphabet)
        cands += r.evaluated - len(inst.alphabet)
        used = r.threads
        solved += r.status == O.FOUND
    el = time.perf_counter() - t0
    return {"value": uniques / el, "unit": UNIT, "cores": used, "kind": "port",
            "sample": f"{solved} of {len(batch)} batch instances solved in {el:.1f} s "
                      f"(CPU port of the same enumeration, OpenMP, exact uniqueness)",
            "candidate_cs_per_s": cands / el, "seconds": el}


def learned_order_report(ekw, repeats: int = 2):
    """Time-to-minimal-formula with the packaged learned block order against the plain order,
    on held-out Hamming-style instances (4 propositions, 1000 positive traces of length
    20-48, 1000 negatives each a positive with 1-3 bits flipped; hidden formula of size 9),
    best of `repeats` per instance and order.  The minimal cost must be the same."""
    from ltlb200 import api, learned
    specs = [(s, 1000, 9) for s in learned.HELD_OUT_SEEDS]
    insts = list(learned.instances(specs, workers=8, chunk=2))
    kw = dict(ekw, slots_log2=max(ekw.get("slots_log2", 26), 26))
    with api.Engine(**kw) as eng:
        rows = learned.compare(eng, insts, learned.load_scorer(), repeats=repeats)
    s = learned.summarize(rows)
    hard = [r for r in rows if r["cost_plain"] >= 8]
    return {
        "workload": "cfg5 shape: 4 props, 1000 pos (len U[20,48], Bernoulli(0.5)) + 1000 negatives = positives "
                    "with 1-3 flipped bits, hidden formula size 9; held-out seeds "
                    f"{learned.HELD_OUT_SEEDS[0]}-{learned.HELD_OUT_SEEDS[-1]}",
        "instances": s["instances"], "same_cost": s["same_cost"],
        "time_to_minimal_ms": {"plain": s["ms_plain"], "learned": s["ms_learned"]},
        "speedup": s["speedup"],
        "device_ms": {"plain": s["device_ms_plain"], "learned": s["device_ms_learned"]},
        "device_speedup": s["device_speedup"],
        "candidates_before_find": {"plain": s["evaluated_plain"], "learned": s["evaluated_learned"]},
        "cost_ge_8": {"instances": len(hard),
                      "speedup_total_time": (sum(r["ms_plain"] for r in hard) / max(1e-9, sum(r["ms_learned"] for r in hard)))
                      if hard else None,
                      "device_speedup": (sum(r["dev_ms_plain"] for r in hard) /
                                         max(1e-9, sum(r["dev_ms_learned"] for r in hard))) if hard else None},
        "per_instance": [[r["cost_plain"], round(r["ms_plain"], 3), round(r["ms_learned"], 3)] for r in rows],
        "scorer": "scorer_hamming.npy: MLP 32-64-64-1, BF16/FP32, trained on the GPU on 198,070 block records",
        "spec_shape": near_miss_report(ekw),
    }


def near_miss_report(ekw, seeds=range(4), max_cost=8, time_limit_s=20.0):
    """The cfg5 shape as specified: 4 props, 1000 random positives (len U[20,48], Bernoulli(0.5)),
    1000 negatives = positives with 1-3 flipped bits (exact duplicates of positives rejected),
    no planted formula.  Both orders enumerate every level up to max_cost (no separating formula
    exists there), so the learned order has no level of a find to reorder."""
    from ltlb200 import api, gen, learned
    insts = [gen.generate_near_miss(s, 4, 1000, 1000, 20, 48, 0.5) for s in seeds]
    kw = dict(ekw, slots_log2=max(ekw.get("slots_log2", 26), 26))
    with api.Engine(**kw) as eng:
        rows = learned.compare(eng, insts, learned.load_scorer(), repeats=1, max_cost=max_cost,
                               time_limit_s=time_limit_s)
    s = learned.summarize(rows)
    return {"workload": f"4 props, 1000 random pos (len U[20,48], Bernoulli(0.5)) + 1000 negatives = positives "
                        f"with 1-3 flipped bits, no planted formula; seeds {seeds[0]}-{seeds[-1]}; max_cost {max_cost}",
            "found": sum(r["status_plain"] == api.FOUND for r in rows), "instances": s["instances"],
            "same_cost": s["same_cost"], "time_ms": {"plain": s["ms_plain"], "learned": s["ms_learned"]},
            "speedup": s["speedup"]}


def extras(device: int, time_limit: float) -> dict:
    """The cfg1 / cfg3 / cfg4 objects of the line (each skipped with its reason on failure)."""
    from ltlb200 import workloads
    out = {}
    jobs = [("cfg1_vs_reference_binary",
             lambda: workloads.run_cfg1(os.path.join(ROOT, "oracle", "_ref", "ltli6463_measure"),
                                        os.path.join(ROOT, "tests", "golden", "inputs"))),
            ("cfg3", lambda: workloads.run_cfg3(time_limit_s=time_limit, device=device)),
            ("cfg4", lambda: workloads.run_cfg4(device=device))]
    for key, job in jobs:
        t0 = time.perf_counter()
        try:
            out[key] = job()
        except Exception as exc:  # a failed extra must not lose the main line
            out[key] = {"error": f"{type(exc).__name__}: {exc}"}
        out[key]["wall_s"] = time.perf_counter() - t0
    return out


def run_reference(a):
    ws, rank, local = dist()
    if rank != 0:
        return 0
    batch = make_batch(seeds_of(a.seeds, 0))
    per_step = max(5.0, min(a.cpu_sample_s, 60.0))
    for _ in range(a.warmup):
        cpu_baseline(batch[:1], per_step / 4)
    vals, secs = [], []
    last = None
    for _ in range(a.steps):
        last = cpu_baseline(batch, per_step)
        vals.append(last["value"])
        secs.append(last["seconds"])
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * statistics.median(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "seeds": a.seeds, "parallelism": "cpu"},
            "cpu_baseline": {**last, "value": value},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_workload(a):
    """The cfg3 / cfg4 lines (one GPU; other ranks exit)."""
    import torch
    ws, rank, local = dist()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    load_package()
    from ltlb200 import workloads
    if a.workload == "cfg3":
        rep = workloads.run_cfg3(time_limit_s=a.time_limit, device=local)
        ex = rep["exact"]
        line = {"metric": "unique CS/s; completeness loss of relaxed (64-bit hash) uniqueness", "value":
                ex["unique_cs_per_s"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "u64",
                "data": "synthetic", "config": {"workload": rep["workload"]}, **rep}
    else:
        rep = workloads.run_cfg4(device=local)
        line = {"metric": "instances/s and unique CS/s of a batched run", "value": rep["instances_per_s"],
                "unit": "instances/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u64", "data": "synthetic",
                "config": {"workload": rep["workload"]}, **rep}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(a):
    import torch
    ws, rank, local = dist()
    if ws > 1:
        import torch.distributed as D
        D.init_process_group(backend="nccl", timeout=datetime.timedelta(seconds=300),
                             device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    load_package()
    from ltlb200 import api
    batch = make_batch(seeds_of(a.seeds, rank))
    ekw = dict(device=local, slots_log2=a.slots_log2, cache_bytes=int(a.cache_gb * (1 << 30)), small_rows=a.small_rows,
               right_chunk=a.right_chunk, unary_rows=a.unary_rows, left_tile=a.left_tile,
               block_threads=a.block_threads)
    eng = api.Engine(**ekw)
    bkw = dict(ekw, cache_bytes=int(a.slot_cache_gb * (1 << 30)), slots_log2=a.slot_slots_log2)
    pool = api.Batch(workers=a.slots, **bkw) if a.slots > 0 else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    opts = dict(neg_type=1, max_cost=a.max_cost, stop_at_found=not a.no_stop)

    def seq_step():
        return [eng.learn(inst, record_levels=True, **opts) for inst in batch]

    def batch_step():
        return pool.learn(batch, **opts) if pool else seq_step()

    for _ in range(a.warmup):
        if pool:
            pool.learn(batch, **opts)
        seq_step()
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            import torch.distributed as D
            D.barrier()

    step_ms, kern_ms, launches = [], [], 0
    uniq_e2e = cand_e2e = uniq_seq = cand_seq = 0
    level_launches = 0  # level-kernel launches of the one-at-a-time pass (one per learn that ran levels)
    ttm, costs = [], []
    h2d = d2h = 0
    with Clocks(local, enabled=not a.no_clocks) as clk:
        for _ in range(a.steps):
            flush.fill_(1)  # L2 flush between timed steps (256 MiB write)
            torch.cuda.synchronize()
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            res = batch_step()  # blocks until every engine's stream is idle
            e1.record()
            torch.cuda.synchronize()
            barrier()
            step_ms.append(e0.elapsed_time(e1))
            launches += 2 if pool else sum(r.launches for r in res)  # the batch call: its start and level launches
            for inst, r in zip(batch, res):
                assert r.status == api.FOUND or a.no_stop, (r.status, r.formula)
                uniq_e2e += r.rows - len(inst.alphabet)
                cand_e2e += r.evaluated - len(inst.alphabet)
                ttm.append(r.device_ms)
                costs.append(r.cost)
                h2d += len(inst.alphabet) * inst.n * 8 + inst.n * 12  # letter CSs + word metadata
                d2h += len(r.formula) + 64
            flush.fill_(2)
            torch.cuda.synchronize()
            seq = seq_step() if pool else res
            kern_ms.append(sum(r.device_ms for r in seq))
            for inst, r in zip(batch, seq):
                uniq_seq += r.rows - len(inst.alphabet)
                cand_seq += r.evaluated - len(inst.alphabet)
                level_launches += 1 if r.levels else 0  # one persistent level-kernel launch per learn
    clocks = clk.summary()
    K = a.steps
    step_t = sum(step_ms) / 1e3
    kern_t = sum(kern_ms) / 1e3
    n = batch[0].n
    tot = [float(uniq_e2e), float(cand_e2e), float(uniq_seq), float(cand_seq)]
    if ws > 1:
        step_t, kern_t, tot = reduce_over_ranks(step_t, kern_t, tot, "cuda")
    if rank == 0:
        peak, peak_kind = measured_peak_gbs()
        per_unit = 8 * n + 8
        alg_bytes = (cand_seq + uniq_seq) * per_unit  # this rank's bytes over its own kernel time
        achieved = alg_bytes / (sum(kern_ms) / 1e3) / 1e9
        tpc = profile_traffic_per_candidate()
        nl = max(1, level_launches)
        line = {
            "metric": METRIC, "value": tot[2] / kern_t, "unit": UNIT, "n_gpus": ws, "steps": K,
            "warmup": a.warmup, "ms_per_step": 1e3 * kern_t / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "seeds_per_rank": a.seeds, "instances_per_step": len(batch) * ws,
                       "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"instances x{ws} ranks; one persistent launch per GPU drains the batch "
                                      f"through {a.slots} instance slots",
                       "value": "unique CS / summed device time of the learns, one instance at a time "
                                "(one persistent launch each); ms_per_step is that time per step",
                       "e2e": "unique CS / CUDA-event time of ltlg_batch_learn on host traces"},
            "time_to_minimal_formula_ms": {"mean": statistics.mean(ttm), "median": statistics.median(ttm),
                                           "max": max(ttm), "min_cost": min(costs), "max_cost": max(costs),
                                           "note": "device time of each instance inside the batch launch, "
                                                   "from its slot's set-up to its result"},
            "candidate_cs_per_s": tot[3] / kern_t,
            "e2e": {"value": tot[0] / step_t, "unit": UNIT, "h2d_bytes_per_step": h2d // K,
                    "d2h_bytes_per_step": d2h // K, "candidate_cs_per_s": tot[1] / step_t,
                    "ms_per_step": 1e3 * step_t / K},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (tpc * cand_seq / nl) if tpc else None,
                         "alg_bytes_per_launch": alg_bytes / nl,
                         "kernel": "level_kernel", "bytes_per_unit": per_unit,
                         "units": "candidates evaluated + uniques stored",
                         "timing": "CUDA events on the engine stream around each learn's persistent launch "
                                   "(every level, the device planner included), summed over the "
                                   "one-at-a-time pass",
                         "traffic_source": "ncu DRAM bytes per candidate of the cost-8 level_kernel launch "
                                           "(profiles/level_kernel_cfg2.txt) x mean candidates per launch"},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if ws == 1 and not a.no_learned:
            line["learned_order"] = learned_order_report(ekw)
        if ws == 1 and not a.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(batch, a.cpu_sample_s)
    if pool:
        pool.close()
    eng.close()
    if rank == 0:
        if ws == 1 and not a.no_extras:  # after the timed buffers are released: cfg3 wants most of HBM
            line.update(extras(local, a.time_limit))
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as D
        D.destroy_process_group()
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "cfg2":
        return run_workload(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
