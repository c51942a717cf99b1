"""Learned block ordering: training records, training on the GPU, and the plain-vs-learned
comparison at identical minimal cost.

The scorer (csrc/order.cuh, csrc/mlp.cu) rates each (operator, left cost, right cost) block
of a level; with ``order=ORDER_LEARNED`` the engine's planner drains the level's blocks
highest score first.  Every lower level is exhausted before, and the level itself still runs
to its end unless a find stops it, so the cost found equals the plain enumerator's; only the
time to the find changes.

Records come from plain-enumerator runs (``Engine.label_blocks``): one per block of the level
holding the find, labelled 1 when the block holds an accepting candidate.  The instance family
is the Hamming-style shape (4 propositions, positives of length 20-48 with Bernoulli(0.5) bits,
each negative a positive with 1-3 bits flipped, exact duplicates of positives rejected).

    python ltl-learning-on-gpus_b200/learned_cli.py collect --out records.npz     # ~200k records
    python ltl-learning-on-gpus_b200/learned_cli.py train --records records.npz --out scorer.npy
    python ltl-learning-on-gpus_b200/learned_cli.py compare --scorer scorer.npy    # held-out seeds
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from . import api, gen

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SCORER = os.path.join(HERE, "scorer_hamming.npy")

NF, H = api.SCORER_FEATURES, 64
PARAMS = api.SCORER_PARAMS

# The packaged scorer was trained on records of seeds fs * 1000003 + npos * 7919 + i
# (fs 6..10, npos 40/100/200, i < 1600); these seeds (hidden formula size 9, 1000 + 1000
# traces) were held out for the comparison with the plain order.
HELD_OUT_SEEDS = tuple(range(900333, 900349))
TRAIN_SPECS = dict(fsizes=(6, 7, 8, 9, 10), npos=(40, 100, 200), per=1600)


def training_specs(fsizes=TRAIN_SPECS["fsizes"], npos=TRAIN_SPECS["npos"], per=TRAIN_SPECS["per"]):
    """(seed, npos, fsize) of the packaged scorer's training instances."""
    return [(fs * 1000003 + n * 7919 + i, n, fs) for fs in fsizes for n in npos for i in range(per)]


def hamming_instance(seed: int, npos: int = 1000, nneg: int = 1000, fsize: int = 6) -> gen.Instance:
    """The Hamming-style shape: 4 propositions, lengths 20-48, Bernoulli(0.5), 1-3 flips."""
    return gen.generate_hamming(seed, 4, npos, nneg, 20, 48, 0.5, fsize)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (the packed FP32 layout of the C ABI)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, dtype=np.float32)
    w1, b1 = 0, H * NF
    w2 = b1 + H
    b2 = w2 + H * H
    w3 = b2 + H
    p[w1:b1] = rng.normal(0.0, np.sqrt(2.0 / NF), H * NF)
    p[w2:b2] = rng.normal(0.0, np.sqrt(2.0 / H), H * H)
    p[w3:w3 + H] = rng.normal(0.0, np.sqrt(1.0 / H), H)
    return p


def load_scorer(path: str = DEFAULT_SCORER) -> np.ndarray:
    p = np.load(path).astype(np.float32)
    if p.size != PARAMS:
        raise ValueError(f"{path}: expected {PARAMS} parameters, got {p.size}")
    return p


def _hamming_spec(spec):
    seed, npos, fsize = spec
    return hamming_instance(seed, npos, npos, fsize)


def instances(specs, workers: int = 0, chunk: int = 64):
    """Hamming-style instances for (seed, npos, fsize) specs, in order.  With workers > 1 the
    generator (plain Python) runs in that many child interpreters, `chunk` specs each."""
    from .workloads import generate_many
    full = [(seed, 4, npos, npos, 20, 48, 0.5, fs) for seed, npos, fs in specs]
    yield from generate_many("generate_hamming", full, workers=workers, chunk=chunk)


def collect(engine: api.Engine, seeds, make=hamming_instance, log=None, insts=None, **opts):
    """Training records of the given seeds (or of the instances `insts`, one per seed):
    (features [k, 32], labels [k], meta list)."""
    feats, labels, meta = [], [], []
    it = iter(insts) if insts is not None else None
    for s in seeds:
        inst = next(it) if it is not None else make(s)
        res, m, x, y = engine.label_blocks(inst, neg_type=1, **opts)
        for d in m:
            d["seed"] = s
        feats.append(x)
        labels.append(y)
        meta.extend(m)
        if log:
            log(f"seed {s}: cost {res.cost} blocks {len(y)} won {int(y.sum())} {res.seconds * 1e3:.1f} ms")
    X = np.concatenate(feats) if feats else np.zeros((0, NF), np.float32)
    Y = np.concatenate(labels).astype(np.float32) if labels else np.zeros(0, np.float32)
    return X, Y, meta


def train(X, Y, epochs=30, batch=1024, lr=2e-3, pos_weight=None, seed=0, weight_decay=1e-4):
    """Adam on the GPU (api.scorer_train).  pos_weight defaults to negatives / positives."""
    if pos_weight is None:
        npos = max(1.0, float(Y.sum()))
        pos_weight = float(len(Y) - npos) / npos
    p0 = init_params(seed)
    return api.scorer_train(p0, X, Y, epochs=epochs, batch=batch, lr=lr, pos_weight=pos_weight, seed=seed,
                            weight_decay=weight_decay)


def compare(engine: api.Engine, instances, params: np.ndarray, repeats: int = 1, **opts):
    """Plain vs learned order on each instance: cost (must match), time to the find (host
    wall and device), candidates evaluated before the find."""
    engine.set_scorer(params)
    rows = []
    for inst in instances:
        best = {}
        for order in (api.ORDER_PLAIN, api.ORDER_LEARNED):
            rs = [engine.learn(inst, neg_type=1, order=order, **opts) for _ in range(repeats)]
            best[order] = min(rs, key=lambda x: x.seconds)
        p, l = best[api.ORDER_PLAIN], best[api.ORDER_LEARNED]
        rows.append(dict(cost_plain=p.cost, cost_learned=l.cost, status_plain=p.status, status_learned=l.status,
                         ms_plain=p.seconds * 1e3, ms_learned=l.seconds * 1e3,
                         dev_ms_plain=p.device_ms, dev_ms_learned=l.device_ms,
                         evaluated_plain=p.evaluated, evaluated_learned=l.evaluated,
                         formula_plain=p.formula, formula_learned=l.formula))
    return rows


def summarize(rows) -> dict:
    same = all(r["cost_plain"] == r["cost_learned"] and r["status_plain"] == r["status_learned"] for r in rows)
    mean = lambda k: float(np.mean([r[k] for r in rows]))
    mp, ml = mean("ms_plain"), mean("ms_learned")
    dp, dl = mean("dev_ms_plain"), mean("dev_ms_learned")
    return dict(instances=len(rows), same_cost=same, ms_plain=mp, ms_learned=ml, speedup=mp / ml if ml else None,
                device_ms_plain=dp, device_ms_learned=dl, device_speedup=dp / dl if dl else None,
                evaluated_plain=mean("evaluated_plain"), evaluated_learned=mean("evaluated_learned"))


def _seeds(spec: str):
    a, b = spec.split("-")
    return range(int(a), int(b) + 1)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="learned_cli.py")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--per", type=int, default=TRAIN_SPECS["per"], help="instances per (fsize, npos) pair")
    c.add_argument("--workers", type=int, default=16)
    c.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--records", required=True, nargs="+")
    t.add_argument("--out", required=True)
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--seed", type=int, default=0)
    m = sub.add_parser("compare")
    m.add_argument("--scorer", default=DEFAULT_SCORER)
    m.add_argument("--seeds", default=f"{HELD_OUT_SEEDS[0]}-{HELD_OUT_SEEDS[-1]}")
    m.add_argument("--npos", type=int, default=1000)
    m.add_argument("--fsize", type=int, default=9)
    m.add_argument("--repeats", type=int, default=2)
    a = ap.parse_args(argv)
    if a.cmd == "train":
        X = np.concatenate([np.load(r)["X"] for r in a.records])
        Y = np.concatenate([np.load(r)["Y"] for r in a.records])
        p, curve = train(X, Y, epochs=a.epochs, seed=a.seed)
        np.save(a.out, p)
        print(f"{len(Y)} records, {int(Y.sum())} positive; loss {curve[0]:.4f} -> {curve[-1]:.4f}")
        return 0
    with api.Engine(slots_log2=26, cache_bytes=16 << 30) as eng:
        if a.cmd == "collect":
            t0 = time.time()
            specs = training_specs(per=a.per)
            X, Y, meta = collect(eng, [s[0] for s in specs], insts=instances(specs, workers=a.workers, chunk=50))
            np.savez_compressed(a.out, X=X, Y=Y, cost=np.array([d["cost"] for d in meta], np.int32),
                                op=np.array(["~&|XFGU".index(d["op"]) for d in meta], np.int32),
                                seed=np.array([d["seed"] for d in meta], np.int64))
            print(f"{len(Y)} records, {int(Y.sum())} positive, {time.time() - t0:.1f} s")
        else:
            insts = [hamming_instance(s, a.npos, a.npos, a.fsize) for s in _seeds(a.seeds)]
            rows = compare(eng, insts, load_scorer(a.scorer), repeats=a.repeats)
            print(summarize(rows))
    return 0


if __name__ == "__main__":
    sys.exit(main())
