"""Shared helpers for the tests (fixtures on disk, oracle comparisons)."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def fixture_path(name):
    return os.path.join(GOLDEN, "inputs", name)


def load_fixture(name):
    from ltlb200 import gen
    with open(fixture_path(name)) as f:
        return gen.from_scarlet_text(f.read())


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)["runs"]


def reference_runs():
    p = os.path.join(GOLDEN, "reference_runs.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def row_set(rows: np.ndarray) -> set:
    return {r.tobytes() for r in np.ascontiguousarray(rows, dtype=np.uint64)}


def lensum(inst):
    return int(np.asarray(inst.lengths).sum())


def last_round_gap(costs):
    """Levels the reference runs on the fly after the one that overflowed: the first cost
    difference that matches an operator's reach (ltli6463.cu:1202-1206)."""
    c1, c2, c3, c4, c5, c6, c7, c8 = costs
    return min(c2, c1 + c3, c1 + c4, c5, c6, c7, c1 + c8)


def on_the_fly_cases(inst, costs, max_cost=14):
    """(k, cache rows) for caches that hold exactly the rows through level k while level k + 1
    has new CSs: the overflow then stores nothing of level k + 1, so the regime that follows
    is deterministic.  The cache holds at least one row beyond the letters."""
    import oracle as O

    ex = O.learn(inst, costs=costs, neg_type=1, max_cost=max_cost)
    assert ex.status == O.FOUND
    return ex, [(k, ex.level_start[k + 1]) for k in range(costs[0] + 1, ex.cost - 1)
                if ex.level_start[k + 2] > ex.level_start[k + 1] > len(inst.alphabet)]



def edge_instance(pos_steps, neg_steps, alphabet="pq"):
    """An instance from explicit step masks (lists of lists of ints), empty traces allowed."""
    from ltlb200 import gen
    traces = list(pos_steps) + list(neg_steps)
    offs = np.zeros(len(traces) + 1, dtype=np.int32)
    for i, t in enumerate(traces):
        offs[i + 1] = offs[i] + len(t)
    steps = np.array([m for t in traces for m in t], dtype=np.uint32)
    return gen.Instance(len(pos_steps), len(neg_steps), alphabet, steps, offs)


P_BIT, Q_BIT = 1 << (ord("p") - 97), 1 << (ord("q") - 97)


def edge_cases():
    """Inputs at the domain's edges: an empty side, a trace of no steps, one-step traces, a
    trace of the maximum 63 steps, duplicate traces, and one trace on both sides."""
    P, Q = P_BIT, Q_BIT
    return {
        "no_negatives": edge_instance([[P, Q], [P | Q]], []),
        "no_positives": edge_instance([], [[P], [Q, 0, P]]),
        "empty_trace": edge_instance([[P, 0, Q]], [[], [Q]]),
        "one_step_traces": edge_instance([[P], [P | Q]], [[Q], [0]]),
        "max_length_trace": edge_instance([[P if k % 3 else Q for k in range(63)]], [[Q] * 63, [P] * 5]),
        "duplicate_traces": edge_instance([[P, Q], [P, Q]], [[Q, P], [Q, P]]),
        "contradiction": edge_instance([[P, Q]], [[P, Q]]),
    }
