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
