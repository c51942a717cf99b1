"""The reference's divide-and-conquer entry (code/dc.py:368-387, runDC) on this library:

    python ltl-learning-on-gpus_b200/dc_cli.py input.trace [--algo rand|det] [--window 64]
        [--costs 1,1,1,1,1,1,1,1] [--max-cost 500] [--rlx 3] [--neg 2] [--timeout 2000] [--reference-keys]

prints the reference's three lines: "Size(P, N): (p, n)", "Time: t s", "LTL: formula".
Sub-problems are learned in process by one engine (the reference runs its enumerator binary
once per sub-problem) and formulas are checked on the device.  Uniqueness is exact, as this
library's ltli6463 is by default; --reference-keys selects the reference's relaxed keys of
type --rlx.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from __graft_entry__ import load_package  # noqa: E402

load_package()
from ltlb200 import api, divide  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser(prog="dc_cli.py")
    ap.add_argument("trace")
    ap.add_argument("--algo", choices=["rand", "det"], default="rand")
    ap.add_argument("--window", type=int, default=64)
    ap.add_argument("--costs", default="1,1,1,1,1,1,1,1")
    ap.add_argument("--max-cost", type=int, default=500)
    ap.add_argument("--rlx", type=int, default=3, help="the reference's RlxUnqChkTyp")
    ap.add_argument("--neg", type=int, default=2, help="the reference's NegType")
    ap.add_argument("--timeout", type=float, default=2000.0)
    ap.add_argument("--reference-keys", action="store_true",
                    help="the reference's relaxed keys of type --rlx instead of exact uniqueness")
    ap.add_argument("--exact", action="store_true", help="exact uniqueness (the default)")
    a = ap.parse_args(argv)
    inst = api.read_scarlet(a.trace)
    out = divide.run_dc(inst, algo=a.algo, window=a.window, timeout_s=a.timeout,
                        costs=tuple(int(c) for c in a.costs.split(",")), max_cost=a.max_cost, rlx_type=a.rlx,
                        neg_type=a.neg, key_mode=api.KEY_REF if a.reference_keys else api.KEY_EXACT)
    print(f"Size(P, N): ({inst.num_pos}, {inst.num_neg})")
    print(f"Time: {round(out['seconds'], 3)}s")
    print(f"LTL: {out['formula']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
