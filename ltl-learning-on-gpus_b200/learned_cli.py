"""Command line of the learned block order (records, training, comparison):

    python ltl-learning-on-gpus_b200/learned_cli.py collect --out records.npz
    python ltl-learning-on-gpus_b200/learned_cli.py train --records records.npz --out scorer.npy
    python ltl-learning-on-gpus_b200/learned_cli.py compare --scorer scorer.npy
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from __graft_entry__ import load_package  # noqa: E402

load_package()
from ltlb200 import learned  # noqa: E402

if __name__ == "__main__":
    sys.exit(learned.main())
