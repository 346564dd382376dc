"""Writes tests/golden/*.npz from the oracle (run from the repo root:
``python tests/golden/make_golden.py``). The files pin the oracle's current
output so a change to the restatement shows up as a test diff."""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import gen, oracle_lib  # noqa: E402

orc = oracle_lib.load()
here = os.path.dirname(os.path.abspath(__file__))
p = gen.bvh_prims(257, 0.0)
nodes, order, depth = orc.build(p, 4)
np.savez_compressed(os.path.join(here, "bvh_257.npz"), prims=p, nodes=nodes, order=order, depth=np.uint32(depth))
print("wrote bvh_257.npz")
