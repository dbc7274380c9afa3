"""The halo-transfer oracle (oracle/halo.py) against the reference library's
own ops_halo_transfer (golden dumps from oracle/ref_drivers/halo_cases.cpp,
tests/golden/halo_cases.npz): bit for bit, including the flipped, swapped and
double -> float cases."""
import os

import numpy as np

from halo_cases import CASES, DM, initial, refill
from oracle import halo as ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "halo_cases.npz")


def test_oracle_matches_reference():
    g = np.load(GOLDEN)
    arrays = initial()
    meta = {k: ([0, 0], [DM, DM]) for k in arrays}
    for c, halos in enumerate(CASES):
        refill(arrays)
        ref.transfer(arrays, meta, halos)
        for name in ("a", "b", "bf"):
            assert np.array_equal(arrays[name], g[f"case{c}_{name}"]), (c, name)
