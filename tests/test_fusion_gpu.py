"""Loop-chain fusion on the B200 path: every tuning candidate of the fused
chain kernel (each tile shape, read-only dats from HBM or staged in shared
memory) run on every CloverLeaf 2D chain it fits, against the reference
build's golden fields (bit for bit), dt (exact) and summaries (1e-12).

The autotuner times these candidates against the unfused loops and keeps
the fastest, so a wrong candidate would otherwise only show on the run that
happens to tune it; here each one runs a whole deck."""
import os

import numpy as np
import pytest

from ops_b200 import apps
from ops_b200 import ops as O

from test_clover_gpu import FIELDS, REL_SUM, as_reference_columns, config2_deck

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu
N_CANDIDATES = 10


@pytest.mark.parametrize("cand", range(N_CANDIDATES))
@pytest.mark.parametrize("name,nx,ny,steps,seed", [("clover_64x64_s30", 64, 64, 30, 2),
                                                    ("clover_100x70_s25", 100, 70, 25, 5)])
def test_candidate_matches_golden(gpu_runtime, tmp_path, cand, name, nx, ny, steps, seed):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    O.set_option("tile_candidate", cand)
    try:
        O.reset_counters()
        summ, _ = apps.cloverleaf(config2_deck(nx, ny, steps, seed), dump_dir=str(tmp_path))
        fs = O.fusion_stats()
    finally:
        O.set_option("tile_candidate", -1)
    assert fs["chains"] > 0, "no chain ran fused"
    assert fs["fused_bytes"] < fs["loop_bytes"]
    ours = as_reference_columns(summ)
    np.testing.assert_allclose(ours[:, 1:], g["summaries"][:, 1:], rtol=REL_SUM, atol=0)
    assert np.array_equal(summ[1:steps + 1, 7], g["dts"])
    for f in FIELDS:
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        assert np.array_equal(got, ext), f


def test_candidate_option_is_checked(gpu_runtime):
    with pytest.raises(O.OpsError):
        O.set_option("tile_candidate", N_CANDIDATES)
    with pytest.raises(O.OpsError):
        O.set_option("tile_candidate", -2)
