"""The headline configurations at their full stated sizes against the
reference's own OpenMP build (fixtures made by
`python tests/golden/make_golden.py fullsize` from oracle/_ref).

* Laplace 4096^2, 1000 iterations (config 1): every iteration's max|delta|
  exactly, and the final field bit for bit (SHA-256 of the full extent).
* CloverLeaf 2D 3840^2, 200 steps (config 2, the bench deck): dt of every
  step exactly, the five field-summary sums of every step to 1e-12 relative
  (FP64 sums in another order), and every dumped field bit for bit
  (SHA-256), with the loop-chain fuser on (the default) -- the path the
  bench times.
* TeaLeaf 4096^2 Jacobi-PCG (config 4, the reference's loop-chain solver):
  the iteration count exactly, the temperature summary to 1e-12 relative.
"""
import hashlib
import os

import numpy as np
import pytest

from ops_b200 import apps, seeded

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REL_SUM = 1e-12
pytestmark = pytest.mark.gpu


def _load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"fixture {path} missing: run tests/golden/make_golden.py fullsize")
    return np.load(path)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_laplace_4096_1000_iterations(gpu_runtime):
    g = _load("fullsize_laplace_4096_it1000")
    n, iters, seed = int(g["imax"]), int(g["iters"]), int(g["seed"])
    A, errs, _ = apps.laplace2d(seeded.laplace_field(n, n, seed), iters)
    assert errs.shape == g["errors"].shape
    assert np.array_equal(errs, g["errors"])
    assert _sha(A) == str(g["field_sha256"])


def test_cloverleaf_3840_200_steps(gpu_runtime, tmp_path):
    g = _load("fullsize_clover_3840_s200")
    n, steps = 3840, 200
    deck = apps.clover_deck(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.04,
                            timestep_rise=1.5, max_timestep=0.04, end_step=steps, summary_frequency=1,
                            states=seeded.clover_config2_states(n, n, 2))
    assert apps.clover_deck_text(deck) == str(g["deck"])
    summ, _ = apps.cloverleaf(deck, dump_dir=str(tmp_path))
    ref = g["summaries"]
    ours = np.stack([summ[:, 0], summ[:, 2], summ[:, 3], summ[:, 3] / summ[:, 2], summ[:, 6] / summ[:, 2],
                     summ[:, 4], summ[:, 5], summ[:, 4] + summ[:, 5]], axis=1)
    assert ours.shape == ref.shape
    assert np.array_equal(ours[:, 0], ref[:, 0])
    assert np.array_equal(summ[1:steps + 1, 7], g["dts"])
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=REL_SUM, atol=0)
    for name, digest, shape in zip(g["field_names"], g["field_sha256"], g["field_shapes"]):
        got = np.fromfile(str(tmp_path / (str(name) + ".bin"))).reshape(tuple(shape))
        assert _sha(got) == str(digest), str(name)


def test_tealeaf_4096_pcg(gpu_runtime):
    g = _load("fullsize_tea_4096_pcg")
    n = 4096
    deck = apps.tea_deck(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.004,
                         end_step=1, summary_frequency=1, max_iters=200000, eps=1e-10, solver=1, preconditioner=1,
                         states=seeded.tea_config4_states(n, n, 4))
    assert apps.tea_deck_text(deck) == str(g["deck"])
    summ, solves, _ = apps.tealeaf(deck)
    assert np.array_equal(solves[:, 0].astype(np.int64), g["iters"])
    ref = g["summaries"]
    ours = np.stack([summ[:, 0], summ[:, 2], summ[:, 3], summ[:, 3] / summ[:, 2], summ[:, 4], summ[:, 5]], axis=1)
    assert ours.shape == ref.shape
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=REL_SUM, atol=0)
