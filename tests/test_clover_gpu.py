"""CloverLeaf 2D hydro on the B200 path vs the reference's own OpenMP build
(golden fixtures made by tests/golden/make_golden.py from oracle/_ref).

Per-cell fields are compared bit for bit (same operation order, no FMA
contraction); dt per step is a min-reduction and must match exactly; the
field-summary sums (volume, mass, energies, pressure) are FP64 sums whose
order differs from the reference's OpenMP order, so they are held to the
north-star bound of 1e-12 relative."""
import glob
import os

import numpy as np
import pytest

from ops_b200 import apps, seeded

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
          "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y"]
REL_SUM = 1e-12
pytestmark = pytest.mark.gpu


def config2_deck(nx, ny, steps, seed, freq=1):
    return apps.clover_deck(x_cells=nx, y_cells=ny, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0,
                            initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=steps,
                            summary_frequency=freq, states=seeded.clover_config2_states(nx, ny, seed))


def as_reference_columns(s):
    """Our rows (step, time, vol, mass, ie, ke, press, dt) in the reference's
    printed form (step, vol, mass, density, pressure, ie, ke, total)."""
    return np.stack([s[:, 0], s[:, 2], s[:, 3], s[:, 3] / s[:, 2], s[:, 6] / s[:, 2], s[:, 4], s[:, 5],
                     s[:, 4] + s[:, 5]], axis=1)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "clover_*.npz"))))
def test_matches_reference_golden(gpu_runtime, path, tmp_path):
    g = np.load(path)
    name = os.path.basename(path)[:-4]
    (nx, ny), steps, seed = {"clover_64x64_s30": ((64, 64), 30, 2), "clover_100x70_s25": ((100, 70), 25, 5)}[name]
    deck = config2_deck(nx, ny, steps, seed)
    assert apps.clover_deck_text(deck) == str(g["deck"])
    summ, _ = apps.cloverleaf(deck, dump_dir=str(tmp_path))
    ref = g["summaries"]
    ours = as_reference_columns(summ)
    assert ours.shape == ref.shape
    assert np.array_equal(ours[:, 0], ref[:, 0])
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=REL_SUM, atol=0)
    # dt of every step: exact
    assert np.array_equal(summ[1:steps + 1, 7], g["dts"])
    for f in FIELDS:
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        assert np.array_equal(got, ext), f


def test_bm_short_known_answer(gpu_runtime):
    """apps/c/CloverLeaf/clover_bm_short.in (960^2, 87 steps): final kinetic
    energy 1.19316898756307 within the reference's 0.001 % (field_summary.cpp:91-99)."""
    deck = apps.clover_deck(x_cells=960, y_cells=960, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0,
                            initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=87,
                            summary_frequency=10,
                            states=[dict(density=0.2, energy=1.0),
                                    dict(density=1.0, energy=2.5, geometry="rectangle", xmin=0.0, xmax=5.0,
                                         ymin=0.0, ymax=2.0)])
    summ, _ = apps.cloverleaf(deck)
    ke = summ[-1, 5]
    assert abs(100.0 * (ke / 1.19316898756307) - 100.0) < 0.001


def test_summary_invariants_and_determinism(gpu_runtime):
    """The mesh volume is invariant; two runs agree bit for bit (reductions
    finish in a fixed order)."""
    deck = config2_deck(200, 150, 15, 9)
    a, _ = apps.cloverleaf(deck)
    b, _ = apps.cloverleaf(deck)
    assert np.array_equal(a, b)
    np.testing.assert_allclose(a[:, 2], a[0, 2], rtol=1e-13)   # volume
