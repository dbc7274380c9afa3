"""CloverLeaf 3D hydro on the B200 path vs the reference's own OpenMP build
(golden fixtures made by `python tests/golden/make_golden.py clover3d` from
oracle/_ref/bin/cloverleaf3d).

As for 2D: per-cell fields bit for bit, dt of every step exactly, the field
summary sums (whose summation order differs from the reference's) to 1e-12
relative. The reference's own known answer (clover_bm_short.in, 96^3,
87 steps, field_summary.cpp:90-106) is checked at its 0.001 % bound."""
import glob
import os

import numpy as np
import pytest

from ops_b200 import apps, seeded

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ["density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0"]
REL_SUM = 1e-12
pytestmark = pytest.mark.gpu

CASES = {"clover3d_24x20x16_s40": (24, 20, 16, 40, 6, 0.04), "clover3d_18x14x22_s30": (18, 14, 22, 30, 9, 1.0)}


def deck3d(nx, ny, nz, steps, seed, max_dt, freq=1):
    return apps.clover3d_deck(x_cells=nx, y_cells=ny, z_cells=nz, xmax=10.0, ymax=10.0, zmax=10.0,
                              initial_timestep=0.04, timestep_rise=1.5, max_timestep=max_dt, end_step=steps,
                              summary_frequency=freq, states=seeded.clover3d_states(nx, ny, nz, seed))


def as_reference_columns(s):
    """Our rows (step, time, vol, mass, ie, ke, press, dt) in the reference's
    printed form (step, vol, mass, density, pressure, ie, ke, total)."""
    return np.stack([s[:, 0], s[:, 2], s[:, 3], s[:, 3] / s[:, 2], s[:, 6] / s[:, 2], s[:, 4], s[:, 5],
                     s[:, 4] + s[:, 5]], axis=1)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "clover3d_*.npz"))))
def test_matches_reference_golden(gpu_runtime, path, tmp_path):
    g = np.load(path)
    nx, ny, nz, steps, seed, max_dt = CASES[os.path.basename(path)[:-4]]
    deck = deck3d(nx, ny, nz, steps, seed, max_dt)
    assert apps.clover3d_deck_text(deck) == str(g["deck"])
    summ, _ = apps.cloverleaf3d(deck, dump_dir=str(tmp_path))
    ref = g["summaries"]
    ours = as_reference_columns(summ)
    assert ours.shape == ref.shape
    assert np.array_equal(ours[:, 0], ref[:, 0])
    assert np.array_equal(summ[1:steps + 1, 7], g["dts"])
    for f in FIELDS:
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        assert np.array_equal(got, ext), f
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=REL_SUM, atol=0)


def test_bm_short_known_answer(gpu_runtime):
    """apps/c/CloverLeaf_3D/clover_bm_short.in (96^3, 87 steps): final kinetic
    energy 20.0546870878964 within the reference's 0.001 %."""
    deck = apps.clover3d_deck(x_cells=96, y_cells=96, z_cells=96, xmax=10.0, ymax=10.0, zmax=10.0,
                              initial_timestep=0.1, max_timestep=0.1, end_step=87, end_time=1000.1,
                              summary_frequency=10,
                              states=[dict(density=0.2, energy=1.0),
                                      dict(density=1.0, energy=2.5, geometry="cuboid", xmin=0.0, xmax=5.0,
                                           ymin=0.0, ymax=2.0, zmin=0.0, zmax=4.0)])
    summ, _ = apps.cloverleaf3d(deck)
    ke = summ[-1, 5]
    assert abs(100.0 * (ke / 20.0546870878964) - 100.0) < 0.001


def test_determinism_and_volume(gpu_runtime):
    """Two runs agree bit for bit; the mesh volume is invariant."""
    deck = deck3d(40, 36, 30, 12, 3, 1.0)
    a, _ = apps.cloverleaf3d(deck)
    b, _ = apps.cloverleaf3d(deck)
    assert np.array_equal(a, b)
    np.testing.assert_allclose(a[:, 2], a[0, 2], rtol=1e-13)
