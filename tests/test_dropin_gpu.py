"""Reference applications, unmodified, running on OPS-B200 through the drop-in
API: their sources translated by the legacy translator with the sm100a
target and linked against ops_b200/dropin/ops_dropin.cu and libops_b200.so
(built by ops_b200/dropin/build_apps.py from the reference tree).

* apps/c/laplace2d_tutorial/step7: the app's own known-answer check
  (laplace2d.cpp:134-139, final error within 0.001 % of 2.421354960840227e-03).
  Its boundary values come from sin/exp, which the device's math library and
  the host's may round differently, so this one is not held to bit equality.
* apps/c/CloverLeaf: the 64x64, 30-step deck of the golden fixture made by
  the reference's own OpenMP build (tests/golden/clover_64x64_s30.npz): dt of
  every step exactly, the field summaries to 1e-12 relative, and every dumped
  field bit for bit.
* apps/c/CloverLeaf_3D and apps/c/TeaLeaf (Jacobi, CG and PPCG decks): the
  same bars against their goldens (below).
"""
import os
import subprocess

import numpy as np
import pytest

from ops_b200.dropin import build_apps

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
          "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y"]
pytestmark = pytest.mark.gpu


def _binary(name):
    exe = build_apps.binary(name)
    if exe is None:
        pytest.fail(f"drop-in app {name} was not built (ops_b200/dropin/build_apps.py needs the reference tree)")
    return exe


def test_laplace_step7_known_answer(tmp_path):
    r = subprocess.run([_binary("laplace2d_step7")], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "This run is considered PASSED" in r.stdout, r.stdout[-2000:]


def test_cloverleaf_matches_reference_golden(tmp_path):
    g = np.load(os.path.join(GOLDEN, "clover_64x64_s30.npz"))
    (tmp_path / "clover.in").write_text(str(g["deck"]))
    env = dict(os.environ, OPS_B200_PRINT_FULL="1", OPS_B200_DUMP_DIR=str(tmp_path))
    r = subprocess.run([_binary("cloverleaf")], cwd=tmp_path, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = (tmp_path / "clover.out").read_text()
    summ = np.array([[float(x) for x in l.split()[1:9]] for l in out.splitlines() if l.strip().startswith("step:")])
    dts = np.array([float(l.split()[7]) for l in r.stdout.splitlines() if l.strip().startswith("Step ")])
    ref = g["summaries"]
    assert summ.shape == ref.shape
    assert np.array_equal(summ[:, 0], ref[:, 0])
    np.testing.assert_allclose(summ[:, 1:], ref[:, 1:], rtol=1e-12, atol=0)
    assert np.array_equal(dts, g["dts"])
    for f in FIELDS:
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        assert np.array_equal(got, ext), f


def _run_app(name, tmp_path, deck_file, deck_text):
    (tmp_path / deck_file).write_text(deck_text)
    env = dict(os.environ, OPS_B200_PRINT_FULL="1", OPS_B200_DUMP_DIR=str(tmp_path))
    r = subprocess.run([_binary(name)], cwd=tmp_path, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.parametrize("case", ["tea_kat_jacobi", "tea_cg_jacdiag_64", "tea_ppcg_jacdiag_64"])
def test_tealeaf_matches_reference_golden(tmp_path, case):
    """apps/c/TeaLeaf unmodified: solver iteration counts exactly, field
    summaries to 1e-12; the Jacobi deck's fields bit for bit (its sums are
    per cell; CG and PPCG take dot products in another order)."""
    g = np.load(os.path.join(GOLDEN, case + ".npz"))
    stdout = _run_app("tealeaf", tmp_path, "tea.in", str(g["deck"]))
    out = (tmp_path / "tea.out").read_text()
    summ = np.array([[float(x) for x in l.split()[1:7]] for l in out.splitlines() if l.strip().startswith("step:")])
    iters = np.array([int(l.split()[-1]) for l in stdout.splitlines() if l.strip().startswith("Iteration count")])
    assert np.array_equal(iters, g["iters"])
    np.testing.assert_allclose(summ, g["summaries"], rtol=1e-12, atol=0)
    if case == "tea_kat_jacobi":
        for f in ("u", "energy1", "density"):
            ext = g["f_" + f]
            got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
            assert np.array_equal(got, ext), f


def test_cloverleaf3d_matches_reference_golden(tmp_path):
    """apps/c/CloverLeaf_3D unmodified (3D accessors, edge dats in all three
    directions): dt of every step exactly, summaries to 1e-12, the dumped
    fields bit for bit."""
    g = np.load(os.path.join(GOLDEN, "clover3d_24x20x16_s40.npz"))
    stdout = _run_app("cloverleaf3d", tmp_path, "clover.in", str(g["deck"]))
    out = (tmp_path / "clover.out").read_text()
    summ = np.array([[float(x) for x in l.split()[1:9]] for l in out.splitlines() if l.strip().startswith("step:")])
    dts = np.array([float(l.split()[7]) for l in stdout.splitlines() if l.strip().startswith("Step ")])
    assert summ.shape == g["summaries"].shape
    np.testing.assert_allclose(summ, g["summaries"], rtol=1e-12, atol=0)
    assert np.array_equal(dts, g["dts"])
    for f in ("density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0"):
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        assert np.array_equal(got, ext), f
