"""TeaLeaf 2D implicit heat conduction on the B200 path vs the reference's own
OpenMP build (golden fixtures made by tests/golden/make_golden.py from
oracle/_ref, `python tests/golden/make_golden.py tea`).

Jacobi: every per-cell operation matches the reference's order, so u, energy1
and density are compared bit for bit and the iteration counts exactly. CG:
alpha and beta come from FP64 dot products whose summation order differs from
the reference's, so u carries rounding differences of a few ulps per
iteration; the iteration counts must still match exactly, the fields hold to
1e-10 of their maximum and the field summaries to 1e-12 relative. Chebyshev
and PPCG: the same bars, plus the iteration at which the polynomial phase
took over, Chebyshev's iteration estimate and the PPCG inner-iteration count
exactly, and the eigenvalue bounds (from the CG coefficients through the QL
eigenvalue solve) to 1e-10 relative."""
import glob
import os

import numpy as np
import pytest

from ops_b200 import apps, seeded

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REL_SUM = 1e-12
REL_FIELD_CG = 1e-10
pytestmark = pytest.mark.gpu

TEA_IN = [dict(density=100.0, energy=0.0001),
          dict(density=0.1, energy=25.0, geometry="rectangle", xmin=0.0, xmax=1.0, ymin=1.0, ymax=2.0),
          dict(density=0.1, energy=0.1, geometry="rectangle", xmin=1.0, xmax=6.0, ymin=1.0, ymax=2.0),
          dict(density=0.1, energy=0.1, geometry="rectangle", xmin=5.0, xmax=6.0, ymin=1.0, ymax=8.0),
          dict(density=0.1, energy=0.1, geometry="rectangle", xmin=5.0, xmax=10.0, ymin=7.0, ymax=8.0)]

CASES = {
    "tea_kat_jacobi": dict(x_cells=10, y_cells=10, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=10,
                           max_iters=1000, eps=1e-15, solver=0, summary_frequency=10, states=TEA_IN),
    "tea_cg_jacdiag_64": dict(x_cells=64, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=2,
                              max_iters=5000, eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
                              states=seeded.tea_config4_states(64, 64, 4)),
    "tea_cg_plain_100x70": dict(x_cells=100, y_cells=70, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=1,
                                max_iters=5000, eps=1e-10, solver=1, preconditioner=0, summary_frequency=1,
                                states=seeded.tea_config4_states(100, 70, 7)),
    "tea_cheby_plain_96": dict(x_cells=96, y_cells=96, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=3,
                               max_iters=5000, eps=1e-10, solver=2, preconditioner=0, summary_frequency=1,
                               states=seeded.tea_config4_states(96, 96, 4)),
    "tea_cheby_jacdiag_80x64": dict(x_cells=80, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.04,
                                    end_step=2, max_iters=5000, eps=1e-10, solver=2, preconditioner=1,
                                    summary_frequency=1, states=seeded.tea_config4_states(80, 64, 11)),
    "tea_ppcg_plain_96": dict(x_cells=96, y_cells=96, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=3,
                              max_iters=5000, eps=1e-10, solver=3, preconditioner=0, summary_frequency=1,
                              states=seeded.tea_config4_states(96, 96, 4)),
    "tea_ppcg_jacdiag_64": dict(x_cells=64, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=2,
                                max_iters=5000, eps=1e-10, solver=3, preconditioner=1, summary_frequency=1,
                                ch_cg_presteps=10, ch_cg_epslim=0.5, ppcg_inner_steps=12,
                                states=seeded.tea_config4_states(64, 64, 5)),
}
REL_EIG = 1e-10
COL = {k: i for i, k in enumerate(apps.TEA_SOLVE_COLS)}


def as_reference_columns(s):
    """Our rows (step, time, vol, mass, ie, temp) in the reference's printed
    form (step, vol, mass, density, ie, temp)."""
    return np.stack([s[:, 0], s[:, 2], s[:, 3], s[:, 3] / s[:, 2], s[:, 4], s[:, 5]], axis=1)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "tea_*.npz"))))
def test_matches_reference_golden(gpu_runtime, path, tmp_path):
    g = np.load(path)
    name = os.path.basename(path)[:-4]
    kw = CASES[name]
    deck = apps.tea_deck(**kw)
    assert apps.tea_deck_text(deck) == str(g["deck"])
    summ, solves, _ = apps.tealeaf(deck, dump_dir=str(tmp_path))
    assert np.array_equal(solves[:, 0].astype(np.int64), g["iters"])
    if kw["solver"] in (2, 3):
        switched = solves[:, COL["switch_iteration"]] > 0
        assert np.array_equal(solves[switched, COL["switch_iteration"]].astype(np.int64), g["poly_switch"])
        eig = solves[switched][:, [COL["eigmin"], COL["eigmax"]]]
        np.testing.assert_allclose(eig, g["poly_eig"], rtol=REL_EIG, atol=0)
        if kw["solver"] == 2:
            assert np.array_equal(solves[switched, COL["est_itc"]].astype(np.int64), g["poly_est_itc"])
        else:
            assert np.array_equal(solves[:, COL["ppcg_inner_iterations"]].astype(np.int64), g["poly_ppcg"])
    ours = as_reference_columns(summ)
    ref = g["summaries"]
    assert ours.shape == ref.shape
    assert np.array_equal(ours[:, 0], ref[:, 0])
    # the golden build prints the summaries with 17 significant digits (oracle/ref_drivers/fullprec_hook.h)
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=REL_SUM, atol=0)
    jacobi = kw["solver"] == 0
    for f in ("density", "energy1", "u"):
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        if jacobi or f == "density":
            assert np.array_equal(got, ext), f
        else:
            np.testing.assert_allclose(got, ext, rtol=0, atol=REL_FIELD_CG * np.abs(ext).max(), err_msg=f)


def test_tea_in_known_answer(gpu_runtime):
    """apps/c/TeaLeaf/tea.in (10x10, 10 steps, Jacobi): the reference checks
    the final temperature against 157.55084183279294 within 0.001 %
    (apps/c/TeaLeaf/field_summary.cpp:84-97)."""
    deck = apps.tea_deck(**CASES["tea_kat_jacobi"])
    summ, _, _ = apps.tealeaf(deck)
    temp = summ[-1, 5]
    assert abs(100.0 * (temp / 157.55084183279294) - 100.0) < 0.001


def test_cg_determinism_and_invariants(gpu_runtime):
    """Two runs agree bit for bit (reductions finish in a fixed order); the
    mesh volume and the mass are invariant over the steps."""
    deck = apps.tea_deck(x_cells=150, y_cells=90, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=3,
                         max_iters=5000, eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
                         states=seeded.tea_config4_states(150, 90, 11))
    a, sa, _ = apps.tealeaf(deck)
    b, sb, _ = apps.tealeaf(deck)
    assert np.array_equal(a, b) and np.array_equal(sa[:, :6], sb[:, :6])   # column 6 is the solve's time
    np.testing.assert_allclose(a[:, 2], a[0, 2], rtol=1e-13)
    np.testing.assert_allclose(a[:, 3], a[0, 3], rtol=1e-13)
    assert (sa[:, 2] < 1e-10).all()


@pytest.mark.parametrize("name", ["tea_cg_jacdiag_64", "tea_cg_plain_100x70"])
def test_fused_solver_matches_reference_golden(gpu_runtime, name, tmp_path):
    """The device-resident CG (alpha, beta and the stop test on the GPU) keeps
    the reference's per-cell arithmetic and stopping rule: iteration counts
    exact, summaries to 1e-12, fields to the CG tolerance."""
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    deck = apps.tea_deck(fused=1, **CASES[name])
    summ, solves, _ = apps.tealeaf(deck, dump_dir=str(tmp_path))
    assert np.array_equal(solves[:, 0].astype(np.int64), g["iters"])
    np.testing.assert_allclose(as_reference_columns(summ)[:, 1:], g["summaries"][:, 1:], rtol=REL_SUM, atol=0)
    for f in ("energy1", "u"):
        ext = g["f_" + f]
        got = np.fromfile(str(tmp_path / (f + ".bin"))).reshape(ext.shape)
        np.testing.assert_allclose(got, ext, rtol=0, atol=REL_FIELD_CG * np.abs(ext).max(), err_msg=f)
    assert (solves[:, 2] < 1e-10).all()        # the stopping quantity
    assert (solves[:, 4] > 0).all() and (solves[:, 4] < 1e-8).all()   # true FP64 residual ratio


def test_fused_matches_loop_chain(gpu_runtime, tmp_path):
    """Fused and loop-by-loop CG on a 300x200 seeded problem: same iteration
    counts, solutions equal to rounding."""
    kw = dict(x_cells=300, y_cells=200, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=2, max_iters=5000,
              eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
              states=seeded.tea_config4_states(300, 200, 13))
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    a, sa, _ = apps.tealeaf(apps.tea_deck(**kw), dump_dir=str(tmp_path / "a"))
    b, sb, _ = apps.tealeaf(apps.tea_deck(fused=1, **kw), dump_dir=str(tmp_path / "b"))
    assert np.array_equal(sa[:, 0], sb[:, 0])
    np.testing.assert_allclose(a[:, 2:], b[:, 2:], rtol=REL_SUM, atol=0)
    ua = np.fromfile(str(tmp_path / "a" / "u.bin"))
    ub = np.fromfile(str(tmp_path / "b" / "u.bin"))
    np.testing.assert_allclose(ub, ua, rtol=0, atol=REL_FIELD_CG * np.abs(ua).max())


def test_true_residual_stop(gpu_runtime):
    """true_residual_stop: the FP64 solve runs until ||u0 - A u|| < 1e-10 ||r0||,
    which takes at least as many iterations as TeaLeaf's sqrt|r.z| test."""
    kw = dict(x_cells=256, y_cells=192, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=1, max_iters=20000,
              eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
              states=seeded.tea_config4_states(256, 192, 21))
    _, sa, _ = apps.tealeaf(apps.tea_deck(fused=1, **kw))
    _, sb, _ = apps.tealeaf(apps.tea_deck(fused=1, true_residual_stop=1, **kw))
    assert sb[0, 0] >= sa[0, 0]
    assert sb[0, 4] < 1.5e-10          # recomputed FP64 residual; the recursive one met 1e-10


@pytest.mark.parametrize("precond", [1, 0])
def test_mixed_precision_reaches_fp64_residual(gpu_runtime, precond, tmp_path):
    """FP32 PCG under FP64 reliable updates: the FP64 residual ||u0 - A u|| /
    ||r0|| ends below 1e-10 and the solution agrees with the FP64 solve to the
    accuracy that residual implies."""
    kw = dict(x_cells=256, y_cells=192, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=1, max_iters=20000,
              eps=1e-10, solver=1, preconditioner=precond, summary_frequency=1,
              states=seeded.tea_config4_states(256, 192, 21))
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    a, sa, _ = apps.tealeaf(apps.tea_deck(fused=1, **kw), dump_dir=str(tmp_path / "a"))
    b, sb, _ = apps.tealeaf(apps.tea_deck(fused=1, mixed=1, reliable_delta=0.1, **kw), dump_dir=str(tmp_path / "b"))
    assert sb[0, 4] < 1e-10 and sb[0, 2] < 1e-10
    assert sb[0, 5] >= 5                       # reliable updates: one per decade at least
    assert sb[0, 0] < 2.0 * sa[0, 0]           # the search direction survives the updates
    ua = np.fromfile(str(tmp_path / "a" / "u.bin"))
    ub = np.fromfile(str(tmp_path / "b" / "u.bin"))
    assert np.linalg.norm(ub - ua) / np.linalg.norm(ua) < 1e-8
    np.testing.assert_allclose(b[:, 2:4], a[:, 2:4], rtol=1e-12, atol=0)   # volume and mass: untouched by the solve
