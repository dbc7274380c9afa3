"""Pins the CPU oracle to the reference (no GPU needed)."""
import glob
import os
import subprocess

import numpy as np
import pytest

import oracle
from ops_b200 import seeded

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_seeded_rng_matches_c(orc):
    ks = np.array([0, 1, 2, 17, 12345, 2**40 + 3], dtype=np.uint64)
    for seed in (0, 1, 5, 2**63 + 11):
        py = seeded.sm64_at(seed, ks)
        c = [orc.oracle_sm64_at(seed, int(k)) for k in ks]
        assert [int(v) for v in py] == c
        assert np.array_equal(seeded.u01(seed, ks), np.array([orc.oracle_sm64_u01(seed, int(k)) for k in ks]))


def _oracle_laplace(orc, field, iters):
    A = np.ascontiguousarray(field.copy())
    errs = np.zeros(max(iters, 1))
    jmax, imax = A.shape[0] - 2, A.shape[1] - 2
    orc.oracle_laplace_run(imax, jmax, iters, A.ctypes.data, errs.ctypes.data)
    return A, errs[:iters]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "laplace_seeded_*.npz"))))
def test_laplace_oracle_matches_reference_golden(orc, path):
    g = np.load(path)
    imax, jmax, iters, seed = int(g["imax"]), int(g["jmax"]), int(g["iters"]), int(g["seed"])
    init = seeded.laplace_field(imax, jmax, seed)
    A, errs = _oracle_laplace(orc, init, iters)
    assert np.array_equal(A, g["field"])          # bit-exact
    assert np.array_equal(errs, g["errors"])


def test_laplace_oracle_step7_known_answer(orc):
    """apps/c/laplace2d_tutorial/step7/laplace2d.cpp:134-138: 4094^2, 100
    iterations, final max|delta| = 2.421354960840227e-03 (the reference
    passes within 0.001 %)."""
    imax = jmax = 4094
    A = np.zeros((jmax + 2, imax + 2))
    orc.oracle_laplace_step7_init(imax, jmax, A.ctypes.data)
    _, errs = _oracle_laplace(orc, A, 100)
    rel = abs(errs[-1] / 2.421354960840227e-03 - 1.0)
    assert rel < 1e-5
    assert rel < 1e-12  # the reference's own build reproduces it to 6.9e-14


def test_laplace_oracle_matches_reference_binary(orc, tmp_path):
    exe = oracle.reference_binary("laplace2d_seeded")
    if exe is None:
        pytest.skip("reference build (oracle/_ref) not present")
    imax, jmax, iters, seed = 203, 77, 40, 9
    dump = str(tmp_path / "A.bin")
    r = subprocess.run([exe, str(imax), str(jmax), str(iters), str(seed), dump], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120, check=True,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    ref_errs = np.array([float(l.split()[3]) for l in r.stdout.splitlines() if l.startswith("iter ")])
    ref = np.fromfile(dump).reshape(jmax + 2, imax + 2)
    A, errs = _oracle_laplace(orc, seeded.laplace_field(imax, jmax, seed), iters)
    assert np.array_equal(A, ref)
    assert np.array_equal(errs, ref_errs)
