"""Regenerates the golden fixtures in tests/golden from the reference itself.

Runs the reference's OpenMP apps built by oracle/build_ref.sh (oracle/_ref/bin,
this container only: it needs the reference tree to build) and stores their
outputs as small .npz files that travel with the tests. The fixtures pin the
oracle (oracle/src) and the B200 path to the reference's own results.

    python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

# (imax, jmax, iters, seed). The reference app itself fails on degenerate
# grids (1x1 segfaults, 2x1 does not terminate), so those edge cases are
# checked against the oracle only.
LAPLACE_CASES = [
    (37, 23, 25, 11),
    (64, 64, 50, 1),
    (130, 7, 9, 5),
]


def laplace():
    exe = oracle.reference_binary("laplace2d_seeded")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/laplace2d_seeded missing: run oracle/build_ref.sh")
    for imax, jmax, iters, seed in LAPLACE_CASES:
        with tempfile.TemporaryDirectory() as td:
            dump = os.path.join(td, "A.bin")
            r = subprocess.run([exe, str(imax), str(jmax), str(iters), str(seed), dump], cwd=td,
                               capture_output=True, text=True, check=True, timeout=120,
                               env=dict(os.environ, OMP_NUM_THREADS="1"))
            errs = [float(l.split()[3]) for l in r.stdout.splitlines() if l.startswith("iter ")]
            field = np.fromfile(dump, dtype=np.float64).reshape(jmax + 2, imax + 2)
        name = os.path.join(HERE, f"laplace_seeded_{imax}x{jmax}_it{iters}_s{seed}.npz")
        np.savez_compressed(name, field=field, errors=np.array(errs), imax=imax, jmax=jmax, iters=iters,
                            seed=seed)
        print("wrote", name)


if __name__ == "__main__":
    laplace()
