"""The halo-transfer cases of oracle/ref_drivers/halo_cases.cpp (shared by the
CPU oracle test and the GPU parity test): two 20 x 20 blocks with a depth-2
ring, dats a, b (double) and bf (float). Before each case the interiors are
refilled with tag + 100 x + y + 0.25 (0.5 for bf); the rings keep what the
earlier cases wrote, as in the driver."""
import numpy as np

SIZE, DM, DP = 20, -2, 2
# per case: halos as (src, dst, iter, from_base, to_base, from_dir, to_dir)
CASES = [
    [("a", "b", [2, 20], [18, 0], [-2, 0], [1, 2], [1, 2]), ("b", "a", [2, 20], [0, 0], [20, 0], [1, 2], [1, 2])],
    [("a", "b", [20, 2], [0, 18], [0, -2], [1, 2], [1, 2]), ("b", "a", [20, 2], [0, 0], [0, 20], [1, 2], [1, 2])],
    [("a", "b", [2, 20], [0, 0], [20, 0], [1, 2], [1, -2]), ("b", "a", [2, 20], [18, 0], [-2, 0], [1, -2], [1, 2])],
    [("a", "b", [20, 2], [0, 0], [0, 20], [1, 2], [-1, 2]), ("b", "a", [20, 2], [0, 18], [0, -2], [-1, 2], [1, 2])],
    [("a", "b", [2, 20], [18, 0], [0, -2], [1, 2], [2, 1]), ("b", "a", [2, 20], [0, 0], [20, 0], [2, 1], [1, 2])],
    [("a", "bf", [3, 20], [17, 0], [-2, 0], [1, 2], [1, 2])],
]
TAGS = {"a": 10000.0, "b": 20000.0, "bf": 20000.0}


def initial():
    ext = SIZE - DM + DP
    out = {}
    x, y = np.meshgrid(np.arange(SIZE), np.arange(SIZE))
    for name, off, dt in (("a", 0.25, np.float64), ("b", 0.25, np.float64), ("bf", 0.5, np.float32)):
        arr = np.zeros((ext, ext), dtype=dt)
        arr[-DM:-DM + SIZE, -DM:-DM + SIZE] = (TAGS[name] + 100.0 * x + y + off).astype(dt)
        out[name] = arr
    return out


def refill(arrays):
    """Rewrite the interiors, keep the rings."""
    fresh = initial()
    for name, arr in arrays.items():
        arr[-DM:-DM + SIZE, -DM:-DM + SIZE] = fresh[name][-DM:-DM + SIZE, -DM:-DM + SIZE]
    return arrays
