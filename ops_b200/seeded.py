"""Seeded synthetic inputs (counter-based SplitMix64, numpy uint64).

The k-th output of the stream `seed` is mix(seed + (k+1) * GAMMA) with the
SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014); uniform doubles take
its top 53 bits. Identical bit for bit to the C definition used on the
reference side (oracle/src/seeded_rng.h), which a CPU test checks.
"""
import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def sm64_at(seed, k):
    """Raw 64-bit outputs for counter array k (any integer array)."""
    k = np.asarray(k, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (k + np.uint64(1)) * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def u01(seed, k):
    """Uniform doubles in [0, 1)."""
    return (sm64_at(seed, k) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform(seed, k, lo, hi):
    return lo + (hi - lo) * u01(seed, k)


def laplace_field(imax, jmax, seed):
    """Laplace initial field: full (jmax+2) x (imax+2) extent, zero interior,
    ring cell (x, y) = u01(seed, (y+1)*(imax+2) + (x+1))."""
    W, H = imax + 2, jmax + 2
    k = np.arange(W * H, dtype=np.uint64).reshape(H, W)
    A = u01(seed, k)
    A[1:-1, 1:-1] = 0.0
    return np.ascontiguousarray(A)


def clover_rectangles(x_cells, y_cells, seed, n=4, xmin=0.0, xmax=10.0, ymin=0.0, ymax=10.0):
    """n seeded rectangles with corners on grid lines, density U[0.5, 2] and
    energy U[1, 3]: rectangle i draws counters 8i..8i+5 of stream `seed`."""
    states = []
    for i in range(n):
        u = u01(seed, np.arange(8 * i, 8 * i + 6, dtype=np.uint64))
        w = max(1, int(x_cells * (0.05 + 0.25 * u[0])))
        h = max(1, int(y_cells * (0.05 + 0.25 * u[1])))
        x0 = int(u[2] * (x_cells - w))
        y0 = int(u[3] * (y_cells - h))
        dx = (xmax - xmin) / x_cells
        dy = (ymax - ymin) / y_cells
        states.append(dict(density=float(0.5 + 1.5 * u[4]), energy=float(1.0 + 2.0 * u[5]), geometry="rectangle",
                           xmin=xmin + x0 * dx, xmax=xmin + (x0 + w) * dx, ymin=ymin + y0 * dy,
                           ymax=ymin + (y0 + h) * dy))
    return states


def clover_config2_states(x_cells, y_cells, seed=2):
    """Background rho=0.2, e=1.0 plus four seeded rectangles."""
    return [dict(density=0.2, energy=1.0)] + clover_rectangles(x_cells, y_cells, seed)


def clover3d_cuboids(x_cells, y_cells, z_cells, seed, n=3, lo=0.0, hi=10.0):
    """n seeded cuboids with corners on grid planes, density U[0.5, 2] and
    energy U[1, 3]: cuboid i draws counters 12i..12i+7 of stream `seed`."""
    states = []
    cells = (x_cells, y_cells, z_cells)
    for i in range(n):
        u = u01(seed, np.arange(12 * i, 12 * i + 8, dtype=np.uint64))
        box = {}
        for a, (name, c) in enumerate(zip("xyz", cells)):
            w = max(1, int(c * (0.1 + 0.3 * u[a])))
            c0 = int(u[3 + a] * (c - w))
            d = (hi - lo) / c
            box[name + "min"] = lo + c0 * d
            box[name + "max"] = lo + (c0 + w) * d
        states.append(dict(density=float(0.5 + 1.5 * u[6]), energy=float(1.0 + 2.0 * u[7]), geometry="cuboid", **box))
    return states


def clover3d_states(x_cells, y_cells, z_cells, seed=6):
    """Background rho=0.2, e=1.0 plus three seeded cuboids."""
    return [dict(density=0.2, energy=1.0)] + clover3d_cuboids(x_cells, y_cells, z_cells, seed)


def normal(seed, k):
    """Standard normal doubles (Box-Muller on counter pairs 2k, 2k+1)."""
    k = np.asarray(k, dtype=np.uint64)
    u1 = u01(seed, 2 * k)
    u2 = u01(seed, 2 * k + np.uint64(1))
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def trid_system(shape, solvedim, seed, dtype=np.float64):
    """ADI test systems (config 3): per line a = c = -lam, b = 1 + 2 lam with
    lam ~ U[0.1, 1], d ~ N(0, 1). `shape` is numpy order (z, y, x)."""
    nd = len(shape)
    ax = nd - 1 - solvedim                      # numpy axis of the solve dimension
    lshape = list(shape)
    lshape[ax] = 1
    nlines = int(np.prod(lshape))
    lam = uniform(seed, np.arange(nlines, dtype=np.uint64), 0.1, 1.0).reshape(lshape)
    lam = np.broadcast_to(lam, shape)
    a = (-lam).astype(dtype)
    c = (-lam).astype(dtype)
    b = (1.0 + 2.0 * lam).astype(dtype)
    d = normal(seed + 1, np.arange(int(np.prod(shape)), dtype=np.uint64)).reshape(shape).astype(dtype)
    return np.ascontiguousarray(a), np.ascontiguousarray(b), np.ascontiguousarray(c), np.ascontiguousarray(d)


def tea_config4_states(x_cells, y_cells, seed=4, n=16, xmin=0.0, xmax=10.0, ymin=0.0, ymax=10.0):
    """Implicit-heat problem: background rho=1 with energy U[0,1] plus n
    seeded rectangles (corners on grid lines) with rho log-uniform in
    [0.1, 100] and energy U[0,1]; rectangle i draws counters 8i..8i+5."""
    bg = float(u01(seed, np.array([10 ** 6], dtype=np.uint64))[0])
    states = [dict(density=1.0, energy=bg)]
    for i in range(n):
        u = u01(seed, np.arange(8 * i, 8 * i + 6, dtype=np.uint64))
        w = max(1, int(x_cells * (0.05 + 0.25 * u[0])))
        h = max(1, int(y_cells * (0.05 + 0.25 * u[1])))
        x0 = int(u[2] * (x_cells - w))
        y0 = int(u[3] * (y_cells - h))
        dx = (xmax - xmin) / x_cells
        dy = (ymax - ymin) / y_cells
        states.append(dict(density=float(10.0 ** (-1.0 + 3.0 * u[4])), energy=float(u[5]), geometry="rectangle",
                           xmin=xmin + x0 * dx, xmax=xmin + (x0 + w) * dx, ymin=ymin + y0 * dy,
                           ymax=ymin + (y0 + h) * dy))
    return states
