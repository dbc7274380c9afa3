"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference's single-process halo transfer
(ops_halo_transfer, ops/c/src/sequential/ops_host_singlenode.cpp:172 and
ops/c/src/core/ops_device_singlenode_common.cpp:262-346 with its copy kernels
ops/c/src/cuda/ops_cuda_rt_support.cu:55-160): dat dimension i walks buffer
dimension |dir_i| - 1 of the iteration box, backwards when dir_i < 0, from
logical index base_i; the source is packed in that order and unpacked into
the target with the target's own bases and directions. Halos of a group are
applied in order; a float <-> double pair converts through the narrower type.
"""
import numpy as np


def _coords(iter_size, base, dirs, b):
    """Array-free logical coordinates of dat dimension i for buffer coords b."""
    out = []
    for i in range(len(dirs)):
        bd = abs(dirs[i]) - 1
        j = b[bd] if dirs[i] > 0 else iter_size[bd] - 1 - b[bd]
        out.append(base[i] + j)
    return out


def transfer(arrays, meta, halos):
    """arrays: name -> full-extent array, index order (z, y, x) reversed from OPS
    dimension order (x fastest); meta: name -> (base, d_m) lists in OPS order;
    halos: list of (src, dst, iter_size, from_base, to_base, from_dir, to_dir)."""
    for src, dst, it, fb, tb, fd, td in halos:
        nd = len(it)
        grids = np.meshgrid(*[np.arange(n) for n in it], indexing="ij")
        b = [g.ravel() for g in grids]
        sc = _coords(it, fb, fd, b)
        dc = _coords(it, tb, td, b)
        sbase, sdm = meta[src]
        dbase, ddm = meta[dst]
        sidx = tuple(sc[i] - sbase[i] - sdm[i] for i in reversed(range(nd)))
        didx = tuple(dc[i] - dbase[i] - ddm[i] for i in reversed(range(nd)))
        vals = arrays[src][sidx]
        if arrays[src].dtype != arrays[dst].dtype:
            narrow = min(arrays[src].dtype.itemsize, arrays[dst].dtype.itemsize)
            vals = vals.astype(np.float32 if narrow == 4 else np.float64)
        arrays[dst][didx] = vals.astype(arrays[dst].dtype)
    return arrays
