"""Python mirror of the OPS C/C++ API over the OPS-B200 C-ABI.

Names, argument order and meaning follow ops/c/include/ops_lib_core.h and
ops_seq_v2.h; failures raise OpsError (the reference throws OPSException,
ops/c/include/ops_exceptions.h:46-77). Kernels are the registered sm_100a
loop kernels, named "<app>/<kernel>" where <kernel> is the reference's kernel
function name (e.g. "laplace2d/apply_stencil").

    ops_init(0)
    grid = ops_decl_block(2, "grid")
    A = ops_decl_dat(grid, 1, [nx, ny], [0, 0], [-1, -1], [1, 1], None, "double", "A")
    ...
    ops_par_loop("laplace2d/apply_stencil", "apply stencil", grid, 2, [0, nx, 0, ny],
                 ops_arg_dat(A, 1, S5, "double", OPS_READ),
                 ops_arg_dat(Anew, 1, S0, "double", OPS_WRITE),
                 ops_arg_reduce(h_err, 1, "double", OPS_MAX))
    err = ops_reduction_result(h_err)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import OpsError, check, lib

OPS_READ, OPS_WRITE, OPS_RW, OPS_INC, OPS_MIN, OPS_MAX = 0, 1, 2, 3, 4, 5
OPS_HOST, OPS_DEVICE = 1, 2

_TYPES = {"double": (np.float64, 8), "float": (np.float32, 4), "int": (np.int32, 4),
          "long long": (np.int64, 8), "ll": (np.int64, 8)}


class ops_block:
    def __init__(self, h, dims, name):
        self.index, self.dims, self.name = h, dims, name


class ops_dat:
    def __init__(self, h, block, dim, size, d_m, d_p, type_, name):
        self.index, self.block, self.dim, self.type, self.name = h, block, dim, type_, name
        self.d_m, self.d_p = list(d_m), list(d_p)
        # Full extent including halos (ops_dat_core::size).
        self.size = [s - m + p for s, m, p in zip(size, d_m, d_p)]

    @property
    def dtype(self):
        return _TYPES[self.type][0]

    def extent_shape(self):
        """numpy shape of the full extent, slowest dimension first."""
        shp = list(reversed(self.size))
        if self.dim > 1:
            shp.append(self.dim)
        return tuple(shp)


class ops_stencil:
    def __init__(self, h, dims, points, name):
        self.index, self.dims, self.points, self.name = h, dims, points, name


class ops_reduction:
    def __init__(self, h, size, type_, name):
        self.index, self.size, self.type, self.name = h, size, type_, name


def _iarr(v):
    a = (ctypes.c_int * len(v))(*[int(x) for x in v])
    return a


# what the diagnostic and timing output report: the diagnostics level given
# to ops_init and the blocks and dats declared since
_STATE = {"diags": 0, "blocks": [], "dats": []}


def ops_init(device=0, diags=0):
    """ops_init. As in the reference, diags > 1 times every loop (per-kernel
    CUDA-event timing, read by ops_timing_output) and diags > 2 enables
    ops_diagnostic_output."""
    check(lib().ops_b200_init(device, diags))
    _STATE["diags"] = diags
    check(lib().ops_b200_set_kernel_timing(1 if diags > 1 else 0))


def ops_exit():
    check(lib().ops_b200_exit())


def ops_decl_block(dims, name):
    b = ops_block(check(lib().ops_b200_decl_block(dims, name.encode())), dims, name)
    _STATE["blocks"].append(b)
    return b


def ops_decl_dat(block, dim, size, base, d_m, d_p, data, type_, name, stride=None):
    """ops_decl_dat; `data` (numpy array or None) holds the full extent.
    `stride` (the multigrid overload's coarsening factor) only matters to the
    reference's MPI decomposition and is accepted and ignored here."""
    dtype, ts = _TYPES[type_]
    buf = None
    if data is not None:
        buf = np.ascontiguousarray(data, dtype=dtype)
    h = check(lib().ops_b200_decl_dat(block.index, dim, _iarr(size), _iarr(base), _iarr(d_m), _iarr(d_p),
                                      buf.ctypes.data if buf is not None else None, ts, type_.encode(),
                                      name.encode()))
    d = ops_dat(h, block, dim, size, d_m, d_p, type_, name)
    d.base = list(base)
    _STATE["dats"].append(d)
    return d


def ops_decl_stencil(dims, points, sten, name):
    return ops_stencil(check(lib().ops_b200_decl_stencil(dims, points, _iarr(sten), name.encode())), dims,
                       points, name)


def ops_decl_strided_stencil(dims, points, sten, stride, name):
    return ops_stencil(check(lib().ops_b200_decl_strided_stencil(dims, points, _iarr(sten), _iarr(stride),
                                                                 name.encode())), dims, points, name)


def ops_decl_restrict_stencil(dims, points, sten, stride, name):
    """ops_decl_restrict_stencil: at loop point x, the dat at x * stride + offset."""
    return ops_stencil(check(lib().ops_b200_decl_restrict_stencil(dims, points, _iarr(sten), _iarr(stride),
                                                                  name.encode())), dims, points, name)


def ops_decl_prolong_stencil(dims, points, sten, stride, name):
    """ops_decl_prolong_stencil: at loop point x, the dat at floor(x / stride) + offset."""
    return ops_stencil(check(lib().ops_b200_decl_prolong_stencil(dims, points, _iarr(sten), _iarr(stride),
                                                                 name.encode())), dims, points, name)


def ops_decl_reduction_handle(size, type_, name):
    return ops_reduction(check(lib().ops_b200_decl_reduction_handle(size, type_.encode(), name.encode())), size,
                         type_, name)


def _ivec(v):
    a = np.ascontiguousarray(v, dtype=np.int32)
    return a, a.ctypes.data


def ops_decl_halo(from_dat, to_dat, iter_size, from_base, to_base, from_dir, to_dir):
    """ops_decl_halo (ops/c/include/ops_lib_core.h:888); returns a halo handle."""
    arrs = [_ivec(v) for v in (iter_size, from_base, to_base, from_dir, to_dir)]
    f = from_dat.index if hasattr(from_dat, "index") else int(from_dat)
    t = to_dat.index if hasattr(to_dat, "index") else int(to_dat)
    return check(lib().ops_b200_decl_halo(f, t, *[p for _, p in arrs]))


def ops_decl_halo_group(halos):
    """ops_decl_halo_group (ops_lib_core.h:902); returns a group handle."""
    a, p = _ivec(list(halos))
    return check(lib().ops_b200_decl_halo_group(len(a), p))


def ops_halo_transfer(group):
    """ops_halo_transfer (ops_lib_core.h:911)."""
    check(lib().ops_b200_halo_transfer(group))


def loops_skipped():
    """Loops dropped as redundant since ops_init (see ops_b200_loops_skipped)."""
    v = ctypes.c_longlong(0)
    check(lib().ops_b200_loops_skipped(ctypes.byref(v)))
    return v.value


def ops_timers():
    """ops_timers: (cpu seconds, wall-clock seconds)."""
    c, e = ctypes.c_double(0.0), ctypes.c_double(0.0)
    check(lib().ops_b200_timers(ctypes.byref(c), ctypes.byref(e)))
    return c.value, e.value


def ops_decl_const(name, dim, type_, data):
    arr = np.ascontiguousarray(np.atleast_1d(data), dtype=_TYPES[type_][0]) if type_ in _TYPES else data
    check(lib().ops_b200_decl_const(name.encode(), dim, type_.encode(),
                                    arr.ctypes.data if isinstance(arr, np.ndarray) else ctypes.addressof(arr)))


ops_update_const = ops_decl_const


def ops_arg_dat(dat, dim, stencil, type_, acc):
    return _lib.Arg(_lib.ARG_DAT, dat.index, stencil.index, dim, acc, 1, -1, 0, None), None


def ops_arg_dat_opt(dat, dim, stencil, type_, acc, flag):
    return _lib.Arg(_lib.ARG_DAT, dat.index, stencil.index, dim, acc, 1 if flag else 0, -1, 0, None), None


def ops_arg_gbl(data, dim, type_, acc):
    arr = np.ascontiguousarray(np.atleast_1d(data), dtype=_TYPES[type_][0])
    return _lib.Arg(_lib.ARG_GBL, -1, -1, dim, acc, 1, -1, arr.itemsize, arr.ctypes.data), arr


def ops_arg_reduce(handle, dim, type_, acc):
    return _lib.Arg(_lib.ARG_REDUCE, -1, -1, dim, acc, 1, handle.index, 0, None), None


def ops_arg_idx():
    return _lib.Arg(_lib.ARG_IDX, -1, -1, 1, OPS_READ, 1, -1, 4, None), None


def ops_par_loop(kernel, name, block, dim, rng, *args):
    """Queue one loop; `kernel` is a registered kernel name."""
    arr = (_lib.Arg * max(1, len(args)))()
    keep = []
    for i, (a, k) in enumerate(args):
        arr[i] = a
        keep.append(k)
    check(lib().ops_b200_par_loop(kernel.encode(), name.encode(), block.index, dim, _iarr(rng), len(args), arr))


def ops_execute():
    check(lib().ops_b200_execute())


def ops_reduction_result(handle, count=None):
    """Returns the reduced value(s) as a numpy array (or a scalar for width 1)."""
    dtype, ts = _TYPES[handle.type]
    n = handle.size // ts
    out = np.zeros(n, dtype=dtype)
    check(lib().ops_b200_reduction_result(handle.index, out.ctypes.data))
    return out[0] if n == 1 else out


def ops_dat_set_data(dat, data):
    buf = np.ascontiguousarray(data, dtype=dat.dtype)
    check(lib().ops_b200_dat_set_data(dat.index, buf.ctypes.data, buf.nbytes))


def ops_dat_fetch_data(dat):
    """The dat's data: the full extent, or the rank's owned part of a block
    partitioned across ranks (ops_dat_get_extents)."""
    _, size = ops_dat_get_extents(dat)
    shp = list(reversed(size)) + ([dat.dim] if dat.dim > 1 else [])
    out = np.zeros(tuple(shp), dtype=dat.dtype)
    check(lib().ops_b200_dat_fetch_data(dat.index, out.ctypes.data, out.nbytes))
    return out


def ops_dat_get_extents(dat):
    nd = dat.block.dims
    disp = (ctypes.c_int * nd)()
    size = (ctypes.c_int * nd)()
    check(lib().ops_b200_dat_get_extents(dat.index, disp, size))
    return list(disp), list(size)


def ops_dat_get_raw_pointer(dat, memspace):
    ptr = ctypes.c_void_p()
    stride = (ctypes.c_int * 3)()
    check(lib().ops_b200_dat_get_raw_pointer(dat.index, memspace, ctypes.byref(ptr), stride))
    return ptr.value, list(stride)


def ops_dat_release_raw_data(dat, acc):
    check(lib().ops_b200_dat_release_raw_data(dat.index, acc))


def set_option(name, value):
    check(lib().ops_b200_set_option(name.encode(), int(value)))


def counters():
    k, g, l = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    check(lib().ops_b200_counters(ctypes.byref(k), ctypes.byref(g), ctypes.byref(l)))
    return {"kernels": k.value, "graphs": g.value, "loops": l.value}


def fusion_stats():
    """Loop-chain fusion since the last counter reset: fused kernels launched,
    loops they replaced, and the compulsory bytes fused vs as separate loops."""
    c, n, fb, lb = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
    check(lib().ops_b200_fusion_stats(ctypes.byref(c), ctypes.byref(n), ctypes.byref(fb), ctypes.byref(lb)))
    return {"chains": c.value, "loops": n.value, "fused_bytes": fb.value, "loop_bytes": lb.value}


def set_kernel_timing(on):
    check(lib().ops_b200_set_kernel_timing(int(on)))


def kernel_time(kernel):
    n, ms = ctypes.c_longlong(), ctypes.c_double()
    check(lib().ops_b200_kernel_time(kernel.encode(), ctypes.byref(n), ctypes.byref(ms)))
    return n.value, ms.value


def kernel_stats():
    """{kernel name: (launches, total_ms, alg_bytes)} of the timed kernels."""
    n = check(lib().ops_b200_kernel_stats(None, 0))
    arr = (_lib.KernelStat * max(n, 1))()
    check(lib().ops_b200_kernel_stats(arr, n))
    return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms, arr[i].alg_bytes) for i in range(n)}


def clear_kernel_timing():
    check(lib().ops_b200_clear_kernel_timing())


def reset_counters():
    check(lib().ops_b200_reset_counters())


def ops_tridMultiDimBatch(ndim, solvedim, rng, a, b, c, d, params=None):
    """ops_tridMultiDimBatch: solve along `solvedim` over `rng`, result in d."""
    check(lib().ops_b200_tridMultiDimBatch(ndim, solvedim, _iarr(rng), a.index, b.index, c.index, d.index))


def ops_tridMultiDimBatch_Inc(ndim, solvedim, rng, a, b, c, d, u, params=None):
    """ops_tridMultiDimBatch_Inc: solve along `solvedim` over `rng`, add the result to u."""
    check(lib().ops_b200_tridMultiDimBatch_Inc(ndim, solvedim, _iarr(rng), a.index, b.index, c.index, d.index,
                                               u.index))


def trid_batch(elem_size, solvedim, systems, stream=None):
    """Raw strided batch over device pointers; `systems` is a list of dicts with
    a, b, c, d, u (ints, u may be None), dims and pads (lists)."""
    arr = (_lib.TridSystem * max(1, len(systems)))()
    for i, s in enumerate(systems):
        t = arr[i]
        t.a, t.b, t.c, t.d = s["a"], s["b"], s["c"], s["d"]
        t.u = s.get("u")
        t.ndim = len(s["dims"])
        for k in range(3):
            t.dims[k] = s["dims"][k] if k < t.ndim else 1
            t.pads[k] = s["pads"][k] if k < t.ndim else 1
    check(lib().ops_b200_trid_batch(elem_size, solvedim, len(systems), arr, stream))


# ---- output, timing and host-data calls of the reference's single-process
# backend (ops/c/src/core/ops_dummy_singlenode.cpp, ops_lib_core.cpp)

def ops_printf(fmt, *args):
    """ops_printf (ops_dummy_singlenode.cpp:413): printf on the one process."""
    print(fmt % args if args else fmt, end="", flush=True)


def ops_fprintf(stream, fmt, *args):
    """ops_fprintf (ops_dummy_singlenode.cpp:457): fprintf to an open text stream."""
    stream.write(fmt % args if args else fmt)


def ops_partition(routine=None, opts=None):
    """ops_partition / ops_partition_opts: splits the blocks declared so far
    across the ranks of the transport set by ops_b200.dist (slabs along each
    block's outermost dimension); with one process it does nothing, as in the
    reference's single-process backends (ops_dummy_singlenode.cpp:892-899).
    `opts` (the reference's decomposition hints) is accepted and ignored."""
    check(lib().ops_b200_partition((routine or "").encode()))


def ops_timing_output(stream=None):
    """ops_timing_output (ops_lib_core.cpp:1468-1626): with diags > 1, one
    line per loop kernel (name, launches, mean seconds per call with its
    spread, MPI time, bandwidth) and the total kernel time. Here every launch
    is timed with CUDA events on the runtime stream; the spread and the MPI
    time are 0 (the per-launch times are not kept, and there is no MPI), and
    the bandwidth is the loop's algorithmic bytes over its time in GiB/s,
    the reference's unit."""
    import sys
    stream = stream or sys.stdout
    if _STATE["diags"] <= 1:
        return
    st = kernel_stats()
    if not st:
        return
    width = max(len(k) for k in st)
    stream.write("\n\n%s  Count Time     MPI-time     Bandwidth(GB/s)\n" % "Name".ljust(width))
    stream.write("-" * (width + 31) + "\n")
    total = 0.0
    for name, (count, ms, byt) in st.items():
        t = ms * 1e-3
        bw = byt / (t * 1024 ** 3) if t > 0 else 0.0
        stream.write("%s%-5d %-6f (%-6f) %-6f (%-6f)  %-13.2f\n" % (name.ljust(width + 2), count, t, 0.0, 0.0, 0.0, bw))
        total += t
    stream.write("Total kernel time: %g\n" % total)


def ops_diagnostic_output():
    """ops_diagnostic_output (ops_lib_core.cpp:1214-1262): with diags > 2, the
    declared blocks and dats with their sizes, bases, halo depths and memory."""
    if _STATE["diags"] <= 2:
        return
    ops_printf("\n OPS diagnostic output\n --------------------\n")
    ops_printf("\n block dimension\n -------------------\n")
    for b in _STATE["blocks"]:
        ops_printf(" %15s %15dD \n", b.name, b.dims)
    ops_printf("\n %15s %15s %15s %10s %10s %10s %15s %15s\n", "data", "item/point", "[block_size]", "[base]",
               "[d_m]", "[d_p]", "memory(MBytes)", "block")
    ops_printf(" " + "-" * 73 + "\n")
    tot = 0.0
    for d in _STATE["dats"]:
        nd = d.block.dims
        mem = float(np.prod(d.size[:nd])) * d.dim * np.dtype(d.dtype).itemsize
        tot += mem
        br = lambda v: "".join("[%d]" % x for x in v[:nd])  # noqa: E731
        ops_printf(" %15s %15d %s %s %s %s  %15.3f  %15s\n", d.name, d.dim, br(d.size), br(getattr(d, "base", [0] * nd)),
                   br(d.d_m), br(d.d_p), mem / (1024.0 * 1024.0), d.block.name)
    ops_printf(" Total Memory Allocated for ops_dats (GBytes) : %.3f\n", tot / (1024.0 ** 3))


def ops_get_data(dat):
    """ops_get_data (ops_lib_core.cpp:2366): the reference copies the device
    copy of the dat to its host storage. Dats here live on the device only;
    this returns the host copy of the full extent (as ops_dat_fetch_data)."""
    return ops_dat_fetch_data(dat)


def ops_put_data(dat, data):
    """ops_put_data (ops_lib_core.cpp:2382): the reference uploads the dat's
    host storage to the device; here the host data is passed in (the full
    extent, as ops_dat_set_data)."""
    ops_dat_set_data(dat, data)


def ops_print_dat_to_txtfile(dat, file_name):
    """ops_print_dat_to_txtfile (ops_lib_core.cpp:1272-1420): appends the
    dat's name, dim, extent, element size and every value of the full extent
    (x fastest; FP64 as " %3.10lf", FP32 as "%e ", integers as "%d ") to a
    text file, one row of x per line."""
    vals = ops_dat_fetch_data(dat)
    nd = dat.block.dims
    es = np.dtype(dat.dtype).itemsize
    with open(file_name, "a") as fp:
        fp.write("ops_dat:  %s \n" % dat.name)
        fp.write("ops_dat dim:  %d \n" % dat.dim)
        fp.write("block Dims : %d " % nd + "".join("[%d]" % x for x in dat.size[:nd]) + "\n")
        fp.write("elem size %d \n" % (es * dat.dim))
        if np.issubdtype(vals.dtype, np.floating):
            fmt = " %3.10lf" if vals.dtype == np.float64 else "%e "
        else:
            fmt = "%d "
        rows = vals.reshape(-1, dat.size[0] * dat.dim)
        for row in rows:
            fp.write("".join(fmt % v for v in row) + "\n")


class ops_tridsolver_params:
    """ops_tridsolver_params (ops/c/include/ops_tridiag.h:45-72): strategy and
    tuning of Tridsolver's multi-process solves, held by the C-ABI struct
    ops_b200_tridsolver_params. The reference's single-process backends
    ignore every setter (ops_tridiag.cpp:48-76); so does this one. The values
    given are kept for callers that read them back (None until set)."""
    GATHER_SCATTER, ALLGATHER, JACOBI, PCR, LATENCY_HIDING_INTERLEAVED, LATENCY_HIDING_TWO_STEP = range(6)

    def __init__(self, block, strategy=None):
        from ._lib import TridsolverParams
        self._p = TridsolverParams()
        handle = block if isinstance(block, int) else getattr(block, "index", -1)
        check(lib().ops_b200_tridsolver_params_init(ctypes.byref(self._p), int(handle),
                                                     -1 if strategy is None else int(strategy)))
        self.block, self.strategy = block, strategy
        self.jacobi = self.batch_size = self.cuda_opts = self.cuda_sync = None

    def set_jacobi_params(self, rtol, atol, maxiter):
        check(lib().ops_b200_tridsolver_params_set_jacobi_params(ctypes.byref(self._p), rtol, atol, maxiter))
        self.jacobi = (rtol, atol, maxiter)

    def set_batch_size(self, batch_size):
        check(lib().ops_b200_tridsolver_params_set_batch_size(ctypes.byref(self._p), batch_size))
        self.batch_size = batch_size

    def set_cuda_opts(self, opt_x, opt_y, opt_z):
        check(lib().ops_b200_tridsolver_params_set_cuda_opts(ctypes.byref(self._p), opt_x, opt_y, opt_z))
        self.cuda_opts = (opt_x, opt_y, opt_z)

    def set_cuda_sync(self, sync):
        check(lib().ops_b200_tridsolver_params_set_cuda_sync(ctypes.byref(self._p), sync))
        self.cuda_sync = sync


__all__ = [n for n in dir() if n.startswith("ops_")] + ["OpsError", "set_option", "counters", "reset_counters",
                                                          "fusion_stats",
                                                          "set_kernel_timing", "kernel_time", "clear_kernel_timing",
                                                          "trid_batch", "OPS_READ", "OPS_WRITE", "OPS_RW", "OPS_INC",
                                                          "OPS_MIN", "OPS_MAX", "OPS_HOST", "OPS_DEVICE"]
