"""ctypes binding of the OPS-B200 C-ABI (include/ops_b200.h).

The shared library is built in-tree (ops_b200/libops_b200.so, see build.py).
There is no fallback: if the library is missing or cannot be loaded, every
entry point of this package raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libops_b200.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOTFOUND, ERR_TIMEOUT, ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6
READ, WRITE, RW, INC, MIN, MAX = 0, 1, 2, 3, 4, 5
ARG_GBL, ARG_DAT, ARG_IDX, ARG_REDUCE = 0, 1, 2, 3
HOST, DEVICE = 1, 2


class OpsError(RuntimeError):
    """A failed C-ABI call (mirrors OPSException, ops/c/include/ops_exceptions.h:46)."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Arg(ctypes.Structure):
    _fields_ = [("argtype", ctypes.c_int), ("dat", ctypes.c_int), ("stencil", ctypes.c_int),
                ("dim", ctypes.c_int), ("acc", ctypes.c_int), ("opt", ctypes.c_int),
                ("reduction", ctypes.c_int), ("elem_size", ctypes.c_int), ("gbl", ctypes.c_void_p)]


class TridSystem(ctypes.Structure):
    _fields_ = [("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("c", ctypes.c_void_p), ("d", ctypes.c_void_p),
                ("u", ctypes.c_void_p), ("ndim", ctypes.c_int), ("dims", ctypes.c_int * 3),
                ("pads", ctypes.c_int * 3)]


class TridsolverParams(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("strategy", ctypes.c_int), ("jacobi_rtol", ctypes.c_double),
                ("jacobi_atol", ctypes.c_double), ("jacobi_maxiter", ctypes.c_int), ("batch_size", ctypes.c_int),
                ("cuda_opts", ctypes.c_int * 3), ("cuda_sync", ctypes.c_int)]


class KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 96), ("launches", ctypes.c_longlong), ("total_ms", ctypes.c_double),
                ("alg_bytes", ctypes.c_double)]


class CloverState(ctypes.Structure):
    _fields_ = [("density", ctypes.c_double), ("energy", ctypes.c_double), ("xvel", ctypes.c_double),
                ("yvel", ctypes.c_double), ("geometry", ctypes.c_int), ("xmin", ctypes.c_double),
                ("xmax", ctypes.c_double), ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
                ("radius", ctypes.c_double)]


class CloverDeck(ctypes.Structure):
    _fields_ = [("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("xmin", ctypes.c_double),
                ("ymin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
                ("initial_timestep", ctypes.c_double), ("timestep_rise", ctypes.c_double),
                ("max_timestep", ctypes.c_double), ("end_time", ctypes.c_double), ("end_step", ctypes.c_int),
                ("summary_frequency", ctypes.c_int), ("number_of_states", ctypes.c_int),
                ("states", CloverState * 16)]


class Clover3DState(ctypes.Structure):
    _fields_ = [("density", ctypes.c_double), ("energy", ctypes.c_double), ("xvel", ctypes.c_double),
                ("yvel", ctypes.c_double), ("zvel", ctypes.c_double), ("geometry", ctypes.c_int),
                ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double),
                ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
                ("radius", ctypes.c_double)]


class Clover3DDeck(ctypes.Structure):
    _fields_ = [("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("z_cells", ctypes.c_int),
                ("xmin", ctypes.c_double), ("ymin", ctypes.c_double), ("zmin", ctypes.c_double),
                ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
                ("initial_timestep", ctypes.c_double), ("timestep_rise", ctypes.c_double),
                ("max_timestep", ctypes.c_double), ("end_time", ctypes.c_double), ("end_step", ctypes.c_int),
                ("summary_frequency", ctypes.c_int), ("number_of_states", ctypes.c_int),
                ("states", Clover3DState * 16)]


class TeaDeck(ctypes.Structure):
    _fields_ = [("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("xmin", ctypes.c_double),
                ("ymin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
                ("initial_timestep", ctypes.c_double), ("end_time", ctypes.c_double), ("end_step", ctypes.c_int),
                ("summary_frequency", ctypes.c_int), ("max_iters", ctypes.c_int), ("eps", ctypes.c_double),
                ("coefficient", ctypes.c_int), ("preconditioner", ctypes.c_int), ("solver", ctypes.c_int),
                ("reflective_boundary", ctypes.c_int), ("check_result", ctypes.c_int),
                ("number_of_states", ctypes.c_int), ("states", CloverState * 24),
                ("fused", ctypes.c_int), ("mixed", ctypes.c_int), ("true_residual_stop", ctypes.c_int),
                ("reliable_delta", ctypes.c_double), ("ch_cg_presteps", ctypes.c_int),
                ("ch_cg_epslim", ctypes.c_double), ("ppcg_inner_steps", ctypes.c_int)]


class Msg(ctypes.Structure):
    _fields_ = [("peer", ctypes.c_int), ("send", ctypes.c_void_p), ("send_bytes", ctypes.c_size_t),
                ("recv", ctypes.c_void_p), ("recv_bytes", ctypes.c_size_t)]


EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(Msg), ctypes.c_int)
ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


class HeatSystem(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("pitch", ctypes.c_longlong),
                ("Kx", ctypes.c_void_p), ("Ky", ctypes.c_void_p), ("u0", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("rx", ctypes.c_double), ("ry", ctypes.c_double)]


class HeatSystem3D(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("pitch", ctypes.c_longlong),
                ("plane", ctypes.c_longlong), ("Kx", ctypes.c_void_p), ("Ky", ctypes.c_void_p),
                ("Kz", ctypes.c_void_p), ("u0", ctypes.c_void_p), ("u", ctypes.c_void_p), ("rx", ctypes.c_double),
                ("ry", ctypes.c_double), ("rz", ctypes.c_double)]


class HeatStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("updates", ctypes.c_int), ("converged", ctypes.c_int),
                ("fallbacks", ctypes.c_int), ("initial_residual", ctypes.c_double),
                ("final_residual", ctypes.c_double), ("seconds", ctypes.c_double), ("launches", ctypes.c_longlong)]


class HeatBatch(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("h", ctypes.c_int), ("w", ctypes.c_int), ("pitch", ctypes.c_longlong),
                ("image", ctypes.c_longlong), ("r", ctypes.c_void_p), ("Kx", ctypes.c_void_p),
                ("Ky", ctypes.c_void_p), ("rx", ctypes.c_double), ("ry", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OpsError(ERR_STATE, f"{LIB_PATH} is missing: build it with `python ops_b200/build.py`")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def check(rc):
    if rc < 0:
        msg = lib().ops_b200_last_error().decode()
        raise OpsError(rc, msg)
    return rc


def _declare(L):
    i, d, P, cp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p
    sz, ll = ctypes.c_size_t, ctypes.c_longlong
    sig = {
        "ops_b200_last_error": ([], cp),
        "ops_b200_init": ([i, i], i),
        "ops_b200_exit": ([], i),
        "ops_b200_decl_block": ([i, cp], i),
        "ops_b200_decl_dat": ([i, i, P, P, P, P, P, i, cp, cp], i),
        "ops_b200_decl_stencil": ([i, i, P, cp], i),
        "ops_b200_decl_strided_stencil": ([i, i, P, P, cp], i),
        "ops_b200_decl_restrict_stencil": ([i, i, P, P, cp], i),
        "ops_b200_decl_prolong_stencil": ([i, i, P, P, cp], i),
        "ops_b200_decl_reduction_handle": ([i, cp, cp], i),
        "ops_b200_decl_halo": ([i, i, P, P, P, P, P], i),
        "ops_b200_decl_halo_group": ([i, P], i),
        "ops_b200_halo_transfer": ([i], i),
        "ops_b200_timers": ([P, P], i),
        "ops_b200_loops_skipped": ([P], i),
        "ops_b200_decl_const": ([cp, i, cp, P], i),
        "ops_b200_update_const": ([cp, i, cp, P], i),
        "ops_b200_par_loop": ([cp, cp, i, i, P, i, P], i),
        "ops_b200_has_kernel": ([cp], i),
        "ops_b200_execute": ([], i),
        "ops_b200_reduction_result": ([i, P], i),
        "ops_b200_dat_set_data": ([i, P, sz], i),
        "ops_b200_dat_fetch_data": ([i, P, sz], i),
        "ops_b200_dat_get_extents": ([i, P, P], i),
        "ops_b200_dat_get_raw_pointer": ([i, i, P, P], i),
        "ops_b200_dat_release_raw_data": ([i, i], i),
        "ops_b200_set_option": ([cp, i], i),
        "ops_b200_counters": ([P, P, P], i),
        "ops_b200_reset_counters": ([], i),
        "ops_b200_release_spare_storage": ([P], i),
        "ops_b200_fusion_stats": ([P, P, P, P], i),
        "ops_b200_set_transport_host": ([i, i, EXCHANGE_FN, ALLGATHER_FN, P], i),
        "ops_b200_nccl_unique_id": ([P], i),
        "ops_b200_set_transport_nccl": ([P, i, i], i),
        "ops_b200_partition": ([cp], i),
        "ops_b200_rank_info": ([P, P, P], i),
        "ops_b200_block_slab": ([i, P, P, P, P, P], i),
        "ops_b200_slab_window": ([i, i, i, i, i, i, P, P, P, P, P, P], i),
        "ops_b200_transport_selftest": ([], i),
        "ops_b200_tridsolver_params_init": ([P, i, i], i),
        "ops_b200_tridsolver_params_set_jacobi_params": ([P, d, d, i], i),
        "ops_b200_tridsolver_params_set_batch_size": ([P, i], i),
        "ops_b200_tridsolver_params_set_cuda_opts": ([P, i, i, i], i),
        "ops_b200_tridsolver_params_set_cuda_sync": ([P, i], i),
        "ops_b200_set_kernel_timing": ([i], i),
        "ops_b200_kernel_time": ([cp, P, P], i),
        "ops_b200_clear_kernel_timing": ([], i),
        "ops_b200_kernel_stats": ([P, i], i),
        "ops_b200_app_laplace2d": ([i, i, i, i, P, P, P, P], i),
        "ops_b200_app_cloverleaf": ([P, i, P, i, P, P, cp], i),
        "ops_b200_app_cloverleaf3d": ([P, i, P, i, P, P, cp], i),
        "ops_b200_app_tealeaf": ([P, P, i, P, P, i, P, P, cp], i),
        "ops_b200_tridMultiDimBatch": ([i, i, P, i, i, i, i], i),
        "ops_b200_tridMultiDimBatch_Inc": ([i, i, P, i, i, i, i, i], i),
        "ops_b200_trid_batch": ([i, i, i, P, P], i),
        "ops_b200_conv3x3_bf16": ([P, P, P, P, P, i, i, i, i, i, i, P], i),
        "ops_b200_heat_solve": ([P, i, i, ctypes.c_double, i, i, P, P, P], i),
        "ops_b200_heat_solve3d": ([P, i, ctypes.c_double, i, P, P], i),
        "ops_b200_heat_mg_apply": ([P, P, P, P, P], i),
        "ops_b200_lmg_create": ([ctypes.c_ulonglong], i),
        "ops_b200_lmg_destroy": ([i], i),
        "ops_b200_lmg_num_params": ([], i),
        "ops_b200_lmg_get_params": ([i, P], i),
        "ops_b200_lmg_set_params": ([i, P], i),
        "ops_b200_lmg_get_grads": ([i, P], i),
        "ops_b200_lmg_apply": ([i, P, P, P], i),
        "ops_b200_lmg_train_step": ([i, P, P, i, ctypes.c_double, P, P], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
