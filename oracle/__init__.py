"""ORACLE — test infrastructure only, never part of the product path.

CPU restatements of the reference OPS algorithms on the accelerated path
(plain C under oracle/src, one function per reference routine, each citing
the reference file:line it follows), plus a recipe (build_ref.sh) that
compiles the reference's own OpenMP apps into oracle/_ref for pinning.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, and only as the checker. The product (ops_b200) never imports
it and has no CPU fallback.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "src")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "bin")
CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
# No fast-math and no contraction: every operation rounds as written.
CFLAGS = ["-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-std=c11", "-fopenmp"]

_lib = None


def _sources():
    return sorted(os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".c"))


def build():
    """Compile oracle/src/*.c into oracle/_build/liboracle.so (incremental)."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    deps = srcs + [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".h")]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [CC] + CFLAGS + ["-I" + SRC, "-o", LIB] + srcs + ["-lm"]
    subprocess.run(cmd, check=True)
    return LIB


def build_reference(ref_root=None):
    """Build the reference OpenMP apps into oracle/_ref (needs the reference
    tree: `ref_root`, else the OPS_REFERENCE_ROOT environment variable)."""
    ref_root = ref_root or os.environ.get("OPS_REFERENCE_ROOT")
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "ops", "c", "src")):
        return False
    subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), ref_root], check=True,
                   stdout=subprocess.DEVNULL)
    return True


def reference_binary(name):
    """Path of a reference app built by build_ref.sh, or None."""
    p = os.path.join(REF_BIN, name)
    return p if os.path.exists(p) else None


def lib():
    """The oracle shared library (built on first use)."""
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        _declare(_lib)
    return _lib


def _declare(L):
    c_int, c_double, c_u64, c_size = ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_size_t
    P = ctypes.c_void_p
    L.oracle_laplace_run.argtypes = [c_int, c_int, c_int, P, P]
    L.oracle_laplace_run.restype = None
    L.oracle_laplace_seed.argtypes = [c_int, c_int, c_u64, P]
    L.oracle_laplace_seed.restype = None
    L.oracle_laplace_step7_init.argtypes = [c_int, c_int, P]
    L.oracle_laplace_step7_init.restype = None
    L.oracle_sm64_at.argtypes = [c_u64, c_u64]
    L.oracle_sm64_at.restype = c_u64
    L.oracle_sm64_u01.argtypes = [c_u64, c_u64]
    L.oracle_sm64_u01.restype = c_double
    for name, args, res in _EXTRA_DECLS:
        if hasattr(L, name):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res


# Declarations of the other oracle modules: (name, argtypes, restype).
_P = ctypes.c_void_p
_EXTRA_DECLS = [
    ("oracle_trid_batch_d", [_P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P], None),
    ("oracle_trid_batch_s", [_P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P], None),
]
