"""Builds the OPS-B200 shared library (ops_b200/libops_b200.so) for sm_100a.

Every CUDA/C++ source under ops_b200/csrc is compiled by nvcc for
`-gencode arch=compute_100a,code=sm_100a` and linked into one shared library
that exports the C-ABI of include/ops_b200.h. The build is incremental: an
object is rebuilt when its source or any header under csrc/ or include/ is
newer. No GPU is needed to build.

Floating point: FP64 stencil kernels are compiled with --fmad=false so that
every cell update rounds exactly as the reference's x86-64 CPU build
(which has no fused multiply-add); files listed in FMAD_OK keep contraction.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libops_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
# Sources whose arithmetic may contract to FMA (no bit-parity requirement).
FMAD_OK = {"tridiag.cu", "heat_mg.cu"}


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _headers():
    hs = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                hs.append(os.path.join(d, f))
    return hs


def _compile(src, newest_header):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
        return obj, None
    fmad = [] if os.path.basename(src) in FMAD_OK else ["--fmad=false"]
    # Host-only .cpp files include the device headers too, so every source
    # goes through the CUDA front end.
    lang = ["-x", "cu"]
    cmd = [NVCC] + ARCH + COMMON + fmad + lang + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    hs = _headers()
    newest = max([os.path.getmtime(h) for h in hs] + [os.path.getmtime(__file__)])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, newest), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("\n".join(errs))
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
