"""Builds reference OPS applications, unmodified, on OPS-B200.

    python ops_b200/dropin/build_apps.py [reference_root] [app ...]

For each application its sources are copied from the reference tree into
ops_b200/dropin/_apps/<name>/ (the translator writes next to its inputs),
translated by the reference's legacy translator with the sm100a target
(sm100a_target.py), and compiled: the translated host files with g++ and
the reference's compiler flags, sm100a/<app>_kernels.cu with nvcc for
sm_100a (--fmad=false, so the kernels round like the reference's CPU build),
and linked with the drop-in API (ops_dropin.cu, compiled against the
reference's headers) and libops_b200.so into ops_b200/dropin/_apps/bin/<name>.
The reference root defaults to $OPS_REFERENCE_ROOT. Nothing from the
reference is kept in the repository: _apps/ is build output.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(HERE, "_apps")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CLOVER_OPS = ("clover_leaf.cpp initialise_chunk.cpp generate.cpp ideal_gas.cpp update_halo.cpp field_summary.cpp "
              "viscosity.cpp calc_dt.cpp PdV.cpp revert.cpp accelerate.cpp flux_calc.cpp advec_cell.cpp advec_mom.cpp "
              "reset_field.cpp").split()
CLOVER_OTHER = "start.cpp time_step.cpp build_field.cpp read_input.cpp initialise.cpp advection.cpp".split()

TEA_OPS = ("tea_leaf.cpp field_summary.cpp generate.cpp initialise_chunk.cpp start.cpp set_field.cpp tea_leaf_cg.cpp "
           "tea_leaf_cheby.cpp tea_leaf_common.cpp tea_leaf_jacobi.cpp tea_leaf_ppcg.cpp update_halo.cpp").split()


def _other_cpp(ref, srcrel, opsf):
    """The application's remaining .cpp files (compiled as they are)."""
    d = os.path.join(ref, srcrel)
    return sorted(f for f in os.listdir(d) if f.endswith(".cpp") and f not in opsf)


# name: (source directory in the reference tree, registry prefix, OPS files, other files or None = all others)
APPS = {
    "laplace2d_step7": ("apps/c/laplace2d_tutorial/step7", "laplace2d", ["laplace2d.cpp"], []),
    "cloverleaf": ("apps/c/CloverLeaf", "cloverleaf_dropin", CLOVER_OPS, CLOVER_OTHER),
    "cloverleaf3d": ("apps/c/CloverLeaf_3D", "cloverleaf3d_dropin", CLOVER_OPS, CLOVER_OTHER),
    "tealeaf": ("apps/c/TeaLeaf", "tealeaf_dropin", TEA_OPS, None),
}


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("failed: " + " ".join(cmd) + "\n" + r.stdout[-4000:] + r.stderr[-4000:])


def _newer(target, deps):
    return os.path.exists(target) and all(os.path.getmtime(target) >= os.path.getmtime(d) for d in deps)


def _lib_headers():
    """The library headers the shim and the generated loop stubs compile
    against: a change to any of them (a struct's layout) rebuilds both."""
    hs = [os.path.join(PKG, "csrc", f) for f in os.listdir(os.path.join(PKG, "csrc")) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(ROOT, "include", "ops_b200.h")]


def shim_object(ref):
    inc = os.path.join(ref, "ops", "c", "include")
    obj = os.path.join(OUT, "obj", "ops_dropin.o")
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    deps = [os.path.join(HERE, "ops_dropin.cu"), os.path.join(HERE, "ops_dropin.h")] + _lib_headers()
    if not _newer(obj, deps):
        _run([NVCC] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I" + inc,
                              "-I" + os.path.join(PKG, "csrc"), "-I" + HERE, "-I" + os.path.join(ROOT, "include"),
                              "-x", "cu", "-c", os.path.join(HERE, "ops_dropin.cu"), "-o", obj], cwd=HERE)
    return obj


def build_app(ref, name):
    srcrel, prefix, opsf, other = APPS[name]
    if other is None:
        other = _other_cpp(ref, srcrel, opsf)
    src = os.path.join(ref, srcrel)
    inc = os.path.join(ref, "ops", "c", "include")
    wd = os.path.join(OUT, name)
    exe = os.path.join(OUT, "bin", name)
    deps = [os.path.join(src, f) for f in os.listdir(src)] + [
        os.path.join(HERE, f) for f in ("sm100a_target.py", "ops_dropin.cu", "ops_dropin.h", "build_apps.py")
    ] + _lib_headers()
    if _newer(exe, deps):
        return exe
    if os.path.isdir(wd):
        shutil.rmtree(wd)
    os.makedirs(wd)
    for f in os.listdir(src):
        if f.endswith((".h", ".cpp")):
            shutil.copy(os.path.join(src, f), wd)
    _run([sys.executable, os.path.join(HERE, "sm100a_target.py"), "--legacy",
          os.path.join(ref, "ops_translator_legacy", "c"), "--app", prefix] + opsf, cwd=wd)
    cxxflags = ["-O3", "-fPIC", "-ffloat-store", "-std=c++17", "-Dgnu", "-w", "-I" + inc, "-I."]
    objs = []
    for f in [x[:-4] + "_ops.cpp" for x in opsf] + other:
        o = os.path.join(wd, os.path.basename(f)[:-4] + ".o")
        _run([CXX] + cxxflags + ["-c", f, "-o", o], cwd=wd)
        objs.append(o)
    ko = os.path.join(wd, "kernels.o")
    _run([NVCC] + ARCH + ["-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                          "-w", "-I" + inc, "-I" + os.path.join(PKG, "csrc"), "-I" + HERE,
                          "-I" + os.path.join(ROOT, "include"), "-I.", "-x", "cu", "-c",
                          os.path.join("sm100a", prefix + "_kernels.cu"), "-o", ko], cwd=wd)
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    _run([NVCC] + ARCH + ["-o", exe] + objs + [ko, shim_object(ref), "-L" + PKG, "-lops_b200",
                                               "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../../.."], cwd=wd)
    return exe


def build(ref=None, names=None):
    ref = ref or os.environ.get("OPS_REFERENCE_ROOT")
    if not ref or not os.path.isdir(os.path.join(ref, "ops", "c", "include")):
        return []
    return [build_app(ref, n) for n in (names or sorted(APPS))]


def binary(name):
    """Path of a built drop-in application, or None."""
    p = os.path.join(OUT, "bin", name)
    return p if os.path.exists(p) else None


if __name__ == "__main__":
    args = sys.argv[1:]
    ref = args.pop(0) if args and os.path.isdir(args[0]) else None
    for e in build(ref, args or None):
        print("built", e)
