"""sm100a target for the reference's legacy OPS translator.

    python ops_b200/dropin/sm100a_target.py --legacy <ops_translator_legacy/c> --app <name> <OPS source files>

Run in the application's source directory, like the translator itself
(ops_translator_legacy/c/ops.py). The reference's translator does the
parsing and rewrites each source file into <file>_ops.cpp (its
parse_source_files and generate_ops_files, ops.py:468-845, imported from the
given directory: no reference code is copied); this target then writes
sm100a/<app>_kernels.cu in place of the reference's backend targets (the
CUDA one is ops_translator_legacy/c/ops_gen_mpi_cuda.py:60). For every
kernel that file holds:

  * a device functor whose call operator is the application's own kernel
    function (its text from the app's *_kernel.h, taken by the translator's
    util.get_kernel_func_text), with ACC<T> bound to the OPS-B200 accessor of
    the loop's dimension, a reduction pointer replaced by the runtime's
    thread-local accumulator RED<T, dim> and an ops_arg_idx pointer by IDX;
  * its registration with the runtime as "<app>/<kernel>";
  * ops_par_loop_<kernel>(name, block, dim, range, args...), which queues
    the loop on the runtime through opsb_dropin_par_loop.

and once: the application's global constants as __constant__ symbols
registered with the runtime, ops_decl_const_char (the reference's backends
generate it too) and ops_init_backend. Compiled with --fmad=false, every
kernel keeps the reference's floating-point results.
"""
import argparse
import os
import re
import sys


def _load_legacy(legacy_dir):
    sys.path.insert(0, legacy_dir)
    import ops as legacy  # noqa: E402  (the reference's ops_translator_legacy/c/ops.py)
    import util  # noqa: E402
    return legacy, util


def _split_top(text, sep=","):
    """Split at `sep` outside (), <>, [] and {}."""
    out, depth, cur = [], 0, ""
    for ch in text:
        if ch in "(<[{":
            depth += 1
        elif ch in ")>]}":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [p.strip() for p in out]


def _param_name(p):
    m = re.search(r"([A-Za-z_]\w*)\s*(\[[^\]]*\])?\s*$", p)
    if not m:
        raise ValueError(f"cannot find the parameter name in '{p}'")
    return m.group(1)


def _split_function(text, name):
    """(parameter text, body text) of `void name(params) { body }`."""
    m = re.search(r"\bvoid\s+" + re.escape(name) + r"\s*\(", text)
    if not m:
        raise ValueError(f"kernel {name}: function not found")
    i = m.end()
    depth = 1
    j = i
    while depth:
        if text[j] == "(":
            depth += 1
        elif text[j] == ")":
            depth -= 1
        j += 1
    params = text[i:j - 1]
    b0 = text.index("{", j)
    depth, k = 1, b0 + 1
    while depth:
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
        k += 1
    return params, text[b0 + 1:k - 1]


def _const_info(c):
    name = c["name"].replace('"', "").strip()
    dim = str(c["dim"]).strip()
    return name, c["type"].strip(), dim


_READ = 1  # the translator's access numbering (ops_translator_legacy/c/config.py): READ 1 ... MIN 6
_MAX_CONST_ELEMS = 64  # device slots of a constant array whose length is a run-time value


def generate(app, consts, kernels, util, src_dir="."):
    """Text of sm100a/<app>_kernels.cu."""
    out = []
    w = out.append
    w("// Generated by the OPS-B200 sm100a target of the OPS legacy translator.")
    w("// Each ops_par_loop of the application runs its own kernel function as a")
    w("// device functor on the OPS-B200 runtime (ops_b200/dropin).")
    w('#include "ops_lib_core.h"')
    w('#include "ops_dropin.h"')
    if os.path.exists(os.path.join(src_dir, "user_types.h")):
        w('#include "user_types.h"')
    w("")
    w("void ops_init_backend() {}")
    w("")
    # constants: device symbols, registered with the runtime, and the names
    # the kernel bodies use mapped onto them
    cinfo = [_const_info(c) for c in consts]
    seen = set()
    cinfo = [c for c in cinfo if not (c[0] in seen or seen.add(c[0]))]
    for name, typ, dim in cinfo:
        if dim.isdigit() and int(dim) == 1:
            w(f"__constant__ {typ} opsb_c_{name};")
        elif dim.isdigit():
            w(f"__constant__ {typ} opsb_c_{name}[{dim}];")
        else:
            w(f"__constant__ {typ} opsb_c_{name}[{_MAX_CONST_ELEMS}];  // length set at run time ({dim})")
    w("")
    w("void ops_decl_const_char(OPS_instance *instance, int dim, char const *type, int size, char *data,")
    w("                         char const *name) {")
    w("  (void)instance;")
    w("  (void)type;")
    for name, typ, dim in cinfo:
        w(f'  if (!strcmp(name, "{name}")) {{')
        if not dim.isdigit():
            w(f"    if (dim > {_MAX_CONST_ELEMS}) {{")
            w("      OPSException ex(OPS_INVALID_ARGUMENT);")
            w(f'      ex << "constant {name}: at most {_MAX_CONST_ELEMS} elements on the device";')
            w("      throw ex;")
            w("    }")
        w(f"    if ((size_t)dim * size > sizeof(opsb_c_{name})) {{")
        w("      OPSException ex(OPS_INVALID_ARGUMENT);")
        w(f'      ex << "constant {name} is larger than its declaration";')
        w("      throw ex;")
        w("    }")
        w("    cudaStream_t s = opsb_dropin_const_begin();")
        w(f'    opsb_dropin_const_done(cudaMemcpyToSymbolAsync(opsb_c_{name}, data, (size_t)dim * size, 0,')
        w(f'                                                   cudaMemcpyHostToDevice, s), "{name}");')
        w("    return;")
        w("  }")
    w("  OPSException ex(OPS_INVALID_ARGUMENT);")
    w('  ex << "ops_decl_const: no constant named " << name << " in the translated application";')
    w("  throw ex;")
    w("}")
    w("")
    # kernel functors
    for name, *_ in cinfo:
        w(f"#define {name} opsb_c_{name}")
    for k in kernels:
        name, nargs = k["name"], int(k["nargs"])
        dim = int(str(k["dim"]).strip())
        text = util.get_kernel_func_text(name, src_dir, k["arg_type"])
        params, body = _split_function(text, name)
        plist = _split_top(params)
        if len(plist) != nargs:
            raise ValueError(f"kernel {name}: {len(plist)} parameters for {nargs} loop arguments")
        newp = []
        for i, p in enumerate(plist):
            at, acc = k["arg_type"][i], int(k["accs"][i])
            if at == "ops_arg_gbl" and acc != _READ:
                d = str(k["dims"][i]).strip()
                if not d.isdigit():
                    raise ValueError(f"kernel {name}: reduction width '{d}' must be a number")
                newp.append(f"opsb::RED<{k['typs'][i].strip()}, {d}> &{_param_name(p)}")
            elif at == "ops_arg_idx":
                newp.append(f"const opsb::IDX &{_param_name(p)}")
            else:
                newp.append(p)
        acc_t = {1: "opsb::ACC2<T>", 2: "opsb::ACC2<T>", 3: "opsb::ACC3<T>"}[dim]
        w(f"struct opsb_k_{name} {{")
        w(f'  static constexpr const char *kname = "{app}/{name}";')
        w(f"  template <class T> using ACC = {acc_t};")
        w("  __device__ void operator()(" + ",\n      ".join(newp) + ") const {")
        w(body.rstrip())
        w("  }")
        w("};")
        w(f"OPSB_REGISTER_LOOP(opsb_k_{name});")
        w("")
    for name, *_ in cinfo:
        w(f"#undef {name}")
    w("")
    # host stubs
    for k in kernels:
        name, nargs = k["name"], int(k["nargs"])
        args = ", ".join(f"ops_arg arg{i}" for i in range(nargs))
        w(f"void ops_par_loop_{name}(char const *name, ops_block block, int dim, int *range, {args}) {{")
        w(f'  static const opsb::LoopInfo *loop = opsb_dropin_find_loop("{app}/{name}");')
        w(f"  ops_arg args[{nargs}] = {{" + ", ".join(f"arg{i}" for i in range(nargs)) + "};")
        w(f"  opsb_dropin_par_loop(loop, name, block, dim, range, args, {nargs});")
        w("}")
        w("")
    return "\n".join(out) + "\n"


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--legacy", required=True, help="the reference's ops_translator_legacy/c directory")
    ap.add_argument("--app", required=True, help="application name (kernel registry prefix)")
    ap.add_argument("sources", nargs="+")
    a = ap.parse_args(argv)
    legacy, util = _load_legacy(a.legacy)
    texts, loop_args, kernels_in_files, kernels, consts, _soa = legacy.parse_source_files(a.sources)
    legacy.generate_ops_files(a.sources, texts, loop_args, kernels_in_files, kernels)
    os.makedirs("sm100a", exist_ok=True)
    with open(os.path.join("sm100a", f"{a.app}_kernels.cu"), "w") as f:
        f.write(generate(a.app, consts, kernels, util))
    return 0


if __name__ == "__main__":
    sys.exit(main())
