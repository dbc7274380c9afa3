"""The sm100a translator target on the reference's Laplace step7 app (CPU
only: translation, no device). Needs the reference tree
(OPS_REFERENCE_ROOT); skipped where it is absent."""
import os
import shutil
import subprocess
import sys

import pytest

REF = os.environ.get("OPS_REFERENCE_ROOT")
HERE = os.path.dirname(os.path.abspath(__file__))
TARGET = os.path.join(os.path.dirname(HERE), "ops_b200", "dropin", "sm100a_target.py")
pytestmark = pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF or "", "ops_translator_legacy")),
                                reason="reference tree not available (OPS_REFERENCE_ROOT)")


def test_step7_translation(tmp_path):
    src = os.path.join(REF, "apps", "c", "laplace2d_tutorial", "step7")
    for f in os.listdir(src):
        if f.endswith((".h", ".cpp")):
            shutil.copy(os.path.join(src, f), tmp_path)
    subprocess.run([sys.executable, TARGET, "--legacy", os.path.join(REF, "ops_translator_legacy", "c"), "--app",
                    "lap", "laplace2d.cpp"], cwd=tmp_path, check=True, capture_output=True)
    host = (tmp_path / "laplace2d_ops.cpp").read_text()
    gen = (tmp_path / "sm100a" / "lap_kernels.cu").read_text()
    # every loop became a call of the generated stub, every stub exists
    for k in ("set_zero", "left_bndcon", "right_bndcon", "apply_stencil", "copy"):
        assert f"ops_par_loop_{k}(" in host
        assert f"void ops_par_loop_{k}(char const *name, ops_block block" in gen
        assert f'kname = "lap/{k}"' in gen
    # the reduction became the runtime's accumulator, the index argument IDX
    assert "opsb::RED<double, 1> &error" in gen
    assert "const opsb::IDX &idx" in gen
    # constants: device symbols, copied by ops_decl_const_char
    for c in ("imax", "jmax", "pi"):
        assert f"__constant__" in gen and f"opsb_c_{c}" in gen
        assert f'if (!strcmp(name, "{c}"))' in gen
