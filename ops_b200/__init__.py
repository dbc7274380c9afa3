"""OPS-B200: a B200-native (sm_100a) execution backend for the OPS
structured-mesh DSL.

The compute path is the in-tree shared library libops_b200.so (CUDA kernels
for sm_100a plus the C++ runtime), reached through its C-ABI
(include/ops_b200.h). `ops_b200.ops` mirrors the OPS C/C++ API names on top
of it; `ops_b200.apps` runs the reference app drivers restated on the
runtime. Nothing here computes on the CPU.
"""
from ._lib import OpsError, lib, check  # noqa: F401

__all__ = ["OpsError", "lib", "check"]
