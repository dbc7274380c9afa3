"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the learned-preconditioner network pieces (no reference
counterpart: the reference has no learned preconditioner), used to check the
sm_100a kernels: BF16 rounding and the 3x3 NHWC convolution in FP32 on
BF16-rounded values.
"""
import numpy as np


def to_bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_ulp(a):
    """Spacing of BF16 values in the binade of each |a| (8 significant bits)."""
    m = np.maximum(np.abs(np.asarray(a, dtype=np.float64)), 1e-30)
    return 2.0 ** (np.floor(np.log2(m)) - 7)


def conv3x3(x, w, bias=None):
    """y[n,h,w,co] = sum over taps (dy,dx) and ci of x[n,h+dy,w+dx,ci] * w[tap,co,ci]
    (+ bias[co]), zero padding, tap = (dy+1)*3 + (dx+1); float64 sums, FP32 result."""
    n, h, wd, ci = x.shape
    co = w.shape[1]
    xp = np.zeros((n, h + 2, wd + 2, ci), dtype=np.float64)
    xp[:, 1:-1, 1:-1, :] = x
    y = np.zeros((n, h, wd, co), dtype=np.float64)
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        patch = xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + wd, :]
        y += patch @ w[tap].astype(np.float64).T
    if bias is not None:
        y += bias
    return y.astype(np.float32)
