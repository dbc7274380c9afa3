"""Learned multigrid preconditioner: Python mirror of the C-ABI building
blocks. Device buffers are torch CUDA tensors (plumbing); the arithmetic is
the library's sm_100a kernels."""
import ctypes

from ._lib import check, lib

CONV_BIAS_RELU, CONV_BIAS, CONV_MASK, CONV_PLAIN = 0, 1, 2, 3


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def conv3x3(x, w, y, bias=None, mask=None, mode=CONV_PLAIN, stream=None):
    """y = conv3x3(x, w) on the tensor cores. x [n,h,w,cin] bf16, w [9,cout,cin]
    bf16, y [n,h,w,cout] bf16, bias [cout] fp32, mask like y (mode 2)."""
    n, h, wd, cin = x.shape
    cout = w.shape[1]
    assert tuple(w.shape) == (9, cout, cin) and tuple(y.shape) == (n, h, wd, cout)
    for t in (x, w, y, bias, mask):
        assert t is None or (t.is_cuda and t.is_contiguous())
    check(lib().ops_b200_conv3x3_bf16(_ptr(x), _ptr(w), _ptr(bias), _ptr(mask), _ptr(y), n, h, wd, cin, cout, mode,
                                      None if stream is None else ctypes.c_void_p(stream)))
