"""Learned-preconditioner kernels on the B200 vs the numpy oracle (oracle/cnn.py).

The 3x3 convolution runs on the tcgen05 tensor cores with BF16 operands and
FP32 accumulation; inputs are BF16 values, so the oracle's result differs
from the kernel's only by summation order (about 1e-6 relative) before the
final rounding to BF16: outputs must agree to one BF16 unit in the last place
of their binade."""
import numpy as np
import pytest

from oracle import cnn as ref

pytestmark = pytest.mark.gpu
PAIRS = [(16, 16), (16, 32), (32, 16), (32, 32), (32, 64), (64, 32), (64, 64)]


def bf16_tensor(a):
    import torch
    return torch.from_numpy(ref.to_bf16(a)).to(torch.bfloat16).cuda()


def as_np(t):
    return t.float().cpu().numpy()


def close_bf16(got, want):
    tol = ref.bf16_ulp(want) * 1.0001 + 1e-5   # near zero: FP32 summation order, ~1e-6 absolute
    bad = np.abs(got.astype(np.float64) - want) > tol
    assert not bad.any(), f"{bad.sum()} of {bad.size} beyond one BF16 ulp; max {np.abs(got - want).max()}"


@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("shape", [(1, 8, 128), (2, 37, 45), (1, 16, 16), (3, 5, 300)])
def test_conv3x3_matches_oracle(gpu_runtime, cin, cout, shape):
    import torch
    from ops_b200 import cnn
    rng = np.random.default_rng(cin * 100 + cout + sum(shape))
    n, h, w = shape
    x = ref.to_bf16(rng.standard_normal((n, h, w, cin)).astype(np.float32))
    wt = ref.to_bf16((rng.standard_normal((9, cout, cin)) / np.sqrt(9 * cin)).astype(np.float32))
    b = rng.standard_normal(cout).astype(np.float32) * 0.1
    y = torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda")
    cnn.conv3x3(bf16_tensor(x), bf16_tensor(wt), y, bias=torch.from_numpy(b).cuda(), mode=cnn.CONV_BIAS)
    close_bf16(as_np(y), ref.to_bf16(ref.conv3x3(x, wt, b)))
    cnn.conv3x3(bf16_tensor(x), bf16_tensor(wt), y, bias=torch.from_numpy(b).cuda(), mode=cnn.CONV_BIAS_RELU)
    close_bf16(as_np(y), ref.to_bf16(np.maximum(ref.conv3x3(x, wt, b), 0)))


def test_conv3x3_mask_and_plain(gpu_runtime):
    import torch
    from ops_b200 import cnn
    rng = np.random.default_rng(7)
    x = ref.to_bf16(rng.standard_normal((2, 20, 70, 32)).astype(np.float32))
    wt = ref.to_bf16((rng.standard_normal((9, 16, 32)) / 17).astype(np.float32))
    m = ref.to_bf16(rng.standard_normal((2, 20, 70, 16)).astype(np.float32))
    y = torch.empty((2, 20, 70, 16), dtype=torch.bfloat16, device="cuda")
    cnn.conv3x3(bf16_tensor(x), bf16_tensor(wt), y, mode=cnn.CONV_PLAIN)
    want = ref.conv3x3(x, wt)
    close_bf16(as_np(y), ref.to_bf16(want))
    cnn.conv3x3(bf16_tensor(x), bf16_tensor(wt), y, mask=bf16_tensor(m), mode=cnn.CONV_MASK)
    close_bf16(as_np(y), ref.to_bf16(np.where(m > 0, want, 0)))
