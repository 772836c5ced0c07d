"""Accuracy of the FP32 exponentials that the FP32-mixed real-space kernels
use in place of expf (p3mx_exp_check through the C ABI), over the range the
pair kernel meets, x = -(alpha r)^2 <= 0, against the FP64 exp of the same
FP32 inputs, down to x = -87 (below ln(FLT_MIN) = -87.34 the results are
subnormal and the hardware ex2 flushes them to zero, a term far below any
force the kernel sums):
  exp_fast (e^x = 2^y_hi (1 + y_lo ln 2), y = x log2 e split error-free,
  2^y_hi by the hardware ex2): relative error <= 2^-20;
  one ex2 of x log2(e) rounded to FP32 (the force-only kernel's form): the
  rounding of the constant and of the product costs up to |x| 2^-23 (each
  2^-24 |x log2 e| ln 2 = 2^-24 |x|), so <= 2^-21 + |x| 2^-23 (1e-5 at
  x = -87, 1.2e-6 at the real-space cutoff's x ~ -10);
  CUDA's expf: <= 2 ulp (2^-22).
"""
import numpy as np
import pytest
import torch

from espresso_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(x):
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    out = torch.empty(3 * len(x), dtype=torch.float32, device=dev)
    assert lib.p3mx_exp_check(len(x), _lib.dptr(xd), _lib.dptr(out), None) == 0
    torch.cuda.synchronize(dev)
    return out.cpu().numpy().reshape(3, -1)


def test_fp32_exponentials_over_the_pair_range():
    x = np.linspace(-87.0, 0.0, 1 << 20, dtype=np.float32)
    x = np.concatenate([x, -np.random.default_rng(5).uniform(0, 87, 1 << 18).astype(np.float32)])
    ref = np.exp(x.astype(np.float64))
    fast, ex2, expf = _run(x)
    rel = lambda y: np.abs(y.astype(np.float64) - ref) / ref
    assert rel(fast).max() <= 2.0 ** -20
    bound = 2.0 ** -21 + np.abs(x.astype(np.float64)) * 2.0 ** -23
    assert np.all(rel(ex2) <= bound), (rel(ex2) / bound).max()
    assert rel(expf).max() <= 2.0 ** -22
    # exp_fast gains over the plain form where |x| is large
    far = x < -40
    assert rel(fast)[far].max() < rel(ex2)[far].max()


def test_exponentials_at_the_ends():
    x = np.array([0.0, -1e-7, -1.0, -87.0, -88.0, -100.0], dtype=np.float32)
    fast, ex2, expf = _run(x)
    ref = np.exp(x.astype(np.float64))
    assert fast[0] == 1.0 and ex2[0] == 1.0
    np.testing.assert_allclose(fast[:4], ref[:4], rtol=2.0 ** -20, atol=0)
    # subnormal results flush to zero, never to anything larger
    assert np.all(fast[4:] <= 1.2e-38) and np.all(fast[4:] >= 0.0)
