"""The tcgen05 building blocks: one-CTA GEMM through the C ABI with 3-term
BF16 splits (tolerances: 1 product ~ BF16 rounding 1e-2; 3 products <=
1e-4; 6 products <= 2e-6 norm-wise relative vs an FP64 product)."""
import ctypes as C

import numpy as np
import pytest
import torch

from exoplasim_b200 import _lib
from tests._util import relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 16), (64, 32), (128, 64), (256, 64)])
def test_tc_selftest_split_products(N, K):
    rng = np.random.default_rng(N + K)
    A = rng.standard_normal((128, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    dA = torch.as_tensor(A, device="cuda")
    dB = torch.as_tensor(B, device="cuda")
    errs = {}
    for nprod in (1, 3, 6):
        dC = torch.full((128, N), float("nan"), device="cuda")
        s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.call("exotx_tc_selftest", C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                  C.c_void_p(dC.data_ptr()), N, K, nprod, s)
        got = dC.cpu().numpy()
        assert np.all(np.isfinite(got))
        errs[nprod] = relerr(got, ref)
    assert errs[1] < 2e-2
    assert errs[3] < 1e-4
    assert errs[6] < 2e-6
    assert errs[6] < errs[3] < errs[1]
