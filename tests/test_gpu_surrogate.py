"""The traveltime surrogate's tensor-core kernels (tcgen05 + TMEM) against
float64 references computed on the host."""
import numpy as np
import pytest

import kirch_datuming_b200 as kd

pytestmark = pytest.mark.gpu


def test_tensor_core_operand_views():
    # X W^T (forward layer), X W (backward through a layer), X^T W (weight
    # gradient): BF16 inputs, FP32 accumulation -> products are exact, only
    # the FP32 sums round
    import torch
    g = torch.Generator().manual_seed(7)
    X = torch.randn(128, 128, generator=g).to(torch.bfloat16)
    W = torch.randn(128, 128, generator=g).to(torch.bfloat16)
    D = kd.tc_selftest(X.cuda(), W.cuda()).cpu().double().numpy()
    x, w = X.double().numpy(), W.double().numpy()
    for got, ref in ((D[0], x @ w.T), (D[1], x @ w), (D[2], x.T @ w)):
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-6
