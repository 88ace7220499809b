"""The warm-start CNN's CUDA kernels (tensor-core implicit GEMMs with TF32
operands) against the CPU restatement (oracle/cnn_ref.py, which rounds the
same operands to TF32): forward pass and the gradients of one training step
(FP32 device sums against float64 ones, checked norm-wise at 1e-5 / 1e-4),
at a size that spans several GEMM tiles and K chunks, and a few Adam steps
that reduce the loss of a fixed batch."""
import numpy as np
import pytest

import cnn_ref as R
from verb4d_b200.learned import CNN

pytestmark = pytest.mark.gpu
CH = (4, 8, 8, 1)


# tolerances (forward, gradients), norm-wise: the tensor cores accumulate a
# product sum in FP32 without rounding each addition to nearest, so the wider
# layers (K = 288 products per output, four layers) differ from the exact
# sum by more than the narrow test network
@pytest.mark.parametrize("B,H,W,CH,TF,TG", [(3, 9, 7, CH, 1e-5, 1e-4),
                                           (5, 31, 31, (4, 32, 32, 32, 1), 2e-3, 1e-2)])
def test_forward_and_gradients_match_cpu(gpu, B, H, W, CH, TF, TG):
    import torch

    rng = np.random.default_rng(0)
    net = CNN(H, W, B, channels=CH, seed=1)
    p = net.params()
    x = rng.standard_normal((B, 4, H, W)).astype(np.float32)
    t = rng.standard_normal((B, 1, H, W)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(t).cuda()
    out = torch.zeros((B, 1, H, W), device="cuda")
    net.forward(xd.data_ptr(), out.data_ptr(), B)
    torch.cuda.synchronize()
    acts = R.forward(p.astype(np.float64), CH, x.astype(np.float64))
    ref = acts[-1]
    ef = np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max()
    print("forward error %.2e" % ef)
    assert ef <= TF
    loss = net.train_step(xd.data_ptr(), td.data_ptr(), B, 0.0)   # gradients only
    _, g = net.params(with_grad=True)
    rloss, rg = R.gradients(p.astype(np.float64), CH, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - rloss) <= TF * rloss
    eg = np.abs(g - rg).max() / np.abs(rg).max()
    print("gradient error %.2e" % eg)
    assert eg <= TG
    net.close()


def test_adam_reduces_loss(gpu):
    import torch

    rng = np.random.default_rng(2)
    B, H, W = 8, 11, 11
    net = CNN(H, W, B, channels=CH, seed=3)
    x = torch.from_numpy(rng.standard_normal((B, 4, H, W)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal((B, 1, H, W)).astype(np.float32)).cuda()
    first = net.train_step(x.data_ptr(), t.data_ptr(), B, 1e-2)
    for _ in range(200):
        last = net.train_step(x.data_ptr(), t.data_ptr(), B, 1e-2)
    assert last < 0.5 * first
    net.close()
