"""Tensor-core (tcgen05) BF16 GEMM and MLP kernels against a PyTorch FP32
reference of the same operation on the same BF16-rounded inputs.

Tolerance: FP32 accumulation of BF16 products, relative 1e-5 of the output
scale (the reference product is computed in FP64 from the BF16 values)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def gemm(A, B, bias=None, act=0, transA=False, transB=False):
    """C = A B^T through msgb_gemm_bf16; A, B BF16 CUDA tensors (possibly transposed views)."""
    from beamax_b200 import _lib

    M, K = A.shape
    N = B.shape[0]
    C32 = torch.empty((M, N), dtype=torch.float32, device=A.device)
    C16 = torch.empty((M, N), dtype=torch.bfloat16, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    g = _lib.Gemm(A=A.data_ptr(), sAm=A.stride(0), sAk=A.stride(1), B=B.data_ptr(), sBn=B.stride(0),
                  sBk=B.stride(1), M=M, N=N, K=K, bias=bias.data_ptr() if bias is not None else None, act=act,
                  C32=C32.data_ptr(), ldc32=N, C16=C16.data_ptr(), ldc16=N, error_flag=err.data_ptr())
    _lib.check(_lib.lib().msgb_gemm_bf16(_lib.ref(g), torch.cuda.current_stream().cuda_stream), "gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C32, C16


# K-contiguous operands run the TMA-fed persistent kernel (the larger cases
# give every CTA several tiles: the A ring and both TMEM accumulators wrap);
# transposed operands run the element-staging kernel.
@pytest.mark.parametrize("M,N,K", [(128, 256, 256), (300, 256, 64), (128, 16, 256), (1000, 128, 16),
                                   (256, 64, 200), (4096, 256, 256), (56909, 256, 256), (20000, 16, 8),
                                   (5000, 48, 256)])
def test_gemm_matches_fp64_reference(M, N, K):
    dev = _dev()
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(dev)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(dev)
    bias = torch.randn(N, generator=g).to(dev)
    C32, C16 = gemm(A, B, bias=bias, act=1)
    ref = A.double() @ B.double().T + bias.double()
    scale = ref.abs().max()
    assert (C32.double() - ref).abs().max() <= 1e-5 * scale
    silu = ref * torch.sigmoid(ref)
    assert (C16.double() - silu).abs().max() <= 1e-2 * silu.abs().max()


def test_gemm_transposed_operands():
    dev = _dev()
    g = torch.Generator(device="cpu").manual_seed(5)
    At = torch.randn(192, 384, generator=g).to(torch.bfloat16).to(dev)   # stored K x M
    Bt = torch.randn(192, 256, generator=g).to(torch.bfloat16).to(dev)   # stored K x N
    C32, _ = gemm(At.T, Bt.T)
    ref = At.double().T @ Bt.double()
    assert (C32.double() - ref).abs().max() <= 1e-5 * ref.abs().max()


def test_mlp_forward_backward_match_oracle():
    """Gradients of the hand-written backward against the FP64 oracle of the
    same BF16 rounding points (oracle/mlp.py); 2e-3 relative per tensor, and
    the output within one BF16 unit in the last place of its largest entry (a
    product that rounds to the other side of a BF16 value in one layer moves
    the output by that much)."""
    from beamax_b200.surrogate import IN_PAD, MLP
    from oracle import mlp as orc

    dev = _dev()
    net = MLP(7, 12, width=256, depth=4, device=dev, seed=3)
    g = torch.Generator(device="cpu").manual_seed(1)
    for l in range(len(net.b)):  # non-zero biases exercise the bias path (seeded)
        net.b[l].copy_(0.1 * torch.randn(net.b[l].shape, generator=g))
    X = torch.zeros(384, IN_PAD)
    X[:, :7] = torch.randn(384, 7, generator=g)
    X16 = X.to(torch.bfloat16).to(dev)
    out, acts, pres = net.forward(X16, keep=True)
    dY = torch.randn(384, IN_PAD, generator=g)
    dY[:, 12:] = 0
    gW, gb = net.backward(dY.to(dev), acts, pres)
    W = [w.cpu().numpy() for w in net.W]
    b = [x.cpu().numpy() for x in net.b]
    Zr, ar, pr = orc.forward(W, b, X16.float().cpu().numpy())
    assert np.max(np.abs(out.cpu().numpy() - Zr)) <= 2.0 ** -8 * np.max(np.abs(Zr))
    gWr, gbr = orc.backward(W, ar, pr, dY.numpy())
    for l in range(len(W)):
        assert np.linalg.norm(gW[l].cpu().numpy() - gWr[l]) <= 2e-3 * np.linalg.norm(gWr[l]), l
        assert np.linalg.norm(gb[l].cpu().numpy() - gbr[l]) <= 2e-3 * np.linalg.norm(gbr[l]) + 1e-12, l


def test_mlp_training_reduces_loss():
    from beamax_b200.surrogate import MLP

    dev = _dev()
    g = torch.Generator(device="cpu").manual_seed(0)
    X = torch.rand(16384, 4, generator=g) * 2 - 1
    Y = torch.stack([torch.sin(2 * X[:, 0]) * X[:, 1], X[:, 2] * X[:, 3], torch.cos(X[:, 0] + X[:, 3])], 1)
    net = MLP(4, 3, width=128, depth=3, device=dev, seed=0)
    losses = net.train(X.to(dev), Y.to(dev), epochs=30, batch=1024, lr=3e-3, lr_min=1e-4)
    assert losses[-1] < 0.02 * losses[0], losses
