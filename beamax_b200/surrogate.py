"""Beam-trajectory surrogate: a BF16 MLP on the tcgen05 tensor cores.

An MLP (``in -> width x depth (SiLU) -> out``; 4 hidden layers of width 256 by
default) maps a beam's launch data and a time to its state, parametrised
relative to the homogeneous solution at the launch speed c(x0):

  inputs  x0 / L, mode * p0/|p0|, log10 w, log10 beta_min, log10 beta_max, t / T
  targets (x(t) - x_hom(t)) / L, (p(t) - p0) / |p0|,
          M(t)^-1 - M_hom(t)^-1 (packed, scaled by |p0| / (c0 T)),
          log A(t) - log A_hom(t)

(M^-1 stays bounded where M itself grows.)  Targets are standardised with
training-set statistics.  Training data are RK4 trajectories from
``msgb_rk4_trajectories``.  Every matrix product of training and inference
runs in ``msgb_gemm_bf16`` (FP32 accumulation in tensor memory); SiLU
backward, bias gradients (fixed-order column sums) and Adam are libmsgb
kernels too.  PyTorch only allocates buffers and assembles features.

Residual check used to decide whether to trust a prediction: the Hamiltonian
invariant c(x(t)) |p(t)| = c(x0) |p0| (G is homogeneous of degree 1 in p) and
an RK4 spot check on a sample of beams; beams that fail fall back to RK4.
"""

from __future__ import annotations

import ctypes
import math
from typing import List, Optional

import numpy as np

from . import _lib

IN_PAD = 16
OUT_PAD = 16


def _st():
    import torch

    return torch.cuda.current_stream().cuda_stream


class MLP:
    """MLP with FP32 master weights, BF16 compute copies and Adam state."""

    def __init__(self, in_dim: int, out_dim: int, width: int = 256, depth: int = 4, device="cuda", seed: int = 0):
        import torch

        if in_dim > IN_PAD or out_dim > OUT_PAD:
            raise ValueError("in/out dims must be <= 16")
        if width % 16 or width > 256:
            raise ValueError("width must be a multiple of 16 <= 256")
        self.in_dim, self.out_dim, self.width, self.depth = in_dim, out_dim, width, depth
        self.dims = [IN_PAD] + [width] * depth + [OUT_PAD]
        self.device = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W: List = []
        self.b: List = []
        for l in range(len(self.dims) - 1):
            fan_in = self.dims[l] if l > 0 else in_dim
            w = torch.randn(self.dims[l + 1], self.dims[l], generator=g) * math.sqrt(2.0 / fan_in)
            if l == 0:
                w[:, in_dim:] = 0.0
            if l == len(self.dims) - 2:
                w *= 0.1
                w[out_dim:, :] = 0.0
            self.W.append(w.to(self.device))
            self.b.append(torch.zeros(self.dims[l + 1], device=self.device))
        self.W16 = [w.to(torch.bfloat16) for w in self.W]
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)

    # ------------------------------------------------------------------ core
    def _gemm(self, A, sAm, sAk, B, sBn, sBk, M, N, K, bias=None, act=0, C32=None, ldc32=0, C16=None, ldc16=0):
        g = _lib.Gemm(A=A.data_ptr(), sAm=sAm, sAk=sAk, B=B.data_ptr(), sBn=sBn, sBk=sBk, M=M, N=N, K=K,
                      bias=bias.data_ptr() if bias is not None else None, act=act,
                      C32=C32.data_ptr() if C32 is not None else None, ldc32=ldc32,
                      C16=C16.data_ptr() if C16 is not None else None, ldc16=ldc16, error_flag=self.err.data_ptr())
        _lib.check(_lib.lib().msgb_gemm_bf16(_lib.ref(g), _st()), "msgb_gemm_bf16")

    def forward(self, X16, keep: bool = False):
        """X16: (B, 16) BF16.  Returns FP32 outputs (B, 16) and, with keep, the
        per-layer BF16 activations and FP32 pre-activations."""
        import torch

        Bsz = X16.shape[0]
        H = X16
        acts, pres = [X16], []
        L = len(self.W)
        for l in range(L):
            N, K = self.dims[l + 1], self.dims[l]
            last = l == L - 1
            Z = torch.empty((Bsz, N), dtype=torch.float32, device=self.device) if (keep or last) else None
            Hn = None if last else torch.empty((Bsz, N), dtype=torch.bfloat16, device=self.device)
            self._gemm(H, K, 1, self.W16[l], K, 1, Bsz, N, K, bias=self.b[l], act=0 if last else 1,
                       C32=Z, ldc32=N, C16=Hn, ldc16=N)
            if keep:
                pres.append(Z)
            if not last:
                acts.append(Hn)
                H = Hn
            else:
                out = Z
        return (out, acts, pres) if keep else out

    def backward(self, dY, acts, pres):
        """Gradients of sum(dY * Y) w.r.t. weights and biases (FP32)."""
        import torch

        L = len(self.W)
        Bsz = dY.shape[0]
        gW = [None] * L
        gb = [None] * L
        dZ32 = dY.contiguous()
        dZ16 = torch.empty(dZ32.shape, dtype=torch.bfloat16, device=self.device)
        _lib.check(_lib.lib().msgb_to_bf16(dZ32.data_ptr(), dZ32.numel(), dZ16.data_ptr(), _st()), "to_bf16")
        for l in range(L - 1, -1, -1):
            N, K = self.dims[l + 1], self.dims[l]
            H = acts[l]
            gw = torch.empty((N, K), dtype=torch.float32, device=self.device)
            # dW = dZ^T H: A(n, b) = dZ[b, n], B(k, b) = H[b, k]
            self._gemm(dZ16, 1, N, H, 1, K, N, K, Bsz, C32=gw, ldc32=K)
            gbv = torch.empty(N, dtype=torch.float32, device=self.device)
            _lib.check(_lib.lib().msgb_colsum(dZ32.data_ptr(), Bsz, N, N, gbv.data_ptr(), _st()), "colsum")
            gW[l], gb[l] = gw, gbv
            if l > 0:
                dH = torch.empty((Bsz, K), dtype=torch.float32, device=self.device)
                # dH = dZ W: A = dZ (b, n), B(k, n) = W[n, k]
                self._gemm(dZ16, N, 1, self.W16[l], 1, K, Bsz, K, N, C32=dH, ldc32=K)
                nz32 = torch.empty_like(dH)
                nz16 = torch.empty(dH.shape, dtype=torch.bfloat16, device=self.device)
                _lib.check(_lib.lib().msgb_silu_backward(dH.data_ptr(), pres[l - 1].data_ptr(), dH.numel(),
                                                         nz32.data_ptr(), nz16.data_ptr(), _st()), "silu_backward")
                dZ32, dZ16 = nz32, nz16
        return gW, gb

    def adam(self, gW, gb, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        for l in range(len(self.W)):
            _lib.check(_lib.lib().msgb_adam(self.W[l].data_ptr(), gW[l].data_ptr(), self.mW[l].data_ptr(),
                                            self.vW[l].data_ptr(), self.W[l].numel(), lr, b1, b2, eps,
                                            self.step_count, self.W16[l].data_ptr(), _st()), "adam")
            _lib.check(_lib.lib().msgb_adam(self.b[l].data_ptr(), gb[l].data_ptr(), self.mb[l].data_ptr(),
                                            self.vb[l].data_ptr(), self.b[l].numel(), lr, b1, b2, eps,
                                            self.step_count, None, _st()), "adam")

    def check_tensor_cores(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core wait ran out in msgb_gemm_bf16")

    def train(self, X, Y, epochs: int = 10, batch: int = 8192, lr: float = 1e-3, seed: int = 0,
              lr_min: Optional[float] = None):
        """Minimise the mean squared error of standardised targets.  X (n, in)
        and Y (n, out) FP32 CUDA tensors.  Returns the per-epoch losses."""
        import torch

        n = X.shape[0]
        Xp = torch.zeros((n, IN_PAD), dtype=torch.bfloat16, device=self.device)
        Xp[:, :self.in_dim] = X.to(torch.bfloat16)
        Yp = torch.zeros((n, OUT_PAD), dtype=torch.float32, device=self.device)
        Yp[:, :self.out_dim] = Y
        g = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        total_steps = epochs * max(1, n // batch)
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.device)
            acc = 0.0
            nb = max(1, n // batch)
            for i in range(nb):
                if lr_min is not None:
                    cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * k / max(1, total_steps)))
                else:
                    cur = lr
                idx = perm[i * batch:(i + 1) * batch]
                xb, yb = Xp[idx].contiguous(), Yp[idx]
                out, acts, pres = self.forward(xb, keep=True)
                diff = out - yb
                acc += float((diff[:, :self.out_dim] ** 2).mean())
                dY = (2.0 / (xb.shape[0] * self.out_dim)) * diff
                dY[:, self.out_dim:] = 0.0
                gW, gb = self.backward(dY, acts, pres)
                self.adam(gW, gb, lr=cur)
                k += 1
            losses.append(acc / nb)
        self.check_tensor_cores()
        return losses

    def predict(self, X, batch: int = 1 << 16):
        import torch

        n = X.shape[0]
        out = torch.empty((n, self.out_dim), dtype=torch.float32, device=self.device)
        for s in range(0, n, batch):
            xb = torch.zeros((min(batch, n - s), IN_PAD), dtype=torch.bfloat16, device=self.device)
            xb[:, :self.in_dim] = X[s:s + batch].to(torch.bfloat16)
            out[s:s + batch] = self.forward(xb)[:, :self.out_dim]
        self.check_tensor_cores()
        return out

    def state_dict(self):
        return {"dims": self.dims, "in_dim": self.in_dim, "out_dim": self.out_dim,
                "W": [w.cpu() for w in self.W], "b": [b.cpu() for b in self.b]}
