"""Beam-trajectory surrogate: a BF16 MLP on the tcgen05 tensor cores.

An MLP (``in -> width x depth (SiLU) -> out``; 4 hidden layers of width 256 by
default) maps a beam's launch data and a time to its state, parametrised
relative to the homogeneous solution at the launch speed c(x0):

  inputs  x0 / L, mode * p0/|p0|, log10 w, log10 beta_min, log10 beta_max, t / T
  targets (x(t) - x_hom(t)) / L, (p(t) - p0) / |p0|,
          M(t)^-1 - M_hom(t)^-1 (packed, scaled by |p0| / (c0 T)),
          log A(t) - log A_hom(t)

(M^-1 stays bounded where M itself grows.)  Targets are standardised with
training-set statistics.  Training data are trajectories from
``msgb_ode_trajectories``.  Every matrix product of training and inference
runs in ``msgb_gemm_bf16`` (FP32 accumulation in tensor memory); SiLU
backward, bias gradients (fixed-order column sums) and Adam are libmsgb
kernels too.  PyTorch only allocates buffers and assembles features.

Residual check used to decide whether to trust a prediction: the Hamiltonian
invariant c(x(t)) |p(t)| = c(x0) |p0| (G is homogeneous of degree 1 in p) and
a validated position-error bound; beams that fail are integrated by the ODE.
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

        if in_dim > IN_PAD or out_dim > 2 * OUT_PAD:
            raise ValueError("in_dim must be <= 16 and out_dim <= 32")
        if width % 16 or width > 256:
            raise ValueError("width must be a multiple of 16 <= 256")
        self.in_dim, self.out_dim, self.width, self.depth = in_dim, out_dim, width, depth
        self.out_pad = OUT_PAD if out_dim <= OUT_PAD else 2 * OUT_PAD
        self.dims = [IN_PAD] + [width] * depth + [self.out_pad]
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
        """X16: (B, 16) BF16.  Returns FP32 outputs (B, out_pad) and, with keep, the
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
        Yp = torch.zeros((n, self.out_pad), dtype=torch.float32, device=self.device)
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


def _surrogate_dims(d: int):
    S = d * (d + 1) // 2
    return 3 * d + 2, 2 * d + 2 * S + 2


class TrajectorySurrogate:
    """Learned beam propagation for one heterogeneous medium and time grid.

    ``fit`` integrates a random sample of the solver's beams with the ODE
    integrator (``msgb_ode_trajectories``), trains the MLP on their states at
    every ``t_stride``-th time, and measures on held-out beams the largest
    position error of the predictions (``pos_err``, metres) and of the
    straight-ray homogeneous prediction the network corrects
    (``pos_err_straight``).  ``MSGBSolver(surrogate=...)`` then predicts every
    beam and accepts a beam when its Hamiltonian residual stays below
    ``residual_tol`` at every time and ``w |p0| pos_err`` (the phase error the
    validated position error implies) is below ``phase_tol``; the other beams
    are integrated.  The acceptance rule keeps the forward's accuracy; how many
    beams pass it depends on how well the network fits the medium.
    """

    def __init__(self, width: int = 256, depth: int = 4, residual_tol: float = 1e-4, phase_tol: float = 1e-3,
                 seed: int = 0):
        self.width, self.depth, self.seed = width, depth, seed
        self.residual_tol, self.phase_tol = float(residual_tol), float(phase_tol)
        self.mlp: Optional[MLP] = None
        self.stats: dict = {}
        self.pos_err = float("inf")
        self._key = None

    # ------------------------------------------------------------- helpers
    @staticmethod
    def _sub_beams(bt, idx):
        """Beam tensors of the coefficients idx (both modes follow from them)."""
        sel = lambda a: a.index_select(0, idx).contiguous()
        return type(bt)(sel(bt.x0), sel(bt.p0), sel(bt.alpha), sel(bt.a0), sel(bt.a0_unit), sel(bt.omega))

    @staticmethod
    def _io(nb, b_first, nq_t, t_index, ld):
        return _lib.SurrogateIO(nb=nb, b_first=b_first, nq_t=nq_t,
                                t_index=t_index.data_ptr() if t_index is not None else None, ld=ld)

    def _ode_rec64(self, solver, pr, med, bs, nb):
        import torch

        d = pr.ndim
        R = 2 * d + 2 * d * d + 2
        rec = torch.empty((pr.nt, nb, R), dtype=torch.float64, device=self.device)
        status = torch.zeros(nb, dtype=torch.int32, device=self.device)
        tr = _lib.Trajectories(nb=nb, b_first=0, rec64=rec.data_ptr(), status=status.data_ptr())
        opts = solver._ode_opts(None)
        _lib.check(_lib.lib().msgb_ode_trajectories(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(opts),
                                                    _lib.ref(tr), _st()), "msgb_ode_trajectories")
        return rec, status

    def _predict_rows(self, X16):
        """Standardised predictions for BF16 feature rows, in batches."""
        import torch

        n = X16.shape[0]
        Y = torch.empty((n, self.mlp.out_pad), dtype=torch.float32, device=self.device)
        step = 1 << 18
        for s in range(0, n, step):
            Y[s:s + step] = self.mlp.forward(X16[s:s + step])
        return Y

    @staticmethod
    def medium_key(domain, ts):
        kind, m = domain.medium()
        tsn = np.asarray(ts.detach().cpu().numpy() if hasattr(ts, "detach") else ts, np.float64)
        return (id(m) if kind != "constant" else float(m), float(domain.lam), tsn.size, float(tsn[0]),
                float(tsn[-1]))

    # ---------------------------------------------------------------- fit
    def fit(self, solver, domain, sensors, ts, bt, n_train: int = 2048, n_val: int = 256, t_stride: int = 4,
            epochs: int = 30, batch: int = 8192, lr: float = 2e-3, lr_min: float = 1e-5):
        """Train on ODE trajectories of a sample of ``bt``'s beams (both modes)."""
        import torch

        self.device = bt.x0.device
        dev = self.device
        pr, keep_p = solver._problem(domain, sensors, ts, dev)
        med, keep_m = solver._medium(domain, dev)
        d = pr.ndim
        in_dim, out_dim = _surrogate_dims(d)
        g = torch.Generator(device="cpu").manual_seed(self.seed)
        n = bt.n
        perm = torch.randperm(n, generator=g)
        n_train = min(n_train, max(1, n - min(n_val, n // 4)))
        n_val = min(n_val, n - n_train)
        tr_idx = perm[:n_train].to(dev)
        va_idx = perm[n_train:n_train + n_val].to(dev)
        t_index = torch.arange(0, pr.nt, t_stride, dtype=torch.int32)
        if int(t_index[-1]) != pr.nt - 1:
            t_index = torch.cat([t_index, torch.tensor([pr.nt - 1], dtype=torch.int32)])
        t_index = t_index.to(dev)
        self.mlp = MLP(in_dim, out_dim, self.width, self.depth, device=dev, seed=self.seed)
        ld_y = self.mlp.out_pad

        def data(idx, t_idx):
            sub = self._sub_beams(bt, idx)
            bs = sub.beam_set(unit=True)
            nb = 2 * sub.n
            rec, status = self._ode_rec64(solver, pr, med, bs, nb)
            nq = t_idx.numel() if t_idx is not None else pr.nt
            X = torch.empty((nq * nb, IN_PAD), dtype=torch.bfloat16, device=dev)
            Y = torch.empty((nq * nb, ld_y), dtype=torch.float32, device=dev)
            io = self._io(nb, 0, nq, t_idx, IN_PAD)
            _lib.check(_lib.lib().msgb_surrogate_features(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                          X.data_ptr(), _st()), "msgb_surrogate_features")
            io.ld = ld_y
            _lib.check(_lib.lib().msgb_surrogate_targets(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                         rec.data_ptr(), Y.data_ptr(), _st()),
                       "msgb_surrogate_targets")
            return sub, bs, rec, status, X, Y, (keep_p, keep_m)

        _, _, _, st_tr, Xtr, Ytr, _k = data(tr_idx, t_index)
        if int(st_tr.max().item()) != 0:
            raise RuntimeError("ODE integration failed for training beams")
        Yo = Ytr[:, :out_dim]
        mean = Yo.mean(0)
        std = Yo.std(0)
        std = torch.where(std > 1e-12, std, torch.ones_like(std))
        Ys = (Yo - mean) / std
        self.mean_pad = torch.zeros(ld_y, dtype=torch.float32, device=dev)
        self.std_pad = torch.ones(ld_y, dtype=torch.float32, device=dev)
        self.mean_pad[:out_dim] = mean
        self.std_pad[:out_dim] = std
        losses = self.mlp.train(Xtr[:, :in_dim].float(), Ys, epochs=epochs, batch=batch, lr=lr, seed=self.seed,
                                lr_min=lr_min)
        self.stats = {"train_rows": int(Xtr.shape[0]), "train_beams": 2 * int(tr_idx.numel()),
                      "loss_first": losses[0], "loss_last": losses[-1]}
        self._key = self.medium_key(domain, ts)
        if n_val > 0:
            sub, bs, rec, st_va, X, Y, _k = data(va_idx, None)
            nb = 2 * sub.n
            v = self._validate(pr, med, bs, nb, rec, X, d)
            self.stats.update({"val_beams": nb, **v})
            self.pos_err = v["pos_err"]
        return self

    def _records(self, pr, med, bs, nb, Y, rec64=None, status=None, pos_err=None, mean=None, std=None):
        tr = _lib.Trajectories(nb=nb, b_first=0, rec64=rec64.data_ptr() if rec64 is not None else None,
                               status=status.data_ptr() if status is not None else None)
        acc = _lib.SurrogateAccept(residual_tol=self.residual_tol, phase_tol=self.phase_tol,
                                   pos_err=self.pos_err if pos_err is None else pos_err)
        io = self._io(nb, 0, pr.nt, None, Y.shape[1])
        m = self.mean_pad if mean is None else mean
        s = self.std_pad if std is None else std
        _lib.check(_lib.lib().msgb_surrogate_records(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                     Y.data_ptr(), m.data_ptr(), s.data_ptr(), _lib.ref(acc),
                                                     _lib.ref(tr), _st()), "msgb_surrogate_records")

    def _validate(self, pr, med, bs, nb, rec_true, X, d):
        """Largest and RMS position error (m) of the predictions and of straight
        rays over held-out beams and times, and the fraction of beams whose
        Hamiltonian residual exceeds residual_tol."""
        import torch

        Yp = self._predict_rows(X)
        rec = torch.empty_like(rec_true)
        status = torch.zeros(nb, dtype=torch.int32, device=self.device)
        self._records(pr, med, bs, nb, Yp, rec64=rec, status=status, pos_err=0.0)
        e = (rec[..., :d] - rec_true[..., :d]).norm(dim=-1)
        rej = int((status == 3).sum().item())
        # straight rays: zero correction (mean 0, std 0)
        zero = torch.zeros(Yp.shape[1], dtype=torch.float32, device=self.device)
        rec0 = torch.empty_like(rec_true)
        self._records(pr, med, bs, nb, Yp, rec64=rec0, status=status, pos_err=0.0, mean=zero, std=zero)
        e0 = (rec0[..., :d] - rec_true[..., :d]).norm(dim=-1)
        self.mlp.check_tensor_cores()
        rms = lambda v: float(v.square().mean().sqrt().item())
        return {"pos_err": e.max().item(), "pos_err_straight": e0.max().item(), "pos_rms": rms(e),
                "pos_rms_straight": rms(e0), "val_residual_rejected": rej / max(nb, 1)}

    # ------------------------------------------------------------ predict
    def predict_into(self, pr, med, bs, b_first: int, nb: int, tr):
        """Predict records of beams [b_first, b_first + nb) into ``tr`` (their
        status entries: 0 accepted, 3/4 rejected)."""
        import torch

        acc = _lib.SurrogateAccept(residual_tol=self.residual_tol, phase_tol=self.phase_tol, pos_err=self.pos_err)
        # sub-chunks of beams whose feature and prediction rows fit ~1 GiB
        per_beam = pr.nt * (IN_PAD * 2 + self.mlp.out_pad * 4)
        step = max(1, min(nb, (1 << 30) // max(per_beam, 1)))
        for b0 in range(b_first, b_first + nb, step):
            m = min(step, b_first + nb - b0)
            X = torch.empty((pr.nt * m, IN_PAD), dtype=torch.bfloat16, device=self.device)
            io = self._io(m, b0, pr.nt, None, IN_PAD)
            _lib.check(_lib.lib().msgb_surrogate_features(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                          X.data_ptr(), _st()), "msgb_surrogate_features")
            Y = self._predict_rows(X)
            del X
            io = self._io(m, b0, pr.nt, None, Y.shape[1])
            _lib.check(_lib.lib().msgb_surrogate_records(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                         Y.data_ptr(), self.mean_pad.data_ptr(),
                                                         self.std_pad.data_ptr(), _lib.ref(acc), _lib.ref(tr), _st()),
                       "msgb_surrogate_records")
        self.mlp.check_tensor_cores()
