"""Differentiated reconstruction (the one-sided-sensor inverse problem).

A 128^2 version of the reference workload that runs gradient iterations on
1/2 ||A p0 - d||^2 through the adjoint: a seeded vessel phantom (random-walk
tubes, smoothed), a one-sided line sensor, d = A p_true + 1 % noise.
  * FP32 gradients A_S^T (A_S p - d) (S the frozen beam selection) agree with
    FP64 central finite differences (h = 1e-6) along 16 random directions to
    1e-3;
  * 20 gradient steps from p0 = 0 through the torch.autograd wrapper lower
    the data misfit below half of its starting value.  The beam set is the
    true image's, frozen (as a reconstruction warm-started from a prior
    would use): re-selecting from p0 = 0 picks zero coefficients by index,
    whose beams need not reach a one-sided sensor, and then the gradient is 0.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _phantom(N, n_tubes, seed):
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    img = np.zeros(N)
    yy, xx = np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij")
    for _ in range(n_tubes):
        p = rng.uniform(0.15, 0.85, 2) * np.asarray(N)
        th = rng.uniform(0, 2 * np.pi)
        r = rng.uniform(1.0, 3.0)
        val = rng.uniform(0.5, 1.0)
        for _ in range(40):
            th += rng.normal(0, 0.3)
            p = np.clip(p + 1.5 * np.array([np.cos(th), np.sin(th)]), 0, np.asarray(N) - 1)
            img = np.maximum(img, val * ((yy - p[0]) ** 2 + (xx - p[1]) ** 2 <= r * r))
    return ndimage.gaussian_filter(img, 1.0)


def _setup(thr=2048):
    import beamax_b200 as bb

    N = (128, 128)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(3, N, (4, 8, 16), (1, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()
    hom = bb.gb.gb_solvers.solve_hom_diag
    s32 = bb.MSGBSolver(thr, "top_n", 128, "spatial", hom, "scan_real", precision="fp32")
    s64 = bb.MSGBSolver(thr, "top_n", 128, "spatial", hom, "scan_real", precision="fp64")
    return dom, wpt, sens, ts, s32, s64


def _apply(solver, sel, p, dom, sens, ts, wpt):
    """A_S p: the forward with the beam selection S frozen (linear in p)."""
    return solver.forward_frozen(p, dom, sens, ts, wpt, sel).double()


def test_fp32_gradient_matches_fp64_finite_differences():
    dev = _dev()
    dom, wpt, sens, ts, s32, s64 = _setup()
    p_true = torch.from_numpy(_phantom(dom.N, 12, 0)).to(dev)
    rng = np.random.default_rng(1)
    y = s64.forward(p_true, dom, sens, ts, wpt)
    d = y + 0.01 * float(y.abs().max()) * torch.from_numpy(rng.standard_normal(tuple(y.shape))).to(dev)
    sel = s64.last_selection
    p = 0.5 * p_true + 0.1 * torch.from_numpy(rng.standard_normal(dom.N)).to(dev)
    r32 = _apply(s32, sel, p, dom, sens, ts, wpt) - d
    g32 = s32.adjoint(r32.float(), dom, sens, ts, wpt, selection=sel)

    def f(q):
        r = _apply(s64, sel, q, dom, sens, ts, wpt) - d
        return 0.5 * float((r * r).sum())

    h = 1e-6
    fd, an = [], []
    for k in range(16):
        v = torch.from_numpy(np.random.default_rng(100 + k).standard_normal(dom.N)).to(dev)
        fd.append((f(p + h * v) - f(p - h * v)) / (2 * h))
        an.append(float((g32 * v).sum()))
    fd, an = np.asarray(fd), np.asarray(an)
    assert np.linalg.norm(an - fd) <= 1e-3 * np.linalg.norm(fd)


def test_twenty_gradient_steps_through_autograd_reduce_misfit():
    from beamax_b200.solvers.autograd import msgb_forward

    dev = _dev()
    dom, wpt, sens, ts, s32, s64 = _setup()
    p_true = torch.from_numpy(_phantom(dom.N, 12, 3)).to(dev)
    rng = np.random.default_rng(4)
    y = s64.forward(p_true, dom, sens, ts, wpt)
    d = (y + 0.01 * float(y.abs().max()) * torch.from_numpy(rng.standard_normal(tuple(y.shape))).to(dev)).float()
    sel = s64.last_selection
    # step 1 / L, L = ||A_S||^2 by power iteration on the frozen operator
    v = torch.from_numpy(rng.standard_normal(dom.N)).to(dev)
    for _ in range(8):
        w = s32.adjoint(_apply(s32, sel, v, dom, sens, ts, wpt).float(), dom, sens, ts, wpt, selection=sel)
        lam = float(torch.linalg.norm(w))
        v = w / lam
    step = 1.0 / lam
    p = torch.zeros(dom.N, dtype=torch.float64, device=dev, requires_grad=True)
    losses = []
    for _ in range(20):
        out = msgb_forward(p, s32, dom, sens, ts, wpt, selection=sel)
        loss = 0.5 * ((out - d) ** 2).sum()
        losses.append(float(loss))
        (g,) = torch.autograd.grad(loss, p)
        with torch.no_grad():
            p -= step * g
    print("misfit", losses[0], losses[-1])
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0]
