"""Differentiated reconstruction at the configuration-4 size (B200).

512 x 512 grid, dx = 1e-4 m, homogeneous c = 1500 m/s, 4 levels (4, 8, 16,
32), redundancy 2; one-sided line sensor on the first row (512 points);
ground truth: a seeded vessel phantom of 30 random-walk tubes (radius 1-4
cells, intensity U(0.5, 1)) smoothed with sigma = 1 cell; data
d = A p_true + 1 % Gaussian noise.

Beam-set policy (p0 = 0 ties every coefficient at 0, so the selection of the
iterate is meaningless there): the set is chosen once from the data, as the
top_n (65,536) coefficients of q = A_H^T d, the exact transpose over the full
half frame H (524,288 coefficients, 1,048,576 beams), and then frozen, so
the iterations minimise 1/2 ||A_S p - d||^2, a quadratic.
  * FP32 gradients A_S^T (A_S p - d) agree with FP64 central finite
    differences (h = 1e-6) along 16 random directions to 1e-3 relative;
  * 20 gradient steps from p = 0 through the torch.autograd wrapper (step 1/L,
    L = ||A_S||^2 by power iteration) lower the misfit below half its start.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def vessel_phantom(N, n_tubes=30, seed=0):
    """Random-walk tubes (radius U(1, 4) cells, intensity U(0.5, 1)), sigma = 1 smoothing."""
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    img = np.zeros(N)
    for _ in range(n_tubes):
        p = rng.uniform(0.1, 0.9, 2) * np.asarray(N)
        th = rng.uniform(0, 2 * np.pi)
        r = rng.uniform(1.0, 4.0)
        val = rng.uniform(0.5, 1.0)
        for _ in range(int(rng.integers(40, 120))):
            th += rng.normal(0, 0.25)
            p = np.clip(p + 1.5 * np.array([np.cos(th), np.sin(th)]), 0, np.asarray(N) - 1)
            lo = np.maximum(np.floor(p - r).astype(int), 0)
            hi = np.minimum(np.ceil(p + r).astype(int) + 1, N)
            yy, xx = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), indexing="ij")
            blob = (yy - p[0]) ** 2 + (xx - p[1]) ** 2 <= r * r
            sub = img[lo[0]:hi[0], lo[1]:hi[1]]
            img[lo[0]:hi[0], lo[1]:hi[1]] = np.maximum(sub, val * blob)
    return ndimage.gaussian_filter(img, 1.0)


def test_config4_gradients_and_twenty_iterations():
    import beamax_b200 as bb
    from beamax_b200.solvers.autograd import msgb_forward
    from beamax_b200.solvers.msgb_solver import Selection

    dev = _dev()
    N = (512, 512)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(4, N, (4, 8, 16, 32), (1, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()
    hom = bb.gb.gb_solvers.solve_hom_diag
    thr = 65536
    s32 = bb.MSGBSolver(thr, "top_n", 128, "spatial", hom, "scan_real", precision="fp32")
    s64 = bb.MSGBSolver(thr, "top_n", 128, "spatial", hom, "scan_real", precision="fp64")
    rng = np.random.default_rng(4)

    p_true = torch.from_numpy(vessel_phantom(N, 30, 0)).to(dev)
    y = s32.forward(p_true, dom, sens, ts, wpt).double()
    assert tuple(y.shape) == (ts.size, 512)
    d = (y + 0.01 * float(y.abs().max()) * torch.from_numpy(rng.standard_normal(tuple(y.shape))).to(dev))

    # beam set from the data: top_n of MSWPT(A_H^T d), H the full half frame
    half = torch.from_numpy(np.flatnonzero(np.asarray(wpt._half_mask).ravel())).to(dev)
    full = Selection(half, torch.zeros(half.numel(), dtype=torch.complex128, device=dev), wpt.total_coeffs)
    q = s32.adjoint(d.float(), dom, sens, ts, wpt, selection=full)
    sel = s32.select(q, dom, wpt)
    assert int(sel.idx.numel()) == thr

    def apply(solver, p):
        return solver.forward_frozen(p, dom, sens, ts, wpt, sel).double()

    # FP32 gradient against FP64 central differences
    p = 0.5 * q / float(q.abs().max()) + 0.1 * torch.from_numpy(rng.standard_normal(N)).to(dev)
    g32 = s32.adjoint((apply(s32, p) - d).float(), dom, sens, ts, wpt, selection=sel)

    def f(x):
        r = apply(s64, x) - d
        return 0.5 * float((r * r).sum())

    h = 1e-6
    fd, an = [], []
    for k in range(16):
        v = torch.from_numpy(np.random.default_rng(100 + k).standard_normal(N)).to(dev)
        fd.append((f(p + h * v) - f(p - h * v)) / (2 * h))
        an.append(float((g32 * v).sum()))
    fd, an = np.asarray(fd), np.asarray(an)
    assert np.linalg.norm(an - fd) <= 1e-3 * np.linalg.norm(fd)

    # 20 gradient steps from 0 through autograd
    v = torch.from_numpy(rng.standard_normal(N)).to(dev)
    for _ in range(8):
        w = s32.adjoint(apply(s32, v).float(), dom, sens, ts, wpt, selection=sel)
        lam = float(torch.linalg.norm(w))
        v = w / lam
    step = 1.0 / lam
    x = torch.zeros(N, dtype=torch.float64, device=dev, requires_grad=True)
    losses = []
    for _ in range(20):
        out = msgb_forward(x, s32, dom, sens, ts, wpt, selection=sel)
        loss = 0.5 * ((out.double() - d) ** 2).sum()
        losses.append(float(loss.detach()))
        (g,) = torch.autograd.grad(loss, x)
        with torch.no_grad():
            x -= step * g
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses
