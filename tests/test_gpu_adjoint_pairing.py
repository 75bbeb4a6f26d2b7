"""The exact transpose against the reference's principal-symbol adjoint (B200).

Restates the controlled pairing diagnostic of the reference
(examples/diagnostics/msgb_adjoint_pairing.py): a one-sided planar detector,
a smooth high-frequency packet, a sin^2 acquisition taper.  Two different
operators are compared:

* the exact discrete transpose B^T of the windowed forward B f = w * P f
  (the VJP with the top-N set frozen, :156-165) -- its dot-product residual is
  at round-off;
* the principal-symbol continuous adjoint (``adjoint`` with sources,
  data_domain and data_wpt, msgb_solver.py:1235-1386) -- an approximation of
  (dt / dx) B^T, compared by cosine and best-scaled relative error with the
  reference's own ``_fit`` (:62-73), and against the D'Alembert references
  (:189-199) in 1D.

Stated floors (measured on a B200, see the assertions): 1D cosine >= 0.99,
best-scaled error <= 0.1; 2D (64 x 64, detector on the first row) cosine >=
0.9.  They are properties of the approximation, not tolerances of the kernels.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def fit(reference, candidate):
    """msgb_adjoint_pairing.py:62-73: candidate scale, best-scaled error, cosine."""
    eps = np.finfo(float).eps
    reference, candidate = np.ravel(reference), np.ravel(candidate)
    ref_norm, cand_norm = np.linalg.norm(reference), np.linalg.norm(candidate)
    dot = float(np.vdot(candidate, reference).real)
    scale = dot / max(cand_norm ** 2, eps)
    error = float(np.linalg.norm(scale * candidate - reference) / max(ref_norm, eps))
    return scale, error, dot / max(cand_norm * ref_norm, eps)


def packet(x, centre, width, cycles):
    return np.exp(-0.5 * ((x - centre) / width) ** 2) * np.cos(2.0 * np.pi * cycles * (x - centre))


def pairing_1d(n=128, cycles=24.0, top_n=32, speed=1.0):
    """The diagnostic's own case; returns its figures."""
    import beamax_b200 as bb

    gs = bb.gb.gb_solvers
    dx = 1.0 / n
    nt = n
    dt = 1.0 / (speed * nt)
    dom = bb.Domain(N=(n,), dx=(dx,), c=speed, cfl=0.3, periodic=(False,))
    image_wpt = bb.MSWPT(bb.DyadicDecomposition(2, (n,), (4, 8), (1,)), 2, "rectangular")
    ts = np.arange(nt, dtype=np.float64) * dt
    ddom = bb.Domain(N=(nt,), dx=(dt,), c=speed, cfl=0.3, periodic=(False,))
    data_wpt = bb.MSWPT(bb.DyadicDecomposition(2, (nt,), (4, 8), (1,)), 2, "rectangular_mirror")
    mask = np.zeros(n)
    mask[0] = 1.0
    boundary = bb.Sensor(dom, binary_mask=mask)
    image_grid = bb.Sensor(dom, binary_mask=np.ones(n))
    solver = bb.MSGBSolver(top_n, "top_n", 32, "spatial", gs.solve_ODE_base, "all_real",
                           tr_ode_solver=gs.solve_ODE_batch_t)
    x = np.asarray(dom.grid)[..., 0]
    f = packet(x, 0.58, 0.075, cycles)
    window = np.sin(np.pi * np.arange(nt) / (nt - 1)) ** 2
    pf = np.ravel(solver.forward(f, dom, boundary, ts, image_wpt))
    bf = window * pf
    y = pf
    exact = np.ravel(solver.adjoint((window * y).reshape(nt, 1), dom, boundary, ts, image_wpt))
    principal = np.ravel(solver.adjoint(y, dom, image_grid, boundary, ts, ddom, data_wpt, window=window))
    lhs = dt * float(np.vdot(bf, y).real)
    rhs_exact = dt * float(np.vdot(f, exact).real)
    rhs_principal = dx * float(np.vdot(f, principal).real)
    scale, err, cos = fit((dt / dx) * exact, principal)
    _, fwd_err, fwd_cos = fit(0.5 * packet(speed * ts, 0.58, 0.075, cycles), pf)
    _, adj_err, adj_cos = fit(0.5 * window * y / speed, principal)
    return dict(exact_residual=abs(lhs - rhs_exact) / abs(lhs), principal_residual=abs(lhs - rhs_principal) / abs(lhs),
                scale=scale, best_scaled_error=err, cosine=cos, dalembert_forward=(fwd_err, fwd_cos),
                dalembert_adjoint=(adj_err, adj_cos))


def pairing_2d(N=(64, 64), dx=1e-4, c=1500.0, top_n=600, seed=0):
    """A 2D one-sided planar detector (first row), packets heading towards it."""
    import beamax_b200 as bb

    gs = bb.gb.gb_solvers
    dom = bb.Domain(N=N, dx=(dx, dx), c=c, cfl=0.3, periodic=(False, False))
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular")
    T = float(dom.generate_time_domain()[-1])
    nt = 2 * N[0]
    dt = T / (nt - 1)
    ts = np.arange(nt) * dt
    ddom = bb.Domain(N=(nt, N[1]), dx=(dt, dx), c=c, cfl=0.3, periodic=(False, False))
    dwpt = bb.MSWPT(bb.DyadicDecomposition(2, (nt, N[1]), (4, 8), (2, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = 1.0
    boundary = bb.Sensor(dom, binary_mask=mask)
    image_grid = bb.Sensor(dom, binary_mask=np.ones(N))
    solver = bb.MSGBSolver(top_n, "top_n", 64, "spatial", gs.solve_ODE_base, "all_real",
                           tr_ode_solver=gs.solve_ODE_batch_t)
    rng = np.random.default_rng(seed)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    f = np.zeros(N)
    for _ in range(4):
        cen = np.array([rng.uniform(0.3, 0.7) * N[0], rng.uniform(0.3, 0.7) * N[1]])
        th = np.pi + rng.uniform(-0.4, 0.4)  # towards the detector row
        r = xg - cen
        f += np.exp(-np.sum(r * r, -1) / (2 * 4.0 ** 2)) * np.cos(2 * np.pi * 0.2 * (r @ [np.cos(th), np.sin(th)]))
    window = np.sin(np.pi * np.arange(nt) / (nt - 1)) ** 2
    pf = solver.forward(f, dom, boundary, ts, wpt)
    exact = solver.adjoint(window[:, None] * pf, dom, boundary, ts, wpt)
    principal = solver.adjoint(pf, dom, image_grid, boundary, ts, ddom, dwpt, window=window)
    lhs = float(np.sum(window[:, None] * pf * pf))
    rhs = float(np.sum(f * exact))
    scale, err, cos = fit(exact, principal)
    return dict(exact_residual=abs(lhs - rhs) / abs(lhs), scale=scale, best_scaled_error=err, cosine=cos)


def test_exact_transpose_and_principal_adjoint_pairing_1d():
    _dev()
    r = pairing_1d()
    assert r["exact_residual"] <= 1e-12
    assert r["cosine"] >= 0.99 and r["best_scaled_error"] <= 0.1, r
    assert r["dalembert_forward"][1] >= 0.99 and r["dalembert_adjoint"][1] >= 0.99, r


def test_exact_transpose_and_principal_adjoint_pairing_2d_planar():
    _dev()
    r = pairing_2d()
    assert r["exact_residual"] <= 1e-11
    assert r["cosine"] >= 0.9, r
