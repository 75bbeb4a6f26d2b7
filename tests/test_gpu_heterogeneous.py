"""GPU parity of the heterogeneous-medium path (beam ODE, trajectory sums).

Oracles: the oracle's own RK4 and Dormand-Prince 5(4) of coupled_rhs_absorption
(gb/gb_solvers.py:820-867), the same methods with the same step control, for
implementation parity; SciPy DOP853 at rtol = atol = 1e-12 (the reference
test's own oracle, tests/test_gb.py:759-849) for the methods' accuracy.
Tolerances: GPU RK4 equal to the oracle RK4 to round-off and the adaptive
integrator to 1e-9 (1e-5 / 1e-4 with the continuous extension, where step
decisions can flip); against DOP853 rays within 1e-8, M within 1e-4 at the
default rtol 1e-7 (1e-6 at rtol 1e-10), fixed-step M converging at second
order; the FP64 forward within 1e-7 rel-L2 of the oracle sum over oracle
trajectories; FP32 within 1e-3 of FP64; the transpose's dot test at 1e-10.
"""

import ctypes

import numpy as np
import pytest

from oracle import msgb as om
from oracle import ode as oo

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _rk4_states(ndim, x0, p0, alpha, ts, medium, L, periodic=None, substeps=1, ode=None, status=False):
    """Run msgb_ode_trajectories (RK4 with `substeps`, or the given options)
    for beams (positive and negative modes); return rec64 (nt, 2n, R)."""
    from beamax_b200 import _lib

    dev = _dev()
    n = x0.shape[0]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    tsd = T(np.asarray(ts, float))
    sens = T(np.zeros((1, ndim)))
    pr = _lib.Problem(ndim=ndim, c=1.0, nt=len(ts), ts=tsd.data_ptr(), ns=1, sensors=sens.data_ptr())
    for a in range(3):
        pr.L[a] = L[a] if a < ndim else 1.0
        pr.periodic[a] = int(periodic[a]) if periodic is not None and a < ndim else 0
    x0d, p0d = T(x0), T(p0)
    ald = T(np.ascontiguousarray(alpha, np.complex128).view(np.float64))
    a0d = T(np.ones(2 * n))
    om_ = T(np.ones(n))
    bs = _lib.BeamSet(n=n, x0=x0d.data_ptr(), p0=p0d.data_ptr(), alpha=ald.data_ptr(), a0=a0d.data_ptr(),
                      omega=om_.data_ptr())
    R = 2 * ndim + 2 * ndim * ndim + 2
    rec = torch.zeros((len(ts), 2 * n, R), dtype=torch.float64, device=dev)
    stat = torch.full((2 * n,), -1, dtype=torch.int32, device=dev)
    tr = _lib.Trajectories(nb=2 * n, b_first=0, rec64=rec.data_ptr(), status=stat.data_ptr())
    med, keep = medium
    if ode is None:
        ode = _lib.OdeOpts(method=0, substeps=substeps)
    _lib.check(_lib.lib().msgb_ode_trajectories(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(ode),
                                                _lib.ref(tr), torch.cuda.current_stream().cuda_stream), "ode")
    torch.cuda.synchronize()
    if status:
        return rec.cpu().numpy(), stat.cpu().numpy()
    assert (stat.cpu().numpy() == 0).all()
    return rec.cpu().numpy()


def _dopri(rtol=1e-7, atol=1e-9, max_steps=4096, dense=False):
    from beamax_b200 import _lib

    return _lib.OdeOpts(method=1, substeps=1, rtol=rtol, atol=atol, dt0=0.0, max_steps=max_steps,
                        dense_output=int(dense))


def _grid_medium(interp):
    from beamax_b200 import _lib
    from beamax_b200.utils.interp import BOUNDARY_CODE

    dev = _dev()
    med = _lib.Medium()
    med.kind = 1 if interp.method == "linear" else 2
    med.boundary = BOUNDARY_CODE[interp.boundary]
    for a in range(3):
        med.n[a] = interp.coeffs.shape[a] if a < interp.ndim else 1
        med.spacing[a] = interp.spacing[a] if a < interp.ndim else 1.0
        med.origin[a] = interp.origin[a] if a < interp.ndim else 0.0
    c = torch.from_numpy(interp.coeffs).to(dev)
    med.coeffs = c.data_ptr()
    return med, c


def _random_medium(N, dx, amp, corr, seed, method="bspline3"):
    from scipy import ndimage

    from beamax_b200.utils.interp import make_c_function_from_grid

    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(N), corr, mode="wrap")
    g = np.clip(g / np.max(np.abs(g)), -1, 1)
    c = 1500.0 * (1 + amp * g)
    return c, make_c_function_from_grid(c, dx, method=method, boundary="clamp")


def _unpack(rec, d):
    x = rec[..., :d]
    p = rec[..., d:2 * d]
    M = (rec[..., 2 * d:2 * d + 2 * d * d:2] + 1j * rec[..., 2 * d + 1:2 * d + 2 * d * d:2]).reshape(rec.shape[:-1] + (d, d))
    A = rec[..., -2] + 1j * rec[..., -1]
    return x, p, M, A


def _beams3(seed=1):
    rng = np.random.default_rng(seed)
    n = 3
    x0 = rng.uniform(0.25, 0.75, (n, 2)) * 64e-4
    th = rng.uniform(0, 2 * np.pi, n)
    p0 = 2 * np.pi * np.stack([np.cos(th), np.sin(th)], 1)
    alpha = 1j * rng.uniform(0.5, 2.0, (n, 2)) * 1e-3
    return n, x0, p0, alpha


def test_rk4_matches_oracle_rk4_in_sharp_bspline_medium():
    """GPU RK4 == the oracle's RK4 (same method, FP64) to round-off, in a
    6-cell-correlation medium where the C^2 cubic B-spline makes hess c kinked."""
    N, dx = (64, 64), (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.1, 6.0, 3)
    n, x0, p0, alpha = _beams3()
    ts = np.arange(0, 80) * 2e-8
    speed = oo.GridSpeed(c, dx, method="bspline3", boundary="clamp")
    rec = _rk4_states(2, x0, p0, alpha, ts, _grid_medium(interp), (64e-4, 64e-4), substeps=2)
    for b in range(2 * n):
        j, mode = b % n, (1.0 if b < n else -1.0)
        ox, op, oM, oA = oo.rk4(x0[j], p0[j], np.diag(alpha[j]), 1.0, mode, ts, speed, substeps=2)
        gx, gp, gM, gA = _unpack(rec[:, b], 2)
        assert np.max(np.abs(gx - ox)) <= 1e-12 * np.max(np.abs(ox))
        assert np.max(np.abs(gp - op)) <= 1e-12 * np.max(np.abs(op))
        assert np.max(np.abs(gM - oM)) <= 1e-10 * np.max(np.abs(oM))
        assert np.max(np.abs(gA - oA)) <= 1e-10 * np.max(np.abs(oA))


def test_rk4_converges_to_dop853_in_smooth_bspline_medium():
    """Fixed-step accuracy against DOP853 at rtol = atol = 1e-12 in a
    16-cell-correlation medium.  Rays agree to 1e-8 and amplitudes to 1e-6.
    The Hessian of a cubic B-spline is continuous but kinked at every knot,
    so with fixed steps the Riccati variable M converges only at second order:
    within 1e-3 at 2 substeps, 1e-4 at 8."""
    N, dx = (64, 64), (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.1, 16.0, 5)
    n, x0, p0, alpha = _beams3(2)
    ts = np.arange(0, 80) * 2e-8
    speed = oo.GridSpeed(c, dx, method="bspline3", boundary="clamp")
    med = _grid_medium(interp)
    recs = {s: _rk4_states(2, x0, p0, alpha, ts, med, (64e-4, 64e-4), substeps=s) for s in (2, 8)}
    for b in range(2 * n):
        j, mode = b % n, (1.0 if b < n else -1.0)
        xt, pt, Mt, At = oo.solve(x0[j], p0[j], np.diag(alpha[j]), 1.0, mode, ts, speed)
        for s, tol_m in ((2, 1e-3), (8, 1e-4)):
            gx, gp, gM, gA = _unpack(recs[s][:, b], 2)
            assert np.max(np.abs(gx - xt)) <= 1e-8 * np.max(np.abs(xt))
            assert np.max(np.abs(gp - pt)) <= 1e-7 * np.max(np.abs(pt))
            assert np.max(np.abs(gM - Mt)) <= tol_m * np.max(np.abs(Mt))
            assert np.max(np.abs(gA - At)) <= 1e-6 * np.max(np.abs(At))


def test_dopri5_matches_oracle_dopri5_in_sharp_bspline_medium():
    """Adaptive integrator == the oracle's Dormand-Prince 5(4) with the same
    step control (default tolerances).  Steps ending on the save times: equal
    to 1e-9.  Continuous extension: steps are longer and a round-off flip of
    one accept/reject decision changes the step sequence, after which the
    solutions agree to the tolerance: rays 1e-5, M and A 1e-4."""
    N, dx = (64, 64), (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.1, 6.0, 3)
    n, x0, p0, alpha = _beams3()
    ts = np.arange(0, 80) * 2e-8
    speed = oo.GridSpeed(c, dx, method="bspline3", boundary="clamp")
    med = _grid_medium(interp)
    for dense, tol, tol_m in ((False, 1e-9, 1e-9), (True, 1e-5, 1e-4)):
        rec = _rk4_states(2, x0, p0, alpha, ts, med, (64e-4, 64e-4), ode=_dopri(dense=dense))
        for b in range(2 * n):
            j, mode = b % n, (1.0 if b < n else -1.0)
            ox, op, oM, oA, st, steps = oo.dopri5(x0[j], p0[j], np.diag(alpha[j]), 1.0, mode, ts, speed, dense=dense)
            assert st == 0
            gx, gp, gM, gA = _unpack(rec[:, b], 2)
            assert np.max(np.abs(gx - ox)) <= tol * np.max(np.abs(ox))
            assert np.max(np.abs(gp - op)) <= tol * np.max(np.abs(op))
            assert np.max(np.abs(gM - oM)) <= tol_m * np.max(np.abs(oM))
            assert np.max(np.abs(gA - oA)) <= tol_m * np.max(np.abs(oA))


def test_dopri5_accuracy_against_dop853():
    """The adaptive integrator's global error against DOP853 at 1e-12 (steps
    ending on the save times): at the reference's default rtol 1e-7 / atol
    1e-9 rays within 1e-8 and M within 1e-4; at rtol 1e-10 / atol 1e-12, M
    within 1e-6 (it converges with the tolerance, unlike fixed steps)."""
    N, dx = (64, 64), (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.1, 16.0, 5)
    n, x0, p0, alpha = _beams3(2)
    ts = np.arange(0, 80) * 2e-8
    speed = oo.GridSpeed(c, dx, method="bspline3", boundary="clamp")
    med = _grid_medium(interp)
    loose = _rk4_states(2, x0, p0, alpha, ts, med, (64e-4, 64e-4), ode=_dopri())
    tight = _rk4_states(2, x0, p0, alpha, ts, med, (64e-4, 64e-4), ode=_dopri(1e-10, 1e-12, 100000))
    for b in range(2 * n):
        j, mode = b % n, (1.0 if b < n else -1.0)
        xt, pt, Mt, At = oo.solve(x0[j], p0[j], np.diag(alpha[j]), 1.0, mode, ts, speed)
        for rec, tol_m in ((loose, 1e-4), (tight, 1e-6)):
            gx, gp, gM, gA = _unpack(rec[:, b], 2)
            assert np.max(np.abs(gx - xt)) <= 1e-8 * np.max(np.abs(xt))
            assert np.max(np.abs(gp - pt)) <= 1e-8 * np.max(np.abs(pt))
            assert np.max(np.abs(gM - Mt)) <= tol_m * np.max(np.abs(Mt))
            assert np.max(np.abs(gA - At)) <= 1e-6 * np.max(np.abs(At))


def test_dopri5_step_budget_reports_status_and_solver_raises():
    """max_steps counts accepted and rejected steps (with the continuous
    extension; ending steps on the save times adds nt - 1); running out leaves
    status 2 (the host raises, as diffeqsolve does)."""
    import beamax_b200 as bb

    N, dx = (64, 64), (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.1, 6.0, 3)
    n, x0, p0, alpha = _beams3()
    ts = np.arange(0, 80) * 2e-8
    rec, stat = _rk4_states(2, x0, p0, alpha, ts, _grid_medium(interp), (64e-4, 64e-4),
                            ode=_dopri(max_steps=10, dense=True), status=True)
    assert (stat == 2).all()
    assert np.isfinite(rec).all()
    dom, wpt, p0g, sens, tsg, c2, interp2, thr = _het_case(thr=4)
    cfg = bb.gb.gb_solvers.SolverConfig(max_steps=3, dense_output=True)
    solver = bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real", ode_config=cfg)
    with pytest.raises(RuntimeError, match="max_steps"):
        solver.forward(p0g, dom, sens, tsg, wpt)


def test_rk4_1d_linear_medium_matches_closed_form():
    """tests/test_gb.py:669-756: c = a + b x, linear interpolation reproduces it exactly."""
    from beamax_b200.utils.interp import make_c_function_from_grid

    a, b = 1.0, 1.0
    xs = np.arange(0, 400) * 0.01
    interp = make_c_function_from_grid(a + b * xs, (0.01,), method="linear", boundary="clamp")
    ts = np.linspace(0.0, 1.0, 200)
    rec = _rk4_states(1, np.array([[0.1]]), np.array([[1.2]]), np.array([[0.2j]]), ts, _grid_medium(interp), (4.0,),
                      substeps=4)
    x, p, M, A = _unpack(rec[:, 0], 1)
    xr, pr_, Mr, Ar = oo.analytic_1d_linear(0.1, 1.2, 0.2j, 1.0, ts, a, b)
    assert np.allclose(x[:, 0], xr, atol=1e-10, rtol=1e-7)
    assert np.allclose(p[:, 0], pr_, atol=1e-10, rtol=1e-7)
    assert np.allclose(M[:, 0, 0], Mr, atol=1e-10, rtol=1e-7)
    assert np.allclose(A, Ar, atol=1e-10, rtol=1e-7)


def test_rk4_constant_medium_matches_closed_form():
    """solve_ODE_base == solve_hom_diag in a homogeneous medium (tests/test_gb.py:155-171)."""
    from beamax_b200 import _lib

    rng = np.random.default_rng(2)
    n = 4
    x0 = rng.uniform(0, 1e-2, (n, 2))
    th = rng.uniform(0, 2 * np.pi, n)
    p0 = 2 * np.pi * np.stack([np.cos(th), np.sin(th)], 1)
    alpha = 1j * rng.uniform(0.5, 2.0, (n, 2)) * 1e-3
    ts = np.arange(0, 50) * 2e-8
    med = _lib.Medium(kind=0, c=1500.0)
    rec = _rk4_states(2, x0, p0, alpha, ts, (med, None), (1e-2, 1e-2))
    M0 = np.einsum("bd,dj->bdj", alpha, np.eye(2))
    modes = np.r_[np.ones(n), -np.ones(n)]
    xt, pt, Mt, At = om.solve_hom_diag(np.r_[x0, x0], np.r_[p0, p0], np.r_[M0, M0], np.ones(2 * n), modes, ts, 1500.0)
    gx, gp, gM, gA = _unpack(np.moveaxis(rec, 0, 1), 2)
    assert np.max(np.abs(gx - xt)) <= 1e-12 * np.max(np.abs(xt))
    assert np.max(np.abs(gM - Mt)) <= 1e-9 * np.max(np.abs(Mt))
    assert np.max(np.abs(gA - At[..., 0])) <= 1e-9


def _het_case(seed=0, N=(64, 64), thr=24):
    import beamax_b200 as bb

    dx = (1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.08, 5.0, seed)
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=interp)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(seed)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - 32) ** 2, -1) / 40.0) * np.cos(0.9 * xg[..., 0]) + 0.3 * rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::3]
    return dom, wpt, p0, sens, ts, c, interp, thr


def test_heterogeneous_forward_fp64_matches_oracle():
    """GPU FP64 forward (adaptive ODE + dense sum) == the oracle's Dormand-Prince
    trajectories summed with the oracle's summation (gb/core.py:194-329), to
    1e-7 rel-L2 (the phase multiplies position round-off by w |p|)."""
    import beamax_b200 as bb

    _dev()
    dom, wpt, p0, sens, ts, c, interp, thr = _het_case(thr=12)
    solver = bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real")
    out = solver.forward(p0, dom, sens, ts, wpt)
    bt = solver.beams(solver.last_selection, dom, wpt)
    x0, p0s = bt.x0.cpu().numpy(), bt.p0.cpu().numpy()
    al, a0, w = bt.alpha.cpu().numpy(), bt.a0.cpu().numpy(), bt.omega.cpu().numpy()
    speed = oo.GridSpeed(c, dom.dx, method="bspline3", boundary="clamp")
    ref = np.zeros_like(out)
    for j in range(x0.shape[0]):
        for mode in (1.0, -1.0):
            xt, pt, Mt, At, st, _ = oo.dopri5(x0[j], p0s[j], np.diag(al[j]), a0[j], mode, ts, speed)
            assert st == 0
            ref += oo.beam_field(xt, pt, Mt, At, w[j], sens.positions, dom.grid_size, dom.periodic)
    assert om.rel_l2(ref, out) < 1e-7


def test_heterogeneous_fp32_and_adjoint_dot_test():
    import beamax_b200 as bb
    from beamax_b200.solvers.msgb_solver import Selection

    dev = _dev()
    dom, wpt, p0, sens, ts, c, interp, thr = _het_case(seed=1, N=(128, 128), thr=400)
    s64 = bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real")
    s32 = bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real",
                        precision="fp32", trajectory_memory=64 << 20)  # forces several chunks
    y64 = s64.forward(p0, dom, sens, ts, wpt)
    y32 = s32.forward(p0, dom, sens, ts, wpt)
    assert om.rel_l2(y64, y32) < 1e-3
    sel = s64.last_selection
    data = np.random.default_rng(3).standard_normal(y64.shape)
    a64 = s64.adjoint(data, dom, sens, ts, wpt, selection=sel)
    a32 = s32.adjoint(data, dom, sens, ts, wpt, selection=sel)
    assert om.rel_l2(a64, a32) < 1e-3
    q = np.random.default_rng(4).standard_normal(dom.N)
    cq = wpt.forward_device(torch.from_numpy(q).to(dev), scale=0.5, half_mask=True)
    selq = Selection(sel.idx, cq[sel.idx], sel.total_coeffs)
    Aq = s64.sum_forward(s64.beams(selq, dom, wpt), dom, sens, ts).cpu().numpy()
    lhs, rhs = float(np.sum(Aq * data)), float(np.sum(q * a64))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_adjoint_reuses_forward_trajectories():
    """An adjoint right after the forward (same selection, domain and time
    grid) reads the kept trajectory records instead of integrating again; the
    result equals the re-integrating adjoint's."""
    import beamax_b200 as bb

    _dev()
    dom, wpt, p0, sens, ts, c, interp, thr = _het_case(seed=2, N=(64, 64), thr=60)
    ode = bb.gb.gb_solvers.solve_ODE_base
    for precision in ("fp64", "fp32"):
        keep = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", precision=precision)
        fresh = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", precision=precision,
                              keep_trajectories=False)
        y = keep.forward(p0, dom, sens, ts, wpt)
        fresh.forward(p0, dom, sens, ts, wpt)
        assert keep._cached_trajectories(keep.last_selection, dom, ts) is not None
        assert fresh._cached_trajectories(fresh.last_selection, dom, ts) is None
        data = np.random.default_rng(9).standard_normal(y.shape)
        a_keep = keep.adjoint(data, dom, sens, ts, wpt)
        a_fresh = fresh.adjoint(data, dom, sens, ts, wpt)
        assert om.rel_l2(a_fresh, a_keep) < (1e-12 if precision == "fp64" else 1e-6)


def test_adjoint_reuses_the_last_chunk_of_forward_trajectories():
    """Records larger than trajectory_memory are integrated in chunks; the
    adjoint reads the kept last chunk and integrates the others, with the
    result of the adjoint that integrates every chunk."""
    import beamax_b200 as bb

    _dev()
    dom, wpt, p0, sens, ts, c, interp, thr = _het_case(seed=2, N=(64, 64), thr=60)
    ode = bb.gb.gb_solvers.solve_ODE_base
    for precision in ("fp64", "fp32"):
        kw = dict(precision=precision, trajectory_memory=256 << 10)
        keep = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", **kw)
        fresh = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", keep_trajectories=False, **kw)
        y = keep.forward(p0, dom, sens, ts, wpt)
        fresh.forward(p0, dom, sens, ts, wpt)
        cached = keep._cached_trajectories(keep.last_selection, dom, ts)
        assert cached is not None and 0 < cached["tr"].nb < 2 * keep.last_selection.idx.shape[0]
        data = np.random.default_rng(9).standard_normal(y.shape)
        a_keep = keep.adjoint(data, dom, sens, ts, wpt)
        a_fresh = fresh.adjoint(data, dom, sens, ts, wpt)
        assert om.rel_l2(a_fresh, a_keep) < (1e-12 if precision == "fp64" else 1e-6)


def _het3d_case(thr):
    import beamax_b200 as bb

    N, dx = (32, 32, 32), (1e-4, 1e-4, 1e-4)
    c, interp = _random_medium(N, dx, 0.05, 4.0, 21)
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False, False), cfl=0.3, c=interp)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1, 1)), 2, "rectangular_mirror")
    xg = np.stack(np.meshgrid(*[np.arange(n) for n in N], indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - 15.0) ** 2, -1) / 20.0) * np.cos(0.8 * xg[..., 2])
    mask = np.zeros(N)
    mask[:, :, 0] = 1  # planar sensor on the z = 0 face
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::2]
    return dom, wpt, p0, sens, ts, c


def test_heterogeneous_3d_forward_matches_oracle_and_fp32_and_dot_test():
    """3D (the 128^3 configuration's geometry at 32^3): FP64 forward against the
    oracle's Dormand-Prince trajectories summed by the oracle (1e-7 rel-L2),
    FP32 against FP64 (1e-3), and the FP64 transpose's dot test (1e-10)."""
    import beamax_b200 as bb
    from beamax_b200.solvers.msgb_solver import Selection

    dev = _dev()
    dom, wpt, p0, sens, ts, c = _het3d_case(thr=4)
    ode = bb.gb.gb_solvers.solve_ODE_base
    s64 = bb.MSGBSolver(4, "top_n", 64, "spatial", ode, "scan_real")
    s32 = bb.MSGBSolver(4, "top_n", 64, "spatial", ode, "scan_real", precision="fp32")
    y64 = s64.forward(p0, dom, sens, ts, wpt)
    bt = s64.beams(s64.last_selection, dom, wpt)
    x0, p0s = bt.x0.cpu().numpy(), bt.p0.cpu().numpy()
    al, a0, w = bt.alpha.cpu().numpy(), bt.a0.cpu().numpy(), bt.omega.cpu().numpy()
    speed = oo.GridSpeed(c, dom.dx, method="bspline3", boundary="clamp")
    ref = np.zeros_like(y64)
    for j in range(x0.shape[0]):
        for mode in (1.0, -1.0):
            xt, pt, Mt, At, st, _ = oo.dopri5(x0[j], p0s[j], np.diag(al[j]), a0[j], mode, ts, speed)
            assert st == 0
            ref += oo.beam_field(xt, pt, Mt, At, w[j], sens.positions, dom.grid_size, dom.periodic)
    assert om.rel_l2(ref, y64) < 1e-7
    y32 = s32.forward(p0, dom, sens, ts, wpt)
    assert om.rel_l2(y64, y32) < 1e-3
    sel = s64.last_selection
    data = np.random.default_rng(6).standard_normal(y64.shape)
    a64 = s64.adjoint(data, dom, sens, ts, wpt, selection=sel)
    q = np.random.default_rng(7).standard_normal(dom.N)
    cq = wpt.forward_device(torch.from_numpy(q).to(dev), scale=0.5, half_mask=True)
    Aq = s64.sum_forward(s64.beams(Selection(sel.idx, cq[sel.idx], sel.total_coeffs), dom, wpt), dom, sens,
                         ts).cpu().numpy()
    lhs, rhs = float(np.sum(Aq * data)), float(np.sum(q * a64))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_compact_trajectory_store_equals_dense_records():
    """The FP32 path's compact store (a time tile's records kept only when it
    comes within the cutoff of a sensor tile) gives the same bits as storing
    every record when both hold all beams in one chunk: the summation
    evaluates the same triples in the same order.  When the pool runs out (a
    live-tile estimate far too low) and chunks are split and integrated
    again, both directions pair other beams in their paired FP32 sums (a
    pair whose partner needs the direct evaluation is evaluated directly):
    1e-6 rel-L2.  Also when the adjoint reuses the forward's records."""
    import beamax_b200 as bb

    dev = _dev()
    dom, wpt, p0, sens, ts, c, interp, thr = _het_case(seed=4, N=(128, 128), thr=300)
    ode = bb.gb.gb_solvers.solve_ODE_base
    dense = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", precision="fp32",
                          compact_trajectories=False)
    compact = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", precision="fp32")
    tight = bb.MSGBSolver(thr, "top_n", 64, "spatial", ode, "scan_real", precision="fp32",
                          trajectory_memory=4 << 20, keep_trajectories=False)
    compact._live_est = 1.0  # one chunk, as the dense store
    tight._live_est = 0.01  # far below the true fraction: the first pools overflow
    y_d = dense.forward(p0, dom, sens, ts, wpt)
    y_c = compact.forward(p0, dom, sens, ts, wpt)
    y_t = tight.forward(p0, dom, sens, ts, wpt)
    assert len(compact.compact_log) == 1 and len(tight.compact_log) > 2
    assert np.array_equal(y_d, y_c)
    assert om.rel_l2(y_d, y_t) <= 1e-6, om.rel_l2(y_d, y_t)
    assert compact._cached_trajectories(compact.last_selection, dom, ts) is not None
    assert 0.0 < compact._live_est < 1.0
    data = torch.from_numpy(np.random.default_rng(2).standard_normal(y_d.shape)).to(dev).float()
    a_d = dense.adjoint(data, dom, sens, ts, wpt)
    a_c = compact.adjoint(data, dom, sens, ts, wpt)
    a_t = tight.adjoint(data, dom, sens, ts, wpt)
    assert torch.equal(a_d, a_c)
    rel = float(torch.linalg.vector_norm(a_t - a_d) / torch.linalg.vector_norm(a_d))
    assert rel <= 1e-6, rel
