"""GPU parity of MSGB time reversal (MSGBSolver.time_reversal).

Oracle: oracle/tr.py (compute_TR_parameters restated, each beam integrated
back to t = 0 with SciPy DOP853 at rtol = atol = 1e-12, the real field summed
at the image points and doubled).  Tolerances: beam parameters from
msgb_tr_init equal to the oracle's to 1e-12 relative (same formulas in FP64);
the reconstruction within 1e-7 rel-L2 of the oracle's with the GPU's adaptive
integrator at rtol 1e-10 (homogeneous and B-spline media, with absorption).
Setups follow the reference's TR tests: tests/solvers/test_msgb_aggregation.py
:134-186 (frequency-cropped data domain, random boundary data x 0.01, one
line of sources, every grid point as an image point) and
tests/solvers/test_tr_solver.py:88-260.
"""

import numpy as np
import pytest

from oracle import msgb as om
from oracle import ode as oo
from oracle import tr as otr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _setup(N, c=1500.0, dx=1e-4, seed=0):
    """Image domain, its time grid, the cropped data domain (2 N0 time
    samples) with its MSWPT, line sources on the first row, image points."""
    import beamax_b200 as bb

    d = len(N)
    dom = bb.Domain(N=N, dx=(dx,) * d, periodic=(False,) * d, cfl=0.3, c=c)
    ts = dom.generate_time_domain()
    nt = 2 * N[0]
    ddx = float((ts[-1] - ts[0]) / (nt - 1))
    if d == 1:
        Nd, ddxs, aspect = (nt,), (ddx,), (1,)
    else:
        Nd = (nt,) + tuple(N[1:])
        ddxs = (ddx,) + (dx,) * (d - 1)
        m = min(Nd)
        aspect = tuple(v // m for v in Nd)
    ddom = bb.Domain(N=Nd, dx=ddxs, periodic=(False,) * d, cfl=0.3, c=1500.0 if not np.isscalar(c) else c)
    dwpt = bb.MSWPT(bb.DyadicDecomposition(2, Nd, (4, 8), aspect), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[(0,) + (slice(None),) * (d - 1)] = 1
    src = bb.Sensor(dom, binary_mask=mask)
    img = bb.Sensor(dom, binary_mask=np.ones(N))
    data = np.random.default_rng(seed).standard_normal(Nd) * 0.01
    return dom, ts, ddom, dwpt, src, img, data


def _oracle_objects(ddom, dwpt, src, dom):
    d = ddom.ndim
    odom = om.Dom(N=ddom.N, dx=tuple(ddom.dx), periodic=(False,) * d, c=1500.0)
    dec = dwpt.dyadic_decomp
    owpt = om.Wpt(om.Decomp(dec.num_levels, dec.N, dec.num_boxes_levels, dec.box_aspect_ratio), dwpt.redundancy,
                  dwpt.windowing)
    osrc = otr.Sources(np.asarray(src.positions), dom.dx, dom.grid_size)
    return odom, owpt, osrc


def _solver(thr=200, rtol=1e-10, atol=1e-12):
    import beamax_b200 as bb
    from beamax_b200.gb.gb_solvers import SolverConfig

    return bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real",
                         ode_config=SolverConfig(rtol=rtol, atol=atol, max_steps=100000))


def _same_selection(solver, oracle_idx):
    """The GPU's selected indices, checked to be the oracle's set.  Real data
    give conjugate pairs of equal |c|, whose order (by index on exact ties)
    can flip when the two FFTs round the pair's magnitudes differently; the
    parameters are compared in the GPU's order."""
    idx = solver.last_boundary_selection.idx.cpu().numpy()
    assert np.array_equal(np.sort(idx), np.sort(oracle_idx))
    return idx


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize("N", [(32, 32), (64,), (32, 32, 32)])
def test_tr_parameters_match_oracle(N):
    _dev()
    dom, ts, ddom, dwpt, src, img, data = _setup(N, c=1.0 if len(N) == 1 else 1500.0,
                                                 dx=1.0 / N[0] if len(N) == 1 else 1e-4)
    s = _solver()
    _, params = s.time_reversal_with_params(data, dom, img, src, ts, ddom, dwpt)
    pts, Mts, xts, omega, ats, signum, tpair = params
    odom, owpt, osrc = _oracle_objects(ddom, dwpt, src, dom)
    c_pos = om.compute_coefficients(data, np.zeros_like(data), "spatial", odom, owpt, mode="both")[0]
    o_idx, _ = om.threshold_top_n(c_pos, om.effective_top_n(200, owpt))
    idx = _same_selection(s, o_idx)
    vals = c_pos[idx]
    speed = oo.LinearSpeed(float(dom.constant_speed()), np.zeros(len(N)))
    o_pts, o_M, o_x, o_om, o_a, o_sg, o_t0 = otr.tr_parameters(idx, odom, owpt, osrc, speed)
    o_a = o_a * vals
    assert _rel(pts, o_pts) <= 1e-12
    assert _rel(xts, o_x) <= 1e-12 if np.any(o_x) else np.all(xts == 0)
    assert _rel(Mts, o_M) <= 1e-12
    assert _rel(omega, o_om) <= 1e-13
    assert _rel(ats[:, 0], o_a) <= 1e-11
    assert np.array_equal(signum[:, 0], o_sg)
    assert _rel(tpair[:, 0], o_t0) <= 1e-13 and np.all(tpair[:, 1] == 0)


@pytest.mark.parametrize("N", [(32, 32), (64,)])
def test_time_reversal_matches_oracle_homogeneous(N):
    _dev()
    one_d = len(N) == 1
    dom, ts, ddom, dwpt, src, img, data = _setup(N, c=1.0 if one_d else 1500.0, dx=1.0 / N[0] if one_d else 1e-4)
    out = _solver().time_reversal(data, dom, img, src, ts, ddom, dwpt)
    assert out.shape == (int(np.prod(N)),)
    odom, owpt, osrc = _oracle_objects(ddom, dwpt, src, dom)
    speed = oo.LinearSpeed(float(dom.constant_speed()), np.zeros(len(N)))
    ref, _ = otr.time_reversal(data, odom, owpt, osrc, speed, np.asarray(img.positions), dom.grid_size, 200)
    assert np.all(np.isfinite(out))
    assert _rel(out, ref) <= 1e-7


LAM_HET = 2e3
GOLDEN_HET = "golden/tr_het_32x32.npz"


def het_setup():
    """32^2 B-spline medium (5 % contrast, 6-cell correlation), absorption
    lam = 2e3, the homogeneous case's data domain and boundary data."""
    import beamax_b200 as bb
    from scipy import ndimage

    from beamax_b200.utils.interp import make_c_function_from_grid

    N, dx = (32, 32), (1e-4, 1e-4)
    rng = np.random.default_rng(5)
    g = ndimage.gaussian_filter(rng.standard_normal(N), 6.0, mode="wrap")
    cgrid = 1500.0 * (1 + 0.05 * g / np.max(np.abs(g)))
    interp = make_c_function_from_grid(cgrid, dx, method="bspline3", boundary="clamp")
    _, _, ddom, dwpt, _, _, data = _setup(N, c=1500.0)
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=interp, lam=LAM_HET)
    mask = np.zeros(N)
    mask[0, :] = 1
    src = bb.Sensor(dom, binary_mask=mask)
    img = bb.Sensor(dom, binary_mask=np.ones(N))
    ts = np.linspace(0.0, (ddom.N[0] - 1) * ddom.dx[0], ddom.N[0])
    return dom, ts, ddom, dwpt, src, img, data, cgrid


def test_time_reversal_matches_oracle_heterogeneous_with_absorption():
    """Against the oracle's image, committed as a fixture (the oracle's
    Python interpolant makes this case take minutes; tests/golden/
    make_tr_het.py regenerates it)."""
    import os

    _dev()
    dom, ts, ddom, dwpt, src, img, data, _ = het_setup()
    out = _solver().time_reversal(data, dom, img, src, ts, ddom, dwpt)
    gold = np.load(os.path.join(os.path.dirname(__file__), GOLDEN_HET))
    assert np.array_equal(gold["data"], data)
    assert _rel(out, gold["image"]) <= 1e-7


# ---- principal-symbol adjoint (msgb_solver.py:1235-1386) -------------------


def test_adjoint_source_matches_oracle():
    from beamax_b200 import _lib

    dev = _dev()
    rng = np.random.default_rng(11)
    nt, ns, dt = 96, 24, 3e-8
    r = rng.standard_normal((nt, ns))
    c = rng.uniform(1400.0, 1600.0, ns)
    for window in (None, np.hanning(nt), rng.uniform(0.5, 1.0, (nt, ns))):
        ref = otr.form_adjoint_source(r, dt, c, window)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(dev)
        rd, cd = T(r), T(c)
        wd = None if window is None else T(window)
        out = torch.empty((nt, ns), dtype=torch.float64, device=dev)
        nb = _lib.lib().msgb_adjoint_source_workspace_size(nt, ns)
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        _lib.check(_lib.lib().msgb_adjoint_source(rd.data_ptr(), None if wd is None else wd.data_ptr(),
                                                  int(window is not None and np.ndim(window) == 1), nt, ns, dt,
                                                  cd.data_ptr(), out.data_ptr(), ws.data_ptr(), nb,
                                                  torch.cuda.current_stream().cuda_stream), "adjoint source")
        torch.cuda.synchronize()
        assert _rel(out.cpu().numpy(), ref) <= 1e-13


def test_medium_speed_matches_oracle_interpolant():
    import beamax_b200 as bb
    from scipy import ndimage

    from beamax_b200.utils.interp import make_c_function_from_grid

    dev = _dev()
    rng = np.random.default_rng(2)
    N, dx = (24, 20), (1e-4, 2e-4)
    g = ndimage.gaussian_filter(rng.standard_normal(N), 3.0, mode="wrap")
    cgrid = 1500.0 * (1 + 0.1 * g / np.max(np.abs(g)))
    pts = rng.uniform(-2e-4, 1.1 * np.array(N) * dx, (50, 2))
    for method in ("linear", "bspline3"):
        dom = bb.Domain(N=N, dx=dx, periodic=(False, False), c=make_c_function_from_grid(cgrid, dx, method=method,
                                                                                       boundary="clamp"))
        s = _solver()
        got = s._speed_at(dom, torch.from_numpy(pts).to(dev)).cpu().numpy()
        speed = oo.GridSpeed(cgrid, dx, method=method, boundary="clamp")
        ref = np.array([speed.eval(p)[0] for p in pts])
        assert np.max(np.abs(got - ref)) <= 1e-12 * 1500.0


def _oracle_adjoint_params(data, dom, ddom, dwpt, src, thr=200, window=None, idx_from=None):
    odom, owpt, osrc = _oracle_objects(ddom, dwpt, src, dom)
    speed = oo.LinearSpeed(float(dom.constant_speed()), np.zeros(dom.ndim))
    c_src = np.full(np.asarray(src.positions).shape[0], float(dom.constant_speed()))
    F = otr.form_adjoint_source(data, ddom.dx[0], c_src, window)
    coeffs = owpt.forward(F, "spatial")
    idx, vals = om.threshold_top_n(coeffs, om.effective_top_n(thr, owpt))
    if idx_from is not None:
        idx = _same_selection(idx_from, idx)
        vals = coeffs[idx]
    p = otr.adj_parameters(idx, odom, owpt, osrc, speed, 5e-2)
    return p, vals, speed, odom, owpt, osrc


@pytest.mark.parametrize("N", [(32, 32), (64,)])
def test_adjoint_parameters_match_oracle(N):
    _dev()
    one_d = len(N) == 1
    dom, ts, ddom, dwpt, src, img, data = _setup(N, c=1.0 if one_d else 1500.0, dx=1.0 / N[0] if one_d else 1e-4)
    s = _solver()
    _, params = s.adjoint_with_params(data, dom, img, src, ts, ddom, dwpt)
    (o_pts, o_M, o_x, o_om, o_a, o_sg, o_t0), vals, *_ = _oracle_adjoint_params(data, dom, ddom, dwpt, src,
                                                                                 idx_from=s)
    pts, Mts, xts, omega, ats, signum, tpair = params
    assert _rel(pts, o_pts) <= 1e-12
    assert _rel(Mts, o_M) <= 1e-12
    assert _rel(ats[:, 0], o_a * vals) <= 1e-11
    assert _rel(omega, o_om) <= 1e-13 and np.array_equal(signum[:, 0], o_sg)
    assert _rel(tpair[:, 0], o_t0) <= 1e-13
    assert np.any(ats != 0)


@pytest.mark.parametrize("N,window", [((32, 32), None), ((32, 32), "hann"), ((64,), None)])
def test_principal_adjoint_matches_oracle(N, window):
    _dev()
    one_d = len(N) == 1
    dom, ts, ddom, dwpt, src, img, data = _setup(N, c=1.0 if one_d else 1500.0, dx=1.0 / N[0] if one_d else 1e-4)
    w = np.hanning(data.shape[0]) if window == "hann" else None
    out = _solver().adjoint(data, dom, img, src, ts, ddom, dwpt, window=w)
    _, _, speed, odom, owpt, osrc = _oracle_adjoint_params(data, dom, ddom, dwpt, src, window=w)
    ref, _ = otr.principal_adjoint(data, ddom.dx[0], odom, owpt, osrc, speed, speed, np.asarray(img.positions),
                                   dom.grid_size, 200, window=w)
    assert out.shape == (int(np.prod(N)),)
    assert np.all(np.isfinite(out))
    assert _rel(out, ref) <= 1e-7
