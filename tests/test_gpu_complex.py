"""The complex summation (*_complex sum methods, gb/core.py:105-168) and the
complex-input path (msgb_solver.py:635-689) against the oracle, and their
adjoints by dot tests.

Real p0 with a complex sum: the mirrored beams' field sum_b a0 K_b, whose
real part times 2 is the real path's output.  Complex p0: c_pos and c_neg
(compute_coefficients mode="both") selected separately with the uncapped
top_n, c_pos beams on mode +1 and c_neg beams on mode -1, complex sum.
FP64 within 1e-12 rel-L2 of the oracle, FP32 within 1e-3 of FP64; the
adjoints satisfy <A q, d> = <q, A* d> to 1e-10 (FP64).
"""

import numpy as np
import pytest

from oracle import msgb as om

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _case():
    import beamax_b200 as bb

    N = (64, 64)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(11)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - 28.0) ** 2, -1) / 50.0) * np.cos(0.7 * xg[..., 0]) + 0.05 * rng.standard_normal(N)
    q0 = np.exp(-np.sum((xg - 36.0) ** 2, -1) / 40.0) * np.sin(0.5 * xg[..., 1])
    mask = np.zeros(N)
    mask[0, :] = mask[:, 0] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::2]
    odom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    return dom, wpt, p0, q0, sens, ts, odom, ow


def _complex_sum(p0s, M0s, x0s, omg, a0s, modes, ts, sens, dom):
    xt, pt, Mt, At = om.solve_hom_diag(x0s, p0s, M0s, a0s, modes, np.asarray(ts, float), 1500.0)
    return om.gaussian_beam_complex(xt, pt, Mt, At, omg, sens.positions, dom.grid_size, dom.periodic).sum(-1)


def _solver(thr, method, precision="fp64"):
    import beamax_b200 as bb

    return bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, method, precision=precision)


def test_real_input_complex_sum_matches_oracle_and_real_path():
    _dev()
    dom, wpt, p0, q0, sens, ts, odom, ow = _case()
    s_c, s_r = _solver(200, "scan_complex"), _solver(200, "scan_real")
    y_c = s_c.forward(p0, dom, sens, ts, wpt)
    y_r = s_r.forward(p0, dom, sens, ts, wpt)
    assert np.iscomplexobj(y_c)
    bm = om.select_beams(p0, odom, ow, 200)
    ref = _complex_sum(*om.mirrored_params(bm), ts, sens, dom)
    assert om.rel_l2(ref, y_c) < 1e-12
    assert om.rel_l2(y_r, 2.0 * y_c.real) < 1e-12
    y32 = _solver(200, "scan_complex", "fp32").forward(p0, dom, sens, ts, wpt)
    assert om.rel_l2(y_c, y32) < 1e-3


def test_complex_input_matches_oracle():
    _dev()
    dom, wpt, p0, q0, sens, ts, odom, ow = _case()
    z0 = p0 + 1j * q0
    s = _solver(150, "scan_complex")
    y = s.forward(z0, dom, sens, ts, wpt)
    cpos, cneg = om.compute_coefficients(z0, np.zeros_like(z0), "spatial", odom, ow, mode="both")
    n = om.effective_top_n(150, ow, half_frame=False)
    parts = []
    for c, mode in ((cpos, 1.0), (cneg, -1.0)):
        idx, vals = om.threshold_top_n(c, n)
        bm = om.beams_for(idx, vals, odom, ow)
        k = bm.idx.size
        parts.append((bm.p0, bm.M0, bm.x0, bm.omega, bm.a0_unit * bm.coeff, np.full(k, mode)))
    cat = [np.concatenate([parts[0][i], parts[1][i]]) for i in range(6)]
    ref = _complex_sum(*cat, ts, sens, dom)
    assert om.rel_l2(ref, y) < 1e-12
    np.testing.assert_array_equal(np.sort(s.last_selection.pos.idx.cpu().numpy()),
                                  np.sort(om.threshold_top_n(cpos, n)[0]))
    np.testing.assert_array_equal(np.sort(s.last_selection.neg.idx.cpu().numpy()),
                                  np.sort(om.threshold_top_n(cneg, n)[0]))
    y32 = _solver(150, "scan_complex", "fp32").forward(z0, dom, sens, ts, wpt)
    assert om.rel_l2(y, y32) < 1e-3
    y_real = _solver(150, "scan_real").forward(z0, dom, sens, ts, wpt)
    assert om.rel_l2(2.0 * y.real, y_real) < 1e-12


@pytest.mark.parametrize("complex_input", [False, True])
def test_complex_adjoints_dot_test(complex_input):
    dev = _dev()
    dom, wpt, p0, q0, sens, ts, odom, ow = _case()
    s = _solver(150, "scan_complex")
    z0 = p0 + 1j * q0 if complex_input else p0
    y = s.forward(z0, dom, sens, ts, wpt)
    sel = s.last_selection
    rng = np.random.default_rng(5)
    d = rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)
    if complex_input:
        q = rng.standard_normal(dom.N) + 1j * rng.standard_normal(dom.N)
    else:
        q = rng.standard_normal(dom.N)
    Aq = s.forward_frozen(q, dom, sens, ts, wpt, sel)
    img = s.adjoint(d, dom, sens, ts, wpt, selection=sel)
    lhs = np.vdot(Aq, d)                    # <A q, d> = sum conj(Aq) d
    rhs = np.vdot(q, img)                   # <q, A* d>
    if not complex_input:                   # real input: the real inner product
        lhs, rhs = lhs.real, rhs.real
        assert not np.iscomplexobj(img)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
