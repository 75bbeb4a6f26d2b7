"""Pins the FP64 oracle to the reference's own known-answer and identity tests.

Each test names the reference test it restates (paths relative to the beamax
project root).  Random inputs are re-seeded with NumPy because the reference's
JAX threefry streams cannot be reproduced without JAX.
"""

import numpy as np
import pytest

from oracle import msgb as om


def _wpt(num_levels, N, boxes, bar=None, windowing="rectangular", redundancy=2):
    bar = bar or (1,) * len(N)
    dec = om.Decomp(num_levels, N, boxes, bar)
    return om.Wpt(dec, redundancy, windowing)


@pytest.mark.parametrize(
    "N, lengths, retained",
    [((2048,), (32, 64, 128), (4, 6, 12)), ((256, 256), (4, 8, 16), (16, 60, 240))],
)
def test_three_level_tiling(N, lengths, retained):
    """tests/test_decomposition.py:113-130."""
    dec = om.Decomp(3, N, (4, 8, 16), (1,) * len(N))
    assert tuple(int(x) for x in dec.box_lengths) == lengths
    assert tuple(int(x) for x in dec.num_boxes_ndim) == retained


@pytest.mark.parametrize("N", [(64, 64), (32, 32)])
def test_rejects_short_boxes(N):
    """tests/test_decomposition.py:133-141."""
    with pytest.raises(ValueError, match="at least 2 Fourier samples"):
        om.Decomp(3, N, (4, 8, 16), (1, 1))


def test_config3_tiling_as_stated_is_rejected_and_corrected_tiling_is_valid():
    """1024^2 with boxes (4,8,16,32,64) has a level-0 box length of 1."""
    with pytest.raises(ValueError, match="at least 2 Fourier samples"):
        om.Decomp(5, (1024, 1024), (4, 8, 16, 32, 64), (1, 1))
    # 5 levels with (2,4,8,16,32): a 2x2 level-0 grid leaves nothing inside
    # level 1's lattice to cut out, so the centre count check
    # (decomposition.py:529-534) rejects it as well.
    with pytest.raises(ValueError, match="centre count"):
        om.Decomp(5, (1024, 1024), (2, 4, 8, 16, 32), (1, 1))
    dec = om.Decomp(4, (1024, 1024), (4, 8, 16, 32), (1, 1))
    assert tuple(int(x) for x in dec.box_lengths) == (4, 8, 16, 32)
    assert tuple(int(x) for x in dec.num_boxes_ndim) == (16, 60, 240, 960)


@pytest.mark.parametrize("nl", [1, 2])
@pytest.mark.parametrize("N", [(128,), (128, 128), (256, 128)])
def test_decomp_is_dyadic(nl, N):
    """tests/test_decomposition.py:94-110."""
    dec = om.Decomp(nl, N, tuple(2 ** (l + 2) for l in range(nl)), (1,) * len(N))
    for i in range(1, nl):
        assert dec.box_lengths[i] == 2 * dec.box_lengths[i - 1]


@pytest.mark.parametrize("windowing", ["rectangular", "rectangular_mirror"])
@pytest.mark.parametrize("N,bar", [((128,), (1,)), ((128, 128), (1, 1)), ((256, 128), (2, 1))])
def test_partition_of_unity(N, bar, windowing):
    """tests/test_ms_filters.py:60-92: sum g*h == 1, 0 <= g <= 1."""
    dec = om.Decomp(2, N, (4, 8), bar)
    g, h = om.compute_gh_filters(dec, 2, windowing)
    assert np.allclose(np.sum(g * h, axis=0), 1.0, atol=1e-15, rtol=0)
    assert np.all(g >= 0) and np.all(g <= 1)


ROUNDTRIP = [
    (1, (128,), (4,), (1,), "rectangular"),
    (2, (128,), (4, 8), (1,), "rectangular_mirror"),
    (2, (128, 128), (4, 8), (1, 1), "rectangular"),
    (2, (256, 128), (4, 8), (1, 1), "rectangular_mirror"),
    (2, (256, 128), (4, 8), (2, 1), "rectangular"),
    (1, (128, 512), (4,), (1, 4), "rectangular_mirror"),
]


@pytest.mark.parametrize("nl,N,boxes,bar,windowing", ROUNDTRIP)
def test_inverse_forward_identity(nl, N, boxes, bar, windowing):
    """tests/test_transforms.py:108-118 and 121-135."""
    w = _wpt(nl, N, boxes, bar, windowing)
    rng = np.random.default_rng(0)
    f = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    assert np.allclose(w.inverse(w.forward(f)), f, atol=1e-13, rtol=0)
    c = rng.standard_normal(w.total_coeffs)
    f1 = w.inverse(c)
    assert np.allclose(w.inverse(w.forward(f1)), f1, atol=1e-13, rtol=0)


def test_redundancy_one_anisotropic_roundtrip():
    """tests/test_transforms.py:78-86."""
    w = _wpt(2, (64, 32), (4, 8), (2, 1), "rectangular", redundancy=1)
    f = np.random.default_rng(91).standard_normal((64, 32))
    assert np.allclose(w.inverse(w.forward(f)), f, atol=1e-12, rtol=1e-12)


def test_forward_rejects_unwindowed():
    """tests/test_transforms.py:64-75."""
    w = _wpt(1, (64,), (4,), windowing="none")
    with pytest.raises(ValueError, match="does not support windowing='none'"):
        w.forward(np.ones(64))


@pytest.mark.parametrize("nl,N", [(1, (128,)), (2, (128, 128)), (2, (256, 128))])
def test_single_coefficient_equals_frame(nl, N):
    """tests/test_frames.py:359-411."""
    w = _wpt(nl, N, tuple(2 ** (l + 2) for l in range(nl)), windowing="rectangular_mirror")
    dec = w.dyadic_decomp
    rng = np.random.default_rng(1)
    for idx in rng.integers(0, w.total_coeffs, size=3):
        c = np.zeros(w.total_coeffs)
        c[idx] = 1.0
        got = w.inverse(c, "fourier")
        lvl, mi = om.find_tensor_and_multiindex([idx], om.coeff_shapes(w))
        box = mi[0, 0] + w.boxes_cumsum[lvl[0]]
        ref = om.compute_frames(dec, box, mi[1:, 0], dec.fourier_meshgrid, 2, "rectangular_mirror")
        assert np.allclose(ref, got, atol=1e-14, rtol=1e-12)


def test_isotropic_redundancy_two_phases_trivial():
    """tests/test_frames.py:452-466."""
    w = _wpt(2, (64, 64), (4, 8))
    lvl, mi = om.find_tensor_and_multiindex(np.arange(w.total_coeffs), om.coeff_shapes(w))
    box = mi[0] + np.r_[0, np.cumsum(w.dyadic_decomp.num_boxes_ndim)][lvl]
    ph = om.compute_frame_phase(w.dyadic_decomp, box, mi[1:].T, 2)
    assert np.array_equal(ph, np.ones_like(ph))


def test_beam_init_equals_frame_atoms():
    """tests/solvers/test_fwd_solver.py:272-361: sum coeff*GB(t=0) == sum frames."""
    N = (128, 128)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(True, True), cfl=0.354, c=1500.0)
    w = _wpt(2, N, (4, 8))
    dec = w.dyadic_decomp
    rng = np.random.default_rng(0)
    idx = np.unique(rng.integers(0, w.total_coeffs, size=2))
    manual = 0
    lvl, mi = om.find_tensor_and_multiindex(idx, om.coeff_shapes(w))
    for j in range(idx.size):
        box = mi[0, j] + w.boxes_cumsum[lvl[j]]
        manual = manual + om.unitary_ifft(om.compute_frames(dec, box, mi[1:, j], dec.fourier_meshgrid, 2, "none"))
    p0s, M0s, x0s, oms, a0s, modes = om.compute_forward_parameters(idx, w, dom)
    xt, pt, Mt, At = om.solve_hom_diag(x0s, p0s, M0s, a0s, modes, np.array([0.0]), 1500.0)
    G = om.gaussian_beam_complex(xt, pt, Mt, At, oms, dom.grid, dom.grid_size, dom.periodic)
    gb = np.sum(G, axis=-1)[0]
    assert np.allclose(gb, manual, atol=1e-14, rtol=0)


def test_coefficients_dpdt_zero_and_p0_zero():
    """tests/solvers/test_solver_utils.py:24-92."""
    N = (128, 64)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), c=1500.0)
    w = _wpt(2, N, (4, 8))
    f = np.random.default_rng(0).standard_normal(N)
    z = np.zeros(N)
    cp, cn = om.compute_coefficients(f, z, "spatial", dom, w)
    assert np.allclose(cp, cn)
    cp, cn = om.compute_coefficients(z, f, "spatial", dom, w)
    assert np.allclose(cp, -cn)


def test_coefficients_conjugate_pairs():
    """tests/solvers/test_solver_utils.py:231-299."""
    N = (128, 64)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), c=1500.0)
    w = _wpt(2, N, (4, 8), windowing="rectangular_mirror")
    rng = np.random.default_rng(10)
    cp, cn = om.compute_coefficients(rng.standard_normal(N), rng.standard_normal(N), "spatial", dom, w)
    for l in range(2):
        s, e = w.coeffs_cumsum[l], w.coeffs_cumsum[l + 1]
        P = cp[s:e].reshape(w.coeff_shapes[l])
        Q = cn[s:e].reshape(w.coeff_shapes[l])
        nb = P.shape[0]
        for b in range(nb):
            assert np.allclose(P[b], np.conj(Q[nb - b - 1]))


def test_top_n_returns_ascending_magnitudes():
    """tests/solvers/test_msgb_solver_misc.py:515-558 (values 3 then 4)."""
    idx, vals = om.threshold_top_n(np.array([1.0, 4.0, 2.0, 3.0]), 2)
    assert np.array_equal(vals, [3.0, 4.0])
    assert np.array_equal(idx, [3, 1])


def test_top_n_tie_rule():
    """Ties at the threshold keep the higher flat indices (JAX argpartition)."""
    c = np.array([0.0, 5.0, 0.0, 0.0, 5.0, 1.0])
    idx, _ = om.threshold_top_n(c, 4)
    assert list(idx) == [3, 5, 1, 4]


def test_oversized_top_n_matches_half_frame_cap():
    """tests/solvers/test_msgb_solver_misc.py:352-389."""
    N = (16,)
    dom = om.Dom(N=N, dx=(1.0 / 16,), periodic=(True,), c=1.0)
    w = _wpt(1, N, (4,))
    half = sum((e - s) // 2 for s, e in zip(w.coeffs_cumsum[:-1], w.coeffs_cumsum[1:]))
    p0 = np.random.default_rng(37).standard_normal(N)
    sens = dom.grid.reshape(-1, 1)
    ts = np.linspace(0.0, 0.02, 3)
    d1, b1 = om.forward(p0, dom, sens, ts, w, half)
    d2, b2 = om.forward(p0, dom, sens, ts, w, w.total_coeffs)
    assert b1.idx.shape == (half,)
    assert np.all(np.abs(b1.a0_unit * b1.coeff) > 0)
    assert np.allclose(d1, d2, rtol=1e-12, atol=1e-12)
    assert np.array_equal(b1.idx, b2.idx)


def _packet(x, centre, width, cycles):
    return np.exp(-0.5 * ((x - centre) / width) ** 2) * np.cos(2 * np.pi * cycles * (x - centre))


def test_dalembert_1d_forward():
    """examples/diagnostics/msgb_adjoint_pairing.py:189-199: (P f)(0, t) ~= f(c t)/2."""
    n = 128
    dx = 1.0 / n
    dt = 1.0 / n
    dom = om.Dom(N=(n,), dx=(dx,), periodic=(False,), c=1.0)
    w = _wpt(2, (n,), (4, 8))
    x = dom.grid[..., 0]
    f = _packet(x, 0.58, 0.075, 24.0)
    ts = np.arange(n) * dt
    sens = np.zeros((1, 1))
    data, _ = om.forward(f, dom, sens, ts, w, 32)
    ref = 0.5 * _packet(ts, 0.58, 0.075, 24.0)
    assert om.rel_l2(ref, data[:, 0]) < 2e-2


def test_adjoint_dot_product_2d():
    """Exact transpose: <A p0, d> == <p0, A* d> at round-off."""
    N = (64, 64)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), c=1500.0)
    w = _wpt(2, N, (4, 8), windowing="rectangular_mirror")
    rng = np.random.default_rng(3)
    p0 = rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = 1
    mask[:, 0] = 1
    sens = om.sensor_positions_from_mask(dom, mask)
    ts = dom.generate_time_domain()[::8]
    bm = om.select_beams(p0, dom, w, 300)
    Ap = om.forward_hom(bm, dom, sens, ts)
    d = rng.standard_normal(Ap.shape)
    q = rng.standard_normal(N)
    lhs = np.sum(om.forward_hom(om.beams_for(bm.idx, om.compute_coefficients(q, np.zeros(N), "spatial", dom, w, "pos_only")[bm.idx], dom, w), dom, sens, ts) * d)
    rhs = np.sum(q * om.adjoint(bm, dom, sens, ts, w, d))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def test_oracle_dopri5_1d_linear_closed_form():
    """Adaptive Dormand-Prince 5(4) against the closed form for c = a + b x
    (tests/test_gb.py:630-756, rtol 1e-7 / atol 1e-10), in both save modes:
    steps ending on the save times, and the continuous extension (fewer
    steps; the M bound is 2e-7, the global error of this pair at the default
    tolerance being 1.01x the reference test's 1e-7 bound)."""
    from oracle import ode as oo

    a, b = 1.0, 1.0
    xs = np.arange(0, 400) * 0.01
    speed = oo.GridSpeed(a + b * xs, (0.01,), method="linear", boundary="clamp")
    ts = np.linspace(0.0, 1.0, 200)
    xr, pr, Mr, Ar = oo.analytic_1d_linear(0.1, 1.2, 0.2j, 1.0, ts, a, b)
    for dense, rtol_m in ((False, 1e-7), (True, 2e-7)):
        x, p, M, A, status, steps = oo.dopri5(np.array([0.1]), np.array([1.2]), np.array([[0.2j]]), 1.0, 1.0, ts,
                                              speed, dense=dense)
        assert status == 0
        assert (steps < ts.size - 1) if dense else (steps >= ts.size - 1)
        assert np.allclose(x[:, 0], xr, atol=1e-10, rtol=1e-7)
        assert np.allclose(p[:, 0], pr, atol=1e-10, rtol=1e-7)
        assert np.allclose(M[:, 0, 0], Mr, atol=1e-10, rtol=rtol_m)
        assert np.allclose(A, Ar, atol=1e-10, rtol=1e-7)


def test_oracle_dopri5_converges_to_dop853_and_honours_max_steps():
    """Tighter tolerances move the adaptive solution onto DOP853's; a step
    budget that is too small reports status 2."""
    from scipy import ndimage

    from oracle import ode as oo

    rng = np.random.default_rng(5)
    g = ndimage.gaussian_filter(rng.standard_normal((32, 32)), 8.0, mode="wrap")
    c = 1500.0 * (1 + 0.1 * g / np.max(np.abs(g)))
    speed = oo.GridSpeed(c, (1e-4, 1e-4), method="bspline3", boundary="clamp")
    x0, p0, M0 = np.array([16e-4, 15e-4]), np.array([2 * np.pi, 0.3]), np.diag([1e-3j, 2e-3j])
    ts = np.arange(0, 30) * 2e-8
    xt, pt, Mt, At = oo.solve(x0, p0, M0, 1.0, 1.0, ts, speed)
    errs = []
    for rtol in (1e-6, 1e-9):
        x, p, M, A, status, _ = oo.dopri5(x0, p0, M0, 1.0, 1.0, ts, speed, rtol=rtol, atol=rtol * 1e-2,
                                          max_steps=100000)
        assert status == 0
        errs.append(np.max(np.abs(M - Mt)) / np.max(np.abs(Mt)))
    assert errs[1] < 0.1 * errs[0]
    *_, status, steps = oo.dopri5(x0, p0, M0, 1.0, 1.0, ts, speed, max_steps=5, dense=True)
    assert status == 2 and steps == 5
    # ending steps on the save times adds nt - 1 to the budget
    *_, status, steps = oo.dopri5(x0, p0, M0, 1.0, 1.0, ts, speed, max_steps=2)
    assert status == 2 and steps == 2 + ts.size - 1


# ---- time reversal (tests/solvers/test_tr_solver.py:88-260) ----------------


def _tr_1d(mask_idx):
    from oracle import ode as oo
    from oracle import tr as otr

    dom = om.Dom(N=(16,), dx=(0.1,), periodic=(False,), c=1.0)
    wpt = om.Wpt(om.Decomp(1, (16,), (2,), (1,)), 2, "rectangular")
    pos = np.zeros((1, 1))
    pos[0, 0] = (np.arange(16) * 0.1)[mask_idx]
    src = otr.Sources(pos, dom.dx, dom.grid_size)
    idx = np.arange(min(8, wpt.total_coeffs))
    return otr.tr_parameters(idx, dom, wpt, src, oo.LinearSpeed(1.0, np.zeros(1)))


@pytest.mark.parametrize("mask_idx,sign", [(0, 1.0), (-1, -1.0)])
def test_tr_beams_point_inward(mask_idx, sign):
    pts = _tr_1d(mask_idx)[0]
    n = pts[:, 0]
    finite = np.abs(n) > 1e-8
    assert finite.any()
    assert np.all(sign * n[finite] >= 0)


def _tr_2d_data(c, data_dx=(1.0, 1.0)):
    dom = om.Dom(N=(16, 16), dx=data_dx, periodic=(False, False), c=c)
    return dom, om.Wpt(om.Decomp(1, (16, 16), (2,), (1, 1)), 2, "rectangular")


def test_tr_detector_side_from_spatial_domain():
    from oracle import ode as oo
    from oracle import tr as otr

    data_dom, wpt = _tr_2d_data(0.01, (1.0, 0.1))
    pos = np.stack([np.full(16, 15 * 0.1), np.arange(16) * 0.1], 1)
    src = otr.Sources(pos, (0.1, 0.1), (1.6, 1.6))
    idx = np.arange(min(64, wpt.total_coeffs))
    pts = otr.tr_parameters(idx, data_dom, wpt, src, oo.LinearSpeed(0.01, np.zeros(2)))[0]
    lvl, mi = om.find_tensor_and_multiindex(idx, om.coeff_shapes(wpt))
    ch = wpt.dyadic_decomp.centres_ndim[mi[0]] / data_dom.grid_size
    hyper = ch[:, 0] ** 2 - 0.01 ** 2 * np.sum(ch[:, 1:] ** 2, 1) > 1e-10
    assert hyper.any()
    assert np.all(pts[hyper, 0] <= 0)


def test_tr_temporal_carrier_sets_tangential_phase():
    from oracle import ode as oo
    from oracle import tr as otr

    data_dom, wpt = _tr_2d_data(0.3)
    pos = np.stack([np.zeros(16), np.arange(16) * 1.0], 1)
    src = otr.Sources(pos, (1.0, 1.0), (16.0, 16.0))
    idx = np.arange(min(64, wpt.total_coeffs))
    pts, _, _, omega, *_ = otr.tr_parameters(idx, data_dom, wpt, src, oo.LinearSpeed(0.3, np.zeros(2)))
    lvl, mi = om.find_tensor_and_multiindex(idx, om.coeff_shapes(wpt))
    ch = wpt.dyadic_decomp.centres_ndim[mi[0]] / data_dom.grid_size
    tau, k_tan = ch[:, 0], ch[:, 1:]
    ok = (np.abs(tau) > 1e-8) & (np.linalg.norm(k_tan, axis=1) > 1e-8)
    assert ok.any()
    np.testing.assert_allclose(omega[ok], np.abs(tau[ok]))
    np.testing.assert_allclose(omega[ok, None] * pts[ok, 1:], 2 * np.pi * k_tan[ok])


@pytest.mark.parametrize("redundancy", [1, 2])
def test_tr_packet_positions_follow_redundant_anisotropic_support(redundancy):
    from oracle import ode as oo
    from oracle import tr as otr

    data_dom = om.Dom(N=(32, 16), dx=(0.1, 0.3), periodic=(False, False), c=0.01)
    dec = om.Decomp(1, (32, 16), (4,), (2, 1))
    wpt = om.Wpt(dec, redundancy, "rectangular")
    pos = np.stack([np.zeros(16), np.arange(16) * 0.3], 1)
    src = otr.Sources(pos, (0.2, 0.3), (3.2, 4.8))
    shape = tuple(int(v) for v in wpt.coeff_shapes[0])
    k = np.array([shape[1] - 1, shape[2] - 1])
    flat = np.ravel_multi_index((0, k[0], k[1]), shape)
    _, _, x, _, a, _, t0 = otr.tr_parameters(np.array([flat]), data_dom, wpt, src,
                                             oo.LinearSpeed(0.01, np.zeros(2)))
    support = redundancy * dec.box_lengths[0] * np.array([2, 1])
    expect = k * data_dom.grid_size / support
    assert t0[0] == pytest.approx(expect[0])
    assert x[0, 0] == pytest.approx(0.0)
    assert x[0, 1] == pytest.approx(expect[1])
    assert t0[0] < data_dom.grid_size[0] and x[0, 1] < data_dom.grid_size[1]
    ph = om.compute_frame_phase(dec, 0, k, redundancy)
    assert a[0] / abs(a[0]) == pytest.approx(ph)


def test_tr_spatial_hessian_inverts_spacetime_hessian():
    """mT_inverse (tr_solver_utils.py:116-170) is the inverse of mT_forward
    (:64-113) for a spatial Hessian whose lower-right block is the
    spacetime one's."""
    from oracle import ode as oo
    from oracle import tr as otr

    rng = np.random.default_rng(0)
    speed = oo.LinearSpeed(1500.0, np.array([30.0, -20.0]))
    x = np.array([0.0, 1e-3])
    p = np.array([3.0, 1.0])
    S = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
    S = S + S.T
    M = otr.mT_inverse(x, p, S, -1.0, speed)
    gp, gx = otr.gp_gx(x, p, -1.0, speed)
    xd, pd = gp, -gx
    # mT_forward of the spatial result gives S back
    up_left = xd @ M @ xd - pd @ xd
    up_right = (pd - M @ xd)[1:]
    # |x_dot|^2 ~ c^2 = 2.25e6 against O(1) entries: cancellation to ~1e-10
    np.testing.assert_allclose(up_left, S[0, 0], rtol=1e-8)
    np.testing.assert_allclose(up_right, S[0, 1:], rtol=1e-8)
    np.testing.assert_allclose(M[1:, 1:], S[1:, 1:])


# ---- principal-symbol adjoint (tests/solvers/test_adj_solver_utils.py,
# ---- tests/solvers/test_msgb_solver_misc.py:452-578) -----------------------


def test_b_inverse_normal_incidence_sign_and_conjugacy():
    from oracle import tr as otr

    b = otr.principal_b_inverse(np.array([3.0, -3.0]), np.zeros((2, 1)), np.array([2.0, 2.0]))
    assert b[0] == pytest.approx(-1j / (4.0 * np.pi * 2.0 * 3.0))
    assert b[1] == pytest.approx(np.conj(b[0]))


def test_b_inverse_removes_evanescent_and_grazing_modes():
    from oracle import tr as otr

    r = 5e-7
    b = otr.principal_b_inverse(np.array([1.0, 2.0, 1.0, 0.0]),
                                np.array([[1.0], [1.0], [np.sqrt(1.0 - r * r)], [0.0]]),
                                np.array([2.0, 2.0, 1.0, 1.0]))
    assert np.all(b == 0.0)


def test_b_inverse_relative_guard_is_frequency_local():
    from oracle import tr as otr

    tau = np.array([1.0, 1e6])
    b = otr.principal_b_inverse(tau, (tau * np.sqrt(1.0 - 1e-6))[:, None], np.ones(2))
    assert np.all(np.abs(b) > 0)
    assert b[0] / b[1] == pytest.approx(tau[1] / tau[0], rel=1e-6)


def _adj_2d(c0, grad=0.0):
    from oracle import ode as oo
    from oracle import tr as otr

    dom = om.Dom(N=(16, 16), dx=(1.0, 1.0), periodic=(False, False), c=c0)
    wpt = om.Wpt(om.Decomp(1, (16, 16), (2,), (1, 1)), 2, "rectangular")
    pos = np.stack([np.zeros(16), np.arange(16.0)], 1)
    src = otr.Sources(pos, (1.0, 1.0), (16.0, 16.0))
    return dom, wpt, src, oo.LinearSpeed(c0, np.array([0.0, grad]))


def test_adj_parameters_are_tr_geometry_times_b_inverse():
    from oracle import tr as otr

    dom, wpt, src, speed = _adj_2d(0.3, 0.01)
    idx = np.array([0, 5, 256, 261])
    tr = otr.tr_parameters(idx, dom, wpt, src, speed)
    adj = otr.adj_parameters(idx, dom, wpt, src, speed)
    lvl, mi = om.find_tensor_and_multiindex(idx, om.coeff_shapes(wpt))
    ch = wpt.dyadic_decomp.centres_ndim[mi[0]] / dom.grid_size
    c = np.array([speed.eval(x)[0] for x in adj[2]])
    binv = -otr.principal_b_inverse(ch[:, 0], ch[:, 1:], c, 5e-2)
    keep = binv != 0
    for k in (0, 1, 2, 3, 5, 6):
        a, b = np.asarray(tr[k]), np.asarray(adj[k])
        np.testing.assert_allclose(b[keep], a[keep])
    np.testing.assert_allclose(adj[4], tr[4] * binv)


def test_adj_parameters_zero_for_evanescent_packets():
    from oracle import tr as otr

    dom, wpt, src, speed = _adj_2d(10.0)
    idx = np.array([0, 256, 512, 768])
    adj = otr.adj_parameters(idx, dom, wpt, src, speed)
    assert np.all(adj[4] == 0)
    assert np.all(adj[0] == 1.0)
    np.testing.assert_array_equal(adj[1], np.broadcast_to(1j * np.eye(2), adj[1].shape))


def test_adj_parameters_1d():
    from oracle import ode as oo
    from oracle import tr as otr

    dom = om.Dom(N=(16,), dx=(1.0,), periodic=(False,), c=0.5)
    wpt = om.Wpt(om.Decomp(1, (16,), (2,), (1,)), 2, "rectangular")
    src = otr.Sources(np.zeros((1, 1)), (1.0,), (16.0,))
    speed = oo.LinearSpeed(0.5, np.zeros(1))
    idx = np.array([0, 16])
    tr = otr.tr_parameters(idx, dom, wpt, src, speed)
    adj = otr.adj_parameters(idx, dom, wpt, src, speed)
    lvl, mi = om.find_tensor_and_multiindex(idx, om.coeff_shapes(wpt))
    tau = (wpt.dyadic_decomp.centres_ndim[mi[0]] / dom.grid_size)[:, 0]
    binv = -otr.principal_b_inverse(tau, np.zeros((2, 0)), np.full(2, 0.5), 5e-2)
    np.testing.assert_allclose(adj[4], tr[4] * binv)


def test_adjoint_source_spectral_derivative_sign_and_c_squared():
    from oracle import tr as otr

    n, dt, mode = 64, 0.25 / 64, 5
    t = np.arange(n) * dt
    w = 2 * np.pi * mode / (n * dt)
    c = np.array([2.0, 3.0])
    s = otr.form_adjoint_source(np.ones((n, 2)), dt, c, np.sin(w * t))
    np.testing.assert_allclose(s, -(c ** 2) * w * np.cos(w * t)[:, None], rtol=1e-12, atol=1e-10)


def test_adjoint_source_folds_flat_speeds_onto_detector_grid():
    from oracle import tr as otr

    rng = np.random.default_rng(0)
    data = rng.standard_normal((8, 3, 2))
    c = rng.uniform(1.0, 2.0, 6)
    g = otr.form_adjoint_source(data, 0.1, c)
    f = otr.form_adjoint_source(data.reshape(8, 6), 0.1, c)
    np.testing.assert_allclose(g.reshape(8, 6), f, atol=1e-12)
    with pytest.raises(ValueError, match="does not match the data detector grid"):
        otr.form_adjoint_source(np.ones((4, 3, 2)), 0.1, np.ones(5))
