"""GPU parity: every libmsgb entry point against the FP64 oracle (B200 only).

Tolerances: FP64 kernels agree with the oracle to rel-L2 <= 1e-12 (the
reference's own FP64 tests use 1e-12..1e-14); top_n indices are bit-exact on
identical keys; the FP32 path meets rel-L2 <= 1e-3 against the FP64 path.
"""

import numpy as np
import pytest

from oracle import build as ob
from oracle import msgb as om

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _pair(nl, N, boxes, bar=None, windowing="rectangular_mirror", red=2):
    import beamax_b200 as bb

    bar = bar or (1,) * len(N)
    return (bb.MSWPT(bb.DyadicDecomposition(nl, N, boxes, bar), red, windowing),
            om.Wpt(om.Decomp(nl, N, boxes, bar), red, windowing))


MSWPT_CASES = [
    (2, (128,), (4, 8), None, "rectangular", 2),
    (3, (128, 128), (4, 8, 16), None, "rectangular_mirror", 2),
    (2, (128, 64), (4, 8), None, "rectangular", 2),
    (2, (64, 32), (4, 8), (2, 1), "rectangular", 1),
    (2, (256, 128), (4, 8), (2, 1), "rectangular_mirror", 2),
    (2, (32, 32, 32), (4, 8), None, "rectangular_mirror", 2),
]


@pytest.mark.parametrize("nl,N,boxes,bar,win,red", MSWPT_CASES)
def test_mswpt_forward_inverse_adjoint(nl, N, boxes, bar, win, red):
    dev = _dev()
    w, ow = _pair(nl, N, boxes, bar, win, red)
    rng = np.random.default_rng(7)
    f = rng.standard_normal(N)
    c_ref = ow.forward(f)
    c = w.forward(torch.from_numpy(f).to(dev)).cpu().numpy()
    assert om.rel_l2(c_ref, c) < 1e-13
    # complex input
    fc = f + 1j * rng.standard_normal(N)
    assert om.rel_l2(ow.forward(fc), w.forward(torch.from_numpy(fc).to(dev)).cpu().numpy()) < 1e-13
    # inverse and inverse(forward(f)) == f
    cr = rng.standard_normal(w.total_coeffs) + 1j * rng.standard_normal(w.total_coeffs)
    inv_ref = ow.inverse(cr)
    inv = w.inverse(torch.from_numpy(cr).to(dev)).cpu().numpy()
    assert om.rel_l2(inv_ref, inv) < 1e-13
    assert om.rel_l2(fc, w.inverse(w.forward(torch.from_numpy(fc).to(dev))).cpu().numpy()) < 1e-13
    # Hermitian adjoint: oracle and dot-product identity
    adj = w.adjoint(torch.from_numpy(cr).to(dev)).cpu().numpy()
    assert om.rel_l2(ow.adjoint(cr), adj) < 1e-13
    lhs = np.vdot(cr, ow.forward(fc))
    rhs = np.vdot(adj, fc)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_mswpt_fourier_output_single_coefficient_is_frame():
    """tests/test_frames.py:359-411 through the GPU synthesis."""
    dev = _dev()
    w, ow = _pair(2, (128, 128), (4, 8))
    dec = ow.dyadic_decomp
    for idx in (5, 4000, 60000):
        c = np.zeros(w.total_coeffs)
        c[idx] = 1.0
        got = w.inverse(torch.from_numpy(c).to(dev), "fourier").cpu().numpy()
        lvl, mi = om.find_tensor_and_multiindex([idx], om.coeff_shapes(ow))
        ref = om.compute_frames(dec, mi[0, 0] + ow.boxes_cumsum[lvl[0]], mi[1:, 0], dec.fourier_meshgrid, 2,
                                "rectangular_mirror")
        assert np.allclose(ref, got, atol=1e-14, rtol=1e-12)


def _topn_gpu(keys, coeffs, n):
    from beamax_b200 import _lib

    dev = _dev()
    k = torch.from_numpy(np.ascontiguousarray(keys, np.float64)).to(dev)
    c = torch.from_numpy(np.ascontiguousarray(coeffs, np.complex128)).to(dev)
    total = keys.size
    idx = torch.empty(n, dtype=torch.int64, device=dev)
    vals = torch.empty(n, dtype=torch.complex128, device=dev)
    nb = _lib.lib().msgb_topn_workspace_size(total, n)
    ws = torch.empty(nb + 256, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().msgb_topn(k.data_ptr(), torch.view_as_real(c).data_ptr(), total, n, idx.data_ptr(),
                                    torch.view_as_real(vals).data_ptr(), ws.data_ptr(), nb, st), "topn")
    return idx.cpu().numpy(), vals.cpu().numpy()


def test_topn_bit_exact_on_identical_keys():
    rng = np.random.default_rng(0)
    c = rng.standard_normal(100_000) + 1j * rng.standard_normal(100_000)
    c[rng.integers(0, c.size, 2000)] = 0.0          # many exact ties at zero
    c[5:50] = c[3]                                   # ties at a common magnitude
    keys = om.topn_key(c)
    for n in (1, 17, 40_000, 99_990, 100_000):
        ref_idx, ref_val = om.threshold_top_n(c, n)
        idx, vals = _topn_gpu(keys, c, n)
        assert np.array_equal(ref_idx, idx), n
        assert np.array_equal(ref_val, vals)


def test_topn_tie_rule_small():
    c = np.array([0.0, 5.0, 0.0, 0.0, 5.0, 1.0], dtype=np.complex128)
    idx, _ = _topn_gpu(om.topn_key(c), c, 4)
    assert list(idx) == [3, 5, 1, 4]


def _c1_setup(nt_stride=1):
    N = (128, 128)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    dec = om.Decomp(3, N, (4, 8, 16), (1, 1))
    ow = om.Wpt(dec, 2, "rectangular_mirror")
    # two packets as in the reference example (README.md:51-72): frame atoms
    hi = om.compute_frames(dec, 125, np.array([11, 6]), dec.fourier_meshgrid, 2, "none")
    lo = om.compute_frames(dec, 44, np.array([11, 3]), dec.fourier_meshgrid, 2, "none")
    p0 = om.unitary_ifft(hi) + om.unitary_ifft(lo)
    p0 = (p0 / np.max(np.abs(p0))).T.real
    mask = np.zeros(N)
    mask[0, :] = 1
    sens = om.sensor_positions_from_mask(dom, mask)
    ts = dom.generate_time_domain()[::nt_stride]
    return dom, ow, p0, sens, ts


def _bb_objects(dom, ow):
    import beamax_b200 as bb

    d = bb.Domain(N=dom.N, dx=dom.dx, periodic=dom.periodic, cfl=dom.cfl, c=dom.c)
    dec = ow.dyadic_decomp
    w = bb.MSWPT(bb.DyadicDecomposition(dec.num_levels, dec.N, dec.num_boxes_levels, dec.box_aspect_ratio),
                 ow.redundancy, ow.windowing)
    return d, w


def test_beam_init_matches_oracle():
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c1_setup()
    d, w = _bb_objects(dom, ow)
    solver = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    sel = solver.select(p0, d, w)
    bm = om.select_beams(p0, dom, ow, 4096)
    idx = sel.idx.cpu().numpy()
    # same selected set (FFT round-off may swap exact near-ties at the threshold)
    assert np.array_equal(np.sort(idx), np.sort(bm.idx))
    bt = solver.beams(sel, d, w)
    ref = om.beams_for(idx, sel.values.cpu().numpy(), dom, ow)
    assert np.allclose(bt.x0.cpu().numpy(), ref.x0, rtol=1e-14, atol=0)
    assert np.allclose(bt.p0.cpu().numpy(), ref.p0, rtol=1e-14, atol=1e-14)
    assert np.allclose(bt.alpha.cpu().numpy(), np.diagonal(ref.M0, axis1=1, axis2=2), rtol=1e-14, atol=0)
    assert np.allclose(bt.a0_unit.cpu().numpy(), ref.a0_unit, rtol=1e-13, atol=1e-18)
    assert np.allclose(bt.omega.cpu().numpy(), ref.omega, rtol=1e-15, atol=0)


def test_forward_fp64_config1_matches_oracle():
    """Config 1 (128^2, 3 levels, thr 4096, row-0 line sensor), every 4th time sample."""
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c1_setup(nt_stride=4)
    d, w = _bb_objects(dom, ow)
    solver = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    out, params = solver.forward_with_params(p0, d, sens, ts, w)
    sel_idx = solver.last_selection.idx.cpu().numpy()
    bm = om.beams_for(sel_idx, solver.last_selection.values.cpu().numpy(), dom, ow)
    ref = ob.sum_hom(om.beam_table(bm, 1500.0), 1500.0, ts, sens, dom.grid_size, dom.periodic)
    assert out.shape == (ts.size, 128) and out.dtype == np.float64
    assert om.rel_l2(ref, out) < 1e-12
    # end to end against the oracle's own coefficients/selection
    ref_e2e, _ = om.forward(p0, dom, sens, ts, ow, 4096)
    assert om.rel_l2(ref_e2e, out) < 1e-12
    assert params[0].shape == (64, 128, 2) and params[4].shape == (64, 128)


def test_forward_fp32_config1_within_1e3():
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c1_setup(nt_stride=2)
    d, w = _bb_objects(dom, ow)
    s64 = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    s32 = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real",
                        precision="fp32")
    o64 = s64.forward(p0, d, sens, ts, w)
    o32 = s32.forward(p0, d, sens, ts, w)
    assert o32.dtype == np.float32 and np.all(np.isfinite(o32))
    assert om.rel_l2(o64, o32) < 1e-3


def _c2_small():
    """A four-sided 256^2 analogue of config 2 with culling exercised."""
    N = (256, 256)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    ow = om.Wpt(om.Decomp(3, N, (4, 8, 16), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(11)
    x = np.stack(np.meshgrid(np.arange(256), np.arange(256), indexing="ij"), -1).astype(float)
    p0 = np.zeros(N)
    for _ in range(16):
        c = rng.uniform(0.1, 0.9, 2) * 256
        th = rng.uniform(0, 2 * np.pi)
        k = rng.uniform(5, 60)
        r2 = np.sum((x - c) ** 2, -1)
        p0 += rng.standard_normal() * np.exp(-r2 / (2 * 6.0 ** 2)) * np.cos(
            2 * np.pi * k / 256 * ((x - c) @ np.array([np.cos(th), np.sin(th)])))
    p0 /= np.max(np.abs(p0))
    mask = np.zeros(N)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sens = om.sensor_positions_from_mask(dom, mask)
    ts = dom.generate_time_domain()
    return dom, ow, p0, sens, ts


def test_forward_fp32_four_sided_culled_within_1e3():
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c2_small()
    d, w = _bb_objects(dom, ow)
    s64 = bb.MSGBSolver(8192, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    s32 = bb.MSGBSolver(8192, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real",
                        precision="fp32", cutoff=16.0)
    o64 = s64.forward(p0, d, sens, ts, w)
    o32 = s32.forward(p0, d, sens, ts, w)
    dense = 2 * 8192 * ts.size * sens.shape[0]
    assert s32.eval_count() < dense  # culling removed work
    assert om.rel_l2(o64, o32) < 1e-3


def test_adjoint_fp64_matches_oracle_and_dot_test():
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c1_setup(nt_stride=4)
    d, w = _bb_objects(dom, ow)
    solver = bb.MSGBSolver(2048, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    y = solver.forward(p0, d, sens, ts, w)
    sel = solver.last_selection
    rng = np.random.default_rng(5)
    data = rng.standard_normal(y.shape)
    img = solver.adjoint(data, d, sens, ts, w)
    bm = om.beams_for(sel.idx.cpu().numpy(), sel.values.cpu().numpy(), dom, ow)
    ref = om.adjoint(bm, dom, sens, ts, ow, data)
    assert om.rel_l2(ref, img) < 1e-12
    # dot test with the selection frozen: <A q, d> == <q, A^T d>
    q = rng.standard_normal(dom.N)
    cq = w.forward_device(torch.from_numpy(q).cuda(), scale=0.5, half_mask=True)
    from beamax_b200.solvers.msgb_solver import Selection

    selq = Selection(sel.idx, cq[sel.idx], sel.total_coeffs)
    Aq = solver.sum_forward(solver.beams(selq, d, w), d, sens, ts).cpu().numpy()
    lhs = float(np.sum(Aq * data))
    rhs = float(np.sum(q * img))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_adjoint_fp32_dot_test_and_vs_fp64():
    import beamax_b200 as bb

    _dev()
    dom, ow, p0, sens, ts = _c2_small()
    d, w = _bb_objects(dom, ow)
    s64 = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    s32 = bb.MSGBSolver(4096, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real",
                        precision="fp32")
    y = s64.forward(p0, d, sens, ts, w)
    sel = s64.last_selection
    data = np.random.default_rng(1).standard_normal(y.shape)
    a64 = s64.adjoint(data, d, sens, ts, w, selection=sel)
    a32 = s32.adjoint(data, d, sens, ts, w, selection=sel)
    assert om.rel_l2(a64, a32) < 1e-3
    y32 = s32.forward(p0, d, sens, ts, w)
    lhs = float(np.sum(y32.astype(np.float64) * data))
    rhs = float(np.sum(p0 * s32.adjoint(data, d, sens, ts, w)))
    assert abs(lhs - rhs) <= 1e-3 * abs(lhs)


@pytest.mark.parametrize("nd", [1, 3])
def test_sum_fp64_other_dimensions(nd):
    import beamax_b200 as bb

    _dev()
    N = (128,) if nd == 1 else (32, 32, 32)
    boxes = (4, 8)
    dom = om.Dom(N=N, dx=(1e-4,) * nd, periodic=(False,) * nd, c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, boxes, (1,) * nd), 2, "rectangular")
    rng = np.random.default_rng(2)
    p0 = rng.standard_normal(N)
    mask = np.zeros(N)
    mask[(0,) * nd] = 1
    if nd == 3:
        mask[0, :, :] = 1
    sens = om.sensor_positions_from_mask(dom, mask)
    ts = dom.generate_time_domain()[::3]
    d, w = _bb_objects(dom, ow)
    s64 = bb.MSGBSolver(300, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "all_real")
    out = s64.forward(p0, d, sens, ts, w)
    sel = s64.last_selection
    bm = om.beams_for(sel.idx.cpu().numpy(), sel.values.cpu().numpy(), dom, ow)
    ref = om.forward_hom(bm, dom, sens, ts)
    assert om.rel_l2(ref, out) < 1e-12
    s32 = bb.MSGBSolver(300, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "all_real",
                        precision="fp32")
    assert om.rel_l2(ref, s32.forward(p0, d, sens, ts, w)) < 1e-3


def test_periodic_domain_fp64_matches_oracle():
    import beamax_b200 as bb

    _dev()
    N = (64, 64)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(True, True), c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, (4, 8), (1, 1)), 2, "rectangular")
    p0 = np.random.default_rng(4).standard_normal(N)
    sens = dom.grid.reshape(-1, 2)[::37]
    ts = np.linspace(0.0, 4e-6, 9)
    d, w = _bb_objects(dom, ow)
    s = bb.MSGBSolver(500, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "vmap_real")
    out = s.forward(p0, d, sens, ts, w)
    sel = s.last_selection
    bm = om.beams_for(sel.idx.cpu().numpy(), sel.values.cpu().numpy(), dom, ow)
    assert om.rel_l2(om.forward_hom(bm, dom, sens, ts), out) < 1e-12


def test_autograd_backward_is_adjoint():
    import beamax_b200 as bb
    from beamax_b200.solvers.autograd import msgb_forward

    dev = _dev()
    dom, ow, p0, sens, ts = _c1_setup(nt_stride=8)
    d, w = _bb_objects(dom, ow)
    solver = bb.MSGBSolver(1024, "top_n", 128, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    x = torch.from_numpy(p0).to(dev).requires_grad_(True)
    y = msgb_forward(x, solver, d, sens, ts, w)
    g = torch.randn_like(y)
    (y * g).sum().backward()
    ref = solver.adjoint(g, d, sens, ts, w, selection=solver.last_selection)
    assert torch.allclose(x.grad, ref, rtol=0, atol=0)


def test_closed_form_propagators_use_c_at_origin_and_ignore_absorption():
    """solve_hom_diag and solve_hom_general (gb/gb_solvers.py:356-481) take
    c(0) and ignore lam whatever the medium: the forward on a B-spline medium
    with absorption equals the forward on the constant medium c(0) (same
    kernels, bit for bit), and solve_hom_general equals solve_hom_diag."""
    import beamax_b200 as bb
    from scipy import ndimage

    from beamax_b200.utils.interp import make_c_function_from_grid

    _dev()
    N, dx = (64, 64), (1e-4, 1e-4)
    g = ndimage.gaussian_filter(np.random.default_rng(3).standard_normal(N), 6.0, mode="wrap")
    cgrid = 1500.0 * (1 + 0.05 * g / np.max(np.abs(g)))
    interp = make_c_function_from_grid(cgrid, dx, method="bspline3", boundary="clamp")
    c0 = float(np.asarray(interp(np.zeros((1, 2)))).ravel()[0])
    het = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=interp, lam=1e3)
    hom = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=c0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = 1
    ts = hom.generate_time_domain()
    p0 = np.random.default_rng(4).standard_normal(N)
    gs = bb.gb.gb_solvers
    outs = []
    for dom, ode in ((het, gs.solve_hom_diag), (hom, gs.solve_hom_diag), (het, gs.solve_hom_general)):
        s = bb.MSGBSolver(256, "top_n", 64, "spatial", ode, "scan_real")
        outs.append(np.asarray(s.forward(p0, dom, bb.Sensor(dom, binary_mask=mask), ts, wpt)))
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[2], outs[0])
