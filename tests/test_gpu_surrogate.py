"""Trajectory surrogate: target map, training gain, fallback keeps accuracy.

The surrogate has no counterpart in the reference.  Its checks:
  * the target map and its inverse (msgb_surrogate_targets, then
    msgb_surrogate_records on the exact targets) reproduce the ODE records to
    FP32 rounding of the corrections;
  * trained on ODE trajectories, the MLP's held-out RMS position error is at
    least 5x smaller than that of the straight rays it corrects (the gain);
  * with the acceptance rule the FP32 forward stays within 1e-3 rel-L2 of the
    FP64 ODE forward, however many beams the rule accepts.
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


def _case(N=(64, 64), thr=200, seed=0, corr=5.0):
    from scipy import ndimage

    import beamax_b200 as bb
    from beamax_b200.utils.interp import make_c_function_from_grid

    dx = (1e-4, 1e-4)
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(N), corr, mode="wrap")
    c = 1500.0 * (1 + 0.08 * np.clip(g / np.max(np.abs(g)), -1, 1))
    interp = make_c_function_from_grid(c, dx, method="bspline3", boundary="clamp")
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=interp)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - np.asarray(N) / 2) ** 2, -1) / 40.0) * np.cos(0.9 * xg[..., 0])
    p0 = p0 + 0.3 * rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::3]
    return dom, wpt, p0, sens, ts, thr


def _solver(thr, **kw):
    import beamax_b200 as bb

    return bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real", **kw)


def test_target_map_round_trip():
    from beamax_b200 import _lib
    from beamax_b200.surrogate import TrajectorySurrogate

    dev = _dev()
    dom, wpt, p0, sens, ts, thr = _case(thr=24)
    s = _solver(thr)
    bt = s.beams(s.select(p0, dom, wpt), dom, wpt)
    pr, keep = s._problem(dom, sens, ts, dev)
    med, keep_m = s._medium(dom, dev)
    bs = bt.beam_set(unit=True)
    nb = 2 * bt.n
    sur = TrajectorySurrogate()
    sur.device = dev
    rec, status = sur._ode_rec64(s, pr, med, bs, nb)
    assert int(status.max()) == 0
    ld = 16
    st = torch.cuda.current_stream().cuda_stream
    Y = torch.empty((pr.nt * nb, ld), dtype=torch.float32, device=dev)
    io = _lib.SurrogateIO(nb=nb, b_first=0, nq_t=pr.nt, t_index=None, ld=ld)
    _lib.check(_lib.lib().msgb_surrogate_targets(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                 rec.data_ptr(), Y.data_ptr(), st), "targets")
    back = torch.empty_like(rec)
    st2 = torch.full((nb,), -1, dtype=torch.int32, device=dev)
    tr = _lib.Trajectories(nb=nb, b_first=0, rec64=back.data_ptr(), status=st2.data_ptr())
    acc = _lib.SurrogateAccept(residual_tol=1e-6, phase_tol=1.0, pos_err=0.0)
    zero, one = torch.zeros(ld, device=dev), torch.ones(ld, device=dev)
    _lib.check(_lib.lib().msgb_surrogate_records(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(io),
                                                 Y.data_ptr(), zero.data_ptr(), one.data_ptr(), _lib.ref(acc),
                                                 _lib.ref(tr), st), "records")
    torch.cuda.synchronize()
    r, b = rec.cpu().numpy(), back.cpu().numpy()
    d = 2
    # the corrections are FP32 (relative rounding 6e-8 of a deviation up to ~c0 T / 4)
    assert np.max(np.abs(b[..., :d] - r[..., :d])) <= 1e-7 * np.max(np.abs(r[..., :d]))
    assert np.max(np.abs(b[..., d:2 * d] - r[..., d:2 * d])) <= 1e-6 * np.max(np.abs(r[..., d:2 * d]))
    M, Mb = r[..., 2 * d:2 * d + 2 * d * d], b[..., 2 * d:2 * d + 2 * d * d]
    assert np.max(np.abs(Mb - M)) <= 1e-5 * np.max(np.abs(M))
    assert np.max(np.abs(b[..., -2:] - r[..., -2:])) <= 1e-5 * np.max(np.abs(r[..., -2:]))
    # exact states satisfy the Hamiltonian invariant far below 1e-6
    assert (st2.cpu().numpy() == 0).all()


def test_surrogate_training_beats_straight_rays():
    """The gain: on held-out beams the RMS position error is 5x below that of
    the straight rays the network corrects (8 % speed contrast, 10-cell
    correlation, 6,000 training beams)."""
    from beamax_b200.surrogate import TrajectorySurrogate

    _dev()
    dom, wpt, p0, sens, ts, thr = _case(thr=4096, corr=10.0)
    s = _solver(thr)
    bt = s.beams(s.select(p0, dom, wpt), dom, wpt)
    sur = TrajectorySurrogate(seed=1).fit(s, dom, sens, ts, bt, n_train=3000, n_val=256, t_stride=2, epochs=60,
                                          batch=8192, lr=2e-3)
    st = sur.stats
    print("surrogate stats", st)
    assert st["loss_last"] < 0.25 * st["loss_first"]
    assert st["pos_rms"] < st["pos_rms_straight"] / 5
    assert st["pos_err"] < st["pos_err_straight"]


def test_forward_with_surrogate_keeps_accuracy():
    from beamax_b200.surrogate import TrajectorySurrogate

    _dev()
    dom, wpt, p0, sens, ts, thr = _case(thr=300, seed=2)
    ref = _solver(thr)
    y64 = ref.forward(p0, dom, sens, ts, wpt)
    bt = ref.beams(ref.last_selection, dom, wpt)
    sur = TrajectorySurrogate(seed=0).fit(ref, dom, sens, ts, bt, n_train=220, n_val=60, t_stride=2, epochs=20,
                                          batch=4096)
    s32 = _solver(thr, precision="fp32", surrogate=sur)
    y32 = s32.forward(p0, dom, sens, ts, wpt)
    n_beams = 2 * bt.n
    print("accepted", s32.last_surrogate_accepted, "of", n_beams, sur.stats)
    assert 0 <= s32.last_surrogate_accepted <= n_beams
    assert om.rel_l2(y64, y32) < 1e-3
    # accepting every prediction shows what the rule protects against
    loose = TrajectorySurrogate(residual_tol=1e9, phase_tol=1e30, seed=0)
    loose.__dict__.update({k: v for k, v in sur.__dict__.items() if k not in ("residual_tol", "phase_tol")})
    s_all = _solver(thr, precision="fp32", surrogate=loose)
    y_all = s_all.forward(p0, dom, sens, ts, wpt)
    assert s_all.last_surrogate_accepted == n_beams
    err_all = om.rel_l2(y64, y_all)
    print("rel-L2 with every prediction accepted", err_all)
    assert np.isfinite(err_all)
