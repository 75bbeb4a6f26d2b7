"""GPU thresholds other than top_n against the oracle's restatement of
threshold_coefficients (forward_solver_utils.py:14-230).

Indices must match exactly (ascending, the jnp.nonzero order; the -1 padding
of percentile / perc_max_abs describes zero-amplitude beams and is dropped),
values to 1e-13 relative (hard_reassign scales by an energy ratio whose
summation order differs).  The full FP64 forward with each strategy matches
the oracle forward to 1e-12 rel-L2.
"""

import numpy as np
import pytest

import oracle.build as ob
from oracle import msgb as om

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STRATEGIES = [("hard", 0.02), ("percentile", 97.0), ("hard_reassign", 0.1), ("bao_energy", 5.0),
              ("perc_max_abs", 0.05)]


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _case():
    import beamax_b200 as bb

    N = (64, 64)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(7)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - 30.0) ** 2, -1) / 50.0) * np.cos(0.8 * xg[..., 0]) + 0.05 * rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = mask[:, 0] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::2]
    odom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    return dom, wpt, p0, sens, ts, odom, ow


@pytest.mark.parametrize("strategy,val", STRATEGIES)
def test_threshold_matches_oracle(strategy, val):
    import beamax_b200 as bb

    dev = _dev()
    dom, wpt, p0, sens, ts, odom, ow = _case()
    s = bb.MSGBSolver(val, strategy, 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    sel = s.select(p0, dom, wpt)
    coeffs = wpt.forward_device(torch.from_numpy(p0).to(dev), scale=0.5, half_mask=True).cpu().numpy()
    idx, vals = om.threshold_coefficients(coeffs, val, strategy, ow)
    keep = idx >= 0
    idx, vals = idx[keep], vals[keep]
    g_idx, g_vals = sel.idx.cpu().numpy(), sel.values.cpu().numpy()
    assert 0 < idx.size < coeffs.size
    np.testing.assert_array_equal(g_idx, idx)
    assert np.max(np.abs(g_vals - vals)) <= 1e-13 * np.max(np.abs(vals))


@pytest.mark.parametrize("strategy,val", STRATEGIES)
def test_forward_with_threshold_matches_oracle(strategy, val):
    import beamax_b200 as bb

    _dev()
    dom, wpt, p0, sens, ts, odom, ow = _case()
    s = bb.MSGBSolver(val, strategy, 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    y = s.forward(p0, dom, sens, ts, wpt)
    cpos = om.compute_coefficients(p0, np.zeros_like(p0), "spatial", odom, ow, mode="pos_only")
    idx, vals = om.threshold_coefficients(cpos, val, strategy, ow)
    k = idx >= 0  # padding: zero-amplitude beams
    bm = om.beams_for(idx[k], vals[k], odom, ow)
    ref = ob.sum_hom(om.beam_table(bm, 1500.0), 1500.0, ts, sens.positions, dom.grid_size, dom.periodic)
    assert om.rel_l2(ref, y) < 1e-12
