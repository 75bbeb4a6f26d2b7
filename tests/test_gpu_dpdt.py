"""Initial time derivative: c_pos = 0.5 (MSWPT(p0) + i MSWPT(dpdt) / vg)
(forward_solver_utils.py:716-786) on the GPU against the oracle's
compute_coefficients, and the forward with both inputs against the oracle
forward (1e-12 rel-L2); the selection indices must match exactly."""

import numpy as np
import pytest

import oracle.build as ob
from oracle import msgb as om

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def test_dpdt_coefficients_selection_and_forward_match_oracle():
    import beamax_b200 as bb

    dev = _dev()
    N = (64, 64)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(3)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    p0 = np.exp(-np.sum((xg - 30.0) ** 2, -1) / 50.0) * np.cos(0.8 * xg[..., 0])
    dpdt = 3e6 * np.exp(-np.sum((xg - 22.0) ** 2, -1) / 30.0) * np.sin(0.6 * xg[..., 1]) \
        + 1e5 * rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = mask[:, -1] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::2]
    odom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")

    s = bb.MSGBSolver(300, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    x = torch.from_numpy(p0).to(dev)
    dz = torch.from_numpy(dpdt).to(dev)
    c_gpu, _ = s._coefficients_dpdt(x, dz, dom, wpt, branch=1, half_mask=True)
    c_ref = om.compute_coefficients(p0, dpdt, "spatial", odom, ow, mode="pos_only")
    c_gpu = c_gpu.cpu().numpy()
    assert np.max(np.abs(c_gpu - c_ref)) <= 1e-12 * np.max(np.abs(c_ref))
    cn_gpu, _ = s._coefficients_dpdt(x, dz, dom, wpt, branch=-1, half_mask=False)
    _, cn_ref = om.compute_coefficients(p0, dpdt, "spatial", odom, ow, mode="both")
    assert np.max(np.abs(cn_gpu.cpu().numpy() - cn_ref)) <= 1e-12 * np.max(np.abs(cn_ref))

    y = s.forward(p0, dom, sens, ts, wpt, dpdt=dpdt)
    bm = om.select_beams(p0, odom, ow, 300, dpdt=dpdt)
    np.testing.assert_array_equal(np.sort(s.last_selection.idx.cpu().numpy()), np.sort(bm.idx))
    ref = ob.sum_hom(om.beam_table(bm, 1500.0), 1500.0, ts, sens.positions, dom.grid_size, dom.periodic)
    assert om.rel_l2(ref, y) < 1e-12
