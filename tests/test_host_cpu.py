"""CPU tests: the C ABI library, host metadata and argument validation.

No compute is launched here (no GPU); these tests load libmsgb.so, check that
it exports every entry point declared in include/msgb.h, and check the
host-side objects against the oracle and the reference's validation rules.
"""

import os
import re

import numpy as np
import pytest

import beamax_b200 as bb
from beamax_b200 import _lib
from oracle import msgb as om

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "msgb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(msgb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes

    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if getattr(lib, s, None) is None]
    assert not missing, missing
    assert set(declared) <= set(_lib.SIGNATURES), set(declared) - set(_lib.SIGNATURES)
    assert _lib.missing_symbols() == []


def test_version_and_error_strings():
    assert b"sm_100a" in _lib.lib().msgb_version()
    assert isinstance(_lib.last_error(), str)


def test_null_arguments_rejected_without_gpu():
    L = _lib.lib()
    assert L.msgb_sum_fwd_f64(None, None, None, None) == 1
    assert "problem descriptor is NULL" in _lib.last_error()
    assert L.msgb_topn(None, None, 10, 5, None, None, None, 0, None) == 1
    assert L.msgb_mswpt_forward(None, None, 0, 0, 1.0, 0, None, None, None, 0, None) == 1


@pytest.mark.parametrize("nl,N,boxes,bar,win", [
    (3, (128, 128), (4, 8, 16), (1, 1), "rectangular_mirror"),
    (2, (256, 128), (4, 8), (2, 1), "rectangular"),
    (2, (32, 32, 32), (4, 8), (1, 1, 1), "rectangular"),
    (2, (128,), (4, 8), (1,), "rectangular_mirror"),
])
def test_host_metadata_matches_oracle(nl, N, boxes, bar, win):
    w = bb.MSWPT(bb.DyadicDecomposition(nl, N, boxes, bar), 2, win)
    ow = om.Wpt(om.Decomp(nl, N, boxes, bar), 2, win)
    assert np.array_equal(w.dyadic_decomp.centres_ndim, ow.dyadic_decomp.centres_ndim)
    assert w.coeff_shapes == ow.coeff_shapes and w.coeffs_cumsum == ow.coeffs_cumsum
    assert np.array_equal(w.sum_gsquare, ow.sum_gsquare)
    for a, b in zip(w.gfilts_packed, ow.gfilts_packed):
        assert np.array_equal(a, b)
    assert np.array_equal(w.half_mask, ow.half_mask)


def test_lattice_tables_cover_every_box():
    dec = bb.DyadicDecomposition(4, (512, 512), (4, 8, 16, 32), (1, 1))
    w = bb.MSWPT(dec, 2, "rectangular_mirror")
    d, keep = w._descriptor()
    tab = keep["lattice_box"]
    assert sorted(tab[tab >= 0].tolist()) == list(range(dec.total_num_boxes))


def test_decomposition_rejections():
    with pytest.raises(ValueError, match="at least 2 Fourier samples"):
        bb.DyadicDecomposition(5, (1024, 1024), (4, 8, 16, 32, 64), (1, 1))
    with pytest.raises(ValueError, match="expected 15 centres"):
        bb.DyadicDecomposition(5, (1024, 1024), (2, 4, 8, 16, 32), (1, 1))
    with pytest.raises(ValueError, match="must be even"):
        bb.DyadicDecomposition(1, (63, 64), (4,), (1, 1))


def test_solver_validation_messages():
    s = bb.gb.gb_solvers.solve_hom_diag
    with pytest.raises(ValueError, match="thr_strat must be one of"):
        bb.MSGBSolver(10, "bogus", 4, "spatial", s, "scan_real")
    with pytest.raises(ValueError, match="top_n threshold must be a positive integer"):
        bb.MSGBSolver(1.5, "top_n", 4, "spatial", s, "scan_real")
    with pytest.raises(ValueError, match="percentile threshold must lie"):
        bb.MSGBSolver(101, "percentile", 4, "spatial", s, "scan_real")
    with pytest.raises(ValueError, match="sum_method must be one of"):
        bb.MSGBSolver(10, "top_n", 4, "spatial", s, "sum_all")
    with pytest.raises(ValueError, match="batch_size must be positive"):
        bb.MSGBSolver(10, "top_n", 0, "spatial", s, "scan_real")
    with pytest.raises(ValueError, match="Unsupported ode_solver"):
        bb.MSGBSolver(10, "top_n", 4, "spatial", "rk45", "scan_real")
    with pytest.raises(ValueError, match="precision must be"):
        bb.MSGBSolver(10, "top_n", 4, "spatial", s, "scan_real", precision="fp16")


def test_effective_top_n_caps_at_half_frame():
    w = bb.MSWPT(bb.DyadicDecomposition(1, (16,), (4,), (1,)), 2, "rectangular")
    s = bb.MSGBSolver(10_000, "top_n", 4, "spatial", "solve_ODE_base", "all_real")
    assert s._effective_top_n(w, half_frame=True) == w.half_frame_capacity() == 16
    assert s._effective_top_n(w) == w.total_coeffs


def test_time_grid_validation():
    from beamax_b200.solvers.msgb_solver import _validate_time_grid

    assert _validate_time_grid(np.array([0.0])) is None if False else True
    with pytest.raises(ValueError, match="uniformly spaced"):
        _validate_time_grid(np.array([0.0, 1.0, 3.0]))
    assert _validate_time_grid(np.array([0.0]), allow_singleton=True) is None
    assert _validate_time_grid(np.arange(5) * 0.5) == 0.5


def test_domain_and_sensor_match_reference_conventions():
    d = bb.Domain(N=(8, 6), dx=(1e-4, 2e-4), periodic=(False, False), c=1500.0, cfl=0.3)
    od = om.Dom(N=(8, 6), dx=(1e-4, 2e-4), periodic=(False, False), c=1500.0, cfl=0.3)
    assert np.array_equal(d.generate_time_domain(), od.generate_time_domain())
    mask = np.zeros((8, 6))
    mask[0, :] = 1
    mask[:, 0] = 1
    s = bb.Sensor(d, binary_mask=mask)
    assert np.array_equal(s.positions, om.sensor_positions_from_mask(od, mask))
    with pytest.raises(ValueError, match="Cannot provide both"):
        bb.Sensor(d, positions=s.positions, binary_mask=mask)
    with pytest.raises(ValueError, match="half-open domain"):
        bb.Sensor(d, positions=np.array([[1.0, 1.0]]))
    assert d.constant_speed() == 1500.0
    assert bb.Domain(N=(4, 4), dx=(1.0, 1.0), periodic=(True, True), c=lambda x: 2.0 + 0 * x[..., 0]).constant_speed() == 2.0


def test_adjoint_seven_argument_form_is_the_principal_symbol_adjoint():
    """adjoint(data, domain, sensors, sources, ts, data_domain, data_wpt) takes
    the reference's principal-symbol path and its checks (msgb_solver.py:
    1339-1356, 806-856), before any device work."""
    s, dom, ts, ddom, wpt, src, data = _tr_case()
    img = bb.Sensor(dom, binary_mask=np.ones(dom.N))
    per = bb.Domain(N=dom.N, dx=dom.dx, periodic=(True, True), cfl=0.3, c=1500.0)
    with pytest.raises(ValueError, match="non-periodic spatial boundaries"):
        s.adjoint(data, per, img, src, ts, ddom, wpt)
    with pytest.raises(ValueError, match="Unsupported sensor type for `sensors` in adjoint"):
        s.adjoint(data, dom, object(), src, ts, ddom, wpt)
    with pytest.raises(ValueError, match="Boundary data must have shape"):
        s.adjoint(data=data[:, :-1], domain=dom, sensors=img, sources=src, ts=ts, data_domain=ddom,
                  data_wpt=wpt, window=np.ones(data.shape[0]))
    with pytest.raises(TypeError):
        s.adjoint(data, dom, img, src, ts, ddom, wpt, p0=np.zeros(dom.N))


def test_solver_config_matches_reference_checks():
    """SolverConfig (gb/gb_solvers.py:597-703): defaults, validation, precision presets."""
    from beamax_b200.gb.gb_solvers import SolverConfig, ode_method

    cfg = SolverConfig()
    assert (cfg.rtol, cfg.atol, cfg.max_steps, cfg.dt0) == (1e-7, 1e-9, 4096, None)
    assert cfg.method == "dopri5"
    assert SolverConfig.from_precision(use_x64=False).rtol == 1e-4
    assert SolverConfig.from_precision(rtol=1e-5, max_steps=10000).max_steps == 10000
    assert SolverConfig(solver="rk4", substeps=4).method == "rk4"
    for bad in ({"max_steps": 0}, {"max_steps": True}, {"rtol": 0.0}, {"atol": float("nan")}, {"dt0": -1.0},
                {"pcoeff": float("inf")}, {"solver": "euler"}, {"substeps": 0}):
        with pytest.raises(ValueError):
            SolverConfig(**bad)
    with pytest.raises(NotImplementedError):
        SolverConfig(pcoeff=0.3)

    class Tsit5:
        pass

    assert ode_method(Tsit5()) == "dopri5"
    solver = bb.MSGBSolver(8, "top_n", 8, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real")
    assert solver.ode_config == SolverConfig()
    with pytest.raises(TypeError):
        bb.MSGBSolver(8, "top_n", 8, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real", ode_config={})


def _tr_case(N=(32, 32)):
    dom = bb.Domain(N=N, dx=(1e-4,) * len(N), periodic=(False,) * len(N), cfl=0.3, c=1500.0)
    ts = dom.generate_time_domain()
    Nd = (2 * N[0],) + tuple(N[1:])
    ddom = bb.Domain(N=Nd, dx=(float(ts[-1] / (Nd[0] - 1)),) + (1e-4,) * (len(N) - 1),
                     periodic=(False,) * len(N), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, Nd, (4, 8), (2, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = 1
    src = bb.Sensor(dom, binary_mask=mask)
    s = bb.MSGBSolver(200, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real")
    return s, dom, ts, ddom, wpt, src, np.zeros(Nd)


def test_time_reversal_input_checks_match_reference():
    """msgb_solver.py:1079-1082 and :806-856 (checked before any device work)."""
    s, dom, ts, ddom, wpt, src, data = _tr_case()
    img = bb.Sensor(dom, binary_mask=np.ones(dom.N))
    per = bb.Domain(N=dom.N, dx=dom.dx, periodic=(True, True), cfl=0.3, c=1500.0)
    with pytest.raises(ValueError, match="only supports free space boundary"):
        s.time_reversal(data, per, img, src, ts, ddom, wpt)
    with pytest.raises(ValueError, match="Boundary data must have shape"):
        s.time_reversal(data[:-1], dom, img, src, ts, ddom, wpt)
    with pytest.raises(ValueError, match="ts spans"):
        s.time_reversal(data, dom, img, src, ts[:-5], ddom, wpt)
    with pytest.raises(ValueError, match="sources must be a Sensor"):
        s.time_reversal(data, dom, img, np.asarray(src.positions), ts, ddom, wpt)
    tilted = bb.Sensor(dom, positions=np.stack([np.arange(32) * 1e-4, np.arange(32) * 1e-4], 1))
    with pytest.raises(ValueError, match="axis-aligned planar surface"):
        s.time_reversal(data, dom, img, tilted, ts, ddom, wpt)
    half = bb.Sensor(dom, positions=np.stack([np.zeros(16), np.arange(16) * 1e-4], 1))
    with pytest.raises(ValueError, match="detector axes do not match"):
        s.time_reversal(data, dom, img, half, ts, ddom, wpt)


def test_time_reversal_detector_geometry():
    """Normal axis and inward sign of the detector (tr_solver_utils.py:241-251,
    377-393): first row -> axis 0 inward +1, last row -> -1, first column ->
    axis 1."""
    s, dom, ts, ddom, wpt, src, data = _tr_case()
    g = s._tr_geometry(src)
    assert (g.normal_axis, g.normal_value, g.inward) == (0, 0.0, 1.0)
    mask = np.zeros(dom.N)
    mask[-1, :] = 1
    g = s._tr_geometry(bb.Sensor(dom, binary_mask=mask))
    assert (g.normal_axis, g.inward) == (0, -1.0) and g.normal_value == pytest.approx(31e-4)
    mask = np.zeros(dom.N)
    mask[:, 0] = 1
    g = s._tr_geometry(bb.Sensor(dom, binary_mask=mask))
    assert (g.normal_axis, g.normal_value, g.inward) == (1, 0.0, 1.0)


def test_reference_propagator_names_are_accepted():
    """gb_solvers.solve_hom_general and solve_hom_TR (gb/gb_solvers.py:425-594)
    are accepted by name or object; the closed forms are marked as such."""
    gs = bb.gb.gb_solvers
    for ode, closed in ((gs.solve_hom_general, True), ("solve_hom_general", True), (gs.solve_hom_diag, True),
                        (gs.solve_ODE_base, False)):
        s = bb.MSGBSolver(8, "top_n", 8, "spatial", ode, "scan_real", tr_ode_solver=gs.solve_hom_TR)
        assert s.closed_form is closed


def test_bench_reports_the_dominant_kernel():
    """bench.py's roofline object is the kernel with the largest device time
    per step, with its algorithmic cost per work unit: the summation kernels
    (flops per evaluated triple, measured FP32 peak) and, in heterogeneous
    media, the FP32 path's mixed-precision beam ODE (FP32 flops per attempted
    step against the FP32 peak, its FP64 ray flops against the FP64 peak)."""
    import types

    import bench

    args = types.SimpleNamespace(thr=65536, workload="c2")
    peaks = {"fp32": 70.0, "fp32x2": 72.0, "fp32_best": 72.0, "fp64": 36.0, "mufu": 4.6, "method": "probe"}
    r = {"hetero": False, "fwd_evals": 8e10, "adj_evals": 8e10, "t_fwd_kernel": 0.08, "t_adj_kernel": 0.09,
         "t_ode": 0.0, "ode_steps": 0, "ndim": 2}
    first, other = bench.rooflines(r, peaks, 1965.0, args)
    assert (first["kernel"], other[0]["kernel"]) == ("adj32_kernel", "fwd32_kernel")
    assert first["flops_per_eval"] == 40.0 and other[0]["flops_per_eval"] == 36.0
    assert abs(first["frac"] - 8e10 * 40 / 0.09 / 1e12 / 72.0) < 1e-12
    assert abs(first["mufu"]["frac"] - 3 * 8e10 / 0.09 / 1e12 / 4.6) < 1e-12
    r["t_fwd_kernel"] = 0.1
    assert bench.rooflines(r, peaks, 1965.0, args)[0]["kernel"] == "fwd32_kernel"
    r.update(hetero=True, t_ode=4.0, ode_steps=3e9)
    first, other = bench.rooflines(r, peaks, 1965.0, args)
    assert first["kernel"] == "dopri_mix_kernel" and first["bound"] == "fp32"
    f64, f32 = bench.ode_flops_split(2)
    assert f64 + f32 == bench.ode_flops_per_step(2) and 0 < f64 < f32
    f64_3, f32_3 = bench.ode_flops_split(3)
    assert f64_3 + f32_3 == bench.ode_flops_per_step(3) and 0 < f64_3 < f32_3
    assert abs(first["frac"] - 3e9 * f32 / 4.0 / 1e12 / 72.0) < 1e-12
    assert abs(first["fp64"]["frac"] - 3e9 * f64 / 4.0 / 1e12 / 36.0) < 1e-12
    assert [e["kernel"] for e in other] == ["fwd32_kernel<TRAJ>", "adj32_kernel<TRAJ>"]


def test_infer_planar_surface_matches_reference():
    """MSGBSolver._infer_planar_surface (tests/solvers/test_msgb_solver_misc.py:
    116-141): axis, coordinate and implicit function of a planar detector;
    generic positions are rejected."""
    s = bb.MSGBSolver(4, "top_n", 4, "spatial", "solve_hom_diag", "all_real")
    y = np.linspace(0.0, 1.0, 5)
    surface, axis, coord = s._infer_planar_surface(np.stack([np.full_like(y, 2.0), y], 1))
    assert axis == 0 and coord == pytest.approx(2.0)
    assert float(surface(np.array([2.0, 0.5]))) == pytest.approx(0.0)
    assert float(surface(np.array([3.0, 0.5]))) == pytest.approx(1.0)
    with pytest.raises(ValueError, match="planar surface"):
        s._infer_planar_surface(np.array([[0.0, 0.0], [1.0, 0.5], [0.3, 0.8], [0.7, 0.2]]))


def test_forward_rejects_unsupported_sensor_type():
    """tests/solvers/test_msgb_solver_misc.py:160-166."""
    dom = bb.Domain(N=(128,), dx=(1.0 / 128,), periodic=(False,), c=1.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(2, (128,), (4, 8), (1,)), 2, "rectangular")
    s = bb.MSGBSolver(4, "top_n", 4, "spatial", "solve_hom_diag", "all_real")
    with pytest.raises(ValueError, match="Unsupported sensor type"):
        s.forward(np.zeros(dom.N), dom, "not_a_sensor", np.linspace(0.0, 1.0, 8), wpt)


@pytest.mark.parametrize("threshold,strategy,match", [
    (0, "top_n", "positive integer"),
    (1.5, "top_n", "positive integer"),
    (-1.0, "hard", "non-negative"),
    (101.0, "percentile", r"\[0, 100\]"),
    (1.1, "perc_max_abs", r"\[0, 1\]"),
])
def test_threshold_configuration_is_validated(threshold, strategy, match):
    """tests/solvers/test_msgb_solver_misc.py:424-446."""
    with pytest.raises(ValueError, match=match):
        bb.MSGBSolver(threshold, strategy, 4, "spatial", bb.gb.gb_solvers.solve_ODE_base, "all_real")


def test_problem_struct_owns_its_device_arrays():
    """The problem struct keeps the time and sensor arrays it points at alive,
    whatever the caller does with the second return value (a rebound name
    once let the allocator hand the time array to another tensor while the
    kernels still read it)."""
    import gc

    pytest.importorskip("torch")
    dom = bb.Domain(N=(32, 32), dx=(1e-4, 1e-4), c=1500.0, cfl=0.3, periodic=(False, False))
    mask = np.zeros((32, 32))
    mask[0, :] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[:10]
    s = bb.MSGBSolver(64, "top_n", 16, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real")
    pr, held = s._problem(dom, sens, ts, "cpu")
    ptr = held[0].data_ptr()
    del held
    gc.collect()
    assert pr.ts == ptr and pr._owned[0].data_ptr() == ptr
    assert np.array_equal(pr._owned[0].numpy(), np.asarray(ts, np.float64))


def test_callable_sound_speed_is_sampled_once_onto_a_bspline():
    """A Python callable c(x) (geometry.py:176-190) becomes the cubic B-spline
    of its grid samples: equal to c at every node, built once per value of
    c (the device caches and kept trajectories key on that object)."""
    dom = bb.Domain(N=(24, 20), dx=(1e-4, 2e-4), periodic=(False, False), cfl=0.3,
                    c=lambda x: 1500.0 * (1.0 + 0.05 * np.sin(900.0 * x[..., 0]) * np.cos(700.0 * x[..., 1])))
    kind, m = dom.medium()
    assert kind == "grid" and m.method == "bspline3" and m.boundary == "nearest"  # clamp
    assert dom.medium()[1] is m
    xs = np.stack(np.meshgrid(np.arange(24) * 1e-4, np.arange(20) * 2e-4, indexing="ij"), -1)
    ref = 1500.0 * (1.0 + 0.05 * np.sin(900.0 * xs[..., 0]) * np.cos(700.0 * xs[..., 1]))
    assert np.allclose(np.asarray(m(xs.reshape(-1, 2))).reshape(24, 20), ref, rtol=1e-12, atol=1e-9)
    const = bb.Domain(N=(8, 8), dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=lambda x: 1480.0 + 0.0 * x[..., 0])
    assert const.medium() == ("constant", 1480.0)
    dom.c = lambda x: 1500.0 + 0.0 * x[..., 0] + 10.0 * x[..., 1]
    assert dom.medium()[1] is not m


@pytest.mark.parametrize("workload", ["c2", "het512"])
def test_bench_reference_arm_prints_the_contract_line(workload):
    """`bench.py --impl reference` (the CPU restatement on a bounded beam
    sample): one JSON line with the metric, a cpu_baseline describing the run
    and an e2e object with no host-device copies."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload", workload,
                          "--cpu-sample", "2", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=root, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "evals/s"
    assert line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and "2 of" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_compact_store_layout_stays_inside_its_buffer():
    """The compact trajectory store's slot table, block counter, culling boxes
    and record pool, as _compact_tr lays them out in one buffer: disjoint,
    aligned, and inside the buffer for every buffer size (the device kernels
    index them without a bounds check beyond pool_blocks)."""
    torch = pytest.importorskip("torch")
    s = bb.MSGBSolver(64, "top_n", 16, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real", precision="fp32")
    rng = np.random.default_rng(0)
    for _ in range(200):
        d = int(rng.integers(1, 4))
        nt = int(rng.integers(1, 6000))
        nb = int(rng.integers(1, 5000))
        n_tt, block, cull = s._compact_sizes(d, nt)
        size = int(rng.integers(n_tt * nb * 4 + 1024, n_tt * nb * 4 + 2048 + 200 * (block + cull)))
        buf = torch.empty(size, dtype=torch.uint8)
        status = torch.zeros(nb + 8, dtype=torch.int32)
        boxes = torch.zeros((4, 2 * d), dtype=torch.float32)
        tr, blocks, ctr = s._compact_tr(buf, d, nt, 3, nb, status, boxes, 4)
        base = buf.data_ptr()
        slot_end = tr.slot - base + n_tt * nb * 4
        ctr_off, cull_off, pool_off = tr.pool_next - base, tr.pool_cull - base, tr.pool - base
        assert tr.slot == base and slot_end <= ctr_off and ctr_off + 8 <= cull_off
        assert blocks >= 0 and tr.pool_blocks == blocks
        assert cull_off + blocks * cull <= pool_off and pool_off % 256 == 0
        assert pool_off + blocks * block <= size
        assert ctr.numel() == 1 and ctr.data_ptr() == tr.pool_next
        assert tr.status == status.data_ptr() + 4 * 3 and tr.nb == nb and tr.b_first == 3
