"""msgb_sum_fwd_f32_static: the FP32 forward for callers that cannot allocate.

Some hosts have no device allocator to lend this library (an XLA custom call
without a scratch buffer, a runtime whose memory belongs to another
framework's pool), so this entry point takes its scratch from a fixed array
compiled into the library.  Its output must match msgb_sum_fwd_f32 with a
caller workspace on the same inputs.  Two different problems are run back to
back through the shared array, so the second call also shows that what the
first left behind does not leak into its result.  The file sorts last so that
it runs after every other GPU test, and it passes in a fresh process as well.
"""

import ctypes

import numpy as np
import pytest

from oracle import msgb as om

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STATIC_BYTES = 16 << 20


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _case(N, thr, seed, interior_sensors):
    """(problem, beam set, options, tensors kept alive) as MSGBSolver builds them."""
    import beamax_b200 as bb
    from beamax_b200 import _lib

    dev = _dev()
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    wpt = bb.MSWPT(bb.DyadicDecomposition(3, N, (4, 8, 16), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(seed)
    xg = np.stack(np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij"), -1).astype(float)
    ctr = np.asarray(N) / 2
    p0 = np.exp(-np.sum((xg - ctr) ** 2, -1) / 60.0) * np.cos(0.7 * xg[..., 0]) + 0.2 * rng.standard_normal(N)
    mask = np.zeros(N)
    if interior_sensors:
        mask[rng.integers(4, N[0] - 4, 300), rng.integers(4, N[1] - 4, 300)] = 1
    else:
        mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sens = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()[::2]
    solver = bb.MSGBSolver(thr, "top_n", 64, "spatial", bb.gb.gb_solvers.solve_hom_diag, "scan_real",
                           precision="fp32")
    sel = solver.select(p0, dom, wpt)
    bt = solver.beams(sel, dom, wpt)
    pr, keep_p = solver._problem(dom, sens, ts, dev)
    bs = bt.beam_set(unit=False)
    tiling = solver._tiling(dom, sens, dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    opts = _lib.SumOpts(cutoff=solver.cutoff, eval_count=cnt.data_ptr(),
                        tiling=_lib.ref(tiling[0]) if tiling else None)
    return pr, bs, opts, (keep_p, bt, tiling, cnt)


def _with_workspace(pr, bs, opts):
    from beamax_b200 import _lib

    dev = _dev()
    nbytes = _lib.lib().msgb_sum_f32_workspace_size(_lib.ref(pr), bs.n)
    ws = torch.full((nbytes + 256,), 0x5A, dtype=torch.uint8, device=dev)
    out = torch.empty((pr.nt, pr.ns), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().msgb_sum_fwd_f32(_lib.ref(pr), _lib.ref(bs), _lib.ref(opts), ws.data_ptr(), nbytes,
                                           out.data_ptr(), st), "msgb_sum_fwd_f32")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _static(pr, bs, opts):
    from beamax_b200 import _lib

    dev = _dev()
    out = torch.full((pr.nt, pr.ns), float("nan"), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().msgb_sum_fwd_f32_static(_lib.ref(pr), _lib.ref(bs), _lib.ref(opts), out.data_ptr(), st),
               "msgb_sum_fwd_f32_static")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_scratch_forward_matches_workspace_forward_on_two_calls():
    """Two problems of different shapes through the static scratch, each equal
    to the workspace entry point within 1e-6 rel-L2 (the FP32 path's own
    tolerance against FP64 is 1e-3; the same kernels on the same inputs are
    expected to agree far more closely)."""
    first = _case((128, 128), 1500, 0, interior_sensors=False)
    second = _case((256, 256), 4000, 1, interior_sensors=True)
    for pr, bs, opts, _keep in (first, second):
        got = _static(pr, bs, opts)
        want = _with_workspace(pr, bs, opts)
        assert np.isfinite(got).all()
        assert om.rel_l2(want.astype(np.float64), got.astype(np.float64)) < 1e-6


def test_static_scratch_rejects_problems_beyond_its_size():
    """A problem whose scratch exceeds the array fails before any launch, with
    the bytes it needs in the message; the library stays usable."""
    from beamax_b200 import _lib

    pr, bs, opts, keep = _case((128, 128), 1500, 0, interior_sensors=False)
    big = _lib.BeamSet(n=1 << 22, x0=bs.x0, p0=bs.p0, alpha=bs.alpha, a0=bs.a0, omega=bs.omega)
    out = torch.empty((pr.nt, pr.ns), dtype=torch.float32, device=_dev())
    st = torch.cuda.current_stream().cuda_stream
    status = _lib.lib().msgb_sum_fwd_f32_static(_lib.ref(pr), _lib.ref(big), _lib.ref(opts), out.data_ptr(), st)
    assert status == 4  # MSGB_ERR_UNSUPPORTED
    msg = _lib.last_error()
    assert "static scratch" in msg and str(STATIC_BYTES) in msg
    got = _static(pr, bs, opts)
    assert om.rel_l2(_with_workspace(pr, bs, opts).astype(np.float64), got.astype(np.float64)) < 1e-6


def test_static_scratch_forward_allocates_no_device_memory():
    """After a warm-up call (module load, symbol lookup), a further call leaves
    the device's free memory and torch's allocated bytes unchanged: the entry
    point takes its scratch from the array, not from an allocator."""
    from beamax_b200 import _lib

    dev = _dev()
    pr, bs, opts, keep = _case((128, 128), 1500, 0, interior_sensors=False)
    out = torch.empty((pr.nt, pr.ns), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    call = lambda: _lib.check(_lib.lib().msgb_sum_fwd_f32_static(_lib.ref(pr), _lib.ref(bs), _lib.ref(opts),
                                                                  out.data_ptr(), st), "msgb_sum_fwd_f32_static")
    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    alloc0 = torch.cuda.memory_allocated(dev)
    call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.memory_allocated(dev) == alloc0
    assert np.isfinite(out.cpu().numpy()).all()
