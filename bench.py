#!/usr/bin/env python
"""Benchmark: MSGB forward + exact adjoint on one B200 (beamax config 3).

Default workload (``--workload c3``; the configuration the headline metric
is quoted on, and it fits one GPU): 2D 1024 x 1024 grid, dx = 5e-5 m,
c(x) = 1500 (1 + 0.08 g(x)) with g a seeded Gaussian random field of 40-cell
correlation length clipped to [-1, 1] (cubic B-spline interpolant), cfl 0.3
(Nt ~ 5,600); 4 levels, boxes (4, 8, 16, 32), redundancy 2,
rectangular_mirror (the stated 5-level tiling is rejected by the reference's
own validation); p0 = 256 seeded Gaussian wave packets + 8 blobs, max|p0| = 1;
four-sided line sensor (4092 points); thr = 262144 top_n (524288 beams);
adaptive beam ODE (Dormand-Prince 5(4), rtol 1e-7, atol 1e-9; FP64 ray, FP32
Hessian and amplitude on the FP32 path, all FP64 on the FP64 path).
Synthetic seeded data of those shapes; nothing is downloaded.

A step = one forward (p0 -> sensor data) plus one exact adjoint (data ->
image) on the FP32 path (Kahan sums, FP64 anchor phases, Gaussian cutoff;
beams integrated once per step by the mixed-precision ODE: FP64 ray, FP32
Hessian and amplitude).  The dense FP64 path (reference
semantics: every beam at every time and sensor) is run once for comparison
and as the accuracy reference.  ``value`` = dense-equivalent beam-sample
evaluations per second of forward + adjoint (2 * 2n * Nt * Ns per step / step
time).

``--impl reference`` times the CPU restatement of the reference algorithm
(C/OpenMP FP64, dense, all host threads: for heterogeneous workloads the
adaptive beam ODE plus the dense trajectory sums) on a bounded sample of the
selected beams and reports the same metric.

``--workload c2`` (512^2 homogeneous, four-sided sensor, thr 65,536),
``het512`` (config 2's geometry in a 20-cell-correlation medium) and ``c5``
(3D 128^3) measure the other configurations.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adj beam-sample evaluations/s (dense-equivalent), FP32 path at <=1e-3 rel-L2 vs FP64"
UNIT = "evals/s"


# ---------------------------------------------------------------- workload
def level_annuli(N, nbl, nl):
    """Outer half-width (in Fourier index units) of every level's region."""
    N_ref = min(N)
    bls = [N_ref // (nbl[-1] * 2 ** L) for L in range(nl - 1, -1, -1)]
    return [nbl[l] * bls[l] / 2 for l in range(nl)]


def _window(N, c, radius):
    """Index ranges of the box of half-width ``radius`` around ``c``, clipped."""
    return tuple(slice(max(0, int(np.floor(ci - radius))), min(n, int(np.ceil(ci + radius)) + 1))
                 for ci, n in zip(c, N))


def make_p0(N, nbl, n_packets, n_blobs, blob_sigma, seed):
    """Seeded packets and blobs; each Gaussian is evaluated within 9 widths of
    its centre (where it is above e^-40 of its peak)."""
    rng = np.random.default_rng(seed)
    d = len(N)
    radii = [0.0] + level_annuli(N, nbl, len(nbl))
    p0 = np.zeros(N)
    Nm = min(N)

    def local_coords(sl):
        ax = [np.arange(s.start, s.stop, dtype=np.float64) for s in sl]
        return np.stack(np.meshgrid(*ax, indexing="ij"), -1)

    for i in range(n_packets):
        lvl = i % len(nbl)
        kmag = rng.uniform(max(radii[lvl], 1.0), radii[lvl + 1])
        if d == 2:
            th = rng.uniform(0, 2 * np.pi)
            u = np.array([np.cos(th), np.sin(th)])
        else:
            v = rng.standard_normal(d)
            u = v / np.linalg.norm(v)
        c = (0.1 + 0.8 * rng.uniform(size=d)) * np.asarray(N)
        band = max(radii[lvl + 1] - radii[lvl], 1.0)
        width = Nm / (np.pi * band)
        amp = rng.standard_normal()
        sl = _window(N, c, 9.0 * width)
        r = local_coords(sl) - c
        env = np.exp(-np.sum(r * r, -1) / (2 * width ** 2))
        p0[sl] += amp * env * np.cos(2 * np.pi * kmag / Nm * (r @ u))
    for _ in range(n_blobs):
        c = (0.1 + 0.8 * rng.uniform(size=d)) * np.asarray(N)
        amp = rng.standard_normal()
        sl = _window(N, c, 9.0 * blob_sigma)
        r = local_coords(sl) - c
        p0[sl] += amp * np.exp(-np.sum(r * r, -1) / (2 * blob_sigma ** 2))
    return p0 / np.max(np.abs(p0))


def config2(seed=0, thr=65536):
    import beamax_b200 as bb

    N = (512, 512)
    dom = bb.Domain(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    dec = bb.DyadicDecomposition(4, N, (4, 8, 16, 32), (1, 1))
    wpt = bb.MSWPT(dec, 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sensors = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()
    p0 = make_p0(N, (4, 8, 16, 32), 64, 8, 20.0, seed)
    return dict(name=f"config2: 2D 512^2 homogeneous, 4 levels (4,8,16,32), four-sided sensor, thr={thr}",
                domain=dom, wpt=wpt, sensors=sensors, ts=ts, p0=p0, thr=thr, hetero=False)


def random_speed(N, dx, contrast, corr_cells, seed):
    """c = 1500 (1 + contrast g), g a seeded Gaussian random field with the
    given correlation length (cells), scaled to max |g| = 1 and clipped to
    [-1, 1]; cubic B-spline interpolant with clamped boundaries."""
    from scipy import ndimage

    from beamax_b200.utils.interp import make_c_function_from_grid

    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(N), corr_cells, mode="wrap")
    g = np.clip(g / np.max(np.abs(g)), -1.0, 1.0)
    return make_c_function_from_grid(1500.0 * (1.0 + contrast * g), dx, method="bspline3", boundary="clamp")


def heterogeneous(N, dx, corr_cells, n_packets, thr, seed, name):
    import beamax_b200 as bb

    c = random_speed(N, dx, 0.08, corr_cells, seed + 17)
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False), cfl=0.3, c=c)
    dec = bb.DyadicDecomposition(4, N, (4, 8, 16, 32), (1, 1))
    wpt = bb.MSWPT(dec, 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[0, :] = mask[-1, :] = mask[:, 0] = mask[:, -1] = 1
    sensors = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()
    p0 = make_p0(N, (4, 8, 16, 32), n_packets, 8, 20.0 * N[0] / 512, seed)
    return dict(name=name, domain=dom, wpt=wpt, sensors=sensors, ts=ts, p0=p0, thr=thr, hetero=True)


def het512(seed=0, thr=65536):
    return heterogeneous((512, 512), (1e-4, 1e-4), 20.0, 64, thr, seed,
                         f"het512: 2D 512^2, c = 1500 (1 + 0.08 g), 20-cell correlation, 4 levels (4,8,16,32), "
                         f"four-sided sensor, thr={thr}, adaptive ODE")


def config3(seed=0, thr=262144):
    return heterogeneous((1024, 1024), (5e-5, 5e-5), 40.0, 256, thr, seed,
                         f"config3: 2D 1024^2, dx 5e-5, c = 1500 (1 + 0.08 g), 40-cell correlation, 4 levels "
                         f"(4,8,16,32), four-sided sensor, thr={thr}, adaptive ODE")


def config5(seed=0, thr=262144, n_packets=512):
    """3D 128^3, dx 1e-4, c = 1500 (1 + 0.05 g) with a 20-cell correlation
    length, 3 levels (4, 8, 16) per axis, 512 packets + 16 blobs (sigma 6
    cells), planar sensor on the z = 0 face (128 x 128)."""
    import beamax_b200 as bb

    N, dx = (128, 128, 128), (1e-4, 1e-4, 1e-4)
    c = random_speed(N, dx, 0.05, 20.0, seed + 17)
    dom = bb.Domain(N=N, dx=dx, periodic=(False, False, False), cfl=0.3, c=c)
    wpt = bb.MSWPT(bb.DyadicDecomposition(3, N, (4, 8, 16), (1, 1, 1)), 2, "rectangular_mirror")
    mask = np.zeros(N)
    mask[:, :, 0] = 1
    sensors = bb.Sensor(dom, binary_mask=mask)
    ts = dom.generate_time_domain()
    p0 = make_p0(N, (4, 8, 16), n_packets, 16, 6.0, seed)
    return dict(name=f"config5: 3D 128^3, c = 1500 (1 + 0.05 g), 20-cell correlation, 3 levels (4,8,16), "
                     f"planar z=0 sensor 128x128, thr={thr}, adaptive ODE",
                domain=dom, wpt=wpt, sensors=sensors, ts=ts, p0=p0, thr=thr, hetero=True)


WORKLOADS = {"c2": config2, "het512": het512, "c3": config3, "c5": config5}
DEFAULT_THR = {"c2": 65536, "het512": 65536, "c3": 262144, "c5": 262144}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._proc = None

    def start(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self._proc = None

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        time.sleep(0.05)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------- peaks
def measure_peaks(device):
    """FP32 (scalar FFMA and paired FFMA2), FP64 (DFMA) and MUFU throughput of
    this GPU with libmsgb's probe kernels (8 blocks of 256 threads per SM, 8
    independent chains per thread), each timed with CUDA events after one
    warm-up launch.  TFLOP/s (FMA = 2 flops) or, for MUFU, Tops/s."""
    import torch

    from beamax_b200 import _lib

    L = _lib.lib()
    props = torch.cuda.get_device_properties(device)
    blocks, threads = props.multi_processor_count * 8, 256
    sink = torch.empty(blocks * threads, dtype=torch.float32, device=device)
    st = torch.cuda.current_stream(device)
    out = {}
    for name, kind, iters in (("fp32", 0, 200000), ("fp32x2", 1, 100000), ("fp64", 2, 100000), ("mufu", 3, 20000)):
        _lib.check(L.msgb_peak_probe(kind, 1000, blocks, threads, sink.data_ptr(), st.cuda_stream), "probe")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        _lib.check(L.msgb_peak_probe(kind, iters, blocks, threads, sink.data_ptr(), st.cuda_stream), "probe")
        b.record(st)
        torch.cuda.synchronize(device)
        secs = a.elapsed_time(b) / 1e3
        out[name] = L.msgb_peak_probe_ops(kind, iters, blocks, threads) / secs / 1e12
    out["fp32_best"] = max(out["fp32"], out["fp32x2"])
    out["method"] = (f"msgb_peak_probe: {blocks} blocks x {threads} threads, 8 independent chains of FFMA / FFMA2 / "
                     "DFMA / MUFU.SIN per thread, CUDA events, after one warm-up launch; FMA = 2 flops")
    return out


def ode_flops_per_step(d: int) -> float:
    """Algorithmic FP64 flops of one attempted Dormand-Prince step of the beam
    ODE in a cubic B-spline medium (add, multiply, divide, square root, power
    = 1 flop; FMA = 2), counted from the operations of the formulas:
      * c, grad c, Hessian c at a point: per axis the B-spline weights and
        their first and second derivatives (36 flops), then the separable
        tensor-product sums: 2D 4 x 4 x 3 + 4 x 6 FMA, 3D 4^3 x 3 + 16 x 6 +
        4 x 10 FMA, and the 1/spacing scaling: 226 (2D) / 785 (3D);
      * coupled_rhs_absorption on the symmetric Riccati state (G, G_x, G_p,
        G_pp, G_xp, M G_pp, the d(d+1)/2 entries of dM = -(G_xx + G_xp M +
        M G_xp^T + M G_pp M), tr M, G_p^T M G_p and dA): 228 (2D) / 578 (3D);
      * per step: 6 right-hand sides (first same as last), the 20 nonzero
        stage coefficients and 6 stage inputs over the N = 12 (2D) / 20 (3D)
        real state entries, the 7-term error estimate and the RMS error norm
        with |.| of each complex entry: 900 (2D) / 1494 (3D).
    2D: 6 x 454 + 900 = 3624; 3D: 6 x 1363 + 1494 = 9672."""
    return {2: 3624.0, 3: 9672.0}.get(d, 3624.0)


def ode_flops_split(d: int):
    """(FP64, FP32) flops of the same step in the FP32 path's mixed-precision
    integrator, where only the ray is FP64: per right-hand side |p|^2, the
    reciprocal square root, G_p and G_x (16 in 2D / 20 in 3D), and the stage
    combinations and error estimate of the 2d ray entries (1/3 of the 840
    flops of the 12-entry state in 2D, 6/20 of 1434 in 3D); everything else
    (the medium, the Riccati and amplitude terms, their stages, the error
    norm) is FP32."""
    f64 = {2: 6 * 16 + 840 / 3, 3: 6 * 20 + 1434 * 6 / 20}.get(d, 6 * 16 + 840 / 3)
    return f64, ode_flops_per_step(d) - f64


# ---------------------------------------------------------------- ours
def launches_per_step(levels: int) -> int:
    """Kernels of libmsgb launched per step (cuFFT's own kernels excluded)."""
    fwd = levels + 1 + 2 + 1 + (1 + 2 + 1 + 1) + 1  # boxes, key bits, radix sort, take, init, prep(4), sum
    adj = 1 + 5 + 1 + 1 + 1 + levels + 1 + 1        # init, prep+permute, gather, scatter, zero, boxes, synth, real
    return fwd + adj


def run_ours(args, rank, world, device):
    import torch

    import beamax_b200 as bb
    from beamax_b200.solvers.msgb_solver import Selection

    torch.cuda.set_device(device)
    W = WORKLOADS[args.workload](seed=1234 + rank, thr=args.thr)
    dom, wpt, sens, ts, p0 = W["domain"], W["wpt"], W["sensors"], W["ts"], W["p0"]
    ode = bb.gb.gb_solvers.solve_ODE_base if W["hetero"] else bb.gb.gb_solvers.solve_hom_diag
    s32 = bb.MSGBSolver(W["thr"], "top_n", 128, "spatial", ode, "scan_real", precision="fp32", cutoff=args.cutoff)
    s64 = bb.MSGBSolver(W["thr"], "top_n", 128, "spatial", ode, "scan_real", precision="fp64")
    p0_d = torch.from_numpy(p0).to(device)
    nt, ns = ts.size, sens.positions.shape[0]
    n = W["thr"]
    dense_step = 2 * (2 * n) * nt * ns  # forward + adjoint, both modes
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    rng = np.random.default_rng(99 + rank)
    data_probe = torch.from_numpy(rng.standard_normal((nt, ns))).to(device)

    def step():
        y = s32.forward(p0_d, dom, sens, ts, wpt)
        img = s32.adjoint(y, dom, sens, ts, wpt)
        return y, img

    # warm-up (also builds device plans and workspaces)
    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()

    st = torch.cuda.current_stream()

    # timed region
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    times = []
    s32.kernel_timer = []  # events around each summation entry point, inside the timed steps
    steps_ctr = torch.zeros(1, dtype=torch.int64, device=device)
    s32.ode_step_counter = steps_ctr
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        step()
        b.record(st)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / 1e3)
    if world > 1:
        torch.distributed.barrier()
    spans = s32.kernel_timer
    s32.kernel_timer = None
    s32.ode_step_counter = None
    ode_steps = int(steps_ctr.item()) / args.steps

    def span_time(name):
        """Device time per step of every call of one entry point (all chunks)."""
        return sum(a.elapsed_time(b) / 1e3 for nm, a, b, c in spans if nm == name) / args.steps

    def span_evals(name):
        cs = [c for nm, a, b, c in spans if nm == name]
        return int(cs[-1].item()) if cs else 0  # one counter per call, summed over its chunks

    suffix = "_traj" if W["hetero"] else ""
    t_fwd_kernel, fwd_evals = span_time("msgb_sum_fwd_f32" + suffix), span_evals("msgb_sum_fwd_f32" + suffix)
    t_adj_kernel, adj_evals = span_time("msgb_adj_gather_f32" + suffix), span_evals("msgb_adj_gather_f32" + suffix)
    t_ode = span_time("msgb_ode_trajectories")
    total = float(np.sum(times))
    if world > 1:
        t = torch.tensor([total], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total = float(t.item())
    clocks = sampler.stop() if sampler else None

    # e2e through the public API with host buffers (H2D of p0, D2H of data,
    # H2D of data, D2H of the image inside the timed region)
    p0_host = torch.from_numpy(p0).pin_memory()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        y_host = s32.forward(p0_host.numpy(), dom, sens, ts, wpt)
        img_host = s32.adjoint(y_host, dom, sens, ts, wpt)
        b.record(st)
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b) / 1e3)
    e2e_t = float(np.mean(e2e))
    if world > 1:  # the job's end-to-end time is the slowest rank's
        t = torch.tensor([e2e_t], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_t = float(t.item())

    result = {"rank": rank, "t_step": total / args.steps, "t_fwd_kernel": t_fwd_kernel, "t_adj_kernel": t_adj_kernel,
              "t_ode": t_ode, "ode_steps": ode_steps, "ndim": len(dom.N), "hetero": W["hetero"],
              "nt": nt, "ns": ns, "n_beams": 2 * n,
              # heterogeneous: one ODE and one summation call per trajectory chunk, each a prep + main kernel
              "extra_launches": 3 * sum(1 for nm, *_ in spans if "traj" in nm or "ode" in nm),
              "fwd_evals": fwd_evals, "adj_evals": adj_evals, "dense_step": dense_step, "clocks": clocks,
              "e2e_t": e2e_t, "h2d": p0.nbytes + nt * ns * 4, "d2h": nt * ns * 4 + p0.nbytes,
              "levels": wpt.dyadic_decomp.num_levels, "workload": W["name"]}

    # FP64 plain path (dense, reference semantics): once, also the accuracy reference
    s32.release_trajectories()
    if rank == 0 and not args.no_fp64:
        flush.zero_()
        torch.cuda.synchronize()
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(st)
        y64 = s64.forward(p0_d, dom, sens, ts, wpt)
        b.record(st)
        img64 = s64.adjoint(y64, dom, sens, ts, wpt)
        c.record(st)
        torch.cuda.synchronize()
        y32f, img32 = step()
        result["fp64"] = {"fwd_s": a.elapsed_time(b) / 1e3, "adj_s": b.elapsed_time(c) / 1e3}
        rel = lambda r, x: float(torch.linalg.norm(r - x.double()) / torch.linalg.norm(r))
        result["rel_l2_fwd"] = rel(y64, y32f)
        img32b = s32.adjoint(y64.float(), dom, sens, ts, wpt)
        result["rel_l2_adj"] = rel(img64, img32b)
        # dot test of the FP32 transpose
        q = torch.from_numpy(np.random.default_rng(5).standard_normal(dom.N)).to(device)
        cq = wpt.forward_device(q, scale=0.5, half_mask=True)
        selq = Selection(s32.last_selection.idx, cq[s32.last_selection.idx], wpt.total_coeffs)
        Aq = s32.sum_forward(s32.beams(selq, dom, wpt), dom, sens, ts).double()
        At = s32.adjoint(data_probe, dom, sens, ts, wpt, selection=s32.last_selection)
        lhs, rhs = float((Aq * data_probe).sum()), float((q * At).sum())
        result["dot_test_rel"] = abs(lhs - rhs) / abs(lhs)
        # the same difference against |A q| |d|: independent of how small the
        # inner product of the random probe with A q happens to be
        result["dot_test_norm"] = abs(lhs - rhs) / float(torch.linalg.norm(Aq) * torch.linalg.norm(data_probe))
    return result


def run_ode_only(args, device, peaks):
    """The beam ODE alone (``--ode-only``): the workload's selection, then
    msgb_ode_trajectories over every beam (both modes) writing the FP32
    summation records into the compact store, in the chunks the solver's
    forward uses; W untimed and K timed integrations, CUDA events on the
    launching stream."""
    import torch

    import beamax_b200 as bb
    from beamax_b200 import _lib

    torch.cuda.set_device(device)
    W = WORKLOADS[args.workload](seed=1234, thr=args.thr)
    if not W["hetero"]:
        raise SystemExit("--ode-only needs a heterogeneous workload (het512, c3, c5)")
    dom, wpt, sens, ts, p0 = W["domain"], W["wpt"], W["sensors"], W["ts"], W["p0"]
    s = bb.MSGBSolver(W["thr"], "top_n", 128, "spatial", bb.gb.gb_solvers.solve_ODE_base, "scan_real",
                      precision="fp32")
    sel = s.select(torch.from_numpy(p0).to(device), dom, wpt)
    bt = s.beams(sel, dom, wpt)
    pr, keep = s._problem(dom, sens, ts, device)
    med, keep_m = s._medium(dom, device)
    bs = bt.beam_set(unit=False)
    st = torch.cuda.current_stream(device)
    status = torch.zeros(2 * bt.n, dtype=torch.int32, device=device)
    ctr = torch.zeros(1, dtype=torch.int64, device=device)
    tiling = s._tiling(dom, sens, device)
    sopts = _lib.SumOpts(cutoff=s.cutoff, tiling=_lib.ref(tiling[0]) if tiling else None)
    n_chunks = [0]

    def integrate():
        n_chunks[0] = 0
        for _ in s._compact_integrate(pr, med, bs, 0, 2 * bt.n, dom, sens, sopts, device, st.cuda_stream, status):
            n_chunks[0] += 1

    for _ in range(max(args.warmup, 1)):
        integrate()
    torch.cuda.synchronize(device)
    s.ode_step_counter = ctr
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(args.steps):
        integrate()
    b.record(st)
    torch.cuda.synchronize(device)
    secs = a.elapsed_time(b) / 1e3 / args.steps
    steps = int(ctr.item()) / args.steps
    fl = ode_flops_per_step(len(dom.N))
    achieved = steps * fl / secs / 1e12
    line = {"mode": "ode_only", "workload": W["name"], "beams": 2 * bt.n, "nt": pr.nt, "chunks": n_chunks[0],
            "ode_s": secs, "attempted_steps": steps, "steps_per_beam": steps / (2 * bt.n),
            "beam_steps_per_s": steps / secs, "flops_per_step": fl, "achieved_tflops": achieved,
            "peak_fp64_tflops": peaks["fp64"] if peaks else None,
            "frac": achieved / peaks["fp64"] if peaks else None, "status_max": int(status.max().item())}
    print(json.dumps(line), flush=True)
    return 0


def run_gemm_only(args, device, peaks):
    """The surrogate MLP's hidden-layer product alone (``--gemm-only``):
    C16 = SiLU(A W^T + b) with A (M x 256), W (256 x 256) BF16, FP32
    accumulation, M = args.gemm_rows, through msgb_gemm_bf16 (the TMA-fed
    persistent tcgen05 kernel); W untimed and K timed launches, CUDA events.
    Roofline: 2 M N K flops against the measured dense BF16 peak in
    MEASURED_PEAKS.json when present."""
    import torch

    from beamax_b200 import _lib

    torch.cuda.set_device(device)
    M, N, K = args.gemm_rows, 256, 256
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(device)
    W = (torch.randn(N, K, generator=g) / 16).to(torch.bfloat16).to(device)
    b = torch.randn(N, generator=g).to(device)
    C16 = torch.empty((M, N), dtype=torch.bfloat16, device=device)
    err = torch.zeros(1, dtype=torch.int32, device=device)
    gm = _lib.Gemm(A=A.data_ptr(), sAm=K, sAk=1, B=W.data_ptr(), sBn=K, sBk=1, M=M, N=N, K=K, bias=b.data_ptr(),
                   act=1, C32=None, ldc32=0, C16=C16.data_ptr(), ldc16=N, error_flag=err.data_ptr())
    st = torch.cuda.current_stream(device)
    call = lambda: _lib.check(_lib.lib().msgb_gemm_bf16(_lib.ref(gm), st.cuda_stream), "msgb_gemm_bf16")
    for _ in range(max(args.warmup, 1)):
        call()
    torch.cuda.synchronize(device)
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(args.steps):
        call()
    e.record(st)
    torch.cuda.synchronize(device)
    secs = a.elapsed_time(e) / 1e3 / args.steps
    ref = torch.nn.functional.silu(A[:4096].float() @ W.float().T + b)
    rel = float((C16[:4096].float() - ref).norm() / ref.norm())
    flops = 2.0 * M * N * K
    peak_bf16 = None
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        with open(mp) as f:
            peak_bf16 = json.load(f).get("bf16_tflops")
    achieved = flops / secs / 1e12
    hbm = (M * K * 2 + M * N * 2) / secs / 1e9
    print(json.dumps({"mode": "gemm_only", "M": M, "N": N, "K": K, "s_per_launch": secs, "tflops": achieved,
                      "peak_bf16_tflops": peak_bf16, "frac": achieved / peak_bf16 if peak_bf16 else None,
                      "hbm_gbs_moved": hbm, "rel_err_vs_fp32": rel, "error_flag": int(err.item())}), flush=True)
    return 0


def run_surrogate_eval(args, device, peaks):
    """What the learned trajectory surrogate buys (``--surrogate-eval``): on
    the workload's medium, train the MLP on ODE trajectories of a beam sample
    (the library's own BF16 tcgen05 kernels), then time the FP32 forward with
    and without it (CUDA events around each forward, after a warm-up of each)
    and compare both with the FP64 forward: beams accepted, forward time, the
    ODE time saved, rel-L2, and the MLP's inference rate."""
    import torch

    import beamax_b200 as bb
    from beamax_b200.surrogate import TrajectorySurrogate

    torch.cuda.set_device(device)
    W = WORKLOADS[args.workload](seed=1234, thr=args.thr)
    if not W["hetero"]:
        raise SystemExit("--surrogate-eval needs a heterogeneous workload (het512, c3, c5)")
    dom, wpt, sens, ts, p0 = W["domain"], W["wpt"], W["sensors"], W["ts"], W["p0"]
    ode = bb.gb.gb_solvers.solve_ODE_base
    s64 = bb.MSGBSolver(W["thr"], "top_n", 128, "spatial", ode, "scan_real")
    p0_d = torch.from_numpy(p0).to(device)
    y64 = s64.forward(p0_d, dom, sens, ts, wpt)
    bt = s64.beams(s64.last_selection, dom, wpt)
    t0 = time.perf_counter()
    sur = TrajectorySurrogate(seed=0).fit(s64, dom, sens, ts, bt, n_train=args.sur_train, n_val=256, t_stride=4,
                                          epochs=args.sur_epochs, batch=8192)
    torch.cuda.synchronize(device)
    t_fit = time.perf_counter() - t0
    st = torch.cuda.current_stream(device)
    out = {}
    for name, kw in (("without", {}), ("with", {"surrogate": sur})):
        s = bb.MSGBSolver(W["thr"], "top_n", 128, "spatial", ode, "scan_real", precision="fp32", **kw)
        s.forward(p0_d, dom, sens, ts, wpt)  # warm-up
        s.kernel_timer = []
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        y = s.forward(p0_d, dom, sens, ts, wpt)
        b.record(st)
        torch.cuda.synchronize(device)
        t_ode = sum(x.elapsed_time(z) / 1e3 for nm, x, z, _ in s.kernel_timer if nm == "msgb_ode_trajectories")
        out[name] = {"forward_s": a.elapsed_time(b) / 1e3, "ode_s": t_ode,
                     "accepted": s.last_surrogate_accepted, "beams": 2 * bt.n,
                     "rel_l2_vs_fp64": float(torch.linalg.norm(y64 - y.double()) / torch.linalg.norm(y64))}
    # MLP inference rate on one chunk of feature rows
    rows = 1 << 20
    X = torch.zeros((rows, 16), dtype=torch.bfloat16, device=device)
    sur._predict_rows(X)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    sur._predict_rows(X)
    b.record(st)
    torch.cuda.synchronize(device)
    t_inf = a.elapsed_time(b) / 1e3
    widths = list(sur.mlp.dims)
    flops_row = sum(2.0 * widths[i] * widths[i + 1] for i in range(len(widths) - 1))
    line = {"mode": "surrogate_eval", "workload": W["name"], "fit_s": t_fit, "fit_stats": sur.stats,
            "without": out["without"], "with": out["with"],
            "ode_s_saved": out["without"]["ode_s"] - out["with"]["ode_s"],
            "forward_s_saved": out["without"]["forward_s"] - out["with"]["forward_s"],
            "mlp_rows_per_s": rows / t_inf, "mlp_tflops": rows * flops_row / t_inf / 1e12,
            "mlp_flops_per_row": flops_row}
    print(json.dumps(line, default=float), flush=True)
    return 0


def rooflines(r, peaks, sm_mhz, args):
    """Rooflines of the step's kernels, the one with the largest device time
    per step first (``roofline``), the others after it (``roofline_other``).

    * Summation (``fwd32_kernel``, ``adj32_kernel``; ``<TRAJ>`` for the
      trajectory variants): work unit = one evaluated (beam, time, sensor)
      triple, 36 flops for the forward (24 FP32 instructions of a direct
      evaluation, FMA = 2), 40 for the transpose (+ 2 FMA for d conj(z));
      also the MUFU side (3 special-function operations per direct
      evaluation).  Peak: the measured FP32 throughput (the better of FFMA and
      FFMA2) and MUFU throughput of msgb_peak_probe.
    * Beam ODE (``dopri_kernel``): attempted Dormand-Prince steps counted on the
      device x ode_flops_per_step(d); peak: the measured DFMA throughput.
    DRAM traffic per launch: dram__bytes_read.sum + dram__bytes_write.sum of
    the committed one-pass ncu capture of the workload at its default size
    (profiles/dram_traffic_<workload>.json); null where there is none."""
    fp32 = peaks["fp32_best"] if peaks else 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    basis32 = ("measured: " + peaks["method"]) if peaks else f"148 SM x 128 FP32 lanes x 2 x {sm_mhz:.0f} MHz"
    traffic = {}
    prof = os.path.join(ROOT, "profiles", f"dram_traffic_{args.workload}.json")
    if os.path.exists(prof) and args.thr == DEFAULT_THR[args.workload]:
        with open(prof) as f:
            traffic = json.load(f).get("per_launch_bytes", {})
    suffix = "<TRAJ>" if r["hetero"] else ""
    out = []
    for key, name, flops, evals, secs, what in (
            ("fwd", "fwd32_kernel", 36.0, r["fwd_evals"], r["t_fwd_kernel"], "forward summation"),
            ("adj", "adj32_kernel", 40.0, r["adj_evals"], r["t_adj_kernel"], "transpose gather")):
        if secs <= 0:
            continue
        achieved = evals * flops / secs / 1e12
        entry = {"bound": "fp32", "achieved": achieved, "peak": fp32, "unit": "TFLOP/s",
                 "frac": achieved / fp32, "traffic": traffic.get(name), "kernel": name + suffix,
                 "flops_per_eval": flops, "device_s_per_step": secs, "peak_basis": basis32,
                 "timing": f"CUDA events around the {what} entry point inside the timed steps "
                           "(device time per step, all chunks)"}
        if peaks:
            mufu = 3.0 * evals / secs / 1e12
            entry["mufu"] = {"achieved": mufu, "peak": peaks["mufu"], "unit": "Tops/s", "frac": mufu / peaks["mufu"],
                             "ops_per_eval": 3}
        out.append(entry)
    if r["hetero"] and r["t_ode"] > 0 and r["ode_steps"] > 0:
        # the FP32 path's mixed-precision integrator: FP32 for all but the ray
        f64, f32 = ode_flops_split(r["ndim"])
        rate = r["ode_steps"] / r["t_ode"]
        peak64 = peaks["fp64"] if peaks else 148 * 64 * 2 * sm_mhz * 1e6 / 1e12
        a32, a64 = rate * f32 / 1e12, rate * f64 / 1e12
        out.append({"bound": "fp32", "achieved": a32, "peak": fp32, "unit": "TFLOP/s", "frac": a32 / fp32,
                    "fp64": {"achieved": a64, "peak": peak64, "frac": a64 / peak64, "flops_per_step": f64},
                    "traffic": traffic.get("dopri_mix_kernel"), "kernel": "dopri_mix_kernel",
                    "flops_per_step": f32, "flops_per_step_total": f64 + f32,
                    "attempted_steps_per_step": r["ode_steps"], "device_s_per_step": r["t_ode"],
                    "peak_basis": basis32,
                    "timing": "CUDA events around every msgb_ode_trajectories call inside the timed steps; "
                              "attempted steps counted on the device"})
    out.sort(key=lambda e: -e["device_s_per_step"])
    return out[0], out[1:]


CPU_SAMPLE = {"c2": 96, "het512": 64, "c3": 48, "c5": 32}


def cpu_reference(args, warmup=0, steps=1):
    """Dense FP64 C/OpenMP restatement on a bounded sample of the selected
    coefficients (both modes of each), all host threads.  Homogeneous media:
    closed-form beams (oracle/csum.c); heterogeneous media: the adaptive
    Dormand-Prince beam ODE, then the dense trajectory sums (oracle/chet.c).
    The selection itself (MSWPT + top_n + beam init in the NumPy oracle) is
    not timed; everything after it is, `warmup` untimed and `steps` timed
    repetitions of the sample (the reported times are their means)."""
    import oracle.build as ob
    from oracle import msgb as om

    ob.build()
    W = WORKLOADS[args.workload](seed=1234, thr=args.thr)
    dom, wpt, sens, ts, p0 = W["domain"], W["wpt"], W["sensors"], W["ts"], W["p0"]
    odom = om.Dom(N=dom.N, dx=dom.dx, periodic=dom.periodic, cfl=dom.cfl, c=1500.0)
    dec = wpt.dyadic_decomp
    ow = om.Wpt(om.Decomp(dec.num_levels, dec.N, dec.num_boxes_levels, dec.box_aspect_ratio), 2, wpt.windowing)
    t0 = time.perf_counter()
    bm = om.select_beams(p0, odom, ow, W["thr"])
    t_select = time.perf_counter() - t0
    nsample = args.cpu_sample or CPU_SAMPLE[args.workload]
    reps = max(0, warmup) + max(1, steps)
    if not args.cpu_sample and reps > 6:
        # keep the whole run near 6 repetitions' worth of host time
        nsample = max(2, nsample * 6 // reps)
    rng = np.random.default_rng(0)
    pick = np.sort(rng.choice(bm.idx.size, size=nsample, replace=False))
    sub = om.Beams(bm.idx[pick], bm.coeff[pick], bm.p0[pick], bm.M0[pick], bm.x0[pick], bm.omega[pick],
                   bm.a0_unit[pick])
    tab = om.beam_table(sub, 1500.0)
    pos = sens.positions

    def one():
        t_ode = 0.0
        if W["hetero"]:
            cat = lambda a: np.concatenate([a, a])
            mode = np.concatenate([np.ones(nsample), -np.ones(nsample)])
            t0 = time.perf_counter()
            rec, status, _ = ob.het_trajectories(cat(tab["x0"]), cat(tab["p0"]), cat(tab["alpha"]), mode,
                                                 dom.medium()[1], ts)
            t_ode = time.perf_counter() - t0
            amp, om2 = cat(tab["a0"]), cat(tab["omega"])
            t0 = time.perf_counter()
            y = ob.sum_traj(rec, amp, om2, pos, dom.grid_size, dom.periodic)
            t_fwd = time.perf_counter() - t0
            t0 = time.perf_counter()
            ob.adj_traj(rec, om2, pos, dom.grid_size, dom.periodic, y)
            t_adj = time.perf_counter() - t0
        else:
            t0 = time.perf_counter()
            y = ob.sum_hom(tab, 1500.0, ts, pos, dom.grid_size, dom.periodic)
            t_fwd = time.perf_counter() - t0
            t0 = time.perf_counter()
            ob.adj_hom(tab, sub.a0_unit, 1500.0, ts, pos, dom.grid_size, dom.periodic, y)
            t_adj = time.perf_counter() - t0
        return t_ode, t_fwd, t_adj

    for _ in range(max(0, warmup)):
        one()
    t_ode, t_fwd, t_adj = (float(np.mean(v)) for v in zip(*[one() for _ in range(max(1, steps))]))
    what = ("adaptive Dormand-Prince beam ODE + dense FP64 trajectory sums, forward + exact adjoint (oracle/chet.c)"
            if W["hetero"] else "dense FP64 closed-form beams, forward + exact adjoint (oracle/csum.c)")
    what += f", {max(1, steps)} timed repetitions after {max(0, warmup)} untimed"
    evals = 2 * (2 * nsample) * ts.size * pos.shape[0]
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    t_all = t_ode + t_fwd + t_adj
    value = evals / t_all
    full_s = t_all * W["thr"] / nsample
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{nsample} of {W['thr']} selected coefficients ({2 * nsample} beams), all {ts.size} times x "
                      f"{pos.shape[0]} sensors; {what}, C/OpenMP on {cores} host threads; ODE {t_ode:.2f} s, "
                      f"sums {t_fwd:.2f} + {t_adj:.2f} s; full step extrapolated linearly in beams: {full_s:.0f} s",
            "select_s": t_select, "t_ode_s": t_ode, "t_fwd_s": t_fwd, "t_adj_s": t_adj, "workload": W["name"]}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cutoff", type=float, default=16.0)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3",
                    help="c3: config 3 (the headline); c2 / het512 / c5: the other configurations")
    ap.add_argument("--thr", type=int, default=None, help="top_n (default: the workload's; smaller for profiling)")
    ap.add_argument("--cpu-sample", type=int, default=None, help="coefficients timed by the CPU baseline")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-peaks", action="store_true")
    ap.add_argument("--ode-only", action="store_true", help="time the beam ODE alone (heterogeneous workloads)")
    ap.add_argument("--gemm-only", action="store_true", help="time the surrogate's 256 x 256 layer GEMM alone")
    ap.add_argument("--gemm-rows", type=int, default=1 << 20)
    ap.add_argument("--surrogate-eval", action="store_true", help="train the trajectory surrogate and measure its gain")
    ap.add_argument("--sur-train", type=int, default=3000)
    ap.add_argument("--sur-epochs", type=int, default=40)
    args = ap.parse_args()
    if args.thr is None:
        args.thr = DEFAULT_THR[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        r = cpu_reference(args, warmup=args.warmup, steps=args.steps)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": r["workload"], "sample": r["sample"]},
                "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch

    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    peaks = None if args.no_peaks else measure_peaks(device)
    if args.ode_only:
        return run_ode_only(args, device, peaks)
    if args.gemm_only:
        return run_gemm_only(args, device, peaks)
    if args.surrogate_eval:
        return run_surrogate_eval(args, device, peaks)
    r = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_reference(args)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as e:  # reported, never fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}
    t_step = r["t_step"]
    value = world * r["dense_step"] / t_step
    clk = r["clocks"] or {}
    sm_mhz = clk.get("sm_mhz") or 1965.0
    roof, roof_other = rooflines(r, peaks, sm_mhz, args)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": r["workload"], "global_batch": world, "parallelism": f"replicas{world}",
                   "nt": r["nt"], "ns": r["ns"], "beams": r["n_beams"],
                   "l2": "flushed (256 MiB write) between timed steps", "cutoff_efolds": args.cutoff},
        "e2e": {"value": world * r["dense_step"] / r["e2e_t"], "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "ms_per_step": r["e2e_t"] * 1e3},
        "gpu_launches": args.steps * launches_per_step(r["levels"]) + r["extra_launches"],
        "roofline": roof,
        "roofline_other": roof_other,
        "kernels": {"fwd32_s": r["t_fwd_kernel"], "adj32_s": r["t_adj_kernel"], "fwd_evals": r["fwd_evals"],
                    "adj_evals": r["adj_evals"], "dense_evals_per_step": r["dense_step"],
                    "fwd_evals_per_s": r["fwd_evals"] / r["t_fwd_kernel"] if r["t_fwd_kernel"] else None,
                    "adj_evals_per_s": r["adj_evals"] / r["t_adj_kernel"] if r["t_adj_kernel"] else None,
                    "ode_s_per_step": r["t_ode"], "ode_attempted_steps_per_step": r["ode_steps"]},
        "peaks_measured": peaks,
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    if "fp64" in r:
        f = r["fp64"]
        line["fp64_plain"] = {"fwd_ms": f["fwd_s"] * 1e3, "adj_ms": f["adj_s"] * 1e3,
                              "value": r["dense_step"] / (f["fwd_s"] + f["adj_s"]),
                              "speedup_fp32_vs_fp64": (f["fwd_s"] + f["adj_s"]) / t_step}
        line["rel_l2_fwd_vs_fp64"] = r["rel_l2_fwd"]
        line["rel_l2_adj_vs_fp64"] = r["rel_l2_adj"]
        line["dot_test_rel_fp32"] = r["dot_test_rel"]
        line["dot_test_norm_fp32"] = r["dot_test_norm"]
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
