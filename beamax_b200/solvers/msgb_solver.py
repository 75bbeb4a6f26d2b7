"""``MSGBSolver``: MSGB forward operator and its exact transpose on a B200.

Drop-in for beamax's ``MSGBSolver`` (solvers/msgb_solvers/msgb_solver.py:
358-1386) on the forward path.  ``forward(p0, domain, sensors, ts, wpt)``
runs, all on the GPU through libmsgb.so:

1. ``msgb_mswpt_forward``  - coefficients c_pos = 0.5 * MSWPT(p0) * half_mask
   (compute_coefficients, forward_solver_utils.py:716-786) plus top_n keys;
2. ``msgb_topn``           - the ``thr`` largest, ties by index (:65-89);
3. ``msgb_beam_init``      - beam data (compute_forward_parameters, :255-373);
4. ``msgb_sum_fwd_f64`` (dense, reference semantics) or ``msgb_sum_fwd_f32``
   (Gaussian cutoff, Kahan sums) - both branches (modes +1/-1) of every beam
   with solve_hom_diag fused in (gb/core.py:194-329).

``adjoint(data, domain, sensors, ts, wpt)`` is the exact transpose of that
map with the beam selection frozen (the reference's jax.vjp pattern,
examples/diagnostics/msgb_adjoint_pairing.py:156-165): per-beam gathers
(``msgb_adj_gather_*``), a scatter to coefficient space and the Hermitian
adjoint of the MSWPT.  The reference's own principal-symbol ``adjoint`` (seven
arguments, msgb_solver.py:1235-1386) is a different operator; called with
those arguments, ``adjoint`` computes it, and ``time_reversal`` the time
reversal (:984-1111), both from boundary data with ``msgb_tr_init`` and
``msgb_tr_final_states``.
"""

from __future__ import annotations

import collections
import contextlib
import ctypes
import math
from dataclasses import dataclass, replace
from numbers import Integral, Real
from typing import Optional, Tuple

import numpy as np

from .. import _lib
from .._device import DeviceCache, as_device_f64, default_device, workspace
from ..geometry import Domain, Sensor
from ..gb.gb_solvers import CLOSED_FORM, SolverConfig, solver_name
from ..transforms import MSWPT

_cache = DeviceCache()


def _validate_time_grid(ts, *, allow_singleton: bool = False) -> Optional[float]:
    """msgb_solver.py:41-65."""
    ts_np = np.asarray(ts.detach().cpu().numpy() if hasattr(ts, "detach") else ts)
    if ts_np.ndim != 1 or ts_np.size == 0:
        raise ValueError("ts must be a non-empty one-dimensional array.")
    if not np.all(np.isfinite(ts_np)):
        raise ValueError("ts must contain only finite values.")
    if ts_np.size == 1:
        if allow_singleton:
            return None
        raise ValueError("ts must be one-dimensional with at least two points.")
    diffs = np.diff(ts_np)
    if np.any(diffs <= 0) or not np.allclose(diffs, diffs[0], rtol=1e-6, atol=0.0):
        raise ValueError("ts must be finite, strictly increasing, and uniformly spaced.")
    return float(diffs[0])


@dataclass
class Selection:
    """Frozen beam selection: flat coefficient indices and their c_pos values (device)."""

    idx: "object"      # (n,) int64 CUDA tensor
    values: "object"   # (n,) complex128 CUDA tensor
    total_coeffs: int


@dataclass
class BranchSelection:
    """The complex-input path's two selections (msgb_solver.py:635-689): c_pos
    coefficients drive mode +1 beams, c_neg coefficients mode -1 beams."""

    pos: Selection
    neg: Selection

    @property
    def total_coeffs(self) -> int:
        return self.pos.total_coeffs


@dataclass
class BeamTensors:
    x0: "object"
    p0: "object"
    alpha: "object"    # complex128 (n, d)
    a0: "object"       # complex128 (n,)
    a0_unit: "object"  # complex128 (n,)
    omega: "object"
    modes: int = 0     # 0 both branches (mirrored), 1 only mode +1, 2 only mode -1

    @property
    def n(self) -> int:
        return int(self.omega.shape[0])

    def beam_set(self, unit: bool = False) -> _lib.BeamSet:
        import torch

        a0 = self.a0_unit if unit else self.a0
        return _lib.BeamSet(n=self.n, x0=self.x0.data_ptr(), p0=self.p0.data_ptr(),
                            alpha=torch.view_as_real(self.alpha).data_ptr(),
                            a0=torch.view_as_real(a0).data_ptr(), omega=self.omega.data_ptr(), modes=self.modes)

    def with_amplitude(self, factor, modes=None):
        """The same beams with a0 and a0_unit multiplied by ``factor``."""
        return BeamTensors(self.x0, self.p0, self.alpha, self.a0 * factor, self.a0_unit * factor, self.omega,
                           self.modes if modes is None else modes)


class MSGBSolver:
    """Multiscale Gaussian beam solver (msgb_solver.py:358-534 options and checks).

    Extra keyword-only options (no reference counterpart):
      precision: "fp64" (dense, reference semantics) or "fp32" (FP32
        evaluation, Kahan-compensated sums, FP64 anchor phases, Gaussian cutoff).
      cutoff: e-folds of the Gaussian envelope beyond which the FP32 path skips
        a (beam, time tile, sensor tile) triple.
      rk4_substeps: RK4 steps per save interval when ``ode_config.solver`` is
        "rk4" (overrides ``ode_config.substeps`` when > 1).
      trajectory_memory: bytes of device memory for trajectory records (at
        most what the device has free less 4 GiB); beams are propagated and
        summed in chunks that fit.  The FP32 path stores a (time tile, beam)
        block of records only when it comes within the cutoff of a sensor
        tile (a compact store, typically 35-40 % of the tiles at the
        configuration-3 geometry), so far more beams fit per chunk.
      surrogate: a fitted ``beamax_b200.surrogate.TrajectorySurrogate`` for the
        medium and time grid; heterogeneous beams are predicted by it and the
        ones it does not accept are integrated.
      keep_trajectories: in heterogeneous media, keep the last forward's
        trajectory records on the device so that an adjoint with the same
        selection, domain and time grid does not integrate those beams again:
        all of them when they fit in trajectory_memory, else the last chunk
        of beams (when the device has room for it beside the chunk buffer).
      compact_trajectories: the FP32 path's compact record store (default);
        False stores every (time, beam) record (the same results, more memory).
    """

    def __init__(self, thr, thr_strat: str, batch_size: int, input_type: str, ode_solver, sum_method: str,
                 tr_ode_solver=None, sharding=None, ode_config=None, adjoint_relative_guard: float = 5e-2,
                 *, precision: str = "fp64", cutoff: float = 16.0, rk4_substeps: int = 1,
                 trajectory_memory: int = 96 << 30, surrogate=None, keep_trajectories: bool = True,
                 compact_trajectories: bool = True):
        valid_thresholds = {"hard", "top_n", "percentile", "hard_reassign", "bao_energy", "perc_max_abs"}
        if thr_strat not in valid_thresholds:
            raise ValueError(f"thr_strat must be one of {', '.join(sorted(valid_thresholds))}; got {thr_strat!r}.")
        if isinstance(thr, bool) or not isinstance(thr, Real):
            raise ValueError(f"thr must be a finite real scalar; got {thr!r}.")
        if not math.isfinite(float(thr)):
            raise ValueError(f"thr must be finite; got {thr!r}.")
        if thr_strat == "top_n":
            if not isinstance(thr, Integral) or int(thr) <= 0:
                raise ValueError("top_n threshold must be a positive integer.")
            thr = int(thr)
        elif thr_strat == "percentile":
            if not 0 <= float(thr) <= 100:
                raise ValueError("percentile threshold must lie in [0, 100].")
            thr = float(thr)
        elif thr_strat in {"hard_reassign", "perc_max_abs"}:
            if not 0 <= float(thr) <= 1:
                raise ValueError(f"{thr_strat} threshold must lie in [0, 1].")
            thr = float(thr)
        else:
            if float(thr) < 0:
                raise ValueError(f"{thr_strat} threshold must be non-negative.")
            thr = float(thr)
        if input_type not in {"spatial", "fourier"}:
            raise ValueError(f"input_type must be 'spatial' or 'fourier'; got {input_type!r}.")
        if batch_size <= 0:
            raise ValueError(f"batch_size must be positive; got {batch_size}.")
        if not 0.0 <= adjoint_relative_guard < 1.0:
            raise ValueError(f"adjoint_relative_guard must lie in [0, 1); got {adjoint_relative_guard}.")
        valid_sum = {"all_real", "scan_real", "vmap_real", "all_complex", "scan_complex", "vmap_complex"}
        if sum_method not in valid_sum:
            raise ValueError(f"sum_method must be one of {', '.join(sorted(valid_sum))}; got {sum_method!r}.")
        if precision not in ("fp64", "fp32"):
            raise ValueError(f"precision must be 'fp64' or 'fp32'; got {precision!r}.")
        self.thr = thr
        self.thr_strat = thr_strat
        self.batch_size = batch_size
        self.input_type = input_type
        self.ode_solver = ode_solver
        self.ode_solver_name = solver_name(ode_solver)
        self.closed_form = self.ode_solver_name in CLOSED_FORM
        self.tr_ode_solver = ode_solver if tr_ode_solver is None else tr_ode_solver
        self.sharding = sharding
        if ode_config is None:
            ode_config = SolverConfig.from_precision()
        if not isinstance(ode_config, SolverConfig):
            raise TypeError("ode_config must be a beamax_b200.gb.gb_solvers.SolverConfig")
        self.ode_config = ode_config
        self.adjoint_relative_guard = float(adjoint_relative_guard)
        self.use_real = "real" in sum_method
        self.aggregate_method = "scan" if "scan" in sum_method else ("vmap" if "vmap" in sum_method else "all")
        self.sum_method = sum_method
        self.precision = precision
        self.cutoff = float(cutoff)
        if int(rk4_substeps) < 1:
            raise ValueError("rk4_substeps must be a positive integer.")
        self.rk4_substeps = max(int(rk4_substeps), ode_config.substeps)
        self.trajectory_memory = int(trajectory_memory)
        self.surrogate = surrogate
        self.keep_trajectories = bool(keep_trajectories)
        self.compact_trajectories = bool(compact_trajectories)
        self._traj_cache = None
        self._traj_owner = None
        self._live_est = 0.5  # fraction of (time tile, beam) pairs the compact store keeps
        self._compact_kept = None
        # (b_first, nb, pool blocks, blocks taken) of the last 256 compact integrations
        self.compact_log = collections.deque(maxlen=256)
        # When set to a list, every FP32 summation entry point call appends
        # (name, start event, end event, evaluation counter) recorded on the
        # launching stream around the call.
        self.kernel_timer = None
        # When set to a one-element int64 CUDA tensor, the adaptive ODE adds the
        # number of attempted steps (accepted + rejected) of every integration to it.
        self.ode_step_counter = None
        self.last_surrogate_accepted: Optional[int] = None
        self._accepted = None
        self.last_selection: Optional[Selection] = None
        self.last_eval_count: Optional[int] = None

    # ------------------------------------------------------------- helpers
    def _effective_top_n(self, wpt: MSWPT, *, half_frame: bool = False):
        """msgb_solver.py:536-549."""
        if self.thr_strat != "top_n":
            return self.thr
        cap = wpt.half_frame_capacity() if half_frame else wpt.total_coeffs
        return min(int(self.thr), int(cap))

    @staticmethod
    def _sensor_positions(sensors) -> np.ndarray:
        if isinstance(sensors, Sensor):
            return sensors.positions
        if hasattr(sensors, "detach"):
            return sensors.detach().cpu().numpy()
        if isinstance(sensors, np.ndarray):
            return sensors
        raise ValueError("Unsupported sensor type")

    def _problem(self, domain: Domain, sensors, ts, device):
        import torch

        kind, m = domain.medium()
        if kind == "constant":
            c = float(m)
        elif self.closed_form:
            # solve_hom_diag / solve_hom_general propagate at c(0) (gb_solvers.py:356-422)
            c = float(np.asarray(m(np.zeros((1, domain.ndim)))).ravel()[0])
        else:
            c = float(np.max(m.values))  # unused by the trajectory kernels
        pos = np.ascontiguousarray(self._sensor_positions(sensors), np.float64)
        if pos.ndim != 2 or pos.shape[1] != domain.ndim:
            raise ValueError(f"sensor positions must have shape (Ns, {domain.ndim})")
        ts_np = np.ascontiguousarray(ts.detach().cpu().numpy() if hasattr(ts, "detach") else np.asarray(ts),
                                     np.float64)
        ts_d = torch.from_numpy(ts_np).to(device)
        sens_key = sensors if isinstance(sensors, Sensor) else None
        if sens_key is not None:
            sd = _cache.get(sens_key, ("pos", str(device)), lambda: torch.from_numpy(pos).to(device))
        else:
            sd = torch.from_numpy(pos).to(device)
        L = domain.grid_size
        pr = _lib.Problem()
        pr.ndim = domain.ndim
        for a in range(3):
            pr.periodic[a] = int(domain.periodic[a]) if a < domain.ndim else 0
            pr.L[a] = float(L[a]) if a < domain.ndim else 1.0
        pr.c = float(c)
        pr.nt = ts_np.size
        pr.ts = ts_d.data_ptr()
        pr.ns = pos.shape[0]
        pr.sensors = sd.data_ptr()
        pr._owned = (ts_d, sd)  # the device arrays live as long as the struct that points at them
        return pr, (ts_d, sd)

    def _tiling(self, domain: Domain, sensors, device):
        """Run-based sensor tiling (cached per Sensor object), or None."""
        import torch

        from ..sensor_layout import build_tiling

        def make():
            t = build_tiling(self._sensor_positions(sensors), domain.dx)
            if t is None:
                return None
            order, offs = t
            od = torch.from_numpy(order).to(device)
            fd = torch.from_numpy(offs).to(device)
            st = _lib.SensorTiling(n_tiles=offs.size - 1, order=od.data_ptr(), tile_offsets=fd.data_ptr())
            return st, od, fd

        if isinstance(sensors, Sensor):
            return _cache.get(sensors, ("tiling", str(device), tuple(domain.dx)), make)
        return make()

    # ------------------------------------------------------------- pipeline
    def select(self, p0, domain: Domain, wpt: MSWPT, dpdt=None) -> Selection:
        """c_pos on the GPU, then the threshold (msgb_solver.py:570-612)."""
        import torch

        x = as_device_f64(p0)
        dz = None
        if dpdt is not None:
            dz = as_device_f64(dpdt, x.device)
            if not bool((dz != 0).any()):
                dz = None
        if x.is_complex() or (dz is not None and dz.is_complex()):
            return self._select_branches(x, dz, domain, wpt)
        if dz is None:
            coeffs, keys = wpt.forward_device(x, self.input_type, scale=0.5, half_mask=True, keys=True)
        else:
            coeffs, keys = self._coefficients_dpdt(x, dz, domain, wpt, branch=1, half_mask=True)
        return self._select_from(coeffs, keys, wpt, x.device, self._effective_top_n(wpt, half_frame=True))

    def _select_branches(self, x, dz, domain: Domain, wpt: MSWPT) -> BranchSelection:
        """Complex input (msgb_solver.py:635-689): c_pos and c_neg of
        compute_coefficients(mode="both") thresholded separately with the
        uncapped top_n (no half-frame mask)."""
        if dz is None:
            c, k = wpt.forward_device(x, self.input_type, scale=0.5, keys=True)
            cp, kp, cn, kn = c, k, c, k
        else:
            cp, kp = self._coefficients_dpdt(x, dz, domain, wpt, branch=1, half_mask=False)
            cn, kn = self._coefficients_dpdt(x, dz, domain, wpt, branch=-1, half_mask=False)
        n = self._effective_top_n(wpt)
        return BranchSelection(self._select_from(cp, kp, wpt, x.device, n), self._select_from(cn, kn, wpt, x.device, n))

    def _select_from(self, coeffs, keys, wpt: MSWPT, dev, n) -> Selection:
        import torch

        if self.thr_strat != "top_n":
            return self._select_masked(coeffs, keys, wpt, dev)
        idx = torch.empty(n, dtype=torch.int64, device=dev)
        vals = torch.empty(n, dtype=torch.complex128, device=dev)
        nbytes = _lib.lib().msgb_topn_workspace_size(wpt.total_coeffs, n)
        ws = workspace(dev, "topn", nbytes)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_topn(keys.data_ptr(), torch.view_as_real(coeffs).data_ptr(), wpt.total_coeffs,
                                        n, idx.data_ptr(), torch.view_as_real(vals).data_ptr(), ws.data_ptr(),
                                        nbytes, st), "msgb_topn")
        return Selection(idx, vals, wpt.total_coeffs)

    def _coefficients_dpdt(self, x, dz, domain: Domain, wpt: MSWPT, branch: int, half_mask: bool):
        """c = 0.5 (MSWPT(p0) + branch i MSWPT(dpdt) / vg) and its keys
        (forward_solver_utils.py:716-786) via msgb_coefficients_dpdt."""
        import torch

        dev = x.device
        a = wpt.forward_device(x, self.input_type, scale=1.0)
        b = wpt.forward_device(dz, self.input_type, scale=1.0)
        med, keep_m = self._medium(domain, dev)
        d = domain.ndim
        L = (ctypes.c_double * 3)(*[float(v) for v in domain.grid_size], *([1.0] * (3 - d)))
        out = torch.empty_like(a)
        keys = torch.empty(a.shape[0], dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_coefficients_dpdt(wpt.plan(dev), L, _lib.ref(med), torch.view_as_real(a).data_ptr(),
                                                     torch.view_as_real(b).data_ptr(), int(branch), int(half_mask),
                                                     torch.view_as_real(out).data_ptr(), keys.data_ptr(), st),
                   "msgb_coefficients_dpdt")
        return out, keys

    _THR_CODE = {"hard": 0, "percentile": 1, "hard_reassign": 2, "bao_energy": 3, "perc_max_abs": 4}

    def _select_masked(self, coeffs, keys, wpt: MSWPT, dev) -> Selection:
        """hard / percentile / hard_reassign / bao_energy / perc_max_abs
        (forward_solver_utils.py:14-178) via msgb_threshold; one device-to-host
        read of the selected count."""
        import torch

        total = wpt.total_coeffs
        idx = torch.empty(total, dtype=torch.int64, device=dev)
        vals = torch.empty(total, dtype=torch.complex128, device=dev)
        count = torch.zeros(1, dtype=torch.int64, device=dev)
        nbytes = _lib.lib().msgb_threshold_workspace_size(total)
        ws = workspace(dev, "threshold", nbytes)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_threshold(self._THR_CODE[self.thr_strat], float(self.thr), keys.data_ptr(),
                                             torch.view_as_real(coeffs).data_ptr(), total, wpt.plan(dev),
                                             idx.data_ptr(), torch.view_as_real(vals).data_ptr(), count.data_ptr(),
                                             ws.data_ptr(), nbytes, st), "msgb_threshold")
        n = int(count.item())
        return Selection(idx[:n].clone(), vals[:n].clone(), total)

    def beams(self, sel: Selection, domain: Domain, wpt: MSWPT) -> BeamTensors:
        """Beam data for a selection (compute_forward_parameters, a0 *= coefficient)."""
        import torch

        dev = sel.idx.device
        n = int(sel.idx.shape[0])
        d = domain.ndim
        x0 = torch.empty((n, d), dtype=torch.float64, device=dev)
        p0 = torch.empty((n, d), dtype=torch.float64, device=dev)
        al = torch.empty((n, d), dtype=torch.complex128, device=dev)
        a0 = torch.empty(n, dtype=torch.complex128, device=dev)
        a0u = torch.empty(n, dtype=torch.complex128, device=dev)
        om = torch.empty(n, dtype=torch.float64, device=dev)
        out = _lib.BeamOut(x0=x0.data_ptr(), p0=p0.data_ptr(), alpha=torch.view_as_real(al).data_ptr(),
                           a0=torch.view_as_real(a0).data_ptr(), omega=om.data_ptr(),
                           a0_unit=torch.view_as_real(a0u).data_ptr())
        L = (ctypes.c_double * 3)(*[float(v) for v in domain.grid_size], *([1.0] * (3 - d)))
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_beam_init(wpt.plan(dev), L, sel.idx.data_ptr(),
                                             torch.view_as_real(sel.values).data_ptr(), n, _lib.ref(out), st),
                   "msgb_beam_init")
        return BeamTensors(x0, p0, al, a0, a0u, om)

    # ------------------------------------------------------------- heterogeneous
    def _medium(self, domain: Domain, device):
        import torch

        from ..utils.interp import BOUNDARY_CODE

        kind, m = domain.medium()
        med = _lib.Medium()
        med.lam = float(domain.lam)
        if kind == "constant":
            med.kind = 0
            med.c = float(m)
            return med, None
        med.kind = 1 if m.method == "linear" else 2
        med.boundary = BOUNDARY_CODE[m.boundary]
        for a in range(3):
            med.n[a] = m.coeffs.shape[a] if a < m.ndim else 1
            med.spacing[a] = float(m.spacing[a]) if a < m.ndim else 1.0
            med.origin[a] = float(m.origin[a]) if a < m.ndim else 0.0
        coeffs = _cache.get(m, ("coeffs", str(device)), lambda: torch.from_numpy(m.coeffs).to(device))
        med.coeffs = coeffs.data_ptr()
        med.c = float(np.max(m.values))
        if self.precision == "fp32":
            # FP32 copy for the FP32 path's medium evaluation: offsets from the
            # mean keep FP32's relative precision on the variation of c
            c_ref = float(np.mean(m.coeffs))
            c32 = _cache.get(m, ("coeffs32", str(device)),
                             lambda: torch.from_numpy((m.coeffs - c_ref).astype(np.float32)).to(device))
            med.coeffs32 = c32.data_ptr()
            med.c_ref = c_ref
            return med, (coeffs, c32)
        return med, coeffs

    @staticmethod
    def heterogeneous(domain: Domain) -> bool:
        return domain.medium()[0] != "constant" or domain.lam != 0.0

    def _integrates(self, domain: Domain) -> bool:
        """The beams go through the ODE kernels: a heterogeneous or absorbing
        medium with an ODE propagator (the closed forms ignore both, as the
        reference's do)."""
        return not self.closed_form and self.heterogeneous(domain)

    def _chunks(self, domain: Domain, nt: int, nbeam: int, fp64: bool, budget: Optional[int] = None):
        d = domain.ndim
        S = d * (d + 1) // 2
        n_tt = (nt + 31) // 32
        per = nt * ((2 * d + 2 * d * d + 2) * 8 if fp64 else (16 * d + 8 * S + 8)) + n_tt * (2 * d + 1) * 4
        chunk = max(1, min(nbeam, (budget or self.trajectory_memory) // max(per, 1)))
        return [(b, min(chunk, nbeam - b)) for b in range(0, nbeam, chunk)], per, n_tt

    def _ode_opts(self, ts):
        cfg = self.ode_config
        if cfg.method == "rk4":
            return _lib.OdeOpts(method=0, substeps=self.rk4_substeps)
        return _lib.OdeOpts(method=1, substeps=1, rtol=float(cfg.rtol), atol=float(cfg.atol),
                            dt0=float(cfg.dt0) if cfg.dt0 is not None else 0.0, max_steps=int(cfg.max_steps),
                            dense_output=int(bool(cfg.dense_output)),
                            medium_fp32=int(self.precision == "fp32"))

    def _mode_chunks(self, domain: Domain, nt: int, bt: BeamTensors, fp64: bool):
        """Chunks over the beams of the summed branches: [0, 2n), [0, n) (mode
        +1 only) or [n, 2n) (mode -1 only)."""
        n = bt.n
        lo, hi = {0: (0, 2 * n), 1: (0, n), 2: (n, 2 * n)}[bt.modes]
        budget = self._trajectory_budget(bt.x0.device)
        if self.keep_trajectories and (fp64 or not self._compact()):
            budget //= 2  # the dense path may hold a kept chunk beside the chunk buffer
        chunks, per, n_tt = self._chunks(domain, nt, hi - lo, fp64, budget)
        return [(lo + b, nb) for b, nb in chunks], per, n_tt

    def _trajectories(self, pr, med, bs, b_first, nb, fp64, per, n_tt, dev, st, status, buf=None):
        if buf is None:
            buf = workspace(dev, "traj", per * nb + 4096)
        base = buf.data_ptr()
        d = pr.ndim
        S = d * (d + 1) // 2
        rec_bytes = pr.nt * nb * ((2 * d + 2 * d * d + 2) * 8 if fp64 else (16 * d + 8 * S + 8))
        cull_off = (rec_bytes + 255) // 256 * 256
        tr = _lib.Trajectories(nb=nb, b_first=b_first, rec64=base if fp64 else None, rec32=None if fp64 else base,
                               cull=None if fp64 else base + cull_off,
                               status=status.data_ptr() + 4 * b_first)
        opts = self._ode_opts(None)
        if self.ode_step_counter is not None:
            opts.step_count = self.ode_step_counter.data_ptr()
        if self.surrogate is not None:
            self.surrogate.predict_into(pr, med, bs, b_first, nb, tr)
            acc = (status[b_first:b_first + nb] == 0).sum()
            self._accepted = acc if self._accepted is None else self._accepted + acc
            opts.only_flagged = 1
        with self._kernel_span("msgb_ode_trajectories", None):
            _lib.check(_lib.lib().msgb_ode_trajectories(_lib.ref(pr), _lib.ref(med), _lib.ref(bs), _lib.ref(opts),
                                                        _lib.ref(tr), st), "msgb_ode_trajectories")
        return tr, buf

    # ---- compact FP32 trajectory store -----------------------------------
    def _compact(self) -> bool:
        """FP32 records are kept only for (time tile, beam) pairs within the
        cutoff of some sensor tile (the summation skips the others anyway)."""
        return (self.compact_trajectories and self.precision == "fp32" and self.surrogate is None
                and self.cutoff > 0)

    def _live_boxes(self, pr, opts, domain, sensors, dev, st):
        """The summation's sensor-tile boxes (n_tiles, 2 d) on the device."""
        import torch

        def make():
            n = int(_lib.lib().msgb_sum_f32_tile_count(_lib.ref(pr), _lib.ref(opts)))
            nbytes = _lib.lib().msgb_sum_f32_traj_workspace_size(_lib.ref(pr), 0)
            ws = workspace(dev, "sum32traj", nbytes)
            boxes = torch.empty((max(n, 1), 2 * pr.ndim), dtype=torch.float32, device=dev)
            _lib.check(_lib.lib().msgb_sum_f32_tile_boxes(_lib.ref(pr), _lib.ref(opts), ws.data_ptr(), nbytes,
                                                          boxes.data_ptr(), st), "msgb_sum_f32_tile_boxes")
            return boxes, n

        if isinstance(sensors, Sensor):
            return _cache.get(sensors, ("live_boxes", str(dev), tuple(domain.dx), pr.nt), make)
        return make()

    @staticmethod
    def _compact_sizes(d: int, nt: int):
        S = d * (d + 1) // 2
        n_tt = (nt + 31) // 32
        block = 32 * (16 * d + 8 * S + 8)          # one time tile of FP32 records
        cull = (2 * d + 1) * 4
        return n_tt, block, cull

    def _trajectory_budget(self, dev) -> int:
        """Bytes for one chunk of trajectory records: trajectory_memory, or
        what the device has free less 4 GiB of headroom.  Free includes the
        memory torch's allocator holds in its cache (freed tensors, e.g. the
        previous step's records), which it hands out again."""
        import torch

        free, _ = torch.cuda.mem_get_info(dev)
        free += torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
        return int(max(1 << 20, min(self.trajectory_memory, free - (4 << 30))))

    def _compact_chunk_beams(self, d, nt, nbeam, budget):
        """Beams per chunk for the estimated fraction of live tiles (each beam
        may also leave one block that no live tile took)."""
        n_tt, block, cull = self._compact_sizes(d, nt)
        per_beam = n_tt * 4 + self._live_est * n_tt * (block + cull) + (block + cull)
        return int(max(1, min(nbeam, (budget - 4096) // max(per_beam, 1))))

    def _compact_tr(self, buf, d, nt, b_first, nb, status, boxes, n_boxes):
        """Lay out the slot table, counter, culling boxes and record blocks of
        one chunk in buf; returns (Trajectories, blocks, counter view)."""
        n_tt, block, cull = self._compact_sizes(d, nt)
        base = buf.data_ptr()
        al = lambda x: (x + 255) // 256 * 256
        slot_b = al(n_tt * nb * 4)
        ctr_off = slot_b
        rest = buf.numel() - slot_b - 512
        blocks = max(0, rest // (block + cull) - 2)
        cull_off = slot_b + 256
        pool_off = al(cull_off + blocks * cull)
        blocks = max(0, min(blocks, (buf.numel() - pool_off) // block))
        tr = _lib.Trajectories(nb=nb, b_first=b_first, status=status.data_ptr() + 4 * b_first,
                               slot=base, pool=base + pool_off, pool_cull=base + cull_off, pool_blocks=blocks,
                               pool_next=base + ctr_off, live_boxes=boxes.data_ptr(), n_boxes=n_boxes,
                               live_cutoff=float(self.cutoff))
        ctr = buf[ctr_off:ctr_off + 8].view(dtype=__import__("torch").int64)
        return tr, blocks, ctr

    def _compact_integrate(self, pr, med, bs, lo, hi, domain, sensors, opts, dev, st, status, keep=False,
                           skip=None):
        """Integrate beams [lo, hi) into compact chunks, yielding (tr, first,
        last) per chunk in beam order.  A chunk whose pool runs out (more live
        tiles than estimated) is split in two and integrated again.  skip:
        (b_first, nb) of a chunk the caller already holds (not integrated).
        keep: the buffer of the last chunk is returned in self._compact_kept."""
        import torch

        d = pr.ndim
        n_tt, block, cull = self._compact_sizes(d, pr.nt)
        boxes, n_boxes = self._live_boxes(pr, opts, domain, sensors, dev, st)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        lanes = 4 * sms * 64  # the integrator's resident lanes
        todo = []
        ranges = [(lo, hi)] if skip is None else [(lo, skip[0]), (skip[0] + skip[1], hi)]
        budget = self._trajectory_budget(dev)
        cb = 1
        for a, b in ranges:
            if b <= a:
                continue
            cb = self._compact_chunk_beams(d, pr.nt, b - a, budget)
            todo += [(x, min(cb, b - x)) for x in range(a, b, cb)]
        if not todo:
            return
        # the chunk's estimated need (plus one block per integrator lane), not the whole budget
        widest = max(nb for _, nb in todo)
        need = int(widest * n_tt * (4 + self._live_est * (block + cull)) + min(widest, lanes) * (block + cull)
                   + 4096)
        buf = None
        size = min(budget, need)
        while buf is None:
            try:
                buf = torch.empty(size, dtype=torch.uint8, device=dev)
            except torch.OutOfMemoryError:
                # the allocator's cache may be fragmented: return it to the
                # driver and retry once at this size, then halve the chunks
                torch.cuda.empty_cache()
                try:
                    buf = torch.empty(size, dtype=torch.uint8, device=dev)
                except torch.OutOfMemoryError:
                    if widest == 1:
                        raise
                    widest = (widest + 1) // 2
                    todo = [(x, min(widest, b0 + n0 - x)) for b0, n0 in todo for x in range(b0, b0 + n0, widest)]
                    size = int(widest * n_tt * (4 + self._live_est * (block + cull))
                               + min(widest, lanes) * (block + cull) + 4096)
        first = True
        opts_ode = self._ode_opts(None)
        if self.ode_step_counter is not None:
            opts_ode.step_count = self.ode_step_counter.data_ptr()
        while todo:
            b_first, nb = todo.pop(0)
            tr, blocks, ctr = self._compact_tr(buf, d, pr.nt, b_first, nb, status, boxes, n_boxes)
            ctr.zero_()
            with self._kernel_span("msgb_ode_trajectories", None):
                _lib.check(_lib.lib().msgb_ode_trajectories(_lib.ref(pr), _lib.ref(med), _lib.ref(bs),
                                                            _lib.ref(opts_ode), _lib.ref(tr), st),
                           "msgb_ode_trajectories")
            used = int(ctr.item())
            self.compact_log.append((b_first, nb, blocks, used))
            if used > blocks:
                if nb == 1:
                    raise RuntimeError("compact trajectory store: one beam needs more than the budget")
                self._live_est = min(1.0, self._live_est * 2.0)
                todo[:0] = [(b_first, nb // 2), (b_first + nb // 2, nb - nb // 2)]
                continue
            self._live_est = min(1.0, max(0.05, 1.15 * max(0, used - min(nb, lanes)) / max(1, n_tt * nb)))
            if keep and not todo:
                self._compact_kept = buf
            yield tr, first, not todo
            first = False

    def _begin_trajectories(self, domain, ts):
        self._accepted = None
        if self.surrogate is not None:
            if getattr(self.surrogate, "_key", None) != self.surrogate.medium_key(domain, ts):
                raise ValueError("the surrogate was fitted for another medium or time grid")

    @contextlib.contextmanager
    def _kernel_span(self, name, counter):
        if self.kernel_timer is None:
            yield
            return
        import torch

        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        yield
        b.record()
        self.kernel_timer.append((name, a, b, counter))

    def _check_status(self, status):
        """Raise, as the reference's diffeqsolve does, when an integration failed."""
        if self.surrogate is not None:
            self.last_surrogate_accepted = int(self._accepted.item()) if self._accepted is not None else 0
        worst = int(status.max().item()) if status.numel() else 0
        if worst == 2:
            n = int((status == 2).sum().item())
            raise RuntimeError(f"ODE integration reached max_steps={self.ode_config.max_steps} for {n} beam(s); "
                               "raise SolverConfig.max_steps or loosen rtol/atol")
        if worst == 1:
            n = int((status == 1).sum().item())
            raise RuntimeError(f"ODE integration produced a non-finite state for {n} beam(s); "
                               "increase rk4_substeps or use an adaptive solver")

    def _sum_forward_het(self, bt: BeamTensors, domain: Domain, sensors, ts):
        import torch

        dev = bt.x0.device
        pr, keep = self._problem(domain, sensors, ts, dev)
        med, keep_m = self._medium(domain, dev)
        bs = bt.beam_set(unit=False)
        st = torch.cuda.current_stream(dev).cuda_stream
        fp64 = self.precision == "fp64"
        chunks, per, n_tt = self._mode_chunks(domain, pr.nt, bt, fp64)
        status = torch.zeros(2 * bt.n, dtype=torch.int32, device=dev)
        self._begin_trajectories(domain, ts)
        self._traj_cache = None
        keep_buf = None if (not fp64 and self._compact()) else self._keep_buffer(chunks, per, dev)
        last = len(chunks) - 1
        if fp64:
            out = torch.zeros((pr.nt, pr.ns), dtype=torch.float64, device=dev)
            for i, (b_first, nb) in enumerate(chunks):
                tr, buf = self._trajectories(pr, med, bs, b_first, nb, True, per, n_tt, dev, st, status,
                                             keep_buf if i == last else None)
                _lib.check(_lib.lib().msgb_sum_fwd_f64_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr), out.data_ptr(),
                                                            st), "msgb_sum_fwd_f64_traj")
            self._check_status(status)
            self._remember_trajectories(keep_buf, tr, domain, ts, pr.nt)
            return out
        out = torch.empty((pr.nt, pr.ns), dtype=torch.float32, device=dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        tiling = self._tiling(domain, sensors, dev)
        opts = _lib.SumOpts(cutoff=self.cutoff, eval_count=cnt.data_ptr(),
                            tiling=_lib.ref(tiling[0]) if tiling else None)
        if self._compact():
            keep_buf = None  # the compact path keeps its own last chunk
            lo, hi = chunks[0][0], chunks[-1][0] + chunks[-1][1]
            keep_last = self.keep_trajectories and self._traj_owner is not None
            self._compact_kept = None
            # the forward keeps its Kahan state in this workspace from the first
            # chunk to the last: one size (no per-chunk partials), never regrown
            nbytes = _lib.lib().msgb_sum_f32_traj_workspace_size(_lib.ref(pr), 0)
            ws = workspace(dev, "sum32traj", nbytes)
            for tr, first, last in self._compact_integrate(pr, med, bs, lo, hi, domain, sensors, opts, dev, st,
                                                          status, keep=keep_last):
                with self._kernel_span("msgb_sum_fwd_f32_traj", cnt):
                    _lib.check(_lib.lib().msgb_sum_fwd_f32_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr),
                                                                _lib.ref(opts), int(first), int(last), ws.data_ptr(),
                                                                nbytes, out.data_ptr(), st), "msgb_sum_fwd_f32_traj")
            self._eval_counter = cnt
            self._check_status(status)
            self._remember_trajectories(self._compact_kept, tr, domain, ts, pr.nt)
            self._compact_kept = None
            return out
        nbytes = _lib.lib().msgb_sum_f32_traj_workspace_size(_lib.ref(pr), max(nb for _, nb in chunks))
        ws = workspace(dev, "sum32traj", nbytes)
        for i, (b_first, nb) in enumerate(chunks):
            tr, buf = self._trajectories(pr, med, bs, b_first, nb, False, per, n_tt, dev, st, status,
                                         keep_buf if i == last else None)
            with self._kernel_span("msgb_sum_fwd_f32_traj", cnt):
                _lib.check(_lib.lib().msgb_sum_fwd_f32_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr), _lib.ref(opts),
                                                            int(i == 0), int(i == len(chunks) - 1), ws.data_ptr(),
                                                            nbytes, out.data_ptr(), st), "msgb_sum_fwd_f32_traj")
        self._eval_counter = cnt
        self._check_status(status)
        self._remember_trajectories(keep_buf, tr, domain, ts, pr.nt)
        return out

    def _keep_buffer(self, chunks, per, dev):
        """Own memory for the records of the forward's last chunk of beams, so
        that an adjoint with the same selection reads them instead of
        integrating those beams again.  One chunk: the whole step integrates
        once.  Several chunks (records larger than trajectory_memory): the
        last chunk is kept when the device has room for a second buffer."""
        import torch

        if not self.keep_trajectories or self._traj_owner is None:
            return None
        self._traj_cache = None  # free the previous forward's records first
        size = per * chunks[-1][1] + 4096
        if self._trajectory_budget(dev) < size:
            return None
        return torch.empty(size, dtype=torch.uint8, device=dev)

    def release_trajectories(self) -> None:
        """Drop the trajectory records kept for the next adjoint (frees their
        device memory)."""
        self._traj_cache = None

    def _propagation_key(self, domain):
        """What the kept records depend on besides the selection and the time
        grid: the medium object and absorption, the integrator settings and
        the surrogate."""
        kind, m = domain.medium()
        return (kind, float(m) if kind == "constant" else id(m), float(domain.lam), repr(self.ode_config),
                self.rk4_substeps, id(self.surrogate))

    def _remember_trajectories(self, buf, tr, domain, ts, nt):
        """Keep the forward's last chunk of records (they stay on the device
        until the next forward of this solver) for an adjoint with the same
        selection, domain, time grid and propagation settings."""
        if buf is None:
            self._traj_cache = None
            return
        tr.status = None  # the forward's status array is not kept
        self._traj_cache = {"selection": self._traj_owner, "domain": domain, "ts": ts, "nt": nt,
                            "precision": self.precision, "tr": tr, "buf": buf,
                            "key": self._propagation_key(domain)}

    def _cached_trajectories(self, selection, domain, ts):
        c = self._traj_cache
        if (c is not None and c["selection"] is selection and c["domain"] is domain and c["ts"] is ts
                and c["precision"] == self.precision and c["key"] == self._propagation_key(domain)):
            return c
        return None

    def _gather_adjoint_het(self, bt: BeamTensors, domain: Domain, sensors, ts, data, cached=None):
        import torch

        dev = bt.x0.device
        pr, keep = self._problem(domain, sensors, ts, dev)
        med, keep_m = self._medium(domain, dev)
        bs = bt.beam_set(unit=True)
        st = torch.cuda.current_stream(dev).cuda_stream
        fp64 = self.precision == "fp64"
        n = bt.n
        chunks, per, n_tt = self._mode_chunks(domain, pr.nt, bt, fp64)
        g_all = torch.zeros(2 * n, dtype=torch.complex128, device=dev)
        if fp64:
            d = as_device_f64(data, dev).reshape(pr.nt, pr.ns).contiguous()
        elif isinstance(data, torch.Tensor) and data.is_cuda and data.dtype == torch.float32:
            d = data.reshape(pr.nt, pr.ns).contiguous()
        else:
            d = as_device_f64(data, dev).to(torch.float32).reshape(pr.nt, pr.ns).contiguous()
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        tiling = None if fp64 else self._tiling(domain, sensors, dev)
        opts = _lib.SumOpts(cutoff=self.cutoff, eval_count=cnt.data_ptr(),
                            tiling=_lib.ref(tiling[0]) if tiling else None)
        nbytes = 0 if fp64 else _lib.lib().msgb_sum_f32_traj_workspace_size(_lib.ref(pr), max(nb for _, nb in chunks))
        ws = None if fp64 else workspace(dev, "sum32traj", nbytes)
        status = torch.zeros(2 * n, dtype=torch.int32, device=dev)
        self._begin_trajectories(domain, ts)
        kept = (cached["tr"].b_first, cached["tr"].nb) if cached is not None else None
        if not fp64 and self._compact():
            lo, hi = chunks[0][0], chunks[-1][0] + chunks[-1][1]
            trs = []
            if kept is not None and lo <= kept[0] and kept[0] + kept[1] <= hi:
                trs.append(cached["tr"])  # the forward's records for these beams
            else:
                kept = None
            gen = self._compact_integrate(pr, med, bs, lo, hi, domain, sensors, opts, dev, st, status, skip=kept)
            for tr in _chain(trs, (t for t, _, _ in gen)):
                nbytes = _lib.lib().msgb_sum_f32_traj_workspace_size(_lib.ref(pr), tr.nb)
                ws = workspace(dev, "sum32traj", nbytes)
                gp = torch.view_as_real(g_all[tr.b_first:tr.b_first + tr.nb]).data_ptr()
                with self._kernel_span("msgb_adj_gather_f32_traj", cnt):
                    _lib.check(_lib.lib().msgb_adj_gather_f32_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr),
                                                                   _lib.ref(opts), ws.data_ptr(), nbytes,
                                                                   d.data_ptr(), gp, st), "msgb_adj_gather_f32_traj")
            self._eval_counter = cnt
            self._check_status(status)
            return g_all[:n] + g_all[n:]
        for b_first, nb in chunks:
            if (b_first, nb) == kept:
                tr = cached["tr"]  # the forward's records for these beams, in this order
            else:
                tr, _ = self._trajectories(pr, med, bs, b_first, nb, fp64, per, n_tt, dev, st, status)
            gp = torch.view_as_real(g_all[b_first:b_first + nb]).data_ptr()
            if fp64:
                _lib.check(_lib.lib().msgb_adj_gather_f64_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr), d.data_ptr(),
                                                               gp, st), "msgb_adj_gather_f64_traj")
            else:
                with self._kernel_span("msgb_adj_gather_f32_traj", cnt):
                    _lib.check(_lib.lib().msgb_adj_gather_f32_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr),
                                                                   _lib.ref(opts), ws.data_ptr(), nbytes,
                                                                   d.data_ptr(), gp, st), "msgb_adj_gather_f32_traj")
        self._eval_counter = cnt
        self._check_status(status)
        return g_all[:n] + g_all[n:]

    def sum_forward(self, bt: BeamTensors, domain: Domain, sensors, ts):
        """Beam summation at the sensors: (Nt, Ns) float64 (fp64) or float32 (fp32)."""
        import torch

        if self._integrates(domain):
            return self._sum_forward_het(bt, domain, sensors, ts)

        dev = bt.x0.device
        pr, keep = self._problem(domain, sensors, ts, dev)
        bs = bt.beam_set(unit=False)
        st = torch.cuda.current_stream(dev).cuda_stream
        if self.precision == "fp64":
            out = torch.empty((pr.nt, pr.ns), dtype=torch.float64, device=dev)
            _lib.check(_lib.lib().msgb_sum_fwd_f64(_lib.ref(pr), _lib.ref(bs), out.data_ptr(), st),
                       "msgb_sum_fwd_f64")
            return out
        out = torch.empty((pr.nt, pr.ns), dtype=torch.float32, device=dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        tiling = self._tiling(domain, sensors, dev)
        opts = _lib.SumOpts(cutoff=self.cutoff, eval_count=cnt.data_ptr(),
                            tiling=_lib.ref(tiling[0]) if tiling else None)
        nbytes = _lib.lib().msgb_sum_f32_workspace_size(_lib.ref(pr), bt.n)
        ws = workspace(dev, "sum32", nbytes)
        with self._kernel_span("msgb_sum_fwd_f32", cnt):
            _lib.check(_lib.lib().msgb_sum_fwd_f32(_lib.ref(pr), _lib.ref(bs), _lib.ref(opts), ws.data_ptr(),
                                                   nbytes, out.data_ptr(), st), "msgb_sum_fwd_f32")
        self._eval_counter = cnt
        return out

    def gather_adjoint(self, bt: BeamTensors, domain: Domain, sensors, ts, data, _cached=None):
        """Per selected coefficient g_j = sum 2 d conj(K_j) over both modes: (n,) complex128."""
        import torch

        if self._integrates(domain):
            return self._gather_adjoint_het(bt, domain, sensors, ts, data, _cached)

        dev = bt.x0.device
        pr, keep = self._problem(domain, sensors, ts, dev)
        bs = bt.beam_set(unit=True)
        g = torch.empty(bt.n, dtype=torch.complex128, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        if self.precision == "fp64":
            d = as_device_f64(data, dev).reshape(pr.nt, pr.ns).contiguous()
            _lib.check(_lib.lib().msgb_adj_gather_f64(_lib.ref(pr), _lib.ref(bs), d.data_ptr(),
                                                      torch.view_as_real(g).data_ptr(), st), "msgb_adj_gather_f64")
            return g
        if isinstance(data, torch.Tensor) and data.is_cuda and data.dtype == torch.float32:
            d = data.reshape(pr.nt, pr.ns).contiguous()
        else:
            d = as_device_f64(data, dev).to(torch.float32).reshape(pr.nt, pr.ns).contiguous()
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        tiling = self._tiling(domain, sensors, dev)
        opts = _lib.SumOpts(cutoff=self.cutoff, eval_count=cnt.data_ptr(),
                            tiling=_lib.ref(tiling[0]) if tiling else None)
        nbytes = _lib.lib().msgb_sum_f32_workspace_size(_lib.ref(pr), bt.n)
        ws = workspace(dev, "sum32", nbytes)
        with self._kernel_span("msgb_adj_gather_f32", cnt):
            _lib.check(_lib.lib().msgb_adj_gather_f32(_lib.ref(pr), _lib.ref(bs), _lib.ref(opts), ws.data_ptr(),
                                                      nbytes, d.data_ptr(), torch.view_as_real(g).data_ptr(), st),
                       "msgb_adj_gather_f32")
        self._eval_counter = cnt
        return g

    def coefficient_adjoint(self, sel: Selection, g, wpt: MSWPT):
        """Transpose of c_pos[idx] -> image: scatter 0.5 * g (half mask), MSWPT^H, real part."""
        import torch

        dev = g.device
        G = torch.zeros(wpt.total_coeffs, dtype=torch.complex128, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_scatter_coeff_grad(sel.idx.data_ptr(), torch.view_as_real(g).data_ptr(),
                                                      int(sel.idx.shape[0]), 0.5, wpt.plan(dev), 1,
                                                      torch.view_as_real(G).data_ptr(), st),
                   "msgb_scatter_coeff_grad")
        return wpt.adjoint(G, "spatial", real_output=True)

    # ------------------------------------------------------------- public API
    def _check_forward_args(self, p0, domain: Domain, ts, wpt: MSWPT, dpdt):
        shape = tuple(p0.shape)
        if shape != domain.N or (dpdt is not None and tuple(dpdt.shape) != domain.N):
            raise ValueError(f"p0 and dpdt must both have shape {domain.N}; got {shape} and "
                             f"{tuple(dpdt.shape) if dpdt is not None else shape}.")
        if wpt.dyadic_decomp.N != domain.N:
            raise ValueError("wpt grid shape must match domain.N.")
        _validate_time_grid(ts, allow_singleton=True)

    def forward(self, p0, domain: Domain, sensors, ts, wpt: MSWPT, *, dpdt=None):
        """Pressure at the sensors, shape (Nt, Ns) (msgb_solver.py:858-899)."""
        data, _ = self._forward_impl(p0, domain, sensors, ts, wpt, dpdt, want_params=False)
        return data

    def forward_frozen(self, p0, domain: Domain, sensors, ts, wpt: MSWPT, selection: Selection):
        """A_S p0: the forward with the beam selection S frozen, i.e. the
        linear map whose exact transpose ``adjoint(..., selection=S)`` is.
        The coefficients of p0 at S's indices drive S's beams."""
        self._check_forward_args(p0, domain, ts, wpt, None)
        x = as_device_f64(p0)
        if isinstance(selection, BranchSelection):
            c = wpt.forward_device(x, self.input_type, scale=0.5)
            take = lambda s: Selection(s.idx, c[s.idx], s.total_coeffs)
            bts = [replace(self.beams(take(selection.pos), domain, wpt), modes=1),
                   replace(self.beams(take(selection.neg), domain, wpt), modes=2)]
        else:
            c = wpt.forward_device(x, self.input_type, scale=0.5, half_mask=True)
            sel = Selection(selection.idx, c[selection.idx], selection.total_coeffs)
            bts = [self.beams(sel, domain, wpt)]
        out = self._sum_beam_sets(bts, domain, sensors, ts)
        return out if _is_torch(p0) else out.cpu().numpy()

    def forward_with_params(self, p0, domain: Domain, sensors, ts, wpt: MSWPT, *, dpdt=None):
        """Sensor data and the beam parameters (p0s, M0s, x0s, omegas, a0s, modes)
        (msgb_solver.py:901-982), mirrored over the two modes and batched as the
        reference does for scan/vmap aggregation (coeff_index.py:29-87)."""
        return self._forward_impl(p0, domain, sensors, ts, wpt, dpdt, want_params=True)

    def _forward_impl(self, p0, domain, sensors, ts, wpt, dpdt, want_params):
        self._check_forward_args(p0, domain, ts, wpt, dpdt)
        self._sensor_positions(sensors)
        sel = self.select(p0, domain, wpt, dpdt)
        if isinstance(sel, BranchSelection):
            bts = [replace(self.beams(sel.pos, domain, wpt), modes=1), replace(self.beams(sel.neg, domain, wpt), modes=2)]
        else:
            bts = [self.beams(sel, domain, wpt)]
        self._traj_owner = sel if (len(bts) == 1 and self.use_real) else None
        try:
            out = self._sum_beam_sets(bts, domain, sensors, ts)
        finally:
            self._traj_owner = None
        self.last_selection = sel
        result = out if _is_torch(p0) else out.cpu().numpy()
        if not want_params:
            return result, None
        return result, self._params_like_reference(bts, domain, as_numpy=not _is_torch(p0))

    def _sum_beam_sets(self, bts, domain: Domain, sensors, ts):
        """Sum over beam sets: the real field sum_b 2 Re(a0 K_b) (scan_real,
        gb/core.py:194-329) or, for the *_complex sum methods, the complex
        field sum_b a0 K_b (gb/core.py:105-168), which is
        0.5 (S(a0) + i S(-i a0)) with S the real summation."""
        total = None
        for bt in bts:
            part = self.sum_forward(bt, domain, sensors, ts)
            if not self.use_real:
                im = self.sum_forward(bt.with_amplitude(-1j), domain, sensors, ts)
                part = 0.5 * (part + 1j * im)
            total = part if total is None else total + part
        return total

    def _params_like_reference(self, bts, domain: Domain, as_numpy: bool):
        import torch

        d = domain.ndim
        if len(bts) == 1:  # real input: the selection mirrored over both modes
            bt = bts[0]
            parts = [(bt, 1.0), (bt, -1.0)]
        else:              # complex input: c_pos beams (+1), then c_neg beams (-1)
            parts = [(bts[0], 1.0), (bts[1], -1.0)]
        dev = bts[0].omega.device
        eye = torch.eye(d, dtype=torch.complex128, device=dev)
        cat = lambda f: torch.cat([f(bt) for bt, _ in parts], 0)
        modes = torch.cat([torch.full((bt.n,), m, dtype=torch.float64, device=dev) for bt, m in parts])
        params = [cat(lambda b: b.p0), cat(lambda b: b.alpha[:, :, None] * eye), cat(lambda b: b.x0),
                  cat(lambda b: b.omega), cat(lambda b: b.a0), modes]
        if self.aggregate_method in ("scan", "vmap"):
            b = params[0].shape[0]
            nb = (b + self.batch_size - 1) // self.batch_size
            pad = nb * self.batch_size - b
            out = []
            for i, t in enumerate(params):
                if pad:
                    filler = torch.zeros((pad,) + t.shape[1:], dtype=t.dtype, device=t.device) if i == 4 \
                        else t[-1:].expand((pad,) + t.shape[1:])
                    t = torch.cat([t, filler], 0)
                out.append(t.reshape((nb, self.batch_size) + t.shape[1:]))
            params = out
        if as_numpy:
            params = [p.cpu().numpy() for p in params]
        return tuple(params)

    def adjoint(self, data, domain: Domain, sensors, *args, **kwargs):
        """Two operators, told apart by their arguments:

        * ``adjoint(data, domain, sensors, ts, wpt, *, p0=None, selection=None)``:
          the exact transpose A^T d of ``forward`` with the beam selection
          frozen (the selection is ``selection`` if given, else the one made
          from ``p0``, else the one of this solver's last ``forward``); returns
          the image (shape domain.N), float64.
        * ``adjoint(data, domain, sensors, sources, ts, data_domain, data_wpt,
          *, window=None)``: the reference's principal-symbol approximation of
          the continuous PAT adjoint (msgb_solver.py:1235-1386), evaluated at
          the sensor positions; not the transpose of the discrete forward.
        """
        if len(args) > 2 or {"sources", "data_domain", "data_wpt", "window"} & set(kwargs):
            return self.adjoint_with_params(data, domain, sensors, *args, **kwargs)[0]
        return self._exact_adjoint(data, domain, sensors, *args, **kwargs)

    def _exact_adjoint(self, data, domain: Domain, sensors, ts, wpt: MSWPT, *, p0=None,
                       selection: Optional[Selection] = None):
        if wpt.dyadic_decomp.N != domain.N:
            raise ValueError("wpt grid shape must match domain.N.")
        _validate_time_grid(ts, allow_singleton=True)
        if selection is None:
            if p0 is not None:
                selection = self.select(p0, domain, wpt)
            elif self.last_selection is not None and self.last_selection.total_coeffs == wpt.total_coeffs:
                selection = self.last_selection
            else:
                raise ValueError("adjoint needs a beam selection: call forward first or pass p0= or selection=")
        complex_data = _is_complex(data)
        if complex_data and self.use_real:
            raise ValueError("complex data needs a *_complex sum_method (the real path's output is real)")
        if isinstance(selection, BranchSelection):
            if self.use_real:
                raise NotImplementedError("the adjoint of the complex-input path with a real sum_method "
                                          "(a map from complex images to real data) is not implemented")
            img = self._adjoint_branches(data, domain, sensors, ts, wpt, selection)
            return img if _is_torch(data) else img.cpu().numpy()
        # Gather in flat-index order: neighbouring coefficients (same box,
        # adjacent packet positions) have overlapping footprints, so the
        # per-beam warps of a CTA reuse the same data tiles from L1.
        cached = self._cached_trajectories(selection, domain, ts) if self._integrates(domain) else None
        if cached is not None:
            sel_sorted = selection  # the order of the kept trajectory records
        else:
            sel_sorted = _sorted_selection(selection)
        bt = self.beams(sel_sorted, domain, wpt)
        if complex_data:
            g = self._gather_complex(bt, domain, sensors, ts, data)
        else:
            g = self.gather_adjoint(bt, domain, sensors, ts, data, cached)
        img = self.coefficient_adjoint(sel_sorted, g, wpt)
        return img if _is_torch(data) else img.cpu().numpy()

    def _gather_complex(self, bt: BeamTensors, domain: Domain, sensors, ts, data):
        """Hermitian gather for complex data: g_j = sum conj(a0u_j K_j) d
        = 0.5 (G(Re d) + i G(Im d)), G the real gather (sum 2 d conj(a0u K))."""
        d = as_device_f64(data, bt.x0.device)
        gr = self.gather_adjoint(bt, domain, sensors, ts, d.real.contiguous())
        gi = self.gather_adjoint(bt, domain, sensors, ts, d.imag.contiguous())
        return 0.5 * (gr + 1j * gi)

    def _adjoint_branches(self, data, domain: Domain, sensors, ts, wpt: MSWPT, selection: BranchSelection):
        """Hermitian adjoint of the complex-input forward (c_pos beams mode +1,
        c_neg beams mode -1, complex sum): both branches' coefficients are
        0.5 MSWPT(p0) (the dpdt term does not depend on p0), so the image is
        MSWPT^H(0.5 (scatter g_pos + scatter g_neg)), complex."""
        import torch

        dev = selection.pos.idx.device
        G = torch.zeros(wpt.total_coeffs, dtype=torch.complex128, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        for sel, modes in ((selection.pos, 1), (selection.neg, 2)):
            s_sorted = _sorted_selection(sel)
            bt = replace(self.beams(s_sorted, domain, wpt), modes=modes)
            g = self._gather_complex(bt, domain, sensors, ts, data)
            _lib.check(_lib.lib().msgb_scatter_coeff_grad(s_sorted.idx.data_ptr(), torch.view_as_real(g).data_ptr(),
                                                          int(s_sorted.idx.shape[0]), 0.5, wpt.plan(dev), 0,
                                                          torch.view_as_real(G).data_ptr(), st),
                       "msgb_scatter_coeff_grad")
        return wpt.adjoint(G, "spatial", real_output=False)

    # ------------------------------------------------------------- time reversal
    def _validate_boundary_data(self, data, data_domain: Domain, sources, *, ts=None) -> None:
        """msgb_solver.py:806-856: the regular axis-aligned detector grid."""
        shape = tuple(data.shape)
        if shape != tuple(data_domain.N):
            raise ValueError(f"Boundary data must have shape {tuple(data_domain.N)}; got {shape}.")
        if ts is not None:
            _validate_time_grid(ts)
            ts_np = np.asarray(ts.detach().cpu().numpy() if hasattr(ts, "detach") else ts, np.float64)
            data_span = (shape[0] - 1) * data_domain.dx[0]
            acquisition_span = float(ts_np[-1] - ts_np[0])
            if not np.isclose(acquisition_span, data_span, rtol=1e-6, atol=1e-12):
                raise ValueError(f"ts spans {acquisition_span}, but data_domain spans {data_span}.")
        if not isinstance(sources, Sensor):
            raise ValueError("sources must be a Sensor on a regular planar grid.")
        positions = np.asarray(sources.positions, np.float64)
        stds = np.std(positions, axis=0)
        normal_axis = int(np.argmin(stds))
        tolerance = 1e-7 * max(1.0, float(np.max(sources.domain.grid_size)))
        if stds[normal_axis] > tolerance:
            raise ValueError("sources must lie on an axis-aligned planar surface.")
        counts = []
        for axis in (a for a in range(positions.shape[1]) if a != normal_axis):
            values = np.unique(positions[:, axis])
            if values.size > 2 and not np.allclose(np.diff(values), np.diff(values)[0], rtol=1e-6, atol=tolerance):
                raise ValueError("sources must be uniformly spaced on the detector plane.")
            counts.append(int(values.size))
        expected = tuple(counts) if counts else (1,)
        actual = tuple(shape[1:]) or (1,)
        if actual != expected:
            raise ValueError("Boundary data detector axes do not match the source grid: "
                             f"got {actual}, expected {expected}.")
        if math.prod(expected) != positions.shape[0]:
            raise ValueError("sources must form a complete Cartesian detector grid.")

    @staticmethod
    def _infer_planar_surface(sensor_positions, eps: float = 1e-9):
        """msgb_solver.py:755-805: the detector plane x_axis = coord of sensor
        positions (the axis of smallest spread, which must be below eps) and
        its implicit function x -> x[axis] - coord."""
        pos = np.asarray(sensor_positions.detach().cpu().numpy() if hasattr(sensor_positions, "detach")
                         else sensor_positions, dtype=np.float64)
        stds = np.std(pos, axis=0)
        axis = int(np.argmin(stds))
        if stds[axis] > eps:
            raise ValueError("Cannot infer planar surface from sensor positions; please provide `surface`.")
        coord = float(pos[0, axis])

        def surface(x):
            return np.asarray(x, dtype=np.float64)[..., axis] - coord

        return surface, axis, coord

    @staticmethod
    def _tr_geometry(sources: Sensor) -> _lib.TrGeometry:
        """The detector plane (tr_solver_utils.py:173-204, 241-251, 377-393):
        the first constant column of the source positions is the normal axis
        (axis 0 at value 0 when none is), and the normal momentum points into
        the domain."""
        pos = np.asarray(sources.positions, np.float64)
        const = np.nonzero(np.all(pos == pos[0], axis=0))[0]
        axis = int(const[0]) if const.size else 0
        value = float(pos[0, axis]) if const.size else 0.0
        dx = np.asarray(sources.domain.dx, np.float64)
        grid_max = float(np.asarray(sources.domain.grid_size, np.float64)[axis] - dx[axis])
        if np.isclose(value, 0.0):
            inward = 1.0
        elif np.isclose(value, grid_max):
            inward = -1.0
        else:
            inward = float(np.sign(grid_max / 2.0 - value)) or 1.0
        return _lib.TrGeometry(normal_axis=axis, normal_value=value, inward=inward)

    def time_reversal(self, data, domain: Domain, sensors, sources, ts, data_domain: Domain, data_wpt: MSWPT):
        """MSGB time-reversal reconstruction at the positions of ``sensors``
        (msgb_solver.py:984-1041), scaled by 2."""
        return self.time_reversal_with_params(data, domain, sensors, sources, ts, data_domain, data_wpt)[0]

    def time_reversal_with_params(self, data, domain: Domain, sensors, sources, ts, data_domain: Domain,
                                  data_wpt: MSWPT):
        """msgb_solver.py:1043-1111 on the GPU: c_pos = 0.5 MSWPT_data(data)
        (no half-frame mask), the solver's threshold, msgb_tr_init (beams on
        the detector at their data time), msgb_tr_final_states (each beam
        back to t = 0, adaptive FP64 with the solver's tolerances), the FP64
        trajectory sum at the sensor positions, times 2.  Returns the image
        (Ns,) and the beam parameters (pts, Mts, xts, omegas, ats, signum, ts)
        with ts (n, 2) = (start, 0) as compute_TR_parameters returns them."""
        if any(domain.periodic):
            raise ValueError("The MSGB time reversal solver only supports free space boundary conditions.")
        pos = self._sensor_positions(sensors)
        self._validate_boundary_data(data, data_domain, sources, ts=ts)
        self._check_tr_axes(domain, sources, data_domain)
        x = as_device_f64(data)
        if x.is_complex():
            raise ValueError("time reversal takes real boundary data")
        coeffs, keys = data_wpt.forward_device(x, self.input_type, scale=0.5, keys=True)
        sel = self._select_from(coeffs, keys, data_wpt, x.device, self._effective_top_n(data_wpt))
        out, params = self._boundary_beams_to_image(sel, domain, pos, sources, data_domain, data_wpt,
                                                    b_inverse=False)
        return self._tr_output(2.0 * out, params, data)

    def adjoint_with_params(self, data, domain: Domain, sensors, sources, ts, data_domain: Domain,
                            data_wpt: MSWPT, *, window=None):
        """The principal-symbol adjoint (msgb_solver.py:1235-1386) on the GPU:
        F = -c_Gamma^2 d_t(window r) (msgb_adjoint_source), raw MSWPT_data(F)
        coefficients, the solver's threshold (uncapped top_n), the time
        reversal beams with amplitudes times -B^{-1} (msgb_tr_init with
        b_inverse, relative guard ``adjoint_relative_guard``), each back to
        t = 0, the FP64 field at the sensor positions divided by c^2 there.
        Returns (q_T (Ns,), beam parameters)."""
        import torch

        if any(domain.periodic):
            raise ValueError("MSGBSolver.adjoint currently assumes non-periodic spatial "
                             "boundaries in the reconstruction domain.")
        try:
            pos = self._sensor_positions(sensors)
        except ValueError:
            raise ValueError("Unsupported sensor type for `sensors` in adjoint().") from None
        self._validate_boundary_data(data, data_domain, sources, ts=ts)
        self._check_tr_axes(domain, sources, data_domain)
        x = as_device_f64(data)
        if x.is_complex():
            raise ValueError("the principal-symbol adjoint takes real boundary data")
        dev = x.device
        nt = int(x.shape[0])
        ns = int(np.prod(x.shape[1:])) if x.dim() > 1 else 1
        src_pos = torch.from_numpy(np.ascontiguousarray(sources.positions, np.float64)).to(dev)
        if src_pos.shape[0] != ns:
            raise ValueError(f"c_at_sources has {src_pos.shape[0]} detector samples, which does not match "
                             f"the data detector grid {tuple(x.shape[1:])}.")
        c_src = self._speed_at(sources.domain, src_pos)
        w = None
        w_time = 0
        if window is not None:
            w = as_device_f64(window, dev)
            if w.dim() == 1 and x.dim() > 1:
                if w.shape[0] != nt:
                    raise ValueError(f"a time window needs {nt} samples; got {w.shape[0]}")
                w_time = 1
            elif tuple(w.shape) != tuple(x.shape):
                raise ValueError(f"window must have shape {tuple(x.shape)} or ({nt},); got {tuple(w.shape)}")
            w = w.contiguous()
        src = torch.empty_like(x)
        nbytes = _lib.lib().msgb_adjoint_source_workspace_size(nt, ns)
        if nbytes == 0:
            raise RuntimeError("msgb_adjoint_source_workspace_size: " + _lib.last_error())
        ws = workspace(dev, "adjsrc", nbytes)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_adjoint_source(x.contiguous().data_ptr(), None if w is None else w.data_ptr(),
                                                  w_time, nt, ns, float(data_domain.dx[0]), c_src.data_ptr(),
                                                  src.data_ptr(), ws.data_ptr(), nbytes, st), "msgb_adjoint_source")
        coeffs, keys = data_wpt.forward_device(src, self.input_type, scale=1.0, keys=True)
        sel = self._select_from(coeffs, keys, data_wpt, dev, self._effective_top_n(data_wpt))
        out, params = self._boundary_beams_to_image(sel, domain, pos, sources, data_domain, data_wpt,
                                                    b_inverse=True)
        img_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).to(dev)
        c_img = self._speed_at(domain, img_pos)
        return self._tr_output(out / (c_img * c_img), params, data)

    @staticmethod
    def _check_tr_axes(domain: Domain, sources, data_domain: Domain):
        if data_domain.ndim != domain.ndim or sources.domain.ndim != domain.ndim:
            raise ValueError("data_domain, sources and domain must have the same number of axes")

    def _speed_at(self, domain: Domain, points):
        """c(x) of ``domain`` at device points (n, d) (msgb_medium_speed)."""
        import torch

        med, keep = self._medium(domain, points.device)
        c = torch.empty(points.shape[0], dtype=torch.float64, device=points.device)
        st = torch.cuda.current_stream(points.device).cuda_stream
        _lib.check(_lib.lib().msgb_medium_speed(domain.ndim, _lib.ref(med), points.data_ptr(), int(points.shape[0]),
                                                c.data_ptr(), st), "msgb_medium_speed")
        del keep
        return c

    @staticmethod
    def _tr_output(img, params, data):
        if not _is_torch(data):
            img = img.cpu().numpy()
            params = tuple(p.cpu().numpy() for p in params)
        return img, params

    def _boundary_beams_to_image(self, sel: Selection, domain: Domain, pos, sources, data_domain: Domain,
                                 data_wpt: MSWPT, b_inverse: bool):
        """Beams from boundary-data coefficients (msgb_tr_init), each from its
        data time back to t = 0 (msgb_tr_final_states), the FP64 real field
        at ``pos`` (msgb_sum_fwd_f64_traj with nt = 1): compute_TR_result
        (tr_solver_utils.py:677-750).  Returns the field (Ns,) and the
        parameters (pts, Mts, xts, omegas, ats (n, 1), signum (n, 1), ts (n, 2))."""
        import torch

        dev = sel.idx.device
        d = domain.ndim
        n = int(sel.idx.shape[0])
        self.last_boundary_selection = sel
        xs = torch.empty((n, d), dtype=torch.float64, device=dev)
        ps = torch.empty((n, d), dtype=torch.float64, device=dev)
        Ms = torch.empty((n, d, d), dtype=torch.complex128, device=dev)
        a = torch.empty(n, dtype=torch.complex128, device=dev)
        om = torch.empty(n, dtype=torch.float64, device=dev)
        mode = torch.empty(n, dtype=torch.float64, device=dev)
        t0 = torch.empty(n, dtype=torch.float64, device=dev)
        tb = _lib.TrBeams(n=n, x=xs.data_ptr(), p=ps.data_ptr(), M=torch.view_as_real(Ms).data_ptr(),
                          a=torch.view_as_real(a).data_ptr(), omega=om.data_ptr(), mode=mode.data_ptr(),
                          t0=t0.data_ptr())
        geo = self._tr_geometry(sources)
        src_med, keep_s = self._medium(sources.domain, dev)
        Ld = (ctypes.c_double * 3)(*[float(v) for v in data_domain.grid_size], *([1.0] * (3 - d)))
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().msgb_tr_init(data_wpt.plan(dev), Ld, _lib.ref(geo), _lib.ref(src_med),
                                           sel.idx.data_ptr(), torch.view_as_real(sel.values).data_ptr(), n,
                                           int(b_inverse), float(self.adjoint_relative_guard), _lib.ref(tb), st),
                   "msgb_tr_init")
        med, keep_m = self._medium(domain, dev)
        cfg = self.ode_config
        opts = _lib.OdeOpts(method=1, substeps=1, rtol=float(cfg.rtol), atol=float(cfg.atol),
                            dt0=float(cfg.dt0) if cfg.dt0 is not None else 0.0, max_steps=int(cfg.max_steps),
                            dense_output=int(bool(cfg.dense_output)))
        sens = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).to(dev)
        t_img = torch.zeros(1, dtype=torch.float64, device=dev)
        pr = _lib.Problem()
        pr.ndim = d
        L = np.asarray(domain.grid_size, np.float64)
        for ax in range(3):
            pr.periodic[ax] = 0
            pr.L[ax] = float(L[ax]) if ax < d else 1.0
        pr.c = 1.0
        pr.nt = 1
        pr.ts = t_img.data_ptr()
        pr.ns = pos.shape[0]
        pr.sensors = sens.data_ptr()
        nr = 2 * d + 2 * d * d + 2
        rec = torch.empty((n, nr), dtype=torch.float64, device=dev)
        status = torch.zeros(n, dtype=torch.int32, device=dev)
        out = torch.zeros((1, pos.shape[0]), dtype=torch.float64, device=dev)
        if n:
            with self._kernel_span("msgb_tr_final_states", None):
                _lib.check(_lib.lib().msgb_tr_final_states(_lib.ref(pr), _lib.ref(med), _lib.ref(tb), _lib.ref(opts),
                                                           rec.data_ptr(), status.data_ptr(), st),
                           "msgb_tr_final_states")
            worst = int(status.max().item())
            if worst:
                what = "reached max_steps" if worst == 2 else "produced a non-finite state"
                raise RuntimeError(f"time-reversal ODE integration {what} for "
                                   f"{int((status == worst).sum().item())} beam(s)")
            bs = _lib.BeamSet(n=n, x0=xs.data_ptr(), p0=ps.data_ptr(), alpha=torch.view_as_real(Ms).data_ptr(),
                              a0=torch.view_as_real(a).data_ptr(), omega=om.data_ptr(), modes=0)
            tr = _lib.Trajectories(nb=n, b_first=0, rec64=rec.data_ptr(), rec32=None, cull=None, status=None)
            _lib.check(_lib.lib().msgb_sum_fwd_f64_traj(_lib.ref(pr), _lib.ref(bs), _lib.ref(tr), out.data_ptr(), st),
                       "msgb_sum_fwd_f64_traj")
        del keep_s, keep_m
        ts_pair = torch.stack([t0, torch.zeros_like(t0)], dim=1)
        return out[0], (ps, Ms, xs, om, a[:, None], mode[:, None], ts_pair)

    def eval_count(self) -> Optional[int]:
        """Evaluated (beam, time, sensor) triples of the last FP32 call."""
        c = getattr(self, "_eval_counter", None)
        return None if c is None else int(c.item())


def _chain(*its):
    for it in its:
        yield from it


def torch_argsort(x):
    import torch

    return torch.argsort(x)


def _sorted_selection(sel: Selection) -> Selection:
    """The selection in ascending flat-index order, sorted once per
    selection object (a frozen selection reused by many adjoints, as in a
    reconstruction loop, is not sorted again)."""
    cached = getattr(sel, "_sorted", None)
    if cached is None or cached[0] is not sel.idx:
        order = torch_argsort(sel.idx)
        cached = (sel.idx, Selection(sel.idx[order], sel.values[order], sel.total_coeffs))
        sel._sorted = cached
    return cached[1]


def _is_torch(x) -> bool:
    return hasattr(x, "detach") and hasattr(x, "device")


def _is_complex(x) -> bool:
    return x.is_complex() if _is_torch(x) else np.iscomplexobj(x)
