"""FP64 restatement of MSGB time reversal and of the principal-symbol
adjoint (test oracle).

Test infrastructure: only ``tests/`` uses this module, as the checker.

Follows MSGBSolver.time_reversal (solvers/msgb_solvers/msgb_solver.py:
984-1111): boundary data -> c_pos = 0.5 MSWPT_data(data) (compute_coefficients
mode "both", forward_solver_utils.py:716-786) -> uncapped threshold ->
compute_TR_parameters (tr_solver_utils.py:205-440: beams launched from the
detector plane at their data time, spatial Hessian from mT_inverse :116-170,
grazing beams zeroed) -> each beam integrated from its start time back to
t = 0 (solve_ODE_batch_t, diffrax; here SciPy DOP853 at a tight tolerance,
backward in time) -> real field at the image points (gb/core.py:332-425)
summed and doubled.
"""

from __future__ import annotations

import numpy as np
from scipy.integrate import solve_ivp

from . import msgb as om
from . import ode as oo


def find_constant_columns(arr, max_constant_axes=None):
    """tr_solver_utils.py:173-204."""
    arr = np.asarray(arr)
    d = arr.shape[1]
    if max_constant_axes is None:
        max_constant_axes = d
    mask = np.all(arr == arr[0], axis=0)
    axes = np.nonzero(mask)[0][:max_constant_axes]
    axes = np.concatenate([axes, -np.ones(max_constant_axes - axes.size, dtype=int)])
    vals = np.where(axes >= 0, arr[0][np.maximum(axes, 0)], 0.0)
    return mask, vals, axes


def gp_gx(x, p, mode, speed):
    """G_p and G_x of G = mode c(x) |p| (gb_utils.py:48-102)."""
    c, g, _ = speed.eval(x)
    n = np.linalg.norm(p)
    return mode * c * p / n, mode * g * n


def mT_inverse(xT, pT, mT_spc_time, mode, speed):
    """tr_solver_utils.py:116-170 for one beam: spacetime Hessian -> spatial."""
    gp, gx = gp_gx(xT, pT, mode, speed)
    xdot, pdot = gp, -gx
    d = xT.size
    A = mT_spc_time[0, 0]
    B = mT_spc_time[0, 1:]
    C = mT_spc_time[1:, 1:]
    xs, ps = xdot[1:], pdot[1:]
    if xdot[0] == 0.0:
        # grazing beam (no velocity across the detector plane): the spatial
        # Hessian is undefined; the caller replaces it with the reference's
        # safe value i I (tr_solver_utils.py:424-435), as for p_n = 0
        return 1j * np.eye(d)
    upper_right = (ps - C @ xs - B) / xdot[0]
    num = A + pdot[0] * xdot[0] - ps @ xs + xs @ C @ xs + 2 * (B @ xs)
    M = np.zeros((d, d), complex)
    M[0, 0] = num / xdot[0] ** 2
    M[0, 1:] = upper_right
    M[1:, 0] = upper_right
    M[1:, 1:] = C
    return M


class Sources:
    """The detector: positions (Ns, d) and the spatial domain's dx and size."""

    def __init__(self, positions, dx, grid_size):
        self.positions = np.asarray(positions, float)
        self.dx = np.asarray(dx, float)
        self.grid_size = np.asarray(grid_size, float)


def tr_parameters(idx, data_dom: om.Dom, data_wpt: om.Wpt, sources: Sources, speed):
    """compute_TR_parameters (tr_solver_utils.py:205-440) for flat indices idx."""
    _, const_vals, const_axes = find_constant_columns(sources.positions, 1)
    normal_axis = int(const_axes[0]) if const_axes[0] >= 0 else 0
    normal_value = float(const_vals[0]) if const_axes[0] >= 0 else 0.0
    d = sources.positions.shape[1]
    dec = data_wpt.dyadic_decomp
    red = data_wpt.redundancy
    L = np.asarray(data_dom.grid_size, float)
    Nd = np.asarray(data_dom.N)
    lvl, mi = om.find_tensor_and_multiindex(np.asarray(idx), om.coeff_shapes(data_wpt))
    box = mi[0] + np.r_[0, np.cumsum(dec.num_boxes_ndim)][lvl]
    ch = dec.centres_ndim[box] / L
    tau = ch[:, 0]
    k_tan = ch[:, 1:]
    bl = np.asarray(dec.box_lengths)[lvl][:, None] / L * np.asarray(dec.box_aspect_ratio)
    Lls = bl * red
    sig = bl / 2.0
    signum = -np.sign(tau)
    omega = np.maximum(np.abs(tau), 1e-6)
    t0 = mi[1] / Lls[:, 0]
    xstar = (mi[2:].T / Lls[:, 1:]) if d > 1 else np.zeros((idx.size, 0))
    tan_axes = [a for a in range(d) if a != normal_axis]
    B = np.asarray(idx).size
    xts = np.zeros((B, d))
    xts[:, normal_axis] = normal_value
    for j, a in enumerate(tan_axes):
        xts[:, a] = xstar[:, j]
    cxt = np.array([speed.eval(x)[0] for x in xts])
    if d == 1:
        ch_n = ch / np.linalg.norm(ch, axis=1, keepdims=True)
        radic = np.maximum((ch_n[:, 0] / cxt) ** 2 - np.sum(ch_n[:, 1:] ** 2, axis=1), 0.0)
        p_tan = np.zeros((B, 0))
    else:
        tau_abs = np.maximum(np.abs(tau), 1e-6)
        p_tan = cxt[:, None] * k_tan / tau_abs[:, None]
        radic = np.maximum(1.0 - np.sum(p_tan ** 2, axis=1), 0.0)
    p_n = np.sqrt(radic)
    grid_max = sources.grid_size[normal_axis] - sources.dx[normal_axis]
    if np.isclose(normal_value, 0.0):
        inward = 1.0
    elif np.isclose(normal_value, grid_max):
        inward = -1.0
    else:
        inward = np.sign(grid_max / 2.0 - normal_value) or 1.0
    p_n = inward * p_n
    pu = np.zeros((B, d))
    pu[:, normal_axis] = p_n
    for j, a in enumerate(tan_axes):
        pu[:, a] = p_tan[:, j]
    pts = 2.0 * np.pi * pu
    if d != 1:
        pts = pts / cxt[:, None]
    alpha = 2j * (np.pi * sig) ** 2 / omega[:, None]
    Mts = np.stack([mT_inverse(xts[b], pts[b], np.diag(alpha[b]), signum[b], speed) for b in range(B)])
    ats = np.prod(np.sqrt((np.pi * L[None]) / (Lls * Nd[None])) * sig, axis=1)
    local_k = mi[1:].T
    ats = ats * om.compute_frame_phase(dec, box, local_k, red)
    graz = np.abs(pts[:, normal_axis]) == 0.0
    pts[graz] = 1.0
    ats[graz] = 0.0
    Mts[graz] = 1j * np.eye(d)
    return pts, Mts, xts, omega, ats, signum, t0


def time_reversal(data, data_dom: om.Dom, data_wpt: om.Wpt, sources: Sources, speed, image_points, domain_size,
                  thr, periodic=None, rtol=1e-12, atol=1e-12, lam=0.0):
    """The reconstruction at image_points (n, d) from boundary data; speed is
    the medium (oracle.ode.GridSpeed or LinearSpeed), lam the absorption."""
    d = sources.positions.shape[1]
    c_pos = om.compute_coefficients(np.asarray(data, float), np.zeros_like(data), "spatial", data_dom, data_wpt,
                                    mode="both")[0]
    idx, vals = om.threshold_top_n(c_pos, om.effective_top_n(thr, data_wpt, half_frame=False))
    pts, Mts, xts, omega, ats, signum, t0 = tr_parameters(idx, data_dom, data_wpt, sources, speed)
    ats = ats * vals
    periodic = np.zeros(d, bool) if periodic is None else np.asarray(periodic)
    out = np.zeros(len(image_points))
    for b in range(idx.size):
        if ats[b] == 0:
            continue
        y0 = oo._pack_state(xts[b], pts[b], Mts[b], ats[b])
        if t0[b] > 0:
            sol = solve_ivp(lambda t, y: oo.rhs(t, y, signum[b], speed, d, lam), (t0[b], 0.0), y0, method="DOP853",
                            rtol=rtol, atol=atol, t_eval=[0.0])
            y = sol.y[:, -1]
        else:
            y = y0
        xt, pt, Mt, At = oo._unpack_states(y[None], d)
        out += om.gaussian_beam_real_sum(xt[None], pt[None], Mt[None], At[None, :, None], np.array([omega[b]]),
                                         np.asarray(image_points, float), domain_size, periodic)[0]
    return 2.0 * out, (idx, vals, pts, Mts, xts, omega, ats, signum, t0)


# ---- principal-symbol adjoint (msgb_solver.py:68-127, 1168-1386;
# ---- adjoint_solver_utils.py:17-200) ---------------------------------------


def form_adjoint_source(data, dt, c_at_sources, window=None):
    """_form_adjoint_source (msgb_solver.py:68-120): -c^2 d_t(window r), the
    time derivative on the sampled Fourier grid (real part)."""
    data = np.asarray(data, float)
    w = data if window is None else (np.asarray(window, float).reshape((-1,) + (1,) * (data.ndim - 1))
                                     if np.ndim(window) == 1 and data.ndim > 1 else np.asarray(window, float)) * data
    f = np.fft.fftfreq(w.shape[0], d=dt).reshape((-1,) + (1,) * (w.ndim - 1))
    der = np.fft.ifft(2j * np.pi * f * np.fft.fft(w, axis=0), axis=0).real
    c = np.asarray(c_at_sources, float)
    det = der.shape[1:]
    if c.ndim == 1 and c.shape != det:
        if c.size != int(np.prod(det)):
            raise ValueError(f"c_at_sources has {c.size} detector samples, which does not match the data "
                             f"detector grid {det}.")
        c = c.reshape(det)
    return -(c ** 2) * der


def principal_b_inverse(tau, k_tan, c, relative_guard=1e-6):
    """adjoint_solver_utils.py:17-75: -i sign(W) / (2 c sqrt(W^2 - c^2 |Q|^2)),
    W = 2 pi tau, Q = 2 pi k_tan; zero when evanescent or within the guard."""
    tau = np.asarray(tau, float)
    k_tan = np.asarray(k_tan, float).reshape(tau.size, -1)
    c = np.asarray(c, float)
    w = 2.0 * np.pi * tau
    q2 = np.sum((2.0 * np.pi * k_tan) ** 2, axis=1)
    rad = w ** 2 - c ** 2 * q2
    g = np.sqrt(np.maximum(rad, 0.0))
    valid = (rad > 0.0) & (np.abs(w) > 0.0) & (g > relative_guard * np.abs(w))
    out = np.zeros(tau.size, complex)
    out[valid] = -1j * np.sign(w[valid]) / (2.0 * c[valid] * g[valid])
    return out


def adj_parameters(idx, data_dom: om.Dom, data_wpt: om.Wpt, sources: Sources, speed, relative_guard=5e-2):
    """compute_adj_parameters (adjoint_solver_utils.py:78-200)."""
    pts, Mts, xts, omega, ats, signum, t0 = tr_parameters(idx, data_dom, data_wpt, sources, speed)
    dec = data_wpt.dyadic_decomp
    lvl, mi = om.find_tensor_and_multiindex(np.asarray(idx), om.coeff_shapes(data_wpt))
    box = mi[0] + np.r_[0, np.cumsum(dec.num_boxes_ndim)][lvl]
    ch = dec.centres_ndim[box] / np.asarray(data_dom.grid_size, float)
    c = np.array([speed.eval(x)[0] for x in xts])
    binv = -principal_b_inverse(ch[:, 0], ch[:, 1:], c, relative_guard)
    ex = binv == 0.0
    pts = pts.copy()
    Mts = Mts.copy()
    pts[ex] = 1.0
    Mts[ex] = 1j * np.eye(xts.shape[1])
    return pts, Mts, xts, omega, ats * binv, signum, t0


def principal_adjoint(data, dt, data_dom: om.Dom, data_wpt: om.Wpt, sources: Sources, source_speed, speed,
                      image_points, domain_size, thr, window=None, relative_guard=5e-2, rtol=1e-12, atol=1e-12,
                      lam=0.0):
    """MSGBSolver.adjoint, seven-argument form (msgb_solver.py:1235-1386):
    source -> raw MSWPT coefficients -> top_n (uncapped) -> adjoint beams ->
    each back to t = 0 -> real field at the image points, divided by c^2."""
    d = sources.positions.shape[1]
    c_src = np.array([source_speed.eval(x)[0] for x in sources.positions])
    src = form_adjoint_source(data, dt, c_src, window)
    coeffs = data_wpt.forward(src, "spatial")
    idx, vals = om.threshold_top_n(coeffs, om.effective_top_n(thr, data_wpt, half_frame=False))
    pts, Mts, xts, omega, ats, signum, t0 = adj_parameters(idx, data_dom, data_wpt, sources, source_speed,
                                                           relative_guard)
    ats = ats * vals
    out = np.zeros(len(image_points))
    for b in range(idx.size):
        if ats[b] == 0:
            continue
        y0 = oo._pack_state(xts[b], pts[b], Mts[b], ats[b])
        if t0[b] > 0:
            sol = solve_ivp(lambda t, y: oo.rhs(t, y, signum[b], speed, d, lam), (t0[b], 0.0), y0, method="DOP853",
                            rtol=rtol, atol=atol, t_eval=[0.0])
            y = sol.y[:, -1]
        else:
            y = y0
        xt, pt, Mt, At = oo._unpack_states(y[None], d)
        out += om.gaussian_beam_real_sum(xt[None], pt[None], Mt[None], At[None, :, None], np.array([omega[b]]),
                                         np.asarray(image_points, float), domain_size,
                                         np.zeros(d, bool))[0]
    c_img = np.array([speed.eval(x)[0] for x in np.asarray(image_points, float)])
    return out / c_img ** 2, (idx, vals, pts, Mts, xts, omega, ats, signum, t0)
