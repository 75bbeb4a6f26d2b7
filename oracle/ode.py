"""FP64 restatement of the heterogeneous beam ODE (test oracle).

Test infrastructure: only ``tests/``, ``__graft_entry__.smoke`` and
``bench.py``'s CPU legs use this module, as the checker.

* ``GridSpeed`` restates ``make_c_function_from_grid`` (utils/interp.py:
  31-263): linear or cubic B-spline tensor-product interpolation with SciPy's
  ``spline_filter`` prefilter and the reference's boundary maps.  Gradient and
  Hessian are the exact derivatives of that formula (what ``jax.grad`` /
  ``jax.hessian`` of the same code return).
* ``rhs`` restates ``coupled_rhs_absorption`` (gb/gb_solvers.py:787-867).
* ``solve`` integrates it with SciPy DOP853 at a tight tolerance, the reference
  test's own oracle (tests/test_gb.py:759-849), in place of diffrax Tsit5
  (diffrax 0.7.2, gb_solvers.py:706-784), which is not installed here.
"""

from __future__ import annotations

import numpy as np
from scipy import ndimage
from scipy.integrate import solve_ivp

_BOUNDARY = {"clamp": "nearest", "nearest": "nearest", "edge": "nearest", "reflect": "reflect",
             "mirror": "mirror", "wrap": "wrap", "periodic": "wrap"}


def map_indices(idx, n, boundary):
    """utils/interp.py:78-98."""
    if n == 1:
        return np.zeros_like(idx)
    if boundary == "nearest":
        return np.clip(idx, 0, n - 1)
    if boundary == "wrap":
        return np.mod(idx, n)
    if boundary == "reflect":
        r = np.mod(idx, 2 * n)
        return np.where(r < n, r, 2 * n - 1 - r)
    if boundary == "mirror":
        period = 2 * n - 2
        r = np.mod(idx, period)
        return np.where(r < n, r, period - r)
    raise ValueError(boundary)


def _weights(method, t):
    """Weights and their first/second derivatives (utils/interp.py:101-118)."""
    if method == "linear":
        w = np.stack([1.0 - t, t], -1)
        d1 = np.stack([-np.ones_like(t), np.ones_like(t)], -1)
        d2 = np.zeros_like(w)
        return w, d1, d2, (0, 1)
    omt = 1.0 - t
    t2, t3 = t * t, t * t * t
    w = np.stack([omt ** 3 / 6.0, (3 * t3 - 6 * t2 + 4) / 6.0, (-3 * t3 + 3 * t2 + 3 * t + 1) / 6.0, t3 / 6.0], -1)
    d1 = np.stack([-(omt ** 2) / 2.0, 1.5 * t2 - 2 * t, -1.5 * t2 + t + 0.5, t2 / 2.0], -1)
    d2 = np.stack([omt, 3 * t - 2, -3 * t + 1, t], -1)
    return w, d1, d2, (-1, 0, 1, 2)


class GridSpeed:
    """Sound speed interpolated from a grid, with gradient and Hessian."""

    def __init__(self, c_map, spacing, origin=None, method="linear", boundary="clamp"):
        self.values = np.asarray(c_map, dtype=np.float64)
        d = self.values.ndim
        self.spacing = np.asarray(spacing, float)
        self.origin = np.zeros(d) if origin is None else np.asarray(origin, float)
        self.method = method
        self.boundary = _BOUNDARY[boundary]
        if method == "bspline3":
            self.coeffs = ndimage.spline_filter(self.values, order=3, mode=self.boundary)
        elif method == "linear":
            self.coeffs = self.values
        else:
            raise ValueError("method must be 'linear' or 'bspline3'.")

    def eval(self, x):
        """(c, grad c, hessian c) at one point x (d,)."""
        d = self.coeffs.ndim
        u = (np.asarray(x, float) - self.origin) / self.spacing
        i0 = np.floor(u)
        t = u - i0
        w, d1, d2, offs = _weights(self.method, t)
        n = len(offs)
        c = 0.0
        g = np.zeros(d)
        H = np.zeros((d, d))
        for corner in range(n ** d):
            rem = corner
            idx = []
            loc = []
            for ax in range(d):
                k = rem % n
                rem //= n
                loc.append(k)
                idx.append(int(map_indices(np.array(int(i0[ax]) + offs[k]), self.coeffs.shape[ax], self.boundary)))
            v = self.coeffs[tuple(idx)]
            wv = np.prod([w[ax, loc[ax]] for ax in range(d)])
            c += wv * v
            for a in range(d):
                ga = d1[a, loc[a]] * np.prod([w[ax, loc[ax]] for ax in range(d) if ax != a])
                g[a] += ga * v / self.spacing[a]
                for b in range(d):
                    if a == b:
                        hab = d2[a, loc[a]] * np.prod([w[ax, loc[ax]] for ax in range(d) if ax != a])
                    else:
                        hab = d1[a, loc[a]] * d1[b, loc[b]] * np.prod(
                            [w[ax, loc[ax]] for ax in range(d) if ax not in (a, b)])
                    H[a, b] += hab * v / (self.spacing[a] * self.spacing[b])
        return c, g, H

    def __call__(self, x):
        x = np.asarray(x, float)
        flat = x.reshape(-1, x.shape[-1])
        return np.asarray([self.eval(p)[0] for p in flat]).reshape(x.shape[:-1])


class LinearSpeed:
    """c(x) = a + b . x (the reference's analytic test media)."""

    def __init__(self, a, b):
        self.a = float(a)
        self.b = np.asarray(b, float)

    def eval(self, x):
        d = self.b.size
        return self.a + self.b @ np.asarray(x, float), self.b.copy(), np.zeros((d, d))


def rhs(t, y, mode, speed, d, lam=0.0):
    """coupled_rhs_absorption (gb/gb_solvers.py:820-867) on a real-packed state
    y = [x (d), p (d), Re M (d^2), Im M (d^2), Re A, Im A]."""
    x = y[:d]
    p = y[d:2 * d]
    M = (y[2 * d:2 * d + d * d] + 1j * y[2 * d + d * d:2 * d + 2 * d * d]).reshape(d, d)
    A = y[-2] + 1j * y[-1]
    c, gc, hc = speed.eval(x)
    npn = np.linalg.norm(p)
    G = mode * c * npn
    Gx = mode * gc * npn
    Gp = mode * c * p / npn
    Gpp = mode * c * (np.eye(d) / npn - np.outer(p, p) / npn ** 3)
    Gxp = mode * np.outer(gc, p) / npn
    Gxx = mode * hc * npn
    dM = -(Gxx + Gxp @ M + M @ Gxp.T + M @ Gpp @ M)
    dA = -A * (c ** 2 * np.trace(M) - Gx @ Gp - Gp @ M @ Gp + lam * G) / (2 * G)
    return np.concatenate([Gp, -Gx, dM.real.ravel(), dM.imag.ravel(), [dA.real, dA.imag]])


def solve(x0, p0, M0, a0, mode, ts, speed, lam=0.0, rtol=1e-12, atol=1e-12):
    """One beam with DOP853; returns xt (Nt, d), pt, Mt (Nt, d, d), At (Nt,)."""
    d = len(x0)
    M0 = np.asarray(M0, complex)
    y0 = np.concatenate([x0, p0, M0.real.ravel(), M0.imag.ravel(), [np.real(a0), np.imag(a0)]])
    ts = np.asarray(ts, float)
    sol = solve_ivp(lambda t, y: rhs(t, y, mode, speed, d, lam), (ts[0], ts[-1]), y0, method="DOP853",
                    rtol=rtol, atol=atol, t_eval=ts)
    if not sol.success:
        raise RuntimeError(sol.message)
    Y = sol.y.T
    xt = Y[:, :d]
    pt = Y[:, d:2 * d]
    Mt = (Y[:, 2 * d:2 * d + d * d] + 1j * Y[:, 2 * d + d * d:2 * d + 2 * d * d]).reshape(-1, d, d)
    At = Y[:, -2] + 1j * Y[:, -1]
    return xt, pt, Mt, At


def analytic_1d_linear(x0, p0, M0, A0, ts, a, b):
    """tests/test_gb.py:630-667: closed forms for c = a + b x, mode +1, p > 0."""
    dt = np.asarray(ts) - ts[0]
    return ((x0 + a / b) * np.exp(b * dt) - a / b, p0 * np.exp(-b * dt), M0 * np.exp(-2 * b * dt),
            A0 * np.exp(0.5 * b * dt))


def beam_field(xt, pt, Mt, At, omega, sensors, domain_size, periodic):
    """Real field of one beam from its trajectory (gb/core.py:267-303), (Nt, Ns)."""
    from .msgb import gaussian_beam_real_sum

    return gaussian_beam_real_sum(xt[None], pt[None], Mt[None], At[None, :, None], np.array([omega]),
                                  np.asarray(sensors), domain_size, periodic)


def _unpack_states(Y, d):
    Y = np.asarray(Y)
    xt = Y[:, :d]
    pt = Y[:, d:2 * d]
    Mt = (Y[:, 2 * d:2 * d + d * d] + 1j * Y[:, 2 * d + d * d:2 * d + 2 * d * d]).reshape(-1, d, d)
    At = Y[:, -2] + 1j * Y[:, -1]
    return xt, pt, Mt, At


def _pack_state(x0, p0, M0, a0):
    M0 = np.asarray(M0, complex)
    return np.concatenate([x0, p0, M0.real.ravel(), M0.imag.ravel(), [np.real(a0), np.imag(a0)]]).astype(float)


def rk4(x0, p0, M0, a0, mode, ts, speed, substeps=1, lam=0.0):
    """Fixed-step RK4 of ``rhs``, ``substeps`` equal steps per interval [ts[k-1], ts[k]].

    The same method as the GPU integrator's fixed-step option; used to separate
    the method's own error (a cubic B-spline medium is only C^2, so RK4 loses
    order where hess c has kinks) from implementation differences.
    """
    d = len(x0)
    y = _pack_state(x0, p0, M0, a0)
    ts = np.asarray(ts, float)
    f = lambda v: rhs(0.0, v, mode, speed, d, lam)
    out = [y.copy()]
    for k in range(1, ts.size):
        h = (ts[k] - ts[k - 1]) / substeps
        for _ in range(substeps):
            k1 = f(y)
            k2 = f(y + 0.5 * h * k1)
            k3 = f(y + 0.5 * h * k2)
            k4 = f(y + h * k3)
            y = y + h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
        out.append(y.copy())
    return _unpack_states(out, d)


# Dormand & Prince (1980) 5(4) pair: nodes, stage matrix, 5th-order weights
# (= the last stage row, first-same-as-last) and the 4th-order embedded weights.
DP_C = (0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0)
DP_A = ((),
        (1 / 5,),
        (3 / 40, 9 / 40),
        (44 / 45, -56 / 15, 32 / 9),
        (19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729),
        (9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656),
        (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84))
DP_B = (35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0)
DP_BHAT = (5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40)
DP_E = tuple(b - bh for b, bh in zip(DP_B, DP_BHAT))
# Continuous-extension weights (Shampine 1986; Hairer, Norsett & Wanner's dopri5).
DP_D = (-12715105075 / 11282082432, 0.0, 87487479700 / 32700410799, -10690763975 / 1880347072,
        701980252875 / 199316789632, -1453857185 / 822651844, 69997945 / 29380423)


def error_norm(e, y0, y1, d, rtol, atol):
    """RMS over the complex state entries (x, p, M, A) of |e| / (atol + rtol max(|y0|, |y1|)),
    the norm diffrax's PIDController applies (optimistix.rms_norm)."""
    def mags(v):
        x = np.abs(v[:2 * d])
        M = np.hypot(v[2 * d:2 * d + d * d], v[2 * d + d * d:2 * d + 2 * d * d])
        A = np.hypot(v[-2], v[-1])
        return np.concatenate([x, M, [A]])
    r = mags(e) / (atol + rtol * np.maximum(mags(y0), mags(y1)))
    return float(np.sqrt(np.mean(r * r)))


def dense_state(y, y5, ks, h, theta):
    """Dormand-Prince continuous extension (Shampine's 4th-order interpolant,
    the form of Hairer, Norsett & Wanner's dopri5 contd5) at t + theta h."""
    r2 = y5 - y
    r3 = h * ks[0] - r2
    r4 = r2 - h * ks[6] - r3
    r5 = h * sum(c * kk for c, kk in zip(DP_D, ks) if c != 0.0)
    return y + theta * (r2 + (1.0 - theta) * (r3 + theta * (r4 + (1.0 - theta) * r5)))


def dopri5(x0, p0, M0, a0, mode, ts, speed, lam=0.0, rtol=1e-7, atol=1e-9, max_steps=4096, dt0=None,
           dense=False):
    """Adaptive Dormand-Prince 5(4) of ``rhs`` with the state saved at every ts.

    Step control (the GPU integrator's, step for step): error norm as
    ``error_norm``; accept when it is <= 1; next step h * clip(0.9 err^(-1/5),
    0.2, 10) (at most 1 after a rejection, and for the step that follows an
    accepted step that came right after a rejection).  Save times: by default
    a step that would pass the next save time is shortened to end on it (the
    proposal it replaced is kept for the next step); with ``dense`` steps
    follow the error control alone (the last one shortened to end at ts[-1])
    and save times inside a step are read from the continuous extension
    (``dense_state``), as diffrax's SaveAt(ts) reads its solver's interpolant.
    ``max_steps`` counts accepted and rejected steps over the whole solve, as
    diffrax does (plus nt - 1 when steps end on the save times, the steps a
    solver reading its interpolant would not take) (gb/gb_solvers.py:756-783 builds that solve: Tsit5,
    PIDController(rtol, atol), SaveAt(ts), dt0 = ts[1] - ts[0]).
    Returns (xt, pt, Mt, At, status, steps); status 0 ok, 1 non-finite,
    2 max_steps reached (later save times then hold the last state).
    """
    d = len(x0)
    y = _pack_state(x0, p0, M0, a0)
    ts = np.asarray(ts, float)
    nt = ts.size
    f = lambda v: rhs(0.0, v, mode, speed, d, lam)
    h = float(dt0) if dt0 is not None else (ts[1] - ts[0] if nt > 1 else 0.0)
    out = [y.copy()]
    steps, status = 0, 0
    k1 = f(y)
    t = ts[0]
    k = 1
    rejected = False
    budget = max_steps + (0 if dense else nt - 1)  # landings on save times do not count
    while k < nt and status == 0:
        if steps >= budget:
            status = 2
            break
        target = ts[-1] if dense else ts[k]
        hh, last = h, False
        if t + hh >= target:
            hh, last = target - t, True
        ks = [k1]
        for s in range(1, 7):
            acc = np.zeros_like(y)
            for j, a in enumerate(DP_A[s]):
                if a != 0.0:
                    acc = acc + a * ks[j]
            ks.append(f(y + hh * acc))
        y5 = y + hh * sum(b * kk for b, kk in zip(DP_B, ks) if b != 0.0)
        # stage 7 is evaluated at y + hh * sum(a7j k_j), which is y5 up to rounding
        e = hh * sum(c * kk for c, kk in zip(DP_E, ks))
        err = error_norm(e, y, y5, d, rtol, atol)
        steps += 1
        if not np.isfinite(err):
            h = 0.2 * hh
            rejected = True
            continue
        fac = 10.0 if err == 0.0 else min(10.0, max(0.2, 0.9 * err ** -0.2))
        if err <= 1.0:
            if rejected:
                fac = min(fac, 1.0)
            rejected = False
            t_new = target if last else t + hh
            while k < nt and ts[k] <= t_new:
                out.append(y5.copy() if ts[k] == t_new else dense_state(y, y5, ks, hh, (ts[k] - t) / hh))
                k += 1
            t = t_new
            y = y5
            k1 = ks[6]
            h = max(hh * fac, h) if (last and not dense) else hh * fac
            if not np.all(np.isfinite(y)):
                status = 1
        else:
            h = hh * min(1.0, fac)
            rejected = True
    while len(out) < nt:
        out.append(y.copy())
    return _unpack_states(out, d) + (status, steps)
