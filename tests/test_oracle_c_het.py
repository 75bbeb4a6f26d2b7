"""CPU tests of the oracle's C restatement of the heterogeneous path
(oracle/chet.c): the adaptive Dormand-Prince trajectories equal the NumPy
oracle's (oracle/ode.py:dopri5, the same method step for step), the dense
trajectory sum equals the NumPy summation (gb/core.py:194-329 restated), and
the transpose passes the dot-product test.  These pin the C code that the
GPU parity tests at full configuration sizes and the timed CPU baseline use.
"""

import numpy as np
import pytest

from oracle import build as ob
from oracle import msgb as om
from oracle import ode as oo


def _medium(N=(32, 32), dx=(1e-4, 1e-4), seed=3, contrast=0.1, corr=4.0):
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal(N), corr, mode="wrap")
    g = np.clip(g / np.max(np.abs(g)), -1, 1)
    c = 1500.0 * (1 + contrast * g)
    return c, oo.GridSpeed(c, dx, method="bspline3", boundary="clamp")


def _beams(n, N, dx, seed=0):
    rng = np.random.default_rng(seed)
    L = np.asarray(N) * np.asarray(dx)
    x0 = (0.2 + 0.6 * rng.uniform(size=(n, 2))) * L
    th = rng.uniform(0, 2 * np.pi, n)
    p0 = 2 * np.pi * np.stack([np.cos(th), np.sin(th)], -1)
    alpha = 1j * rng.uniform(2e6, 8e6, size=(n, 2)) + rng.uniform(-1e5, 1e5, size=(n, 2))
    omega = rng.uniform(2e3, 8e3, n)
    return x0, p0, alpha, omega


@pytest.fixture(scope="module", autouse=True)
def _built():
    ob.build()


def test_c_dopri5_equals_numpy_dopri5():
    N, dx = (32, 32), (1e-4, 1e-4)
    c, speed = _medium(N, dx)
    x0, p0, alpha, _ = _beams(4, N, dx)
    ts = np.arange(0, 60) * 0.3 * 1e-4 / 1650.0
    mode = np.array([1.0, -1.0, 1.0, -1.0])
    rec, status, steps = ob.het_trajectories(x0, p0, alpha, mode, speed, ts)
    assert np.all(status == 0) and np.all(steps >= ts.size - 1)
    for b in range(4):
        xt, pt, Mt, At, st, nsteps = oo.dopri5(x0[b], p0[b], np.diag(alpha[b]), 1.0, mode[b], ts, speed)
        assert st == 0 and nsteps == steps[b]
        r = rec[b]
        assert np.max(np.abs(r[:, :2] - xt)) <= 1e-14 * np.max(np.abs(xt)) + 1e-18
        assert np.max(np.abs(r[:, 2:4] - pt)) <= 1e-12 * np.max(np.abs(pt))
        Mc = (r[:, 4:12:2] + 1j * r[:, 5:12:2]).reshape(-1, 2, 2)
        assert np.max(np.abs(Mc - Mt)) <= 1e-10 * np.max(np.abs(Mt))
        assert np.max(np.abs(r[:, 12] + 1j * r[:, 13] - At)) <= 1e-10


def test_c_trajectory_sum_equals_numpy_sum_and_dot_test():
    N, dx = (32, 32), (1e-4, 1e-4)
    c, speed = _medium(N, dx, seed=5)
    x0, p0, alpha, omega = _beams(6, N, dx, seed=1)
    ts = np.arange(0, 40) * 0.3 * 1e-4 / 1650.0
    mode = np.where(np.arange(6) % 2 == 0, 1.0, -1.0)
    rec, status, _ = ob.het_trajectories(x0, p0, alpha, mode, speed, ts)
    assert np.all(status == 0)
    L = np.asarray(N) * np.asarray(dx)
    sens = np.stack([np.arange(32) * 1e-4, np.zeros(32)], -1)
    rng = np.random.default_rng(2)
    amp = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    out = ob.sum_traj(rec, amp, omega, sens, L, (False, False))
    ref = np.zeros_like(out)
    for b in range(6):
        r = rec[b]
        xt, pt = r[:, :2], r[:, 2:4]
        Mt = (r[:, 4:12:2] + 1j * r[:, 5:12:2]).reshape(-1, 2, 2)
        At = amp[b] * (r[:, 12] + 1j * r[:, 13])
        ref += oo.beam_field(xt, pt, Mt, At, omega[b], sens, L, (False, False))
    assert om.rel_l2(ref, out) < 1e-12
    data = rng.standard_normal(out.shape)
    g = ob.adj_traj(rec, omega, sens, L, (False, False), data)
    lhs = float(np.sum(out * data))
    rhs = float(np.real(np.sum(amp * np.conj(g))))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
