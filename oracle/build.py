"""Build recipe for the oracle's C restatement (test infrastructure).

``python -m oracle.build`` compiles ``csum.c`` (homogeneous closed-form
beams) and ``chet.c`` (heterogeneous media: B-spline sound speed, adaptive
Dormand-Prince beam ODE, summation over trajectories) with gcc and OpenMP into
``oracle/_build/liboracle_msgb.so``.  ``load()`` returns a ctypes handle with
typed entry points.  The reference itself is pure Python/JAX, so there are no
reference sources to compile here.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle_msgb.so")
SRCS = [os.path.join(HERE, "csum.c"), os.path.join(HERE, "chet.c")]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(s) for s in SRCS):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-o", tmp, *SRCS, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        path = LIB if os.path.exists(LIB) else build()
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I64 = ctypes.c_int64
        args = [ctypes.c_int, I64, P, P, P, P, P, ctypes.c_double, I64, P, I64, P, P, P]
        lib.oracle_sum_hom.argtypes = args + [P]
        lib.oracle_sum_hom.restype = ctypes.c_int
        lib.oracle_adj_hom.argtypes = args + [P, P]
        lib.oracle_adj_hom.restype = ctypes.c_int
        D = ctypes.c_double
        lib.oracle_het_traj.argtypes = [ctypes.c_int, I64, P, P, P, P, ctypes.c_int, ctypes.c_int, P, P, P, P, D, D,
                                        D, D, I64, D, I64, P, P, P, P]
        lib.oracle_het_traj.restype = ctypes.c_int
        lib.oracle_sum_traj.argtypes = [ctypes.c_int, I64, P, P, P, I64, I64, P, P, P, P]
        lib.oracle_sum_traj.restype = ctypes.c_int
        lib.oracle_adj_traj.argtypes = [ctypes.c_int, I64, P, P, I64, I64, P, P, P, P, P]
        lib.oracle_adj_traj.restype = ctypes.c_int
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _common(tab, c, ts, sens, L, periodic):
    d = tab["x0"].shape[1]
    x0 = np.ascontiguousarray(tab["x0"], np.float64)
    p0 = np.ascontiguousarray(tab["p0"], np.float64)
    al = np.ascontiguousarray(tab["alpha"], np.complex128)
    om = np.ascontiguousarray(tab["omega"], np.float64)
    ts = np.ascontiguousarray(ts, np.float64)
    sens = np.ascontiguousarray(np.asarray(sens, np.float64).reshape(-1, d))
    L = np.ascontiguousarray(L, np.float64)
    per = np.ascontiguousarray(np.asarray(periodic, np.int32))
    keep = (x0, p0, al, om, ts, sens, L, per)
    return d, keep


def sum_hom(tab, c, ts, sens, L, periodic):
    """Dense FP64 forward over both modes; returns (Nt, Ns)."""
    lib = load()
    d, (x0, p0, al, om, ts, sens, L, per) = _common(tab, c, ts, sens, L, periodic)
    a0 = np.ascontiguousarray(tab["a0"], np.complex128)
    out = np.zeros((ts.size, sens.shape[0]))
    rc = lib.oracle_sum_hom(d, x0.shape[0], _p(x0), _p(p0), _p(al), _p(a0), _p(om), float(c),
                            ts.size, _p(ts), sens.shape[0], _p(sens), _p(L), _p(per), _p(out))
    if rc:
        raise RuntimeError(f"oracle_sum_hom failed: {rc}")
    return out


def adj_hom(tab, a0_unit, c, ts, sens, L, periodic, data):
    """Per-beam coefficient gradient g_b (complex, (n,))."""
    lib = load()
    d, (x0, p0, al, om, ts, sens, L, per) = _common(tab, c, ts, sens, L, periodic)
    a0 = np.ascontiguousarray(a0_unit, np.complex128)
    data = np.ascontiguousarray(data, np.float64).reshape(ts.size, sens.shape[0])
    g = np.zeros(x0.shape[0], np.complex128)
    rc = lib.oracle_adj_hom(d, x0.shape[0], _p(x0), _p(p0), _p(al), _p(a0), _p(om), float(c),
                            ts.size, _p(ts), sens.shape[0], _p(sens), _p(L), _p(per), _p(data), _p(g))
    if rc:
        raise RuntimeError(f"oracle_adj_hom failed: {rc}")
    return g


_BOUNDARY_CODE = {"clamp": 0, "nearest": 0, "edge": 0, "wrap": 1, "periodic": 1, "reflect": 2, "mirror": 3}


def het_trajectories(x0, p0, alpha, mode, medium, ts, rtol=1e-7, atol=1e-9, max_steps=4096, dt0=0.0, lam=0.0):
    """Adaptive Dormand-Prince trajectories of nb beams (amplitude from 1).

    medium: ("constant", c) or a grid interpolant with ``coeffs``, ``spacing``,
    ``origin``, ``method`` ("linear" / "bspline3") and ``boundary`` attributes
    (oracle.ode.GridSpeed or beamax_b200.utils.interp's interpolant).
    Returns (rec (nb, nt, 2d + 2d^2 + 2), status (nb), steps (nb))."""
    lib = load()
    x0 = np.ascontiguousarray(x0, np.float64)
    nb, d = x0.shape
    p0 = np.ascontiguousarray(p0, np.float64).reshape(nb, d)
    al = np.ascontiguousarray(alpha, np.complex128).reshape(nb, d)
    mo = np.ascontiguousarray(np.broadcast_to(np.asarray(mode, np.float64), (nb,)))
    ts = np.ascontiguousarray(ts, np.float64)
    n = np.ones(3, np.int32)
    sp = np.ones(3)
    org = np.zeros(3)
    if isinstance(medium, tuple) and medium[0] == "constant":
        kind, bnd, coeffs, c = 0, 0, np.zeros(1), float(medium[1])
    else:
        kind = 1 if medium.method == "linear" else 2
        bnd = _BOUNDARY_CODE[medium.boundary]
        coeffs = np.ascontiguousarray(medium.coeffs, np.float64)
        n[:d] = coeffs.shape
        sp[:d] = medium.spacing
        org[:d] = medium.origin
        c = float(np.max(coeffs))
    rl = 2 * d + 2 * d * d + 2
    rec = np.zeros((nb, ts.size, rl))
    status = np.zeros(nb, np.int32)
    steps = np.zeros(nb, np.int64)
    rc = lib.oracle_het_traj(d, nb, _p(x0), _p(p0), _p(al), _p(mo), kind, bnd, _p(n), _p(sp), _p(org), _p(coeffs),
                             c, float(lam), float(rtol), float(atol), int(max_steps), float(dt0), ts.size, _p(ts),
                             _p(rec), _p(status), _p(steps))
    if rc:
        raise RuntimeError(f"oracle_het_traj failed: {rc}")
    return rec, status, steps


def sum_traj(rec, amp, omega, sens, L, periodic, out=None):
    """Dense FP64 sum over trajectory records (nb, nt, RL): adds into out (nt, ns)."""
    lib = load()
    rec = np.ascontiguousarray(rec, np.float64)
    nb, nt, rl = rec.shape
    d = int(round((-2 + np.sqrt(4 + 8 * (rl - 2))) / 4))
    amp = np.ascontiguousarray(amp, np.complex128)
    om = np.ascontiguousarray(omega, np.float64)
    sens = np.ascontiguousarray(np.asarray(sens, np.float64).reshape(-1, d))
    L = np.ascontiguousarray(L, np.float64)
    per = np.ascontiguousarray(np.asarray(periodic, np.int32))
    if out is None:
        out = np.zeros((nt, sens.shape[0]))
    rc = lib.oracle_sum_traj(d, nb, _p(rec), _p(amp), _p(om), nt, sens.shape[0], _p(sens), _p(L), _p(per), _p(out))
    if rc:
        raise RuntimeError(f"oracle_sum_traj failed: {rc}")
    return out


def adj_traj(rec, omega, sens, L, periodic, data):
    """Per-beam complex gradient of the dense sum over records (nb, nt, RL)."""
    lib = load()
    rec = np.ascontiguousarray(rec, np.float64)
    nb, nt, rl = rec.shape
    d = int(round((-2 + np.sqrt(4 + 8 * (rl - 2))) / 4))
    om = np.ascontiguousarray(omega, np.float64)
    sens = np.ascontiguousarray(np.asarray(sens, np.float64).reshape(-1, d))
    L = np.ascontiguousarray(L, np.float64)
    per = np.ascontiguousarray(np.asarray(periodic, np.int32))
    data = np.ascontiguousarray(data, np.float64).reshape(nt, sens.shape[0])
    g = np.zeros(nb, np.complex128)
    rc = lib.oracle_adj_traj(d, nb, _p(rec), _p(om), nt, sens.shape[0], _p(sens), _p(L), _p(per), _p(data), _p(g))
    if rc:
        raise RuntimeError(f"oracle_adj_traj failed: {rc}")
    return g


if __name__ == "__main__":
    print(build(force=True))
