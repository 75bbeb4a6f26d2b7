"""Build recipe for the oracle's C restatement (test infrastructure).

``python -m oracle.build`` compiles ``csum.c`` with gcc and OpenMP into
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
SRC = os.path.join(HERE, "csum.c")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
    subprocess.run(cmd, check=True)
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


if __name__ == "__main__":
    print(build(force=True))
