"""JAX binding of the beam summation: XLA FFI custom calls + ``jax.custom_vjp``.

For beamax users who stay in JAX: ``beam_sum`` is the real Gaussian-beam
summation of the MSGB forward with both branches of every selected
coefficient (what ``_compute_forward_result_jit`` computes in
``MSGBSolver.forward_with_params``, solvers/msgb_solvers/msgb_solver.py:
958-977, for the real sum methods), run by libmsgb's CUDA kernels as XLA
custom calls.  It is linear in the amplitudes ``a0``; its VJP with respect to
``a0`` is the exact transpose (``msgb_adj_gather_*``), so ``jax.grad``
through ``beam_sum`` and the reference's own differentiable ``jnp`` MSWPT
gives the exact adjoint with the selection frozen (the pattern of
examples/diagnostics/msgb_adjoint_pairing.py:156-165).

The C++ handlers (``msgb_xla_ffi.cc``) are compiled by ``build()`` against
jaxlib's FFI headers (``jax.ffi.include_dir()``) and linked to libmsgb.so.
Without JAX this module imports and ``available()`` is False; every other
function then raises ImportError.
"""

from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np

try:  # JAX is optional: the torch / C ABI path does not need it
    import jax
    import jax.numpy as jnp
except ImportError:  # pragma: no cover - exercised where JAX is absent
    jax = None
    jnp = None

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
SRC = os.path.join(HERE, "msgb_xla_ffi.cc")
LIB = os.path.join(HERE, "libmsgb_xla_ffi.so")

# (XLA custom-call target, exported handler symbol)
TARGETS = {
    "msgb_sum_fwd_f64": "MsgbSumFwdF64",
    "msgb_sum_fwd_f32": "MsgbSumFwdF32",
    "msgb_adj_gather_f64": "MsgbAdjGatherF64",
    "msgb_adj_gather_f32": "MsgbAdjGatherF32",
}

_registered = False


def available() -> bool:
    """True when JAX is importable (the handlers can then be built and registered)."""
    return jax is not None


def _require():
    if jax is None:
        raise ImportError("beamax_b200.jax_ffi needs jax (not installed); use the torch / C ABI path "
                          "(beamax_b200.MSGBSolver) instead")


def build(force: bool = False) -> str:
    """Compile the FFI handlers into libmsgb_xla_ffi.so (needs jax's FFI headers and libmsgb.so)."""
    _require()
    from .. import build as core

    lib = core.build()
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                                                          os.path.getmtime(lib)):
        return LIB
    cxx = shutil.which("g++") or "g++"
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(core._nvcc())), "include")
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", SRC, "-o", LIB, "-I" + jax.ffi.include_dir(),
           "-I" + cuda_inc, "-I" + os.path.join(ROOT, "include"), "-L" + PKG, "-lmsgb",
           "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True)
    return LIB


def register() -> None:
    """Build (if needed) and register the four handlers as CUDA custom-call targets."""
    global _registered
    _require()
    if _registered:
        return
    lib = ctypes.CDLL(build())
    for target, sym in TARGETS.items():
        jax.ffi.register_ffi_target(target, jax.ffi.pycapsule(getattr(lib, sym)), platform="CUDA")
    _registered = True


def _attrs(c, L, periodic):
    return dict(c=np.float64(c), L=np.asarray(L, np.float64), periodic=np.asarray(periodic, np.int64))


def beam_sum(a0, x0, p0, alpha, omega, ts, sensors, *, c, L, periodic, precision="fp64", cutoff=16.0):
    """sum_j sum_{mode = +1, -1} 2 Re[a0_j K_{j,mode}(t, s)], shape (nt, ns).

    a0 (n,) complex: amplitudes including the coefficients; x0, p0 (n, d);
    alpha (n, d) complex, the diagonal of M0; omega (n,); ts (nt,); sensors
    (ns, d); homogeneous sound speed c (solve_hom_diag), domain size L and
    periodic flags.  precision "fp64" (dense, the reference's semantics) or
    "fp32" (Gaussian cutoff, Kahan sums).  Differentiable in a0 (custom_vjp);
    the other inputs are treated as constants."""
    _require()
    register()
    attrs = _attrs(c, L, periodic)
    nt, ns = int(np.shape(ts)[0]), int(np.shape(sensors)[0])
    n = int(np.shape(a0)[0])
    fp32 = precision == "fp32"
    consts = (jnp.asarray(x0, jnp.float64), jnp.asarray(p0, jnp.float64), jnp.asarray(alpha, jnp.complex128))
    tail = (jnp.asarray(omega, jnp.float64), jnp.asarray(ts, jnp.float64), jnp.asarray(sensors, jnp.float64))

    def fwd_call(a):
        if fp32:
            call = jax.ffi.ffi_call("msgb_sum_fwd_f32", jax.ShapeDtypeStruct((nt, ns), jnp.float32))
            return call(*consts, a, *tail, cutoff=np.float64(cutoff), **attrs)
        call = jax.ffi.ffi_call("msgb_sum_fwd_f64", jax.ShapeDtypeStruct((nt, ns), jnp.float64))
        return call(*consts, a, *tail, **attrs)

    @jax.custom_vjp
    def f(a):
        return fwd_call(a)

    def f_fwd(a):
        return fwd_call(a), None

    def f_bwd(_, d):
        unit = jnp.ones((n,), jnp.complex128)
        if fp32:
            call = jax.ffi.ffi_call("msgb_adj_gather_f32", jax.ShapeDtypeStruct((n,), jnp.complex128))
            g = call(*consts, unit, *tail, jnp.asarray(d, jnp.float32), cutoff=np.float64(cutoff), **attrs)
        else:
            call = jax.ffi.ffi_call("msgb_adj_gather_f64", jax.ShapeDtypeStruct((n,), jnp.complex128))
            g = call(*consts, unit, *tail, jnp.asarray(d, jnp.float64), **attrs)
        # g_j = sum 2 d conj(K_j); JAX's cotangent of a real output with
        # respect to a complex input is d<d, y>/d Re a - i d<d, y>/d Im a = conj(g).
        return (jnp.conj(g),)

    f.defvjp(f_fwd, f_bwd)
    return f(jnp.asarray(a0, jnp.complex128))
