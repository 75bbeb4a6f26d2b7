"""FP64 CPU oracle for the MSGB forward operator and its exact transpose.

TEST INFRASTRUCTURE ONLY.  This package is a plain NumPy/SciPy (and C, see
``csum.c``) restatement of the reference beamax 0.2.2 algorithm for the MSGB
hot path.  It exists to check the CUDA implementation in ``beamax_b200``; it is
never the thing measured or shipped.  Only ``tests/``, ``__graft_entry__.smoke``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it, and only as the checker.

Parity status: the reference is JAX code that cannot run on this machine (no
jax/jaxlib/equinox/diffrax).  The restatement is pinned against the reference's
own known-answer and identity tests (ported in ``tests/test_oracle_pins.py``):
box lengths/counts, Sum g*h = 1, inverse(forward(f)) = f, single coefficient ==
frame atom, beam init == frame atom at t = 0, D'Alembert 1D forward, top_n
ordering, oversized top_n == half-frame cap.  The reference ships no golden
vectors, so bit-level agreement with JAX's FFT/Tsit5 is unpinned; every pin
above is an exact identity or analytic answer.
"""
