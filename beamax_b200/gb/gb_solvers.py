"""Beam ODE solvers selectable through ``MSGBSolver(ode_solver=...)``.

The reference passes Python functions (beamax gb/gb_solvers.py:356-422
``solve_hom_diag`` and :940-1014 ``solve_ODE_base``).  Here the same names are
identifiers that select a libmsgb propagation kernel:

* ``solve_hom_diag`` - closed-form homogeneous propagation (Sherman-Morrison
  Hessian, closed-form amplitude), fused into the summation kernels.
* ``solve_ODE_base`` - the general ray/Riccati/amplitude ODE.  In a
  homogeneous medium its exact solution is the closed form above, so the same
  fused kernels are used; heterogeneous media use the RK4 integrator.

Reference functions passed by object are recognised by their ``__name__``.
"""

from __future__ import annotations


class SolverId:
    def __init__(self, name: str):
        self.__name__ = name
        self.name = name

    def __repr__(self) -> str:
        return f"<beamax_b200 ODE solver {self.name}>"

    def __call__(self, *args, **kwargs):
        raise TypeError(f"{self.name} is evaluated inside the CUDA summation kernels; "
                        "pass it to MSGBSolver(ode_solver=...) instead of calling it")


solve_hom_diag = SolverId("solve_hom_diag")
solve_ODE_base = SolverId("solve_ODE_base")
solve_ODE_batch_t = SolverId("solve_ODE_batch_t")

KNOWN = {"solve_hom_diag", "solve_ODE_base", "solve_ODE_batch_t"}


def solver_name(fn) -> str:
    name = fn if isinstance(fn, str) else getattr(fn, "__name__", None)
    if name not in KNOWN:
        raise ValueError(f"Unsupported ode_solver {fn!r}; expected one of {sorted(KNOWN)}")
    return name
