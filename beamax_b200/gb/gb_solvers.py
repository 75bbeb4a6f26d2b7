"""Beam ODE solvers selectable through ``MSGBSolver(ode_solver=...)``.

The reference passes Python functions (beamax gb/gb_solvers.py:356-422
``solve_hom_diag`` and :940-1014 ``solve_ODE_base``).  Here the same names are
identifiers that select a libmsgb propagation kernel:

* ``solve_hom_diag`` - closed-form homogeneous propagation (Sherman-Morrison
  Hessian, closed-form amplitude), fused into the summation kernels.  As in
  the reference, the speed is c at the origin (``c(zeros(d))``, :356-422) and
  the absorption ``lam`` is ignored, whatever the medium.
* ``solve_hom_general`` - the closed form for a general initial Hessian
  (:425-481: M0 (I + c t P_perp M0 / |p|)^-1, a0 / sqrt(det(...))).  The
  solver's beams start with a diagonal Hessian, for which it equals
  ``solve_hom_diag``, so it selects the same fused kernels.
* ``solve_ODE_base`` - the general ray/Riccati/amplitude ODE.  In a
  homogeneous medium its exact solution is the closed form above, so the same
  fused kernels are used; heterogeneous media use ``msgb_ode_trajectories``
  (adaptive Dormand-Prince 5(4), or fixed-step RK4), configured by
  ``SolverConfig``.

Reference functions passed by object are recognised by their ``__name__``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Optional


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
solve_hom_general = SolverId("solve_hom_general")
solve_hom_TR = SolverId("solve_hom_TR")

KNOWN = {"solve_hom_diag", "solve_hom_general", "solve_ODE_base", "solve_ODE_batch_t", "solve_hom_TR"}
# propagators that are closed forms at c(0) (no ODE, absorption ignored)
CLOSED_FORM = {"solve_hom_diag", "solve_hom_general"}


def solver_name(fn) -> str:
    name = fn if isinstance(fn, str) else getattr(fn, "__name__", None)
    if name not in KNOWN:
        raise ValueError(f"Unsupported ode_solver {fn!r}; expected one of {sorted(KNOWN)}")
    return name


ADAPTIVE_SOLVERS = {"dopri5", "tsit5", "dopri8"}
FIXED_SOLVERS = {"rk4"}


def ode_method(solver) -> str:
    """Integrator behind a ``SolverConfig.solver`` value: "dopri5" or "rk4".

    Accepts the names above or a diffrax solver object (by class name).  The
    reference's default, diffrax Tsit5, is an explicit 5(4) pair like
    Dormand-Prince 5(4), which runs in its place with the same tolerances.
    """
    name = solver if isinstance(solver, str) else type(solver).__name__
    key = name.lower()
    if key in ADAPTIVE_SOLVERS:
        return "dopri5"
    if key in FIXED_SOLVERS:
        return "rk4"
    raise ValueError(f"Unsupported ODE solver {name!r}; expected one of "
                     f"{sorted(ADAPTIVE_SOLVERS | FIXED_SOLVERS)}")


@dataclass(frozen=True)
class SolverConfig:
    """Integrator settings (gb/gb_solvers.py:597-700, same fields, defaults and checks).

    ``solver`` names the integrator ("tsit5"/"dopri5" adaptive, "rk4" fixed
    step; a diffrax solver object is recognised by its class name).  The step
    controller is the integral controller the reference's default
    coefficients select (pcoeff 0, icoeff 1, dcoeff 0); other coefficients are
    rejected.  ``substeps`` (no reference counterpart) is the number of RK4
    steps per save interval.  ``dense_output`` (no reference counterpart):
    False ends adaptive steps on every save time (at most one save interval
    per step, robust for strongly focusing beams); True lets steps follow the
    error control and reads save times from the continuous extension, as
    diffrax's SaveAt(ts) does.
    """

    solver: Any = "tsit5"
    max_steps: int = 4096
    rtol: float = 1e-7
    atol: float = 1e-9
    pcoeff: float = 0.0
    icoeff: float = 1.0
    dcoeff: float = 0.0
    dt0: Optional[float] = None
    substeps: int = 1
    dense_output: bool = False

    def __post_init__(self) -> None:
        if isinstance(self.max_steps, bool) or not isinstance(self.max_steps, int):
            raise ValueError("max_steps must be a positive integer.")
        if self.max_steps <= 0:
            raise ValueError("max_steps must be a positive integer.")
        for name in ("rtol", "atol"):
            value = float(getattr(self, name))
            if not math.isfinite(value) or value <= 0:
                raise ValueError(f"{name} must be finite and positive.")
        for name in ("pcoeff", "icoeff", "dcoeff"):
            value = float(getattr(self, name))
            if not math.isfinite(value):
                raise ValueError(f"{name} must be finite.")
        if self.dt0 is not None and (not math.isfinite(float(self.dt0)) or float(self.dt0) <= 0):
            raise ValueError("dt0 must be finite and positive when provided.")
        if isinstance(self.substeps, bool) or not isinstance(self.substeps, int) or self.substeps < 1:
            raise ValueError("substeps must be a positive integer.")
        ode_method(self.solver)
        if (float(self.pcoeff), float(self.icoeff), float(self.dcoeff)) != (0.0, 1.0, 0.0):
            raise NotImplementedError("only the integral step controller (pcoeff=0, icoeff=1, dcoeff=0) "
                                      "is implemented")

    @property
    def method(self) -> str:
        return ode_method(self.solver)

    @classmethod
    def from_precision(cls, use_x64: Optional[bool] = None, solver=None, **overrides) -> "SolverConfig":
        """Defaults by precision (gb/gb_solvers.py:633-703).  The integrator
        always runs in FP64, so ``use_x64=None`` selects the FP64 defaults."""
        if use_x64 is None:
            use_x64 = True
        defaults = ({"rtol": 1e-7, "atol": 1e-9, "max_steps": 4096} if use_x64
                    else {"rtol": 1e-4, "atol": 1e-6, "max_steps": 4096})
        defaults.update(overrides)
        if solver is not None:
            defaults["solver"] = solver
        return cls(**defaults)
