"""Beam propagators (identifiers mapped to libmsgb kernels)."""
from . import gb_solvers  # noqa: F401
