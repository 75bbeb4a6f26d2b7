"""MSGB solvers."""
from .msgb_solver import MSGBSolver, Selection  # noqa: F401


def __getattr__(name):
    if name in ("MSGBForward", "msgb_forward"):
        from . import autograd

        return getattr(autograd, name)
    raise AttributeError(name)
