"""beamax_b200: B200-native MSGB forward operator and its exact adjoint.

Public names follow beamax (beamax/__init__.py:14-60): ``Domain``, ``Sensor``,
``DyadicDecomposition``, ``MSWPT`` and, under ``solvers``, ``MSGBSolver``.
Compute runs in libmsgb.so (sm_100a); see ``include/msgb.h`` for the C ABI.
"""

from .decomposition import DyadicDecomposition  # noqa: F401
from .geometry import Domain, Sensor  # noqa: F401
from .transforms import MSWPT  # noqa: F401
from . import gb, utils  # noqa: F401
from .solvers import MSGBSolver  # noqa: F401

__all__ = ["Domain", "Sensor", "DyadicDecomposition", "MSWPT", "MSGBSolver", "gb", "utils", "solvers"]
