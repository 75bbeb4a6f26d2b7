"""Array helpers (beamax utils/arrays.py:237-289)."""

from __future__ import annotations

import numpy as np


def extract_centered_box(arr, box_shape_tuple, center):
    """Wrap-around extraction of a centred box."""
    arr = np.asarray(arr)
    starts = (np.asarray(center) - np.asarray([m // 2 for m in box_shape_tuple])) % np.asarray(arr.shape)
    out = arr
    for ax in range(arr.ndim):
        out = np.take(out, (starts[ax] + np.arange(int(box_shape_tuple[ax]))) % arr.shape[ax], axis=ax)
    return out


def rel_l2(a, b) -> float:
    """``||a - b|| / (||a|| + 1e-30)``."""
    a = np.asarray(a.detach().cpu() if hasattr(a, "detach") else a)
    b = np.asarray(b.detach().cpu() if hasattr(b, "detach") else b)
    return float(np.linalg.norm(a - b) / (np.linalg.norm(a) + 1e-30))
