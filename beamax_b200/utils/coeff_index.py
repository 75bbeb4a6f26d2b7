"""Flat coefficient index <-> (level, box, local index) (beamax utils/coeff_index.py:29-180)."""

from __future__ import annotations

import numpy as np


def batch_data(*args, batch_size, zero_padded_args=()):
    """Pad the leading axis to a multiple of ``batch_size`` and reshape (coeff_index.py:29-87)."""
    if not args:
        raise ValueError("batch_data requires at least one array.")
    if isinstance(batch_size, bool) or not isinstance(batch_size, int) or batch_size <= 0:
        raise ValueError("batch_size must be a positive integer.")
    if any(np.ndim(a) == 0 for a in args):
        raise ValueError("All arrays must have a leading batch dimension.")
    b = args[0].shape[0]
    if b == 0:
        raise ValueError("Cannot batch empty arrays.")
    if any(a.shape[0] != b for a in args[1:]):
        raise ValueError("All arrays must have the same leading dimension.")
    if any(isinstance(i, bool) or not isinstance(i, int) or i < 0 or i >= len(args) for i in zero_padded_args):
        raise ValueError("zero_padded_args contains an invalid argument index.")
    nb = (b + batch_size - 1) // batch_size
    out = []
    for i, a in enumerate(args):
        a = np.asarray(a)
        pad = nb * batch_size - b
        if pad:
            fill = np.zeros((pad,) + a.shape[1:], a.dtype) if i in zero_padded_args \
                else np.broadcast_to(a[-1:], (pad,) + a.shape[1:])
            a = np.concatenate([a, fill], axis=0)
        out.append(a.reshape((nb, batch_size) + a.shape[1:]))
    return tuple(out)


def find_level(dyadic_decomp, box_num):
    """Level of a global box index (coeff_index.py:90-108)."""
    return np.searchsorted(dyadic_decomp.num_boxes_ndim_cumsum, box_num, side="right")


def compute_coeff_shapes(dyadic_decomp, redundancy, levels):
    """(num_boxes_level, *support_shape) per level (coeff_index.py:150-180)."""
    bar = np.asarray(dyadic_decomp.box_aspect_ratio)
    return np.asarray([[int(dyadic_decomp.num_boxes_ndim[l])]
                       + [int(x) for x in bar * redundancy * int(dyadic_decomp.box_lengths[l])]
                       for l in np.atleast_1d(levels)], dtype=np.int64)


def find_tensor_and_multiindex(flat_indices, shapes):
    """(level, multi-index (k, m)) of flat coefficient indices (coeff_index.py:111-147)."""
    flat = np.asarray(flat_indices, dtype=np.int64)
    shapes = np.asarray(shapes, dtype=np.int64)
    cum = np.cumsum(np.prod(shapes, axis=1))
    lvl = np.searchsorted(cum, flat, side="right")
    local = np.where(lvl > 0, flat - np.take(cum, np.maximum(lvl - 1, 0)), flat)
    mi = np.zeros((shapes.shape[1], flat.size), dtype=np.int64)
    for L in np.unique(lvl):
        sel = lvl == L
        mi[:, sel] = np.stack(np.unravel_index(local[sel], tuple(int(x) for x in shapes[L])))
    return lvl, mi
