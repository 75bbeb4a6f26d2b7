"""Sensor tiling for the FP32 summation kernels.

The kernels evaluate Gaussian beams along straight, evenly spaced runs of
sensors with a complex-exponential recurrence (two complex multiplies per
sensor), and cull (beam, time tile, sensor tile) triples by bounding boxes.
This module orders the sensors so that

* every group of up to 16 consecutive sensors lies on one grid line with unit
  step (a run), and
* tiles of 8 groups (128 sensors) are spatially compact: groups are ordered by
  the Morton code of their centres, quantised at the group length.

The result (sorted order and tile offsets) is passed to libmsgb through
``msgb_sensor_tiling``; without it the library falls back to its own
cell-Morton order with fixed 128-sensor tiles.
"""

from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

GS = 16
GROUPS_PER_TILE = 8


def _morton(q: np.ndarray, bits: int = 16) -> np.ndarray:
    q = q.astype(np.uint64)
    d = q.shape[1]
    key = np.zeros(q.shape[0], dtype=np.uint64)
    for b in range(bits - 1, -1, -1):
        for i in range(d):
            key = (key << np.uint64(1)) | ((q[:, i] >> np.uint64(b)) & np.uint64(1))
    return key


def _runs_along(q: np.ndarray, idx: np.ndarray, axis: int):
    """Split the sensors ``idx`` into maximal unit-step runs along ``axis``.

    Returns a list of index arrays, each ordered along the axis.
    """
    d = q.shape[1]
    others = [a for a in range(d) if a != axis]
    sub = q[idx]
    keys = [sub[:, axis]] + [sub[:, o] for o in reversed(others)]
    order = np.lexsort(keys)
    qs = sub[order]
    new = np.ones(len(idx), dtype=bool)
    if len(idx) > 1:
        same_line = np.all(qs[1:, others] == qs[:-1, others], axis=1) if others else np.ones(len(idx) - 1, bool)
        new[1:] = ~(same_line & (qs[1:, axis] == qs[:-1, axis] + 1))
    starts = np.flatnonzero(new)
    ends = np.r_[starts[1:], len(idx)]
    return [idx[order[s:e]] for s, e in zip(starts, ends)]


def build_tiling(positions: np.ndarray, dx, max_tile: int = GS * GROUPS_PER_TILE
                 ) -> Optional[Tuple[np.ndarray, np.ndarray]]:
    """(order, tile_offsets) for grid-aligned sensors, or ``None``.

    ``order[k]`` is the caller's index of the k-th sorted sensor and tile ``i``
    holds sorted sensors ``tile_offsets[i]:tile_offsets[i+1]``.  Returns
    ``None`` when the sensors are not on the grid or do not form runs.
    """
    pos = np.asarray(positions, dtype=np.float64)
    dx = np.asarray(dx, dtype=np.float64)
    ns, d = pos.shape
    if ns == 0:
        return None
    q = np.rint(pos / dx).astype(np.int64)
    if not np.allclose(q * dx, pos, rtol=0, atol=1e-9 * float(np.min(dx))):
        return None
    idx_all = np.arange(ns)
    # run length of every sensor along every axis
    run_len = np.zeros((ns, d), dtype=np.int64)
    for a in range(d):
        for r in _runs_along(q, idx_all, a):
            run_len[r, a] = len(r)
    axis = np.argmax(run_len, axis=1)  # ties -> lowest axis
    groups = []
    for a in range(d):
        members = np.flatnonzero(axis == a)
        if members.size == 0:
            continue
        for r in _runs_along(q, members, a):
            for s in range(0, len(r), GS):
                groups.append(r[s:s + GS])
    mean_len = ns / max(len(groups), 1)
    if mean_len < 4:
        return None
    centres = np.stack([q[g].mean(axis=0) for g in groups])
    cq = np.floor((centres - centres.min(axis=0)) / GS).astype(np.int64)
    gorder = np.argsort(_morton(cq), kind="stable")
    order, offsets, fill = [], [0], 0
    for gi in gorder:
        g = groups[gi]
        if fill + len(g) > max_tile:
            offsets.append(offsets[-1] + fill)
            fill = 0
        order.append(g)
        fill += len(g)
    offsets.append(offsets[-1] + fill)
    order = np.concatenate(order).astype(np.int32)
    return order, np.asarray(offsets, dtype=np.int32)
