"""``DyadicDecomposition``: multi-level dyadic tiling of Fourier space.

Host-side metadata with the reference's attribute names and validation
(beamax decomposition.py:89-541).  Levels run from the innermost
low-frequency region to the outermost; box lengths double with the level and
each level removes the central region that the previous level covers.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import numpy as np


def _is_integral(value) -> bool:
    if isinstance(value, (bool, np.bool_)):
        return False
    if isinstance(value, (int, np.integer)):
        return True
    if isinstance(value, (float, np.floating)):
        return bool(np.isfinite(value) and float(value).is_integer())
    return False


def validate_params(num_levels, N, num_boxes_levels, box_aspect_ratio, boxes_per_dim_levels=None) -> None:
    """Raise ``ValueError`` when the parameters cannot tile the grid (decomposition.py:89-215)."""
    if not isinstance(num_levels, int) or num_levels < 1:
        raise ValueError(f"num_levels must be positive int; got {num_levels}.")
    if not N or any(not _is_integral(x) for x in N):
        raise ValueError(f"N entries must be integers; got {N}.")
    N = tuple(int(x) for x in N)
    if any(n <= 0 for n in N):
        raise ValueError(f"N must be positive; got {N}.")
    if any(n % 2 for n in N):
        raise ValueError(f"N must be even along all axes; got {N}.")
    ndim = len(N)
    if any(not _is_integral(x) for x in box_aspect_ratio):
        raise ValueError(f"box_aspect_ratio entries must be integers; got {box_aspect_ratio}.")
    bar = tuple(int(x) for x in box_aspect_ratio)
    if len(bar) == 0:
        raise ValueError("box_aspect_ratio must be non-empty.")
    if len(bar) != ndim:
        raise ValueError(f"len(box_aspect_ratio)={len(bar)} != ndim={ndim}.")
    if any(x <= 0 for x in bar):
        raise ValueError(f"box_aspect_ratio must be positive; got {bar}.")
    if not any(x == 1 for x in bar):
        raise ValueError("At least one aspect ratio component must equal 1.")
    if ndim == 1 and bar != (1,):
        raise ValueError("For 1D, box_aspect_ratio must be (1,).")
    if any(not _is_integral(x) for x in num_boxes_levels):
        raise ValueError(f"num_boxes_levels entries must be integers; got {num_boxes_levels}.")
    nbl = tuple(int(x) for x in num_boxes_levels)
    if len(nbl) != num_levels:
        raise ValueError(f"len(num_boxes_levels)={len(nbl)} != num_levels={num_levels}.")
    if any(x <= 0 for x in nbl):
        raise ValueError(f"num_boxes_levels must be positive; got {nbl}.")
    if any(nbl[i] > nbl[i + 1] for i in range(num_levels - 1)):
        raise ValueError(f"num_boxes_levels must be non-decreasing with level; got {nbl}.")
    if boxes_per_dim_levels is not None:
        if len(boxes_per_dim_levels) != num_levels:
            raise ValueError(f"len(boxes_per_dim_levels)={len(boxes_per_dim_levels)} != num_levels={num_levels}.")
        for lvl, b in enumerate(boxes_per_dim_levels):
            if len(b) != ndim:
                raise ValueError(f"Level {lvl}: len(boxes_per_dim_levels[lvl])={len(b)} != ndim={ndim}.")
            if any(not _is_integral(x) for x in b):
                raise ValueError(f"Level {lvl}: boxes per axis must be integers; got {b}.")
            if any(int(x) <= 0 for x in b):
                raise ValueError(f"Level {lvl}: boxes per axis must be positive; got {b}.")
            if any(int(x) % 2 for x in b):
                raise ValueError(f"Level {lvl}: boxes per axis must be even for symmetry; got {b}.")
        for ax in range(ndim):
            seq = [int(boxes_per_dim_levels[l][ax]) for l in range(num_levels)]
            if any(seq[i] > seq[i + 1] for i in range(num_levels - 1)):
                raise ValueError(f"boxes_per_dim_levels must be nondecreasing per axis; axis {ax} has {seq}.")
        min_axis = int(np.argmin(np.asarray(N)))
        implied = tuple(int(boxes_per_dim_levels[l][min_axis]) for l in range(num_levels))
        if implied != nbl:
            raise ValueError("boxes_per_dim_levels disagrees with num_boxes_levels on the smallest axis. "
                             f"Expected smallest-axis sequence {nbl}, got {implied}.")
    else:
        scale = np.asarray(N, float) / float(min(N)) / np.asarray(bar, float)
        for boxes in nbl:
            counts = boxes * scale
            if not np.allclose(counts, np.rint(counts), rtol=0.0, atol=1e-12):
                raise ValueError("Derived boxes per axis are non-integral; provide a compatible "
                                 "box_aspect_ratio or explicit boxes_per_dim_levels. "
                                 f"Got counts {counts.tolist()} for {boxes} boxes.")
    N_ref = min(N)
    base = nbl[0]
    if base <= 0 or base > N_ref:
        raise ValueError(f"Invalid base boxes per side: {base} for N_ref={N_ref}.")
    max_levels = int(math.floor(math.log2(N_ref // base)) + 1)
    if not (1 <= num_levels <= max_levels):
        raise ValueError(f"num_levels must be in [1, {max_levels}] (N_ref={N_ref}, base={base}).")
    lengths = [N_ref // (nbl[-1] * 2 ** L) for L in range(num_levels - 1, -1, -1)]
    if any(L < 2 for L in lengths):
        raise ValueError("Every box length must be at least 2 Fourier samples so the "
                         f"Gaussian width is positive; computed {lengths} for N_ref={N_ref}.")
    if any(N_ref % L for L in lengths):
        raise ValueError(f"Box lengths must divide N_ref={N_ref}; computed {lengths}.")


class DyadicDecomposition:
    """Multi-level dyadic tiling (decomposition.py:218-541)."""

    def __init__(self, num_levels: int, N: Tuple[int, ...], num_boxes_levels: Tuple[int, ...],
                 box_aspect_ratio: Tuple[int, ...],
                 boxes_per_dim_levels: Optional[Tuple[Tuple[int, ...], ...]] = None):
        validate_params(num_levels, N, num_boxes_levels, box_aspect_ratio, boxes_per_dim_levels)
        self.num_levels = int(num_levels)
        self.N = tuple(int(x) for x in N)
        self.num_boxes_levels = tuple(int(x) for x in num_boxes_levels)
        self.box_aspect_ratio = tuple(int(x) for x in box_aspect_ratio)
        self.boxes_per_dim_levels = boxes_per_dim_levels
        counts = [self.outer_boxes_per_axis(l) for l in range(self.num_levels)]
        totals = [int(np.prod(c)) for c in counts]
        cut = [t // (2 ** self.ndim) if l < self.num_levels - 1 else 0 for l, t in enumerate(totals)]
        nb = [totals[0]] + [totals[i] - cut[i - 1] for i in range(1, self.num_levels)]
        self.num_boxes_ndim = np.asarray(nb, dtype=np.int32)
        self.centres_ndim = self._centres(nb).astype(np.int32)
        self.total_num_boxes = int(self.num_boxes_ndim.sum())

    @property
    def ndim(self) -> int:
        return len(self.N)

    @property
    def num_boxes_ndim_cumsum(self) -> np.ndarray:
        return np.cumsum(self.num_boxes_ndim)

    @property
    def fourier_meshgrid(self) -> np.ndarray:
        axes = [np.arange(-n // 2, n // 2, dtype=np.int32) for n in self.N]
        return np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)

    @property
    def scaling(self) -> np.ndarray:
        Nv = np.asarray(self.N, float)
        return Nv / Nv.min() / np.asarray(self.box_aspect_ratio)

    @property
    def box_lengths(self) -> np.ndarray:
        """``min(N) // (num_boxes_levels[-1] * 2**(num_levels - 1 - r))`` for level r."""
        N_ref = min(self.N)
        return np.asarray([N_ref // (self.num_boxes_levels[-1] * 2 ** L)
                           for L in range(self.num_levels - 1, -1, -1)], dtype=np.int32)

    def outer_boxes_per_axis(self, lvl: int) -> np.ndarray:
        if self.boxes_per_dim_levels is not None:
            return np.asarray(self.boxes_per_dim_levels[lvl], dtype=np.int64)
        aspect = np.asarray(self.N, float) / float(min(self.N))
        per = self.num_boxes_levels[lvl] * aspect / np.asarray(self.box_aspect_ratio, float)
        out = np.rint(per).astype(np.int64)
        if not np.allclose(per, out, rtol=0.0, atol=1e-12):
            raise ValueError(f"Level {lvl}: non-integral derived box counts {per.tolist()}.")
        return out

    def lattice(self, lvl: int):
        """Per-axis (count, first centre, step) of the level's outer box lattice."""
        step = [int(self.box_lengths[lvl]) * b for b in self.box_aspect_ratio]
        cnt = [int(c) for c in self.outer_boxes_per_axis(lvl)]
        first = [-(c // 2) * s + s // 2 for c, s in zip(cnt, step)]
        return cnt, first, step

    def _centres(self, nb):
        out = []
        bounds_prev = np.zeros(self.ndim, dtype=np.int64)
        for lvl in range(self.num_levels):
            cnt, first, step = self.lattice(lvl)
            axes = [np.arange(first[a], (cnt[a] // 2) * step[a], step[a]) for a in range(self.ndim)]
            mesh = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, self.ndim)
            if mesh.size and np.any(bounds_prev > 0):
                mesh = mesh[~np.all(np.abs(mesh) < bounds_prev, axis=1)]
            if mesh.shape[0] != nb[lvl]:
                raise ValueError(f"Level {lvl}: expected {nb[lvl]} centres, got {mesh.shape[0]}. "
                                 f"(per_axis_counts={cnt})")
            out.append(mesh)
            if mesh.shape[0]:
                bounds_prev = np.max(np.abs(mesh), axis=0) + int(self.box_lengths[lvl]) // 2
        return np.concatenate(out, axis=0)

    def find_level(self, box_num):
        return np.searchsorted(self.num_boxes_ndim_cumsum, box_num, side="right")
