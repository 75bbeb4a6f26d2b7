"""Grid-valued sound speed usable by the GPU beam propagator.

``make_c_function_from_grid`` mirrors beamax utils/interp.py:158-263: the
returned object is callable on the host (NumPy, for inspection) and carries the
interpolation data (grid values, or cubic B-spline coefficients prefiltered
with ``scipy.ndimage.spline_filter`` exactly as the reference does) that the
RK4 kernel evaluates, together with its first and second derivatives, on the
GPU.
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

_BOUNDARY = {"clamp": "nearest", "nearest": "nearest", "edge": "nearest", "reflect": "reflect",
             "mirror": "mirror", "wrap": "wrap", "periodic": "wrap"}
BOUNDARY_CODE = {"nearest": 0, "wrap": 1, "reflect": 2, "mirror": 3}


def canonical_boundary(boundary: str) -> str:
    try:
        return _BOUNDARY[boundary]
    except KeyError as exc:
        raise ValueError(f"Unsupported boundary='{boundary}'. Expected one of: "
                         f"{', '.join(sorted(_BOUNDARY))}") from exc


class GridInterpolant:
    """n-linear or cubic B-spline interpolant of a grid (utils/interp.py:31-263)."""

    def __init__(self, c_map, spacing=None, origin=None, *, method: str = "linear", boundary: str = "clamp",
                 smooth_sigma: Optional[float | Sequence[float]] = None):
        from scipy import ndimage

        method = method.lower()
        boundary = canonical_boundary(boundary)
        values = np.asarray(c_map, dtype=np.float64)
        if values.ndim == 0:
            raise ValueError("c_map must have at least one dimension.")
        if smooth_sigma is not None:
            sigma = np.asarray(smooth_sigma, dtype=float)
            if sigma.ndim == 0:
                sigma = np.full(values.ndim, float(sigma))
            if sigma.shape != (values.ndim,):
                raise ValueError(f"smooth_sigma must be scalar or length {values.ndim}, got shape {sigma.shape}.")
            if np.any(sigma < 0):
                raise ValueError("smooth_sigma entries must be non-negative.")
            values = ndimage.gaussian_filter(values, sigma=tuple(float(s) for s in sigma), mode=boundary)
        if method == "linear":
            coeffs = values
        elif method == "bspline3":
            coeffs = ndimage.spline_filter(values, order=3, mode=boundary)
        else:
            raise ValueError("method must be 'linear' or 'bspline3'.")
        d = values.ndim
        sp = np.asarray(spacing if spacing is not None else (1.0,) * d, dtype=float)
        org = np.asarray(origin if origin is not None else (0.0,) * d, dtype=float)
        if sp.shape != (d,):
            raise ValueError(f"spacing must be length {d}, got shape {sp.shape}.")
        if org.shape != (d,):
            raise ValueError(f"origin must be length {d}, got shape {org.shape}.")
        if not np.all(np.isfinite(sp)) or np.any(sp <= 0):
            raise ValueError("spacing entries must be finite and strictly positive.")
        if not np.all(np.isfinite(org)):
            raise ValueError("origin entries must be finite.")
        self.values = values
        self.coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        self.method = method
        self.boundary = boundary
        self.spacing = sp
        self.origin = org

    @property
    def ndim(self) -> int:
        return self.coeffs.ndim

    def sample_nodes(self, N, dx):
        """Values at the grid nodes k * dx (k = 0 .. N - 1) when those are the
        interpolant's own nodes, else None.  At a node the cubic B-spline
        weights are (1, 4, 1) / 6 and the linear ones (0, 1), so the samples
        are a separable 3-tap filter of the coefficients (same boundary
        rule): O(N) instead of 4^d taps per point."""
        from scipy import ndimage

        if (tuple(self.coeffs.shape) != tuple(N) or np.any(self.origin != 0.0)
                or np.any(self.spacing != np.asarray(dx, dtype=float))):
            return None
        if self.method == "linear":
            return self.coeffs.copy()
        out = self.coeffs
        for ax in range(self.ndim):
            if out.shape[ax] > 1:
                out = ndimage.correlate1d(out, np.array([1.0, 4.0, 1.0]) / 6.0, axis=ax, mode=self.boundary)
        return out

    def _map(self, idx, n):
        if n == 1:
            return np.zeros_like(idx)
        b = self.boundary
        if b == "nearest":
            return np.clip(idx, 0, n - 1)
        if b == "wrap":
            return np.mod(idx, n)
        if b == "reflect":
            r = np.mod(idx, 2 * n)
            return np.where(r < n, r, 2 * n - 1 - r)
        per = 2 * n - 2
        r = np.mod(idx, per)
        return np.where(r < n, r, per - r)

    def __call__(self, coords):
        """Host evaluation at physical coordinates (..., d)."""
        x = (np.asarray(coords, dtype=float) - self.origin) / self.spacing
        if x.ndim == 0 or x.shape[-1] != self.ndim:
            raise ValueError(f"coords must have final dimension {self.ndim}; got shape {x.shape}.")
        i0 = np.floor(x)
        t = x - i0
        if self.method == "linear":
            w = np.stack([1.0 - t, t], -1)
            offs = (0, 1)
        else:
            omt, t2 = 1.0 - t, t * t
            t3 = t2 * t
            w = np.stack([omt ** 3 / 6.0, (3 * t3 - 6 * t2 + 4) / 6.0, (-3 * t3 + 3 * t2 + 3 * t + 1) / 6.0,
                          t3 / 6.0], -1)
            offs = (-1, 0, 1, 2)
        acc = np.zeros(x.shape[:-1])
        n = len(offs)
        for corner in range(n ** self.ndim):
            rem, wt, gi = corner, np.ones(x.shape[:-1]), []
            for ax in range(self.ndim):
                k = rem % n
                rem //= n
                gi.append(self._map(i0[..., ax].astype(np.int64) + offs[k], self.coeffs.shape[ax]))
                wt = wt * w[..., ax, k]
            acc = acc + wt * self.coeffs[tuple(gi)]
        return acc


def make_c_function_from_grid(c_map, spacing=None, origin=None, *, method: str = "linear", boundary: str = "clamp",
                              smooth_sigma=None) -> GridInterpolant:
    """utils/interp.py:158-263."""
    return GridInterpolant(c_map, spacing, origin, method=method, boundary=boundary, smooth_sigma=smooth_sigma)
