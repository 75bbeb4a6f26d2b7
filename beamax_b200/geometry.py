"""Host-side ``Domain`` and ``Sensor`` with the reference's fields and checks.

Restates beamax geometry.py:15-616 (validation messages and ordering
conventions included) as NumPy objects; device copies of sensor positions and
time grids are made by the solver, once per object and device.
"""

from __future__ import annotations

from typing import Callable, Optional, Tuple, Union

import numpy as np

Param = Optional[Union[Callable, float, int, np.ndarray]]


class Domain:
    """Axis-aligned rectangular domain with spacing and medium fields (geometry.py:15-400)."""

    def __init__(self, N: Tuple[int, ...], dx: Tuple[float, ...], periodic: Tuple[bool, ...],
                 cfl: float = 0.3, c: Param = 1500.0, density: Param = 1.0,
                 alpha_coeff: Param = None, lam: float = 0.0, alpha_power: Param = None) -> None:
        N_values = np.asarray(N)
        if N_values.ndim != 1 or N_values.size == 0:
            raise ValueError("N must contain at least one spatial dimension.")
        if any(isinstance(n, (bool, np.bool_)) or not isinstance(n, (int, np.integer)) for n in N_values):
            raise ValueError(f"N entries must be integers; got {N}.")
        N = tuple(int(n) for n in N_values)
        if any(n <= 0 for n in N):
            raise ValueError(f"N entries must be positive; got {N}.")
        if len(dx) != len(N):
            raise ValueError(f"dx must have length {len(N)}, got {len(dx)}.")
        dx_arr = np.asarray(dx, dtype=float)
        if not np.all(np.isfinite(dx_arr)) or np.any(dx_arr <= 0):
            raise ValueError(f"dx entries must be finite and positive; got {dx}.")
        if len(periodic) != len(N):
            raise ValueError(f"periodic must have length {len(N)}, got {len(periodic)}.")
        if any(not isinstance(p, (bool, np.bool_)) for p in periodic):
            raise ValueError(f"periodic entries must be boolean; got {periodic}.")
        if not np.isfinite(cfl) or cfl <= 0:
            raise ValueError(f"cfl must be finite and positive; got {cfl}.")
        if not np.isfinite(lam) or lam < 0:
            raise ValueError(f"lam must be finite and non-negative; got {lam}.")

        def _validate(name, value, *, allow_none, strictly_positive):
            if value is None:
                if allow_none:
                    return None
                raise ValueError(f"{name} cannot be None.")
            if callable(value):
                return value
            arr = np.asarray(value)
            if arr.ndim != 0 and tuple(arr.shape) != N:
                raise ValueError(f"{name} must be scalar, callable, or have shape {N}; got {arr.shape}.")
            if not np.all(np.isfinite(arr)):
                raise ValueError(f"{name} must contain only finite values.")
            if strictly_positive and np.any(arr <= 0):
                raise ValueError(f"{name} must be strictly positive.")
            if not strictly_positive and np.any(arr < 0):
                raise ValueError(f"{name} must be non-negative.")
            return value if arr.ndim == 0 else np.asarray(value, dtype=float)

        self.N = N
        self.dx = tuple(float(x) for x in dx_arr)
        self.periodic = tuple(bool(p) for p in periodic)
        self.cfl = float(cfl)
        self.c = _validate("c", c, allow_none=False, strictly_positive=True)
        self.density = _validate("density", density, allow_none=True, strictly_positive=True)
        self.alpha_coeff = _validate("alpha_coeff", alpha_coeff, allow_none=True, strictly_positive=False)
        self.lam = float(lam)
        self.alpha_power = _validate("alpha_power", alpha_power, allow_none=True, strictly_positive=False)

    # geometry.py:226-283
    @property
    def grid_size(self) -> np.ndarray:
        return np.asarray(self.N) * np.asarray(self.dx)

    @property
    def xmax(self) -> float:
        return float(np.linalg.norm(self.grid_size))

    @property
    def k_max(self) -> float:
        return float(np.pi * np.min(1 / np.asarray(self.dx)))

    @property
    def ndim(self) -> int:
        return len(self.N)

    @property
    def grid(self) -> np.ndarray:
        return np.stack(self.generate_meshgrid()[0], axis=-1)

    def _eval(self, p):
        from .utils.interp import GridInterpolant

        if p is None:
            return None
        if isinstance(p, GridInterpolant):
            nodes = p.sample_nodes(self.N, self.dx)
            if nodes is not None:
                return nodes
        arr = np.asarray(p(self.grid) if callable(p) else p, dtype=float)
        if arr.ndim == 0:
            arr = np.broadcast_to(arr, self.N)
        elif tuple(arr.shape) != self.N:
            raise ValueError(f"Medium field evaluated to shape {arr.shape}; expected {self.N}.")
        return arr

    @property
    def sound_speed_array(self) -> np.ndarray:
        """c on the grid; evaluated once per sound-speed object (a 3D cubic
        interpolant takes seconds to sample at 128^3 points)."""
        cached = getattr(self, "_c_grid_cache", None)
        if cached is not None and cached[0] is self.c:
            return cached[1]
        arr = self._eval(self.c)
        self._c_grid_cache = (self.c, arr)
        return arr

    @property
    def density_array(self):
        return self._eval(self.density)

    def compute_max_speed(self) -> float:
        return float(np.max(self.sound_speed_array))

    def compute_min_speed(self) -> float:
        return float(np.min(self.sound_speed_array))

    def compute_max_freq(self) -> float:
        return self.compute_max_speed() / (2 * min(self.dx))

    def generate_meshgrid(self):
        """geometry.py:352-374: spatial 0..(N-1)*dx and Fourier -N//2..N//2-1."""
        sp = [np.arange(0, self.N[i], 1) * self.dx[i] for i in range(self.ndim)]
        fr = [np.arange(-self.N[i] // 2, self.N[i] // 2, 1) for i in range(self.ndim)]
        return np.meshgrid(*sp, indexing="ij"), np.meshgrid(*fr, indexing="ij")

    def generate_time_domain(self) -> np.ndarray:
        """geometry.py:387-400: ``arange(0, ||L|| / c_min, cfl * min(dx) / c_max)``."""
        dt = self.cfl * min(self.dx) / self.compute_max_speed()
        tmax = self.xmax / self.compute_min_speed()
        return np.arange(0, tmax, dt)

    def medium(self):
        """The sound speed as the GPU propagator sees it.

        Returns ``("constant", c)`` for a homogeneous medium and
        ``("grid", interpolant)`` for a grid-valued speed (n-linear, wrap
        boundary when every axis is periodic, clamp otherwise, as
        geometry.py:191-203) or a ``GridInterpolant``.  Any other callable
        c(x) (geometry.py:176-190 accepts one) is sampled once at the grid
        nodes on the host and interpolated by the cubic B-spline of those
        samples (same boundary rule): it equals c at every node and carries
        the continuous gradient and Hessian the ray and Riccati equations
        need; between nodes it differs from c by the interpolation error of
        the samples.  The interpolant is built once per value of ``c`` and
        reused, so the device caches and the kept trajectories key on one
        object.
        """
        from .utils.interp import GridInterpolant, make_c_function_from_grid

        c = self.constant_speed()
        if c is not None:
            return "constant", c
        if isinstance(self.c, GridInterpolant):
            return "grid", self.c
        cached = getattr(self, "_medium_cache", None)
        if cached is not None and cached[0] is self.c:
            return "grid", cached[1]
        boundary = "wrap" if all(self.periodic) else "clamp"
        if not callable(self.c):
            interp = make_c_function_from_grid(np.asarray(self.c, float), spacing=self.dx,
                                               origin=(0.0,) * self.ndim, boundary=boundary)
        else:
            interp = make_c_function_from_grid(np.asarray(self.sound_speed_array, float), spacing=self.dx,
                                               origin=(0.0,) * self.ndim, method="bspline3", boundary=boundary)
        self._medium_cache = (self.c, interp)
        return "grid", interp

    def constant_speed(self) -> Optional[float]:
        """The sound speed when the medium is homogeneous, else ``None``.
        A grid interpolant is constant exactly when its grid values are (both
        n-linear and B-spline interpolation reproduce constants), which is
        checked on the values without evaluating the interpolant."""
        from .utils.interp import GridInterpolant

        if isinstance(self.c, GridInterpolant):
            v = float(self.c.values.flat[0])
            return v if np.all(self.c.values == v) else None
        if callable(self.c):
            arr = self.sound_speed_array
            v = float(arr.flat[0])
            return v if np.all(arr == v) else None
        arr = np.asarray(self.c, dtype=float)
        if arr.ndim == 0:
            return float(arr)
        v = float(arr.flat[0])
        return v if np.all(arr == v) else None


class Sensor:
    """Receiver geometry from positions or a binary mask (geometry.py:403-616)."""

    def __init__(self, domain: Domain, positions=None, binary_mask=None) -> None:
        if positions is None and binary_mask is None:
            raise ValueError("Either positions or binary_mask must be provided")
        if positions is not None and binary_mask is not None:
            raise ValueError("Cannot provide both positions and binary_mask")
        self.domain = domain
        if positions is not None:
            positions = self._normalize_positions(positions)
            self._positions = positions
            self._binary_mask = self._positions_to_mask(positions)
        else:
            binary_mask = self._normalize_mask(binary_mask)
            self._binary_mask = binary_mask
            self._positions = self._mask_to_positions(binary_mask)

    def _normalize_positions(self, positions) -> np.ndarray:
        positions = np.asarray(positions, dtype=float)
        if positions.ndim == 1:
            positions = positions[None, :]
        if positions.ndim != 2 or positions.shape[1] != self.domain.ndim:
            raise ValueError("positions must have shape (Ns, ndim) or (ndim,), "
                             f"got {positions.shape} for ndim={self.domain.ndim}.")
        if not np.all(np.isfinite(positions)):
            raise ValueError("positions must contain only finite values.")
        upper = np.asarray(self.domain.grid_size)
        if np.any(positions < 0) or np.any(positions >= upper):
            raise ValueError("positions must lie inside the half-open domain [0, N*dx).")
        idx = np.rint(positions / np.asarray(self.domain.dx)).astype(int)
        idx = np.clip(idx, 0, np.asarray(self.domain.N) - 1)
        if np.unique(idx, axis=0).shape[0] != idx.shape[0]:
            raise ValueError("positions must map to distinct grid points after quantisation.")
        return positions

    def _normalize_mask(self, mask) -> np.ndarray:
        mask = np.asarray(mask)
        if tuple(mask.shape) != tuple(self.domain.N):
            raise ValueError(f"binary_mask must have shape {self.domain.N}, got {mask.shape}.")
        if not np.all(np.isfinite(mask)):
            raise ValueError("binary_mask must contain only finite values.")
        if not np.all((mask == 0) | (mask == 1)):
            raise ValueError("binary_mask must contain only binary values 0 and 1.")
        if not bool(np.any(mask == 1)):
            raise ValueError("binary_mask must contain at least one positive active entry.")
        return mask

    def _positions_to_mask(self, positions) -> np.ndarray:
        idx = np.round(positions / np.asarray(self.domain.dx)).astype(int)
        idx = np.clip(idx, 0, np.asarray(self.domain.N) - 1)
        mask = np.zeros(self.domain.N)
        mask[tuple(idx.T)] = 1
        return mask

    def _mask_to_positions(self, mask) -> np.ndarray:
        """Row-major order of ``where(mask > 0)`` times dx (geometry.py:575-590)."""
        idx = np.nonzero(np.asarray(mask) > 0)
        return np.stack(idx, axis=1) * np.asarray(self.domain.dx)

    @property
    def positions(self) -> np.ndarray:
        return self._positions

    @property
    def binary_mask(self) -> np.ndarray:
        return self._binary_mask
