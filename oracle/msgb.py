"""FP64 NumPy restatement of the reference MSGB forward path (test oracle).

Test infrastructure: only ``tests/``, ``__graft_entry__.smoke`` and
``bench.py``'s CPU legs use this module, as the checker.

Every function cites the reference file:line it restates (paths relative to
the beamax project root).  The restatement keeps the reference's operation
order where that order is visible in the source, so that FP64 results agree to
round-off.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Optional, Sequence, Tuple, Union

import numpy as np

# --------------------------------------------------------------------------
# utils/fft.py:5-72
# --------------------------------------------------------------------------


def unitary_fft(arr: np.ndarray) -> np.ndarray:
    """``fftshift(fftn(arr, norm="ortho"))`` (utils/fft.py:5-20)."""
    return np.fft.fftshift(np.fft.fftn(arr, norm="ortho"))


def unitary_ifft(arr: np.ndarray) -> np.ndarray:
    """``ifftn(ifftshift(arr), norm="ortho")`` (utils/fft.py:23-38)."""
    return np.fft.ifftn(np.fft.ifftshift(arr), norm="ortho")


def convert_space(array, input_space: str, target_space: str):
    """utils/fft.py:41-72."""
    if input_space == target_space:
        return array
    if input_space == "spatial" and target_space == "fourier":
        return unitary_fft(array)
    if input_space == "fourier" and target_space == "spatial":
        return unitary_ifft(array)
    raise ValueError("Invalid conversion.")


# --------------------------------------------------------------------------
# utils/arrays.py:237-289
# --------------------------------------------------------------------------


def extract_centered_box(arr: np.ndarray, box_shape, center) -> np.ndarray:
    """Wrap-around gather of a centred box (utils/arrays.py:237-268)."""
    S = arr.shape
    c = np.asarray(center, dtype=np.int64)
    half = np.asarray([m // 2 for m in box_shape], dtype=np.int64)
    starts = (c - half) % np.asarray(S)
    out = arr
    for axis in range(arr.ndim):
        idx = (starts[axis] + np.arange(int(box_shape[axis]))) % S[axis]
        out = np.take(out, idx, axis=axis)
    return out


def rel_l2(a, b) -> float:
    """``||a-b|| / (||a|| + 1e-30)`` (utils/arrays.py:271-289)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / (np.linalg.norm(a) + 1e-30))


# --------------------------------------------------------------------------
# decomposition.py
# --------------------------------------------------------------------------


def _is_integral(value) -> bool:
    """decomposition.py:28-36."""
    if isinstance(value, (bool, np.bool_)):
        return False
    if isinstance(value, (int, np.integer)):
        return True
    if isinstance(value, (float, np.floating)):
        return bool(np.isfinite(value) and float(value).is_integer())
    return False


def validate_params(num_levels, N, num_boxes_levels, box_aspect_ratio,
                    boxes_per_dim_levels=None) -> None:
    """decomposition.py:89-215 (the same checks, in the same order)."""
    if not isinstance(num_levels, int) or num_levels < 1:
        raise ValueError(f"num_levels must be positive int; got {num_levels}.")
    if not N or any(not _is_integral(x) for x in N):
        raise ValueError(f"N entries must be integers; got {N}.")
    N = tuple(int(x) for x in N)
    if any(n <= 0 for n in N):
        raise ValueError(f"N must be positive; got {N}.")
    if not all(n % 2 == 0 for n in N):
        raise ValueError(f"N must be even along all axes; got {N}.")
    ndim = len(N)
    if any(not _is_integral(x) for x in box_aspect_ratio):
        raise ValueError("box_aspect_ratio entries must be integers.")
    bar = tuple(int(x) for x in box_aspect_ratio)
    if len(bar) != ndim:
        raise ValueError(f"len(box_aspect_ratio)={len(bar)} != ndim={ndim}.")
    if any(x <= 0 for x in bar):
        raise ValueError("box_aspect_ratio must be positive.")
    if not any(x == 1 for x in bar):
        raise ValueError("At least one aspect ratio component must equal 1.")
    nbl = tuple(int(x) for x in num_boxes_levels)
    if len(nbl) != num_levels:
        raise ValueError("len(num_boxes_levels) != num_levels.")
    if any(x <= 0 for x in nbl):
        raise ValueError("num_boxes_levels must be positive.")
    if any(nbl[i] > nbl[i + 1] for i in range(num_levels - 1)):
        raise ValueError("num_boxes_levels must be non-decreasing with level.")
    if boxes_per_dim_levels is None:
        scale = np.asarray(N, float) / float(min(N)) / np.asarray(bar, float)
        for boxes in nbl:
            counts = boxes * scale
            if not np.allclose(counts, np.rint(counts), rtol=0.0, atol=1e-12):
                raise ValueError("Derived boxes per axis are non-integral.")
    N_ref = min(N)
    base = nbl[0]
    if base <= 0 or base > N_ref:
        raise ValueError(f"Invalid base boxes per side: {base} for N_ref={N_ref}.")
    max_levels = int(math.floor(math.log2(N_ref // base)) + 1)
    if not (1 <= num_levels <= max_levels):
        raise ValueError(f"num_levels must be in [1, {max_levels}].")
    box_lengths = [N_ref // (nbl[-1] * (2 ** L)) for L in range(num_levels - 1, -1, -1)]
    if any(L < 2 for L in box_lengths):
        raise ValueError(
            "Every box length must be at least 2 Fourier samples so the "
            f"Gaussian width is positive; computed {box_lengths} for N_ref={N_ref}."
        )
    if any(N_ref % L != 0 for L in box_lengths):
        raise ValueError(f"Box lengths must divide N_ref={N_ref}; computed {box_lengths}.")


class Decomp:
    """Restatement of ``DyadicDecomposition`` (decomposition.py:218-541)."""

    def __init__(self, num_levels, N, num_boxes_levels, box_aspect_ratio,
                 boxes_per_dim_levels=None):
        validate_params(num_levels, N, num_boxes_levels, box_aspect_ratio,
                        boxes_per_dim_levels)
        self.num_levels = int(num_levels)
        self.N = tuple(int(x) for x in N)
        self.num_boxes_levels = tuple(int(x) for x in num_boxes_levels)
        self.box_aspect_ratio = tuple(int(x) for x in box_aspect_ratio)
        self.boxes_per_dim_levels = boxes_per_dim_levels
        nb = self._num_boxes()
        self.num_boxes_ndim = np.asarray(nb, dtype=np.int64)
        self.centres_ndim = self._centres(nb).astype(np.int64)
        self.total_num_boxes = int(self.num_boxes_ndim.sum())

    @property
    def ndim(self):
        return len(self.N)

    @property
    def num_boxes_ndim_cumsum(self):
        return np.cumsum(self.num_boxes_ndim)

    @property
    def fourier_meshgrid(self):
        """decomposition.py:343-354."""
        axes = [np.arange(-n // 2, n // 2) for n in self.N]
        return np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)

    @property
    def box_lengths(self):
        """decomposition.py:370-386."""
        N_ref = min(self.N)
        return np.asarray([N_ref // (self.num_boxes_levels[-1] * 2 ** L)
                           for L in range(self.num_levels - 1, -1, -1)], dtype=np.int64)

    def _outer(self, lvl):
        """decomposition.py:390-423."""
        if self.boxes_per_dim_levels is not None:
            return np.asarray(self.boxes_per_dim_levels[lvl], dtype=np.int64)
        aspect = np.asarray(self.N, float) / float(min(self.N))
        per = self.num_boxes_levels[lvl] * aspect / np.asarray(self.box_aspect_ratio, float)
        return np.rint(per).astype(np.int64)

    def _num_boxes(self):
        """decomposition.py:425-452."""
        totals, cut = [], []
        for L in range(self.num_levels):
            t = int(np.prod(self._outer(L)))
            totals.append(t)
            cut.append(t // (2 ** self.ndim) if L < self.num_levels - 1 else 0)
        return [totals[0]] + [totals[i] - cut[i - 1] for i in range(1, self.num_levels)]

    def _centres(self, nb):
        """decomposition.py:454-541."""
        bar = self.box_aspect_ratio
        bls = [int(x) for x in self.box_lengths]
        out = []
        bounds_prev = np.zeros(self.ndim, dtype=np.int64)
        for lvl in range(self.num_levels):
            step_len = bls[lvl]
            counts = self._outer(lvl)
            per_axis = []
            for ax in range(self.ndim):
                step = step_len * bar[ax]
                half = int(counts[ax]) // 2
                per_axis.append(np.arange(-half * step + step // 2, half * step, step))
            mesh = np.stack(np.meshgrid(*per_axis, indexing="ij"), -1).reshape(-1, self.ndim)
            if mesh.size > 0 and np.any(bounds_prev > 0):
                keep = ~np.all(np.abs(mesh) < bounds_prev, axis=1)
                mesh = mesh[keep]
            if mesh.shape[0] != nb[lvl]:
                raise ValueError("centre count mismatch")
            out.append(mesh)
            if mesh.shape[0] > 0:
                bounds_prev = np.max(np.abs(mesh), axis=0) + step_len // 2
        return np.concatenate(out, axis=0)

    def find_level(self, box):
        """utils/coeff_index.py:90-108 (searchsorted, side='right')."""
        return np.searchsorted(self.num_boxes_ndim_cumsum, box, side="right")


# --------------------------------------------------------------------------
# transforms.py
# --------------------------------------------------------------------------


def windowed_gaussian(centre, meshgrid, box_length, bar, N, redundancy, windowing):
    """transforms.py:36-96 (compute_windowed_gaussian)."""
    bar = np.asarray(bar)
    Nf = np.asarray(N)
    sigma = (int(box_length) // 2) * bar
    diff = (meshgrid - centre + Nf / 2) % Nf - Nf / 2
    g = np.exp(-np.sum(np.square(diff / sigma), axis=-1))
    if windowing == "none":
        return g
    ws = box_length * bar * (redundancy / 2)
    if windowing == "rectangular":
        w = np.all((-ws <= diff) & (diff < ws), axis=-1)
    elif windowing == "rectangular_mirror":
        w = np.all(np.abs(diff) < ws, axis=-1)
    else:
        raise ValueError(f"Invalid windowing function: {windowing}")
    return g * w.astype(float)


def validate_transform(redundancy, windowing):
    """transforms.py:22-33."""
    if redundancy not in (1, 2):
        raise ValueError(f"redundancy must be 1 or 2; got {redundancy}.")
    if windowing not in ("none", "rectangular", "rectangular_mirror"):
        raise ValueError(f"Unknown windowing mode {windowing!r}.")
    if redundancy == 1 and windowing == "rectangular_mirror":
        raise ValueError("redundancy=1 with windowing='rectangular_mirror' leaves uncovered bins")


def filter_idx(dec: Decomp, box, redundancy, windowing):
    """transforms.py:99-138 (single_filter_idx)."""
    lvl = int(dec.find_level(box))
    return windowed_gaussian(dec.centres_ndim[box], dec.fourier_meshgrid,
                             dec.box_lengths[lvl], dec.box_aspect_ratio, dec.N,
                             redundancy, windowing)


def compute_frame_phase(dec: Decomp, boxidx, k, redundancy):
    """transforms.py:193-226."""
    boxidx = np.asarray(boxidx)
    level = dec.find_level(boxidx)
    bl = dec.box_lengths[level]
    if np.ndim(bl) > 0:
        bl = bl[..., None]
    support = bl * redundancy * np.asarray(dec.box_aspect_ratio)
    half = support // 2
    centre = dec.centres_ndim[boxidx]
    parity = (centre + np.asarray(dec.N) // 2) // half
    sign = 1 - 2 * (parity & 1)
    rolls = sign * (half // 2)
    cycles = np.sum((centre - rolls) * np.asarray(k) / support, axis=-1)
    cycles = np.remainder(cycles, 1.0)
    return np.exp(2 * np.pi * 1j * cycles)


def compute_frames(dec: Decomp, boxidx, k, fourier_space, redundancy, windowing):
    """transforms.py:309-354 (frame atom in Fourier space)."""
    lvl = int(dec.find_level(boxidx))
    support = dec.box_lengths[lvl] * redundancy * np.asarray(dec.box_aspect_ratio)
    g = filter_idx(dec, boxidx, redundancy, windowing)
    scaled = np.einsum("...d,d->...", fourier_space, np.asarray(k) / support)
    norm = float(np.prod(support)) ** (-0.5)
    ph = compute_frame_phase(dec, boxidx, k, redundancy)
    return norm * ph * np.exp(-2 * np.pi * 1j * scaled) * g


class Wpt:
    """Restatement of ``MSWPT`` (transforms.py:357-912)."""

    def __init__(self, dec: Decomp, redundancy: int, windowing: str):
        validate_transform(redundancy, windowing)
        self.dyadic_decomp = dec
        self.redundancy = redundancy
        self.windowing = windowing
        mesh = dec.fourier_meshgrid
        ssq = np.zeros(dec.N)
        Nv0 = np.asarray(dec.N)
        sup = [dec.box_lengths[l] * np.asarray(dec.box_aspect_ratio) * redundancy for l in range(dec.num_levels)]
        if windowing != "none" and all(np.all(s <= Nv0) for s in sup):
            # Windowed filters vanish outside their box's support patch, so the
            # full-grid sum (transforms.py:511-555) only receives +0.0 elsewhere;
            # accumulating over the patches alone gives the same values.
            for i in range(dec.total_num_boxes):
                lvl = int(dec.find_level(i))
                S = sup[lvl]
                c = dec.centres_ndim[i]
                j = np.stack(np.meshgrid(*[np.arange(x) for x in S], indexing="ij"), -1)
                kg = (c + Nv0 // 2 - S // 2 + j) % Nv0
                g = windowed_gaussian(c, kg - Nv0 // 2, dec.box_lengths[lvl], dec.box_aspect_ratio, dec.N,
                                      redundancy, windowing)
                ssq[tuple(np.moveaxis(kg, -1, 0))] += np.square(g)
        else:
            for i in range(dec.total_num_boxes):
                ssq = ssq + np.square(filter_idx(dec, i, redundancy, windowing))
        if not np.all(np.isfinite(ssq)) or not np.all(ssq > 0):
            raise ValueError("The dyadic decomposition leaves uncovered Fourier bins.")
        self.sum_gsquare = ssq
        self.boxes_cumsum = tuple([0] + [int(x) for x in dec.num_boxes_ndim_cumsum])
        bar = np.asarray(dec.box_aspect_ratio)
        self.coeff_shapes = tuple(
            tuple([int(dec.num_boxes_ndim[l])] + [int(x) for x in bar * redundancy * dec.box_lengths[l]])
            for l in range(dec.num_levels))
        cs = [0]
        for sh in self.coeff_shapes:
            cs.append(cs[-1] + int(np.prod(sh)))
        self.coeffs_cumsum = tuple(cs)
        self.total_coeffs = cs[-1]
        self.box_shapes = [tuple(int(x) for x in (dec.box_lengths[l] * bar * redundancy / 2).astype(int))
                           for l in range(dec.num_levels)]
        self.support_shapes = [tuple(2 * x for x in bs) for bs in self.box_shapes]
        seg = [cs[i + 1] - cs[i] for i in range(dec.num_levels)]
        self.half_mask = np.concatenate(
            [np.concatenate([np.ones(L // 2), np.zeros(L - L // 2)]) for L in seg])
        Nv = np.asarray(dec.N)
        cen = dec.centres_ndim + Nv // 2
        self.gfilts_packed = []
        for l in range(dec.num_levels):
            start = self.boxes_cumsum[l]
            g = filter_idx(dec, start, redundancy, windowing)
            self.gfilts_packed.append(extract_centered_box(g, self.support_shapes[l], cen[start]))
        del mesh

    # transforms.py:591-694 plus 696-733
    def _fwd_rolls(self, level, centre_shifted):
        bhs = np.asarray(self.box_shapes[level])
        ri = (centre_shifted + np.asarray(self.dyadic_decomp.N) // 2) // bhs
        sign = 1 - 2 * (ri & 1)
        return sign * (bhs // 2)

    def forward(self, data, input_type="spatial"):
        """MSWPT.forward (transforms.py:696-733, _compute_coeffs 591-694)."""
        if self.windowing == "none":
            raise ValueError("MSWPT.forward does not support windowing='none'")
        dec = self.dyadic_decomp
        ft = convert_space(np.asarray(data), input_type, "fourier") / self.sum_gsquare
        Nv = np.asarray(dec.N)
        cen = dec.centres_ndim + Nv // 2
        axes = tuple(range(dec.ndim))
        out = np.zeros(self.total_coeffs, dtype=np.complex128)
        for l in range(dec.num_levels):
            s, e = self.boxes_cumsum[l], self.boxes_cumsum[l + 1]
            blk = np.zeros(self.coeff_shapes[l], dtype=np.complex128)
            for i in range(e - s):
                c = cen[s + i]
                patch = extract_centered_box(ft, self.support_shapes[l], c)
                sf = self.gfilts_packed[l] * patch
                sf = np.roll(sf, tuple(int(r) for r in self._fwd_rolls(l, c)), axis=axes)
                blk[i] = unitary_ifft(sf)
            out[self.coeffs_cumsum[l]:self.coeffs_cumsum[l + 1]] = blk.ravel()
        return out

    def _synth_fourier(self, coeffs, rolls_kind):
        """Fourier-domain accumulation shared by inverse and the Hermitian adjoint.

        ``rolls_kind='inverse'`` uses the inverse's roll convention
        (transforms.py:822-824: ``(centre + N//2) // box_len``);
        ``'forward'`` uses the forward's (transforms.py:626,666:
        ``(centre + N//2 + N//2) // box_len``), as the exact adjoint needs.
        """
        dec = self.dyadic_decomp
        Nv = np.asarray(dec.N)
        ft = np.zeros(dec.N, dtype=np.complex128)
        for l in range(dec.num_levels):
            s, e = self.boxes_cumsum[l], self.boxes_cumsum[l + 1]
            S = np.asarray(self.support_shapes[l])
            blk = np.asarray(coeffs[self.coeffs_cumsum[l]:self.coeffs_cumsum[l + 1]]).reshape(self.coeff_shapes[l])
            bl = np.asarray(self.box_shapes[l])
            for i in range(e - s):
                centre = dec.centres_ndim[s + i]
                if rolls_kind == "inverse":
                    ri = (centre + Nv // 2) // bl
                else:
                    ri = (centre + Nv // 2 + Nv // 2) // bl
                rolls = (1 - 2 * (ri & 1)) * (bl // 2)
                fh = unitary_fft(blk[i])
                un = fh
                for ax in range(dec.ndim):
                    idx = (np.arange(S[ax]) + rolls[ax]) % S[ax]
                    un = np.take(un, idx, axis=ax)
                contrib = self.gfilts_packed[l] * un
                c0 = (centre + Nv // 2) % Nv
                starts = (c0 - S // 2) % Nv
                grids = np.meshgrid(*[(starts[k] + np.arange(S[k])) % Nv[k] for k in range(dec.ndim)],
                                    indexing="ij")
                np.add.at(ft, tuple(grids), contrib)
        return ft

    def inverse(self, coeffs, output_type="spatial"):
        """MSWPT.inverse (transforms.py:735-850)."""
        ft = self._synth_fourier(coeffs, "inverse")
        return convert_space(ft, "fourier", output_type)

    def adjoint(self, coeffs, output_type="spatial"):
        """Hermitian adjoint of ``forward`` (spatial input), complex output.

        forward = unitary_ifft per box o roll(+r) o (g *) o extract o (/ sum g^2)
        o unitary_fft.  Each factor's adjoint is taken in reverse order:
        unitary_ifft^H = unitary_fft, roll(+r)^H = roll(-r), extract^H =
        periodic scatter-add, (/ sum g^2) and (g *) are real diagonal,
        unitary_fft^H = unitary_ifft.
        """
        ft = self._synth_fourier(coeffs, "forward") / self.sum_gsquare
        return convert_space(ft, "fourier", output_type)


def compute_gh_filters(dec: Decomp, redundancy, windowing):
    """transforms.py:266-306."""
    g = np.stack([filter_idx(dec, i, redundancy, windowing) for i in range(dec.total_num_boxes)])
    ssq = np.sum(g ** 2, axis=0)
    return g, g / ssq


# --------------------------------------------------------------------------
# utils/coeff_index.py
# --------------------------------------------------------------------------


def coeff_shapes(wpt: Wpt):
    return np.asarray(wpt.coeff_shapes, dtype=np.int64)


def find_tensor_and_multiindex(flat, shapes):
    """utils/coeff_index.py:111-147.  Returns (level, (1+d, m) multi-index)."""
    flat = np.asarray(flat, dtype=np.int64)
    prods = np.prod(shapes, axis=1)
    cum = np.cumsum(prods)
    lvl = np.searchsorted(cum, flat, side="right")
    local = np.where(lvl > 0, flat - np.take(cum, np.maximum(lvl - 1, 0)), flat)
    mi = np.zeros((shapes.shape[1], flat.size), dtype=np.int64)
    for j in range(flat.size):
        mi[:, j] = np.unravel_index(int(local[j]), tuple(int(x) for x in shapes[lvl[j]]))
    return lvl, mi


def batch_data(*args, batch_size, zero_padded_args=()):
    """utils/coeff_index.py:29-87."""
    b = args[0].shape[0]
    nb = (b + batch_size - 1) // batch_size
    out = []
    for i, a in enumerate(args):
        pad = nb * batch_size - a.shape[0]
        if pad:
            if i in zero_padded_args:
                p = np.zeros((pad,) + a.shape[1:], dtype=a.dtype)
            else:
                p = np.broadcast_to(a[-1:], (pad,) + a.shape[1:])
            a = np.concatenate([a, p], axis=0)
        out.append(a.reshape((nb, batch_size) + a.shape[1:]))
    return tuple(out)


# --------------------------------------------------------------------------
# geometry.py (minimal Domain)
# --------------------------------------------------------------------------


@dataclass
class Dom:
    """Minimal restatement of ``Domain`` (geometry.py:15-400)."""

    N: Tuple[int, ...]
    dx: Tuple[float, ...]
    periodic: Tuple[bool, ...]
    cfl: float = 0.3
    c: Union[float, Callable, np.ndarray] = 1500.0
    lam: float = 0.0

    @property
    def ndim(self):
        return len(self.N)

    @property
    def grid_size(self):
        return np.asarray(self.N) * np.asarray(self.dx)

    @property
    def grid(self):
        sp = [np.arange(0, self.N[i], 1) * self.dx[i] for i in range(self.ndim)]
        return np.stack(np.meshgrid(*sp, indexing="ij"), axis=-1)

    def c_fn(self, x):
        if callable(self.c):
            return self.c(x)
        v = np.asarray(self.c, dtype=float)
        if v.ndim == 0:
            return v + np.zeros(np.asarray(x).shape[:-1])
        raise NotImplementedError("grid-valued c: use oracle.ode")

    def sound_speed_array(self):
        if callable(self.c):
            return np.asarray(self.c(self.grid))
        v = np.asarray(self.c, dtype=float)
        return np.broadcast_to(v, self.N) if v.ndim == 0 else v

    def generate_time_domain(self):
        """geometry.py:387-400."""
        c = self.sound_speed_array()
        dt = self.cfl * min(self.dx) / np.max(c)
        tmax = np.linalg.norm(self.grid_size) / np.min(c)
        return np.arange(0, tmax, dt)


def sensor_positions_from_mask(dom: Dom, mask) -> np.ndarray:
    """geometry.py:575-590: ``stack(where(mask > 0)) * dx`` (row-major)."""
    idx = np.nonzero(np.asarray(mask) > 0)
    return np.stack(idx, axis=1) * np.asarray(dom.dx)


# --------------------------------------------------------------------------
# solvers/msgb_solvers/forward_solver_utils.py
# --------------------------------------------------------------------------


def threshold_top_n(coeff, val):
    """forward_solver_utils.py:65-89, with JAX's argpartition semantics.

    ``jnp.argpartition(a, k)`` (jax 0.10) is ``top_k(-a, k+1)`` for the bottom
    set (ties: lower index first, i.e. lower index counts as smaller) and the
    remaining rows in index order; ``[-N:]`` therefore keeps the last N keys of
    the ordering (|c| ascending, index ascending), and the stable ``argsort``
    of their magnitudes returns them in that same ascending order.  Net
    contract: sort by (|c|, index) ascending and keep the last N.
    """
    coeff = np.asarray(coeff)
    N = min(int(val), int(coeff.shape[0]))
    if N <= 0:
        raise ValueError("top_n threshold must be a positive integer.")
    key = topn_key(coeff)
    order = np.lexsort((np.arange(coeff.size), key))  # primary key, then index
    idx = order[-N:]
    return idx.astype(np.int64), coeff[idx]


def topn_key(coeff) -> np.ndarray:
    """Magnitude used for selection: ``sqrt(re*re + im*im)``, each step IEEE-rounded.

    ``jnp.abs`` of a complex is a hypot; this form is within one ulp of it and
    is reproduced bit-for-bit by the GPU selector (no FMA contraction).
    """
    c = np.asarray(coeff)
    if np.iscomplexobj(c):
        re = np.ascontiguousarray(c.real)
        im = np.ascontiguousarray(c.imag)
        return np.sqrt(re * re + im * im)
    return np.abs(c)


def threshold_coefficients(coeffs, val, strategy="hard", wpt=None):
    """forward_solver_utils.py:181-230 (hard, top_n, percentile, hard_reassign,
    bao_energy, perc_max_abs at :14-178)."""
    def hard(c):
        idx = np.nonzero(np.abs(c) > val)[0]
        return idx, c[idx]

    def percentile(c):
        thresh = np.percentile(np.abs(c), val)
        mask = np.abs(c) > thresh
        idx = np.full(c.shape[0], -1, dtype=np.int64)
        nz = np.nonzero(mask)[0]
        idx[: nz.size] = nz
        values = np.where(idx >= 0, c[idx], 0.0)
        return idx, values

    def hard_reassign(c):
        max_abs = np.max(np.abs(c))
        thr = np.where((max_abs > 0) & (np.abs(c) >= val * max_abs), c, 0)
        re = np.sum(np.abs(thr) ** 2)
        te = np.sum(np.abs(c) ** 2)
        ratio = np.sqrt(te / (re if re > 0 else 1)) if re > 0 else 0.0
        r = thr * ratio
        idx = np.nonzero(np.abs(r) > 0)[0]
        return idx, r[idx]

    def bao(c):
        if wpt is None:
            raise ValueError("bao_energy thresholding requires wpt.")
        dec = wpt.dyadic_decomp
        sh = coeff_shapes(wpt)
        lvl, mi = find_tensor_and_multiindex(np.arange(c.shape[0]), sh)
        box = mi[0] + np.r_[0, np.cumsum(dec.num_boxes_ndim)][lvl]
        nx = np.linalg.norm(dec.centres_ndim[box], axis=1) ** dec.ndim
        idx = np.nonzero(np.abs(c * nx) > val)[0]
        return idx, c[idx]

    def perc_max(c):
        thresh = np.max(np.abs(c)) * val
        mask = np.abs(c) > thresh
        idx = np.full(c.shape[0], -1, dtype=np.int64)
        nz = np.nonzero(mask)[0]
        idx[: nz.size] = nz
        values = np.where(idx >= 0, c[idx], 0.0)
        return idx, values

    funcs = {"hard": hard, "top_n": lambda c: threshold_top_n(c, val),
             "percentile": percentile, "hard_reassign": hard_reassign,
             "bao_energy": bao, "perc_max_abs": perc_max}
    if strategy not in funcs:
        raise ValueError(f"Invalid thresholding strategy: {strategy}")
    f = funcs[strategy]
    return (f(coeffs[0]), f(coeffs[1])) if isinstance(coeffs, tuple) else f(np.asarray(coeffs))


def coefficient_positions(lvl, mi, wpt: Wpt, dom: Dom):
    """forward_solver_utils.py:233-252."""
    dec = wpt.dyadic_decomp
    local = mi[1:, :].T
    support = dec.box_lengths[lvl][:, None] * np.asarray(dec.box_aspect_ratio) * wpt.redundancy
    return local * dom.grid_size / support


def compute_forward_parameters(idx, wpt: Wpt, dom: Dom, sign=1):
    """forward_solver_utils.py:255-373 (one sign branch, compute_params)."""
    dec = wpt.dyadic_decomp
    gs = dom.grid_size
    bls = dec.box_lengths
    bar = np.asarray(dec.box_aspect_ratio)
    Nv = np.asarray(dom.N)
    lvl, mi = find_tensor_and_multiindex(idx, coeff_shapes(wpt))
    box = mi[0] + np.r_[0, np.cumsum(dec.num_boxes_ndim)][lvl]
    centres = dec.centres_ndim[box, :] / gs
    norm = np.linalg.norm(centres, axis=-1, keepdims=True)
    p0s = 2 * np.pi * centres / norm
    bl = bls[lvl][:, None] / gs * bar
    Lls = bl * wpt.redundancy
    sig = bl / 2
    alphas = 2j * (np.pi * sig) ** 2 / norm
    d = dom.ndim
    M0s = np.einsum("bd,dj->bdj", alphas, np.eye(d))
    a0s = np.prod(np.sqrt((np.pi * gs[None, :]) / (Lls * Nv[None, :])) * sig, axis=1)
    local_k = mi[1:, :].T
    a0s = a0s * compute_frame_phase(dec, box, local_k, wpt.redundancy)
    x0s = coefficient_positions(lvl, mi, wpt, dom)
    om = norm[:, 0]
    modes = sign * np.ones(p0s.shape[0])
    return p0s, M0s, x0s, om, a0s, modes


def compute_coefficients(p0, dpdt, input_type, dom: Dom, wpt: Wpt, mode="both"):
    """forward_solver_utils.py:716-786."""
    a = wpt.forward(p0, input_type)
    b = wpt.forward(dpdt, input_type)
    dec = wpt.dyadic_decomp
    lvl, mi = find_tensor_and_multiindex(np.arange(wpt.total_coeffs), coeff_shapes(wpt))
    xb = coefficient_positions(lvl, mi, wpt, dom)
    box = mi[0] + np.r_[0, np.cumsum(dec.num_boxes_ndim)][lvl]
    pb = 2 * np.pi * dec.centres_ndim[box] / dom.grid_size
    vg = dom.c_fn(xb) * np.linalg.norm(pb, axis=-1)  # G(x, p, mode=1) gb_utils.py:11-41
    cpos = 0.5 * (a + 1j * b / vg)
    if mode == "pos_only":
        return cpos * wpt.half_mask
    if mode == "both":
        return cpos, 0.5 * (a - 1j * b / vg)
    raise ValueError(f"Invalid mode: {mode}")


def effective_top_n(thr, wpt: Wpt, half_frame=False):
    """msgb_solver.py:536-549."""
    if half_frame:
        cap = sum((e - s) // 2 for s, e in zip(wpt.coeffs_cumsum[:-1], wpt.coeffs_cumsum[1:]))
    else:
        cap = wpt.total_coeffs
    return min(int(thr), int(cap))


# --------------------------------------------------------------------------
# gb/gb_solvers.py: closed-form homogeneous propagation
# --------------------------------------------------------------------------


def compute_m_hom_diag(p0, normp, alpha0, c0, ts):
    """gb/gb_solvers.py:306-353 (Sherman-Morrison)."""
    d = p0.shape[1]
    P = p0[:, None, :, None]
    C = c0[:, :, None, None]
    A0 = alpha0[:, None, :, None]
    NP = normp[:, :, None, None]
    T = ts[None, :, None, None]
    eye = np.eye(d)[None, None]
    N0 = A0 * eye
    Ad = 1 + C * T * A0 / NP
    Ainv = (1 / Ad) * eye
    u = -C * T * P / NP ** 3
    vT = np.einsum("btij,btik->btjk", np.broadcast_to(P, (p0.shape[0], 1, d, 1)), np.broadcast_to(N0, (p0.shape[0], 1, d, d)))
    Ainv_u = Ainv @ u
    vT_Ainv = vT @ Ainv
    scalar = 1 + vT_Ainv @ u
    Y = Ainv - (Ainv_u @ vT_Ainv) / scalar
    return N0 @ Y


def compute_amp_hom_diag(p0, normp, alpha0, c0, ts, a0):
    """gb/gb_solvers.py:194-303 (2D formula for d < 3, 3D formula for d == 3)."""
    d = p0.shape[-1]
    if d == 3:
        p1, p2, p3 = p0[:, 0] ** 2, p0[:, 1] ** 2, p0[:, 2] ** 2
        a1, a2, a3 = alpha0[:, 0][:, None], alpha0[:, 1][:, None], alpha0[:, 2][:, None]
        tsc = c0 * ts / normp ** 4
        t1 = c0 * a2 * a3 * ts + (a2 + a3) * normp
        t2 = c0 * a1 * a3 * ts + (a1 + a3) * normp
        t3 = c0 * a1 * a2 * ts + (a1 + a2) * normp
        den = 1 + tsc * (p1[:, None] * t1 + p2[:, None] * t2 + p3[:, None] * t3)
        return a0[:, None] / np.sqrt(den)
    if d < 3:
        ap = np.sum(np.square(p0) * alpha0[:, ::-1], axis=1, keepdims=True) / normp ** 3
        return a0[..., None] / (1 + c0 * ts[None, :] * ap) ** ((d - 1) / 2)
    raise ValueError("Currently only 1D, 2D and 3D are supported.")


def solve_hom_diag(x0, p0, M0, a0, mode, ts, c_const):
    """gb/gb_solvers.py:356-422 with constant c."""
    d = p0.shape[-1]
    nt = ts.shape[0]
    c0 = c_const * np.asarray(mode, float)[..., None]
    normp = np.linalg.norm(p0, axis=-1, keepdims=True)
    xt = x0[:, None, :] + c0[:, None, :] * (p0 / normp)[:, None, :] * ts[None, :, None]
    pt = np.repeat(p0[:, None, :], nt, axis=1)
    alpha0 = np.diagonal(M0, axis1=1, axis2=2)
    Mt = compute_m_hom_diag(p0, normp, alpha0, c0, ts)
    At = compute_amp_hom_diag(p0, normp, alpha0, c0, ts, a0)[:, :, None]
    return xt, pt, Mt, At


# --------------------------------------------------------------------------
# gb/core.py: beam summation
# --------------------------------------------------------------------------


def wrap_position(x, domain_size, periodic):
    """gb/core.py:16-36."""
    return np.where(np.asarray(periodic), x % domain_size, x)


def safe_angle(z, eps=1e-12):
    """gb/core.py:171-191."""
    re = np.real(z)
    im = np.imag(z)
    re = np.where((re == 0) & (im == 0), eps, re)
    return np.arctan2(im, re)


def gaussian_beam_real_sum(xt, pt, Mt, At, omega, sensors, domain_size, periodic):
    """gb/core.py:194-329 (compute_gaussian_beam_real after the ODE)."""
    xt = wrap_position(xt, domain_size, periodic)
    d = sensors.shape[-1]
    sf = sensors.reshape(-1, d)
    nt = xt.shape[1]
    dom = np.asarray(domain_size, float)
    pm = np.asarray(periodic, float)
    acc = np.zeros((nt, sf.shape[0]))
    for b in range(xt.shape[0]):
        Mr = Mt[b].real
        Mi = Mt[b].imag
        A = At[b, :, 0]
        delta = sf[None, :, :] - xt[b][:, None, :]
        delta = delta - dom * np.round(delta / dom) * pm
        phi_lin = np.einsum("tsd,td->ts", delta, pt[b])
        phi_q = 0.5 * np.einsum("tsd,tde,tse->ts", delta, Mr, delta)
        chi = 0.5 * np.einsum("tsd,tde,tse->ts", delta, Mi, delta)
        phase = omega[b] * (phi_lin + phi_q) + safe_angle(A[:, None])
        acc = acc + 2.0 * np.abs(A[:, None]) * np.cos(phase) * np.exp(-omega[b] * chi)
    return acc.reshape((nt,) + sensors.shape[:-1])


def gaussian_beam_complex(xt, pt, Mt, At, omega, sensors, domain_size, periodic):
    """gb/core.py:39-168: complex field per beam, shape (Nt, *S, b)."""
    xt = wrap_position(xt, domain_size, periodic)
    d = sensors.shape[-1]
    sf = sensors.reshape(-1, d)
    dom = np.asarray(domain_size, float)
    diff = sf[None, None] - xt[:, :, None, :]
    diff = np.where(np.asarray(periodic), diff - dom * np.round(diff / dom), diff)
    phase = np.einsum("btd,btsd->bts", pt, diff) + 0.5 * np.einsum("btij,btsi,btsj->bts", Mt, diff, diff)
    gb = At[:, :, 0][:, :, None] * np.exp(1j * omega[:, None, None] * phase)
    out = np.moveaxis(gb, 0, -1)
    return out.reshape((xt.shape[1],) + sensors.shape[:-1] + (xt.shape[0],))


# --------------------------------------------------------------------------
# msgb_solver.py: the forward pipeline and its exact transpose
# --------------------------------------------------------------------------


@dataclass
class Beams:
    """Per selected coefficient beam data (positive branch; the mirror reuses it)."""

    idx: np.ndarray      # (n,) int64 flat coefficient indices
    coeff: np.ndarray    # (n,) complex coefficient values c_pos[idx]
    p0: np.ndarray       # (n, d)
    M0: np.ndarray       # (n, d, d)
    x0: np.ndarray       # (n, d)
    omega: np.ndarray    # (n,)
    a0_unit: np.ndarray  # (n,) complex, before multiplying by the coefficient


def select_beams(p0, dom: Dom, wpt: Wpt, thr, thr_strat="top_n", input_type="spatial", dpdt=None):
    """msgb_solver.py:570-612: coefficients -> threshold -> beam init."""
    if dpdt is None:
        dpdt = np.zeros_like(p0)
    cpos = compute_coefficients(p0, dpdt, input_type, dom, wpt, mode="pos_only")
    t = effective_top_n(thr, wpt, half_frame=True) if thr_strat == "top_n" else thr
    idx, vals = threshold_coefficients(cpos, t, thr_strat, wpt)
    return beams_for(idx, vals, dom, wpt)


def beams_for(idx, vals, dom: Dom, wpt: Wpt) -> Beams:
    p0s, M0s, x0s, om, a0s, _ = compute_forward_parameters(idx, wpt, dom)
    return Beams(np.asarray(idx), np.asarray(vals), p0s, M0s, x0s, om, a0s)


def mirrored_params(bm: Beams):
    """msgb_solver.py:612-619: a0 *= coeff, params duplicated, modes [+1, -1]."""
    a0 = bm.a0_unit * bm.coeff
    cat = lambda a: np.concatenate([a, a])
    n = bm.p0.shape[0]
    modes = np.concatenate([np.ones(n), -np.ones(n)])
    return cat(bm.p0), cat(bm.M0), cat(bm.x0), cat(bm.omega), cat(a0), modes


def forward_hom(bm: Beams, dom: Dom, sensors, ts):
    """Real forward (scan_real, solve_hom_diag) for constant c."""
    p0s, M0s, x0s, om, a0s, modes = mirrored_params(bm)
    xt, pt, Mt, At = solve_hom_diag(x0s, p0s, M0s, a0s, modes, np.asarray(ts, float), float(dom.c))
    return gaussian_beam_real_sum(xt, pt, Mt, At, om, np.asarray(sensors, float),
                                  dom.grid_size, dom.periodic)


def forward(p0, dom: Dom, sensors, ts, wpt: Wpt, thr, thr_strat="top_n", dpdt=None):
    bm = select_beams(np.asarray(p0, float), dom, wpt, thr, thr_strat, dpdt=dpdt)
    return forward_hom(bm, dom, sensors, ts), bm


def beam_kernels_hom(bm: Beams, dom: Dom, sensors, ts):
    """K_b(t, s) with contribution = 2 Re[coeff_b K_b], for both branches.

    Returns (K_plus, K_minus), each (n, Nt, Ns) complex.  For the real field
    ``2|A| cos(w phi + arg A) exp(-w chi) = 2 Re[A exp(i w (phi + i chi))]``
    and ``A(t) = coeff * a0_unit * h(t)``.
    """
    out = []
    n = bm.p0.shape[0]
    sens = np.asarray(sensors, float).reshape(-1, dom.ndim)
    for sgn in (1.0, -1.0):
        xt, pt, Mt, At = solve_hom_diag(bm.x0, bm.p0, bm.M0, bm.a0_unit, sgn * np.ones(n),
                                        np.asarray(ts, float), float(dom.c))
        G = gaussian_beam_complex(xt, pt, Mt, At, bm.omega, sens, dom.grid_size, dom.periodic)
        out.append(np.moveaxis(G, -1, 0))
    return out[0], out[1]


def adjoint_coeff_grad(bm: Beams, dom: Dom, sensors, ts, data):
    """Exact transpose down to the selected coefficients: g_b = sum 2 d conj(K_b)."""
    Kp, Km = beam_kernels_hom(bm, dom, sensors, ts)
    d = np.asarray(data, float).reshape(Kp.shape[1], -1)
    return 2.0 * np.einsum("bts,ts->b", np.conj(Kp) + np.conj(Km), d)


def adjoint(bm: Beams, dom: Dom, sensors, ts, wpt: Wpt, data):
    """Exact transpose of ``forward`` with the selection frozen (real p0)."""
    g = adjoint_coeff_grad(bm, dom, sensors, ts, data)
    G = np.zeros(wpt.total_coeffs, dtype=np.complex128)
    # c_pos = 0.5 * a_coeff * half_mask (dpdt = 0); both factors are real.
    np.add.at(G, bm.idx, 0.5 * g * wpt.half_mask[bm.idx])
    return np.real(wpt.adjoint(G, "spatial"))


def beam_table(bm: Beams, c_const: float):
    """Flat arrays for the C oracle: a0 includes the coefficient."""
    return dict(x0=np.ascontiguousarray(bm.x0, float),
                p0=np.ascontiguousarray(bm.p0, float),
                alpha=np.ascontiguousarray(np.diagonal(bm.M0, axis1=1, axis2=2), np.complex128),
                a0=np.ascontiguousarray(bm.a0_unit * bm.coeff, np.complex128),
                omega=np.ascontiguousarray(bm.omega, float))
