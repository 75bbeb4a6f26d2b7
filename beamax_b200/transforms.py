"""``MSWPT``: the multiscale wave-packet transform, analysis on the GPU.

The constructor builds the reference's static metadata on the host (beamax
transforms.py:423-589: sum of squared filters, coefficient shapes and offsets,
packed per-level filters, conjugate half mask) and, on first use on a CUDA
device, uploads it once into a ``msgb_mswpt`` plan of libmsgb.so.  ``forward``,
``inverse`` and ``adjoint`` run the sm_100a kernels; there is no CPU path.
"""

from __future__ import annotations

import ctypes
from typing import Dict, Tuple

import numpy as np

from . import _lib
from ._device import as_device_f64, workspace
from .decomposition import DyadicDecomposition


def _validate_transform_configuration(redundancy: int, windowing: str) -> None:
    """transforms.py:22-33."""
    if redundancy not in (1, 2):
        raise ValueError(f"redundancy must be 1 or 2; got {redundancy}.")
    if windowing not in ("none", "rectangular", "rectangular_mirror"):
        raise ValueError(f"Unknown windowing mode {windowing!r}.")
    if redundancy == 1 and windowing == "rectangular_mirror":
        raise ValueError("redundancy=1 with windowing='rectangular_mirror' leaves "
                         "uncovered Fourier bins, so the canonical-dual analysis is "
                         "undefined; use windowing='rectangular' or redundancy=2.")


def _gaussian_on_patch(centre, k_grid, box_length, bar, N, redundancy, windowing):
    """compute_windowed_gaussian (transforms.py:36-96) at grid indices ``k_grid``.

    ``k_grid`` holds shifted Fourier indices (meshgrid value = k - N//2).
    """
    bar = np.asarray(bar)
    Nf = np.asarray(N)
    mesh = k_grid - Nf // 2
    sigma = (int(box_length) // 2) * bar
    diff = (mesh - centre + Nf / 2) % Nf - Nf / 2
    g = np.exp(-np.sum(np.square(diff / sigma), axis=-1))
    if windowing == "none":
        return g
    ws = box_length * bar * (redundancy / 2)
    if windowing == "rectangular":
        w = np.all((-ws <= diff) & (diff < ws), axis=-1)
    else:
        w = np.all(np.abs(diff) < ws, axis=-1)
    return g * w.astype(float)


class MSWPT:
    """Multiscale wave-packet transform (transforms.py:357-912)."""

    def __init__(self, dyadic_decomp: DyadicDecomposition, redundancy: int = 2,
                 windowing: str = "rectangular"):
        _validate_transform_configuration(redundancy, windowing)
        self.dyadic_decomp = dyadic_decomp
        self.redundancy = int(redundancy)
        self.windowing = windowing
        dec = dyadic_decomp
        nd = dec.ndim
        bar = np.asarray(dec.box_aspect_ratio)
        Nv = np.asarray(dec.N)
        self.boxes_cumsum = tuple([0] + [int(x) for x in dec.num_boxes_ndim_cumsum])
        self.coeff_shapes = tuple(
            tuple([int(dec.num_boxes_ndim[l])] + [int(x) for x in bar * redundancy * int(dec.box_lengths[l])])
            for l in range(dec.num_levels))
        cs = [0]
        for sh in self.coeff_shapes:
            cs.append(cs[-1] + int(np.prod(sh)))
        self.coeffs_cumsum = tuple(cs)
        self.total_coeffs = int(cs[-1])
        self.max_box_length = int(int(dec.box_lengths[-1]) * max(dec.box_aspect_ratio) * (redundancy / 2))
        self._box_shapes = [tuple(int(x) for x in (int(dec.box_lengths[l]) * bar * redundancy / 2).astype(int))
                            for l in range(dec.num_levels)]
        self._support_shapes = [tuple(2 * x for x in b) for b in self._box_shapes]
        seg = [cs[i + 1] - cs[i] for i in range(dec.num_levels)]
        self._half_mask = np.concatenate(
            [np.concatenate([np.ones(L // 2), np.zeros(L - L // 2)]) for L in seg])
        # Packed per-level filters and sum of squares over every box's support.
        ssq = np.zeros(dec.N)
        self.gfilts_packed = []
        self._box_level = np.repeat(np.arange(dec.num_levels), dec.num_boxes_ndim).astype(np.int32)
        for l in range(dec.num_levels):
            S = np.asarray(self._support_shapes[l])
            s, e = self.boxes_cumsum[l], self.boxes_cumsum[l + 1]
            bl = int(dec.box_lengths[l])
            if np.any(S > Nv) or windowing == "none":
                # Supports that wrap onto themselves (or an untruncated Gaussian):
                # evaluate every filter on the whole grid as the reference does.
                kg = np.stack(np.meshgrid(*[np.arange(n) for n in dec.N], indexing="ij"), -1)
                for b in range(s, e):
                    g = _gaussian_on_patch(dec.centres_ndim[b], kg, bl, bar, dec.N, redundancy, windowing)
                    ssq = ssq + np.square(g)
                    if b == s:
                        self.gfilts_packed.append(self._extract(g, tuple(S), dec.centres_ndim[b] + Nv // 2))
                continue
            j = np.stack(np.meshgrid(*[np.arange(x) for x in S], indexing="ij"), -1)
            for b in range(s, e):
                c = dec.centres_ndim[b]
                kg = (c + Nv // 2 - S // 2 + j) % Nv
                g = _gaussian_on_patch(c, kg, bl, bar, dec.N, redundancy, windowing)
                ssq[tuple(np.moveaxis(kg, -1, 0))] += np.square(g)
                if b == s:
                    self.gfilts_packed.append(g)
        if not np.all(np.isfinite(ssq)) or not np.all(ssq > 0):
            raise ValueError("The dyadic decomposition leaves uncovered Fourier bins; "
                             "choose compatible grid, box counts, and aspect ratios.")
        self.sum_gsquare = ssq
        self.complex_dtype = np.complex128
        self._plans: Dict[int, int] = {}
        self._keep = None

    @staticmethod
    def _extract(arr, shape, centre):
        out = arr
        starts = (np.asarray(centre) - np.asarray([m // 2 for m in shape])) % np.asarray(arr.shape)
        for ax in range(arr.ndim):
            out = np.take(out, (starts[ax] + np.arange(shape[ax])) % arr.shape[ax], axis=ax)
        return out

    # ------------------------------------------------------------ device plan
    def _descriptor(self):
        dec = self.dyadic_decomp
        nd = dec.ndim
        L = dec.num_levels
        goff = np.zeros(L, np.int64)
        gparts, o = [], 0
        for l in range(L):
            goff[l] = o
            gparts.append(np.ascontiguousarray(self.gfilts_packed[l], np.float64).ravel())
            o += gparts[-1].size
        lat_cnt = np.zeros((L, nd), np.int32)
        lat_first = np.zeros((L, nd), np.int32)
        lat_step = np.zeros((L, nd), np.int32)
        lat_off = np.zeros(L, np.int64)
        tables, o = [], 0
        for l in range(L):
            cnt, first, step = dec.lattice(l)
            lat_cnt[l], lat_first[l], lat_step[l] = cnt, first, step
            lat_off[l] = o
            tab = -np.ones(int(np.prod(cnt)), np.int32)
            s, e = self.boxes_cumsum[l], self.boxes_cumsum[l + 1]
            ii = (dec.centres_ndim[s:e] - np.asarray(first)) // np.asarray(step)
            tab[np.ravel_multi_index(tuple(ii.T), tuple(cnt))] = np.arange(s, e, dtype=np.int32)
            tables.append(tab)
            o += tab.size
        keep = dict(
            box_length=np.ascontiguousarray(dec.box_lengths, np.int32),
            box_level=np.ascontiguousarray(self._box_level, np.int32),
            centres=np.ascontiguousarray(dec.centres_ndim, np.int32),
            box_shape=np.ascontiguousarray(self._box_shapes, np.int32),
            coeffs_cumsum=np.ascontiguousarray(self.coeffs_cumsum, np.int64),
            boxes_cumsum=np.ascontiguousarray(self.boxes_cumsum, np.int32),
            gfilt=np.concatenate(gparts), gfilt_offset=goff,
            sum_gsquare=np.ascontiguousarray(self.sum_gsquare, np.float64).ravel(),
            lattice_counts=lat_cnt, lattice_first=lat_first, lattice_step=lat_step,
            lattice_offset=lat_off, lattice_box=np.concatenate(tables))
        d = _lib.MswptDesc()
        d.ndim = nd
        for a in range(3):
            d.N[a] = dec.N[a] if a < nd else 1
            d.aspect[a] = dec.box_aspect_ratio[a] if a < nd else 1
        d.redundancy = self.redundancy
        d.num_levels = L
        d.total_boxes = dec.total_num_boxes
        for k, v in keep.items():
            setattr(d, k, v.ctypes.data_as(ctypes.c_void_p))
        return d, keep

    def plan(self, device) -> int:
        """The libmsgb plan for ``device`` (created on first use)."""
        import torch

        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("MSWPT device plans need a CUDA device; there is no CPU path")
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        if idx not in self._plans:
            with torch.cuda.device(idx):
                d, keep = self._descriptor()
                h = ctypes.c_void_p()
                _lib.check(_lib.lib().msgb_mswpt_create(_lib.ref(d), ctypes.byref(h)), "msgb_mswpt_create")
                self._plans[idx] = h.value
        return self._plans[idx]

    def __del__(self):
        try:
            for h in getattr(self, "_plans", {}).values():
                _lib.lib().msgb_mswpt_destroy(h)
        except Exception:
            pass

    # ------------------------------------------------------------ transforms
    def forward_device(self, data, input_type: str = "spatial", *, scale: float = 1.0,
                       half_mask: bool = False, keys: bool = False):
        """Coefficients (and optionally top_n keys) as CUDA tensors."""
        import torch

        if self.windowing == "none":
            raise ValueError("MSWPT.forward does not support windowing='none': the fast "
                             "local-patch implementation truncates an otherwise global "
                             "Gaussian, so it cannot provide an exact analysis/synthesis "
                             "pair. Use 'rectangular' or 'rectangular_mirror'.")
        if input_type not in ("spatial", "fourier"):
            raise ValueError("Invalid conversion.")
        x = as_device_f64(data)
        if tuple(x.shape) != self.dyadic_decomp.N:
            raise ValueError(f"data must have shape {self.dyadic_decomp.N}; got {tuple(x.shape)}")
        is_complex = x.is_complex()
        if input_type == "fourier" and not is_complex:
            x = x.to(torch.complex128)
            is_complex = True
        x = x.contiguous()
        plan = self.plan(x.device)
        out = torch.empty(self.total_coeffs, dtype=torch.complex128, device=x.device)
        kt = torch.empty(self.total_coeffs, dtype=torch.float64, device=x.device) if keys else None
        nbytes = _lib.lib().msgb_mswpt_workspace_size(plan)
        ws = workspace(x.device, "mswpt", nbytes)
        st = torch.cuda.current_stream(x.device).cuda_stream
        _lib.check(_lib.lib().msgb_mswpt_forward(
            plan, x.data_ptr(), int(is_complex), int(input_type == "fourier"), float(scale),
            int(half_mask), out.data_ptr(), kt.data_ptr() if keys else None, ws.data_ptr(), nbytes, st),
            "msgb_mswpt_forward")
        return (out, kt) if keys else out

    def forward(self, data, input_type: str = "spatial"):
        """MSWPT.forward (transforms.py:696-733); returns a complex128 CUDA tensor."""
        return self.forward_device(data, input_type)

    def _synthesis(self, coeffs, mode: int, real_output: bool, output_type: str):
        import torch

        if output_type not in ("spatial", "fourier"):
            raise ValueError("Invalid conversion.")
        c = as_device_f64(coeffs)
        if c.numel() != self.total_coeffs:
            raise ValueError(f"coeffs must have {self.total_coeffs} entries; got {c.numel()}")
        c = c.to(torch.complex128).reshape(-1).contiguous()
        plan = self.plan(c.device)
        m = mode | (2 if output_type == "fourier" else 0)
        dt = torch.float64 if real_output else torch.complex128
        out = torch.empty(self.dyadic_decomp.N, dtype=dt, device=c.device)
        nbytes = _lib.lib().msgb_mswpt_workspace_size(plan)
        ws = workspace(c.device, "mswpt", nbytes)
        st = torch.cuda.current_stream(c.device).cuda_stream
        _lib.check(_lib.lib().msgb_mswpt_synthesis(plan, c.data_ptr(), m, int(real_output), out.data_ptr(),
                                                   ws.data_ptr(), nbytes, st), "msgb_mswpt_synthesis")
        return out

    def inverse(self, coeffs, output_type: str = "spatial"):
        """MSWPT.inverse (transforms.py:735-850); complex128 CUDA tensor."""
        return self._synthesis(coeffs, 0, False, output_type)

    def adjoint(self, coeffs, output_type: str = "spatial", real_output: bool = False):
        """Hermitian adjoint of ``forward`` (spatial input)."""
        return self._synthesis(coeffs, 1, real_output, output_type)

    # ------------------------------------------------------------ metadata
    @property
    def half_mask(self) -> np.ndarray:
        return self._half_mask

    def half_frame_capacity(self) -> int:
        """Number of coefficients kept by the conjugate half mask."""
        return sum((e - s) // 2 for s, e in zip(self.coeffs_cumsum[:-1], self.coeffs_cumsum[1:]))
