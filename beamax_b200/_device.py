"""Device plumbing: tensor conversion, cached device copies and workspaces.

PyTorch is used only for device memory, streams and host<->device copies; all
compute runs in libmsgb.so.
"""

from __future__ import annotations

import threading
import weakref
from typing import Dict, Tuple

import numpy as np

_ws_lock = threading.Lock()
_workspaces: Dict[Tuple[int, str], "object"] = {}


def default_device():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("beamax_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    return torch.device("cuda", torch.cuda.current_device())


def as_device_f64(x, device=None):
    """A CUDA float64 / complex128 tensor for ``x`` (NumPy array, scalar or tensor)."""
    import torch

    if isinstance(x, torch.Tensor):
        dev = x.device if x.is_cuda else (torch.device(device) if device is not None else default_device())
        t = x.to(dev)
        if t.is_complex():
            return t.to(torch.complex128)
        return t.to(torch.float64)
    arr = np.asarray(x)
    dev = torch.device(device) if device is not None else default_device()
    if np.iscomplexobj(arr):
        return torch.from_numpy(np.ascontiguousarray(arr, np.complex128)).to(dev)
    return torch.from_numpy(np.ascontiguousarray(arr, np.float64)).to(dev)


def workspace(device, name: str, nbytes: int):
    """A 256-byte aligned scratch buffer of at least ``nbytes`` bytes (cached, grown on demand)."""
    import torch

    dev = torch.device(device)
    key = (dev.index if dev.index is not None else torch.cuda.current_device(), name)
    with _ws_lock:
        buf = _workspaces.get(key)
        if buf is None or buf.numel() < nbytes:
            # release the smaller buffer before allocating the larger one
            _workspaces.pop(key, None)
            buf = None
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
            _workspaces[key] = buf
    assert buf.data_ptr() % 256 == 0
    return buf


class DeviceCache:
    """Per-object, per-device cache of derived device tensors (weakly keyed)."""

    def __init__(self):
        self._store = weakref.WeakKeyDictionary()

    def get(self, obj, key, make):
        d = self._store.get(obj)
        if d is None:
            d = {}
            self._store[obj] = d
        if key not in d:
            d[key] = make()
        return d[key]
