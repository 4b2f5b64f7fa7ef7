"""Device plumbing: streams, grow-only workspaces and pinned staging buffers.

PyTorch is used only to own device memory and streams; every kernel the
stages launch comes from the gmf CUDA library.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native


def require_cuda(device=None) -> torch.device:
    """The CUDA device to run on; raises when none is available (there is no
    CPU fallback for the alignment kernels)."""
    if not torch.cuda.is_available():
        raise RuntimeError("graphmambaformer_b200 needs a CUDA GPU (sm_100a); none is available")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dev.type != "cuda":
        raise RuntimeError(f"graphmambaformer_b200 runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def stream_handle(stream: Optional[torch.cuda.Stream], device: torch.device) -> int:
    s = stream if stream is not None else torch.cuda.current_stream(device)
    return int(s.cuda_stream)


def bind(device: torch.device, stream_ptr: int) -> None:
    """Calls on the legacy stream run on the library's selected device."""
    if stream_ptr == 0:
        _native.check("gmf_set_device", _native.lib().gmf_set_device(device.index))


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


class Workspace:
    """Grow-only device scratch buffer per device (never shrinks, so repeated
    calls do not allocate)."""

    def __init__(self):
        self._buf: dict[int, torch.Tensor] = {}

    def get(self, device: torch.device, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        cur = self._buf.get(device.index)
        if cur is None or cur.numel() < nbytes:
            grow = max(nbytes, int(cur.numel() * 1.25) if cur is not None else 0)
            cur = torch.empty(grow, dtype=torch.uint8, device=device)
            self._buf[device.index] = cur
        return cur


WORKSPACE = Workspace()


def to_device(a: np.ndarray, device: torch.device, stream=None, pinned: bool = True) -> torch.Tensor:
    """Host numpy -> device tensor through a pinned staging copy (async on the
    current stream)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if pinned and t.numel() > 0:
        t = t.pin_memory()
    return t.to(device, non_blocking=True)


def np_ptr(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)
