"""Autotuner of the batched banded-SW form.

The batched form (``gmf_banded_sw``) chooses a kernel shape per pair: 8 or
16 lanes per pair for narrow bands, a warp for wide ones, 2 / 4 / 8
cooperating warps for long pairs with wide bands, and overlaps the class
kernels on side streams.  Where those boundaries pay off depends on the
workload's mix of lengths and bands, so they are knobs
(:class:`SwTuning`, the C ABI's ``gmf_sw_tuning``).  The autotuner times
candidate settings on a sample of the workload, one knob at a time (coordinate
descent, a few passes), keeps the fastest, and refuses any setting whose
results differ from the reference run's in any field -- the knobs change
scheduling only, so a difference would be a bug.

Settings can be cached in a JSON file keyed by GPU name and a coarse workload
signature (length and band histograms), so a service tunes once per workload
shape.  The reference has no counterpart: its batched kernel has one shape.
"""

from __future__ import annotations

import json
import os
from dataclasses import asdict, dataclass, field, replace
from typing import Callable, Optional

import numpy as np

from . import _native


@dataclass(frozen=True)
class SwTuning:
    l8_max_w: int = 61
    l16_max_w: int = 125
    coop_min_strips: tuple = (4, 8, 16)
    warps_per_block: int = 4
    side_streams: int = 1

    def to_c(self) -> _native.GmfSwTuning:
        t = _native.GmfSwTuning()
        t.l8_max_w = int(self.l8_max_w)
        t.l16_max_w = int(self.l16_max_w)
        for i, v in enumerate(self.coop_min_strips):
            t.coop_min_strips[i] = int(v)
        t.warps_per_block = int(self.warps_per_block)
        t.side_streams = int(self.side_streams)
        return t

    @staticmethod
    def from_c(t: _native.GmfSwTuning) -> "SwTuning":
        return SwTuning(int(t.l8_max_w), int(t.l16_max_w), tuple(int(v) for v in t.coop_min_strips),
                        int(t.warps_per_block), int(t.side_streams))

    def valid(self) -> bool:
        return 0 <= self.l8_max_w <= self.l16_max_w and all(v >= 0 for v in self.coop_min_strips) \
            and 1 <= self.warps_per_block <= 4 and self.side_streams in (0, 1)


DEFAULT = SwTuning()

# Values tried per knob (each must keep the setting valid to be tried).
KNOBS: dict = {
    "l8_max_w": (0, 29, 61, 125),
    "l16_max_w": (61, 125, 253, 509),
    "coop_min_strips": ((4, 8, 16), (2, 4, 8), (8, 16, 32), (0, 0, 0)),
    "warps_per_block": (2, 4),
    "side_streams": (1, 0),
}


def _bind(device) -> None:
    import torch

    torch.cuda.set_device(device)
    _native.check("gmf_set_device", _native.lib().gmf_set_device(torch.device(device).index or 0))


def get_tuning(device=None) -> SwTuning:
    """The tuning in force on ``device`` (default: the current device)."""
    import ctypes

    if device is not None:
        _bind(device)
    t = _native.GmfSwTuning()
    _native.check("gmf_sw_get_tuning", _native.lib().gmf_sw_get_tuning(ctypes.byref(t)))
    return SwTuning.from_c(t)


def set_tuning(tuning: SwTuning, device=None) -> None:
    import ctypes

    if not tuning.valid():
        raise ValueError(f"invalid tuning {tuning}")
    if device is not None:
        _bind(device)
    _native.check("gmf_sw_set_tuning", _native.lib().gmf_sw_set_tuning(ctypes.byref(tuning.to_c())))


def coordinate_descent(start: SwTuning, evaluate: Callable[[SwTuning], Optional[float]],
                       knobs: Optional[dict] = None, passes: int = 2) -> tuple:
    """Minimise ``evaluate`` (ms, or None for a rejected setting) one knob at
    a time.  Returns (best setting, its ms, list of (setting, ms) trials)."""
    knobs = knobs or KNOBS
    trials: list = []
    cache: dict = {}

    def ev(t: SwTuning):
        if t not in cache:
            cache[t] = evaluate(t)
            trials.append((t, cache[t]))
        return cache[t]

    best = start
    best_ms = ev(start)
    if best_ms is None:
        raise RuntimeError("the starting tuning was rejected")
    for _ in range(passes):
        improved = False
        for name, values in knobs.items():
            for v in values:
                cand = replace(best, **{name: v})
                if cand == best or not cand.valid():
                    continue
                ms = ev(cand)
                if ms is not None and ms < best_ms:
                    best, best_ms, improved = cand, ms, True
        if not improved:
            break
    return best, best_ms, trials


def signature(query_len: np.ndarray, half_band: np.ndarray) -> str:
    """Coarse workload key: fractions of DP area per (log2 length, log2
    band) bucket, rounded to tenths."""
    ql = np.maximum(np.asarray(query_len, np.int64), 1)
    W = 2 * np.asarray(half_band, np.int64) + 1
    area = (ql * W).astype(np.float64)
    lb = np.minimum(np.log2(ql).astype(int), 20)
    wb = np.minimum(np.log2(W).astype(int), 13)
    hist: dict = {}
    for a, b, c in zip(lb, wb, area):
        hist[(int(a), int(b))] = hist.get((int(a), int(b)), 0.0) + c
    tot = sum(hist.values()) or 1.0
    parts = [f"{a}:{b}:{round(v / tot, 1)}" for (a, b), v in sorted(hist.items()) if round(v / tot, 1) > 0]
    return ",".join(parts)


@dataclass
class TuneReport:
    best: SwTuning
    best_ms: float
    default_ms: float
    trials: list = field(default_factory=list)

    def as_dict(self) -> dict:
        return {"best": asdict(self.best), "best_ms": self.best_ms, "default_ms": self.default_ms,
                "trials": len(self.trials)}


def autotune_sw(pairs, params, device=None, traceback: bool = True, reps: int = 3, passes: int = 2,
                knobs: Optional[dict] = None, apply: bool = True) -> TuneReport:
    """Tune the batched form on ``pairs`` (a PairSet sample of the workload)
    with scoring ``params`` (a GmfSwParams).  Every candidate's results are
    compared field by field with the default setting's; a candidate that
    differs is rejected.  The best setting is applied to the device unless
    ``apply`` is false."""
    import torch

    from . import extension
    from .device import require_cuda

    dev = require_cuda(device)
    _bind(dev)
    before = get_tuning()
    dp = extension.upload_pairs(pairs, dev)
    out = extension.SWOutputs.allocate(dp, traceback)
    ws = torch.empty(max(extension.workspace_bytes(dp, traceback), 256), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def run():
        extension.launch_banded_sw(dp, params, traceback, out=out, workspace=ws, stream=stream)

    def snapshot():
        r = extension.fetch(out, dp.n)
        cig = [tuple(r.cigar(b)) for b in range(dp.n)] if traceback else []
        return (r.score.tobytes(), r.query_end.tobytes(), r.target_end.tobytes(),
                None if r.query_start is None else r.query_start.tobytes(),
                None if r.target_start is None else r.target_start.tobytes(), cig)

    set_tuning(DEFAULT)
    run()
    reference = snapshot()

    def evaluate(t: SwTuning) -> Optional[float]:
        set_tuning(t)
        run()  # warm (kernel images, side streams)
        torch.cuda.synchronize(dev)
        if snapshot() != reference:
            return None
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    try:
        best, best_ms, trials = coordinate_descent(DEFAULT, evaluate, knobs, passes)
    finally:
        set_tuning(before)
    default_ms = next(ms for t, ms in trials if t == DEFAULT)
    if apply:
        set_tuning(best)
    return TuneReport(best, best_ms, default_ms, trials)


class TuningCache:
    """JSON file of tuned settings: {gpu name: {workload signature: setting}}."""

    def __init__(self, path: str):
        self.path = path
        self.data: dict = {}
        if os.path.exists(path):
            with open(path) as fh:
                self.data = json.load(fh)

    def get(self, gpu: str, sig: str) -> Optional[SwTuning]:
        d = self.data.get(gpu, {}).get(sig)
        if d is None:
            return None
        d = dict(d)
        d["coop_min_strips"] = tuple(d["coop_min_strips"])
        return SwTuning(**d)

    def put(self, gpu: str, sig: str, t: SwTuning) -> None:
        self.data.setdefault(gpu, {})[sig] = asdict(t)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(self.data, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def tuned_for(pairs, params, device=None, cache_path: Optional[str] = None, **kw) -> SwTuning:
    """The cached setting for this GPU and workload shape, or a fresh
    autotune on ``pairs`` (stored in the cache when one is given); the
    setting is applied to the device either way."""
    import torch

    from .device import require_cuda

    dev = require_cuda(device)
    gpu = torch.cuda.get_device_name(dev)
    sig = signature(pairs.query_len, pairs.half_band)
    cache = TuningCache(cache_path) if cache_path else None
    hit = cache.get(gpu, sig) if cache else None
    if hit is not None:
        set_tuning(hit, dev)
        return hit
    rep = autotune_sw(pairs, params, dev, **kw)
    if cache:
        cache.put(gpu, sig, rep.best)
    return rep.best
