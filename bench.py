#!/usr/bin/env python
"""Benchmark of the alignment hot path on B200 GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  The headline ``value`` is banded-SW GCUPS of the
extension workload (in-band DP cells per second, traceback included) with
inputs resident in HBM; ``e2e`` is the same metric through the public session
API with host inputs (pinned H2D copy, kernel, D2H of scores, coordinates and
CIGARs, every step); ``chain`` reports chaining anchors/s of the HiFi chaining
workload the same two ways.  Workloads are seeded synthetic data (no public
dataset).  Multi-GPU runs are replicas: every rank aligns its own shard-sized
copy of the workload (weak scaling, no collective on the data path); times
are device-measured per rank and the max over ranks is reported.

``--impl reference`` times the reference algorithm's CPU restatement (the C
oracle, all host cores) on the same workloads and prints the same line with
``"impl": "reference"``.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "banded-SW GCUPS & chain anchors/s, batched vs plain on 1 B200; p50/p99 ms"
INT_OPS_PER_CELL = 11  # scalar-equivalent integer ops per DP cell (E, F, H, sub, best)
TB_BYTES_PER_CELL = 0.5  # 4 traceback bits per cell written to the workspace


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="extension_pairs_150bp",
                   choices=["extension_pairs_150bp", "extension_pairs_mixed"])
    p.add_argument("--pairs", type=int, default=10_000)
    p.add_argument("--chain-reads", type=int, default=5_000)
    p.add_argument("--no-chain", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-case", action="store_true",
                   help="small single-GPU case for ncu captures (no timing JSON)")
    return p.parse_args()


# --------------------------------------------------------------------------- #
# workloads
# --------------------------------------------------------------------------- #
def sw_workload(name: str, n_pairs: int, seed: int):
    from graphmambaformer_b200 import synth

    if name == "extension_pairs_150bp":
        ps = synth.extension_pairs_150bp(n_pairs=n_pairs, seed=seed)
        params = (2, 4, 4, 2, 0)
        desc = dict(workload=name, pairs=len(ps), read_len=150, half_band=32, band_offset=32,
                    scoring="match 2, mismatch 4, open 4, extend 2, x_drop off")
    else:
        ps = synth.extension_pairs_mixed(n_pairs=n_pairs, seed=seed)
        params = (2, 4, 4, 2, 0)
        desc = dict(workload=name, pairs=len(ps), read_len="lognormal 150-20000",
                    half_band="32-500 (32 + 0.02 len)", scoring="2/4/4/2")
    desc["cells"] = ps.cells()
    return ps, params, desc


def chain_workload(n_reads: int, seed: int):
    from graphmambaformer_b200 import synth

    b = synth.chaining_reads_hifi(n_reads=n_reads, seed=seed)
    return b, dict(workload="chaining_reads_hifi", reads=len(b), anchors=b.n_anchors,
                   read_len="15 kb +-20%", lookback=50, max_gap=5000, k=15, w=10)


# --------------------------------------------------------------------------- #
# helpers
# --------------------------------------------------------------------------- #
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout
                for line in out.strip().splitlines():
                    f = [x.strip() for x in line.split(",")]
                    if self.uuid and self.uuid not in f[0]:
                        continue
                    self.rows.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if "Active" == r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measure_int_peak(device) -> dict:
    """Integer-ALU throughput of this GPU (scalar int32 add/max chains)."""
    import ctypes

    import torch

    from graphmambaformer_b200 import build

    lib = ctypes.CDLL(build.PROBE_LIB)
    lib.gmf_probe_int.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_void_p]
    lib.gmf_probe_int_ops.restype = ctypes.c_double
    lib.gmf_probe_int_ops.argtypes = [ctypes.c_int] * 4
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    blocks, threads, iters = sms * 8, 256, 4096
    out = torch.empty(blocks * threads, dtype=torch.int32, device=device)
    s = torch.cuda.current_stream(device)
    res = {}
    for kind, name in ((0, "int32_add_max"), (1, "int32_dpx_viaddmax"), (2, "int16x2_add_max")):
        best = 0.0
        for _ in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            lib.gmf_probe_int(kind, blocks, threads, iters, ctypes.c_void_p(out.data_ptr()),
                              ctypes.c_void_p(s.cuda_stream))
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = max(best, lib.gmf_probe_int_ops(kind, blocks, threads, iters) / (ms * 1e-3))
        res[name] = best / 1e12  # Tops/s
    return res


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def load_traffic():
    """Per-cell DRAM traffic of the SW kernel from the committed ncu summary
    (bytes per DP cell), or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return {}
    out = {}
    for line in open(path):
        if "=" in line and not line.startswith("#"):
            k, v = line.split("=", 1)
            try:
                out[k.strip()] = float(v.split()[0])
            except ValueError:
                pass
    return out


# --------------------------------------------------------------------------- #
# B200 arm
# --------------------------------------------------------------------------- #
def run_b200(args):
    import torch
    import torch.distributed as dist

    from graphmambaformer_b200 import chaining, extension
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.session import ChainSession, ExtensionSession

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", device_id=device, timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    # ---- SW workload (each rank its own shard-sized replica) ----
    ps, params, desc = sw_workload(args.workload, args.pairs, seed=1 + 1000 * rank)
    sw_p = extension.sw_params(*params)
    dp = extension.upload_pairs(ps, device)
    out = extension.SWOutputs.allocate(dp, True)
    ws = torch.empty(extension.workspace_bytes(dp, True), dtype=torch.uint8, device=device)
    flush = torch.empty(320 * 1024 * 1024 // 4, dtype=torch.int32, device=device)  # > 126 MB L2
    stream = torch.cuda.current_stream(device)

    def sw_step():
        extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=stream)

    for _ in range(max(args.warmup, 3)):
        sw_step()
    torch.cuda.synchronize(device)
    # correctness guard: the timed launch must report no workspace/capacity error
    err = int(out.error_flags.item())
    if err:
        raise RuntimeError(f"SW kernel reported error flags {err}")
    uuid = str(torch.cuda.get_device_properties(device).uuid) if hasattr(
        torch.cuda.get_device_properties(device), "uuid") else ""
    sampler = ClockSampler(uuid)
    step_ms = []
    with sampler:
        barrier()
        torch.cuda.synchronize(device)
        for _ in range(args.steps):
            flush.zero_()  # evict L2 between timed steps (outside the timed events)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sw_step()
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize(device)
        barrier()
    # the plain per-batch form (one warp per pair, int32 cells) on the same batch
    plain_ms = []
    for _ in range(max(args.warmup, 3)):
        extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=stream, form="plain")
    torch.cuda.synchronize(device)
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=stream, form="plain")
        e1.record(stream)
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
    cells_rank = desc["cells"]
    ms_rank = float(np.mean(step_ms))
    ms = max_over_ranks(ms_rank)
    total_cells = sum_over_ranks(float(cells_rank))
    gcups = total_cells / (ms * 1e-3) / 1e9

    # ---- e2e through the session API (host inputs, pinned H2D, D2H) ----
    sess = ExtensionSession(device, *params, traceback=True)
    for _ in range(max(args.warmup, 3)):
        sess.align(ps)
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sess.align(ps)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    barrier()
    e2e_step = max_over_ranks(float(np.mean(e2e_ms)))
    plain_step = max_over_ranks(float(np.mean(plain_ms)))
    e2e_gcups = total_cells / (e2e_step * 1e-3) / 1e9

    # ---- chaining ----
    chain = None
    if not args.no_chain:
        cb, cdesc = chain_workload(args.chain_reads, seed=2 + 1000 * rank)
        cfg = ChainingConfig(max_lookback=50, max_gap=5000)
        da = chaining.upload_anchors(cb, device)
        cout = chaining.ChainOutputs.allocate(da, cfg.max_chains)
        for _ in range(max(args.warmup, 3)):
            chaining.launch_chain_batch(da, cfg, out=cout, stream=stream)
        torch.cuda.synchronize(device)
        barrier()
        cms = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            chaining.launch_chain_batch(da, cfg, out=cout, stream=stream)
            e1.record(stream)
            e1.synchronize()
            cms.append(e0.elapsed_time(e1))
        barrier()
        c_ms = max_over_ranks(float(np.mean(cms)))
        anchors_total = sum_over_ranks(float(cb.n_anchors))
        csess = ChainSession(cfg, device)
        for _ in range(2):
            csess.chain(cb)
        barrier()
        ce = []
        for _ in range(max(2, args.steps // 4)):
            t0 = time.perf_counter()
            csess.chain(cb)
            ce.append((time.perf_counter() - t0) * 1e3)
        barrier()
        ce_ms = max_over_ranks(float(np.mean(ce)))
        chain = {
            "value": anchors_total / (c_ms * 1e-3), "unit": "anchors/s", "ms_per_step": c_ms,
            "config": cdesc, "gpu_launches_per_step": 3,
            "e2e": {"value": anchors_total / (ce_ms * 1e-3), "unit": "anchors/s", "ms_per_step": ce_ms,
                    "h2d_bytes_per_step": csess.h2d_bytes, "d2h_bytes_per_step": csess.d2h_bytes},
        }

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    # ---- roofline (rank 0, single-GPU kernel figures) ----
    peaks, peak_src = load_peaks()
    ip = measure_int_peak(device)
    int_peak = ip["int32_add_max"]
    achieved_int = INT_OPS_PER_CELL * cells_rank / (ms_rank * 1e-3) / 1e12
    traffic = load_traffic()
    tpc = traffic.get("sw_bytes_per_cell")
    alg_bytes = TB_BYTES_PER_CELL * cells_rank + int(ps.query.size + ps.target.size)
    line = {
        "metric": METRIC,
        "value": gcups,
        "unit": "GCUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded, reference simulator error model)",
        "config": dict(desc, parallelism=f"replicas x{world}", l2="flushed between timed steps",
                       traceback="on (CIGAR per pair)", kernel="gmf_banded_sw batched: device classifier + int16x2 work-queue kernels"),
        "e2e": {"value": e2e_gcups, "unit": "GCUPS", "ms_per_step": e2e_step,
                "h2d_bytes_per_step": sess.h2d_bytes, "d2h_bytes_per_step": sess.d2h_bytes,
                "timing": "wall clock around ExtensionSession.align (synchronous)"},
        "plain": {"value": total_cells / (plain_step * 1e-3) / 1e9, "unit": "GCUPS",
                  "ms_per_step": plain_step, "form": "gmf_banded_sw_plain: one warp per pair, int32, one launch",
                  "batched_over_plain": plain_step / ms},
        "gpu_launches": args.steps * 5,
        "roofline": {"bound": "int", "achieved": achieved_int, "peak": int_peak, "unit": "Tops/s",
                     "frac": achieved_int / int_peak, "peak_source": "int32 add/max probe, this GPU",
                     "ops_per_cell": INT_OPS_PER_CELL,
                     "traffic": (tpc * cells_rank) if tpc else None},
        "roofline_hbm": {"bound": "hbm", "achieved": alg_bytes / (ms_rank * 1e-3) / 1e9,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": alg_bytes / (ms_rank * 1e-3) / 1e9 / peaks["hbm_gbs"],
                         "peak_source": peak_src, "traffic": (tpc * cells_rank) if tpc else None},
        "int_probe_tops": ip,
        "clocks": sampler.summary(),
    }
    if chain:
        line["chain"] = chain
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ps, params, cells_rank)
    return line


# --------------------------------------------------------------------------- #
# CPU baseline / reference arm
# --------------------------------------------------------------------------- #
def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(ps, params, cells, sample_pairs: int = 10_000) -> dict:
    from oracle import oracle

    n = min(sample_pairs, len(ps))
    qs = [ps.q(b) for b in range(n)]
    ts = [ps.t(b) for b in range(n)]
    from graphmambaformer_b200.synth import band_cells

    cs = int(band_cells(ps.query_len[:n], ps.target_len[:n], ps.half_band[:n], ps.band_offset[:n]).sum())
    th = host_threads()
    t0 = time.perf_counter()
    oracle.sw_batch(qs, ts, ps.half_band[:n], ps.band_offset[:n], *params, threads=th)
    dt = time.perf_counter() - t0
    return {"value": cs / dt / 1e9, "unit": "GCUPS", "cores": th, "kind": "port",
            "sample": f"{n} pairs ({cs} cells) of the same workload, SW + traceback, C oracle"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle import oracle

    ps, params, desc = sw_workload(args.workload, args.pairs, seed=1)
    th = host_threads()
    n = len(ps)
    if desc["workload"] != "extension_pairs_150bp":
        n = min(n, 2000)
    qs = [ps.q(b) for b in range(n)]
    ts = [ps.t(b) for b in range(n)]
    from graphmambaformer_b200.synth import band_cells

    cells = int(band_cells(ps.query_len[:n], ps.target_len[:n], ps.half_band[:n], ps.band_offset[:n]).sum())
    for _ in range(max(args.warmup, 3) if args.warmup else 0):
        oracle.sw_batch(qs[:200], ts[:200], ps.half_band[:200], ps.band_offset[:200], *params, threads=th)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.sw_batch(qs, ts, ps.half_band[:n], ps.band_offset[:n], *params, threads=th)
        times.append(time.perf_counter() - t0)
    ms = float(np.mean(times)) * 1e3
    gcups = cells / (ms * 1e-3) / 1e9
    sample = f"{n} pairs ({cells} cells) per step, SW + traceback, C restatement of the reference"
    line = {
        "impl": "reference", "metric": METRIC, "value": gcups, "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "float32", "data": "synthetic (seeded)",
        "config": dict(desc, parallelism="host threads"),
        "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": th, "kind": "port", "sample": sample},
        "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_chain:
        cb, cdesc = chain_workload(min(args.chain_reads, 1000), seed=2)
        lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
        t0 = time.perf_counter()
        oracle.chain_batch(cb.read_off, cb.read_pos, cb.ref_pos, cb.length, cb.strand, lut,
                           max_lookback=50, threads=th)
        dt = time.perf_counter() - t0
        line["chain"] = {"value": cb.n_anchors / dt, "unit": "anchors/s", "ms_per_step": dt * 1e3,
                         "config": cdesc, "cores": th}
    return line


def profile_case(args):
    """A small case for ncu: 2,000 pairs of the 150 bp workload, 3 launches."""
    import torch

    from graphmambaformer_b200 import extension

    ps, params, _ = sw_workload(args.workload, 2000, seed=1)
    dp = extension.upload_pairs(ps, "cuda:0")
    for _ in range(3):
        extension.launch_banded_sw(dp, extension.sw_params(*params), True)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": "done", "cells_per_launch": ps.cells()}))


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    line = run_reference(args) if args.impl == "reference" else run_b200(args)
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
