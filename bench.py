#!/usr/bin/env python
"""Benchmark of the alignment hot path on B200 GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  The headline ``value`` is banded-SW GCUPS (in-band
DP cells per second, traceback and CIGARs included) of the batched form on
the mixed-length extension workload: 100,000 pairs with log-normal lengths
from 150 bp to 20 kb, Illumina / HiFi / ONT error profiles and bands growing
with length from 32 to 432, inputs resident in HBM.  ``plain`` is the plain
per-batch form (one warp per pair, int32 cells, one launch) on the same
batch; ``e2e`` is the same metric through the public ``ExtensionSession``
API with host inputs (pinned H2D copy, kernels, D2H of scores, coordinates
and CIGARs, every step).  ``extension_150bp`` reports the 10,000-pair 150 bp
workload the same two ways and ``chain`` the chaining anchors/s of the HiFi
chaining workload.  Workloads are seeded synthetic data (no public
dataset).  Multi-GPU runs are replicas: every rank aligns its own shard-sized
copy of the workload (weak scaling, no collective on the data path); times
are device-measured per rank and the max over ranks is reported.

``--impl reference`` times the reference algorithm's CPU restatement (the C
oracle, all host cores) on a bounded, length-stratified sample of the same
workload and prints the same line with ``"impl": "reference"``.
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
CHAIN_OPS_PER_EVAL = 10  # f64 / int ops per chaining predecessor evaluation (gap, score, penalty, compares)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="extension_pairs_mixed",
                   choices=["extension_pairs_150bp", "extension_pairs_mixed"])
    p.add_argument("--pairs", type=int, default=0, help="pairs of the headline workload (0: its default)")
    p.add_argument("--chain-reads", type=int, default=5_000)
    p.add_argument("--no-chain", action="store_true")
    p.add_argument("--no-150bp", action="store_true")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--long-reads", type=int, default=2000,
                   help="reads of the long-read stress leg (2,000 = the full configuration; 0 skips it)")
    p.add_argument("--wfa-pairs", type=int, default=20_000, help="pairs of the WFA leg (0: skip it)")
    p.add_argument("--sam-records", type=int, default=25_000, help="records of the SAM leg (0: skip it)")
    p.add_argument("--serve-loads", default="10000,20000,50000,100000,200000",
                   help="offered loads of the serving leg, reads/s")
    p.add_argument("--serve-requests", type=int, default=600,
                   help="requests per load point (at least 1.5 s of arrivals at that load)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-case", action="store_true",
                   help="small single-GPU case for ncu captures (no timing JSON)")
    p.add_argument("--profile-longest", type=int, default=0,
                   help="with --profile-case: the N largest pairs (by DP area) of the workload")
    p.add_argument("--profile-chain", type=int, default=0,
                   help="with --profile-case: chain N reads of the HiFi chaining workload instead")
    return p.parse_args()


# --------------------------------------------------------------------------- #
# workloads
# --------------------------------------------------------------------------- #
def sw_workload(name: str, n_pairs: int, seed: int):
    from graphmambaformer_b200 import synth

    if not n_pairs:
        n_pairs = 10_000 if name == "extension_pairs_150bp" else 100_000
    if name == "extension_pairs_150bp":
        ps = synth.extension_pairs_150bp(n_pairs=n_pairs, seed=seed)
        params = (2, 4, 4, 2, 0)
        desc = dict(workload=name, pairs=len(ps), read_len=150, half_band=32, band_offset=32,
                    scoring="match 2, mismatch 4, open 4, extend 2, x_drop off")
    else:
        ps = synth.extension_pairs_mixed(n_pairs=n_pairs, seed=seed)
        params = (2, 4, 4, 2, 0)
        desc = dict(workload=name, pairs=len(ps), read_len="lognormal(7.0, 1.2) clipped to 150-20000",
                    profiles="Illumina 1% sub / HiFi 0.1% / ONT 5% (60% indels), one third each",
                    half_band="clip(32 + 0.02 len, 32, 500)", band_offset=32,
                    scoring="match 2, mismatch 4, open 4, extend 2, x_drop off")
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
    # float64 add / max (the chaining DP's arithmetic)
    lib.gmf_probe_f64.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_void_p]
    outd = torch.empty(blocks * threads, dtype=torch.float64, device=device)
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        lib.gmf_probe_f64(blocks, threads, iters, ctypes.c_void_p(outd.data_ptr()), ctypes.c_void_p(s.cuda_stream))
        e1.record(s)
        e1.synchronize()
        best = max(best, 4.0 * 8.0 * iters * blocks * threads / (e0.elapsed_time(e1) * 1e-3))
    res["f64_add_max"] = best / 1e12
    return res


def chain_pair_evaluations(batch, lookback: int) -> int:
    """Predecessor evaluations of the chaining DP: per read and strand with
    n anchors, sum over i < n of min(i, lookback)."""
    r = np.repeat(np.arange(len(batch.read_off) - 1), np.diff(batch.read_off))
    plus = np.bincount(r[batch.strand > 0], minlength=len(batch.read_off) - 1).astype(np.int64)
    minus = np.diff(batch.read_off).astype(np.int64) - plus
    h = int(lookback)
    total = 0
    for n in (plus, minus):
        small = n <= h
        total += int((n[small] * (n[small] - 1) // 2).sum())
        total += int((h * (h - 1) // 2 + (n[~small] - h) * h).sum())
    return total


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


def launches_per_call(max_half_band: int, traceback: bool) -> int:
    """Kernels one gmf_banded_sw call launches: the classifier, one kernel per
    pair class that can be populated (the cooperative classes only when the
    widest band reaches their period range), and the deferred walk."""
    W = 2 * max_half_band + 1
    P = max(W + 2, 128)
    P = (P + 3) & ~3
    coop = sum(1 for pmin in (8 * 132, 4 * 132, 2 * 132) if P >= pmin)
    return 1 + coop + 3 + 1 + (1 if traceback else 0)


def time_device(fn, steps, stream, flush):
    """Per-step device time of ``fn`` with CUDA events on ``stream``; the L2
    is flushed (a 320 MB write) before every step, outside the events."""
    import torch

    out = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


# --------------------------------------------------------------------------- #
# B200 arm
# --------------------------------------------------------------------------- #
def run_b200(args):
    import torch
    import torch.distributed as dist

    from graphmambaformer_b200 import chaining, extension
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.session import ChainSession, ExtensionSession, pin_anchors

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

    warm = max(args.warmup, 3)
    # CPU baselines are timed on rank 0 of a one-GPU run only
    args.no_cpu_baseline = args.no_cpu_baseline or world > 1 or rank != 0
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(320 * 1024 * 1024 // 4, dtype=torch.int32, device=device)  # > 126 MB L2

    def sw_leg(name, n_pairs, seed, clocks=None, keep_result=False):
        """Batched and plain device timing plus e2e of one SW workload."""
        ps, params, desc = sw_workload(name, n_pairs, seed=seed)
        sw_p = extension.sw_params(*params)
        dp = extension.upload_pairs(ps, device)
        out = extension.SWOutputs.allocate(dp, True)
        ws = torch.empty(extension.workspace_bytes(dp, True), dtype=torch.uint8, device=device)

        def step(form):
            return lambda: extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=stream,
                                                      form=form)

        for _ in range(warm):
            step("batched")()
        torch.cuda.synchronize(device)
        if int(out.error_flags.item()):  # the timed launches must report no workspace/capacity error
            raise RuntimeError(f"SW kernels reported error flags {int(out.error_flags.item())}")
        barrier()
        torch.cuda.synchronize(device)
        if clocks is not None:
            with clocks:
                b_ms = time_device(step("batched"), args.steps, stream, flush)
        else:
            b_ms = time_device(step("batched"), args.steps, stream, flush)
        barrier()
        # the same call captured once as a CUDA graph (classifier, class kernels forked onto side streams
        # and joined, deferred walk) and replayed: one graph launch per step
        from graphmambaformer_b200 import _native

        _native.check("gmf_set_device", _native.lib().gmf_set_device(device.index))
        cap = torch.cuda.Stream(device)
        cap.wait_stream(stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cap, capture_error_mode="thread_local"):
            extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=cap)
        stream.wait_stream(cap)
        for _ in range(warm):
            graph.replay()
        torch.cuda.synchronize(device)
        barrier()
        g_ms = time_device(graph.replay, args.steps, stream, flush)
        torch.cuda.synchronize(device)
        if int(out.error_flags.item()):
            raise RuntimeError(f"SW kernels reported error flags {int(out.error_flags.item())}")
        barrier()
        result = extension.fetch(out, dp.n) if keep_result else None  # outputs of the last timed call
        del graph
        for _ in range(warm):
            step("plain")()
        torch.cuda.synchronize(device)
        p_ms = time_device(step("plain"), args.steps, stream, flush)
        barrier()
        sess = ExtensionSession(device, *params, traceback=True)
        for _ in range(warm):
            sess.align(ps)
        barrier()
        e_ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            sess.align(ps)
            e_ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
        sess_io = (sess.h2d_bytes, sess.d2h_bytes)
        ws_bytes = int(ws.numel())
        del ws, out, sess
        torch.cuda.empty_cache()  # the context allocates through the library's own runtime
        # end to end through the C ABI on host buffers: gmf_batch_submit + gmf_batch_wait per step
        from graphmambaformer_b200.context import AlignContext

        ctx = AlignContext(local, slots=1)
        for _ in range(min(warm, 2)):
            r = ctx.align(ps, sw_p)
        barrier()
        c_ms = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = ctx.align(ps, sw_p)
            c_ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
        ctx.close()
        # the same through a two-slot context: step i+1 is submitted before step i is waited for, so one
        # batch's copies overlap the other's kernels (every step still copies its inputs and results)
        ctx2 = AlignContext(local, slots=2)
        for _ in range(2):
            ctx2.align(ps, sw_p)
        barrier()
        t0 = time.perf_counter()
        prev = None
        for _ in range(args.steps):
            cur = ctx2.submit(ps, sw_p)
            if prev is not None:
                ctx2.wait(prev)
            prev = cur
        ctx2.wait(prev)
        c2_ms = (time.perf_counter() - t0) * 1e3 / args.steps
        barrier()
        ctx2.close()
        ctx_io = (int(ps.query.size + ps.target.size + 16 * (len(ps) + 1) + 12 * len(ps)),
                  int(48 * len(ps) + 12 + 4 * len(r.cigar_words)))
        pipe = None
        if ws_bytes < 8 << 30:  # several batches in flight when three arenas fit comfortably
            ctx3 = AlignContext(local, slots=3)
            for _ in range(3):  # every slot's arena and staging allocated before timing
                ctx3.align(ps, sw_p)
            barrier()
            t0 = time.perf_counter()
            inflight = []
            for _ in range(args.steps):
                inflight.append(ctx3.submit(ps, sw_p))
                if len(inflight) == 3:
                    ctx3.wait(inflight.pop(0))
            for t in inflight:
                ctx3.wait(t)
            pipe = (time.perf_counter() - t0) * 1e3 / args.steps
            barrier()
            ctx3.close()
        cells = float(desc["cells"])
        total = sum_over_ranks(cells)
        b = max_over_ranks(float(np.mean(b_ms)))
        gr = max_over_ranks(float(np.mean(g_ms)))
        pl = max_over_ranks(float(np.mean(p_ms)))
        e = max_over_ranks(float(np.mean(e_ms)))
        c = max_over_ranks(float(np.mean(c_ms)))
        c2 = max_over_ranks(c2_ms)
        pp = max_over_ranks(pipe) if pipe is not None else None
        return dict(ps=ps, params=params, desc=desc, cells=cells, total=total, batched_ms=b, graph_ms=gr, plain_ms=pl,
                    e2e_ms=c2, sync_ms=c, session_ms=e, pipelined_ms=pp, rank_ms=float(np.mean(b_ms)),
                    sess_io=sess_io, ctx_io=ctx_io, launches=launches_per_call(dp.max_half_band, True),
                    result=result)

    # ---- autotuned scheduling of the batched form (on a 10% sample of the
    # headline workload; outside every timed region) ----
    tuning = None
    if not args.no_autotune:
        from graphmambaformer_b200 import autotune

        ps_s, params_s, _ = sw_workload(args.workload, args.pairs, seed=1 + 1000 * rank)
        rng = np.random.default_rng(99)
        sample = ps_s.subset(np.sort(rng.choice(len(ps_s), size=max(1, len(ps_s) // 10), replace=False)))
        rep = autotune.autotune_sw(sample, extension.sw_params(*params_s), device, reps=2, passes=1)
        tuning = dict(rep.as_dict(), sample_pairs=len(sample))
        del ps_s, sample

    uuid = str(getattr(torch.cuda.get_device_properties(device), "uuid", ""))
    sampler = ClockSampler(uuid)
    head = sw_leg(args.workload, args.pairs, 1 + 1000 * rank, clocks=sampler,
                  keep_result=not args.no_cpu_baseline)
    small = None
    if not args.no_150bp and args.workload != "extension_pairs_150bp":
        # its own scheduling knobs, tuned on the whole batch (a call takes a fraction of a millisecond, and
        # a 10% sample of it is launch-bound, which once steered the knobs to a slower class split); the
        # headline's are put back afterwards for the legs that run the mixed workload
        from graphmambaformer_b200 import autotune

        head_tuning = autotune.get_tuning(device)
        small_tuning = None
        if not args.no_autotune:
            ps_s, params_s, _ = sw_workload("extension_pairs_150bp", 0, seed=11 + 1000 * rank)
            small_tuning = autotune.autotune_sw(ps_s, extension.sw_params(*params_s), device, reps=5,
                                                passes=1).as_dict()
            del ps_s
        small = sw_leg("extension_pairs_150bp", 0, 11 + 1000 * rank)
        small["tuning"] = small_tuning or "defaults"
        autotune.set_tuning(head_tuning, device)

    # ---- chaining ----
    chain = None
    if not args.no_chain:
        cb, cdesc = chain_workload(args.chain_reads, seed=2 + 1000 * rank)
        cfg = ChainingConfig(max_lookback=50, max_gap=5000)
        da = chaining.upload_anchors(cb, device)
        cout = chaining.ChainOutputs.allocate(da, cfg.max_chains)

        def cstep():
            chaining.launch_chain_batch(da, cfg, out=cout, stream=stream)

        for _ in range(warm):
            cstep()
        torch.cuda.synchronize(device)
        barrier()
        cms = time_device(cstep, args.steps, stream, flush)
        barrier()
        c_ms = max_over_ranks(float(np.mean(cms)))
        anchors_total = sum_over_ranks(float(cb.n_anchors))
        csess = ChainSession(cfg, device)
        pcb = pin_anchors(cb)  # the batch as a service holds it: page-locked host columns
        for _ in range(2):
            csess.chain(pcb)
        barrier()
        ce = []
        for _ in range(max(2, args.steps // 4)):
            t0 = time.perf_counter()
            csess.chain(pcb)
            ce.append((time.perf_counter() - t0) * 1e3)
        barrier()
        ce_ms = max_over_ranks(float(np.mean(ce)))
        evals = chain_pair_evaluations(cb, cfg.max_lookback)
        chain = {
            "value": anchors_total / (c_ms * 1e-3), "unit": "anchors/s", "ms_per_step": c_ms,
            "pair_evaluations_per_step": evals,
            "config": cdesc, "gpu_launches_per_step": 3,
            "e2e": {"value": anchors_total / (ce_ms * 1e-3), "unit": "anchors/s", "ms_per_step": ce_ms,
                    "h2d_bytes_per_step": csess.h2d_bytes, "d2h_bytes_per_step": csess.d2h_bytes},
        }

    # ---- long-read stress: 50-100 kb ONT-like reads, h = 200 chaining, gap SW ----
    longr = None
    if args.long_reads > 0:
        longr = long_read_leg(args, device, stream, flush, seed=6 + 1000 * rank, warm=warm)

    # ---- serving loop: Poisson requests of 1-64 mixed-profile reads ----
    serve = None
    if not args.no_serve:
        serve = serve_leg(args, device, seed=7 + 1000 * rank)

    # ---- wavefront alignment (the extension's algorithm="wfa" variant) ----
    wfa_res = None
    if args.wfa_pairs > 0:
        wfa_res = wfa_leg(args, device, stream, flush, seed=8 + 1000 * rank, warm=warm)

    # ---- SAM text of alignment records ----
    sam_res = None
    if args.sam_records > 0:
        sam_res = sam_leg(args, device, stream, flush, warm=warm)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    # ---- roofline (rank 0, single-GPU figures of the headline call) ----
    peaks, peak_src = load_peaks()
    ip = measure_int_peak(device)
    int_peak = ip["int32_add_max"]
    cells_rank, ms_rank = head["cells"], head["rank_ms"]
    achieved_int = INT_OPS_PER_CELL * cells_rank / (ms_rank * 1e-3) / 1e12
    traffic = load_traffic()
    tpc = traffic.get("sw_bytes_per_cell")
    ps = head["ps"]
    alg_bytes = TB_BYTES_PER_CELL * cells_rank + int(ps.query.size + ps.target.size)
    gcups = head["total"] / (head["batched_ms"] * 1e-3) / 1e9
    plain_gcups = head["total"] / (head["plain_ms"] * 1e-3) / 1e9
    line = {
        "metric": METRIC,
        "value": gcups,
        "unit": "GCUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warm,
        "ms_per_step": head["batched_ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u16x2 / int32 (exact integer scores)",
        "data": "synthetic (seeded, reference simulator error model)",
        "config": dict(head["desc"], parallelism=f"replicas x{world}", l2="flushed between timed steps",
                       traceback="on (CIGAR per pair)",
                       form="batched: device classifier, class kernels on side streams, deferred walk",
                       tuning=tuning or "defaults"),
        "e2e": {"value": head["total"] / (head["e2e_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                "ms_per_step": head["e2e_ms"], "h2d_bytes_per_step": head["ctx_io"][0],
                "d2h_bytes_per_step": head["ctx_io"][1],
                "timing": "wall clock of K steps through the C ABI on host buffers (gmf_batch_submit, "
                          "gmf_batch_wait) with two batches in flight on a two-slot context, per step",
                "sync": {"value": head["total"] / (head["sync_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                         "ms_per_step": head["sync_ms"],
                         "timing": "submit + wait of one batch at a time (one-slot context)"},
                "session": {"value": head["total"] / (head["session_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                            "ms_per_step": head["session_ms"], "h2d_bytes_per_step": head["sess_io"][0],
                            "d2h_bytes_per_step": head["sess_io"][1],
                            "timing": "wall clock around ExtensionSession.align (Python API)"}},
        "graph": {"value": head["total"] / (head["graph_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                  "ms_per_step": head["graph_ms"],
                  "form": "the same call captured once as a CUDA graph and replayed (one graph launch per step)"},
        "plain": {"value": plain_gcups, "unit": "GCUPS", "ms_per_step": head["plain_ms"],
                  "form": "gmf_banded_sw_plain: one warp per pair, int32 cells, one launch",
                  "batched_over_plain": gcups / plain_gcups},
        "gpu_launches": args.steps * head["launches"],
        "roofline": {"bound": "int", "kernel": "gmf_banded_sw (all kernels of one call)",
                     "achieved": achieved_int, "peak": int_peak, "unit": "Tops/s",
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
    if small:
        line["extension_150bp"] = {
            "value": small["total"] / (small["batched_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
            "ms_per_step": small["batched_ms"], "config": small["desc"],
            "graph": small["total"] / (small["graph_ms"] * 1e-3) / 1e9,
            "plain": small["total"] / (small["plain_ms"] * 1e-3) / 1e9,
            "e2e": {"value": small["total"] / (small["e2e_ms"] * 1e-3) / 1e9, "unit": "GCUPS",
                    "h2d_bytes_per_step": small["ctx_io"][0], "d2h_bytes_per_step": small["ctx_io"][1],
                    "timing": "two batches in flight on a two-slot context",
                    "sync": small["total"] / (small["sync_ms"] * 1e-3) / 1e9,
                    "pipelined": (None if small["pipelined_ms"] is None else
                                  {"value": small["total"] / (small["pipelined_ms"] * 1e-3) / 1e9,
                                   "unit": "GCUPS", "ms_per_step": small["pipelined_ms"],
                                   "timing": "three batches in flight on a three-slot context"}),
                    "session": small["total"] / (small["session_ms"] * 1e-3) / 1e9},
            "gpu_launches_per_step": small["launches"], "tuning": small["tuning"]}
    if chain:
        # about 10 f64/int ops per predecessor evaluation, against this GPU's f64 add/max rate
        ach = CHAIN_OPS_PER_EVAL * chain["pair_evaluations_per_step"] / (chain["ms_per_step"] * 1e-3) / 1e12
        chain["roofline"] = {"bound": "f64 issue", "achieved": ach, "peak": ip["f64_add_max"], "unit": "Tops/s",
                             "frac": ach / ip["f64_add_max"], "ops_per_evaluation": CHAIN_OPS_PER_EVAL,
                             "peak_source": "f64 add/max probe, this GPU"}
        line["chain"] = chain
    if serve:
        line["serving"] = serve
    if longr:
        line["long_reads"] = longr
    if wfa_res:
        line["wfa"] = wfa_res
    if sam_res:
        sam_res["roofline"]["peak"] = peaks["hbm_gbs"]
        sam_res["roofline"]["frac"] = sam_res["roofline"]["achieved"] / peaks["hbm_gbs"]
        sam_res["roofline"]["peak_source"] = peak_src
        line["sam"] = sam_res
    if not args.no_cpu_baseline:
        line["cpu_baseline"], line["parity"] = cpu_baseline(ps, head["params"], head["result"])
    return line


def wfa_leg(args, device, stream, flush, seed: int, warm: int) -> dict:
    """Wavefront alignment of mixed-length reads against their source stretch
    (graphmambaformer_b200.wfa): device time of the distance pass alone and of
    the full alignment (distance pass, history pass, walk), end-to-end time of
    align_wfa_pairs (host lists in, distances and CIGARs out), and the oracle
    on a sample of the pairs on the host cores."""
    import torch

    from graphmambaformer_b200 import synth, wfa

    qs, ts = synth.wfa_pairs_mixed(n_pairs=args.wfa_pairs, seed=seed)
    md = 4096
    dp = wfa.upload_wfa_pairs(qs, ts, device)
    dist = torch.empty(dp.n, dtype=torch.int32, device=device)

    def dstep():
        wfa.wfa_distances(dp, md, stream, out=dist)

    for _ in range(warm):
        dstep()
    torch.cuda.synchronize(device)
    h_dist = dist.to("cpu").numpy().copy()
    d_ms = float(np.mean(time_device(dstep, args.steps, stream, flush)))

    def astep():
        wfa.wfa_distances(dp, md, stream, out=dist)
        wfa._run_align(dp, dist, h_dist, int(stream.cuda_stream))

    for _ in range(warm):
        astep()
    torch.cuda.synchronize(device)
    a_ms = float(np.mean(time_device(astep, max(2, args.steps // 2), stream, flush)))
    # end to end: the pairs as page-locked CSR arrays (WfaBatch) in, distances and CIGARs out
    wb = wfa.WfaBatch.of(qs, ts).pinned()
    wfa.align_wfa_batch(wb, md, device=device)
    e = []
    for _ in range(max(2, args.steps // 4)):
        t0 = time.perf_counter()
        r = wfa.align_wfa_batch(wb, md, device=device)
        e.append((time.perf_counter() - t0) * 1e3)
    e_ms = float(np.mean(e))
    # the same from Python lists of per-pair arrays (the reference's calling form)
    el = []
    for _ in range(2):
        t0 = time.perf_counter()
        wfa.align_wfa_pairs(qs, ts, md, device=device)
        el.append((time.perf_counter() - t0) * 1e3)
    el_ms = float(np.mean(el))
    n = len(qs)
    bases = int(sum(len(q) + len(t) for q, t in zip(qs, ts)))
    hist = int(np.sum(np.where(h_dist >= 0, (h_dist.astype(np.int64) + 1) ** 2, 0)))
    out = {
        "value": n / (a_ms * 1e-3), "unit": "alignments/s", "ms_per_step": a_ms,
        "bases_per_s": bases / (a_ms * 1e-3),
        "distance_only": {"value": n / (d_ms * 1e-3), "unit": "alignments/s", "ms_per_step": d_ms},
        "e2e": {"value": n / (e_ms * 1e-3), "unit": "alignments/s", "ms_per_step": e_ms,
                "h2d_bytes_per_step": bases + 16 * (n + 1),
                # distances, op counts, CIGAR starts and lengths, two counters, the CIGAR words
                "d2h_bytes_per_step": 32 * n + 12 + 4 * int(len(r.cigar_words)),
                "timing": "align_wfa_batch on page-locked CSR pairs",
                "from_lists": {"value": n / (el_ms * 1e-3), "ms_per_step": el_ms,
                               "timing": "align_wfa_pairs on Python lists of per-pair arrays"}},
        "config": {"workload": "wfa_pairs_mixed", "pairs": n, "read_len": "lognormal(7.0, 1.2) clipped to 150-20000",
                   "profiles": "Illumina / HiFi / ONT thirds", "target": "the read's source stretch",
                   "max_distance": md, "bases": bases, "mean_distance": float(h_dist[h_dist >= 0].mean()),
                   "max_distance_seen": int(h_dist.max()), "history_entries": hist},
        "gpu_launches_per_step": 3,
    }
    if not args.no_cpu_baseline:
        from oracle import oracle

        rng = np.random.default_rng(1)
        idx = rng.permutation(n)
        t0 = time.perf_counter()
        done, done_bases = 0, 0
        for b in idx:
            oracle.wfa_align(qs[b], ts[b], md)
            done += 1
            done_bases += len(qs[b]) + len(ts[b])
            if time.perf_counter() - t0 > 10.0:
                break
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": done / dt, "unit": "alignments/s", "bases_per_s": done_bases / dt,
                               "cores": 1, "kind": "port",
                               "sample": f"{done} random pairs of the workload, oracle_wfa_align, one thread"}
    return out


def sam_records_workload(n: int, seed: int):
    """Alignment records of mixed-length reads (150 bp - 20 kb, both
    strands, soft clips, every 31st unmapped) with their reads, as objects
    (ReadAlignments, reads with seq / quals / modality) and as arrays
    (RecordTable, names, ASCII bases, qualities, offsets)."""
    from types import SimpleNamespace

    from graphmambaformer_b200.records import OPS, AlignmentRecord, ReadAlignments, RecordTable

    rng = np.random.default_rng(seed)
    lens = np.clip(rng.lognormal(7.0, 1.2, size=n), 150, 20_000).astype(np.int64)
    pool = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=int(lens.sum()))
    qual = np.zeros(int(lens.sum()), np.uint8)
    results, reads, o = [], [], 0
    cols = {k: [] for k in ("ref_id", "ref_start", "ref_end", "strand", "mapq")}
    words, nwords = [], []
    for i, L in enumerate(lens):
        L = int(L)
        seq = pool[o: o + L].tobytes().decode()
        cl, cr = int(rng.integers(0, 40)), int(rng.integers(0, 40))
        mid = L - cl - cr
        cigar = [("S", cl), ("=", mid // 3), ("X", 1), ("=", mid // 3), ("I", 2), ("=", mid - 2 * (mid // 3) - 3),
                 ("D", 3), ("S", cr)]
        cigar = [x for x in cigar if x[1] > 0]
        rs = int(rng.integers(0, 10 ** 8))
        rec = AlignmentRecord(read_id=f"read{i}", read_len=L, ref_id=0, ref_start=rs, ref_end=rs + mid,
                              strand=1 if i % 2 else -1, mapq=int(rng.integers(0, 61)), cigar=cigar,
                              is_mapped=i % 31 != 0)
        q = rng.integers(0, 60, size=L) if i % 4 == 0 else None
        if q is not None:
            qual[o: o + L] = q
        o += L
        results.append(ReadAlignments(read_id=rec.read_id, read_len=L, records=[rec]))
        reads.append(SimpleNamespace(read_id=rec.read_id, seq=seq, quals=q.tolist() if q is not None else None,
                                     modality="ont"))
        w = [(m << 4) | OPS.index(op) for op, m in cigar] if rec.is_mapped else []
        words.extend(w)
        nwords.append(len(w))
        for k, v in (("ref_id", 0 if rec.is_mapped else -1), ("ref_start", rs), ("ref_end", rs + mid),
                     ("strand", rec.strand), ("mapq", rec.mapq)):
            cols[k].append(v)
    woff = np.zeros(n + 1, np.int64)
    np.cumsum(nwords, out=woff[1:])
    seq_off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=seq_off[1:])
    table = RecordTable(read=np.arange(n, dtype=np.int64), ref_id=np.array(cols["ref_id"], np.int64),
                        ref_start=np.array(cols["ref_start"], np.int64), ref_end=np.array(cols["ref_end"], np.int64),
                        strand=np.array(cols["strand"], np.int8), mapq=np.array(cols["mapq"], np.int32),
                        is_primary=np.ones(n, bool), cigar=np.array(words, np.uint32), cigar_off=woff)
    arrays = dict(table=table, names=[r.read_id for r in reads], seq=pool, seq_off=seq_off, qual=qual)
    return results, reads, arrays


def sam_leg(args, device, stream, flush, warm: int) -> dict:
    """SAM text of alignment records (graphmambaformer_b200.records): device
    time of gmf_sam_count + scan + gmf_sam_fill on device-resident records;
    end to end from the host layout (render_sam: copies in, kernels, text
    out); the host layout itself (sam_records) timed apart; the oracle's
    Python rendering on a sample."""
    import ctypes

    import torch

    from graphmambaformer_b200 import _native
    from graphmambaformer_b200.device import to_device
    from graphmambaformer_b200.records import render_sam, render_sam_array, sam_batch, sam_records

    results, reads, arrays = sam_records_workload(args.sam_records, seed=9)
    t0 = time.perf_counter()
    b = sam_records(results, reads, "ont", False, {0: 10 ** 9})
    layout_ms = (time.perf_counter() - t0) * 1e3
    # the same records held as arrays: bases and qualities in page-locked memory, as a service keeps them
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    seq_p, qual_p = pin(arrays["seq"]), pin(arrays["qual"])

    def table_layout():
        return sam_batch(arrays["table"], arrays["names"], seq_p, arrays["seq_off"], qual_p, "ont", False,
                         {0: 10 ** 9})

    bt = table_layout()
    for f in ("names", "name_off", "seq", "seq_off", "qual", "contig", "contig_names", "contig_off", "ref_start",
              "ref_end", "strand", "mapq", "cigar", "cigar_start", "cigar_len", "tags", "tag_off"):
        if not np.array_equal(getattr(bt, f), getattr(b, f)):
            raise RuntimeError(f"the array layout differs from the object layout in {f}")
    t0 = time.perf_counter()
    table_layout()
    table_layout_ms = (time.perf_counter() - t0) * 1e3
    n = len(b)
    d = {k: to_device(getattr(b, k), device) for k in ("names", "name_off", "seq", "seq_off", "qual", "contig",
                                                        "contig_names", "contig_off", "ref_start", "ref_end",
                                                        "strand", "mapq", "cigar", "cigar_start", "cigar_len",
                                                        "tags", "tag_off")}
    p = {k: v.data_ptr() for k, v in d.items()}
    rec = _native.GmfSamRecords(n, p["names"], p["name_off"], p["seq"], p["seq_off"], p["qual"], p["contig"],
                                p["contig_names"], p["contig_off"], len(b.contig_off) - 1, p["ref_start"],
                                p["ref_end"], p["strand"], p["mapq"], p["cigar"], p["cigar_start"], p["cigar_len"],
                                None, None, p["tags"], p["tag_off"], int(np.diff(b.seq_off).max()))
    lens = torch.empty(n, dtype=torch.int64, device=device)
    off = torch.zeros(n + 1, dtype=torch.int64, device=device)
    sp = int(stream.cuda_stream)
    lib = _native.lib()
    _native.check("gmf_sam_count", lib.gmf_sam_count(ctypes.byref(rec), ctypes.c_void_p(lens.data_ptr()),
                                                     ctypes.c_void_p(sp)))
    torch.cumsum(lens, 0, out=off[1:])
    total = int(off[-1].item())
    text = torch.empty(total, dtype=torch.uint8, device=device)

    def step():
        lib.gmf_sam_count(ctypes.byref(rec), ctypes.c_void_p(lens.data_ptr()), ctypes.c_void_p(sp))
        torch.cumsum(lens, 0, out=off[1:])
        lib.gmf_sam_fill(ctypes.byref(rec), ctypes.c_void_p(off.data_ptr()), ctypes.c_void_p(text.data_ptr()),
                         ctypes.c_void_p(sp))

    for _ in range(warm):
        step()
    torch.cuda.synchronize(device)
    ms = float(np.mean(time_device(step, args.steps, stream, flush)))
    # algorithmic bytes of one step: both passes read each record's 69 B of fields and its CIGAR words; the
    # fill pass reads names, bases, qualities and tags once and writes the text; the count pass writes 8 B
    read_b = int(2 * (69 * n + 4 * b.cigar.size) + b.names.size + b.seq.size + b.qual.size + b.tags.size)
    alg = read_b + total + 8 * n
    h2d = int(sum(getattr(b, k).nbytes for k in ("names", "name_off", "seq", "seq_off", "qual", "contig",
                                                  "contig_names", "contig_off", "ref_start", "ref_end", "strand",
                                                  "mapq", "cigar", "cigar_start", "cigar_len", "tags", "tag_off")))
    keep = [render_sam_array(table_layout(), device) for _ in range(2)]  # both page-locked text buffers made
    del keep
    e = []
    for _ in range(max(2, args.steps // 4)):
        t0 = time.perf_counter()
        out = render_sam_array(table_layout(), device)
        e.append((time.perf_counter() - t0) * 1e3)
    e_ms = float(np.mean(e))
    eb = []
    for _ in range(2):
        t0 = time.perf_counter()
        render_sam(b, device)
        eb.append((time.perf_counter() - t0) * 1e3)
    eb_ms = float(np.mean(eb))
    res = {
        "value": n / (ms * 1e-3), "unit": "records/s", "ms_per_step": ms,
        "text_gb_per_s": total / (ms * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "unit": "GB/s",
                     "bytes_per_step": alg, "text_bytes": total},
        "e2e": {"value": n / (e_ms * 1e-3), "unit": "records/s", "ms_per_step": e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": len(out),
                "timing": "sam_batch + render_sam_array: record table and page-locked read columns in, "
                          "SAM text out in page-locked memory",
                "from_layout_bytes": {"value": n / (eb_ms * 1e-3), "ms_per_step": eb_ms,
                                      "timing": "render_sam on a ready layout, text as bytes"}},
        "host_layout_ms": layout_ms,
        "table_layout_ms": table_layout_ms,
        "config": {"workload": "sam_records_mixed", "records": n, "bases": int(b.seq.size),
                   "read_len": "lognormal(7.0, 1.2) clipped to 150-20000", "strands": "alternating",
                   "qualities": "every 4th read", "unmapped": "every 31st"},
        "gpu_launches_per_step": 3,
    }
    if not args.no_cpu_baseline:
        from oracle import sam

        t0 = time.perf_counter()
        k = 0
        while k < n and time.perf_counter() - t0 < 10.0:
            r, rd = results[k].records[0], reads[k]
            sam.render(sam.segment(vars(r), rd.seq, rd.quals, "ont", {0: 0}), ["ref0"])
            k += 1
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": k / dt, "unit": "records/s", "cores": 1, "kind": "port",
                               "sample": f"first {k} records, oracle segment + render (Python), one thread"}
    return res


def long_read_leg(args, device, stream, flush, seed: int, warm: int) -> dict:
    """Long-read stress: ONT-like reads of 50-100 kb on a 50 Mb reference,
    chained with a 200-anchor window; banded SW over the primary chain's gaps
    (graphmambaformer_b200.longreads).  Device times of the chaining call and
    of the gap-SW call, each the mean of the timed steps."""
    import torch

    from graphmambaformer_b200 import chaining, longreads, synth
    from graphmambaformer_b200.config import ChainingConfig

    from graphmambaformer_b200.seeding import DeviceMinimizerIndex

    # raw (k=15, w=10) minimizer anchors from the reference's index semantics, found on the device
    pool = synth.long_reads_ont(n_reads=args.long_reads, seed=seed,
                                seeder=lambda ref: DeviceMinimizerIndex(ref, k=15, w=10, max_occ=200, device=device))
    al = longreads.LongReadAligner(torch.from_numpy(pool.ref).to(device), device)
    prim, _ = al.primary_chains(pool.reads, pool.anchors)
    seg = al.segments(pool.reads, prim)
    cfg = ChainingConfig(max_lookback=200)
    da = chaining.upload_anchors(pool.anchors, device)
    cout = chaining.ChainOutputs.allocate(da, cfg.max_chains)

    def cstep():
        chaining.launch_chain_batch(da, cfg, out=cout, stream=stream)

    for _ in range(warm):
        cstep()
    torch.cuda.synchronize(device)
    c_ms = float(np.mean(time_device(cstep, args.steps, stream, flush)))
    # gap SW: the segments as a resident pair batch
    from graphmambaformer_b200 import extension

    qs, ts = [], []
    for i in range(len(seg)):
        read = pool.reads[int(seg.read[i])]
        frame = read if seg.strand[i] > 0 else synth.reverse_complement(read)
        qs.append(frame[seg.q_start[i]: seg.q_start[i] + seg.q_len[i]])
        ts.append(pool.ref[seg.t_start[i]: seg.t_start[i] + seg.t_len[i]])
    ps = synth.PairSet.from_lists(qs, ts, seg.half_band, seg.band_offset)
    dp = extension.upload_pairs(ps, device)
    sw_p = extension.params_from_config(al.ecfg)
    out = extension.SWOutputs.allocate(dp, True)
    ws = torch.empty(extension.workspace_bytes(dp, True), dtype=torch.uint8, device=device)

    def sstep():
        extension.launch_banded_sw(dp, sw_p, True, out=out, workspace=ws, stream=stream)

    for _ in range(warm):
        sstep()
    torch.cuda.synchronize(device)
    s_ms = float(np.mean(time_device(sstep, args.steps, stream, flush)))
    cells = ps.cells()
    del out, ws, dp
    torch.cuda.empty_cache()
    # wide segmentation: 8 kb segments with half bands up to 2,000; run as calls of <= 5e10 cells each
    # (0.5 B of traceback bits per cell)
    segw = al.segments(pool.reads, prim, mode=longreads.WIDE)
    qw, tw_ = [], []
    for i in range(len(segw)):
        read = pool.reads[int(segw.read[i])]
        frame = read if segw.strand[i] > 0 else synth.reverse_complement(read)
        qw.append(frame[segw.q_start[i]: segw.q_start[i] + segw.q_len[i]])
        tw_.append(pool.ref[segw.t_start[i]: segw.t_start[i] + segw.t_len[i]])
    psw = synth.PairSet.from_lists(qw, tw_, segw.half_band, segw.band_offset)
    wcells = synth.band_cells(psw.query_len, psw.target_len, psw.half_band, psw.band_offset).astype(np.float64)
    cut = np.searchsorted(np.cumsum(wcells), np.arange(5e10, wcells.sum() + 5e10, 5e10))
    bounds = np.unique(np.concatenate([[0], np.minimum(cut + 1, len(psw))]))
    calls = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        dpc = extension.upload_pairs(psw.subset(np.arange(lo, hi)), device)
        calls.append((dpc, extension.SWOutputs.allocate(dpc, True)))
    wsw = torch.empty(max(extension.workspace_bytes(c[0], True) for c in calls), dtype=torch.uint8, device=device)
    # the scheduling knobs tuned for these uniform wide pairs on a sample (results checked identical)
    from graphmambaformer_b200 import autotune

    before = autotune.get_tuning(device)
    rng = np.random.default_rng(3)
    sample = psw.subset(np.sort(rng.choice(len(psw), size=min(len(psw), 400), replace=False)))
    wrep = autotune.autotune_sw(sample, sw_p, device, reps=2, passes=1)
    del sample

    def wstep():
        for dpc, outc in calls:
            extension.launch_banded_sw(dpc, sw_p, True, out=outc, workspace=wsw, stream=stream)

    wstep()
    torch.cuda.synchronize(device)
    w_ms = float(np.mean(time_device(wstep, max(1, min(args.steps, 3)), stream, flush)))
    w_cells = float(wcells.sum())
    autotune.set_tuning(before, device)
    wide = {"value": w_cells / (w_ms * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": w_ms, "segments": len(segw),
            "cells": w_cells, "max_half_band": int(segw.half_band.max()),
            "median_half_band": float(np.median(segw.half_band)), "calls_per_step": len(calls),
            "tuning": dict(wrep.as_dict(), sample_pairs=400),
            "segmentation": "primary chain cut at anchors >= 8 kb apart; band clip(32 + |drift| + len/4, 32, 2000)"}
    del calls, wsw
    torch.cuda.empty_cache()
    return {"reads": len(pool), "anchors": pool.anchors.n_anchors,
            "chain": {"value": pool.anchors.n_anchors / (c_ms * 1e-3), "unit": "anchors/s", "ms_per_step": c_ms,
                      "lookback": 200},
            "gap_sw": {"value": cells / (s_ms * 1e-3) / 1e9, "unit": "GCUPS", "ms_per_step": s_ms,
                       "segments": len(seg), "cells": cells, "max_half_band": int(seg.half_band.max()),
                       "scoring": "extension defaults 2/4/6/2, x-drop 600"},
            "wide_sw": wide,
            "config": {"reference": "50 Mb uniform", "reads": "ONT-like 5% error (60% indels), 50-100 kb",
                       "anchors": "raw (k=15, w=10) minimizer hits of the reference's index semantics "
                                  "(max_occ 200), found on the device",
                       "segmentation": "primary chain cut at anchors >= 1 kb apart; band clip(32 + |drift| + "
                                       "len/50, 32, 2000)",
                       "sample": f"{len(pool)} of the configuration's 2,000 reads" if len(pool) < 2000 else "full"}}


def serve_leg(args, device, seed: int) -> dict:
    """p50/p99 request latency and throughput of the serving loop at a fixed
    offered load: Poisson arrivals of requests of 1-64 reads drawn from a
    pool of mixed-profile reads (lengths 150 bp - 20 kb) on a 10 Mb
    reference kept on the device, 8 GB working-memory budget."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex
    from graphmambaformer_b200.serving import AlignServer, serve_stream

    pool = synth.mixed_read_pool(n_reads=2000, seed=seed, ref_len=10_000_000)
    index = DeviceMinimizerIndex(pool.ref, k=15, w=10, max_occ=200, device=device)
    srv = AlignServer(pool.ref, device, budget_bytes=8 << 30, workers=4, max_batch_reads=1024, index=index).start()
    loads = [float(x) for x in str(args.serve_loads).split(",") if x]
    points = []
    try:
        # warm-up at the highest load, so every worker's grow-only buffers reach full size first
        warm = synth.poisson_requests(120, max(loads), len(pool), seed=seed + 1)
        serve_stream(srv, pool, warm)
        for i, load in enumerate(loads):
            srv.completed.clear()
            srv.batches = 0
            n_req = max(args.serve_requests, int(1.5 * load / 32.5))  # 1-64 reads per request, 32.5 on average
            reqs = synth.poisson_requests(n_req, load, len(pool), seed=seed + 2 + i)
            st = serve_stream(srv, pool, reqs)
            points.append({"offered_reads_per_s": load, "achieved_reads_per_s": st["reads_per_s"],
                           "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                           "requests": st["requests"], "reads": st["reads"], "batches": st["batches"]})
    finally:
        srv.stop()
    return {**points[-1], "loads": points,
            "config": {"reference": "10 Mb uniform and its (k=15, w=10) minimizer index, resident on the device",
                       "requests": "1-64 bare reads, Poisson arrivals; seeding, chaining and extension on the GPU",
                       "reads": "pool of 2,000 mixed-profile reads (150 bp - 20 kb)",
                       "budget": "8 GB", "workers": 4, "max_batch_reads": 1024,
                       "index_bytes": index.bytes}}


# --------------------------------------------------------------------------- #
# CPU baseline / reference arm
# --------------------------------------------------------------------------- #
def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def stratified_sample(ps, max_cells: float, seed: int = 0) -> np.ndarray:
    """Pair indices of a sample of ``ps`` covering every length decile in
    proportion, about ``max_cells`` in-band cells in total."""
    from graphmambaformer_b200.synth import band_cells

    cells = band_cells(ps.query_len, ps.target_len, ps.half_band, ps.band_offset).astype(np.float64)
    if cells.sum() <= max_cells:
        return np.arange(len(ps))
    rng = np.random.default_rng(seed)
    frac = max_cells / cells.sum()
    order = np.argsort(ps.query_len, kind="stable")
    picks = []
    for dec in np.array_split(order, 10):
        k = max(1, int(round(len(dec) * frac)))
        picks.append(rng.choice(dec, size=min(k, len(dec)), replace=False))
    return np.sort(np.concatenate(picks))


def oracle_sw_rate(ps, params, idx, threads, want_out=False):
    """GCUPS of the C oracle (the reference algorithm, SW + traceback) on the
    pairs ``idx`` of ``ps``; returns (gcups, cells, seconds), plus the
    oracle's outputs when ``want_out``."""
    from graphmambaformer_b200.synth import band_cells
    from oracle import oracle

    qs = [ps.q(int(b)) for b in idx]
    ts = [ps.t(int(b)) for b in idx]
    cs = float(band_cells(ps.query_len[idx], ps.target_len[idx], ps.half_band[idx], ps.band_offset[idx]).sum())
    t0 = time.perf_counter()
    res = oracle.sw_batch(qs, ts, ps.half_band[idx], ps.band_offset[idx], *params, threads=threads)
    dt = time.perf_counter() - t0
    return (cs / dt / 1e9, cs, dt, res) if want_out else (cs / dt / 1e9, cs, dt)


def sw_mismatches(got, want, idx) -> int:
    """Pairs of ``idx`` whose GPU result (``got``, indexed by pair) differs
    from the oracle's (``want``, indexed by sample position) in any field:
    score, ends, starts, op counts or CIGAR."""
    bad = 0
    for k, b in enumerate(idx):
        b = int(b)
        same = (np.float32(got.score[b]) == want.score[k] and got.query_end[b] == want.query_end[k]
                and got.target_end[b] == want.target_end[k] and got.query_start[b] == want.query_start[k]
                and got.target_start[b] == want.target_start[k]
                and np.array_equal(got.op_counts[b], want.counts[k]) and got.cigar(b) == want.cigars[k])
        bad += 0 if same else 1
    return bad


def cpu_baseline(ps, params, got=None, max_cells: float = 6e9):
    """The oracle timed on a stratified sample of the workload; its outputs
    are compared with the GPU's outputs ``got`` of the same pairs.  Returns
    (cpu_baseline dict, parity dict or None)."""
    th = host_threads()
    idx = stratified_sample(ps, max_cells)
    gcups, cs, dt, want = oracle_sw_rate(ps, params, idx, th, want_out=True)
    base = {"value": gcups, "unit": "GCUPS", "cores": th, "kind": "port",
            "sample": f"{len(idx)} pairs ({cs:.3g} cells, every length decile) of the same workload, "
                      f"SW + traceback, C restatement of the reference, {dt:.1f} s"}
    parity = None
    if got is not None:
        parity = {"pairs": int(len(idx)), "mismatches": sw_mismatches(got, want, idx),
                  "fields": "score, ends, starts, op counts, CIGAR of the last timed call vs the oracle"}
    return base, parity


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    ps, params, desc = sw_workload(args.workload, args.pairs, seed=1)
    th = host_threads()
    idx = stratified_sample(ps, 2e9)
    warm_idx = idx[:: max(1, len(idx) // 20)]
    for _ in range(max(args.warmup, 3) if args.warmup else 0):
        oracle_sw_rate(ps, params, warm_idx[:4], th)
    times, cells = [], 0.0
    for _ in range(args.steps):
        _, cells, dt = oracle_sw_rate(ps, params, idx, th)
        times.append(dt)
    ms = float(np.mean(times)) * 1e3
    gcups = cells / (ms * 1e-3) / 1e9
    sample = (f"{len(idx)} pairs ({cells:.3g} cells, every length decile) per step, SW + traceback, "
              f"C restatement of the reference")
    line = {
        "impl": "reference", "metric": METRIC, "value": gcups, "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "float32", "data": "synthetic (seeded)",
        "config": dict(desc, parallelism="host threads"),
        "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": th, "kind": "port", "sample": sample},
        "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_chain:
        from oracle import oracle

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
    """A small single-GPU case for ncu captures: 2,000 pairs of the chosen
    workload (or its N largest pairs), 3 launches of the batched form; or N
    reads of the HiFi chaining workload, 3 launches of the chaining batch."""
    import torch

    from graphmambaformer_b200 import extension

    if args.profile_chain:
        from graphmambaformer_b200 import chaining
        from graphmambaformer_b200.config import ChainingConfig

        cb, _ = chain_workload(args.profile_chain, seed=2)
        cfg = ChainingConfig(max_lookback=50, max_gap=5000)
        da = chaining.upload_anchors(cb, "cuda:0")
        out = chaining.ChainOutputs.allocate(da, cfg.max_chains)
        for _ in range(3):
            chaining.launch_chain_batch(da, cfg, out=out)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "done", "anchors_per_launch": cb.n_anchors}))
        return
    if args.profile_longest:
        ps, params, _ = sw_workload(args.workload, args.pairs, seed=1)
        area = ps.query_len.astype(np.int64) * (2 * ps.half_band.astype(np.int64) + 1)
        ps = ps.subset(np.sort(np.argsort(-area, kind="stable")[: args.profile_longest]))
    else:
        ps, params, _ = sw_workload(args.workload, args.pairs or 2000, seed=1)
    dp = extension.upload_pairs(ps, "cuda:0")
    for _ in range(3):
        extension.launch_banded_sw(dp, extension.sw_params(*params), True)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": "done", "cells_per_launch": ps.cells()}))


def _r(x, nd=4):
    """A figure rounded to ``nd`` significant digits (None stays None)."""
    if x is None:
        return None
    return float(f"{float(x):.{nd}g}")


def compact_summary(line: dict) -> dict:
    """The figures of every leg in a few hundred bytes.  It goes last on the
    line, so that a reader keeping only the end of a long line still sees
    them."""
    s = {"headline_gcups": _r(line.get("value")), "graph_gcups": _r(line.get("graph", {}).get("value")),
         "e2e_gcups": _r(line.get("e2e", {}).get("value")),
         "int_frac": _r(line.get("roofline", {}).get("frac"), 3)}
    pl = line.get("plain")
    if pl:
        s["plain_gcups"] = _r(pl["value"])
        s["batched_over_plain"] = _r(pl["batched_over_plain"], 3)
    sm = line.get("extension_150bp")
    if sm:
        s["bp150"] = {"gcups": _r(sm["value"]), "graph": _r(sm.get("graph")), "plain": _r(sm["plain"]),
                      "e2e": _r(sm["e2e"]["value"])}
    ch = line.get("chain")
    if ch:
        s["chain"] = {"anchors_s": _r(ch["value"]), "ms": _r(ch["ms_per_step"]), "e2e_anchors_s": _r(ch["e2e"]["value"]),
                      "f64_frac": _r(ch.get("roofline", {}).get("frac"), 3)}
    sv = line.get("serving")
    if sv:
        s["serving"] = [{"offered": int(p["offered_reads_per_s"]), "achieved": _r(p["achieved_reads_per_s"]),
                         "p50_ms": _r(p["p50_ms"], 3), "p99_ms": _r(p["p99_ms"], 3)} for p in sv["loads"]]
    lr = line.get("long_reads")
    if lr:
        s["long_reads"] = {"reads": lr["reads"], "chain_anchors_s": _r(lr["chain"]["value"]),
                           "gap_sw_gcups": _r(lr["gap_sw"]["value"]), "max_half_band": lr["gap_sw"]["max_half_band"]}
        if "wide_sw" in lr:
            s["long_reads"]["wide_sw_gcups"] = _r(lr["wide_sw"]["value"])
            s["long_reads"]["wide_max_half_band"] = lr["wide_sw"]["max_half_band"]
    wf = line.get("wfa")
    if wf:
        s["wfa"] = {"aln_s": _r(wf["value"]), "e2e_aln_s": _r(wf.get("e2e", {}).get("value")),
                    "lists_aln_s": _r(wf.get("e2e", {}).get("from_lists", {}).get("value"))}
    sa = line.get("sam")
    if sa:
        s["sam"] = {"records_s": _r(sa["value"]), "e2e_records_s": _r(sa.get("e2e", {}).get("value")),
                    "e2e_ms": _r(sa.get("e2e", {}).get("ms_per_step"), 3), "table_layout_ms": _r(sa.get("table_layout_ms"), 3)}
    if line.get("parity"):
        s["parity"] = {k: line["parity"][k] for k in ("pairs", "mismatches")}
    cb = line.get("cpu_baseline")
    if cb:
        s["cpu_gcups"] = _r(cb["value"])
    return s


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    line = run_reference(args) if args.impl == "reference" else run_b200(args)
    if line is not None:
        if args.impl != "reference":
            line["summary"] = compact_summary(line)
        print(json.dumps(line))


if __name__ == "__main__":
    main()
