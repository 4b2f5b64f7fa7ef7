"""The allocation-free chaining entry point, gmf_chain_batch_noalloc.

Some callers cannot allocate device memory: a plugin host that passes only
its own input and output buffers, a process whose HBM is all held by a pool
it does not control, or a latency-bound loop that must not call cudaMalloc /
cudaFree because they synchronise the device.  For them the library keeps a
fixed scratch array per GPU and this entry point takes no workspace.

The test calls it through the C ABI twice in a row, on two different batches,
and checks each result against gmf_chain_batch (the entry point with a
caller-supplied workspace) on the same inputs: bit-identical scores, spans,
flags and members, like every chaining parity test here.  The second call
also shows that what the first call left in the shared scratch does not leak
into the next result.  A batch larger than the scratch is refused on the host
with GMF_ERR_LIMIT before anything is launched.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(da, cfg, out):
    from graphmambaformer_b200 import _native, chaining
    from graphmambaformer_b200.device import ptr, stream_handle

    cp = chaining.chain_params(cfg)
    lut = chaining.LUTS.get(da.device, cfg.max_gap, cfg.gap_open, cfg.gap_extend, cfg.log_coeff)
    batch = _native.GmfAnchorBatch(da.n_reads, ptr(da.read_off), ptr(da.read_pos), ptr(da.ref_pos),
                                   ptr(da.length), ptr(da.strand))
    res = _native.GmfChainResults(ptr(out.n_chains), ptr(out.score), ptr(out.strand), ptr(out.span),
                                  ptr(out.is_primary), ptr(out.n_members), ptr(out.members))
    sp = stream_handle(None, da.device)
    return _native.lib().gmf_chain_batch_noalloc(
        ctypes.byref(batch), ctypes.byref(cp), ctypes.c_void_p(lut.data_ptr()), lut.numel(),
        da.n_anchors, ctypes.byref(res), ctypes.c_void_p(sp))


def _same(a, b):
    assert np.array_equal(a.n_chains, b.n_chains)
    R = len(a.n_chains)
    for r in range(R):
        k = int(a.n_chains[r])
        assert np.array_equal(a.score[r, :k].view(np.int64), b.score[r, :k].view(np.int64)), r
        for name in ("strand", "span", "is_primary", "n_members"):
            assert np.array_equal(getattr(a, name)[r, :k], getattr(b, name)[r, :k]), (name, r)
        lo = int(a.read_off[r])
        m = int(a.n_members[r, :k].sum())
        assert np.array_equal(a.members[lo: lo + m], b.members[lo: lo + m]), r


def test_noalloc_chaining_matches_workspace_form_twice():
    import torch

    from graphmambaformer_b200 import _native, chaining, synth
    from graphmambaformer_b200.config import ChainingConfig

    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    batches = [synth.chaining_reads_hifi(n_reads=24, seed=901, ref_len=2_000_000, mean_len=15_000),
               synth.chaining_reads_hifi(n_reads=40, seed=902, ref_len=2_000_000, mean_len=6_000)]
    for b in batches:
        a = chaining.AnchorCSR.of(b)
        assert _native.lib().gmf_chain_workspace_bytes(len(a), int(a.read_off[-1])) \
            <= _native.CHAIN_NOALLOC_SCRATCH_BYTES
        da = chaining.upload_anchors(a, "cuda:0")
        want = chaining.fetch_chains(chaining.launch_chain_batch(da, cfg), a.read_off)
        out = chaining.ChainOutputs.allocate(da, cfg.max_chains)
        for t in (out.n_chains, out.score, out.strand, out.span, out.is_primary, out.n_members, out.members):
            t.fill_(-7)  # stale values must all be overwritten
        st = _noalloc(da, cfg, out)
        assert st == _native.GMF_OK, _native.status_string(st)
        got = chaining.fetch_chains(out, a.read_off)
        torch.cuda.synchronize()
        assert int(want.n_chains.sum()) > 0
        _same(got, want)


def test_noalloc_chaining_refuses_batches_beyond_its_scratch():
    import torch

    from graphmambaformer_b200 import _native, chaining
    from graphmambaformer_b200.config import ChainingConfig

    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    a = chaining.AnchorCSR(np.array([0, 4], np.int64), np.arange(4, dtype=np.int32),
                           np.arange(4, dtype=np.int32), np.full(4, 15, np.int32), np.ones(4, np.int8))
    da = chaining.upload_anchors(a, "cuda:0")
    out = chaining.ChainOutputs.allocate(da, cfg.max_chains)
    too_many = _native.CHAIN_NOALLOC_SCRATCH_BYTES // 16  # claims far more anchors than fit
    da_big = chaining.DeviceAnchors(da.n_reads, too_many, da.read_off, da.read_pos, da.ref_pos,
                                    da.length, da.strand, da.device)
    assert _noalloc(da_big, cfg, out) == _native.GMF_ERR_LIMIT  # refused before any launch
    assert _noalloc(da, cfg, out) == _native.GMF_OK
    torch.cuda.synchronize()
    assert int(out.n_chains[0].item()) >= 0


def test_noalloc_chaining_reports_reads_it_could_not_chain():
    """An understated n_anchors leaves the later reads outside the scratch's
    sorted layout: those reads get zero chains, the call still returns
    GMF_OK, and gmf_chain_noalloc_error_flags reports bit 4.  A correct call
    afterwards clears the word again."""
    import torch

    from graphmambaformer_b200 import _native, chaining, synth
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.device import stream_handle

    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    b = synth.chaining_reads_hifi(n_reads=6, seed=903, ref_len=2_000_000, mean_len=6_000)
    a = chaining.AnchorCSR.of(b)
    da = chaining.upload_anchors(a, "cuda:0")
    want = chaining.fetch_chains(chaining.launch_chain_batch(da, cfg), a.read_off)
    assert (want.n_chains > 0).all()
    flags = torch.full((1,), -1, dtype=torch.int32, device="cuda:0")
    sp = stream_handle(None, da.device)

    def error_flags():
        st = _native.lib().gmf_chain_noalloc_error_flags(ctypes.c_void_p(flags.data_ptr()), ctypes.c_void_p(sp))
        assert st == _native.GMF_OK, _native.status_string(st)
        return int(flags.item())

    short = chaining.DeviceAnchors(da.n_reads, int(a.read_off[2]), da.read_off, da.read_pos, da.ref_pos,
                                   da.length, da.strand, da.device)  # room for the first two reads only
    out = chaining.ChainOutputs.allocate(da, cfg.max_chains)
    assert _noalloc(short, cfg, out) == _native.GMF_OK
    got = chaining.fetch_chains(out, a.read_off)
    assert np.array_equal(got.n_chains[:2], want.n_chains[:2])
    assert (got.n_chains[2:] == 0).all()
    assert error_flags() & 4
    assert _noalloc(da, cfg, out) == _native.GMF_OK
    _same(chaining.fetch_chains(out, a.read_off), want)
    assert error_flags() == 0
