"""The allocation-free compaction scan (fpg_compaction_indices_static).

Some callers cannot call cudaMalloc -- their device memory belongs to another
allocator, or an allocation would stall a latency-critical loop -- so this
entry point keeps its scratch in a static device array of the library and
writes only into the caller's buffers.  This test calls it through the C ABI
and checks its indices and active count against the existing fpg_compact
(integer results: bit-exact), on two calls in a row with different inputs,
so that scratch left by the first call cannot leak into the second.

The file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from flexpart_gpu.records import PARTICLE_DTYPE

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")


def _flags(n, seed, density):
    rng = np.random.default_rng(seed)
    return (rng.random(n) < density).astype(np.uint32)


def _existing(ctx, flags):
    """Indices and count from fpg_compact (allocating handles)."""
    n = len(flags)
    rec = np.zeros(n, PARTICLE_DTYPE)
    rec["flags"] = flags
    p = api.Particles(ctx, n)
    p.upload(rec)
    comp = api.Compaction(ctx, n)
    idx = api.DeviceArray(ctx, n, np.uint32)
    count = comp.compact(p, idx)
    return idx.numpy()[:count], count


def _buffers(ctx, flags):
    """Device input and output buffers of one call (uploaded, synchronised)."""
    n = len(flags)
    return (api.DeviceArray.from_numpy(ctx, flags), api.DeviceArray(ctx, n, np.uint32),
            api.DeviceArray(ctx, 1, np.uint32))


def _enqueue(ctx, bufs):
    """Queues one call on the context's stream, with no host synchronisation."""
    d_flags, d_idx, d_cnt = bufs
    st = api._lib.lib.fpg_compaction_indices_static(ctx.h, ctypes.c_void_p(d_flags.ptr), d_flags.n,
                                                    ctypes.c_void_p(d_idx.ptr), ctypes.c_void_p(d_cnt.ptr), None)
    assert st == 0, api._lib.lib.fpg_status_string(st)
    return bufs


def _result(bufs):
    _, d_idx, d_cnt = bufs
    count = int(d_cnt.numpy()[0])
    return d_idx.numpy()[:count], count


def _static(ctx, flags):
    bufs = _enqueue(ctx, _buffers(ctx, flags))
    ctx.synchronize()
    return _result(bufs)


def test_static_scan_matches_fpg_compact_twice():
    ctx = api.Context(0)
    # 3,000,001 slots are 1465 tiles: the single-CTA scan then runs two tiles
    # per thread with a shorter range on the last busy thread
    for n, seed, density in ((300_001, 1, 0.9), (70_000, 2, 0.3), (3_000_001, 3, 0.55)):
        flags = _flags(n, seed, density)
        ref_idx, ref_count = _existing(ctx, flags)
        idx, count = _static(ctx, flags)
        assert count == ref_count == int(flags.sum())
        assert np.array_equal(idx, ref_idx)


def test_static_scan_back_to_back_on_one_stream():
    """Two calls queued on one stream with no host synchronisation between
    them share the scratch array in turn; each result matches fpg_compact."""
    ctx = api.Context(0)
    fa = _flags(2_500_003, 4, 0.2)
    fb = _flags(400_000, 5, 0.8)
    a, b = _buffers(ctx, fa), _buffers(ctx, fb)
    _enqueue(ctx, a)
    _enqueue(ctx, b)
    ctx.synchronize()
    for flags, bufs in ((fa, a), (fb, b)):
        ref_idx, ref_count = _existing(ctx, flags)
        idx, count = _result(bufs)
        assert count == ref_count == int(flags.sum())
        assert np.array_equal(idx, ref_idx)


def test_static_scan_limits():
    ctx = api.Context(0)
    lib = api._lib.lib
    d_cnt = api.DeviceArray(ctx, 1, np.uint32)
    too_big = (65536 * 2048) + 1
    st = lib.fpg_compaction_indices_static(ctx.h, ctypes.c_void_p(d_cnt.ptr), too_big, ctypes.c_void_p(d_cnt.ptr),
                                           ctypes.c_void_p(d_cnt.ptr), None)
    assert st == -4          # FPG_ERR_VALUE_TOO_LARGE, rejected before any launch
    d_cnt.upload(np.array([123], np.uint32))
    assert lib.fpg_compaction_indices_static(ctx.h, None, 0, None, ctypes.c_void_p(d_cnt.ptr), None) == 0
    assert int(d_cnt.numpy()[0]) == 0
