"""clue_make_clusters_noalloc: the pipeline for callers that cannot allocate device memory.

Such callers (a runtime that hands out every byte of device memory from its own pool, or a
latency-critical path that cannot take cudaMalloc's implicit synchronisation) pass their own
device inputs and outputs; the entry point keeps its intermediate buffers in a fixed 6 MiB
file-scope device array.  These tests call it through the C ABI and compare every output with
the allocating entry point clue_make_clusters, bit for bit (the tolerance of the flat-kernel
parity tests; the exponential kernel takes the same density sweep in both, so it matches bit
for bit too), on two different calls in a row so that contents left in the shared array by
the first call cannot leak into the second, and at the largest request that fits in 8
dimensions.  This file sorts last so that a stop-at-first-
failure run has executed every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_run(fn_noalloc, ctx, coords, weight, params, kernel, metric):
    import torch
    from cluestering_alpaka3_b200 import capi
    ndim, n = coords.shape
    dc = torch.from_numpy(np.ascontiguousarray(coords)).cuda()
    dw = torch.from_numpy(weight).cuda()
    outs = {k: torch.full((n,), -7, dtype=dt, device="cuda") for k, dt in
            (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
             ("nearest_higher", torch.int32), ("delta", torch.float32))}
    o = capi._Outputs()
    for k, v in outs.items():
        setattr(o, k, v.data_ptr())
    p, kk, m = params.struct(), kernel.struct(), metric.struct(ndim)
    info = capi._RunInfo()
    torch.cuda.synchronize()
    if fn_noalloc:
        st = capi.lib.clue_make_clusters_noalloc(ctypes.byref(p), ctypes.byref(kk), ctypes.byref(m), ndim, n,
                                                  ctypes.c_void_p(dc.data_ptr()), ctypes.c_void_p(dw.data_ptr()),
                                                  ctypes.byref(o), None, ctypes.byref(info))
    else:
        st = capi.lib.clue_make_clusters(ctx.handle, ctypes.byref(p), ctypes.byref(kk), ctypes.byref(m), ndim, n,
                                         ctypes.c_void_p(dc.data_ptr()), ctypes.c_void_p(dw.data_ptr()),
                                         ctypes.byref(o), capi.MEM_DEVICE, None, ctypes.byref(info))
    capi.check(st)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}, info


def test_noalloc_matches_allocating_entry_point(gpu_context):
    from cluestering_alpaka3_b200 import capi, synthetic
    rng = np.random.default_rng(2024)
    cases = [synthetic.blobs_2d_16k(n=20000, seed=77), None]
    # second call: different size, dimensionality and data than the first
    c3 = np.concatenate([rng.normal(c, 0.8, size=(600, 3)) for c in rng.uniform(0, 40, size=(6, 3))]).T
    c3 = np.ascontiguousarray(c3.astype(np.float32))
    w3 = rng.uniform(0.5, 1.5, size=c3.shape[1]).astype(np.float32)
    for call, wl in enumerate(cases):
        if wl is not None:
            coords, weight, params = wl.coords, wl.weight, capi.Params(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
        else:
            coords, weight, params = c3, w3, capi.Params(dc=1.0, rhoc=3.0, dm=1.5)
        kernel, metric = capi.FlatKernel(0.5), capi.Metric()
        got, info_a = _device_run(True, None, coords, weight, params, kernel, metric)
        ref, info_b = _device_run(False, gpu_context, coords, weight, params, kernel, metric)
        for k in ("cluster_index", "is_seed", "nearest_higher"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"call {call}: {k}")
        for k in ("rho", "delta"):
            np.testing.assert_array_equal(got[k].view(np.uint32), ref[k].view(np.uint32), err_msg=f"call {call}: {k}")
        assert info_a.n_clusters == info_b.n_clusters > 0
        assert info_a.n_seeds == info_b.n_seeds


def test_noalloc_exponential_kernel_and_8d_limit(gpu_context):
    # The exponential kernel takes the symmetric density sweep in both entry points (the fixed
    # scratch holds its buffers), so the outputs agree bit for bit here too; in 8 dimensions
    # (three float4 words per record) the largest request that fits is a little below 32768
    # points: it runs and agrees, one point more is refused with the limit in the message.
    import re
    from cluestering_alpaka3_b200 import capi
    from parity_util import random_blobs
    rng = np.random.default_rng(77)
    c2, w2 = random_blobs(rng, 12000, 2, nblobs=8, extent=60.0)
    p2 = capi.Params(dc=2.0, rhoc=4.0, dm=3.0)
    got, ia = _device_run(True, None, c2, w2, p2, capi.ExponentialKernel(1.0, 1.0), capi.Metric())
    ref, ib = _device_run(False, gpu_context, c2, w2, p2, capi.ExponentialKernel(1.0, 1.0), capi.Metric())
    for k in ("cluster_index", "is_seed", "nearest_higher", "rho", "delta"):
        np.testing.assert_array_equal(got[k].view(np.uint32), ref[k].view(np.uint32), err_msg=f"exp: {k}")
    assert ia.n_clusters == ib.n_clusters > 0

    p8 = capi.Params(dc=3.0, rhoc=3.0, dm=4.0)
    ps, ks, ms = p8.struct(), capi.FlatKernel(0.5).struct(), capi.Metric().struct(8)
    o = capi._Outputs()
    o.cluster_index = 16  # never dereferenced: the request is refused before any work
    st = capi.lib.clue_make_clusters_noalloc(ctypes.byref(ps), ctypes.byref(ks), ctypes.byref(ms), 8, 32768,
                                             ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.byref(o), None, None)
    assert st == capi.ERR_CAPACITY
    limit = int(re.search(r"at most (\d+) in 8 dimensions", capi.last_error()).group(1))
    assert 29000 < limit < 32768
    c8, w8 = random_blobs(rng, limit, 8, nblobs=6, extent=40.0)
    got, ia = _device_run(True, None, c8, w8, p8, capi.FlatKernel(0.5), capi.Metric())
    ref, ib = _device_run(False, gpu_context, c8, w8, p8, capi.FlatKernel(0.5), capi.Metric())
    for k in ("cluster_index", "is_seed", "nearest_higher", "rho", "delta"):
        np.testing.assert_array_equal(got[k].view(np.uint32), ref[k].view(np.uint32), err_msg=f"8-D: {k}")
    st = capi.lib.clue_make_clusters_noalloc(ctypes.byref(ps), ctypes.byref(ks), ctypes.byref(ms), 8, limit + 1,
                                             ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.byref(o), None, None)
    assert st == capi.ERR_CAPACITY and f"at most {limit}" in capi.last_error()


def test_noalloc_rejects_oversized_requests():
    from cluestering_alpaka3_b200 import capi
    p, k, m = capi.Params(dc=1.0, rhoc=1.0).struct(), capi.FlatKernel(0.5).struct(), capi.Metric().struct(2)
    o = capi._Outputs()
    o.cluster_index = 16  # never dereferenced: the size check comes first
    st = capi.lib.clue_make_clusters_noalloc(ctypes.byref(p), ctypes.byref(k), ctypes.byref(m), 2, 32769,
                                             ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.byref(o), None, None)
    assert st == capi.ERR_CAPACITY
    assert "32768" in capi.last_error()
