"""The allocation-free entry point ufsecp_gpu_ext_verify_jobs_noalloc.

It serves callers that cannot call cudaMalloc (their GPU memory is owned by
another allocator or framework, or they run under a fixed device-memory
budget): they hand over device buffers they own and the library allocates
nothing, keeping the work-queue kernel's scratch in a static device array.
This test calls it through the C ABI on device-resident mixed ECDSA / BIP-340
jobs, twice in a row with different jobs, and requires verdicts bit-identical
to the existing entry point ufsecp_gpu_ext_verify_jobs on the same items (and
to the oracle).  It is kept in its own file so that it runs after every other
test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import ecdsa_corpus, schnorr_corpus

pytestmark = pytest.mark.gpu


def _device_jobs(torch, specs):
    """specs: [(kind, msgs, pubs, sigs)] host arrays -> device tensors + C job array."""
    keep, arr = [], (uf.Job * len(specs))()
    for k, (kind, m, p, s) in enumerate(specs):
        n = len(m)
        dm = torch.from_numpy(np.ascontiguousarray(m)).cuda()
        dp = torch.from_numpy(np.ascontiguousarray(p)).cuda()
        ds = torch.from_numpy(np.ascontiguousarray(s)).cuda()
        do = torch.full((max(n, 1),), 0xEE, dtype=torch.uint8, device="cuda")
        keep.append((dm, dp, ds, do))
        arr[k] = uf.Job(kind, 0, n, dm.data_ptr(), dp.data_ptr(), ds.data_ptr(), do.data_ptr())
    return keep, arr


def _run_noalloc(gpu_ctx, torch, specs):
    """Runs the entry point on device copies of `specs`; returns the verdicts and
    the device's free bytes just before and just after the call (inputs, outputs
    and the stream are created before the first reading)."""
    keep, arr = _device_jobs(torch, specs)
    L = uf.load_library()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = L.ufsecp_gpu_ext_verify_jobs_noalloc(gpu_ctx.handle, arr, len(specs), stream.cuda_stream)
    assert rc == uf.UFSECP_OK, gpu_ctx.last_error_msg()
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    return [keep[k][3][:len(specs[k][1])].cpu().numpy() for k in range(len(specs))], free_before, free_after


def test_no_alloc_matches_existing_entry_point_twice(gpu_ctx, oracle):
    import torch
    e = ecdsa_corpus(oracle, 1500, seed=91, tamper=0.1)
    s = schnorr_corpus(oracle, 2500, seed=92, tamper=0.1)
    first = [(1,) + tuple(x[:1000] for x in s), (0,) + tuple(x[:700] for x in e), (1,) + tuple(x[1000:1001] for x in s),
             (0,) + tuple(x[700:700] for x in e), (0,) + tuple(x[700:1500] for x in e)]
    second = [(0,) + tuple(x[:33] for x in e), (1,) + tuple(x[1001:2500] for x in s)]
    for call, specs in enumerate((first, second)):
        got, free_before, free_after = _run_noalloc(gpu_ctx, torch, specs)
        if call == 1:
            # the point of this entry point: once a device has seen its first
            # call, a call takes no device memory at all
            assert free_after == free_before, (free_before, free_after)
        want = gpu_ctx.verify_jobs(specs)                      # the existing entry point
        for g, w, (kind, m, p, sg) in zip(got, want, specs):
            assert g.shape == w.shape
            assert (g == w).all()
            ref = oracle.ecdsa_verify_batch(m, p, sg) if kind == 0 else oracle.schnorr_verify_batch(m, p, sg)
            assert (g == ref).all()


def test_no_alloc_rejects_too_many_jobs(gpu_ctx):
    L = uf.load_library()
    n = uf_max = 1024
    arr = (uf.Job * (uf_max + 1))()
    rc = L.ufsecp_gpu_ext_verify_jobs_noalloc(gpu_ctx.handle, arr, uf_max + 1, None)
    assert rc == uf.UFSECP_ERR_BAD_INPUT
    assert "1024" in gpu_ctx.last_error_msg()
    assert L.ufsecp_gpu_ext_verify_jobs_noalloc(None, arr, n, None) == uf.UFSECP_ERR_NULL_ARG
