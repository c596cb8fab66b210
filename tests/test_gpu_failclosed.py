"""Fail-closed behaviour under backend errors, and request cancellation.

The reference's C ABI layer clears a call's result buffer before the work and
again after any non-OK backend return (src/cpu/src/ufsecp_gpu_impl.cpp:117-140),
and its engine hook declines on any operational error so that the engine's CPU
path answers (src/gpu/src/gpu_engine_hook.cpp:1-23).  Here the failures are
injected on the host (ufsecp_gpu_ext_inject_fault: the (after + 1)-th fault
point of a context fails as an allocation failure, a launch failure or a
thrown std::bad_alloc; the failing step is simply not made, nothing faults on
the device).  Every result byte of a failed call must read 0 although earlier
chunks of the same call had verdicts written, the right code must come back,
and the context must keep working.  The serving loop must end a failed
request with its code (not hang) and its verdicts cleared, and its cancel
call / cancellation token must release a request's buffers.
"""
import ctypes
import threading
import time

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import schnorr_corpus, ecdsa_corpus

pytestmark = pytest.mark.gpu

KINDS = [(1, uf.UFSECP_ERR_GPU_MEMORY), (2, uf.UFSECP_ERR_GPU_LAUNCH), (3, uf.UFSECP_ERR_GPU_MEMORY)]


@pytest.fixture(scope="module")
def valid_big(oracle):
    """300,000 valid BIP-340 items (a 2,000-item corpus tiled): five pipeline
    chunks of the host-buffer call (16k, 32k, 64k, 128k, the rest)."""
    m, x, s = schnorr_corpus(oracle, 2000, seed=901, tamper=0.0)
    reps = 150
    return tuple(np.ascontiguousarray(np.concatenate([a] * reps)) for a in (m, x, s))


def _arm(ctx, after, kind):
    assert uf.load_library().ufsecp_gpu_ext_inject_fault(ctx.handle, after, kind) == uf.UFSECP_OK


@pytest.mark.parametrize("kind,code", KINDS)
def test_verify_batch_recleared_after_a_mid_call_failure(gpu_ctx, valid_big, kind, code):
    m, x, s = valid_big
    n = len(m)
    L = uf.load_library()
    out = np.full(n, 7, np.uint8)
    # chunk 4's launch fails: chunks 0 and 1 have had their verdicts copied out by then
    _arm(gpu_ctx, 4, kind)
    rc = L.ufsecp_gpu_schnorr_verify_batch(gpu_ctx.handle, m.ctypes.data, x.ctypes.data, s.ctypes.data, n,
                                           out.ctypes.data)
    assert rc == code
    assert not out.any()
    assert (gpu_ctx.schnorr_verify_batch(m, x, s) == 1).all()        # the context keeps working


def test_verify_batch_first_chunk_failure(gpu_ctx, oracle):
    m, p, s = ecdsa_corpus(oracle, 3000, seed=902, tamper=0.0)
    L = uf.load_library()
    out = np.full(len(m), 7, np.uint8)
    _arm(gpu_ctx, 0, 2)
    rc = L.ufsecp_gpu_ecdsa_verify_batch(gpu_ctx.handle, m.ctypes.data, p.ctypes.data, s.ctypes.data, len(m),
                                         out.ctypes.data)
    assert rc == uf.UFSECP_ERR_GPU_LAUNCH and not out.any()
    assert (gpu_ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()


def test_device_call_failure_code(gpu_ctx, valid_big):
    import torch
    m, x, s = (torch.from_numpy(a.reshape(-1)).cuda() for a in valid_big)
    n = len(valid_big[0])
    d_out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    L = uf.load_library()
    torch.cuda.synchronize()
    _arm(gpu_ctx, 0, 1)
    rc = L.ufsecp_gpu_ext_schnorr_verify_device(gpu_ctx.handle, m.data_ptr(), x.data_ptr(), s.data_ptr(), n,
                                                d_out.data_ptr(), None)
    assert rc == uf.UFSECP_ERR_GPU_MEMORY
    gpu_ctx.schnorr_verify_device(m.data_ptr(), x.data_ptr(), s.data_ptr(), n, d_out.data_ptr(), 0)
    torch.cuda.synchronize()
    assert bool(d_out.all())


@pytest.mark.parametrize("kind,code", KINDS)
def test_verify_jobs_fail_closed(gpu_ctx, valid_big, kind, code):
    m, x, s = valid_big
    jobs = [(1, m[:150_000], x[:150_000], s[:150_000]), (1, m[150_000:], x[150_000:], s[150_000:])]
    tab, keep, out_all, offs = uf._job_table(jobs)
    out_all[:] = 7
    L = uf.load_library()
    _arm(gpu_ctx, 2, kind)          # the third sub-call's launch fails, two are on the device or done
    rc = L.ufsecp_gpu_ext_verify_jobs(gpu_ctx.handle, tab.ctypes.data_as(ctypes.POINTER(uf.Job)), len(jobs))
    assert rc == code
    assert not out_all.any()
    got = gpu_ctx.verify_jobs(jobs)
    assert all(g.all() for g in got)


def test_rlc_fail_closed_during_bisection(gpu_ctx, oracle):
    m, x, s = schnorr_corpus(oracle, 4096, seed=903, tamper=0.0)
    m = m.copy()
    m[1234, 3] ^= 1
    L = uf.load_library()
    out = np.full(len(m), 7, np.uint8)
    bok = np.full(1, 7, np.uint8)
    seed = np.arange(32, dtype=np.uint8)
    _arm(gpu_ctx, 1, 1)             # round 0 runs, the first bisection round fails
    rc = L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, m.ctypes.data, x.ctypes.data, s.ctypes.data, len(m),
                                             len(m), seed.ctypes.data, 0, out.ctypes.data, bok.ctypes.data)
    assert rc == uf.UFSECP_ERR_GPU_MEMORY
    assert not out.any() and not bok.any()
    _arm(gpu_ctx, 0, 3)
    rc = L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, m.ctypes.data, x.ctypes.data, s.ctypes.data, len(m),
                                             len(m), seed.ctypes.data, 0, out.ctypes.data, bok.ctypes.data)
    assert rc == uf.UFSECP_ERR_GPU_MEMORY and not out.any()
    got, _ = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=len(m), seed32=bytes(range(32)))
    assert (got == oracle.schnorr_verify_batch(m, x, s)).all()


def test_inject_gating(gpu_ctx):
    L = uf.load_library()
    assert L.ufsecp_gpu_ext_inject_fault(None, 0, 1) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_ext_inject_fault(gpu_ctx.handle, 0, 4) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_inject_fault(gpu_ctx.handle, 0, 0) == uf.UFSECP_OK     # disarm


# ---------------------------------------------------------------- serving --
@pytest.fixture(scope="module")
def served(oracle):
    m, x, s = schnorr_corpus(oracle, 3000, seed=904, tamper=0.05)
    return m, x, s, oracle.schnorr_verify_batch(m, x, s)


def test_server_request_fails_closed(served):
    m, x, s, want = served
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=2, max_launch_items=1024) as srv:
        _arm(sctx, 1, 2)            # the second launch fails: a piece of the 3000-item request
        rid = srv.submit([(1, m, x, s)])
        outs = srv._keep[rid][1]
        with pytest.raises(uf.UfsecpError) as ei:
            srv.wait(rid, 30_000)
        assert ei.value.code == uf.UFSECP_ERR_GPU_LAUNCH
        assert not outs[0].any()
        got = srv.wait(srv.submit([(1, m, x, s)]), 30_000)      # the server keeps serving
        assert (got[0] == want).all()


def test_server_cancel_pending_and_completed(served):
    m, x, s, want = served
    big = tuple(np.ascontiguousarray(np.concatenate([a] * 20)) for a in (m, x, s))
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=1, max_launch_items=4096) as srv:
        first = srv.submit([(1,) + big])                        # 60,000 items: 15 launches on one slot
        second = srv.submit([(1, m, x, s)])
        outs2 = srv._keep[second][1]
        assert srv.cancel(second, 30_000) == uf.UFSECP_OK       # dropped before or while it ran
        assert not outs2[0].any()
        assert srv.cancel(second, 1000) == uf.UFSECP_ERR_BAD_INPUT
        got = srv.wait(first, 60_000)
        assert (got[0] == np.concatenate([want] * 20)).all()
        third = srv.submit([(1, m, x, s)])
        outs3 = srv._keep[third][1]
        while srv.stats()["pending_requests"] or srv.stats()["requests_done"] < 2:
            time.sleep(0.01)
        time.sleep(0.05)
        assert srv.cancel(third, 30_000) == uf.UFSECP_OK        # completed before the call: verdicts stay
        assert (outs3[0] == want).all()


def test_server_cancellation_token(served):
    m, x, s, want = served
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=1, max_launch_items=512) as srv:
        rid = srv.submit_cancellable([(1, m, x, s)], lambda: True)
        outs = srv._keep[rid][1]
        with pytest.raises(uf.UfsecpError) as ei:
            srv.wait(rid, 30_000)
        assert ei.value.code == uf.UFSECP_ERR_CANCELLED
        assert not outs[0].any()
        # a token that turns after the first poll: the first piece ran, the rest is dropped, nothing reads valid
        polls = []
        rid = srv.submit_cancellable([(1, m, x, s)], lambda: polls.append(1) or len(polls) > 1)
        outs = srv._keep[rid][1]
        with pytest.raises(uf.UfsecpError) as ei:
            srv.wait(rid, 30_000)
        assert ei.value.code == uf.UFSECP_ERR_CANCELLED and not outs[0].any()
        # a token that never fires changes nothing
        rid = srv.submit_cancellable([(1, m, x, s)], lambda: False)
        assert (srv.wait(rid, 30_000)[0] == want).all()


@pytest.mark.parametrize("kind,code", KINDS)
def test_rlc_jobs_fail_closed(gpu_ctx, valid_big, kind, code):
    """Kind 2 jobs (BIP-340 by RLC) mixed with kind 1 jobs: a failure in the
    queue part (while the RLC items are being staged) or in the first RLC
    round leaves every verdict byte of the call cleared."""
    m, x, s = valid_big
    jobs = [(1, m[:100_000], x[:100_000], s[:100_000]), (2, m[100_000:200_000], x[100_000:200_000],
                                                          s[100_000:200_000]), (2, m[200_000:], x[200_000:], s[200_000:])]
    L = uf.load_library()
    for after, only_rlc in ((0, False), (0, True)):
        js = jobs[1:] if only_rlc else jobs
        tab, keep, out_all, offs = uf._job_table(js)
        out_all[:] = 7
        _arm(gpu_ctx, after, kind)
        rc = L.ufsecp_gpu_ext_verify_jobs(gpu_ctx.handle, tab.ctypes.data_as(ctypes.POINTER(uf.Job)), len(js))
        assert rc == code
        assert not out_all.any()
    got = gpu_ctx.verify_jobs(jobs)
    assert all(g.all() for g in got)
