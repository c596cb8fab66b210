"""Serving loop (ufsecp_gpu_ext_server_*): continuous batching of verify requests.

The property that matters: every request's verdicts are the same whether it is
verified alone (one plain per-kind call) or inside the mix the server builds
from whatever else is in flight, and equal to the oracle.  Requests of
log-uniform sizes in [1, 4096], ECDSA / BIP-340 / both, with repeated keys and
tampered signatures, are submitted from several threads at once; launches must
overlap (more than one slot in flight), large requests are cut across launches,
and the memory budget bounds the bytes in flight.
"""
import threading

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import ecdsa_corpus, schnorr_corpus

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pools(oracle):
    e = ecdsa_corpus(oracle, 6000, seed=501, tamper=0.05)
    s = schnorr_corpus(oracle, 9000, seed=502, tamper=0.05)
    return e, s


def _requests(pools, n_req, seed):
    (em, ep, es), (sm, sp, ss) = pools
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_req):
        size = int(np.clip(np.exp(rng.uniform(0, np.log(4096))), 1, 4096))
        n_e = int(round(size * 0.3)) if rng.random() < 0.8 else (size if rng.random() < 0.5 else 0)
        n_s = size - n_e
        jobs = []
        if n_e:
            idx = rng.integers(0, len(em), n_e)      # keys repeat across requests
            jobs.append((0, em[idx], ep[idx], es[idx]))
        if n_s:
            idx = rng.integers(0, len(sm), n_s)
            jobs.append((1, sm[idx], sp[idx], ss[idx]))
        reqs.append(jobs)
    return reqs


def _alone(ctx, jobs):
    return [ctx.ecdsa_verify_batch(m, p, s) if k == 0 else ctx.schnorr_verify_batch(m, p, s) for k, m, p, s in jobs]


def _oracle(oracle, jobs):
    return [oracle.ecdsa_verify_batch(m, p, s) if k == 0 else oracle.schnorr_verify_batch(m, p, s)
            for k, m, p, s in jobs]


def test_results_same_alone_and_in_the_mix(gpu_ctx, oracle, pools):
    reqs = _requests(pools, 240, seed=7)
    results = [None] * len(reqs)
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=4, max_launch_items=8192) as srv:
        def client(lo, hi):
            ids = [(i, srv.submit(reqs[i])) for i in range(lo, hi)]
            for i, rid in ids:
                results[i] = srv.wait(rid)
        threads = [threading.Thread(target=client, args=(k * 60, (k + 1) * 60)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = srv.stats()
    assert st["requests_done"] == len(reqs)
    assert st["items_done"] == sum(len(m) for jobs in reqs for _, m, _, _ in jobs)
    assert st["peak_slots_in_flight"] > 1            # launches overlapped on the device
    assert st["launches"] < len(reqs)                 # requests were batched together
    assert 0 < st["p50_us"] <= st["p99_us"] <= st["max_us"]
    for jobs, got in zip(reqs, results):
        alone = _alone(gpu_ctx, jobs)
        want = _oracle(oracle, jobs)
        assert len(got) == len(jobs)
        for g, a, w in zip(got, alone, want):
            assert (g == a).all() and (g == w).all()


def test_large_request_is_cut_across_launches(oracle, pools):
    (em, ep, es), (sm, sp, ss) = pools
    rng = np.random.default_rng(9)
    idx = rng.integers(0, len(sm), 150_000)
    jobs = [(1, sm[idx], sp[idx], ss[idx]), (0, em[:1000], ep[:1000], es[:1000])]
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=2, max_launch_items=65536) as srv:
        out = srv.wait(srv.submit(jobs))
        st = srv.stats()
    assert st["launches"] >= 3
    assert (out[0] == oracle.schnorr_verify_batch(*jobs[0][1:])).all()
    assert (out[1] == oracle.ecdsa_verify_batch(*jobs[1][1:])).all()


def test_memory_budget_bounds_bytes_in_flight(oracle, pools):
    reqs = _requests(pools, 60, seed=11)
    with uf.GpuContext(0) as sctx:
        with uf.Server(sctx, slots=4, max_launch_items=4096) as probe:
            reserved = probe.stats()["reserved_bytes"]          # fixed staging of 4 slots
        budget = reserved + (1 << 20)                          # room for ~4000 items in flight
        with uf.Server(sctx, slots=4, max_launch_items=4096, memory_budget_bytes=budget) as srv:
            ids = [srv.submit(r) for r in reqs]
            outs = [srv.wait(i) for i in ids]
            st = srv.stats()
    assert st["reserved_bytes"] == reserved
    assert reserved < st["peak_budget_bytes"] <= budget
    for jobs, got in zip(reqs, outs):
        for g, w in zip(got, _oracle(oracle, jobs)):
            assert (g == w).all()


def test_server_gating(gpu_ctx):
    L = uf.load_library()
    h = uf._vp()
    bad = uf.ServerConfig(0, 1024, 8 << 30, 0, 0)
    assert L.ufsecp_gpu_ext_server_create(gpu_ctx.handle, bad, h) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_server_create(None, None, h) == uf.UFSECP_ERR_NULL_ARG
    with uf.GpuContext(0) as sctx, uf.Server(sctx) as srv:
        assert L.ufsecp_gpu_ext_server_wait(srv._h, 12345, 1) == uf.UFSECP_ERR_BAD_INPUT
        arr = (uf.Job * 1)()
        arr[0] = uf.Job(2, 0, 1, None, None, None, None)
        rid = uf.ctypes.c_uint64()
        assert L.ufsecp_gpu_ext_server_submit(srv._h, arr, 1, rid) == uf.UFSECP_ERR_BAD_INPUT
        # an empty request completes at once
        assert L.ufsecp_gpu_ext_server_submit(srv._h, arr, 0, rid) == uf.UFSECP_OK
        assert L.ufsecp_gpu_ext_server_wait(srv._h, rid.value, 1000) == uf.UFSECP_OK


@pytest.mark.parametrize("cache_log2", [1, 8, 17])
def test_resident_key_cache_keeps_verdicts(oracle, pools, cache_log2):
    """Same requests with no cache, a tiny cache that overflows (256 slots, many
    keys) and a 2^17-slot cache: identical verdicts, and hits when cached."""
    reqs = _requests(pools, 80, seed=13)
    reqs = reqs + reqs            # the second pass sees every key again
    with uf.GpuContext(0) as sctx, uf.Server(sctx, slots=2, max_launch_items=4096,
                                             key_cache_log2=cache_log2) as srv:
        outs = [srv.wait(srv.submit(r)) for r in reqs]
        st = srv.stats()
    for jobs, got in zip(reqs, outs):
        for g, w in zip(got, _oracle(oracle, jobs)):
            assert (g == w).all()
    if cache_log2 == 1:
        assert st["cache_lookups"] == 0
    else:
        assert st["cache_lookups"] > 0 and st["cache_hits"] > 0
        if cache_log2 == 17:
            assert st["cache_hits"] >= st["cache_lookups"] // 3
