"""Mixed ECDSA / BIP-340 batches through ufsecp_gpu_ext_verify_jobs (one
persistent work-queue launch per call, CUDA graphs per capacity bucket):
verdicts must equal the per-kind plain calls and the oracle item for item."""
import ctypes

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import ecdsa_corpus, schnorr_corpus

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def corpora(oracle):
    e = ecdsa_corpus(oracle, 6000, seed=81, tamper=0.05)
    s = schnorr_corpus(oracle, 6000, seed=82, tamper=0.05)
    return e, s, oracle.ecdsa_verify_batch(*e), oracle.schnorr_verify_batch(*s)


def _slice(c, lo, hi):
    return tuple(x[lo:hi] for x in c)


def test_mixed_uneven_batches(gpu_ctx, corpora):
    (e, s, we, ws) = corpora
    rng = np.random.default_rng(5)
    jobs, want = [], []
    pe = ps = 0
    for k in range(60):
        kind = int(rng.random() < 0.3) ^ 1          # ~70% BIP-340
        size = int(np.exp(rng.uniform(0, np.log(300))))
        if k % 17 == 0:
            size = 0
        if kind == 0:
            size = min(size, 6000 - pe)
            jobs.append((0,) + _slice(e, pe, pe + size))
            want.append(we[pe:pe + size])
            pe += size
        else:
            size = min(size, 6000 - ps)
            jobs.append((1,) + _slice(s, ps, ps + size))
            want.append(ws[ps:ps + size])
            ps += size
    got = gpu_ctx.verify_jobs(jobs)
    assert len(got) == len(jobs)
    for g, w in zip(got, want):
        assert (g == w).all()


@pytest.mark.parametrize("lanes", [1, 2])
def test_queue_lanes_per_signature(gpu_ctx, corpora, lanes):
    """Small mixed layouts run the one-lane or the two-lane queue kernels
    (ufsecp_gpu_ext_set_lanes for both kinds); both give the oracle's verdicts
    over every bucket shape, and switching back and forth replays no stale
    graph."""
    (e, s, we, ws) = corpora
    old = [gpu_ctx.get_lanes(k) for k in (0, 1)]
    try:
        for k in (0, 1):
            gpu_ctx.set_lanes(k, lanes, 1 << 16)
        for n_e, n_s in [(1, 0), (0, 1), (17, 33), (255, 257), (1000, 3000), (6000, 6000)]:
            jobs = [(0,) + _slice(e, 0, n_e), (1,) + _slice(s, 0, n_s)]
            ge, gs = gpu_ctx.verify_jobs(jobs)
            assert (ge == we[:n_e]).all() and (gs == ws[:n_s]).all()
    finally:
        for k in (0, 1):
            gpu_ctx.set_lanes(k, *((2, old[k][1]) if old[k][0] == 2 else (1, 0)))


def test_graph_buckets_replay(gpu_ctx, corpora):
    """Repeated calls hitting the same and different capacity buckets stay exact."""
    (e, s, we, ws) = corpora
    for n_e, n_s in [(1, 1), (255, 0), (0, 257), (300, 900), (300, 900), (2000, 3000), (5, 5999), (6000, 6000)]:
        jobs = [(0,) + _slice(e, 0, n_e), (1,) + _slice(s, 0, n_s)]
        ge, gs = gpu_ctx.verify_jobs(jobs)
        assert (ge == we[:n_e]).all() and (gs == ws[:n_s]).all()


def test_direct_path_large(gpu_ctx, oracle):
    """A call above 65,536 items is cut into sub-calls on two batch slots (a
    job split across them keeps its verdicts in place)."""
    base = 4096
    m, x, s = schnorr_corpus(oracle, base, seed=83, tamper=0.1)
    w = oracle.schnorr_verify_batch(m, x, s)
    reps = 20
    big = (1, np.tile(m, (reps, 1)), np.tile(x, (reps, 1)), np.tile(s, (reps, 1)))
    me, pe, se = ecdsa_corpus(oracle, 777, seed=84, tamper=0.1)
    we = oracle.ecdsa_verify_batch(me, pe, se)
    gs, ge = gpu_ctx.verify_jobs([big, (0, me, pe, se)])
    assert (gs == np.tile(w, reps)).all() and (ge == we).all()


def test_large_call_many_subcalls(gpu_ctx, oracle):
    """Large jobs of both kinds and small ones between them, over more than two
    65,536-item sub-calls (each slot reused), keep every verdict in place."""
    base = 2048
    m, x, s = schnorr_corpus(oracle, base, seed=85, tamper=0.1)
    ws = oracle.schnorr_verify_batch(m, x, s)
    me, pe, se = ecdsa_corpus(oracle, base, seed=86, tamper=0.1)
    we = oracle.ecdsa_verify_batch(me, pe, se)
    tile = lambda a, n: np.ascontiguousarray(np.tile(a, (-(-n // base), 1))[:n])
    sizes = [(0, 40_000), (1, 70_001), (0, 3), (1, 0), (0, 30_001), (1, 65_536), (0, 1), (1, 17)]
    jobs, want = [], []
    for kind, n in sizes:
        if kind == 0:
            jobs.append((0, tile(me, n), tile(pe, n), tile(se, n)))
            want.append(np.tile(we, -(-n // base) if n else 1)[:n])
        else:
            jobs.append((1, tile(m, n), tile(x, n), tile(s, n)))
            want.append(np.tile(ws, -(-n // base) if n else 1)[:n])
    got = gpu_ctx.verify_jobs(jobs)
    for g, w in zip(got, want):
        assert g.shape == w.shape and (g == w).all()


def test_jobs_buffer_forms(gpu_ctx, corpora):
    """Jobs given as read-only arrays, bytes, 2-D arrays and lists verify like flat arrays."""
    (e, s, we, ws) = corpora
    ro = [np.frombuffer(a.tobytes(), np.uint8) for a in e]
    jobs = [(0,) + tuple(ro), (1, bytes(s[0]), bytearray(s[1]), s[2].reshape(-1, 64)),
            (1, s[0][:3].tolist(), s[1][:3], s[2][:3]), (0, e[0][:0], e[1][:0], e[2][:0])]
    got = gpu_ctx.verify_jobs(jobs)
    assert (got[0] == we).all() and (got[1] == ws).all() and (got[2] == ws[:3]).all() and got[3].size == 0


def test_same_verdicts_as_plain_calls(gpu_ctx, corpora):
    (e, s, we, ws) = corpora
    ge, gs = gpu_ctx.verify_jobs([(0,) + e, (1,) + s])
    assert (ge == gpu_ctx.ecdsa_verify_batch(*e)).all()
    assert (gs == gpu_ctx.schnorr_verify_batch(*s)).all()


def test_jobs_gating(gpu_ctx):
    L = uf.load_library()
    h = gpu_ctx.handle
    assert L.ufsecp_gpu_ext_verify_jobs(None, None, 1) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_ext_verify_jobs(h, None, 0) == uf.UFSECP_OK
    out = np.full(4, 7, np.uint8)
    j = (uf.Job * 1)(uf.Job(0, 0, 4, None, None, None, out.ctypes.data))
    assert L.ufsecp_gpu_ext_verify_jobs(h, j, 1) == uf.UFSECP_ERR_NULL_ARG
    assert (out == 0).all()                      # cleared before the NULL check
    buf = np.zeros(64 * 4, np.uint8)
    j = (uf.Job * 1)(uf.Job(3, 0, 4, buf.ctypes.data, buf.ctypes.data, buf.ctypes.data, out.ctypes.data))
    assert L.ufsecp_gpu_ext_verify_jobs(h, j, 1) == uf.UFSECP_ERR_BAD_INPUT


def test_job_ranges_equal_job_lists(gpu_ctx, corpora):
    """verify_job_ranges (job table built by vector operations from index
    ranges of per-kind corpora) gives the verdicts of the same jobs passed as a
    job list, and leaves items no job covers at 0."""
    (e, s, we, ws) = corpora
    rng = np.random.default_rng(17)
    kinds, starts, counts = [], [], []
    for kind, n in ((0, 6000), (1, 6000)):
        pos = 0
        while pos < n - 400:
            c = int(rng.integers(0, 300))
            kinds.append(kind)
            starts.append(pos)
            counts.append(c)
            pos += c + int(rng.integers(0, 3))          # small gaps: uncovered items
    got = gpu_ctx.verify_job_ranges({0: e, 1: s}, kinds, starts, counts)
    covered = {0: np.zeros(6000, bool), 1: np.zeros(6000, bool)}
    for k, st, c in zip(kinds, starts, counts):
        covered[k][st:st + c] = True
    for k, w in ((0, we), (1, ws)):
        assert (got[k][covered[k]] == w[covered[k]]).all()
        assert (got[k][~covered[k]] == 0).all()
    with pytest.raises(ValueError):
        gpu_ctx.verify_job_ranges({0: e}, [0], [5990], [20])


def _flip_bit(c, idx):
    m, x, s = (a.copy() for a in c)
    for i in idx:
        s[i, 40] ^= 0x04
    return m, x, s


@pytest.mark.parametrize("pattern", ["valid", "one_invalid", "dense"])
def test_rlc_job_kind(gpu_ctx, oracle, corpora, pattern):
    """Kind 2 jobs (BIP-340 checked by one RLC batch over all of the call's
    kind 2 items, locate step and bisection down to per-item verdicts) mixed
    with kind 0 / 1 jobs: every verdict equals the oracle's, for all-valid
    items, one invalid item in a segment and dense invalid items, with the
    default and with small segment lengths."""
    (e, s, we, ws) = corpora
    clean = schnorr_corpus(oracle, 5000, seed=83, tamper=0.0)
    if pattern == "one_invalid":
        clean = _flip_bit(clean, [1234])
    elif pattern == "dense":
        clean = _flip_bit(clean, range(7, 5000, 9))
    want_rlc = oracle.schnorr_verify_batch(*clean)
    for segment in (0, 256, 1000):
        jobs = [(0,) + _slice(e, 0, 700), (2,) + _slice(clean, 0, 1500) + (segment,), (1,) + _slice(s, 0, 900),
                (2,) + _slice(clean, 1500, 1501), (2,) + _slice(clean, 1501, 1501), (2,) + _slice(clean, 1501, 5000)]
        got = gpu_ctx.verify_jobs(jobs)
        assert (got[0] == we[:700]).all() and (got[2] == ws[:900]).all()
        assert (np.concatenate([got[1], got[3], got[4], got[5]]) == want_rlc).all(), segment


def test_rlc_job_kind_gating(gpu_ctx):
    L = uf.load_library()
    m = np.zeros((4, 32), np.uint8)
    x = np.zeros((4, 32), np.uint8)
    sg = np.zeros((4, 64), np.uint8)
    out = np.full(4, 7, np.uint8)
    tab = np.zeros(1, uf._JOB_DTYPE)
    tab[0] = (3, 0, 4, m.ctypes.data, x.ctypes.data, sg.ctypes.data, out.ctypes.data)
    P = ctypes.POINTER(uf.Job)
    assert L.ufsecp_gpu_ext_verify_jobs(gpu_ctx.handle, tab.ctypes.data_as(P), 1) == uf.UFSECP_ERR_BAD_INPUT
    assert not out.any()
    tab[0]["kind"] = 2
    out[:] = 7
    assert L.ufsecp_gpu_ext_verify_jobs(gpu_ctx.handle, tab.ctypes.data_as(P), 1) == uf.UFSECP_OK
    assert not out.any()                       # s = 0 fails the strict parse
    assert L.ufsecp_gpu_ext_verify_jobs_noalloc(gpu_ctx.handle, tab.ctypes.data_as(P), 1, None) == \
        uf.UFSECP_ERR_BAD_INPUT


def test_rlc_job_kind_beyond_one_pass(gpu_ctx):
    """More kind 2 items than one RLC pass takes (2^24): the jobs are cut
    between passes (one job straddles the boundary) and every verdict lands
    in its own job's buffer.  Items are a GPU-signed, all-valid 2^20 corpus
    tiled, with three invalid items (one flipped bit of s) on both sides of
    the cut; verdicts by construction."""
    import torch
    from ultrafastsecp256k1_b200.autotune import signed_batch
    base = 1 << 20
    d_m, d_x, d_s = signed_batch(gpu_ctx, torch, 1, base, seed=97)
    d_s.view(base, 64)[::50, 40] ^= 0x04   # undo signed_batch's flips: an all-valid corpus
    m0, x0, s0 = (t.cpu().numpy().reshape(base, -1) for t in (d_m, d_x, d_s))
    want0 = np.ones(base, np.uint8)
    reps, extra = 16, 5000
    n = reps * base + extra
    m = np.concatenate([m0] * reps + [m0[:extra]])
    x = np.concatenate([x0] * reps + [x0[:extra]])
    s = np.concatenate([s0] * reps + [s0[:extra]])
    want = np.concatenate([want0] * reps + [want0[:extra]])
    for i in ((1 << 24) - 3, (1 << 24) + 11, n - 2):
        s[i, 40] ^= 0x02
        want[i] = 0
    cut = (1 << 24) - 1000               # a job across the first pass's end
    jobs = [(2, m[:cut], x[:cut], s[:cut]), (2, m[cut:cut + 3000], x[cut:cut + 3000], s[cut:cut + 3000]),
            (2, m[cut + 3000:], x[cut + 3000:], s[cut + 3000:])]
    got = np.concatenate(gpu_ctx.verify_jobs(jobs))
    assert got.shape == want.shape and (got == want).all()
