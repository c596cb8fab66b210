"""Resident key table of ufsecp_gpu_ext_verify_jobs (ufsecp_gpu_ext_set_key_table).

Before the verify kernels, a resolve pass gives every item its key's slot and a
build pass decompresses each new key and builds its 1P..8P table in the slot
(or marks an x off the curve as bad); the verify kernels then copy the table.
The verdicts must never depend on the table: with no table, a table that
overflows, a cold table and a warm one (every key already resident, including
the bad ones) they equal the oracle item for item.  The corpus repeats keys
(few distinct keys, many signatures each) and mixes in every key edge case:
bad prefixes, x >= p, x off the curve (repeated, so the second call meets the
cached bad mark), and the other parity of a real key (the same x in a
different slot).
"""
import numpy as np
import pytest

from conftest import P, flip_random_bits, rand_keys

pytestmark = pytest.mark.gpu


def _offcurve(x):
    while True:
        x = (x + 1) % P
        if pow((x ** 3 + 7) % P, (P - 1) // 2, P) != 1:
            return x


def _keyed_corpus(oracle, kind, n, n_keys, seed):
    rng = np.random.default_rng(seed)
    pool = rand_keys(rng, n_keys)
    sks = pool[rng.integers(0, n_keys, n)]
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    if kind == 0:
        pubs, sigs, ok = oracle.ecdsa_sign_batch(msgs, sks)
        pubs = pubs.reshape(n, 33).copy()
    else:
        aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
        pubs, sigs, ok = oracle.schnorr_sign_batch(msgs, sks, aux)
        pubs = pubs.reshape(n, 32).copy()
    assert ok.all()
    sigs = sigs.reshape(n, 64).copy()
    flip_random_bits(rng, (msgs, sigs), 0.05)
    # key edge cases, each class on a few repeated keys
    bad_x = [_offcurve(int(rng.integers(1, 1 << 62))) for _ in range(3)]
    big_x = [P + int(rng.integers(0, 977)) for _ in range(2)]
    off = 1 if kind == 0 else 0
    for i in range(0, n, 7):
        c = (i // 7) % 5
        if c == 0:
            pubs[i, off:] = np.frombuffer(bad_x[i % 3].to_bytes(32, "big"), np.uint8)
        elif c == 1:
            pubs[i, off:] = np.frombuffer(big_x[i % 2].to_bytes(32, "big"), np.uint8)
        elif c == 2 and kind == 0:
            pubs[i, 0] = (0x00, 0x04)[i % 2]
        elif c == 3 and kind == 0:
            pubs[i, 0] ^= 0x01          # 02 <-> 03: the other point with this x
    return msgs, pubs, sigs


@pytest.fixture(scope="module")
def keyed(oracle):
    e = _keyed_corpus(oracle, 0, 3000, 150, seed=601)
    s = _keyed_corpus(oracle, 1, 5000, 250, seed=602)
    we = oracle.ecdsa_verify_batch(*e)
    ws = oracle.schnorr_verify_batch(*s)
    assert 0 < we.sum() < len(we) and 0 < ws.sum() < len(ws)
    return e, s, we, ws


def _jobs(e, s, cut=37):
    """Uneven mixed jobs over both corpora."""
    jobs = []
    for c, kind in ((e, 0), (s, 1)):
        n = len(c[0])
        lo = 0
        k = 0
        while lo < n:
            hi = min(n, lo + cut + 97 * (k % 5))
            jobs.append((kind,) + tuple(x[lo:hi] for x in c))
            lo, k = hi, k + 1
    return jobs


def _check(got, jobs, we, ws):
    pos = {0: 0, 1: 0}
    for g, (kind, m, p, s) in zip(got, jobs):
        w = (we if kind == 0 else ws)[pos[kind]:pos[kind] + len(m)]
        pos[kind] += len(m)
        assert (g == w).all()


def test_key_table_cold_warm_and_off(gpu_ctx, keyed):
    e, s, we, ws = keyed
    jobs = _jobs(e, s)
    try:
        gpu_ctx.set_key_table(16)
        _check(gpu_ctx.verify_jobs(jobs), jobs, we, ws)          # cold: keys built in this call
        st1 = gpu_ctx.key_table_stats()
        assert st1["slots"] == 1 << 16 and st1["lookups"] > 0
        _check(gpu_ctx.verify_jobs(jobs), jobs, we, ws)          # warm: every parsed key resident
        st2 = gpu_ctx.key_table_stats()
        looked = st2["lookups"] - st1["lookups"]
        assert looked == st1["lookups"]
        assert st2["hits"] - st1["hits"] == looked
        gpu_ctx.set_key_table(0)
        _check(gpu_ctx.verify_jobs(jobs), jobs, we, ws)
        assert gpu_ctx.key_table_stats()["slots"] == 0
    finally:
        gpu_ctx.set_key_table(18)


def test_key_table_overflow(gpu_ctx, oracle):
    """256 slots for 2,000 distinct keys: most keys find no slot and are verified
    the plain way, in the same launches as the keys that found one."""
    e = _keyed_corpus(oracle, 0, 2500, 1000, seed=611)
    s = _keyed_corpus(oracle, 1, 2500, 1000, seed=612)
    we = oracle.ecdsa_verify_batch(*e)
    ws = oracle.schnorr_verify_batch(*s)
    jobs = _jobs(e, s, cut=300)
    try:
        gpu_ctx.set_key_table(8)
        for _ in range(2):
            _check(gpu_ctx.verify_jobs(jobs), jobs, we, ws)
        st = gpu_ctx.key_table_stats()
        assert st["slots"] == 256 and 0 < st["hits"] < st["lookups"]
    finally:
        gpu_ctx.set_key_table(18)


def test_key_table_large_call(gpu_ctx, keyed):
    """A call above one sub-call (the direct, non-graph path, two batch slots):
    the sub-calls share one table."""
    e, s, we, ws = keyed
    reps = 16
    E = tuple(np.ascontiguousarray(np.concatenate([x] * reps)) for x in e)
    S = tuple(np.ascontiguousarray(np.concatenate([x] * reps)) for x in s)
    got = gpu_ctx.verify_jobs([(0,) + E, (1,) + S])
    assert (got[0] == np.concatenate([we] * reps)).all()
    assert (got[1] == np.concatenate([ws] * reps)).all()


def test_key_table_gating(gpu_ctx):
    import ultrafastsecp256k1_b200 as uf
    L = uf.load_library()
    assert L.ufsecp_gpu_ext_set_key_table(gpu_ctx.handle, 7) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_set_key_table(gpu_ctx.handle, 25) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_set_key_table(None, 18) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_ext_key_table_stats(gpu_ctx.handle, None) == uf.UFSECP_ERR_NULL_ARG
