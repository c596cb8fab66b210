"""RLC batch verification of BIP-340 signatures on the GPU.

ufsecp_gpu_ext_schnorr_verify_rlc[_device] must give, item for item, the
verdicts of the per-signature verify (the oracle and ufsecp_gpu_schnorr_verify_batch)
for every batch size, window width and invalid-item pattern: one batch of
64 / 512 / 4096 / 16384 with no or one invalid item (bisection down to a
32-item leaf), many ragged batches with 1% invalid, parse failures (r >= p,
s = 0 or >= n, x >= p, x or r off the curve) from the golden edge corpus and
the BIP-340 vectors, and repeated items (equal points in one bucket).

The reference-shaped calls ufsecp_gpu_ext_schnorr_batch_verify and
ufsecp_gpu_ext_schnorr_batch_identify_invalid are compared with the
reference library's own ufsecp_schnorr_batch_verify and
ufsecp_schnorr_batch_identify_invalid (src/cpu/src/impl/ufsecp_taproot.cpp:703,
:849) on the same 128-byte rows: return codes, the parse gate's order and the
invalid indices.
"""
import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import P, load_golden, schnorr_corpus

pytestmark = pytest.mark.gpu

SEED = bytes(range(32))


def _flip(msgs, i, byte=5, bit=4):
    msgs[i, byte] ^= 1 << bit


def _bisection(n, bad, leaf=32, fanout=8):
    """Rounds and leaf items of the verifier's split policy for one invalid item."""
    rounds, leaves, segs = 0, 0, [(0, n)]
    while segs:
        rounds += 1
        nxt = []
        for st, ln in segs:
            if not st <= bad < st + ln:
                continue
            if ln <= leaf:
                leaves += ln
                continue
            parts = min(fanout, ln)
            nxt += [(st + ln * q // parts, ln * (q + 1) // parts - ln * q // parts) for q in range(parts)]
        segs = nxt
    return rounds, leaves


@pytest.mark.parametrize("bad", [0, 1])
@pytest.mark.parametrize("n", [64, 512, 4096, 16384])
def test_rlc_one_batch(gpu_ctx, oracle, n, bad):
    m, x, s = schnorr_corpus(oracle, n, seed=1000 + n, tamper=0.0)
    if bad:
        _flip(m, int(np.random.default_rng(n).integers(0, n)))
    out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=n, seed32=SEED)
    want = oracle.schnorr_verify_batch(m, x, s)
    assert int(want.sum()) == n - bad
    assert (out == want).all()
    assert (out == gpu_ctx.schnorr_verify_batch(m, x, s)).all()
    assert bok.tolist() == [0 if bad else 1]
    st = gpu_ctx.rlc_stats()
    if bad:
        # the locate round finds the single invalid item: check + locate, one candidate verified
        assert st["rounds"] == 2 and st["leaf_items"] == 1 and st["located"] == 1
    else:
        assert st["rounds"] == 1 and st["leaf_items"] == 0 and st["segments"] == 1
    if bad:
        # bisection alone: eight-way splits down to the leaf (<= 32 items) that holds it
        try:
            gpu_ctx.set_rlc_locate(False)
            out2, _ = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=n, seed32=SEED)
            assert (out2 == want).all()
            st = gpu_ctx.rlc_stats()
            rounds, leaf = _bisection(n, int(np.flatnonzero(want == 0)[0]))
            assert st["rounds"] == rounds and st["leaf_items"] == leaf and st["located"] == 0
        finally:
            gpu_ctx.set_rlc_locate(True)


@pytest.mark.parametrize("where", ["first", "last", "two", "three_spread"])
def test_rlc_locate_positions_and_multiples(gpu_ctx, oracle, where):
    """The locate step at the segment's first and last position (j = 1 and
    j = len), and with two or three invalid items in one segment (no multiple
    matches: the segment is bisected and its children located)."""
    n = 4096
    m, x, s = schnorr_corpus(oracle, n, seed=1300, tamper=0.0)
    m = m.copy()
    bad = {"first": [0], "last": [n - 1], "two": [100, 101], "three_spread": [7, 2000, 4095]}[where]
    for i in bad:
        _flip(m, i)
    out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=n, seed32=SEED)
    want = oracle.schnorr_verify_batch(m, x, s)
    assert (out == want).all()
    assert sorted(np.flatnonzero(out == 0).tolist()) == bad
    st = gpu_ctx.rlc_stats()
    if len(bad) == 1:
        assert st["located"] == 1 and st["leaf_items"] == 1
    elif where == "two":
        # adjacent items share every child down to a leaf: bisection alone finds them
        assert st["located"] == 0
    else:
        # the first split separates them: each child is located
        assert st["located"] == 3


def test_rlc_locate_segment_limits(gpu_ctx, oracle):
    """A 65,535-item batch (the longest a locate round searches) and a
    69,632-item one (longer: bisected first, then its failing child located),
    one invalid item each; tiled corpora (repeated items share buckets)."""
    m0, x0, s0 = schnorr_corpus(oracle, 4096, seed=1301, tamper=0.0)
    for n, bad_i in ((65535, 40000), (69632, 69000)):
        reps = -(-n // 4096)
        m, x, s = (np.ascontiguousarray(np.concatenate([a] * reps)[:n]) for a in (m0, x0, s0))
        _flip(m, bad_i)
        out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=n, seed32=SEED)
        assert np.flatnonzero(out == 0).tolist() == [bad_i]
        assert bok.tolist() == [0]
        st = gpu_ctx.rlc_stats()
        assert st["located"] == 1 and st["leaf_items"] == 1
        assert st["rounds"] == (2 if n <= 65535 else 3)


def test_rlc_many_ragged_batches_dense_invalid(gpu_ctx, oracle):
    n = 20000
    m, x, s = schnorr_corpus(oracle, n, seed=77, tamper=0.01)
    want = oracle.schnorr_verify_batch(m, x, s)
    for bs in (1000, 4096, 0):
        out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=bs, seed32=SEED)
        assert (out == want).all(), bs
        step = bs or n
        assert bok.tolist() == [int(want[i:i + step].all()) for i in range(0, n, step)]


def test_rlc_many_batches_sparse_invalid(gpu_ctx, oracle):
    n = 16 * 1024
    m, x, s = schnorr_corpus(oracle, n, seed=78, tamper=0.0)
    bad = [3, 5000, 5001, 16383]
    for i in bad:
        _flip(m, i)
    out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=1024, seed32=SEED)
    want = oracle.schnorr_verify_batch(m, x, s)
    assert (out == want).all()
    assert sorted(np.flatnonzero(out == 0).tolist()) == bad
    assert bok.tolist() == [0 if k in (0, 4, 15) else 1 for k in range(16)]
    # only the failing batches are bisected; leaves are 32-item pieces
    assert gpu_ctx.rlc_stats()["leaf_items"] <= 32 * len(bad)


def test_rlc_edge_corpus_and_bip340_vectors(gpu_ctx, oracle):
    vecs, _, edge = load_golden()
    em, ex, es = edge["schnorr_msgs"], edge["schnorr_pubs"], edge["schnorr_sigs"]
    vm = np.array([np.frombuffer(bytes.fromhex(v["msg"]), np.uint8) for v in vecs])
    vx = np.array([np.frombuffer(bytes.fromhex(v["pk"]), np.uint8) for v in vecs])
    vs = np.array([np.frombuffer(bytes.fromhex(v["sig"]), np.uint8) for v in vecs])
    m = np.concatenate([em, vm])
    x = np.concatenate([ex, vx])
    s = np.concatenate([es, vs])
    want = np.concatenate([edge["schnorr_ref_valid"].astype(np.uint8),
                           np.array([1 if v["ref_valid"] else 0 for v in vecs], np.uint8)])
    assert (oracle.schnorr_verify_batch(m, x, s) == want).all()
    for bs in (0, 100, 33):
        out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=bs, seed32=SEED)
        assert (out == want).all(), bs


@pytest.mark.parametrize("wbits", [4, 5, 7, 9, 12, 16])
def test_rlc_window_bits(gpu_ctx, oracle, wbits):
    n = 700
    m, x, s = schnorr_corpus(oracle, n, seed=79, tamper=0.0)
    _flip(m, 123)
    out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=350, seed32=SEED, window_bits=wbits)
    want = oracle.schnorr_verify_batch(m, x, s)
    assert (out == want).all()
    assert bok.tolist() == [0, 1]
    assert gpu_ctx.rlc_stats()["window_bits"] == wbits


def test_rlc_repeated_items(gpu_ctx, oracle):
    m, x, s = schnorr_corpus(oracle, 40, seed=80, tamper=0.0)
    _flip(m, 7)
    idx = np.array([i % 40 for i in range(400)] + [0] * 50 + [7] * 10)
    m, x, s = m[idx].copy(), x[idx].copy(), s[idx].copy()
    want = oracle.schnorr_verify_batch(m, x, s)
    out, _ = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=0, seed32=SEED, window_bits=4)
    assert (out == want).all()
    out, _ = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=0, seed32=SEED)
    assert (out == want).all()


@pytest.mark.parametrize("chunk", [2, 3, 7, 12, 16, 256])
def test_rlc_chunk_sizes(gpu_ctx, oracle, chunk):
    """Any bucket chunk (one point per thread up to whole buckets) gives the same verdicts."""
    m, x, s = schnorr_corpus(oracle, 60, seed=82, tamper=0.0)
    _flip(m, 11)
    idx = np.array([i % 60 for i in range(1500)] + [3] * 200)
    m, x, s = m[idx].copy(), x[idx].copy(), s[idx].copy()
    want = oracle.schnorr_verify_batch(m, x, s)
    tuned = gpu_ctx.get_rlc_chunk(4096)
    gpu_ctx.set_rlc_chunk(chunk)
    try:
        assert gpu_ctx.get_rlc_chunk(4096) == chunk and gpu_ctx.get_rlc_chunk(64) == chunk
        for wbits in (4, 0):
            for bs in (0, 256):
                out, bok = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=bs, seed32=SEED, window_bits=wbits)
                assert (out == want).all(), (wbits, bs)
    finally:
        gpu_ctx.set_rlc_chunk(0)
    assert gpu_ctx.get_rlc_chunk(4096) == tuned


@pytest.mark.parametrize("affine", [1, 0])
def test_rlc_affine_and_jacobian_chunk_sums(oracle, monkeypatch, affine):
    """Chunks summed in affine coordinates with block-shared inversions (up to
    16 points) or by mixed Jacobian additions give the same verdicts, repeated
    items (equal points in one bucket) included."""
    monkeypatch.setenv("UFSECP_B200_RLC_AFFINE", str(affine))
    m, x, s = schnorr_corpus(oracle, 80, seed=83, tamper=0.0)
    _flip(m, 7)
    idx = np.array([i % 80 for i in range(3000)] + [5] * 300 + [9] * 97)
    m, x, s = m[idx].copy(), x[idx].copy(), s[idx].copy()
    want = oracle.schnorr_verify_batch(m, x, s)
    with uf.GpuContext(0) as ctx:
        for chunk in (4, 8, 13, 16):
            ctx.set_rlc_chunk(chunk)
            for bs in (0, 512):
                out, _ = ctx.schnorr_verify_rlc(m, x, s, batch_size=bs, seed32=SEED)
                assert (out == want).all(), (chunk, bs)


def test_rlc_chunk_bounds(gpu_ctx):
    for bad in (1, 257):
        with pytest.raises(uf.UfsecpError):
            gpu_ctx.set_rlc_chunk(bad)
    assert 2 <= gpu_ctx.get_rlc_chunk(4096) <= 256


def test_rlc_seed_does_not_change_verdicts(gpu_ctx, oracle):
    m, x, s = schnorr_corpus(oracle, 3000, seed=81, tamper=0.003)
    want = oracle.schnorr_verify_batch(m, x, s)
    for k in range(3):
        out, _ = gpu_ctx.schnorr_verify_rlc(m, x, s, batch_size=1024, seed32=bytes([k]) * 32)
        assert (out == want).all()


def test_rlc_device_buffers(gpu_ctx, oracle):
    import torch
    n = 5000
    m, x, s = schnorr_corpus(oracle, n, seed=82, tamper=0.002)
    dm, dx, ds = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (m, x, s))
    do = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    bok = gpu_ctx.schnorr_verify_rlc_device(dm.data_ptr(), dx.data_ptr(), ds.data_ptr(), n, do.data_ptr(),
                                            batch_size=2048, seed32=SEED, stream=stream.cuda_stream)
    stream.synchronize()
    want = oracle.schnorr_verify_batch(m, x, s)
    assert (do.cpu().numpy() == want).all()
    assert bok.tolist() == [int(want[i:i + 2048].all()) for i in range(0, n, 2048)]


def test_rlc_gating(gpu_ctx):
    L = uf.load_library()
    z = np.zeros(64, np.uint8)
    out = np.full(4, 7, np.uint8)
    assert L.ufsecp_gpu_ext_schnorr_verify_rlc(None, z.ctypes.data, z.ctypes.data, z.ctypes.data, 1, 0,
                                               z.ctypes.data, 0, out.ctypes.data, None) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, None, None, None, 0, 0, None, 0, None,
                                               None) == uf.UFSECP_OK
    rc = L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, None, z.ctypes.data, z.ctypes.data, 1, 0,
                                             z.ctypes.data, 0, out.ctypes.data, None)
    assert rc == uf.UFSECP_ERR_NULL_ARG and out[0] == 0          # cleared before the NULL check
    rc = L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, z.ctypes.data, z.ctypes.data, z.ctypes.data, 1, 0,
                                             z.ctypes.data, 3, out.ctypes.data, None)
    assert rc == uf.UFSECP_ERR_BAD_INPUT                          # window_bits outside 4..16
    rc = L.ufsecp_gpu_ext_schnorr_verify_rlc(gpu_ctx.handle, z.ctypes.data, z.ctypes.data, z.ctypes.data,
                                             (1 << 24) + 1, 0, z.ctypes.data, 0, out.ctypes.data, None)
    assert rc == uf.UFSECP_ERR_BAD_INPUT


# ---- the reference's batch API --------------------------------------------------

def _rows(m, x, s):
    return np.ascontiguousarray(np.concatenate([x, m, s], axis=1))


def _int_be(v: int) -> np.ndarray:
    return np.frombuffer(v.to_bytes(32, "big"), np.uint8)


def test_batch_api_matches_reference(gpu_ctx, oracle, reflib):
    m, x, s = schnorr_corpus(oracle, 3000, seed=83, tamper=0.0)
    rows = _rows(m, x, s)
    assert gpu_ctx.schnorr_batch_verify(rows) == reflib.schnorr_batch_verify_rows(rows) == uf.UFSECP_OK
    rc, idx, tot = gpu_ctx.schnorr_batch_identify_invalid(rows)
    assert (rc, idx, tot) == reflib.schnorr_batch_identify_invalid_rows(rows) == (0, [], 0)
    # invalid items: tampered messages, an off-curve key, an off-curve R
    bad = [10, 11, 2999]
    for i in bad:
        rows[i, 32 + 3] ^= 0x01
    x_off = int.from_bytes(bytes(rows[500, :32]), "big")
    while True:          # an x < p with no curve point (x^3 + 7 not a square)
        x_off = (x_off + 1) % P
        if pow((x_off ** 3 + 7) % P, (P - 1) // 2, P) != 1:
            break
    rows[500, :32] = _int_be(x_off)
    rows[600, 64:96] = _int_be(x_off)
    want_idx = sorted(bad + [500, 600])
    assert gpu_ctx.schnorr_batch_verify(rows) == reflib.schnorr_batch_verify_rows(rows) == uf.UFSECP_ERR_VERIFY_FAIL
    got = gpu_ctx.schnorr_batch_identify_invalid(rows)
    assert got == reflib.schnorr_batch_identify_invalid_rows(rows) == (0, want_idx, len(want_idx))
    # capacity below the count: the first `capacity` indices, the full total
    got = gpu_ctx.schnorr_batch_identify_invalid(rows, capacity=2)
    assert got == reflib.schnorr_batch_identify_invalid_rows(rows, capacity=2) == (0, want_idx[:2], len(want_idx))


def test_batch_api_parse_gate_order(gpu_ctx, oracle, reflib):
    m, x, s = schnorr_corpus(oracle, 64, seed=84, tamper=0.0)
    base = _rows(m, x, s)
    cases = []
    r = base.copy(); r[7, :32] = _int_be(P + 5); cases.append(r)                    # x >= p -> BAD_PUBKEY
    r = base.copy(); r[9, 64:96] = _int_be(P); cases.append(r)                      # r >= p -> BAD_SIG
    r = base.copy(); r[9, 96:] = 0; cases.append(r)                                 # s = 0 -> BAD_SIG
    r = base.copy(); r[9, 96:] = 0xFF; r[20, :32] = _int_be(P); cases.append(r)     # first failing row wins
    r = base.copy(); r[9, :32] = _int_be(P + 1); r[9, 96:] = 0; cases.append(r)    # key tested before sig
    for r in cases:
        want = reflib.schnorr_batch_verify_rows(r)
        assert want in (uf.UFSECP_ERR_BAD_PUBKEY, uf.UFSECP_ERR_BAD_SIG)
        assert gpu_ctx.schnorr_batch_verify(r) == want
        assert gpu_ctx.schnorr_batch_identify_invalid(r)[0] == reflib.schnorr_batch_identify_invalid_rows(r)[0]
    assert gpu_ctx.schnorr_batch_verify(base[:0]) == uf.UFSECP_OK


def _tree_digest(m, x, s):
    """The RLC seed's input binding written out with hashlib: per item
    SHA-256(r || s || x || m), 16-way tree, then SHA-256(root || le32 n)."""
    import hashlib
    n = len(m)
    level = [hashlib.sha256(s[i].tobytes() + x[i].tobytes() + m[i].tobytes()).digest() for i in range(n)]
    while len(level) > 1:
        level = [hashlib.sha256(b"".join(level[k:k + 16])).digest() for k in range(0, len(level), 16)]
    root = level[0] if level else bytes(32)
    return hashlib.sha256(root + n.to_bytes(4, "little")).digest()


@pytest.mark.parametrize("n", [0, 1, 15, 16, 17, 257, 4099])
def test_rlc_input_digest_matches_hashlib(gpu_ctx, oracle, n):
    m, x, s = schnorr_corpus(oracle, max(n, 1), seed=777 + n, tamper=0.05)
    m, x, s = m[:n], x[:n], s[:n]
    assert gpu_ctx.rlc_input_digest(m, x, s) == _tree_digest(m, x, s)
    if n:
        m2 = m.copy()
        m2[n - 1, 0] ^= 1
        assert gpu_ctx.rlc_input_digest(m2, x, s) != gpu_ctx.rlc_input_digest(m, x, s)


def test_rlc_uses_resident_keys(oracle):
    """Keys left in the context's key table by a mixed-job call give the RLC
    prep their y without a square root (entry 0 of the slot's table), and a
    key the table knows to be off the curve fails as lift_x would: verdicts
    equal the oracle's with and without resident keys."""
    m, x, s = schnorr_corpus(oracle, 3000, seed=91, tamper=0.03)
    x = x.copy()
    x[::37, 7] ^= 0x10                    # some keys off the curve (the oracle decides which)
    idx = np.array([i % 3000 for i in range(6000)])
    m, x, s = m[idx].copy(), x[idx].copy(), s[idx].copy()
    want = oracle.schnorr_verify_batch(m, x, s)
    with uf.GpuContext(0) as ctx:
        out0, _ = ctx.schnorr_verify_rlc(m, x, s, batch_size=512, seed32=SEED)
        assert ctx.rlc_stats()["key_hits"] == 0         # no table made yet
        assert (out0 == want).all()
        assert all((g == w).all() for g, w in zip(ctx.verify_jobs([(1, m, x, s)]), [want]))
        out1, _ = ctx.schnorr_verify_rlc(m, x, s, batch_size=512, seed32=SEED)
        st = ctx.rlc_stats()
        assert (out1 == want).all()
        assert st["key_hits"] >= 0.9 * len(m)
        ctx.set_key_table(0)
        out2, _ = ctx.schnorr_verify_rlc(m, x, s, batch_size=512, seed32=SEED)
        assert (out2 == want).all() and ctx.rlc_stats()["key_hits"] == 0
