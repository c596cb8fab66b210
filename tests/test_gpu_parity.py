"""Parity of the sm_100a verify path with the oracle, through the C ABI.

Bit-exact per-signature verdicts are required everywhere.  Small cases are
compared item by item with the oracle; the full-size configurations (4096
ECDSA, 1,048,576 BIP-340 in one launch) are compared against verdicts that are
known by construction (oracle-verified seed corpora tiled across the launch,
tampered copies)."""
import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import N, P, ecdsa_corpus, load_golden, opaque_rows_corpus, rand_keys, schnorr_corpus

pytestmark = pytest.mark.gpu

LAM = 0x5363AD4CC05C30E0A5261C028812645A122E22EA20816678DF02967C1B23BD72


def be(v):
    return int(v).to_bytes(32, "big")


def _cat(hexes):
    return np.frombuffer(b"".join(bytes.fromhex(h) for h in hexes), np.uint8)


# ------------------------------------------------------------ building blocks --
def test_diag_field_and_scalar(gpu_ctx):
    rng = np.random.default_rng(1)
    special = [0, 1, 2, P - 1, P, P + 1, 2**256 - 1, 2**255, N - 1, N]
    vals = special + [int.from_bytes(rng.bytes(32), "big") for _ in range(4000)]
    a = vals
    b = vals[7:] + vals[:7]
    ab = np.frombuffer(b"".join(be(x) + be(y) for x, y in zip(a, b)), np.uint8)
    out = gpu_ctx.diag(1, ab)
    assert [int.from_bytes(r.tobytes(), "big") for r in out] == [x * y % P for x, y in zip(a, b)]
    out = gpu_ctx.diag(2, np.frombuffer(b"".join(be(x) for x in a), np.uint8))
    assert [int.from_bytes(r.tobytes(), "big") for r in out] == [x * x % P for x in a]
    nz = [x for x in a if x % P]
    out = gpu_ctx.diag(3, np.frombuffer(b"".join(be(x) for x in nz), np.uint8))
    assert [int.from_bytes(r.tobytes(), "big") for r in out] == [pow(x, -1, P) for x in nz]
    an = [x % N for x in a]
    bn = [x % N for x in b]
    out = gpu_ctx.diag(5, np.frombuffer(b"".join(be(x) + be(y) for x, y in zip(an, bn)), np.uint8))
    assert [int.from_bytes(r.tobytes(), "big") for r in out] == [x * y % N for x, y in zip(an, bn)]
    nzn = [x for x in an if x]
    out = gpu_ctx.diag(6, np.frombuffer(b"".join(be(x) for x in nzn), np.uint8))
    assert [int.from_bytes(r.tobytes(), "big") for r in out] == [pow(x, -1, N) for x in nzn]


M32 = (1 << 32) - 1
K = (1 << 32) + 977


def _fold_paths(t):
    """Which rare paths the device reduction of the 512-bit t takes in its
    second fold: (top >= 2^32, carry past limb 2, wrap past 2^256)."""
    L, H = t % 2**256, t >> 256
    sf = L + 977 * H + (H << 32)
    s, top = sf % 2**256, sf >> 256
    tl, th = top & M32, top >> 32
    s0, s1, s2 = s & M32, (s >> 32) & M32, (s >> 64) & M32
    x = s0 + ((tl * 977) & M32)
    y = s1 + ((tl * 977) >> 32) + (x >> 32)
    z = s2 + th + (y >> 32)
    c = z >> 32
    y2 = (y & M32) + tl
    c += ((z & M32) + (y2 >> 32)) >> 32
    return th, c, (s + top * K) >> 256


def _add_paths(a, b):
    """(carry past limb 1 after the +K fold, second wrap) of the device a + b."""
    sm = a + b
    if sm < 2**256:
        return 0, 0
    r = sm - 2**256
    return int(((r & (2**64 - 1)) + K) >> 64), int(r + K >= 2**256)


def _sub_paths(a, b):
    """(borrow past limb 1 after the -K fold, second borrow) of the device a - b."""
    if a >= b:
        return 0, 0
    r = a - b + 2**256
    return int((r & (2**64 - 1)) < K), int(r < K)


def _shift_paths(a, k):
    """(carry past limb 1 after folding the shifted-out bits, wrap past 2^256)
    of the device a * 2^k."""
    r, top = (a << k) % 2**256, a >> (256 - k)
    return int(((r & (2**64 - 1)) + top * K) >> 64), int(r + top * K >= 2**256)


def _hard_field_pairs(rng):
    """Operand pairs that drive the device field code into its rare carry paths."""
    pairs = []
    # reduction, carry past limb 2 in the second fold: b = 2^96 and a chosen so
    # that L + H*K = 2^256 + s with limbs 1 and 2 of s all ones
    kinv = pow(K, -1, 2**96)
    for _ in range(64):
        X = int(rng.integers(0, 2**32)) | (M32 << 32) | (M32 << 64)
        H = X * kinv % 2**96
        if H * K <= X:
            continue
        L = 2**256 + X - H * K
        pairs.append(((H << 160) | (L >> 96), 2**96))
    # top >= 2^32 and a wrap: operands near 2^256
    for d1 in range(0, 40, 3):
        for d2 in range(0, 40, 7):
            pairs.append((2**256 - 1 - d1, 2**256 - 1 - d2))
    # add: sums 2^256 + r with limb 1 of r all ones, and r >= 2^256 - K
    for _ in range(32):
        r = int.from_bytes(rng.bytes(32), "big") | (M32 << 32)
        pairs.append((2**256 - 1, (r + 1) % 2**256))
    pairs += [(2**256 - 1, 2**256 - 1 - d) for d in range(0, 3000, 97)]
    # sub: borrows with limb 1 of a - b + 2^256 zero, and a tiny with b near 2^256
    for _ in range(32):
        r = int.from_bytes(rng.bytes(32), "big") & ~(M32 << 32)
        a = int(rng.integers(0, 2**20))
        pairs.append((a, (a - r) % 2**256))
    pairs += [(d, 2**256 - 1 - e) for d in range(0, 5) for e in range(0, 2000, 401)]
    # shifts: a * 2^k with limb 1 of the shifted value all ones, and near 2^256
    for k in (2, 3):
        for _ in range(16):
            r = (int.from_bytes(rng.bytes(32), "big") | (M32 << 32)) & ~((1 << k) - 1)
            top = int(rng.integers(1, 1 << k))
            pairs.append((((top << 256) | r) >> k, 1))
    pairs += [(2**256 - 1 - d, 3) for d in range(0, 64, 5)]
    return pairs


def test_diag_ptx_field_rare_paths(gpu_ctx):
    """The field code the verify kernels run (PTX carry chains) on random
    weakly reduced operands and on pairs built to reach every rare carry path
    of the reduction, the add, the sub and the shifts by 2 and 3; the models
    above confirm that each path is reached."""
    rng = np.random.default_rng(11)
    pairs = _hard_field_pairs(rng)
    pairs += [(int.from_bytes(rng.bytes(32), "big"), int.from_bytes(rng.bytes(32), "big")) for _ in range(2000)]
    special = [0, 1, 2, P - 1, P, P + 1, 2**256 - 1, 2**255, N - 1, N, K, 2**256 - K]
    pairs += [(x, y) for x in special for y in special]
    fold = [_fold_paths(a * b) for a, b in pairs] + [_fold_paths(a * a) for a, _ in pairs]
    assert all(any(f[k] for f in fold) for k in range(3)), "a reduction path is not reached"
    assert all(any(_add_paths(a, b)[k] for a, b in pairs) for k in range(2)), "an add path is not reached"
    assert all(any(_sub_paths(a, b)[k] for a, b in pairs) for k in range(2)), "a sub path is not reached"
    for sh in (2, 3):
        assert all(any(_shift_paths(a, sh)[k] for a, _ in pairs) for k in range(2)), "a shift path is not reached"
    data = np.frombuffer(b"".join(be(a) + be(b) for a, b in pairs), np.uint8)
    out = gpu_ctx.diag(11, data)
    got = [[int.from_bytes(r[32 * k:32 * k + 32].tobytes(), "big") for k in range(6)] for r in out]
    want = [[a * b % P, a * a % P, (a + b) % P, (a - b) % P, 4 * a % P, 8 * a % P] for a, b in pairs]
    bad = [(i, pairs[i]) for i in range(len(pairs)) if got[i] != want[i]]
    assert not bad, bad[:4]


def test_diag_sqrt_glv_challenge(gpu_ctx):
    import hashlib
    rng = np.random.default_rng(2)
    xs = [int.from_bytes(rng.bytes(32), "big") % P for _ in range(2000)]
    out = gpu_ctx.diag(4, np.frombuffer(b"".join(be(x) for x in xs), np.uint8))
    for x, r in zip(xs, out):
        qr = pow(x, (P - 1) // 2, P) in (0, 1)
        assert bool(r[0]) == qr
        if qr:
            y = int.from_bytes(r[1:].tobytes(), "big")
            assert y * y % P == x
    ks = [0, 1, N - 1, LAM] + [int.from_bytes(rng.bytes(32), "big") % N for _ in range(4000)]
    out = gpu_ctx.diag(7, np.frombuffer(b"".join(be(k) for k in ks), np.uint8))
    for k, r in zip(ks, out):
        k1 = int.from_bytes(r[:16].tobytes(), "big") * (-1 if r[32] else 1)
        k2 = int.from_bytes(r[16:32].tobytes(), "big") * (-1 if r[33] else 1)
        assert (k1 + k2 * LAM - k) % N == 0
    tag = hashlib.sha256(b"BIP0340/challenge").digest()
    data = [rng.bytes(96) for _ in range(1000)]
    out = gpu_ctx.diag(10, np.frombuffer(b"".join(data), np.uint8))
    for d, r in zip(data, out):
        assert r.tobytes() == hashlib.sha256(tag + tag + d).digest()


def test_diag_gen_mul_vs_oracle(gpu_ctx, oracle):
    rng = np.random.default_rng(3)
    ks = [1, 2, 3, N - 1, N - 2, 2**128, LAM] + [int.from_bytes(rng.bytes(32), "big") % N for _ in range(500)]
    out = gpu_ctx.diag(8, np.frombuffer(b"".join(be(k) for k in ks), np.uint8))
    for k, r in zip(ks, out):
        x, y = oracle.gen_mul(be(k))
        assert r[:32].tobytes() == x and r[32:].tobytes() == y
    out = gpu_ctx.diag(8, np.frombuffer(be(0) + be(N), np.uint8))
    assert not out.any()


def test_diag_dual_mul_exceptional(gpu_ctx, oracle):
    """a*G + b*P including results at infinity and doublings inside the adds."""
    rng = np.random.default_rng(4)
    rows, want = [], []
    for i in range(64):
        d = int.from_bytes(rng.bytes(32), "big") % (N - 1) + 1
        X, Y = (int.from_bytes(v, "big") for v in oracle.gen_mul(be(d)))
        if Y & 1:
            d = N - d
        a, b = (int.from_bytes(rng.bytes(32), "big") % N for _ in range(2))
        if i == 0:
            a, b = (N - d) % N, 1          # a*G + P = infinity
        elif i == 1:
            a, b = d, 1                    # = 2P
        elif i == 2:
            a, b = 0, 3
        elif i == 3:
            a, b = 5, 0
        rows.append(be(a) + be(X) + be(b))
        want.append((a + b * d) % N)
    out = gpu_ctx.diag(9, np.frombuffer(b"".join(rows), np.uint8))
    for r, k in zip(out, want):
        if k == 0:
            assert r[0] == 0
        else:
            x, y = oracle.gen_mul(be(k))
            assert r[0] == 1 and r[1:33].tobytes() == x and r[33:].tobytes() == y


# ---------------------------------------------------------------- golden data --
def test_bip340_vectors(gpu_ctx):
    vecs, _, _ = load_golden()
    got = gpu_ctx.schnorr_verify_batch(_cat(v["msg"] for v in vecs), _cat(v["pk"] for v in vecs),
                                       _cat(v["sig"] for v in vecs))
    assert list(got) == [int(v["ref_valid"]) for v in vecs]


def test_wycheproof_ecdsa(gpu_ctx):
    _, wy, _ = load_golden()
    got = gpu_ctx.ecdsa_verify_batch(wy["msgs"], wy["pubs"], wy["sigs"])
    assert (got == wy["ref_valid"]).all()


def test_edge_corpus(gpu_ctx):
    _, _, e = load_golden()
    assert (gpu_ctx.ecdsa_verify_batch(e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"]) == e["ecdsa_ref_valid"]).all()
    assert (gpu_ctx.schnorr_verify_batch(e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
            == e["schnorr_ref_valid"]).all()


# ---------------------------------------------------------- seeded workloads --
def test_ecdsa_4096_tampered(gpu_ctx, oracle):
    """Plain ECDSA verify, 4096 signatures, 10% with one flipped bit in msg, r or s."""
    m, p, s = ecdsa_corpus(oracle, 4096, seed=20261203, tamper=0.10)
    want = oracle.ecdsa_verify_batch(m, p, s)
    got = gpu_ctx.ecdsa_verify_batch(m, p, s)
    assert (got == want).all()
    assert 0.85 * 4096 < want.sum() < 0.95 * 4096


def _offcurve_x(rng):
    while True:
        x = int.from_bytes(rng.bytes(32), "big") % P
        if pow((x**3 + 7) % P, (P - 1) // 2, P) != 1:
            return x


def test_schnorr_1m_one_launch(gpu_ctx, oracle):
    """BIP-340, 1,048,576 signatures in one launch: 1% flipped bits in s or R.x,
    0.1% x-only keys off the curve.  16,384 oracle-verified items tiled 64x."""
    base = 16384
    rng = np.random.default_rng(7)
    m, x, s = schnorr_corpus(oracle, base, seed=8, tamper=0.0)
    for i in rng.choice(base, size=base // 100, replace=False):
        bit = int(rng.integers(0, 256))
        s[i, (0 if rng.integers(0, 2) else 32) + bit // 8] ^= 1 << (bit % 8)
    for i in rng.choice(base, size=max(1, base // 1000), replace=False):
        x[i] = np.frombuffer(be(_offcurve_x(rng)), np.uint8)
    want = oracle.schnorr_verify_batch(m, x, s)
    reps = (1 << 20) // base
    got = gpu_ctx.schnorr_verify_batch(np.tile(m, (reps, 1)), np.tile(x, (reps, 1)), np.tile(s, (reps, 1)))
    assert got.shape == (1 << 20,)
    assert (got == np.tile(want, reps)).all()


def test_chunked_host_call(gpu_ctx, oracle):
    """A call larger than one device chunk (2^22 items) keeps per-item order."""
    base = 4096
    m, x, s = schnorr_corpus(oracle, base, seed=9, tamper=0.05)
    want = oracle.schnorr_verify_batch(m, x, s)
    n = (1 << 22) + 4099
    reps = -(-n // base)
    got = gpu_ctx.schnorr_verify_batch(np.tile(m, (reps, 1))[:n], np.tile(x, (reps, 1))[:n],
                                       np.tile(s, (reps, 1))[:n])
    assert (got == np.tile(want, reps)[:n]).all()


@pytest.mark.parametrize("n", [16383, 16384, 16385, 49151, 49153, 114688, 131072, 131073, 245761, 393217])
def test_host_pipeline_chunk_edges(gpu_ctx, oracle, n):
    """Host-buffer calls are cut into chunks of 16384, 32768, 65536 and then
    131072 items over three staging slots: sizes on and around those edges keep
    every verdict in place (ECDSA with collect, BIP-340 plain)."""
    base = 2048
    m, x, s = schnorr_corpus(oracle, base, seed=300, tamper=0.1)
    want = oracle.schnorr_verify_batch(m, x, s)
    reps = -(-n // base)
    tile = lambda a: np.ascontiguousarray(np.tile(a, (reps, 1))[:n])
    assert (gpu_ctx.schnorr_verify_batch(tile(m), tile(x), tile(s)) == np.tile(want, reps)[:n]).all()
    me, pe, se = ecdsa_corpus(oracle, base, seed=301, tamper=0.1)
    we = oracle.ecdsa_verify_batch(me, pe, se)
    kb = np.full(n, 0x5A, np.uint8)
    gpu_ctx.ecdsa_verify_collect(tile(me), tile(pe), tile(se), kb)
    w = np.tile(we, reps)[:n]
    assert ((kb == 0) == (w == 1)).all() and (kb[w == 0] == 0x5A).all()


@pytest.mark.parametrize("n", [1, 2, 31, 127, 129, 1000])
def test_ragged_sizes(gpu_ctx, oracle, n):
    m, p, s = ecdsa_corpus(oracle, n, seed=100 + n, tamper=0.3)
    assert (gpu_ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
    m, x, s = schnorr_corpus(oracle, n, seed=200 + n, tamper=0.3)
    assert (gpu_ctx.schnorr_verify_batch(m, x, s) == oracle.schnorr_verify_batch(m, x, s)).all()


def test_collect_semantics(gpu_ctx, oracle):
    m, p, s = ecdsa_corpus(oracle, 777, seed=31, tamper=0.2)
    want = oracle.ecdsa_verify_batch(m, p, s)
    kb = np.full(777, 0xA5, np.uint8)
    gpu_ctx.ecdsa_verify_collect(m, p, s, kb)
    assert ((kb == 0) == (want == 1)).all() and (kb[want == 0] == 0xA5).all()
    m, x, s = schnorr_corpus(oracle, 555, seed=32, tamper=0.2)
    want = oracle.schnorr_verify_batch(m, x, s)
    kb = np.arange(1, 556, dtype=np.uint32).astype(np.uint8) | 1
    before = kb.copy()
    gpu_ctx.schnorr_verify_collect(m, x, s, kb)
    assert ((kb == 0) == (want == 1)).all() and (kb[want == 0] == before[want == 0]).all()


def test_gpu_signers_match_oracle(gpu_ctx, oracle):
    import torch
    n = 512
    rng = np.random.default_rng(41)
    sks = rand_keys(rng, n)
    sks[0] = 0                               # invalid key -> ok = 0
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dm, dk, da = dev(msgs), dev(sks), dev(aux)
    for kind, ps in ((0, 33), (1, 32)):
        dp = torch.zeros(n * ps, dtype=torch.uint8, device="cuda")
        ds = torch.zeros(n * 64, dtype=torch.uint8, device="cuda")
        dok = torch.zeros(n, dtype=torch.uint8, device="cuda")
        gpu_ctx.sign_device(kind, dm.data_ptr(), dk.data_ptr(), da.data_ptr(), n, dp.data_ptr(), ds.data_ptr(),
                            dok.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        if kind == 0:
            p2, s2, ok2 = oracle.ecdsa_sign_batch(msgs[1:], sks[1:])
        else:
            p2, s2, ok2 = oracle.schnorr_sign_batch(msgs[1:], sks[1:], aux[1:])
        ok = dok.cpu().numpy()
        assert ok[0] == 0 and ok[1:].all()
        assert (dp.cpu().numpy()[ps:] == p2).all() and (ds.cpu().numpy()[64:] == s2).all()


def test_device_api_matches_host_api(gpu_ctx, oracle):
    import torch
    m, p, s = ecdsa_corpus(oracle, 3000, seed=51, tamper=0.1)
    want = gpu_ctx.ecdsa_verify_batch(m, p, s)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dm, dp, ds = dev(m), dev(p), dev(s)
    dout = torch.full((3000,), 7, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    gpu_ctx.ecdsa_verify_device(dm.data_ptr(), dp.data_ptr(), ds.data_ptr(), 3000, dout.data_ptr(), stream)
    torch.cuda.synchronize()
    assert (dout.cpu().numpy() == want).all()
    m, x, s = schnorr_corpus(oracle, 3000, seed=52, tamper=0.1)
    want = gpu_ctx.schnorr_verify_batch(m, x, s)
    dm, dx, ds = dev(m), dev(x), dev(s)
    gpu_ctx.schnorr_verify_device(dm.data_ptr(), dx.data_ptr(), ds.data_ptr(), 3000, dout.data_ptr(), 0)
    gpu_ctx_stream_sync(gpu_ctx)
    assert (dout.cpu().numpy() == want).all()


def gpu_ctx_stream_sync(ctx):
    import torch
    s = torch.cuda.ExternalStream(ctx.stream())
    s.synchronize()


def test_abi_gating_with_context(gpu_ctx):
    L = uf.load_library()
    h = gpu_ctx.handle
    out = np.full(4, 9, np.uint8)
    # count == 0: OK, buffers untouched
    assert L.ufsecp_gpu_ecdsa_verify_batch(h, None, None, None, 0, out.ctypes.data) == 0 and (out == 9).all()
    # over the 2^26 cap
    assert L.ufsecp_gpu_schnorr_verify_batch(h, 1, 1, 1, (1 << 26) + 1, out.ctypes.data) == uf.UFSECP_ERR_BAD_INPUT
    # output cleared before the NULL-input check
    assert L.ufsecp_gpu_ecdsa_verify_batch(h, None, None, None, 4, out.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert (out == 0).all()
    # collect: NULL check before the cap check, key buffer not cleared
    kb = np.full(4, 3, np.uint8)
    assert L.ufsecp_gpu_ecdsa_verify_collect(h, None, None, None, 4, kb.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert (kb == 3).all()
    # invalid inputs are verdicts, not errors (all-zero rows: bad pubkey prefix)
    res = np.full(2, 5, np.uint8)
    z = np.zeros(2 * 64, np.uint8)
    assert L.ufsecp_gpu_ecdsa_verify_lbtc_columns(h, z.ctypes.data, z.ctypes.data, z.ctypes.data, 2,
                                                  res.ctypes.data) == uf.UFSECP_OK
    assert (res == 0).all()
    # operations outside the verify path report UNSUPPORTED
    L.ufsecp_gpu_generator_mul_batch.argtypes = [uf._vp, uf._vp, uf.ctypes.c_size_t, uf._vp]
    assert L.ufsecp_gpu_generator_mul_batch(h, z.ctypes.data, 1, res.ctypes.data) == uf.UFSECP_ERR_GPU_UNSUPPORTED
    assert gpu_ctx.is_ready()
    info = uf.device_info(0)
    assert info.compute_units > 0 and info.global_mem_bytes > 0


@pytest.mark.parametrize("variant", range(12))
def test_every_kernel_variant_matches_oracle(gpu_ctx, oracle, variant):
    """The code-size variants (0..8) and the window-width variants (9: 3-bit P /
    18-bit G windows, 10: 5-bit P, 11: 16-bit G) of ufsecp_gpu_ext_set_variant
    compute identical verdicts."""
    _, wy, e = load_golden()
    m, p, s = ecdsa_corpus(oracle, 700, seed=60 + variant, tamper=0.2)
    mx, x, sx = schnorr_corpus(oracle, 700, seed=70 + variant, tamper=0.2)
    old = (gpu_ctx.get_variant(0)[0], gpu_ctx.get_variant(1)[0])
    old_small = (gpu_ctx.get_small_variant(0), gpu_ctx.get_small_variant(1))
    try:
        gpu_ctx.set_variant(0, variant)
        gpu_ctx.set_variant(1, variant)
        assert (gpu_ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
        assert (gpu_ctx.schnorr_verify_batch(mx, x, sx) == oracle.schnorr_verify_batch(mx, x, sx)).all()
        assert (gpu_ctx.ecdsa_verify_batch(wy["msgs"], wy["pubs"], wy["sigs"]) == wy["ref_valid"]).all()
        assert (gpu_ctx.ecdsa_verify_batch(e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"])
                == e["ecdsa_ref_valid"]).all()
        assert (gpu_ctx.schnorr_verify_batch(e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
                == e["schnorr_ref_valid"]).all()
    finally:
        gpu_ctx.set_variant(0, old[0])
        gpu_ctx.set_variant(1, old[1])
        for k in (0, 1):
            gpu_ctx.set_small_variant(k, *old_small[k])


@pytest.mark.parametrize("group", [64, 128])
def test_inversion_groups_match_oracle(gpu_ctx, oracle, group):
    """Block-wide batch inversion (ufsecp_gpu_ext_set_inversion_group): one
    inversion per block of 64 / 128 signatures for the table, the BIP-340 final
    Z and the ECDSA s.  Groups that hold invalid items (failed parses,
    off-curve keys, tampered signatures, results at infinity from the edge
    corpus) and partial last groups give the per-signature verdicts, through
    the compact, opaque-row and collect forms, small and chunked calls."""
    import ctypes
    _, wy, e = load_golden()
    saved = [(gpu_ctx.get_variant(k)[0], gpu_ctx.get_small_variant(k), gpu_ctx.get_lanes(k),
              gpu_ctx.get_inversion_group(k)) for k in (0, 1)]
    try:
        for k in (0, 1):
            gpu_ctx.set_variant(k, 4)              # no small-launch or two-lane path: every call is grouped
            gpu_ctx.set_inversion_group(k, group)
            assert gpu_ctx.get_inversion_group(k) == group
        assert (gpu_ctx.ecdsa_verify_batch(wy["msgs"], wy["pubs"], wy["sigs"]) == wy["ref_valid"]).all()
        assert (gpu_ctx.ecdsa_verify_batch(e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"])
                == e["ecdsa_ref_valid"]).all()
        assert (gpu_ctx.schnorr_verify_batch(e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
                == e["schnorr_ref_valid"]).all()
        for n in (1, 63, 129, 700):
            m, p, s = ecdsa_corpus(oracle, n, seed=900 + n, tamper=0.25)
            assert (gpu_ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
            mx, x, sx = schnorr_corpus(oracle, n, seed=950 + n, tamper=0.25)
            assert (gpu_ctx.schnorr_verify_batch(mx, x, sx) == oracle.schnorr_verify_batch(mx, x, sx)).all()
            kb = np.full(n, 5, np.uint8)
            got = gpu_ctx.schnorr_verify_collect(mx, x, sx, kb)
            assert (got == np.where(oracle.schnorr_verify_batch(mx, x, sx) == 1, 0, 5)).all()
        rows = opaque_rows_corpus(oracle, 600, seed=990)
        L = uf.load_library()
        L.ufsecp_gpu_ecdsa_verify_opaque_rows.argtypes = [uf._vp, uf._vp, ctypes.c_size_t, ctypes.c_size_t, uf._vp]
        got = np.full(len(rows), 9, np.uint8)
        assert L.ufsecp_gpu_ecdsa_verify_opaque_rows(gpu_ctx.handle, rows.ctypes.data, 129, len(rows),
                                                     got.ctypes.data) == uf.UFSECP_OK
        assert (got == oracle.ecdsa_verify_opaque_rows(rows, 129)).all()
        # a call of several pipeline chunks (16k, 32k, 64k, 128k items ...)
        mx, x, sx = schnorr_corpus(oracle, 3000, seed=991, tamper=0.05)
        want = oracle.schnorr_verify_batch(mx, x, sx)
        big = [np.ascontiguousarray(np.concatenate([a] * 70)) for a in (mx, x, sx)]
        assert (gpu_ctx.schnorr_verify_batch(*big) == np.concatenate([want] * 70)).all()
    finally:
        for k in (0, 1):
            v, small, lanes, grp = saved[k]
            gpu_ctx.set_variant(k, v)
            gpu_ctx.set_small_variant(k, *small)
            gpu_ctx.set_lanes(k, *lanes)
            gpu_ctx.set_inversion_group(k, grp)


def test_two_lanes_per_signature_match_oracle(gpu_ctx, oracle):
    """Two threads per signature (ufsecp_gpu_ext_set_lanes): the golden sets,
    the edge corpus, tampered corpora of odd sizes (partial warps) and the
    collect form give the one-lane verdicts."""
    _, wy, e = load_golden()
    old = [gpu_ctx.get_lanes(k) for k in (0, 1)]
    try:
        for k in (0, 1):
            gpu_ctx.set_lanes(k, 2, 1 << 22)
            assert gpu_ctx.get_lanes(k) == (2, 1 << 22)
        assert (gpu_ctx.ecdsa_verify_batch(wy["msgs"], wy["pubs"], wy["sigs"]) == wy["ref_valid"]).all()
        assert (gpu_ctx.ecdsa_verify_batch(e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"])
                == e["ecdsa_ref_valid"]).all()
        assert (gpu_ctx.schnorr_verify_batch(e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
                == e["schnorr_ref_valid"]).all()
        for n in (1, 17, 700):
            m, p, s = ecdsa_corpus(oracle, n, seed=800 + n, tamper=0.25)
            assert (gpu_ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
            m, x, s = schnorr_corpus(oracle, n, seed=900 + n, tamper=0.25)
            assert (gpu_ctx.schnorr_verify_batch(m, x, s) == oracle.schnorr_verify_batch(m, x, s)).all()
        m, p, s = ecdsa_corpus(oracle, 333, seed=33, tamper=0.3)
        want = oracle.ecdsa_verify_batch(m, p, s)
        kb = np.full(333, 0x77, np.uint8)
        gpu_ctx.ecdsa_verify_collect(m, p, s, kb)
        assert ((kb == 0) == (want == 1)).all() and (kb[want == 0] == 0x77).all()
    finally:
        for k in (0, 1):
            gpu_ctx.set_lanes(k, *((2, old[k][1]) if old[k][0] == 2 else (1, 0)))


def test_small_launch_variant_from_tuning(oracle, tmp_path, monkeypatch):
    """A tuning file's small-launch variants apply to launches up to their item
    limit and the main variant above it; verdicts match the oracle on both
    sides, and set_variant removes the small-launch variant."""
    import ultrafastsecp256k1_b200 as uf
    tune = tmp_path / "tuning.txt"
    tune.write_text("ecdsa_variant 4\necdsa_small_variant 6\necdsa_small_items 1000\n"
                    "schnorr_variant 8\nschnorr_small_variant 0\nschnorr_small_items 500\n")
    monkeypatch.setenv("UFSECP_B200_TUNING", str(tune))
    monkeypatch.delenv("UFSECP_B200_VARIANT_ECDSA", raising=False)
    monkeypatch.delenv("UFSECP_B200_VARIANT_SCHNORR", raising=False)
    ctx = uf.GpuContext(0)
    try:
        assert ctx.get_variant(0)[0] == 4 and ctx.get_small_variant(0) == (6, 1000)
        assert ctx.get_variant(1)[0] == 8 and ctx.get_small_variant(1) == (0, 500)
        for n in (999, 1000, 1001):
            m, p, s = ecdsa_corpus(oracle, n, seed=500 + n, tamper=0.2)
            assert (ctx.ecdsa_verify_batch(m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
        for n in (499, 500, 501):
            m, x, s = schnorr_corpus(oracle, n, seed=600 + n, tamper=0.2)
            assert (ctx.schnorr_verify_batch(m, x, s) == oracle.schnorr_verify_batch(m, x, s)).all()
        ctx.set_variant(0, 4)
        assert ctx.get_small_variant(0) == (-1, 0)
    finally:
        ctx.close()
