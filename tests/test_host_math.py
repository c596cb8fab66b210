"""The device math headers, compiled for the host by the test harness in
tests/native, checked against the oracle and Python integers (CPU only).  The
same headers are compiled for sm_100a into the product library; the -m gpu
tests check the device results."""
import ctypes
import hashlib
import random

import numpy as np
import pytest

from conftest import N, P, ecdsa_corpus, load_golden, schnorr_corpus

LAM = 0x5363AD4CC05C30E0A5261C028812645A122E22EA20816678DF02967C1B23BD72
GX = 0x79BE667EF9DCBBAC55A06295CE870B07029BFCDB2DCE28D959F2815B16F81798
GY = 0x483ADA7726A3C4655DA4FBFC0E1108A8FD17B448A68554199C47D08FFB10D4B8


def b32(v):
    return int(v).to_bytes(32, "big")


def call1(fn, *args):
    out = ctypes.create_string_buffer(32)
    fn(*[ctypes.c_char_p(a) for a in args], out)
    return int.from_bytes(out.raw, "big")


SPECIAL = [0, 1, 2, P - 1, P - 2, P, P + 1, 2**256 - 1, 2**255, 977, 2**32 + 977, N - 1, N, N + 1]


def _vals(k, seed):
    r = random.Random(seed)
    return SPECIAL + [r.randrange(2**256) for _ in range(k)]


def test_field_ops(host_math):
    vals = _vals(600, 1)
    for i, a in enumerate(vals):
        c = vals[(7 * i + 3) % len(vals)]
        assert call1(host_math.hm_fe_mul, b32(a), b32(c)) == a * c % P
        assert call1(host_math.hm_fe_sqr, b32(a)) == a * a % P
        assert call1(host_math.hm_fe_add, b32(a), b32(c)) == (a + c) % P
        assert call1(host_math.hm_fe_sub, b32(a), b32(c)) == (a - c) % P
        if a % P:
            assert call1(host_math.hm_fe_inv, b32(a)) == pow(a, -1, P)


def test_field_sqrt(host_math):
    r = random.Random(2)
    for _ in range(200):
        a = r.randrange(P)
        out = ctypes.create_string_buffer(32)
        ok = host_math.hm_fe_sqrt(b32(a), out)
        root = int.from_bytes(out.raw, "big")
        assert bool(ok) == (pow(a, (P - 1) // 2, P) in (0, 1))
        if ok:
            assert root * root % P == a


def test_scalar_ops(host_math):
    vals = _vals(600, 3)
    for i, a in enumerate(vals):
        a %= N
        c = vals[(5 * i + 1) % len(vals)] % N
        assert call1(host_math.hm_sc_mul, b32(a), b32(c)) == a * c % N
        if a:
            assert call1(host_math.hm_sc_inv, b32(a)) == pow(a, -1, N)


def test_glv_split(host_math):
    r = random.Random(4)
    ks = [0, 1, N - 1, N // 2, N // 2 + 1, LAM, N - LAM, 2**128, 2**128 - 1] + [r.randrange(N) for _ in range(3000)]
    for k in ks:
        k1 = ctypes.create_string_buffer(16)
        k2 = ctypes.create_string_buffer(16)
        ng = ctypes.create_string_buffer(2)
        host_math.hm_glv(b32(k), k1, k2, ng)
        v1 = int.from_bytes(k1.raw, "big") * (-1 if ng.raw[0] else 1)
        v2 = int.from_bytes(k2.raw, "big") * (-1 if ng.raw[1] else 1)
        assert (v1 + v2 * LAM - k) % N == 0
        assert abs(v1) < 2**128 and abs(v2) < 2**128


@pytest.mark.parametrize("w,nd", [(4, 33), (20, 7)])
def test_booth_recoding(host_math, w, nd):
    r = random.Random(w)
    for k in [0, 1, 2**128 - 1, 2**127, 2**127 - 1] + [r.randrange(2**128) for _ in range(2000)]:
        d = (ctypes.c_int32 * nd)()
        host_math.hm_booth(k.to_bytes(16, "big"), w, d)
        assert sum(d[j] << (w * j) for j in range(nd)) == k
        assert max(abs(x) for x in d) <= 2 ** (w - 1)


def test_challenge_hash(host_math):
    r = random.Random(6)
    tag = hashlib.sha256(b"BIP0340/challenge").digest()
    for _ in range(100):
        rx, px, m = (bytes(r.randrange(256) for _ in range(32)) for _ in range(3))
        out = ctypes.create_string_buffer(32)
        host_math.hm_challenge(rx, px, m, out)
        assert out.raw == hashlib.sha256(tag + tag + rx + px + m).digest()


def _padd(A, B):
    if A is None:
        return B
    if B is None:
        return A
    (x1, y1), (x2, y2) = A, B
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, P) % P
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, P) % P
    x3 = (lam * lam - x1 - x2) % P
    return x3, (lam * (x1 - x3) - y1) % P


def _pmul(k, A):
    R = None
    while k:
        if k & 1:
            R = _padd(R, A)
        A = _padd(A, A)
        k >>= 1
    return R


def test_dual_mul_including_infinity(host_math):
    r = random.Random(7)
    for i in range(40):
        d = r.randrange(1, N)
        Q = _pmul(d, (GX, GY))
        if Q[1] & 1:
            Q, d = (Q[0], P - Q[1]), N - d
        a, c = r.randrange(N), r.randrange(N)
        if i == 0:
            a, c = 0, 5
        if i == 1:
            a, c = 7, 0
        if i == 2:
            a, c = (N - d) % N, 1          # a*G + Q = infinity
        if i == 3:
            a, c = d, 1                    # a*G + Q = 2Q (doubling inside the adds)
        want = _padd(_pmul(a, (GX, GY)), _pmul(c, Q))
        xo, yo = ctypes.create_string_buffer(32), ctypes.create_string_buffer(32)
        rc = host_math.hm_dual_mul(b32(a), b32(Q[0]), b32(c), xo, yo)
        got = None if rc == 0 else (int.from_bytes(xo.raw, "big"), int.from_bytes(yo.raw, "big"))
        assert got == want, i


def _vb(fn, m, p, s):
    m, p, s = (np.ascontiguousarray(x, np.uint8) for x in (m, p, s))
    n = m.size // 32
    out = np.zeros(n, np.uint8)
    fn(m.ctypes.data_as(ctypes.c_void_p), p.ctypes.data_as(ctypes.c_void_p), s.ctypes.data_as(ctypes.c_void_p),
       ctypes.c_size_t(n), out.ctypes.data_as(ctypes.c_void_p))
    return out


def test_verify_logic_on_golden(host_math):
    vecs, wy, e = load_golden()
    cat = lambda hs: np.frombuffer(b"".join(bytes.fromhex(h) for h in hs), np.uint8)
    got = _vb(host_math.hm_schnorr_verify_batch, cat(v["msg"] for v in vecs), cat(v["pk"] for v in vecs),
              cat(v["sig"] for v in vecs))
    assert list(got) == [int(v["ref_valid"]) for v in vecs]
    assert (_vb(host_math.hm_ecdsa_verify_batch, wy["msgs"], wy["pubs"], wy["sigs"]) == wy["ref_valid"]).all()
    assert (_vb(host_math.hm_ecdsa_verify_batch, e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"])
            == e["ecdsa_ref_valid"]).all()
    assert (_vb(host_math.hm_schnorr_verify_batch, e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
            == e["schnorr_ref_valid"]).all()


def test_verify_logic_vs_oracle(host_math, oracle):
    m, p, s = ecdsa_corpus(oracle, 200, seed=21, tamper=0.1)
    assert (_vb(host_math.hm_ecdsa_verify_batch, m, p, s) == oracle.ecdsa_verify_batch(m, p, s)).all()
    m, x, s = schnorr_corpus(oracle, 200, seed=22, tamper=0.1)
    assert (_vb(host_math.hm_schnorr_verify_batch, m, x, s) == oracle.schnorr_verify_batch(m, x, s)).all()


def test_signers_vs_oracle(host_math, oracle):
    rng = np.random.default_rng(9)
    n = 64
    m = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    k = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    k[:, 0] &= 0x7F
    a = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    for kind, ps in ((0, 33), (1, 32)):
        pubs, sigs, ok = np.zeros(n * ps, np.uint8), np.zeros(n * 64, np.uint8), np.zeros(n, np.uint8)
        host_math.hm_sign_batch(kind, vp(m), vp(k), vp(a), ctypes.c_size_t(n), vp(pubs), vp(sigs), vp(ok))
        if kind == 0:
            p2, s2, ok2 = oracle.ecdsa_sign_batch(m, k)
        else:
            p2, s2, ok2 = oracle.schnorr_sign_batch(m, k, a)
        assert ok.all() and (pubs == p2).all() and (sigs == s2).all()
