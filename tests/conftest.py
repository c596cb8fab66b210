"""Shared fixtures.  Tests marked `gpu` need a CUDA device (run with -m gpu);
everything else runs on the CPU (-m "not gpu")."""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
NATIVE = os.path.join(ROOT, "tests", "native")
P = 2**256 - 2**32 - 977
N = 0xFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFEBAAEDCE6AF48A03BBFD25E8CD0364141


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU test")


def _newer(target: str, *sources: str) -> bool:
    return os.path.exists(target) and all(os.path.getmtime(target) >= os.path.getmtime(s) for s in sources)


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle, ORACLE_SO
    src = os.path.join(ROOT, "oracle", "secp_oracle.c")
    if not _newer(ORACLE_SO, src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle import RefLib, ref_available
    if not ref_available():
        pytest.skip("reference library not built (oracle/_ref)")
    return RefLib()


@pytest.fixture(scope="session")
def host_math():
    """Host build of the device math headers (test harness, see tests/native)."""
    import ctypes
    import glob
    so = os.path.join(NATIVE, "libdevmath_host.so")
    src = os.path.join(NATIVE, "devmath_host.cpp")
    hdrs = glob.glob(os.path.join(ROOT, "ultrafastsecp256k1_b200", "csrc", "*.cuh"))
    if not _newer(so, src, *hdrs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", so, src], check=True)
    return ctypes.CDLL(so)


@pytest.fixture(scope="session")
def gpu_ctx():
    import ultrafastsecp256k1_b200 as uf
    ctx = uf.GpuContext(0)
    yield ctx
    ctx.close()


def load_golden():
    import json
    vecs = json.load(open(os.path.join(GOLDEN, "bip340_vectors.json")))
    wy = dict(np.load(os.path.join(GOLDEN, "wycheproof_ecdsa.npz")))
    edge = dict(np.load(os.path.join(GOLDEN, "edge_corpus.npz")))
    return vecs, wy, edge


def rand_keys(rng, n):
    """Private keys uniform in [1, n-1] (rejection sampling)."""
    out = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    for i in range(n):
        while True:
            v = int.from_bytes(out[i].tobytes(), "big")
            if 1 <= v < N:
                break
            out[i] = rng.integers(0, 256, 32, dtype=np.uint8)
    return out


def flip_random_bits(rng, arrs, frac):
    """Flip one random bit in msg, r or s (chosen uniformly) of a `frac` share of items.
    arrs = (msgs[n,32], sigs[n,64]); returns the tampered index set."""
    msgs, sigs = arrs
    n = msgs.shape[0]
    idx = rng.choice(n, size=int(round(frac * n)), replace=False)
    for i in idx:
        where = rng.integers(0, 3)
        bit = int(rng.integers(0, 256))
        if where == 0:
            msgs[i, bit // 8] ^= 1 << (bit % 8)
        elif where == 1:
            sigs[i, bit // 8] ^= 1 << (bit % 8)
        else:
            sigs[i, 32 + bit // 8] ^= 1 << (bit % 8)
    return set(int(i) for i in idx)


def ecdsa_corpus(oracle, n, seed, tamper=0.1):
    rng = np.random.default_rng(seed)
    sks = rand_keys(rng, n)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    pubs, sigs, ok = oracle.ecdsa_sign_batch(msgs, sks)
    assert ok.all()
    pubs = pubs.reshape(n, 33)
    sigs = sigs.reshape(n, 64)
    flip_random_bits(rng, (msgs, sigs), tamper)
    return msgs, pubs, sigs


def schnorr_corpus(oracle, n, seed, tamper=0.01):
    rng = np.random.default_rng(seed)
    sks = rand_keys(rng, n)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    xs, sigs, ok = oracle.schnorr_sign_batch(msgs, sks, aux)
    assert ok.all()
    xs = xs.reshape(n, 32)
    sigs = sigs.reshape(n, 64)
    flip_random_bits(rng, (msgs, sigs), tamper)
    return msgs, xs, sigs


def opaque_rows_corpus(oracle, n, seed, stride=129):
    """ECDSA rows [msg 32 | pubkey 33 | opaque sig 64 | tail] in the libsecp
    in-memory signature layout (r, s as 32-byte little-endian), with high-S
    twins, one-bit tampering, r / s = 0, r / s >= n, bad prefixes, x >= p and
    off-curve keys, and random tail bytes when stride > 129."""
    rng = np.random.default_rng(seed)
    msgs, pubs, sigs = ecdsa_corpus(oracle, n, seed, tamper=0.0)
    opaque = np.concatenate([sigs[:, 31::-1], sigs[:, :31:-1]], axis=1)   # BE r||s -> LE r, LE s
    rows = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    rows[:, :32] = msgs
    rows[:, 32:65] = pubs
    rows[:, 65:129] = opaque
    le = lambda v: np.frombuffer(v.to_bytes(32, "little"), np.uint8)
    for i in range(n):
        k = i % 12
        if k == 1:      # high-S twin: accepted on this surface
            s_ = int.from_bytes(bytes(rows[i, 97:129]), "little")
            rows[i, 97:129] = le(N - s_)
        elif k == 2:
            rows[i, int(rng.integers(0, 32))] ^= 1 << int(rng.integers(0, 8))
        elif k == 3:
            rows[i, 65:97] = 0
        elif k == 4:
            rows[i, 97:129] = 0
        elif k == 5:
            rows[i, 65:97] = le(N + int(rng.integers(0, 1000)))
        elif k == 6:
            rows[i, 97:129] = le(N + int(rng.integers(0, 1000)))
        elif k == 7:
            rows[i, 32] = 0x04
        elif k == 8:
            rows[i, 33:65] = np.frombuffer((P + int(rng.integers(0, 977))).to_bytes(32, "big"), np.uint8)
        elif k == 9:
            x = int.from_bytes(bytes(rows[i, 33:65]), "big")
            while True:
                x = (x + 1) % P
                if pow((x ** 3 + 7) % P, (P - 1) // 2, P) != 1:
                    break
            rows[i, 33:65] = np.frombuffer(x.to_bytes(32, "big"), np.uint8)
    return np.ascontiguousarray(rows)


def _offcurve(x):
    while True:
        x = (x + 1) % P
        if pow((x ** 3 + 7) % P, (P - 1) // 2, P) != 1:
            return x


def key_corpus(oracle, n, seed):
    """Compressed keys (33 B) and x-only keys (32 B) with invalid classes mixed in:
    prefix 0x00 / 0x04, x >= p, off-curve x."""
    rng = np.random.default_rng(seed)
    _, pubs, _ = ecdsa_corpus(oracle, n, seed, tamper=0.0)
    pubs = pubs.copy()
    xs = pubs[:, 1:].copy()
    for i in range(n):
        k = i % 6
        if k == 1:
            pubs[i, 0] = (0x00, 0x04, 0x05)[i % 3]
        elif k == 2:
            v = np.frombuffer((P + int(rng.integers(0, 977))).to_bytes(32, "big"), np.uint8)
            pubs[i, 1:] = v
            xs[i] = v
        elif k == 3:
            v = np.frombuffer(_offcurve(int.from_bytes(bytes(xs[i]), "big")).to_bytes(32, "big"), np.uint8)
            pubs[i, 1:] = v
            xs[i] = v
    return np.ascontiguousarray(pubs), np.ascontiguousarray(xs)


def tap_tweak(internal_x32: bytes, merkle_root: bytes) -> bytes:
    import hashlib
    tag = hashlib.sha256(b"TapTweak").digest()
    return hashlib.sha256(tag + tag + internal_x32 + merkle_root).digest()


def commitment_corpus(reflib, oracle, n, seed):
    """(internal_x, tweak, tweaked_x, parity) rows: outputs derived by the reference's
    ufsecp_taproot_output_key, with flipped parity / tampered x / off-curve internal keys."""
    import ctypes
    rng = np.random.default_rng(seed)
    _, xs = key_corpus(oracle, n, seed)
    L = reflib.L
    L.ufsecp_taproot_output_key.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                            ctypes.POINTER(ctypes.c_int)]
    ix, tw, tx, par, mr = [], [], [], [], []
    for i in range(n):
        x = bytes(xs[i])
        root = rng.bytes(32)
        out = ctypes.create_string_buffer(32)
        p = ctypes.c_int(0)
        rc = L.ufsecp_taproot_output_key(reflib.ctx(), x, root, out, ctypes.byref(p))
        ox, pp = (out.raw, p.value) if rc == 0 else (rng.bytes(32), 0)
        k = i % 5
        if k == 1:
            pp ^= 1
        elif k == 2:
            ox = bytes([ox[0] ^ 1]) + ox[1:]
        ix.append(x)
        tw.append(tap_tweak(x, root))
        tx.append(ox)
        par.append(pp)
        mr.append(root)
    cat = lambda v: np.frombuffer(b"".join(v), np.uint8).reshape(n, 32)
    return cat(ix), cat(tw), cat(tx), np.array(par, np.uint8), cat(mr)


def msm_corpus(oracle, n, seed):
    """Scalars below n (some 0, some n-1) and valid compressed points (repeats included)."""
    rng = np.random.default_rng(seed)
    _, pubs, _ = ecdsa_corpus(oracle, max(n // 2, 1), seed, tamper=0.0)
    pts = pubs[rng.integers(0, len(pubs), n)]
    ks = rand_keys(rng, n)
    if n > 3:
        ks[1] = 0
        ks[2] = np.frombuffer((N - 1).to_bytes(32, "big"), np.uint8)
    return np.ascontiguousarray(ks), np.ascontiguousarray(pts)
