"""Per-item batch operations next to verify, against the oracle (pinned to the
reference library in test_oracle.py) and hashlib:
ufsecp_gpu_xonly_validate, _pubkey_validate, _commitment_verify,
_tagged_hash and _tagged_hash_var (include/ufsecp/ufsecp_gpu.h)."""
import ctypes
import hashlib

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import commitment_corpus, key_corpus

pytestmark = pytest.mark.gpu

_vp, _sz = uf._vp, ctypes.c_size_t


def _lib():
    L = uf.load_library()
    L.ufsecp_gpu_xonly_validate.argtypes = [_vp, _vp, _sz, _vp]
    L.ufsecp_gpu_pubkey_validate.argtypes = [_vp, _vp, _sz, _vp]
    L.ufsecp_gpu_commitment_verify.argtypes = [_vp] * 5 + [_sz, _vp]
    L.ufsecp_gpu_tagged_hash.argtypes = [_vp, _vp, _vp, _sz, _sz, _vp]
    L.ufsecp_gpu_tagged_hash_var.argtypes = [_vp, _vp, _vp, _vp, _sz, _sz, _vp]
    return L


def test_key_validation(gpu_ctx, oracle):
    L = _lib()
    pubs, xs = key_corpus(oracle, 3000, seed=51)
    out = np.full(len(pubs), 9, np.uint8)
    assert L.ufsecp_gpu_pubkey_validate(gpu_ctx.handle, pubs.ctypes.data, len(pubs), out.ctypes.data) == 0
    assert (out == oracle.pubkey_validate(pubs)).all()
    out2 = np.full(len(xs), 9, np.uint8)
    assert L.ufsecp_gpu_xonly_validate(gpu_ctx.handle, xs.ctypes.data, len(xs), out2.ctypes.data) == 0
    assert (out2 == oracle.xonly_validate(xs)).all()
    assert 0 < out.sum() < len(out) and 0 < out2.sum() < len(out2)


def test_commitment_verify(gpu_ctx, oracle, reflib):
    L = _lib()
    ix, tw, tx, par, _ = commitment_corpus(reflib, oracle, 1500, seed=52)
    # a tweak >= n is reduced; a tweak that cancels the key gives infinity (invalid)
    out = np.full(len(ix), 9, np.uint8)
    rc = L.ufsecp_gpu_commitment_verify(gpu_ctx.handle, ix.ctypes.data, tw.ctypes.data, tx.ctypes.data,
                                        par.ctypes.data, len(ix), out.ctypes.data)
    assert rc == 0
    assert (out == oracle.commitment_verify(ix, tw, tx, par)).all()
    assert 0 < out.sum() < len(out)


@pytest.mark.parametrize("msg_len", [1, 31, 32, 55, 56, 63, 64, 65, 119, 128, 200, 256])
def test_tagged_hash_fixed(gpu_ctx, msg_len):
    L = _lib()
    rng = np.random.default_rng(msg_len)
    tag = hashlib.sha256(b"TapBranch").digest()
    n = 777
    msgs = rng.integers(0, 256, (n, msg_len), dtype=np.uint8)
    out = np.zeros((n, 32), np.uint8)
    th = np.frombuffer(tag, np.uint8).copy()
    assert L.ufsecp_gpu_tagged_hash(gpu_ctx.handle, th.ctypes.data, msgs.ctypes.data, msg_len, n,
                                    out.ctypes.data) == 0
    for i in range(0, n, 37):
        assert out[i].tobytes() == hashlib.sha256(tag + tag + msgs[i].tobytes()).digest()


def test_tagged_hash_var(gpu_ctx):
    L = _lib()
    rng = np.random.default_rng(3)
    tag = hashlib.sha256(b"TapLeaf").digest()
    n, stride = 1000, 256
    lens = rng.integers(1, stride + 1, n).astype(np.uint32)
    msgs = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    out = np.zeros((n, 32), np.uint8)
    th = np.frombuffer(tag, np.uint8).copy()
    assert L.ufsecp_gpu_tagged_hash_var(gpu_ctx.handle, th.ctypes.data, msgs.ctypes.data, lens.ctypes.data,
                                        stride, n, out.ctypes.data) == 0
    for i in range(n):
        assert out[i].tobytes() == hashlib.sha256(tag + tag + msgs[i, :lens[i]].tobytes()).digest()
    bad = lens.copy()
    bad[5] = stride + 1
    assert L.ufsecp_gpu_tagged_hash_var(gpu_ctx.handle, th.ctypes.data, msgs.ctypes.data, bad.ctypes.data,
                                        stride, n, out.ctypes.data) == uf.UFSECP_ERR_BAD_INPUT
    assert (out == 0).all()      # cleared on failure


def test_ops_gating(gpu_ctx):
    L = _lib()
    z = np.zeros(64, np.uint8)
    out = np.full(2, 7, np.uint8)
    assert L.ufsecp_gpu_xonly_validate(None, z.ctypes.data, 2, out.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_xonly_validate(gpu_ctx.handle, None, 2, out.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert (out == 0).all()                       # cleared before the NULL check
    assert L.ufsecp_gpu_tagged_hash(gpu_ctx.handle, z.ctypes.data, z.ctypes.data, 257, 1, z.ctypes.data) == \
        uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_tagged_hash_var(gpu_ctx.handle, z.ctypes.data, z.ctypes.data, z.ctypes.data, 0, 1,
                                        z.ctypes.data) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_pubkey_validate(gpu_ctx.handle, None, 0, None) == uf.UFSECP_OK


@pytest.mark.parametrize("n", [1, 2, 7, 150, 5000, 20000])
def test_msm_matches_oracle(gpu_ctx, oracle, n):
    from conftest import msm_corpus
    L = uf.load_library()
    L.ufsecp_gpu_msm.argtypes = [_vp, _vp, _vp, _sz, _vp]
    ks, pts = msm_corpus(oracle, n, seed=60 + n)
    out = np.full(33, 7, np.uint8)
    rc = L.ufsecp_gpu_msm(gpu_ctx.handle, ks.ctypes.data, pts.ctypes.data, n, out.ctypes.data)
    st, want = oracle.msm(ks, pts)
    assert (rc, out.tobytes()) == (st, want)


def test_msm_error_codes(gpu_ctx, oracle):
    from conftest import N, msm_corpus
    L = uf.load_library()
    L.ufsecp_gpu_msm.argtypes = [_vp, _vp, _vp, _sz, _vp]
    ks, pts = msm_corpus(oracle, 10, seed=70)
    out = np.full(33, 7, np.uint8)
    bad_k = ks.copy()
    bad_k[3] = 0xFF
    bad_p = pts.copy()
    bad_p[2, 0] = 0x05
    # item 2's point fails before item 3's scalar: first bad item in index order wins
    both_k, both_p = bad_k.copy(), bad_p.copy()
    for k, p in ((bad_k, pts), (ks, bad_p), (both_k, both_p)):
        rc = L.ufsecp_gpu_msm(gpu_ctx.handle, k.ctypes.data, p.ctypes.data, 10, out.ctypes.data)
        assert rc == oracle.msm(k, p)[0] and (out == 0).all()
    two_k = np.concatenate([ks[:1], np.frombuffer((N - int.from_bytes(bytes(ks[0]), "big")).to_bytes(32, "big"),
                                                  np.uint8)[None]])
    two_p = np.ascontiguousarray(np.concatenate([pts[:1], pts[:1]]))
    rc = L.ufsecp_gpu_msm(gpu_ctx.handle, two_k.ctypes.data, two_p.ctypes.data, 2, out.ctypes.data)
    assert rc == uf.UFSECP_ERR_ARITH == 7 and (out == 0).all()


@pytest.mark.parametrize("affine", [1, 0])
def test_msm_repeated_and_opposite_points(oracle, monkeypatch, affine):
    """Equal points with equal scalars land in the same bucket of every window,
    so the bucket sums meet P + P (doubling) and P + (-P) (infinity) inside one
    chunk and across chunks; with and without the batch-affine chunk sums."""
    from conftest import msm_corpus
    monkeypatch.setenv("UFSECP_B200_RLC_AFFINE", str(affine))
    L = uf.load_library()
    L.ufsecp_gpu_msm.argtypes = [_vp, _vp, _vp, _sz, _vp]
    ks, pts = msm_corpus(oracle, 8, seed=81)
    neg = pts.copy()
    neg[:, 0] ^= 1                                  # 02 <-> 03: the opposite point
    cases = [
        (np.repeat(ks[:1], 40, 0), np.repeat(pts[:1], 40, 0)),
        (np.concatenate([np.repeat(ks[:1], 40, 0), ks[3:4]]),
         np.concatenate([np.repeat(pts[:1], 20, 0), np.repeat(neg[:1], 20, 0), pts[3:4]])),
        (np.concatenate([np.repeat(ks[:2], 33, 0), np.repeat(ks[:1], 17, 0), ks[4:8]]),
         np.concatenate([np.repeat(pts[:2], 33, 0), np.repeat(neg[:1], 17, 0), pts[4:8]])),
        (np.repeat(ks[:1], 300, 0), np.concatenate([np.repeat(pts[:1], 150, 0), np.repeat(neg[:1], 150, 0)])),
    ]
    with uf.GpuContext(0) as ctx:
        for k, p in cases:
            k, p = np.ascontiguousarray(k), np.ascontiguousarray(p)
            out = np.full(33, 7, np.uint8)
            rc = L.ufsecp_gpu_msm(ctx.handle, k.ctypes.data, p.ctypes.data, len(k), out.ctypes.data)
            st, want = oracle.msm(k, p)
            assert (rc, out.tobytes()) == (st, want)
