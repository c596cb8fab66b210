"""Consensus row / column surfaces: ufsecp_gpu_ecdsa_verify_opaque_rows (and its
alias _lbtc_rows), ufsecp_gpu_ecdsa_verify_lbtc_columns and
ufsecp_gpu_schnorr_verify_lbtc_columns.

The ECDSA surfaces read the libsecp in-memory signature (r then s, little-endian)
and accept high-S; their verdicts must equal the oracle's restatement and, where
the reference library is built, the reference CPU's own
ufsecp_ecdsa_verify_opaque_rows on the same rows (stride 129 and a longer stride
with tail bytes).  The BIP-340 columns must equal the plain BIP-340 verify.
"""
import ctypes

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import load_golden, opaque_rows_corpus, schnorr_corpus

pytestmark = pytest.mark.gpu


def _rows_call(L, name, h, rows, stride, n):
    out = np.full(max(n, 1), 7, np.uint8)
    getattr(L, name).argtypes = [uf._vp, uf._vp, ctypes.c_size_t, ctypes.c_size_t, uf._vp]
    rc = getattr(L, name)(h, rows.ctypes.data, stride, n, out.ctypes.data)
    return rc, out[:n]


@pytest.mark.parametrize("stride", [129, 141])
def test_opaque_rows_match_oracle_and_reference(gpu_ctx, oracle, stride):
    L = uf.load_library()
    rows = opaque_rows_corpus(oracle, 3000, seed=70 + stride, stride=stride)
    want = oracle.ecdsa_verify_opaque_rows(rows, stride)
    assert 0 < int(want.sum()) < len(want) and want[1::12].all()      # high-S twins valid
    for name in ("ufsecp_gpu_ecdsa_verify_opaque_rows", "ufsecp_gpu_ecdsa_verify_lbtc_rows"):
        rc, got = _rows_call(L, name, gpu_ctx.handle, rows, stride, len(rows))
        assert rc == uf.UFSECP_OK
        assert (got == want).all(), name
    from oracle import RefLib, ref_available
    if ref_available():
        rc, ref = RefLib().ecdsa_verify_opaque_rows(rows, stride)
        assert rc == 0 and (ref == want).all()


def test_ecdsa_lbtc_columns_match_rows(gpu_ctx, oracle):
    L = uf.load_library()
    rows = opaque_rows_corpus(oracle, 2500, seed=90)
    d, p, s = (np.ascontiguousarray(rows[:, a:b]) for a, b in ((0, 32), (32, 65), (65, 129)))
    out = np.full(len(rows), 9, np.uint8)
    rc = L.ufsecp_gpu_ecdsa_verify_lbtc_columns(gpu_ctx.handle, d.ctypes.data, p.ctypes.data, s.ctypes.data,
                                                len(rows), out.ctypes.data)
    assert rc == uf.UFSECP_OK
    assert (out == oracle.ecdsa_verify_opaque_rows(rows, 129)).all()


def test_schnorr_lbtc_columns_match_plain(gpu_ctx, oracle):
    L = uf.load_library()
    _, _, edge = load_golden()
    m, x, s = schnorr_corpus(oracle, 3000, seed=91, tamper=0.05)
    m = np.concatenate([m, edge["schnorr_msgs"]])
    x = np.concatenate([x, edge["schnorr_pubs"]])
    s = np.concatenate([s, edge["schnorr_sigs"]])
    out = np.full(len(m), 9, np.uint8)
    rc = L.ufsecp_gpu_schnorr_verify_lbtc_columns(gpu_ctx.handle, m.ctypes.data, x.ctypes.data, s.ctypes.data,
                                                  len(m), out.ctypes.data)
    assert rc == uf.UFSECP_OK
    assert (out == oracle.schnorr_verify_batch(m, x, s)).all()
    assert (out == gpu_ctx.schnorr_verify_batch(m, x, s)).all()


def test_opaque_rows_gating(gpu_ctx):
    L = uf.load_library()
    rows = np.zeros(2 * 129, np.uint8)
    out = np.full(2, 7, np.uint8)
    f = L.ufsecp_gpu_ecdsa_verify_opaque_rows
    f.argtypes = [uf._vp, uf._vp, ctypes.c_size_t, ctypes.c_size_t, uf._vp]
    assert f(None, rows.ctypes.data, 129, 2, out.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert f(gpu_ctx.handle, rows.ctypes.data, 128, 2, out.ctypes.data) == uf.UFSECP_ERR_BAD_INPUT
    assert f(gpu_ctx.handle, None, 129, 2, out.ctypes.data) == uf.UFSECP_ERR_NULL_ARG
    assert (out == 7).all()                      # NULL check comes before clearing
    assert f(gpu_ctx.handle, None, 129, 0, None) == uf.UFSECP_OK
    assert f(gpu_ctx.handle, rows.ctypes.data, 129, 2, out.ctypes.data) == uf.UFSECP_OK
    assert (out == 0).all()
