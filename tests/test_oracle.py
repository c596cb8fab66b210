"""The oracle is pinned before it is trusted: against the BIP-340 vectors and
the Wycheproof-derived ECDSA cases held by the reference's own tests, against
the edge corpus whose verdicts came from running the reference library, and
(where the reference library is built) against that library on fresh seeded
corpora."""
import numpy as np
import pytest

from conftest import N, P, ecdsa_corpus, load_golden, schnorr_corpus


def _cat(hexes):
    return np.frombuffer(b"".join(bytes.fromhex(h) for h in hexes), np.uint8)


def test_bip340_vectors(oracle):
    vecs, _, _ = load_golden()
    assert len(vecs) == 15
    got = oracle.schnorr_verify_batch(_cat(v["msg"] for v in vecs), _cat(v["pk"] for v in vecs),
                                      _cat(v["sig"] for v in vecs))
    for v, g in zip(vecs, got):
        assert bool(g) == v["expect_valid"] == v["ref_valid"], v["name"]


def test_bip340_signing_vectors(oracle):
    vecs, _, _ = load_golden()
    signed = [v for v in vecs if "sk" in v]
    assert len(signed) == 4
    xs, sigs, ok = oracle.schnorr_sign_batch(_cat(v["msg"] for v in signed), _cat(v["sk"] for v in signed),
                                             _cat(v["aux"] for v in signed))
    assert ok.all()
    for i, v in enumerate(signed):
        assert xs[32 * i:32 * i + 32].tobytes().hex() == v["pk"]
        assert sigs[64 * i:64 * i + 64].tobytes().hex() == v["sig"]


def test_wycheproof_ecdsa(oracle):
    _, wy, _ = load_golden()
    got = oracle.ecdsa_verify_batch(wy["msgs"], wy["pubs"], wy["sigs"])
    assert (got == wy["ref_valid"]).all()
    assert wy["ref_valid"].sum() > 0  # large-x / r+n cases are among the valid ones


def test_edge_corpus(oracle):
    _, _, e = load_golden()
    ge = oracle.ecdsa_verify_batch(e["ecdsa_msgs"], e["ecdsa_pubs"], e["ecdsa_sigs"])
    gs = oracle.schnorr_verify_batch(e["schnorr_msgs"], e["schnorr_pubs"], e["schnorr_sigs"])
    assert (ge == e["ecdsa_ref_valid"]).all()
    assert (gs == e["schnorr_ref_valid"]).all()
    # every edge class is present and rejected
    for cls in range(1, len(e["ecdsa_class_names"]) + 1):
        sel = e["ecdsa_class"] == cls
        assert sel.any() and ge[sel].sum() == 0, e["ecdsa_class_names"][cls - 1]
    for cls in range(1, len(e["schnorr_class_names"]) + 1):
        sel = e["schnorr_class"] == cls
        assert sel.any() and gs[sel].sum() == 0, e["schnorr_class_names"][cls - 1]


def test_oracle_vs_reference_library(oracle, reflib):
    m, p, s = ecdsa_corpus(oracle, 256, seed=11, tamper=0.2)
    assert (oracle.ecdsa_verify_batch(m, p, s) == reflib.ecdsa_verify_batch(m, p, s)).all()
    m, x, s = schnorr_corpus(oracle, 256, seed=12, tamper=0.2)
    assert (oracle.schnorr_verify_batch(m, x, s) == reflib.schnorr_verify_batch(m, x, s)).all()


@pytest.mark.parametrize("stride", [129, 141])
def test_opaque_rows_vs_reference_library(oracle, reflib, stride):
    from conftest import opaque_rows_corpus
    rows = opaque_rows_corpus(oracle, 600, seed=31 + stride, stride=stride)
    rc, ref = reflib.ecdsa_verify_opaque_rows(rows, stride)
    assert rc == 0
    got = oracle.ecdsa_verify_opaque_rows(rows, stride)
    assert (got == ref).all()
    assert 0 < int(got.sum()) < len(got)
    assert got[1::12].all()          # high-S twins are accepted on this surface


def test_oracle_signers_vs_reference_library(oracle, reflib):
    rng = np.random.default_rng(5)
    for i in range(16):
        sk = rng.integers(1, 256, 32, dtype=np.uint8).tobytes()
        msg = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        aux = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        pub, sig, ok = oracle.ecdsa_sign_batch(msg, sk)
        assert ok.all() and (pub.tobytes(), sig.tobytes()) == reflib.ecdsa_sign(msg, sk)
        xo, ssig, ok = oracle.schnorr_sign_batch(msg, sk, aux)
        assert ok.all() and (xo.tobytes(), ssig.tobytes()) == reflib.schnorr_sign(msg, sk, aux)


@pytest.mark.parametrize("n", [0, 1, 7])
def test_oracle_batch_sizes(oracle, n):
    m, p, s = ecdsa_corpus(oracle, max(n, 1), seed=3, tamper=0.0)
    got = oracle.ecdsa_verify_batch(m[:n], p[:n], s[:n])
    assert got.shape == (n,) and got.all()


def test_planted_mistake_is_caught(oracle):
    """A deliberately wrong expectation must fail the comparison the GPU tests use."""
    m, p, s = ecdsa_corpus(oracle, 8, seed=4, tamper=0.0)
    good = oracle.ecdsa_verify_batch(m, p, s)
    wrong = good.copy()
    wrong[3] ^= 1
    assert not (good == wrong).all()
