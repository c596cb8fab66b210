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


def test_key_validation_vs_reference_library(oracle, reflib):
    import ctypes
    from conftest import key_corpus
    pubs, xs = key_corpus(oracle, 300, seed=41)
    L = reflib.L
    L.ufsecp_pubkey_parse.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
    out = ctypes.create_string_buffer(33)
    ref = np.array([L.ufsecp_pubkey_parse(reflib.ctx(), bytes(p), 33, out) == 0 for p in pubs], np.uint8)
    assert (oracle.pubkey_validate(pubs) == ref).all()
    # an x-only key is valid iff 02 || x parses
    ref_x = np.array([L.ufsecp_pubkey_parse(reflib.ctx(), b"\x02" + bytes(x), 33, out) == 0 for x in xs], np.uint8)
    assert (oracle.xonly_validate(xs) == ref_x).all()
    assert 0 < ref.sum() < len(ref) and 0 < ref_x.sum() < len(ref_x)


def test_commitment_vs_reference_library(oracle, reflib):
    import ctypes
    from conftest import commitment_corpus
    ix, tw, tx, par, mr = commitment_corpus(reflib, oracle, 200, seed=42)
    L = reflib.L
    L.ufsecp_taproot_verify.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                        ctypes.c_char_p, ctypes.c_size_t]
    ref = np.array([L.ufsecp_taproot_verify(reflib.ctx(), bytes(tx[i]), int(par[i]), bytes(ix[i]), bytes(mr[i]), 32)
                    == 0 for i in range(len(ix))], np.uint8)
    got = oracle.commitment_verify(ix, tw, tx, par)
    assert (got == ref).all()
    assert 0 < ref.sum() < len(ref)


def test_msm_vs_reference_library(oracle, reflib):
    from conftest import msm_corpus
    for n, seed in ((1, 1), (7, 2), (150, 3)):
        ks, pts = msm_corpus(oracle, n, seed)
        assert oracle.msm(ks, pts) == reflib.msm(ks, pts)
    ks, pts = msm_corpus(oracle, 10, 4)
    bad_k = ks.copy()
    bad_k[3] = 0xFF                                       # scalar >= n
    assert oracle.msm(bad_k, pts)[0] == reflib.msm(bad_k, pts)[0] == 5
    bad_p = pts.copy()
    bad_p[5, 0] = 0x04                                    # invalid point
    assert oracle.msm(ks, bad_p)[0] == reflib.msm(ks, bad_p)[0] == 3
    # k P + (n - k) P = infinity
    two_k = np.concatenate([ks[:1], np.frombuffer((N - int.from_bytes(bytes(ks[0]), "big")).to_bytes(32, "big"),
                                                  np.uint8)[None]])
    two_p = np.concatenate([pts[:1], pts[:1]])
    assert oracle.msm(two_k, two_p)[0] == reflib.msm(two_k, two_p)[0] == 7


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
