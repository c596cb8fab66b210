"""Generate the committed golden fixtures for the verify path.

Run where the reference source tree and oracle/_ref exist, never on the GPU box:

    make -C oracle ref REF=<tree> -j8 && UFSECP_REFERENCE=<tree> python tests/golden/make_golden.py

Outputs (all verdicts come from RUNNING the reference's own CPU library,
oracle/_ref/libufsecp_ref.so, through its C ABI ufsecp_ecdsa_verify /
ufsecp_schnorr_verify):

* bip340_vectors.json  -- the BIP-340 vectors held by the reference test
  src/cpu/tests/test_bip340_vectors.cpp, parsed from its text: per vector the
  pubkey, message, signature, the expectation written in that test, and the
  reference library's verdict; vectors 0-3 also carry sk / aux_rand / the
  expected signature (signer pin).
* wycheproof_ecdsa.npz -- ECDSA cases assembled from the Wycheproof-derived
  reference tests audit/test_wycheproof_ecdsa*.cpp: every (pubkey, signature)
  literal found in those files (P1363 64-byte or DER, r,s <= 32 bytes), crossed
  with the Wycheproof message hashes used there, plus the low-S twin of every
  high-S signature.  The verdict is the reference library's.
* edge_corpus.npz -- seeded corpora (keys/messages from numpy PCG64 seeds,
  signatures from the reference signer) with the edge classes of the verify
  path: tampered bits, high-S twins, r = 0, s = 0, r >= n, s >= n, r >= p,
  pubkey x >= p, off-curve x, bad prefix, R = infinity (ECDSA z = -r*d).
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import RefLib  # noqa: E402

# the reference source tree (its test files hold the vectors); no default
REF = os.environ.get("UFSECP_REFERENCE", "")
P = 2**256 - 2**32 - 977
N = 0xFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFEBAAEDCE6AF48A03BBFD25E8CD0364141


def _join_literals(text: str) -> str:
    """Merge adjacent C string literals ("ab" "cd" -> "abcd")."""
    return re.sub(r'"\s*\n?\s*"', "", text)


# --------------------------------------------------------------- BIP-340 --
def bip340_vectors(ref: RefLib):
    path = os.path.join(REF, "src/cpu/tests/test_bip340_vectors.cpp")
    src = _join_literals(open(path).read())
    consts = dict(re.findall(r'static const char\*\s+(\w+)\s*=\s*"([0-9A-Fa-f]+)"', src))

    def val(expr: str) -> str:
        m = re.search(r'"([0-9A-Fa-f]+)"', expr)
        return m.group(1) if m else consts[expr.strip()]

    out = []
    # signing vectors 0-3: one function each
    for m in re.finditer(r"static void test_bip340_sign_vector_(\d+)\(\)\s*\{(.*?)\n\}", src, re.S):
        idx, body = int(m.group(1)), m.group(2)
        sk = re.search(r'Scalar::from_hex\(\s*"([0-9A-Fa-f]{64})"', body).group(1)
        get = lambda name: val(re.search(name + r"\s*=\s*h(?:32|64)\(([^)]*)\)", body).group(1))
        out.append(dict(name=f"V{idx}", sk=sk.lower(), pk=get("pk").lower(), aux=get("aux").lower(),
                        msg=get("msg").lower(), sig=get("expected_sig").lower(), expect_valid=True))
    # verify-only vectors 4-14: one brace block each inside test_bip340_verify_vectors
    body = re.search(r"static void test_bip340_verify_vectors\(\)\s*\{(.*?)\n\}", src, re.S).group(1)
    for blk in re.finditer(r"// Vector (\d+):.*?\{(.*?)CHECK\((!?)schnorr_verify", body, re.S):
        idx, b, neg = int(blk.group(1)), blk.group(2), blk.group(3)
        pk = val(re.search(r"pk\s*=\s*h32\(([^)]*)\)", b).group(1))
        msg = val(re.search(r"msg\s*=\s*h32\(([^)]*)\)", b).group(1))
        sig = val(re.search(r"h64\(([^)]*)\)", b).group(1))
        out.append(dict(name=f"V{idx}", pk=pk.lower(), msg=msg.lower(), sig=sig.lower(),
                        expect_valid=(neg == "")))
    out.sort(key=lambda d: int(d["name"][1:]))
    msgs = np.frombuffer(b"".join(bytes.fromhex(v["msg"]) for v in out), np.uint8)
    pks = np.frombuffer(b"".join(bytes.fromhex(v["pk"]) for v in out), np.uint8)
    sigs = np.frombuffer(b"".join(bytes.fromhex(v["sig"]) for v in out), np.uint8)
    verdicts = ref.schnorr_verify_batch(msgs, pks, sigs)
    for v, r in zip(out, verdicts):
        v["ref_valid"] = bool(r)
        if "sk" in v:
            got = ref.schnorr_sign(bytes.fromhex(v["msg"]), bytes.fromhex(v["sk"]), bytes.fromhex(v["aux"]))
            v["ref_sign_matches"] = got is not None and got[1].hex() == v["sig"] and got[0].hex() == v["pk"]
    return out


# ------------------------------------------------------------ Wycheproof --
def _der_to_rs(b: bytes):
    try:
        if len(b) < 8 or b[0] != 0x30:
            return None
        off = 2 if b[1] < 0x80 else 3
        vals = []
        for _ in range(2):
            if b[off] != 0x02:
                return None
            ln = b[off + 1]
            v = b[off + 2: off + 2 + ln]
            off += 2 + ln
            v = v.lstrip(b"\x00")
            if len(v) > 32:
                return None
            vals.append(v.rjust(32, b"\x00"))
        return vals[0] + vals[1]
    except IndexError:
        return None


def _compress(wx: str, wy: str) -> bytes:
    x = int(wx, 16)
    y = int(wy, 16)
    return bytes([0x02 | (y & 1)]) + x.to_bytes(32, "big")


def wycheproof_cases(ref: RefLib):
    files = sorted(f for f in os.listdir(os.path.join(REF, "audit"))
                   if f.startswith("test_wycheproof_ecdsa") and f.endswith(".cpp") and "sha512" not in f)
    msgs = [hashlib.sha256(b"123400").digest(), hashlib.sha256(b"").digest(),
            hashlib.sha256(b"bitcoin_test").digest()]
    cases = []
    for fi, f in enumerate(files):
        src = _join_literals(open(os.path.join(REF, "audit", f)).read())
        pubs = []
        for m in re.finditer(r'make_pubkey\(\s*"([0-9a-fA-F]{1,66})"\s*,\s*"([0-9a-fA-F]{1,66})"', src):
            pubs.append(_compress(m.group(1), m.group(2)))
        sigs = set()
        for lit in re.findall(r'"([0-9a-fA-F]{16,})"', src):
            if len(lit) % 2:
                continue
            b = bytes.fromhex(lit)
            if len(b) == 64:
                sigs.add(b)
            elif b[0] == 0x30:
                rs = _der_to_rs(b)
                if rs is not None:
                    sigs.add(rs)
        twins = set()
        for s in sigs:
            sv = int.from_bytes(s[32:], "big")
            if 0 < sv < N and sv > N // 2:
                twins.add(s[:32] + (N - sv).to_bytes(32, "big"))
        for pk in dict.fromkeys(pubs):
            for s in sorted(sigs | twins):
                for m in msgs:
                    cases.append((fi, m, pk, s))
    fidx = np.array([c[0] for c in cases], np.uint8)
    M = np.frombuffer(b"".join(c[1] for c in cases), np.uint8).reshape(-1, 32)
    Pk = np.frombuffer(b"".join(c[2] for c in cases), np.uint8).reshape(-1, 33)
    S = np.frombuffer(b"".join(c[3] for c in cases), np.uint8).reshape(-1, 64)
    v = ref.ecdsa_verify_batch(M, Pk, S, threads=8)
    return dict(msgs=M, pubs=Pk, sigs=S, ref_valid=v, file_index=fidx, files=np.array(files))


# ----------------------------------------------------------- edge corpus --
def _rand_sk(rng, n):
    out = np.zeros((n, 32), np.uint8)
    for i in range(n):
        while True:
            b = rng.integers(0, 256, 32, dtype=np.uint8)
            v = int.from_bytes(b.tobytes(), "big")
            if 1 <= v < N:
                out[i] = b
                break
    return out


def _small_curve_x():
    """Smallest x with x^3+7 a square (so x+p is a >= p encoding of a curve x)."""
    x = 1
    while True:
        y2 = (x**3 + 7) % P
        if pow(y2, (P - 1) // 2, P) == 1:
            return x
        x += 1


def _offcurve_x(rng):
    while True:
        x = int.from_bytes(rng.integers(0, 256, 32, dtype=np.uint8).tobytes(), "big") % P
        if pow((x**3 + 7) % P, (P - 1) // 2, P) != 1:
            return x


def edge_corpus(ref: RefLib, seed: int = 20261203, n: int = 768):
    rng = np.random.default_rng(seed)
    sks = _rand_sk(rng, n)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    e_pub = np.zeros((n, 33), np.uint8)
    e_sig = np.zeros((n, 64), np.uint8)
    s_pub = np.zeros((n, 32), np.uint8)
    s_sig = np.zeros((n, 64), np.uint8)
    for i in range(n):
        pk, sg = ref.ecdsa_sign(msgs[i].tobytes(), sks[i].tobytes())
        e_pub[i] = np.frombuffer(pk, np.uint8)
        e_sig[i] = np.frombuffer(sg, np.uint8)
        xo, ss = ref.schnorr_sign(msgs[i].tobytes(), sks[i].tobytes(), aux[i].tobytes())
        s_pub[i] = np.frombuffer(xo, np.uint8)
        s_sig[i] = np.frombuffer(ss, np.uint8)
    e_msg = msgs.copy()
    s_msg = msgs.copy()
    e_cls = np.zeros(n, np.uint8)  # 0 = untouched
    s_cls = np.zeros(n, np.uint8)
    small_x = _small_curve_x()
    be = lambda v: np.frombuffer(int(v).to_bytes(32, "big"), np.uint8)
    # ECDSA edge classes, cycling over indices
    classes_e = ["tamper_msg", "tamper_r", "tamper_s", "high_s", "r_zero", "s_zero", "r_ge_n", "s_ge_n",
                 "pk_x_ge_p", "pk_offcurve", "pk_prefix", "r_inf", "pk_wrong_parity"]
    for j, i in enumerate(range(0, n, 3)):
        c = classes_e[j % len(classes_e)]
        e_cls[i] = 1 + classes_e.index(c)
        if c == "tamper_msg":
            b = rng.integers(0, 256); e_msg[i, b // 8] ^= 1 << (b % 8)
        elif c == "tamper_r":
            b = rng.integers(0, 256); e_sig[i, b // 8] ^= 1 << (b % 8)
        elif c == "tamper_s":
            b = rng.integers(0, 256); e_sig[i, 32 + b // 8] ^= 1 << (b % 8)
        elif c == "high_s":
            s = int.from_bytes(e_sig[i, 32:].tobytes(), "big"); e_sig[i, 32:] = be(N - s)
        elif c == "r_zero":
            e_sig[i, :32] = 0
        elif c == "s_zero":
            e_sig[i, 32:] = 0
        elif c == "r_ge_n":
            e_sig[i, :32] = be(N + int(rng.integers(0, 2**30)))
        elif c == "s_ge_n":
            e_sig[i, 32:] = be(N + int(rng.integers(0, 2**30)))
        elif c == "pk_x_ge_p":
            y2 = (small_x**3 + 7) % P
            e_pub[i, 0] = 2; e_pub[i, 1:] = be(small_x + P)
        elif c == "pk_offcurve":
            e_pub[i, 1:] = be(_offcurve_x(rng))
        elif c == "pk_prefix":
            e_pub[i, 0] = int(rng.choice([0, 1, 4, 5, 6, 7, 0xff]))
        elif c == "r_inf":
            # z = -r*d mod n makes u1*G + u2*Q = w(z + r d)G = infinity
            d = int.from_bytes(sks[i].tobytes(), "big")
            r = int.from_bytes(e_sig[i, :32].tobytes(), "big")
            e_msg[i] = be((-r * d) % N)
        elif c == "pk_wrong_parity":
            e_pub[i, 0] ^= 1
    classes_s = ["tamper_msg", "tamper_r", "tamper_s", "s_zero", "s_ge_n", "r_ge_p", "pk_x_ge_p",
                 "pk_offcurve", "r_offcurve", "neg_s"]
    for j, i in enumerate(range(1, n, 3)):
        c = classes_s[j % len(classes_s)]
        s_cls[i] = 1 + classes_s.index(c)
        if c == "tamper_msg":
            b = rng.integers(0, 256); s_msg[i, b // 8] ^= 1 << (b % 8)
        elif c == "tamper_r":
            b = rng.integers(0, 256); s_sig[i, b // 8] ^= 1 << (b % 8)
        elif c == "tamper_s":
            b = rng.integers(0, 256); s_sig[i, 32 + b // 8] ^= 1 << (b % 8)
        elif c == "s_zero":
            s_sig[i, 32:] = 0
        elif c == "s_ge_n":
            s_sig[i, 32:] = be(N + int(rng.integers(0, 2**30)))
        elif c == "r_ge_p":
            s_sig[i, :32] = be(P + int(rng.integers(0, 2**20)))
        elif c == "pk_x_ge_p":
            s_pub[i] = be(small_x + P)
        elif c == "pk_offcurve":
            s_pub[i] = be(_offcurve_x(rng))
        elif c == "r_offcurve":
            s_sig[i, :32] = be(_offcurve_x(rng))
        elif c == "neg_s":
            s = int.from_bytes(s_sig[i, 32:].tobytes(), "big"); s_sig[i, 32:] = be(N - s)
    e_ref = ref.ecdsa_verify_batch(e_msg, e_pub, e_sig, threads=8)
    s_ref = ref.schnorr_verify_batch(s_msg, s_pub, s_sig, threads=8)
    return dict(seed=np.array([seed]), ecdsa_msgs=e_msg, ecdsa_pubs=e_pub, ecdsa_sigs=e_sig,
                ecdsa_class=e_cls, ecdsa_ref_valid=e_ref, ecdsa_class_names=np.array(classes_e),
                schnorr_msgs=s_msg, schnorr_pubs=s_pub, schnorr_sigs=s_sig,
                schnorr_class=s_cls, schnorr_ref_valid=s_ref, schnorr_class_names=np.array(classes_s),
                sks=sks, aux=aux)


def main():
    ref = RefLib()
    vecs = bip340_vectors(ref)
    with open(os.path.join(HERE, "bip340_vectors.json"), "w") as f:
        json.dump(vecs, f, indent=1)
    print(f"bip340: {len(vecs)} vectors; ref agrees with file expectations:",
          all(v["ref_valid"] == v["expect_valid"] for v in vecs))
    wy = wycheproof_cases(ref)
    np.savez_compressed(os.path.join(HERE, "wycheproof_ecdsa.npz"), **wy)
    print(f"wycheproof: {len(wy['ref_valid'])} cases, {int(wy['ref_valid'].sum())} valid, files={list(wy['files'])}")
    ec = edge_corpus(ref)
    np.savez_compressed(os.path.join(HERE, "edge_corpus.npz"), **ec)
    print("edge corpus: ecdsa valid", int(ec["ecdsa_ref_valid"].sum()), "/", len(ec["ecdsa_ref_valid"]),
          "schnorr valid", int(ec["schnorr_ref_valid"].sum()), "/", len(ec["schnorr_ref_valid"]))


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        sys.exit("set UFSECP_REFERENCE to the reference source tree")
    main()
