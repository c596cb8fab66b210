"""CPU oracle for batch ECDSA / BIP-340 verification -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / reference legs of
``bench.py`` import this package.  The product library (ultrafastsecp256k1_b200)
never imports, links or falls back to anything here.

Two checkers live here:

* ``Oracle`` wraps ``liboracle.so``, the plain-C restatement of the reference's
  CPU verify semantics (``oracle/secp_oracle.c``; every function cites the
  reference file:line it follows).
* ``RefLib`` wraps ``_ref/libufsecp_ref.so``, the reference's own CPU library
  (UltrafastSecp256k1 v4.5.0) compiled from its sources by ``oracle/Makefile``.
  It is used to pin the restatement and as the timed CPU baseline.  Its C ABI
  is called exactly as a reference user would: ``ufsecp_ecdsa_verify(ctx,
  msg32, sig64, pubkey33)`` (src/cpu/src/impl/ufsecp_ecdsa.cpp:244) and
  ``ufsecp_schnorr_verify(ctx, msg32, sig64, pubkey_x32)`` (:992), verdict =
  return code == UFSECP_OK.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libufsecp_ref.so")

# The reference library writes its generator precompute cache (cache_w*.bin,
# ~250 MB) to SECP256K1_CACHE_DIR, else to the working directory
# (src/cpu/src/precompute.cpp:3267-3275); keep it out of the repository.
_CACHE_DIR = os.path.join(tempfile.gettempdir(), "ufsecp_ref_cache")
os.makedirs(_CACHE_DIR, exist_ok=True)
os.environ.setdefault("SECP256K1_CACHE_DIR", _CACHE_DIR)

_u8p = ctypes.POINTER(ctypes.c_uint8)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


def _as_u8(x) -> np.ndarray:
    if isinstance(x, (bytes, bytearray)):
        return np.frombuffer(bytes(x), dtype=np.uint8).copy()
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint8))


class Oracle:
    """ctypes view of liboracle.so (the plain-C restatement)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        self.L = L
        for name in ("oracle_ecdsa_verify_batch", "oracle_schnorr_verify_batch"):
            getattr(L, name).argtypes = [_u8p, _u8p, _u8p, ctypes.c_size_t, _u8p]
            getattr(L, name).restype = None
        L.oracle_msm.argtypes = [_u8p, _u8p, ctypes.c_size_t, _u8p]
        L.oracle_msm.restype = ctypes.c_int
        L.oracle_ops_batch.argtypes = [ctypes.c_int, _u8p, _u8p, _u8p, _u8p, ctypes.c_size_t, _u8p]
        L.oracle_ecdsa_verify_opaque_rows.argtypes = [_u8p, ctypes.c_size_t, ctypes.c_size_t, _u8p]
        L.oracle_ecdsa_sign_batch.argtypes = [_u8p, _u8p, ctypes.c_size_t, _u8p, _u8p, _u8p]
        L.oracle_schnorr_sign_batch.argtypes = [_u8p, _u8p, _u8p, ctypes.c_size_t, _u8p, _u8p, _u8p]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        for name in ("oracle_fe_mul", "oracle_sc_mul"):
            getattr(L, name).argtypes = [_u8p, _u8p, _u8p]
        for name in ("oracle_fe_inv", "oracle_sc_inv"):
            getattr(L, name).argtypes = [_u8p, _u8p]
        L.oracle_gen_mul.argtypes = [_u8p, _u8p, _u8p]
        L.oracle_gen_mul.restype = ctypes.c_int
        L.oracle_sha256.argtypes = [_u8p, ctypes.c_size_t, _u8p]

    def set_threads(self, n: int) -> None:
        self.L.oracle_set_threads(int(n))

    # ---- verify ---------------------------------------------------------
    def ecdsa_verify_batch(self, msgs, pubs33, sigs) -> np.ndarray:
        msgs, pubs33, sigs = _as_u8(msgs), _as_u8(pubs33), _as_u8(sigs)
        n = msgs.size // 32
        assert pubs33.size == 33 * n and sigs.size == 64 * n
        out = np.zeros(n, dtype=np.uint8)
        if n:
            self.L.oracle_ecdsa_verify_batch(_ptr(msgs), _ptr(pubs33), _ptr(sigs), n, _ptr(out))
        return out

    def schnorr_verify_batch(self, msgs, xonly32, sigs) -> np.ndarray:
        msgs, xonly32, sigs = _as_u8(msgs), _as_u8(xonly32), _as_u8(sigs)
        n = msgs.size // 32
        assert xonly32.size == 32 * n and sigs.size == 64 * n
        out = np.zeros(n, dtype=np.uint8)
        if n:
            self.L.oracle_schnorr_verify_batch(_ptr(msgs), _ptr(xonly32), _ptr(sigs), n, _ptr(out))
        return out

    # ---- signing (corpus generation) --------------------------------------
    def ecdsa_verify_opaque_rows(self, rows, stride: int) -> np.ndarray:
        """Rows [msg 32 | pubkey 33 | opaque LE r, s 64 | tail], `stride` bytes apart."""
        rows = _as_u8(rows)
        n = rows.size // stride
        out = np.zeros(n, np.uint8)
        if n:
            self.L.oracle_ecdsa_verify_opaque_rows(_ptr(rows), stride, n, _ptr(out))
        return out

    def _ops(self, op, n, a, b=None, c=None, d=None) -> np.ndarray:
        out = np.zeros(max(n, 1), np.uint8)
        arrs = [_as_u8(x) if x is not None else np.zeros(1, np.uint8) for x in (a, b, c, d)]
        self.L.oracle_ops_batch(op, *[_ptr(x) for x in arrs], n, _ptr(out))
        return out[:n]

    def xonly_validate(self, keys32) -> np.ndarray:
        k = _as_u8(keys32)
        return self._ops(0, k.size // 32, k)

    def pubkey_validate(self, pubs33) -> np.ndarray:
        p = _as_u8(pubs33)
        return self._ops(1, p.size // 33, p)

    def commitment_verify(self, internal_x32, tweak32, tweaked_x32, parity) -> np.ndarray:
        ix = _as_u8(internal_x32)
        return self._ops(2, ix.size // 32, ix, tweak32, tweaked_x32, parity)

    def msm(self, scalars32, points33):
        """(status, compressed sum): status 0 OK, 5 scalar >= n, 3 bad point, 7 infinity."""
        k, p = _as_u8(scalars32), _as_u8(points33)
        out = np.zeros(33, np.uint8)
        st = self.L.oracle_msm(_ptr(k), _ptr(p), k.size // 32, _ptr(out))
        return st, out.tobytes()

    def ecdsa_sign_batch(self, msgs, sks):
        msgs, sks = _as_u8(msgs), _as_u8(sks)
        n = msgs.size // 32
        pubs = np.zeros(33 * n, np.uint8)
        sigs = np.zeros(64 * n, np.uint8)
        ok = np.zeros(n, np.uint8)
        if n:
            self.L.oracle_ecdsa_sign_batch(_ptr(msgs), _ptr(sks), n, _ptr(pubs), _ptr(sigs), _ptr(ok))
        return pubs, sigs, ok

    def schnorr_sign_batch(self, msgs, sks, auxs):
        msgs, sks, auxs = _as_u8(msgs), _as_u8(sks), _as_u8(auxs)
        n = msgs.size // 32
        xs = np.zeros(32 * n, np.uint8)
        sigs = np.zeros(64 * n, np.uint8)
        ok = np.zeros(n, np.uint8)
        if n:
            self.L.oracle_schnorr_sign_batch(_ptr(msgs), _ptr(sks), _ptr(auxs), n, _ptr(xs), _ptr(sigs), _ptr(ok))
        return xs, sigs, ok

    # ---- arithmetic probes -------------------------------------------------
    def _bin(self, fn, a: bytes, b: bytes | None = None) -> bytes:
        out = np.zeros(32, np.uint8)
        args = [_ptr(_as_u8(a))] + ([_ptr(_as_u8(b))] if b is not None else []) + [_ptr(out)]
        fn(*args)
        return out.tobytes()

    def fe_mul(self, a: bytes, b: bytes) -> bytes:
        return self._bin(self.L.oracle_fe_mul, a, b)

    def fe_inv(self, a: bytes) -> bytes:
        return self._bin(self.L.oracle_fe_inv, a)

    def sc_mul(self, a: bytes, b: bytes) -> bytes:
        return self._bin(self.L.oracle_sc_mul, a, b)

    def sc_inv(self, a: bytes) -> bytes:
        return self._bin(self.L.oracle_sc_inv, a)

    def gen_mul(self, k: bytes):
        x = np.zeros(32, np.uint8)
        y = np.zeros(32, np.uint8)
        ok = self.L.oracle_gen_mul(_ptr(_as_u8(k)), _ptr(x), _ptr(y))
        return (x.tobytes(), y.tobytes()) if ok else None

    def sha256(self, data: bytes) -> bytes:
        out = np.zeros(32, np.uint8)
        d = _as_u8(data) if len(data) else np.zeros(1, np.uint8)
        self.L.oracle_sha256(_ptr(d), len(data), _ptr(out))
        return out.tobytes()


class RefLib:
    """ctypes view of the reference CPU library built into oracle/_ref/.

    One ``ufsecp_ctx`` per worker thread (the reference's contexts are
    single-thread, include/ufsecp/ufsecp.h), statically partitioned work.
    """

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(path)
        self.L = L
        L.ufsecp_ctx_create.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        L.ufsecp_ctx_create.restype = ctypes.c_int
        L.ufsecp_ctx_destroy.argtypes = [ctypes.c_void_p]
        for name in ("ufsecp_ecdsa_verify", "ufsecp_schnorr_verify"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _u8p, _u8p, _u8p]
            getattr(L, name).restype = ctypes.c_int
        L.ufsecp_ecdsa_sign.argtypes = [ctypes.c_void_p, _u8p, _u8p, _u8p]
        L.ufsecp_schnorr_sign.argtypes = [ctypes.c_void_p, _u8p, _u8p, _u8p, _u8p]
        L.ufsecp_pubkey_create.argtypes = [ctypes.c_void_p, _u8p, _u8p]
        L.ufsecp_pubkey_xonly.argtypes = [ctypes.c_void_p, _u8p, _u8p]
        L.ufsecp_schnorr_batch_verify.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_size_t]
        L.ufsecp_schnorr_batch_verify.restype = ctypes.c_int
        L.ufsecp_ecdsa_verify_opaque_rows.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_size_t, ctypes.c_size_t, _u8p]
        L.ufsecp_ecdsa_verify_opaque_rows.restype = ctypes.c_int
        L.ufsecp_schnorr_batch_identify_invalid.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_size_t,
                                                           ctypes.POINTER(ctypes.c_size_t),
                                                           ctypes.POINTER(ctypes.c_size_t)]
        L.ufsecp_schnorr_batch_identify_invalid.restype = ctypes.c_int
        L.ufsecp_set_cache_dir.argtypes = [ctypes.c_char_p]
        L.ufsecp_set_cache_dir(_CACHE_DIR.encode())
        self._tls = threading.local()
        self._ctxs = []
        self._lock = threading.Lock()
        # build the library's fixed-base tables once from the cache dir (it saves
        # them to the working directory when the cache dir has no copy yet)
        cwd = os.getcwd()
        try:
            os.chdir(_CACHE_DIR)
            self.ecdsa_sign(bytes(32), bytes(31) + b"\x01")
        finally:
            os.chdir(cwd)

    def ctx(self):
        c = getattr(self._tls, "ctx", None)
        if c is None:
            c = ctypes.c_void_p()
            rc = self.L.ufsecp_ctx_create(ctypes.byref(c))
            if rc != 0:
                raise RuntimeError(f"ufsecp_ctx_create failed: {rc}")
            self._tls.ctx = c
            with self._lock:
                self._ctxs.append(c)
        return c

    def _verify_range(self, fn, msgs, pubs, pstride, sigs, out, lo, hi):
        ctx = self.ctx()
        base_m = msgs.ctypes.data
        base_p = pubs.ctypes.data
        base_s = sigs.ctypes.data
        cast = ctypes.cast
        for i in range(lo, hi):
            rc = fn(ctx, cast(base_m + 32 * i, _u8p), cast(base_s + 64 * i, _u8p),
                    cast(base_p + pstride * i, _u8p))
            out[i] = 1 if rc == 0 else 0

    def _verify(self, fn, msgs, pubs, pstride, sigs, threads):
        msgs, pubs, sigs = _as_u8(msgs), _as_u8(pubs), _as_u8(sigs)
        n = msgs.size // 32
        out = np.zeros(n, np.uint8)
        threads = max(1, min(threads or (os.cpu_count() or 1), n or 1))
        if threads == 1:
            self._verify_range(fn, msgs, pubs, pstride, sigs, out, 0, n)
        else:
            with ThreadPoolExecutor(threads) as ex:
                futs = [ex.submit(self._verify_range, fn, msgs, pubs, pstride, sigs, out,
                                  n * k // threads, n * (k + 1) // threads) for k in range(threads)]
                for f in futs:
                    f.result()
        return out

    def ecdsa_verify_batch(self, msgs, pubs33, sigs, threads: int = 1) -> np.ndarray:
        return self._verify(self.L.ufsecp_ecdsa_verify, msgs, pubs33, 33, sigs, threads)

    def schnorr_verify_batch(self, msgs, xonly32, sigs, threads: int = 1) -> np.ndarray:
        return self._verify(self.L.ufsecp_schnorr_verify, msgs, xonly32, 32, sigs, threads)

    def ecdsa_sign(self, msg32: bytes, sk32: bytes):
        pub = (ctypes.c_uint8 * 33)()
        sig = (ctypes.c_uint8 * 64)()
        m, k = _as_u8(msg32), _as_u8(sk32)
        rc1 = self.L.ufsecp_pubkey_create(self.ctx(), _ptr(k), ctypes.cast(pub, _u8p))
        rc2 = self.L.ufsecp_ecdsa_sign(self.ctx(), _ptr(m), _ptr(k), ctypes.cast(sig, _u8p))
        return (bytes(pub), bytes(sig)) if rc1 == 0 and rc2 == 0 else None

    def schnorr_sign(self, msg32: bytes, sk32: bytes, aux32: bytes):
        xo = (ctypes.c_uint8 * 32)()
        sig = (ctypes.c_uint8 * 64)()
        m, k, a = _as_u8(msg32), _as_u8(sk32), _as_u8(aux32)
        rc1 = self.L.ufsecp_pubkey_xonly(self.ctx(), _ptr(k), ctypes.cast(xo, _u8p))
        rc2 = self.L.ufsecp_schnorr_sign(self.ctx(), _ptr(m), _ptr(k), _ptr(a), ctypes.cast(sig, _u8p))
        return (bytes(xo), bytes(sig)) if rc1 == 0 and rc2 == 0 else None

    def ecdsa_verify_opaque_rows(self, rows, stride: int):
        """ufsecp_ecdsa_verify_opaque_rows: (return code, per-row verdicts)."""
        rows = _as_u8(rows)
        n = rows.size // stride
        out = np.zeros(max(n, 1), np.uint8)
        rc = self.L.ufsecp_ecdsa_verify_opaque_rows(self.ctx(), _ptr(rows), stride, n, _ptr(out))
        return rc, out[:n]

    def msm(self, scalars32, points33):
        """ufsecp_multi_scalar_mul: (return code, compressed sum)."""
        k, p = _as_u8(scalars32), _as_u8(points33)
        out = np.zeros(33, np.uint8)
        self.L.ufsecp_multi_scalar_mul.argtypes = [ctypes.c_void_p, _u8p, _u8p, ctypes.c_size_t, _u8p]
        rc = self.L.ufsecp_multi_scalar_mul(self.ctx(), _ptr(k), _ptr(p), k.size // 32, _ptr(out))
        return rc, out.tobytes()

    def schnorr_batch_verify_rows(self, rows128: np.ndarray) -> int:
        """ufsecp_schnorr_batch_verify over 128-byte rows pk|msg|sig (RLC form)."""
        rows = _as_u8(rows128)
        return self.L.ufsecp_schnorr_batch_verify(self.ctx(), _ptr(rows), rows.size // 128)

    def schnorr_batch_identify_invalid_rows(self, rows128: np.ndarray, capacity: int | None = None):
        """ufsecp_schnorr_batch_identify_invalid: (code, indices, total invalid)."""
        rows = _as_u8(rows128)
        n = rows.size // 128
        cap = n if capacity is None else capacity
        buf = (ctypes.c_size_t * max(cap, 1))()
        cnt = ctypes.c_size_t(cap)
        rc = self.L.ufsecp_schnorr_batch_identify_invalid(self.ctx(), _ptr(rows), n, buf, ctypes.byref(cnt))
        return rc, [buf[i] for i in range(min(cap, cnt.value))], cnt.value


class RefDriver:
    """Times the reference library's per-signature C ABI on all host threads
    (oracle/refdrv.c: one ufsecp_ctx per thread, static partition)."""

    def __init__(self, ref_path: str = REF_SO, drv_path: str = os.path.join(HERE, "librefdrv.so")):
        if not os.path.exists(ref_path):
            raise FileNotFoundError(f"{ref_path} missing")
        if not os.path.exists(drv_path):
            raise FileNotFoundError(f"{drv_path} missing: run `make -C oracle oracle`")
        self.L = ctypes.CDLL(drv_path)
        self.L.refdrv_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        self.L.refdrv_verify.argtypes = [ctypes.c_int, _u8p, _u8p, _u8p, ctypes.c_size_t, _u8p, ctypes.c_int]
        self.L.refdrv_sign.argtypes = [ctypes.c_int, _u8p, _u8p, _u8p, ctypes.c_size_t, _u8p, _u8p, _u8p,
                                       ctypes.c_int]
        rc = self.L.refdrv_open(ref_path.encode(), _CACHE_DIR.encode())
        if rc != 0:
            raise RuntimeError(f"refdrv_open failed: {rc}")

    def verify(self, kind: int, msgs, pubs, sigs, threads: int) -> np.ndarray:
        msgs, pubs, sigs = _as_u8(msgs), _as_u8(pubs), _as_u8(sigs)
        n = msgs.size // 32
        out = np.zeros(n, np.uint8)
        rc = self.L.refdrv_verify(kind, _ptr(msgs), _ptr(pubs), _ptr(sigs), n, _ptr(out), int(threads))
        if rc != 0:
            raise RuntimeError(f"refdrv_verify failed: {rc}")
        return out


    def sign(self, kind: int, msgs, sks, auxs, threads: int):
        """Reference signers on all threads: returns (pubs, sigs, ok)."""
        msgs, sks = _as_u8(msgs), _as_u8(sks)
        auxs = _as_u8(auxs) if auxs is not None else np.zeros(1, np.uint8)
        n = msgs.size // 32
        ps = 33 if kind == 0 else 32
        pubs, sigs, ok = np.zeros(n * ps, np.uint8), np.zeros(n * 64, np.uint8), np.zeros(n, np.uint8)
        self.L.refdrv_sign(kind, _ptr(msgs), _ptr(sks), _ptr(auxs), n, _ptr(pubs), _ptr(sigs), _ptr(ok), int(threads))
        return pubs.reshape(n, ps), sigs.reshape(n, 64), ok


def ref_available() -> bool:
    return os.path.exists(REF_SO)
