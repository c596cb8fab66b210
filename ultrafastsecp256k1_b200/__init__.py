"""ultrafastsecp256k1_b200 -- B200-native batch ECDSA / BIP-340 verification.

The product is the C-ABI shared library ``lib/libufsecp_gpu.so`` (sm_100a
kernels + C++ host runtime) exporting the reference's GPU verify ABI
(``include/ufsecp/ufsecp_gpu.h``) plus B200 additions
(``include/ufsecp/ufsecp_gpu_ext.h``).  This module is a thin ctypes mirror of
that ABI for Python callers, the tests and the benchmark: same function names,
same argument meaning, same error codes (a non-OK code raises
``UfsecpError``).  There is no CPU path: if the library or a CUDA device is
missing, the calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libufsecp_gpu.so")

UFSECP_OK = 0
UFSECP_ERR_NULL_ARG = 1
UFSECP_ERR_BAD_PUBKEY = 3
UFSECP_ERR_BAD_SIG = 4
UFSECP_ERR_BAD_INPUT = 5
UFSECP_ERR_VERIFY_FAIL = 6
UFSECP_ERR_ARITH = 7
UFSECP_ERR_INTERNAL = 9
UFSECP_ERR_CANCELLED = 13
UFSECP_ERR_GPU_UNAVAILABLE = 100
UFSECP_ERR_GPU_DEVICE = 101
UFSECP_ERR_GPU_LAUNCH = 102
UFSECP_ERR_GPU_MEMORY = 103
UFSECP_ERR_GPU_UNSUPPORTED = 104
UFSECP_ERR_GPU_BACKEND = 105
UFSECP_ERR_GPU_QUEUE = 106
UFSECP_GPU_BACKEND_CUDA = 1
MAX_BATCH = 1 << 26

_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_lib: Optional[ctypes.CDLL] = None


class UfsecpError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str = ""):
        self.code = code
        super().__init__(f"{where}: ufsecp error {code}{' (' + msg + ')' if msg else ''}")


class Job(ctypes.Structure):
    """ufsecp_gpu_ext_job_t: one caller batch of a mixed ufsecp_gpu_ext_verify_jobs call."""
    _fields_ = [("kind", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("count", ctypes.c_size_t),
                ("msg_hashes32", _vp), ("pubkeys", _vp), ("sigs64", _vp), ("out_results", _vp)]


CANCEL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


class CancelToken(ctypes.Structure):
    """ufsecp_cancel_token (include/ufsecp/ufsecp_cancel.h)."""
    _fields_ = [("is_cancelled", CANCEL_FN), ("user", ctypes.c_void_p), ("check_interval", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("max_launch_items", ctypes.c_uint32),
                ("memory_budget_bytes", ctypes.c_uint64), ("batch_window_us", ctypes.c_uint32),
                ("key_cache_log2", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests_done", ctypes.c_uint64), ("items_done", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("peak_budget_bytes", ctypes.c_uint64), ("reserved_bytes", ctypes.c_uint64),
                ("pending_requests", ctypes.c_uint64),
                ("peak_slots_in_flight", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("mean_us", ctypes.c_double), ("busy_s", ctypes.c_double), ("span_s", ctypes.c_double),
                ("cache_lookups", ctypes.c_uint64), ("cache_hits", ctypes.c_uint64)]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 128), ("global_mem_bytes", ctypes.c_uint64),
                ("compute_units", ctypes.c_uint32), ("max_clock_mhz", ctypes.c_uint32),
                ("max_threads_per_block", ctypes.c_uint32), ("backend_id", ctypes.c_uint32),
                ("device_index", ctypes.c_uint32)]


# name -> (restype, argtypes) of every symbol the mirror binds
_SIGS = {
    "ufsecp_gpu_backend_count": (ctypes.c_uint32, [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32]),
    "ufsecp_gpu_backend_name": (ctypes.c_char_p, [ctypes.c_uint32]),
    "ufsecp_gpu_is_available": (ctypes.c_int, [ctypes.c_uint32]),
    "ufsecp_gpu_device_count": (ctypes.c_uint32, [ctypes.c_uint32]),
    "ufsecp_gpu_device_info": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(DeviceInfo)]),
    "ufsecp_gpu_ctx_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_uint32, ctypes.c_uint32]),
    "ufsecp_gpu_ctx_destroy": (None, [_vp]),
    "ufsecp_gpu_is_ready": (ctypes.c_int, [_vp]),
    "ufsecp_gpu_last_error": (ctypes.c_int, [_vp]),
    "ufsecp_gpu_last_error_msg": (ctypes.c_char_p, [_vp]),
    "ufsecp_gpu_error_str": (ctypes.c_char_p, [ctypes.c_int]),
    "ufsecp_gpu_ecdsa_verify_batch": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_schnorr_verify_batch": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ecdsa_verify_collect": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_schnorr_verify_collect": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ext_ecdsa_verify_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp, _vp]),
    "ufsecp_gpu_ext_schnorr_verify_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp, _vp]),
    "ufsecp_gpu_ext_verify_jobs": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_size_t]),
    "ufsecp_gpu_ext_verify_jobs_noalloc": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ext_sign_device": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, _vp, ctypes.c_size_t, _vp, _vp, _vp,
                                                  _vp]),
    "ufsecp_gpu_ext_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "ufsecp_gpu_ext_device_props": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                                   ctypes.POINTER(ctypes.c_int)]),
    "ufsecp_gpu_ext_set_variant": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "ufsecp_gpu_ext_get_variant": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(ctypes.c_int)]),
    "ufsecp_gpu_ext_get_small_variant": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                        ctypes.POINTER(ctypes.c_uint32)]),
    "ufsecp_gpu_ext_set_small_variant": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint32]),
    "ufsecp_gpu_ext_set_lanes": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint32]),
    "ufsecp_gpu_ext_get_lanes": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_uint32)]),
    "ufsecp_gpu_ext_set_rlc_chunk": (ctypes.c_int, [_vp, ctypes.c_uint32]),
    "ufsecp_gpu_ext_get_rlc_chunk": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "ufsecp_gpu_ext_imad_peak": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "ufsecp_gpu_ext_diag": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ext_probe": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_float)]),
    "ufsecp_gpu_ext_schnorr_verify_rlc": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp,
                                                         ctypes.c_int, _vp, _vp]),
    "ufsecp_gpu_ext_schnorr_verify_rlc_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t,
                                                                _vp, ctypes.c_int, _vp, _vp, _vp]),
    "ufsecp_gpu_ext_server_create": (ctypes.c_int, [_vp, ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)]),
    "ufsecp_gpu_ext_server_submit": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_size_t,
                                                    ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint32]),
    "ufsecp_gpu_ext_server_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStats), ctypes.c_int]),
    "ufsecp_gpu_ext_server_destroy": (None, [_vp]),
    "ufsecp_gpu_ext_rlc_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_rlc_key_hits": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_verify_batch_sharded": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_size_t, ctypes.c_uint32,
                                                           _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ext_set_key_table": (ctypes.c_int, [_vp, ctypes.c_uint32]),
    "ufsecp_gpu_ext_set_rlc_locate": (ctypes.c_int, [_vp, ctypes.c_int]),
    "ufsecp_gpu_ext_rlc_located": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_set_inversion_group": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "ufsecp_gpu_ext_get_inversion_group": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "ufsecp_gpu_ext_inject_fault": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_int]),
    "ufsecp_gpu_ext_engine_hook_inject_fault": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_int]),
    "ufsecp_gpu_ext_server_submit_cancellable": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_size_t, _vp,
                                                                ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_server_cancel": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint32]),
    "ufsecp_gpu_ext_key_table_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "ufsecp_gpu_ext_rlc_input_digest": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "ufsecp_gpu_ext_schnorr_batch_verify": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    "ufsecp_gpu_ext_schnorr_batch_identify_invalid": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t,
                                                                     ctypes.POINTER(ctypes.c_size_t),
                                                                     ctypes.POINTER(ctypes.c_size_t)]),
}


def lib_path() -> str:
    return LIB_PATH


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libufsecp_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run `python -m ultrafastsecp256k1_b200.build`")
    L = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


_U8 = np.dtype(np.uint8)
# ufsecp_gpu_ext_job_t as a numpy record (the Job structure's layout, 48 bytes)
_JOB_DTYPE = np.dtype([("kind", "<u4"), ("reserved", "<u4"), ("count", "<u8"), ("msg_hashes32", "<u8"),
                       ("pubkeys", "<u8"), ("sigs64", "<u8"), ("out_results", "<u8")])
assert _JOB_DTYPE.itemsize == ctypes.sizeof(Job)


def _u8(x) -> np.ndarray:
    """x as a flat contiguous uint8 array (no copy when it already is one)."""
    if isinstance(x, np.ndarray) and x.dtype == np.uint8 and x.flags.c_contiguous:
        return x.reshape(-1)
    if isinstance(x, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(x), dtype=np.uint8)
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint8)).reshape(-1)


def _buf(x, n_bytes: int, name: str) -> np.ndarray:
    a = _u8(x)
    if a.size != n_bytes:
        raise ValueError(f"{name}: expected {n_bytes} bytes, got {a.size}")
    return a


def _ptr(a: np.ndarray) -> int:
    return a.__array_interface__["data"][0]


_CCHAR = ctypes.c_char


def _addr(a: np.ndarray) -> int:
    """Address of a non-empty contiguous array: through the buffer protocol
    (a third of __array_interface__'s cost), read-only arrays through _ptr."""
    try:
        return ctypes.addressof(_CCHAR.from_buffer(a))
    except (TypeError, ValueError):
        return _ptr(a)


def _flat_u8(x) -> np.ndarray:
    if type(x) is np.ndarray and x.dtype is _U8 and x.flags.c_contiguous:
        return x
    return _u8(x)


def _job_table(jobs):
    """The ufsecp_gpu_ext_job_t table of `jobs` as one numpy record array, the
    input arrays it points into (to keep alive), one verdict buffer for all
    jobs and each job's (offset, count) in it.  The per-job Python work is
    little more than the three buffer addresses."""
    keep, meta = [], []
    total = 0
    for job in jobs:
        kind, m, p, s = job[:4]
        segment = int(job[4]) if len(job) > 4 else 0      # kind 2: RLC segment length (0 = default)
        m, p, s = _flat_u8(m), _flat_u8(p), _flat_u8(s)
        n = m.size >> 5
        if p.size != (33 if kind == 0 else 32) * n:
            raise ValueError(f"pubkeys: expected {(33 if kind == 0 else 32) * n} bytes, got {p.size}")
        if s.size != 64 * n:
            raise ValueError(f"sigs64: expected {64 * n} bytes, got {s.size}")
        keep.append((m, p, s))
        meta.append((kind, segment, n, _addr(m) if n else 0, _addr(p) if n else 0, _addr(s) if n else 0, total))
        total += n
    out_all = np.zeros(max(1, total), np.uint8)
    tab = np.array(meta, _JOB_DTYPE) if meta else np.zeros(1, _JOB_DTYPE)
    if meta:
        o = tab["out_results"]
        o += _addr(out_all)
        o[tab["count"] == 0] = 0
    return tab, keep, out_all, [(t[6], t[2]) for t in meta]


def verify_batch_sharded(ctxs, kind: int, msg_hashes32, pubkeys, sigs64) -> np.ndarray:
    """ufsecp_gpu_ext_verify_batch_sharded: one host-buffer batch cut into
    contiguous shares over the contexts in `ctxs` (GpuContext objects, e.g. one
    per GPU), each share verified on its context in its own host thread;
    kind 0 ECDSA (33-byte keys) / 1 BIP-340 (32-byte keys)."""
    m, p, s = _flat_u8(msg_hashes32), _flat_u8(pubkeys), _flat_u8(sigs64)
    n = m.size >> 5
    out = np.zeros(max(1, n), np.uint8)
    arr = (_vp * max(1, len(ctxs)))(*[c.handle for c in ctxs])
    L = load_library()
    rc = L.ufsecp_gpu_ext_verify_batch_sharded(arr, len(ctxs), kind, _addr(m) if n else None,
                                               _addr(p) if n else None, _addr(s) if n else None, n,
                                               _addr(out) if n else None)
    if rc != UFSECP_OK:
        raise UfsecpError(rc, "verify_batch_sharded")
    return out[:n]


def backend_count() -> int:
    return load_library().ufsecp_gpu_backend_count(None, 0)


def is_available(backend_id: int = UFSECP_GPU_BACKEND_CUDA) -> bool:
    return bool(load_library().ufsecp_gpu_is_available(backend_id))


def device_count(backend_id: int = UFSECP_GPU_BACKEND_CUDA) -> int:
    return int(load_library().ufsecp_gpu_device_count(backend_id))


def device_info(device_index: int = 0, backend_id: int = UFSECP_GPU_BACKEND_CUDA) -> DeviceInfo:
    info = DeviceInfo()
    rc = load_library().ufsecp_gpu_device_info(backend_id, device_index, ctypes.byref(info))
    if rc != UFSECP_OK:
        raise UfsecpError(rc, "ufsecp_gpu_device_info")
    return info


def error_str(code: int) -> str:
    return load_library().ufsecp_gpu_error_str(code).decode()


class GpuContext:
    """One ``ufsecp_gpu_ctx`` (single-thread, like the reference's)."""

    def __init__(self, device_index: int = 0, backend_id: int = UFSECP_GPU_BACKEND_CUDA):
        self.L = load_library()
        self._ctx = _vp()
        rc = self.L.ufsecp_gpu_ctx_create(ctypes.byref(self._ctx), backend_id, device_index)
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "ufsecp_gpu_ctx_create", error_str(rc))

    @property
    def handle(self) -> int:
        return self._ctx.value

    def close(self) -> None:
        if self._ctx:
            self.L.ufsecp_gpu_ctx_destroy(self._ctx)
            self._ctx = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def is_ready(self) -> bool:
        return bool(self.L.ufsecp_gpu_is_ready(self._ctx))

    def last_error(self) -> int:
        return int(self.L.ufsecp_gpu_last_error(self._ctx))

    def last_error_msg(self) -> str:
        return self.L.ufsecp_gpu_last_error_msg(self._ctx).decode()

    def _check(self, rc: int, where: str) -> None:
        if rc != UFSECP_OK:
            raise UfsecpError(rc, where, self.last_error_msg())

    # ---- ufsecp_gpu.h verify calls (host buffers) ----------------------------
    def _verify(self, fn, name, msgs, pubs, pub_sz, sigs, count=None, out=None) -> np.ndarray:
        n = (len(msgs) if isinstance(msgs, (bytes, bytearray)) else np.asarray(msgs).size) // 32 \
            if count is None else count
        m = _buf(msgs, 32 * n, "msg_hashes32")
        p = _buf(pubs, pub_sz * n, "pubkeys")
        s = _buf(sigs, 64 * n, "sigs64")
        if out is None:
            out = np.zeros(n, dtype=np.uint8)
        rc = fn(self._ctx, _ptr(m), _ptr(p), _ptr(s), n, _ptr(out))
        self._check(rc, name)
        return out

    def ecdsa_verify_batch(self, msg_hashes32, pubkeys33, sigs64) -> np.ndarray:
        """ufsecp_gpu_ecdsa_verify_batch: per-item verdicts (1 valid / 0 invalid)."""
        return self._verify(self.L.ufsecp_gpu_ecdsa_verify_batch, "ufsecp_gpu_ecdsa_verify_batch",
                            msg_hashes32, pubkeys33, 33, sigs64)

    def schnorr_verify_batch(self, msg_hashes32, pubkeys_x32, sigs64) -> np.ndarray:
        """ufsecp_gpu_schnorr_verify_batch: per-item BIP-340 verdicts."""
        return self._verify(self.L.ufsecp_gpu_schnorr_verify_batch, "ufsecp_gpu_schnorr_verify_batch",
                            msg_hashes32, pubkeys_x32, 32, sigs64)

    def ecdsa_verify_collect(self, msg_hashes32, pubkeys33, sigs64, key_buffer: np.ndarray) -> np.ndarray:
        """ufsecp_gpu_ecdsa_verify_collect: valid rows of key_buffer become 0 in place."""
        kb = np.ascontiguousarray(key_buffer, dtype=np.uint8)
        return self._verify(self.L.ufsecp_gpu_ecdsa_verify_collect, "ufsecp_gpu_ecdsa_verify_collect",
                            msg_hashes32, pubkeys33, 33, sigs64, count=kb.size, out=kb)

    def schnorr_verify_collect(self, msg_hashes32, pubkeys_x32, sigs64, key_buffer: np.ndarray) -> np.ndarray:
        kb = np.ascontiguousarray(key_buffer, dtype=np.uint8)
        return self._verify(self.L.ufsecp_gpu_schnorr_verify_collect, "ufsecp_gpu_schnorr_verify_collect",
                            msg_hashes32, pubkeys_x32, 32, sigs64, count=kb.size, out=kb)

    # ---- ufsecp_gpu_ext.h -------------------------------------------------------
    def verify_jobs(self, jobs):
        """ufsecp_gpu_ext_verify_jobs: jobs = [(kind, msgs, pubs, sigs[, segment]), ...] with
        kind 0 ECDSA (33-byte keys) / 1 BIP-340 (32-byte keys) / 2 BIP-340 checked by RLC
        (32-byte keys; `segment` = RLC segment length, 0 = default); returns one verdict
        array per job."""
        tab, keep, out_all, offs = _job_table(jobs)
        self._check(self.L.ufsecp_gpu_ext_verify_jobs(self._ctx, tab.ctypes.data_as(ctypes.POINTER(Job)), len(jobs)),
                    "verify_jobs")
        return [out_all[o:o + n] for o, n in offs]

    def verify_job_ranges(self, corpora: dict, kinds, starts, counts) -> dict:
        """ufsecp_gpu_ext_verify_jobs over jobs given as index ranges of per-kind
        corpora: corpora = {kind: (msgs, pubs, sigs)} (contiguous uint8 arrays of
        32 / 33 or 32 / 64 bytes per item), job j = items starts[j] ..
        starts[j] + counts[j] - 1 of corpora[kinds[j]].  The job table is built
        with vector operations (no per-job Python work), so a call of thousands
        of jobs costs what the C ABI call costs.  Returns {kind: verdicts},
        aligned with the corpora (items no job covers stay 0)."""
        kinds = np.asarray(kinds, np.uint32)
        starts = np.asarray(starts, np.uint64)
        counts = np.asarray(counts, np.uint64)
        if not (kinds.shape == starts.shape == counts.shape):
            raise ValueError("kinds, starts and counts differ in length")
        tab = np.zeros(max(1, kinds.size), _JOB_DTYPE)[:kinds.size]
        tab["kind"] = kinds
        tab["count"] = counts
        outs, keep = {}, []
        for k, (m, p, sg) in corpora.items():
            m, p, sg = _flat_u8(m), _flat_u8(p), _flat_u8(sg)
            n = m.size // 32
            ps = 33 if k == 0 else 32
            if p.size != ps * n or sg.size != 64 * n:
                raise ValueError(f"corpus of kind {k}: inconsistent sizes")
            sel = kinds == k
            if (starts[sel] + counts[sel] > n).any():
                raise ValueError(f"a job of kind {k} reaches past its corpus")
            out = np.zeros(max(1, n), np.uint8)
            outs[k] = out[:n]
            keep.append((m, p, sg, out))
            if n and sel.any():
                st = starts[sel]
                tab["msg_hashes32"][sel] = _addr(m) + 32 * st
                tab["pubkeys"][sel] = _addr(p) + ps * st
                tab["sigs64"][sel] = _addr(sg) + 64 * st
                tab["out_results"][sel] = _addr(out) + st
        orphan = ~np.isin(kinds, np.array(list(corpora), np.uint32))
        if (counts[orphan] > 0).any():
            raise ValueError("a job names a kind with no corpus")
        self._check(self.L.ufsecp_gpu_ext_verify_jobs(self._ctx, tab.ctypes.data_as(ctypes.POINTER(Job)), kinds.size),
                    "verify_jobs")
        return outs

    def set_inversion_group(self, kind: int, group: int):
        """ufsecp_gpu_ext_set_inversion_group: 1, 64 or 128 threads share each inversion."""
        self._check(self.L.ufsecp_gpu_ext_set_inversion_group(self._ctx, kind, group), "set_inversion_group")

    def get_inversion_group(self, kind: int) -> int:
        g = ctypes.c_int()
        self._check(self.L.ufsecp_gpu_ext_get_inversion_group(self._ctx, kind, ctypes.byref(g)),
                    "get_inversion_group")
        return g.value

    def set_key_table(self, log2_slots: int):
        """ufsecp_gpu_ext_set_key_table: 0 = no resident key table for verify_jobs,
        8..24 = a new, empty table of 2^log2_slots slots."""
        self._check(self.L.ufsecp_gpu_ext_set_key_table(self._ctx, log2_slots), "set_key_table")

    def key_table_stats(self) -> dict:
        v = (ctypes.c_uint64 * 3)()
        self._check(self.L.ufsecp_gpu_ext_key_table_stats(self._ctx, v), "key_table_stats")
        return {"lookups": v[0], "hits": v[1], "slots": v[2]}

    def schnorr_verify_rlc(self, msg_hashes32, pubkeys_x32, sigs64, batch_size: int = 0, seed32=None,
                           window_bits: int = 0):
        """ufsecp_gpu_ext_schnorr_verify_rlc: RLC batch verify with bisection.
        Returns (per-item verdicts, per-batch all-valid flags)."""
        n = np.asarray(msg_hashes32, np.uint8).size // 32 if not isinstance(msg_hashes32, (bytes, bytearray)) \
            else len(msg_hashes32) // 32
        m = _buf(msg_hashes32, 32 * n, "msg_hashes32")
        p = _buf(pubkeys_x32, 32 * n, "pubkeys_x32")
        s = _buf(sigs64, 64 * n, "sigs64")
        seed = _buf(seed32 if seed32 is not None else os.urandom(32), 32, "seed32")
        out = np.zeros(n, np.uint8)
        nb = 1 if batch_size == 0 or batch_size >= n else -(-n // batch_size)
        bok = np.zeros(max(nb, 1), np.uint8)
        rc = self.L.ufsecp_gpu_ext_schnorr_verify_rlc(self._ctx, _ptr(m), _ptr(p), _ptr(s), n, batch_size,
                                                      _ptr(seed), window_bits, _ptr(out), _ptr(bok))
        self._check(rc, "schnorr_verify_rlc")
        return out, bok[:nb]

    def schnorr_verify_rlc_device(self, d_msgs: int, d_xonly: int, d_sigs: int, count: int, d_out: int,
                                  batch_size: int = 0, seed32=None, window_bits: int = 0, stream: int = 0):
        """Device-buffer RLC verify; returns the per-batch all-valid flags."""
        seed = _buf(seed32 if seed32 is not None else os.urandom(32), 32, "seed32")
        nb = 1 if batch_size == 0 or batch_size >= count else -(-count // batch_size)
        bok = np.zeros(max(nb, 1), np.uint8)
        rc = self.L.ufsecp_gpu_ext_schnorr_verify_rlc_device(self._ctx, d_msgs, d_xonly, d_sigs, count, batch_size,
                                                             _ptr(seed), window_bits, d_out, _ptr(bok),
                                                             stream or None)
        self._check(rc, "schnorr_verify_rlc_device")
        return bok[:nb]

    def rlc_stats(self) -> dict:
        v = (ctypes.c_uint64 * 4)()
        self._check(self.L.ufsecp_gpu_ext_rlc_stats(self._ctx, v), "rlc_stats")
        loc = ctypes.c_uint64()
        self._check(self.L.ufsecp_gpu_ext_rlc_located(self._ctx, ctypes.byref(loc)), "rlc_located")
        kh = ctypes.c_uint64()
        self._check(self.L.ufsecp_gpu_ext_rlc_key_hits(self._ctx, ctypes.byref(kh)), "rlc_key_hits")
        return {"rounds": v[0], "segments": v[1], "leaf_items": v[2], "window_bits": v[3], "located": loc.value,
                "key_hits": kh.value}

    def set_rlc_locate(self, on: bool):
        """ufsecp_gpu_ext_set_rlc_locate: the locate step of RLC verification on / off."""
        self._check(self.L.ufsecp_gpu_ext_set_rlc_locate(self._ctx, 1 if on else 0), "set_rlc_locate")

    def rlc_input_digest(self, msg_hashes32, pubkeys_x32, sigs64) -> bytes:
        """ufsecp_gpu_ext_rlc_input_digest: the SHA-256 tree digest that binds the
        reference-shaped batch API's RLC seed to its inputs."""
        n = len(np.asarray(msg_hashes32, np.uint8).reshape(-1)) // 32
        m = _buf(msg_hashes32, 32 * n, "msg_hashes32")
        p = _buf(pubkeys_x32, 32 * n, "pubkeys_x32")
        s = _buf(sigs64, 64 * n, "sigs64")
        out = np.zeros(32, np.uint8)
        rc = self.L.ufsecp_gpu_ext_rlc_input_digest(self._ctx, _ptr(m) if n else None, _ptr(p) if n else None,
                                                    _ptr(s) if n else None, n, _ptr(out))
        self._check(rc, "rlc_input_digest")
        return out.tobytes()

    def schnorr_batch_verify(self, entries) -> int:
        """ufsecp_gpu_ext_schnorr_batch_verify on rows [x 32 | msg 32 | sig 64]; returns the
        reference's code (0 all valid, 6 VERIFY_FAIL, 3 BAD_PUBKEY, 4 BAD_SIG, ...)."""
        e = np.ascontiguousarray(np.asarray(entries, np.uint8)).reshape(-1)
        return self.L.ufsecp_gpu_ext_schnorr_batch_verify(self._ctx, _ptr(e) if e.size else None, e.size // 128)

    def schnorr_batch_identify_invalid(self, entries, capacity: int = None):
        """Returns (code, invalid indices, total invalid)."""
        e = np.ascontiguousarray(np.asarray(entries, np.uint8)).reshape(-1)
        n = e.size // 128
        cap = n if capacity is None else capacity
        buf = (ctypes.c_size_t * max(cap, 1))()
        cnt = ctypes.c_size_t(cap)
        rc = self.L.ufsecp_gpu_ext_schnorr_batch_identify_invalid(self._ctx, _ptr(e) if e.size else None, n, buf,
                                                                  ctypes.byref(cnt))
        got = min(cnt.value, cap)
        return rc, [buf[i] for i in range(got)], cnt.value

    def ecdsa_verify_device(self, d_msgs: int, d_pubs33: int, d_sigs: int, count: int, d_out: int,
                            stream: int = 0) -> None:
        """Device pointers in / out, enqueued on `stream` (0 = context stream)."""
        self._check(self.L.ufsecp_gpu_ext_ecdsa_verify_device(self._ctx, d_msgs, d_pubs33, d_sigs, count, d_out,
                                                              stream or None), "ecdsa_verify_device")

    def schnorr_verify_device(self, d_msgs: int, d_xonly: int, d_sigs: int, count: int, d_out: int,
                              stream: int = 0) -> None:
        self._check(self.L.ufsecp_gpu_ext_schnorr_verify_device(self._ctx, d_msgs, d_xonly, d_sigs, count, d_out,
                                                                stream or None), "schnorr_verify_device")

    def sign_device(self, kind: int, d_msgs: int, d_sks: int, d_auxs: int, count: int, d_pubs: int, d_sigs: int,
                    d_ok: int, stream: int = 0) -> None:
        """Batch signer for synthetic corpora (device pointers; kind 0 ECDSA, 1 BIP-340)."""
        self._check(self.L.ufsecp_gpu_ext_sign_device(self._ctx, kind, d_msgs, d_sks, d_auxs or None, count, d_pubs,
                                                      d_sigs, d_ok, stream or None), "sign_device")

    def stream(self) -> int:
        s = _vp()
        self._check(self.L.ufsecp_gpu_ext_stream(self._ctx, ctypes.byref(s)), "ext_stream")
        return s.value or 0

    def device_props(self):
        sms, be, bs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.L.ufsecp_gpu_ext_device_props(self._ctx, ctypes.byref(sms), ctypes.byref(be),
                                                       ctypes.byref(bs)), "device_props")
        return {"sm_count": sms.value, "ecdsa_blocks_per_sm": be.value, "schnorr_blocks_per_sm": bs.value}

    def set_variant(self, kind: int, variant: int) -> None:
        self._check(self.L.ufsecp_gpu_ext_set_variant(self._ctx, kind, variant), "set_variant")

    def get_variant(self, kind: int):
        v, b = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.ufsecp_gpu_ext_get_variant(self._ctx, kind, ctypes.byref(v), ctypes.byref(b)),
                    "get_variant")
        return v.value, b.value

    def get_small_variant(self, kind: int):
        """(variant, items): launches of at most `items` items use `variant`; (-1, 0) when none."""
        v, n = ctypes.c_int(), ctypes.c_uint32()
        self._check(self.L.ufsecp_gpu_ext_get_small_variant(self._ctx, kind, ctypes.byref(v), ctypes.byref(n)),
                    "get_small_variant")
        return v.value, n.value

    def set_lanes(self, kind: int, lanes: int, items: int = 0) -> None:
        """lanes 2: calls of at most `items` items run two threads per signature; 1: off."""
        self._check(self.L.ufsecp_gpu_ext_set_lanes(self._ctx, kind, lanes, items), "set_lanes")

    def get_lanes(self, kind: int):
        """(lanes, items) for signature kind 0 ECDSA / 1 BIP-340."""
        l, n = ctypes.c_int(), ctypes.c_uint32()
        self._check(self.L.ufsecp_gpu_ext_get_lanes(self._ctx, kind, ctypes.byref(l), ctypes.byref(n)), "get_lanes")
        return l.value, n.value

    def set_rlc_chunk(self, chunk: int) -> None:
        """Bucket points per RLC chunk thread for every segment (2..256); 0 restores the tuned values."""
        self._check(self.L.ufsecp_gpu_ext_set_rlc_chunk(self._ctx, chunk), "set_rlc_chunk")

    def get_rlc_chunk(self, length: int) -> int:
        """Bucket points per RLC chunk thread for a segment of `length` items."""
        v = ctypes.c_uint32()
        self._check(self.L.ufsecp_gpu_ext_get_rlc_chunk(self._ctx, length, ctypes.byref(v)), "get_rlc_chunk")
        return v.value

    def set_small_variant(self, kind: int, variant: int, items: int = 0) -> None:
        """Launches of at most `items` items use `variant` (-1: none)."""
        self._check(self.L.ufsecp_gpu_ext_set_small_variant(self._ctx, kind, variant, items), "set_small_variant")

    def imad_peak(self) -> float:
        v = ctypes.c_double()
        self._check(self.L.ufsecp_gpu_ext_imad_peak(self._ctx, ctypes.byref(v)), "imad_peak")
        return v.value

    def probe(self, op: int, blocks: int, threads: int, iters: int) -> float:
        """Building-block throughput probe; returns the launch time in ms."""
        ms = ctypes.c_float()
        self._check(self.L.ufsecp_gpu_ext_probe(self._ctx, op, blocks, threads, iters, ctypes.byref(ms)), "probe")
        return ms.value

    _DIAG_IO = {1: (64, 32), 2: (32, 32), 3: (32, 32), 4: (32, 33), 5: (64, 32), 6: (32, 32), 7: (32, 34),
                8: (32, 64), 9: (96, 65), 10: (96, 32), 11: (64, 192)}

    def diag(self, op: int, data) -> np.ndarray:
        isz, osz = self._DIAG_IO[op]
        a = np.ascontiguousarray(np.frombuffer(bytes(data), np.uint8) if isinstance(data, (bytes, bytearray))
                                 else np.asarray(data, np.uint8)).reshape(-1)
        n = a.size // isz
        out = np.zeros(n * osz, np.uint8)
        self._check(self.L.ufsecp_gpu_ext_diag(self._ctx, op, _ptr(a), n, _ptr(out)), "ext_diag")
        return out.reshape(n, osz)


class Server:
    """Serving loop over one context (ufsecp_gpu_ext_server_*): submit requests
    of ECDSA / BIP-340 jobs from any thread, wait for their verdicts."""

    def __init__(self, ctx: GpuContext, slots: int = 8, max_launch_items: int = 1 << 16,
                 memory_budget_bytes: int = 8 << 30, batch_window_us: int = 0, key_cache_log2: int = 18):
        """key_cache_log2: 0 or 1 = no resident key table, 8..24 = a table of 2^k slots (default 18)."""
        self.L = ctx.L
        self._ctx = ctx
        cfg = ServerConfig(slots, max_launch_items, memory_budget_bytes, batch_window_us, key_cache_log2)
        h = _vp()
        rc = self.L.ufsecp_gpu_ext_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h))
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "server_create", ctx.last_error_msg())
        self._h = h
        self._keep = {}

    def submit(self, jobs) -> int:
        """jobs = [(kind, msgs, pubs, sigs), ...]; returns the request id.  The verdict
        arrays are returned by wait()."""
        tab, keep, out_all, offs = _job_table(jobs)
        rid = ctypes.c_uint64()
        rc = self.L.ufsecp_gpu_ext_server_submit(self._h, tab.ctypes.data_as(ctypes.POINTER(Job)), len(jobs),
                                                 ctypes.byref(rid))
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "server_submit")
        self._keep[rid.value] = (keep, [out_all[o:o + n] for o, n in offs], tab)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = 60_000):
        """Verdict arrays of request `rid`, one per job.  A failed or cancelled
        request raises UfsecpError with its code (its verdicts were cleared); a
        timeout raises with UFSECP_ERR_GPU_QUEUE and keeps the request."""
        rc = self.L.ufsecp_gpu_ext_server_wait(self._h, rid, timeout_ms)
        if rc == UFSECP_ERR_GPU_QUEUE:
            raise UfsecpError(rc, "server_wait")
        keep = self._keep.pop(rid)
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "server_wait")
        return keep[1]

    def submit_cancellable(self, jobs, is_cancelled, check_interval: int = 0) -> int:
        """submit() with a cancellation token: is_cancelled() -> bool is polled by
        the server before each launch that would take a piece of the request."""
        tab, keep, out_all, offs = _job_table(jobs)
        fn = CANCEL_FN(lambda user: 1 if is_cancelled() else 0)
        tok = CancelToken(fn, None, check_interval)
        rid = ctypes.c_uint64()
        rc = self.L.ufsecp_gpu_ext_server_submit_cancellable(self._h, tab.ctypes.data_as(ctypes.POINTER(Job)),
                                                             len(jobs), ctypes.byref(tok), ctypes.byref(rid))
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "server_submit_cancellable")
        self._keep[rid.value] = (keep, [out_all[o:o + n] for o, n in offs], tab, fn, tok)
        return rid.value

    def cancel(self, rid: int, timeout_ms: int = 60_000) -> int:
        """ufsecp_gpu_ext_server_cancel; returns its code.  On UFSECP_OK the server
        no longer touches the request's buffers."""
        rc = self.L.ufsecp_gpu_ext_server_cancel(self._h, rid, timeout_ms)
        if rc == UFSECP_OK:
            self._keep.pop(rid, None)
        return rc

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        rc = self.L.ufsecp_gpu_ext_server_stats(self._h, ctypes.byref(st), 1 if reset else 0)
        if rc != UFSECP_OK:
            raise UfsecpError(rc, "server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_ if f != "reserved"}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.L.ufsecp_gpu_ext_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
