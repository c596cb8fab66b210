"""The engine hook provider ufsecp_gpu_ext_engine_columns_hook, installed into
the reference engine itself (oracle/_ref, the reference CPU library compiled
from its sources) with secp256k1::install_gpu_columns_verify_hook, exactly as
the reference's own GPU host layer does (src/gpu/src/gpu_engine_hook.cpp:81-104).

The reference's column entry points secp256k1::ecdsa_batch_verify_opaque_columns
and secp256k1::schnorr_batch_verify_bip340_columns then consult the hook.  On a
machine without a CUDA device the hook must decline (-1) and the engine's CPU
path must produce the verdicts; with a device the GPU must handle the calls.
Either way the verdicts equal the oracle's.
"""
import ctypes

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import opaque_rows_corpus, schnorr_corpus

INSTALL = "_ZN9secp256k131install_gpu_columns_verify_hookEPDoFiiPKhS1_S1_mPhE"
ECDSA_COLS = "_ZN9secp256k133ecdsa_batch_verify_opaque_columnsEPKhS1_S1_mPhm"
SCHNORR_COLS = "_ZN9secp256k135schnorr_batch_verify_bip340_columnsEPKhS1_S1_mPhm"


def _engine(reflib):
    L = reflib.L
    for name in (INSTALL, ECDSA_COLS, SCHNORR_COLS):
        if not hasattr(L, name):
            pytest.skip(f"reference engine symbol {name} not exported")
    getattr(L, INSTALL).argtypes = [ctypes.c_void_p]
    getattr(L, INSTALL).restype = ctypes.c_void_p
    for name in (ECDSA_COLS, SCHNORR_COLS):
        getattr(L, name).argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        getattr(L, name).restype = ctypes.c_bool
    return L


def _counters(L):
    L.ufsecp_gpu_ext_engine_hook_counters.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 2
    h, d = ctypes.c_uint64(), ctypes.c_uint64()
    L.ufsecp_gpu_ext_engine_hook_counters(ctypes.byref(h), ctypes.byref(d))
    return h.value, d.value


def _run(oracle, reflib):
    E = _engine(reflib)
    U = uf.load_library()
    hook = ctypes.cast(U.ufsecp_gpu_ext_engine_columns_hook, ctypes.c_void_p).value
    prev = getattr(E, INSTALL)(hook)
    try:
        before = _counters(U)
        rows = opaque_rows_corpus(oracle, 700, seed=17)
        d, p, s = (np.ascontiguousarray(rows[:, a:b]) for a, b in ((0, 32), (32, 65), (65, 129)))
        out = np.full(len(rows), 9, np.uint8)
        all_ok = getattr(E, ECDSA_COLS)(d.ctypes.data, p.ctypes.data, s.ctypes.data, len(rows), out.ctypes.data, 1)
        want = oracle.ecdsa_verify_opaque_rows(rows, 129)
        assert (out == want).all() and all_ok == bool(want.all())
        m, x, sg = schnorr_corpus(oracle, 600, seed=18, tamper=0.02)
        out2 = np.full(len(m), 9, np.uint8)
        all_ok2 = getattr(E, SCHNORR_COLS)(m.ctypes.data, x.ctypes.data, sg.ctypes.data, len(m), out2.ctypes.data, 1)
        want2 = oracle.schnorr_verify_batch(m, x, sg)
        assert (out2 == want2).all() and all_ok2 == bool(want2.all())
        after = _counters(U)
    finally:
        getattr(E, INSTALL)(prev)
    return before, after


def test_hook_declines_without_a_device(oracle, reflib):
    if uf.device_count() > 0:
        pytest.skip("a CUDA device is present (covered by the gpu test)")
    before, after = _run(oracle, reflib)
    assert after[0] == before[0] and after[1] >= before[1] + 2      # both calls declined -> CPU path


@pytest.mark.gpu
def test_hook_handles_engine_calls_on_the_gpu(oracle, reflib):
    before, after = _run(oracle, reflib)
    assert after[0] == before[0] + 2 and after[1] == before[1]      # both calls ran on the GPU
    uf.load_library().ufsecp_gpu_ext_engine_hook_release()


@pytest.mark.gpu
def test_hook_declines_on_a_backend_error(oracle, reflib):
    """A backend failure inside the hook (injected on the host: the hook's
    context fails its next launch) makes the hook decline that call; the
    engine's CPU path answers it with the right verdicts, and the next call is
    handled on the GPU again."""
    U = uf.load_library()
    U.ufsecp_gpu_ext_engine_hook_release()
    assert U.ufsecp_gpu_ext_engine_hook_inject_fault(0, 2) == uf.UFSECP_OK    # first launch of the hook fails
    before, after = _run(oracle, reflib)
    assert after[1] == before[1] + 1 and after[0] == before[0] + 1     # one declined (CPU answered), one handled
    U.ufsecp_gpu_ext_engine_hook_release()
