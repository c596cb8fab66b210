"""One host-buffer batch over several contexts (ufsecp_gpu_ext_verify_batch_sharded):
contiguous shares, one host thread per context, verdicts item for item equal
to the oracle and to the single-context call.  The box runs one GPU, so the
contexts here share it; with one context per GPU the shares run on all of them."""
import ctypes

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import ecdsa_corpus, schnorr_corpus

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctxs():
    cs = [uf.GpuContext(0) for _ in range(3)]
    yield cs
    for c in cs:
        c.close()


@pytest.mark.parametrize("n_ctx", [1, 2, 3])
def test_sharded_equals_oracle(oracle, ctxs, n_ctx):
    me, pe, se = ecdsa_corpus(oracle, 5001, seed=141, tamper=0.05)
    ms, xs, ss = schnorr_corpus(oracle, 4999, seed=142, tamper=0.05)
    got_e = uf.verify_batch_sharded(ctxs[:n_ctx], 0, me, pe, se)
    got_s = uf.verify_batch_sharded(ctxs[:n_ctx], 1, ms, xs, ss)
    assert (got_e == oracle.ecdsa_verify_batch(me, pe, se)).all()
    assert (got_s == oracle.schnorr_verify_batch(ms, xs, ss)).all()
    assert (got_s == ctxs[0].schnorr_verify_batch(ms, xs, ss)).all()


def test_sharded_fewer_items_than_contexts(oracle, ctxs):
    ms, xs, ss = schnorr_corpus(oracle, 2, seed=143, tamper=0.0)
    assert (uf.verify_batch_sharded(ctxs, 1, ms, xs, ss) == 1).all()


def test_sharded_gating_and_fail_closed(oracle, ctxs):
    L = uf.load_library()
    ms, xs, ss = schnorr_corpus(oracle, 3000, seed=144, tamper=0.0)
    out = np.full(3000, 7, np.uint8)
    dup = (uf._vp * 2)(ctxs[0].handle, ctxs[0].handle)
    assert L.ufsecp_gpu_ext_verify_batch_sharded(dup, 2, 1, ms.ctypes.data, xs.ctypes.data, ss.ctypes.data, 3000,
                                                 out.ctypes.data) == uf.UFSECP_ERR_BAD_INPUT
    arr = (uf._vp * 3)(*[c.handle for c in ctxs])
    # the second share's launch fails: its code comes back and no verdict reads valid
    assert L.ufsecp_gpu_ext_inject_fault(ctxs[1].handle, 0, 2) == uf.UFSECP_OK
    out[:] = 7
    rc = L.ufsecp_gpu_ext_verify_batch_sharded(arr, 3, 1, ms.ctypes.data, xs.ctypes.data, ss.ctypes.data, 3000,
                                               out.ctypes.data)
    assert rc == uf.UFSECP_ERR_GPU_LAUNCH and not out.any()
    assert (uf.verify_batch_sharded(ctxs, 1, ms, xs, ss) == 1).all()      # all contexts keep working
