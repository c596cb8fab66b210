"""C-ABI library checks that need no GPU: it loads, exports every symbol that
include/ufsecp/*.h declares, and gates arguments like the reference ABI layer
(src/cpu/src/ufsecp_gpu_impl.cpp) without touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import ultrafastsecp256k1_b200 as uf
from conftest import ROOT


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(uf.LIB_PATH):
        from ultrafastsecp256k1_b200 import build
        build.build()
    return uf.load_library()


def declared_symbols():
    names = set()
    for h in ("ufsecp_gpu.h", "ufsecp_gpu_ext.h"):
        src = open(os.path.join(ROOT, "include", "ufsecp", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"UFSECP_API\s+[^;(]*?\b(ufsecp_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 48
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_reference_surface_is_complete():
    """Every function of the reference GPU header is declared here too."""
    expected = {
        "ufsecp_gpu_backend_count", "ufsecp_gpu_backend_name", "ufsecp_gpu_is_available", "ufsecp_gpu_device_count",
        "ufsecp_gpu_device_info", "ufsecp_gpu_ctx_create", "ufsecp_gpu_ctx_destroy", "ufsecp_gpu_is_ready",
        "ufsecp_gpu_last_error", "ufsecp_gpu_last_error_msg", "ufsecp_gpu_generator_mul_batch",
        "ufsecp_gpu_ecdsa_verify_batch", "ufsecp_gpu_ecdsa_verify_opaque_rows", "ufsecp_gpu_ecdsa_verify_lbtc_rows",
        "ufsecp_gpu_schnorr_verify_batch", "ufsecp_gpu_ecdsa_verify_lbtc_columns",
        "ufsecp_gpu_schnorr_verify_lbtc_columns", "ufsecp_gpu_ecdsa_verify_collect",
        "ufsecp_gpu_schnorr_verify_collect", "ufsecp_gpu_ecdh_batch", "ufsecp_gpu_hash160_pubkey_batch",
        "ufsecp_gpu_msm", "ufsecp_gpu_xonly_validate", "ufsecp_gpu_commitment_verify", "ufsecp_gpu_tagged_hash",
        "ufsecp_gpu_pubkey_validate", "ufsecp_gpu_tagged_hash_var", "ufsecp_gpu_hash256", "ufsecp_gpu_hash256_var",
        "ufsecp_gpu_frost_verify_partial_batch", "ufsecp_gpu_ecrecover_batch", "ufsecp_gpu_error_str",
        "ufsecp_gpu_zk_knowledge_verify_batch", "ufsecp_gpu_zk_dleq_verify_batch",
        "ufsecp_gpu_bulletproof_verify_batch", "ufsecp_gpu_bip324_aead_encrypt_batch",
        "ufsecp_gpu_bip324_aead_decrypt_batch", "ufsecp_gpu_zk_ecdsa_snark_witness_batch",
        "ufsecp_gpu_zk_schnorr_snark_witness_batch", "ufsecp_bip352_prepare_scan_plan",
        "ufsecp_gpu_bip352_scan_batch",
    }
    assert expected <= declared_symbols()


def test_only_ufsecp_symbols_exported(lib):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", uf.LIB_PATH], capture_output=True, text=True).stdout
    exported = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert exported and all(n.startswith("ufsecp_") for n in exported)


def test_discovery_and_gating_without_device(lib):
    assert lib.ufsecp_gpu_backend_count(None, 0) == 1
    ids = (ctypes.c_uint32 * 4)()
    assert lib.ufsecp_gpu_backend_count(ids, 4) == 1 and ids[0] == uf.UFSECP_GPU_BACKEND_CUDA
    assert lib.ufsecp_gpu_backend_name(1) == b"CUDA"
    assert lib.ufsecp_gpu_backend_name(7) == b"none"
    assert lib.ufsecp_gpu_is_available(2) == 0
    assert lib.ufsecp_gpu_device_count(3) == 0
    assert lib.ufsecp_gpu_is_ready(None) == 0
    assert lib.ufsecp_gpu_last_error(None) == uf.UFSECP_ERR_NULL_ARG
    assert lib.ufsecp_gpu_last_error_msg(None) == b"NULL GPU context"
    assert lib.ufsecp_gpu_ctx_create(None, 1, 0) == uf.UFSECP_ERR_NULL_ARG
    c = ctypes.c_void_p()
    assert lib.ufsecp_gpu_ctx_create(ctypes.byref(c), 2, 0) == uf.UFSECP_ERR_GPU_UNAVAILABLE
    assert not c.value
    # NULL ctx is checked first for every verify entry point
    for name in ("ufsecp_gpu_ecdsa_verify_batch", "ufsecp_gpu_schnorr_verify_batch",
                 "ufsecp_gpu_ecdsa_verify_collect", "ufsecp_gpu_schnorr_verify_collect"):
        assert getattr(lib, name)(None, None, None, None, 4, None) == uf.UFSECP_ERR_NULL_ARG
    assert lib.ufsecp_gpu_ext_diag(None, 1, None, 1, None) == uf.UFSECP_ERR_NULL_ARG
    for code in (0, 1, 5, 9, 100, 104, 106):
        assert lib.ufsecp_gpu_error_str(code)
    assert lib.ufsecp_gpu_error_str(12345) == b"unknown error"


def test_device_info_without_device(lib):
    if uf.device_count() > 0:
        pytest.skip("a device is present")
    info = uf.DeviceInfo()
    assert lib.ufsecp_gpu_device_info(1, 0, ctypes.byref(info)) == uf.UFSECP_ERR_GPU_UNAVAILABLE
    assert lib.ufsecp_gpu_device_info(1, 0, None) == uf.UFSECP_ERR_NULL_ARG
    with pytest.raises(uf.UfsecpError):
        uf.GpuContext(0)


def _reference_tree():
    import sys
    sys.path.insert(0, ROOT)
    from __graft_entry__ import reference_tree
    return reference_tree()


EXAMPLE_BIN = os.path.join(ROOT, "oracle", "_ref", "gpu_example")


def test_reference_c_example_compiles_links_and_runs(tmp_path):
    """The reference's own C example of the GPU API (include/ufsecp/examples/
    gpu_example.c), compiled UNCHANGED against this include/ and linked to
    libufsecp_gpu.so by a C compiler: it must build without warnings of
    missing declarations and run to completion.  Without a device it takes its
    no-device path."""
    import subprocess
    ref = _reference_tree()
    if ref is None:
        pytest.skip("reference source tree not present (the prebuilt binary is run by the gpu test)")
    src = os.path.join(ref, "include", "ufsecp", "examples", "gpu_example.c")
    exe = tmp_path / "gpu_example"
    libdir = os.path.dirname(uf.LIB_PATH)
    cc = subprocess.run(["gcc", "-O2", "-Wall", "-Werror=implicit-function-declaration", "-I",
                         os.path.join(ROOT, "include"), "-o", str(exe), src, "-L", libdir, "-lufsecp_gpu",
                         f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "Compiled GPU backends: 1" in run.stdout
    if uf.device_count() == 0:
        assert "No available GPU device found." in run.stdout


@pytest.mark.gpu
def test_reference_c_example_on_the_gpu():
    """The same example, prebuilt from the reference's source by `make -C oracle
    example`, on a B200: it creates a context, meets UNSUPPORTED for the
    generator multiplication (outside the verify path) and verifies a batch
    through ufsecp_gpu_ecdsa_verify_batch."""
    import subprocess
    if not os.path.exists(EXAMPLE_BIN):
        pytest.skip("oracle/_ref/gpu_example not built (make -C oracle example REF=<reference tree>)")
    run = subprocess.run([EXAMPLE_BIN], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "Using: NVIDIA" in run.stdout
    assert "generator_mul_batch not supported on this backend." in run.stdout
    assert "ecdsa_verify_batch returned: OK" in run.stdout
    assert "Done." in run.stdout


def test_sharded_gating_without_contexts():
    """ufsecp_gpu_ext_verify_batch_sharded's argument checks that need no context."""
    L = uf.load_library()
    buf = np.zeros(64 * 4, np.uint8)
    out = np.full(4, 7, np.uint8)
    nulls = (uf._vp * 2)(None, None)
    a = (buf.ctypes.data, buf.ctypes.data, buf.ctypes.data, 4, out.ctypes.data)
    assert L.ufsecp_gpu_ext_verify_batch_sharded(None, 1, 1, *a) == uf.UFSECP_ERR_NULL_ARG
    assert L.ufsecp_gpu_ext_verify_batch_sharded(nulls, 2, 1, buf.ctypes.data, buf.ctypes.data, buf.ctypes.data, 0,
                                                 out.ctypes.data) == uf.UFSECP_OK
    assert L.ufsecp_gpu_ext_verify_batch_sharded(nulls, 0, 1, *a) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_verify_batch_sharded(nulls, 2, 2, *a) == uf.UFSECP_ERR_BAD_INPUT
    assert L.ufsecp_gpu_ext_verify_batch_sharded(nulls, 2, 1, *a) == uf.UFSECP_ERR_NULL_ARG
    assert (out == 7).all()                      # nothing checked later than the contexts was touched
