"""The host thread pool that splits a chunk's staging copy
(ultrafastsecp256k1_b200/csrc/pack_pool.cpp), built for the host by the test
harness in tests/native (CPU only): every part runs exactly once per run, and
its writes are visible when run() returns, for pools of 1..8 threads and part
counts below, equal to and above the thread count."""
import ctypes
import os
import subprocess

import pytest

from conftest import NATIVE, ROOT, _newer


@pytest.fixture(scope="module")
def pool_lib():
    so = os.path.join(NATIVE, "libpack_pool_host.so")
    src = os.path.join(NATIVE, "pack_pool_host.cpp")
    csrc = os.path.join(ROOT, "ultrafastsecp256k1_b200", "csrc")
    if not _newer(so, src, os.path.join(csrc, "pack_pool.cpp"), os.path.join(csrc, "pack_pool.h")):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", so, src], check=True)
    return ctypes.CDLL(so)


@pytest.mark.parametrize("threads", [1, 2, 4, 8])
@pytest.mark.parametrize("parts", [1, 3, 4, 16])
def test_every_part_once(pool_lib, threads, parts):
    assert pool_lib.pp_check(threads, parts, 200) == 0
