"""Build libufsecp_gpu.so (sm_100a) in-tree.

    python -m ultrafastsecp256k1_b200.build [-j N] [--force]

Every .cu / .cpp under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into _build/ and
linked (static cudart) into ultrafastsecp256k1_b200/lib/libufsecp_gpu.so.
Objects are rebuilt when their source or any csrc/ header is newer.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libufsecp_gpu.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


# kernels_verify.cu (and its building-block probe) is compiled once per
# code-size variant (see csrc/common.cuh)
_VARIANT_FLAGS = [
    ("v0", ["-DUF_VARIANT=0"]),
        ("v1", ["-DUF_VARIANT=1", "-DUF_NOINLINE_POINT"]),
        ("v2", ["-DUF_VARIANT=2", "-DUF_NOINLINE_POINT", "-DUF_NOINLINE_FIELD"]),
        ("v3", ["-DUF_VARIANT=3", "-DUF_NOINLINE_FIELD"]),
        ("v4", ["-DUF_VARIANT=4", "-DUF_NOINLINE_POINT", "-DUF_NOINLINE_FIELD", "-DUF_PTX_MUL"]),
        ("v5", ["-DUF_VARIANT=5", "-DUF_NOINLINE_FIELD", "-DUF_PTX_MUL"]),
        ("v6", ["-DUF_VARIANT=6", "-DUF_NOINLINE_POINT", "-DUF_PTX_MUL"]),
        ("v7", ["-DUF_VARIANT=7", "-DUF_NOINLINE_POINT", "-DUF_NOINLINE_FIELD", "-DUF_PTX_MUL",
                "-DUF_PLAIN_THREADS=64", "-DUF_MIN_BLOCKS=7"]),
        ("v8", ["-DUF_VARIANT=8", "-DUF_NOINLINE_POINT", "-DUF_NOINLINE_FIELD", "-DUF_PTX_MUL", "-DUF_TAB7",
                "-DUF_PLAIN_THREADS=128", "-DUF_MIN_BLOCKS=4"]),
]
# the batched / served kernels are built once, with the code generation that
# measured fastest for the per-signature kernel on B200 (variant 4)
_BEST_FLAGS = ["-DUF_NOINLINE_POINT", "-DUF_NOINLINE_FIELD", "-DUF_PTX_MUL"]
# window-width variants of the per-signature kernel (variant 4's code
# generation): 3-bit P / 18-bit G windows, 5-bit P windows, 16-bit G windows
_WINDOW_FLAGS = [
    ("v9", ["-DUF_VARIANT=9", "-DUF_PWIN=3", "-DUF_GWIN=18"] + _BEST_FLAGS),
    ("v10", ["-DUF_VARIANT=10", "-DUF_PWIN=5"] + _BEST_FLAGS),
    ("v11", ["-DUF_VARIANT=11", "-DUF_GWIN=16"] + _BEST_FLAGS),
]
VARIANTS = {"kernels_verify.cu": _VARIANT_FLAGS + _WINDOW_FLAGS, "kernels_probe.cu": _VARIANT_FLAGS,
            "kernels_queue.cu": [("", _BEST_FLAGS)], "kernels_noalloc.cu": [("", _BEST_FLAGS)],
            "kernels_verify_grp.cu": [("", _BEST_FLAGS)],
            # small calls are latency-bound: the two-lane kernel takes variant 6's
            # code generation (field ops inlined into out-of-line point ops)
            "kernels_pair.cu": [("", ["-DUF_NOINLINE_POINT", "-DUF_PTX_MUL"])],
            "rlc.cu": [("", _BEST_FLAGS)], "kernels_ops.cu": [("", _BEST_FLAGS)],
            # the RLC kernels with one serial chain per segment or window run few
            # threads: field and point operations inlined, for overlap inside a chain
            "rlc_serial.cu": [("", ["-DUF_PTX_MUL"])]}


def _sources():
    """(source, object suffix, extra flags) for every compile job."""
    jobs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        for suffix, flags in VARIANTS.get(os.path.basename(src), [("", [])]):
            jobs.append((src, suffix, flags))
    return jobs


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "ufsecp", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(job, force: bool, verbose: bool) -> str:
    src, suffix, flags = job
    obj = os.path.join(BUILD, os.path.basename(src) + (("." + suffix) if suffix else "") + ".o")
    if not force and os.path.exists(obj):
        newest = max(os.path.getmtime(src), _headers_mtime())
        if os.path.getmtime(obj) >= newest:
            return obj
    cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    if src.endswith(".cu") and verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(jobs: int = 0, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-cudart", "static", "-o", LIB] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, a.v))


if __name__ == "__main__":
    main()
