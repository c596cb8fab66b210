"""Autotuner for the verify kernels.

    python -m ultrafastsecp256k1_b200.autotune [--batch N] [--out PATH]

For each signature kind (ECDSA, BIP-340) it times every verify-kernel variant
(ufsecp_gpu_ext_set_variant; variants 0..8 differ in how much field / point
arithmetic is inlined, i.e. instruction-cache footprint against call
overhead, 9..11 in the P / G window widths: 3 / 18, 5 / 20, 4 / 16 bits
against the default 4 / 20) on a GPU-signed batch, checks that all variants return identical
verdicts, and picks them, plus the inversion group (threads of a block that
share each modular inversion: 1, 64 or 128), a small-launch variant and its
item limit for latency-bound launches (a few warps per SM) and the call size
up to which two lanes per signature beat one; then, for RLC batch verification, it times the
Pippenger window width (the MSM bucket width, 2^(c-1) buckets per window)
for each batch size of 64 / 512 / 4096 / 16384 over the model's choice and
its neighbours and picks the fastest.  The winners go to a tuning file of
"key value" lines:

    ultrafastsecp256k1_b200/tuning/<device name>_<SMs>sm.txt

The C++ backend reads that file at context creation (or the file named by
UFSECP_B200_TUNING).  Prints the measurements as JSON.
"""
from __future__ import annotations

import argparse
import json
import os
import re

import numpy as np

import ultrafastsecp256k1_b200 as uf

TUNING_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")
VARIANTS = 12
# window widths of each variant (kVariantPWin / kVariantGWin in csrc/kernels.h)
P_WINDOW = [4] * 9 + [3, 5, 4]
G_WINDOW = [20] * 9 + [18, 20, 16]
RLC_SIZES = (64, 512, 4096, 16384)


def tuning_path(name: str, sms: int) -> str:
    return os.path.join(TUNING_DIR, f"{re.sub(r'[^A-Za-z0-9]+', '_', name).strip('_')}_{sms}sm.txt")


def signed_batch(ctx, torch, kind: int, n: int, seed: int):
    rng = np.random.default_rng(seed)
    sks = rng.integers(1, 255, (n, 32), dtype=np.uint8)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_m, d_k, d_a = dev(msgs), dev(sks), dev(aux)
    ps = 33 if kind == 0 else 32
    d_p = torch.empty(n * ps, dtype=torch.uint8, device="cuda")
    d_s = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.sign_device(kind, d_m.data_ptr(), d_k.data_ptr(), d_a.data_ptr(), n, d_p.data_ptr(), d_s.data_ptr(),
                    d_ok.data_ptr(), 0)
    torch.cuda.synchronize()
    torch.cuda.ExternalStream(ctx.stream()).synchronize()
    # flip one bit in every 50th signature so the verdicts are not all 1
    s = d_s.view(n, 64)
    s[::50, 40] ^= 0x04
    torch.cuda.synchronize()
    return d_m, d_p, d_s


def time_variant(ctx, torch, kind, bufs, n, reps=3):
    d_m, d_p, d_s = bufs
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    fn = ctx.ecdsa_verify_device if kind == 0 else ctx.schnorr_verify_device
    fn(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, out.data_ptr(), st.cuda_stream)   # warm-up
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        fn(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, out.data_ptr(), st.cuda_stream)
    b.record(st)
    st.synchronize()
    ms = a.elapsed_time(b) / reps
    return n / (ms * 1e-3), out.cpu().numpy()


SMALL_SIZES = (4096, 8192, 16384, 32768, 65536)


def tune_small(ctx, torch, kind, bufs, main: int, reps: int = 10) -> dict:
    """Small launches (a few warps per SM) are latency-bound, where inlining
    the field arithmetic can beat the variant that is fastest at full
    occupancy.  Times every variant at SMALL_SIZES; the fastest at the
    smallest size becomes the small-launch variant, used up to the largest
    size at which it still beats `main` (none if it never does)."""
    rates = {v: {} for v in range(VARIANTS)}
    for v in range(VARIANTS):
        ctx.set_variant(kind, v)
        for n in SMALL_SIZES:
            rates[v][n] = time_variant(ctx, torch, kind, bufs, n, reps)[0]
    ctx.set_variant(kind, main)
    small = max(range(VARIANTS), key=lambda v: rates[v][SMALL_SIZES[0]])
    items = 0
    for n in SMALL_SIZES:
        if small != main and rates[small][n] > rates[main][n]:
            items = n
        else:
            break
    return {"variant": small if items else None, "items": items,
            "sigs_per_s": {str(v): {str(n): r for n, r in rs.items()} for v, rs in rates.items()}}


def tune_lanes(ctx, torch, kind, bufs, reps: int = 10) -> dict:
    """Two lanes per signature against one, with the tuned (small-launch)
    variants in place: the limit is the largest SMALL_SIZES entry up to which
    two lanes stay faster (0: never)."""
    rates = {1: {}, 2: {}}
    for lanes in (1, 2):
        ctx.set_lanes(kind, lanes, 1 << 30)
        for n in SMALL_SIZES:
            rates[lanes][n] = time_variant(ctx, torch, kind, bufs, n, reps)[0]
    ctx.set_lanes(kind, 1)
    items = 0
    for n in SMALL_SIZES:
        if rates[2][n] > rates[1][n]:
            items = n
        else:
            break
    return {"items": items, "sigs_per_s": {str(l): {str(n): r for n, r in rs.items()} for l, rs in rates.items()}}


INV_GROUPS = (1, 64, 128)


def tune_inversion_group(ctx, torch, kind, bufs, n, ref, reps: int = 3) -> dict:
    """Threads per block that share each modular inversion (Montgomery's trick
    across a block, ufsecp_gpu_ext_set_inversion_group): 1 (every signature
    alone, the tuned variant), 64 or 128, timed at the main batch size with the
    main variant in place; every group must reproduce the verdicts."""
    rates = {}
    for g in INV_GROUPS:
        ctx.set_inversion_group(kind, g)
        rate, verdicts = time_variant(ctx, torch, kind, bufs, n, reps)
        if not (verdicts == ref).all():
            raise RuntimeError(f"inversion group {g} disagrees with the variants")
        rates[g] = rate
    best = max(rates, key=rates.get)
    ctx.set_inversion_group(kind, best)
    return {"best": best, "sigs_per_s": {str(g): r for g, r in rates.items()}}


def model_window(n: int) -> int:
    """The backend's cost model (rlc_window_bits in csrc/rlc.cu)."""
    best, cost = 4, float("inf")
    for c in range(4, 17):
        w, b = -(-129 // c), 1 << (c - 1)
        v = (3.0 * n + 2.0) * w + 3.0 * w * b + 0.7 * (w - 1) * c
        if v < cost:
            best, cost = c, v
    return best


def tune_rlc(ctx, torch, total: int = 1 << 18, reps: int = 2) -> dict:
    import time
    d_m, d_p, d_s = signed_batch(ctx, torch, 1, total, seed=91)
    d_s.view(total, 64)[::50, 40] ^= 0x04        # undo the flips: an all-valid corpus
    torch.cuda.synchronize()
    out = torch.zeros(total, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    res = {}
    for size in RLC_SIZES:
        c0 = model_window(size)
        rates = {}
        for c in range(max(4, c0 - 2), min(16, c0 + 2) + 1):
            call = lambda: ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), total,
                                                         out.data_ptr(), batch_size=size, seed32=bytes(32),
                                                         window_bits=c, stream=st.cuda_stream)
            call()
            t0 = time.perf_counter()
            for _ in range(reps):
                call()
            rates[c] = total * reps / (time.perf_counter() - t0)
            if not bool(out.all()):
                raise RuntimeError("RLC rejected a valid corpus while tuning")
        best = max(rates, key=rates.get)
        res[str(size)] = {"model": c0, "best": best, "sigs_per_s": {str(k): v for k, v in rates.items()}}
    return res


RLC_CHUNKS = (4, 6, 8, 12, 16, 24, 32)


def tune_rlc_chunk(ctx, torch, windows: dict, total: int = 1 << 18, reps: int = 2) -> dict:
    """Bucket points per chunk thread per RLC batch size, at the tuned window."""
    import time
    d_m, d_p, d_s = signed_batch(ctx, torch, 1, total, seed=92)
    d_s.view(total, 64)[::50, 40] ^= 0x04        # an all-valid corpus
    torch.cuda.synchronize()
    out = torch.zeros(total, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    res = {}
    try:
        for size in RLC_SIZES:
            c = windows[str(size)]["best"]
            rates = {}
            for chunk in RLC_CHUNKS:
                ctx.set_rlc_chunk(chunk)
                call = lambda: ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), total,
                                                             out.data_ptr(), batch_size=size, seed32=bytes(32),
                                                             window_bits=c, stream=st.cuda_stream)
                call()
                t0 = time.perf_counter()
                for _ in range(reps):
                    call()
                rates[chunk] = total * reps / (time.perf_counter() - t0)
                if not bool(out.all()):
                    raise RuntimeError("RLC rejected a valid corpus while tuning the chunk")
            best = max(rates, key=rates.get)
            res[str(size)] = {"best": best, "sigs_per_s": {str(k): v for k, v in rates.items()}}
    finally:
        ctx.set_rlc_chunk(0)
    return res


def autotune(batch: int = 1 << 18, out_path: str | None = None, write: bool = True) -> dict:
    import torch
    info = uf.device_info(0)
    name = info.name.decode()
    res = {"device": name, "sm_count": info.compute_units, "batch": batch, "kinds": {}}
    with uf.GpuContext(0) as ctx:
        for kind, label in ((0, "ecdsa"), (1, "schnorr")):
            bufs = signed_batch(ctx, torch, kind, batch, seed=77 + kind)
            rates, ref = {}, None
            for v in range(VARIANTS):
                ctx.set_variant(kind, v)
                rate, verdicts = time_variant(ctx, torch, kind, bufs, batch)
                if ref is None:
                    ref = verdicts
                elif not (verdicts == ref).all():
                    raise RuntimeError(f"variant {v} disagrees with variant 0 on {label}")
                rates[v] = rate
            best = max(rates, key=rates.get)
            small = tune_small(ctx, torch, kind, bufs, best)
            ctx.set_variant(kind, best)
            group = tune_inversion_group(ctx, torch, kind, bufs, batch, ref)
            if small["variant"] is not None:
                ctx.set_small_variant(kind, small["variant"], small["items"])
            res["kinds"][label] = {"sigs_per_s": {str(k): r for k, r in rates.items()}, "best": best,
                                   "valid": int(ref.sum()), "small": small, "inversion_group": group,
                                   "lanes": tune_lanes(ctx, torch, kind, bufs)}
        res["rlc_window"] = tune_rlc(ctx, torch)
        res["rlc_chunk"] = tune_rlc_chunk(ctx, torch, res["rlc_window"])
    if write:
        path = out_path or tuning_path(name, info.compute_units)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            for label in ("ecdsa", "schnorr"):
                k = res["kinds"][label]
                f.write(f"{label}_variant {k['best']}\n")
                # the window widths of the chosen variant (informational: the variant number selects them)
                f.write(f"{label}_p_window {P_WINDOW[k['best']]}\n")
                f.write(f"{label}_g_window {G_WINDOW[k['best']]}\n")
                f.write(f"{label}_inv_group {k['inversion_group']['best']}\n")
                if k["small"]["variant"] is not None:
                    f.write(f"{label}_small_variant {k['small']['variant']}\n")
                    f.write(f"{label}_small_items {k['small']['items']}\n")
                if k["lanes"]["items"]:
                    f.write(f"{label}_pair_items {k['lanes']['items']}\n")
            for size, r in res["rlc_window"].items():
                f.write(f"rlc_window_{size} {r['best']}\n")
            for size, r in res["rlc_chunk"].items():
                f.write(f"rlc_chunk_{size} {r['best']}\n")
        res["tuning_file"] = path
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=1 << 18)
    ap.add_argument("--out", default=None)
    ap.add_argument("--no-write", action="store_true")
    a = ap.parse_args()
    print(json.dumps(autotune(a.batch, a.out, not a.no_write), indent=1))


if __name__ == "__main__":
    main()
