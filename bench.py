#!/usr/bin/env python3
"""Benchmark: verified signatures per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one pass of the hot path over one batch: one launch that verifies
the 1,048,576-signature BIP-340 batch (seeded keys, 32-byte x-only keys,
uniform messages, seeded aux_rand; 1% of signatures with one flipped bit in
s or R.x, 0.1% of keys off the curve).  Signatures are made on the GPU by the
library's batch signer (byte-identical to the reference's CPU signer; checked
by the tests).

* value: whole-job sigs/s with inputs resident in HBM (device-pointer entry
  ufsecp_gpu_ext_schnorr_verify_device), CUDA events on the launching stream,
  max over ranks.
* e2e: the same work through the reference ABI call
  ufsecp_gpu_schnorr_verify_batch with host buffers, copies included.
* roofline: integer-pipe (IMAD) bound; achieved = sigs/s x the canonical
  3.33e5 IMAD-class ops per signature, against the device's IMAD issue rate
  measured in this run; HBM bytes of the same launch beside it.
* cpu_baseline: the reference library (oracle/_ref, compiled from the
  reference sources) on all host threads over a bounded sample.
Multi-GPU: one process per GPU (torchrun), every rank verifies its own batch
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "verified sigs/sec on 1 B200 (ECDSA, BIP-340) batched vs plain kernel; p50/p99"
N_ORDER = 0xFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFEBAAEDCE6AF48A03BBFD25E8CD0364141
P_FIELD = 2**256 - 2**32 - 977
W_SIG = 3.33e5            # IMAD-class ops per verified signature (canonical work model)
BYTES_PER_SIG = 32 + 32 + 64 + 1
BATCH = 1 << 20
CPU_SAMPLE = 1 << 20            # the whole headline batch


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the mixed-batch / RLC / serving sections")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers --
def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def profile_traffic():
    """dram bytes per launch of the verify kernel from the committed ncu summary."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while running; entering
    waits for the first sample so the timed region that follows is covered."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clk", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        self.skip = 1      # the sample taken before the timed region started
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        rows = rows[getattr(self, "skip", 0):] or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


def offcurve_x(rng):
    while True:
        x = int.from_bytes(rng.bytes(32), "big") % P_FIELD
        if pow((x**3 + 7) % P_FIELD, (P_FIELD - 1) // 2, P_FIELD) != 1:
            return x


def tamper(rng, xs, sigs, expect):
    """1% of items: one flipped bit in s or R.x; 0.1%: x-only key off the curve."""
    n = xs.shape[0]
    idx = rng.choice(n, size=n // 100, replace=False)
    for i in idx:
        bit = int(rng.integers(0, 256))
        off = 0 if rng.integers(0, 2) else 32
        sigs[i, off + bit // 8] ^= 1 << (bit % 8)
    expect[idx] = 0
    idx = rng.choice(n, size=max(1, n // 1000), replace=False)
    for i in idx:
        xs[i] = np.frombuffer(offcurve_x(rng).to_bytes(32, "big"), np.uint8)
    expect[idx] = 0


def make_schnorr_batch(ctx, torch, n: int, seed: int, invalid: bool = True):
    """Seeded BIP-340 batch, signed on the GPU; returns device tensors, host
    copies and the verdict every item must get (by construction).  invalid=False
    leaves every signature valid."""
    rng = np.random.default_rng(seed)
    sks = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    # keys uniform in [1, n-1]: redraw the (astronomically rare) values outside
    hi = sks[:, 0] == 0xFF
    for i in np.nonzero(hi)[0]:
        while not (0 < int.from_bytes(sks[i].tobytes(), "big") < N_ORDER):
            sks[i] = rng.integers(0, 256, 32, dtype=np.uint8)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_msgs, d_sks, d_aux = dev(msgs), dev(sks), dev(aux)
    d_xs = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    d_sigs = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
    ctx.sign_device(1, d_msgs.data_ptr(), d_sks.data_ptr(), d_aux.data_ptr(), n, d_xs.data_ptr(),
                    d_sigs.data_ptr(), d_ok.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert bool(d_ok.all()), "signer rejected a key"
    del d_sks, d_aux
    xs = d_xs.cpu().numpy().reshape(n, 32)
    sigs = d_sigs.cpu().numpy().reshape(n, 64)
    expect = np.ones(n, np.uint8)
    if invalid:
        tamper(rng, xs, sigs, expect)
    d_xs = dev(xs)
    d_sigs = dev(sigs)
    d_out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    return (d_msgs, d_xs, d_sigs, d_out), (msgs, xs, sigs), expect


def launches_per_call(n: int) -> int:
    """Kernel launches of one ufsecp_gpu_ext_schnorr_verify_device call over n items
    (large calls are cut into launches of 131,072 on two streams)."""
    chunk = 1 << 17
    return 1 if n < 2 * chunk else -(-n // chunk)


def cpu_reference_rate(msgs, xs, sigs, sample: int):
    """Reference library, all host threads, ufsecp_schnorr_verify per signature."""
    from oracle import RefDriver
    drv = RefDriver()
    threads = os.cpu_count() or 1
    m, x, s = msgs[:sample], xs[:sample], sigs[:sample]
    drv.verify(1, m[:2048], x[:2048], s[:2048], threads)          # one-time table set-up
    t0 = time.perf_counter()
    verdicts = drv.verify(1, m, x, s, threads)
    dt = time.perf_counter() - t0
    return sample / dt, threads, verdicts, dt


# -------------------------------------------------------------- reference arm --
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import REF_SO, RefDriver
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
        return 0
    # the reference arm makes its corpus with the reference's own signer, same seeds and tamper rules
    drv = RefDriver()
    threads = os.cpu_count() or 1
    n = min(args.batch, 1 << 17)
    rng = np.random.default_rng(20261203)
    sks = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    xs, sigs, ok = drv.sign(1, msgs, sks, aux, threads)
    expect = ok.copy()
    tamper(rng, xs, sigs, expect)
    per_step = min(n, max(8192, 1500 * threads))
    drv.verify(1, msgs[:2048], xs[:2048], sigs[:2048], threads)
    for _ in range(args.warmup):
        drv.verify(1, msgs[:per_step], xs[:per_step], sigs[:per_step], threads)
    t0 = time.perf_counter()
    agree = 0
    for k in range(args.steps):
        off = (k * per_step) % max(1, n - per_step + 1)
        v = drv.verify(1, msgs[off:off + per_step], xs[off:off + per_step], sigs[off:off + per_step], threads)
        agree += int((v == expect[off:off + per_step]).sum())
    dt = time.perf_counter() - t0
    rate = args.steps * per_step / dt
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "sigs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded BIP-340 corpus (1% flipped bits, 0.1% off-curve keys)",
            "config": {"workload": "bip340_verify_1M_one_launch", "signatures_per_step": per_step,
                       "parallelism": f"{threads} host threads, one ufsecp_ctx each"},
            "cpu_baseline": {"value": rate, "unit": "sigs/s", "cores": threads, "kind": "reference",
                             "sample": f"{per_step} signatures per step from the seeded 1M-signature BIP-340 batch, "
                                       "ufsecp_schnorr_verify per signature"},
            "e2e": {"value": rate, "unit": "sigs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "verdict_agreement": agree / (args.steps * per_step)}
    print(json.dumps(line))
    return 0


# -------------------------------------------------------------------- our arm --
def run_ours(args):
    import torch
    import ultrafastsecp256k1_b200 as uf

    from ultrafastsecp256k1_b200.shard import Ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks.from_env(device="cuda")
    rank = ranks.rank
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    ctx = uf.GpuContext(local)
    n = args.batch
    (d_msgs, d_xs, d_sigs, d_out), (msgs, xs, sigs), expect = make_schnorr_batch(ctx, torch, n,
                                                                                 seed=20261203 + rank)
    torch.cuda.synchronize()   # inputs were written on the default stream
    # an explicit stream: the launches and the events that time them share it
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    def launch():
        ctx.schnorr_verify_device(d_msgs.data_ptr(), d_xs.data_ptr(), d_sigs.data_ptr(), n, d_out.data_ptr(), sptr)

    # ---- device-resident throughput (value) --------------------------------
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    agree = int((d_out.cpu().numpy() == expect).sum())
    imad_peak = ctx.imad_peak()
    barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for k in range(args.steps):
            evs[k][0].record(stream)
            launch()
            evs[k][1].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
    barrier()
    clocks = clk.summary()
    total_ms = max_over_ranks(t_start.elapsed_time(t_end))
    launch_ms = [a.elapsed_time(b) for a, b in evs]
    avg_launch_ms = max_over_ranks(sum(launch_ms) / len(launch_ms))
    total_sigs = sum_over_ranks(float(n * args.steps))
    value = total_sigs / (total_ms * 1e-3)

    # ---- end to end through the reference ABI call (host buffers) ----------
    s_ctx = torch.cuda.ExternalStream(ctx.stream())
    for _ in range(max(1, args.warmup)):
        ctx.schnorr_verify_batch(msgs, xs, sigs)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e_steps = max(2, args.steps // 2)
    e0.record(s_ctx)
    for _ in range(e_steps):
        res = ctx.schnorr_verify_batch(msgs, xs, sigs)
    e1.record(s_ctx)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = sum_over_ranks(float(n * e_steps)) / (e2e_ms * 1e-3)
    e2e_agree = int((res == expect).sum())

    # ---- secondary: plain ECDSA on 4096 and 2^20 signatures ---------------
    c1 = ecdsa_big = None
    mixed = None
    rlc = None
    serving = None
    # single-GPU sections: measured in the one-GPU run only (a multi-GPU run
    # would hold every GPU while rank 0 alone runs them)
    if rank == 0 and world == 1:
        try:
            c1 = bench_c1(ctx, torch)
        except Exception as e:   # reference library missing on this box
            c1 = {"unavailable": str(e)}
        if not args.no_secondary:
            ecdsa_big = ecdsa_plain_rate(ctx, torch, n=1 << 20, reps=3)
            mixed = bench_mixed(ctx, torch)
            rlc = bench_rlc(ctx, torch)
            serving = bench_serving(ctx, torch)

    # ---- CPU baseline (rank 0, one GPU only) --------------------------------
    cpu = None
    ref_agree = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            # every item of the batch: the CPU baseline's sample and the full verdict check at once
            sample = min(CPU_SAMPLE, n)
            rate, threads, verdicts, dt = cpu_reference_rate(msgs, xs, sigs, sample)
            ref_agree = float((verdicts == d_out.cpu().numpy()[:sample]).mean())
            cpu = {"value": rate, "unit": "sigs/s", "cores": threads, "kind": "reference",
                   "sample": f"all {sample:,} signatures of the BIP-340 batch ({dt:.1f} s wall), "
                             "ufsecp_schnorr_verify per signature, one ufsecp_ctx per thread",
                   "verdicts_equal_gpu": ref_agree == 1.0}
        except Exception as e:  # reference library missing on this box
            cpu = {"value": None, "unit": "sigs/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        peaks = measured_peaks()
        traffic = profile_traffic().get("k_verify_schnorr_bytes_per_sig")
        per_launch_s = avg_launch_ms * 1e-3
        sigs_per_rank_s = n / per_launch_s
        achieved = sigs_per_rank_s * W_SIG / 1e9
        peak = imad_peak / 1e9
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        hbm_achieved = n * BYTES_PER_SIG / per_launch_s / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "sigs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic: seeded keys / messages / aux_rand, signed on the GPU (bytes identical to the "
                    "reference signer), 1% one-bit flips in s or R.x, 0.1% off-curve x-only keys",
            "config": {"workload": "bip340_verify_1M_one_launch", "signatures_per_launch": n,
                       "kernel": "plain (one signature per thread)",
                       "parallelism": f"{world} rank(s), one independent batch per GPU",
                       "l2": "inputs 134 MB per launch > 126 MB L2 (no flush needed)"},
            "e2e": {"value": e2e_value, "unit": "sigs/s", "h2d_bytes_per_step": n * 128, "d2h_bytes_per_step": n,
                    "api": "ufsecp_gpu_schnorr_verify_batch (host buffers)",
                    "verdict_agreement": e2e_agree / n},
            "roofline": {"bound": "int", "achieved": achieved, "peak": peak, "unit": "Gop/s",
                         "frac": achieved / peak if peak else None,
                         "traffic": (traffic * n) if traffic else None,
                         "ops_per_sig": W_SIG, "launch_ms": avg_launch_ms,
                         "peak_source": "measured in this run: 32-bit IMAD issue rate (ufsecp_gpu_ext_imad_peak)",
                         "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                                 "frac": hbm_achieved / hbm_peak, "peak_source": "of measured (MEASURED_PEAKS.json)"}},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps * launches_per_call(n),
            "verdict_agreement": ref_agree if ref_agree is not None else agree / n,
            "verdict_agreement_source": ("reference library, every item of the batch" if ref_agree is not None
                                         else "construction (reference library unavailable)"),
            "verdict_agreement_construction": agree / n,
            "secondary": {"ecdsa_4096": c1, "ecdsa_1048576_plain_sigs_per_s": ecdsa_big,
                          "mixed_batches": mixed, "rlc_batch_verify": rlc,
                          "serving": serving},
        }
        print(json.dumps(line))
    del d_msgs, d_xs, d_sigs, d_out
    ctx.close()
    ranks.close()
    return 0


def mixed_workload(ctx, torch, n_batches=2000, seed=3, pool=100_000):
    """Mixed batches: sizes log-uniform in [1, 8192], 70% BIP-340 / 30% ECDSA inside
    each batch, keys drawn Zipf(s=1.1) from a seeded pool, 0.5% one-bit tampering.
    Signed on the GPU.  Returns per-batch (kind-split) host arrays."""
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.exp(rng.uniform(0, np.log(8192), n_batches)).astype(np.int64), 1, 8192)
    total = int(sizes.sum())
    pool_sk = rng.integers(1, 255, (pool, 32), dtype=np.uint8)
    w = 1.0 / np.arange(1, pool + 1) ** 1.1
    key_idx = rng.choice(pool, size=total, p=w / w.sum())
    kinds = (rng.random(total) < 0.7).astype(np.uint8)          # 1 = BIP-340
    msgs = rng.integers(0, 256, (total, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (total, 32), dtype=np.uint8)
    sks = pool_sk[key_idx]
    out = {}
    for kind, ps in ((0, 33), (1, 32)):
        sel = np.nonzero(kinds == kind)[0]
        n = sel.size
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        d_m, d_k, d_a = dev(msgs[sel]), dev(sks[sel]), dev(aux[sel])
        d_p = torch.empty(n * ps, dtype=torch.uint8, device="cuda")
        d_s = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
        d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        ctx.sign_device(kind, d_m.data_ptr(), d_k.data_ptr(), d_a.data_ptr(), n, d_p.data_ptr(), d_s.data_ptr(),
                        d_ok.data_ptr(), 0)
        torch.cuda.ExternalStream(ctx.stream()).synchronize()
        sigs = d_s.cpu().numpy().reshape(n, 64)
        clean = sigs.copy()
        expect = np.ones(n, np.uint8)
        bad = rng.choice(n, size=max(1, n // 200), replace=False)
        for i in bad:
            bit = int(rng.integers(0, 512))
            sigs[i, bit // 8] ^= 1 << (bit % 8)
        expect[bad] = 0
        out[kind] = (sel, msgs[sel], d_p.cpu().numpy().reshape(n, ps), sigs, expect, clean)
    # split back into batches (each batch: its ECDSA items and its BIP-340 items)
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    pos = {0: np.searchsorted(out[0][0], bounds), 1: np.searchsorted(out[1][0], bounds)}
    batches = []
    kinds_j, starts_j, counts_j = [], [], []
    for b in range(n_batches):
        parts = []
        for kind in (0, 1):
            lo, hi = pos[kind][b], pos[kind][b + 1]
            sel, m, p, s, ex, _ = out[kind]
            parts.append((kind, m[lo:hi], p[lo:hi], s[lo:hi], ex[lo:hi]))
            kinds_j.append(kind)
            starts_j.append(lo)
            counts_j.append(hi - lo)
        batches.append(parts)
    # the same jobs as index ranges of the two per-kind corpora
    corpora = {k: tuple(np.ascontiguousarray(a) for a in out[k][1:4]) for k in (0, 1)}
    expects = {k: out[k][4] for k in (0, 1)}
    ranges = (np.array(kinds_j), np.array(starts_j), np.array(counts_j))
    # the BIP-340 items before tampering (an all-valid variant of the same jobs)
    clean1 = (corpora[1][0], corpora[1][1], np.ascontiguousarray(out[1][5]))
    return batches, total, corpora, expects, ranges, clean1


def bench_mixed(ctx, torch):
    """The mixed-batch workload (2000 caller batches) five ways, same items:
    one plain ABI call per batch and kind; ufsecp_gpu_ext_verify_jobs over
    groups of >= 262,144 signatures and over all 2000 batches in one call (job
    lists marshalled per job in Python); the one call with the job table built
    by vector operations from index ranges (what a C / C++ caller pays), with
    the resident key table cold (emptied just before), warm (every key resident
    from the previous call) and off; and the plain one-signature-per-thread
    kernel over the same items already on the device (one launch per kind,
    CUDA events): the ceiling a batched form has to beat.  Each host form runs
    once untimed first (staging buffers, batch slots, streams, graphs), then
    once timed.  Verdicts: every form against the construction, and every item
    against the reference library on the host cores."""
    import time as _t
    batches, total, corpora, expects, (kinds_j, starts_j, counts_j), clean1 = mixed_workload(ctx, torch)

    def plain_pass():
        # the reference-style synchronous call per batch and kind; verdicts
        # are compared after the timed loop
        got, exps = [], []
        t0 = _t.perf_counter()
        for parts in batches:
            for kind, m, p, s, ex in parts:
                if len(m) == 0:
                    continue
                got.append(ctx.ecdsa_verify_batch(m, p, s) if kind == 0 else ctx.schnorr_verify_batch(m, p, s))
                exps.append(ex)
        dt = _t.perf_counter() - t0
        return dt, sum(int((g == ex).sum()) for g, ex in zip(got, exps))

    group_items = 1 << 18

    def batched_pass():
        # groups of consecutive batches packed into one persistent-queue launch;
        # verdicts are compared after the timed loop
        got, exps = [], []
        t0 = _t.perf_counter()
        i = 0
        while i < len(batches):
            jobs, n = [], 0
            while i < len(batches) and (n == 0 or n < group_items):
                for kind, m, p, s, ex in batches[i]:
                    jobs.append((kind, m, p, s))
                    exps.append(ex)
                    n += len(m)
                i += 1
            got += ctx.verify_jobs(jobs)
        dt = _t.perf_counter() - t0
        return dt, sum(int((o == ex).sum()) for o, ex in zip(got, exps))

    def one_call_pass():
        # every batch of both kinds in one ufsecp_gpu_ext_verify_jobs call
        jobs, exps = [], []
        for parts in batches:
            for kind, m, p, s, ex in parts:
                jobs.append((kind, m, p, s))
                exps.append(ex)
        t0 = _t.perf_counter()
        got = ctx.verify_jobs(jobs)
        dt = _t.perf_counter() - t0
        return dt, sum(int((o == ex).sum()) for o, ex in zip(got, exps))

    def ranges_pass():
        t0 = _t.perf_counter()
        got = ctx.verify_job_ranges(corpora, kinds_j, starts_j, counts_j)
        dt = _t.perf_counter() - t0
        return dt, sum(int((got[k] == expects[k]).sum()) for k in (0, 1)), got

    plain_pass()
    t_plain, agree = plain_pass()
    batched_pass()
    t_batched, agree_b = batched_pass()
    one_call_pass()
    t_one, agree_o = one_call_pass()
    ranges_pass()
    ctx.set_key_table(18)                       # emptied in place: the timed call builds every key's table
    t_cold, agree_c, _ = ranges_pass()
    cold_stats = ctx.key_table_stats()
    t_warm, agree_w, got_w = ranges_pass()      # every key resident from the call before
    ctx.set_key_table(0)
    ranges_pass()
    t_off, agree_n, _ = ranges_pass()
    ctx.set_key_table(18)

    # BIP-340 jobs as kind 2 (one RLC batch over all of them, 16384-item
    # segments), on these items (0.5 % invalid) and on the all-valid variant
    kinds_r = np.where(kinds_j == 1, 2, kinds_j)
    n_bip = len(corpora[1][0])

    def jobs_pass(corp, kinds, exps):
        t0 = _t.perf_counter()
        got = ctx.verify_job_ranges(corp, kinds, starts_j, counts_j)
        dt = _t.perf_counter() - t0
        return dt, sum(int((got[k] == exps[k]).sum()) for k in corp)

    ones = np.ones(n_bip, np.uint8)
    rlc_rows = {}
    for label, corp1, exp1 in (("tampered", corpora[1], expects[1]), ("all_valid_bip340", clean1, ones)):
        for kind in (1, 2):
            corp = {0: corpora[0], kind: corp1}
            kinds = kinds_j if kind == 1 else kinds_r
            exps = {0: expects[0], kind: exp1}
            jobs_pass(corp, kinds, exps)
            t, agree_x = jobs_pass(corp, kinds, exps)
            rlc_rows[f"{label}_kind{kind}"] = {"sigs_per_s": total / t, "verdict_agreement": agree_x / total}

    # the plain kernel over the same items, device-resident, one launch per kind
    st = torch.cuda.Stream()
    dev = {k: [torch.from_numpy(a.reshape(-1)).cuda() for a in corpora[k]] for k in (0, 1)}
    d_out = {k: torch.zeros(len(corpora[k][0]), dtype=torch.uint8, device="cuda") for k in (0, 1)}
    torch.cuda.synchronize()

    def plain_kernel():
        for k, f in ((0, ctx.ecdsa_verify_device), (1, ctx.schnorr_verify_device)):
            m, p, sg = dev[k]
            f(m.data_ptr(), p.data_ptr(), sg.data_ptr(), len(d_out[k]), d_out[k].data_ptr(), st.cuda_stream)

    for _ in range(2):
        plain_kernel()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    a.record(st)
    for _ in range(reps):
        plain_kernel()
    b.record(st)
    torch.cuda.synchronize()
    plain_kernel_rate = total * reps / (a.elapsed_time(b) * 1e-3)
    agree_k = sum(int((d_out[k].cpu().numpy() == expects[k]).sum()) for k in (0, 1))

    # every item against the reference library (host cores), outside the timed regions
    ref_agree = None
    try:
        from oracle import RefDriver
        drv = RefDriver()
        thr = os.cpu_count() or 1
        ref_agree = sum(int((drv.verify(k, *corpora[k], thr) == got_w[k]).sum()) for k in (0, 1)) / total
    except Exception as e:   # reference library missing on this box
        ref_agree = f"unavailable: {e}"
    return {"workload": "2000 mixed batches, sizes log-uniform [1, 8192], 70/30 BIP-340/ECDSA, Zipf(1.1) keys "
                        "from a 100k pool, 0.5% invalid",
            "signatures": total, "jobs": int(len(kinds_j)),
            "plain_sigs_per_s": total / t_plain, "batched_sigs_per_s": total / t_batched,
            "batched_over_plain": t_plain / t_batched,
            "plain": "one ufsecp_gpu_{ecdsa,schnorr}_verify_batch call per batch and kind (host buffers, wall clock, "
                     "second pass)",
            "batched": f"ufsecp_gpu_ext_verify_jobs over groups of >= {group_items} signatures (host buffers, wall "
                       "clock, second pass)",
            "batched_one_call_sigs_per_s": total / t_one,
            "batched_one_call": "all 2000 batches in one ufsecp_gpu_ext_verify_jobs call, job list marshalled per "
                                "job in Python (host buffers, wall clock, second pass)",
            "one_call_ranges": {
                "api": "ufsecp_gpu_ext_verify_jobs, job table built by numpy vector operations from per-batch index "
                       "ranges (host buffers, wall clock)",
                "key_table_cold_sigs_per_s": total / t_cold,
                "key_table_warm_sigs_per_s": total / t_warm,
                "key_table_off_sigs_per_s": total / t_off,
                "cold_key_table": {"lookups": cold_stats["lookups"], "hits": cold_stats["hits"]},
                "cold_over_plain_kernel": (total / t_cold) / plain_kernel_rate,
                "warm_over_plain_kernel": (total / t_warm) / plain_kernel_rate},
            "plain_kernel_sigs_per_s": plain_kernel_rate,
            "plain_kernel": "ufsecp_gpu_ext_{ecdsa,schnorr}_verify_device over all items of each kind, one call per "
                            "kind, inputs on the device, CUDA events",
            "rlc_job_kind": {
                "api": "ufsecp_gpu_ext_verify_jobs from index ranges, key table on: the BIP-340 jobs as kind 1 "
                       "(work queue) or kind 2 (one RLC batch over all BIP-340 items, 16384-item segments); the "
                       "ECDSA jobs kind 0 in both; on these items and with the BIP-340 items untampered",
                **rlc_rows},
            "verdict_agreement": {"plain": agree / total, "batched": agree_b / total, "batched_one_call": agree_o / total,
                                  "ranges_cold": agree_c / total, "ranges_warm": agree_w / total,
                                  "ranges_off": agree_n / total, "plain_kernel": agree_k / total,
                                  "reference_library_all_items": ref_agree}}


def bench_rlc(ctx, torch, n: int = 1 << 20, reps: int = 3):
    """RLC batch verify (BIP-340) against the plain kernel on the same n valid
    signatures cut into batches of 64 / 512 / 4096 / 16384, with 0 or 1 invalid
    signature per batch (one flipped bit of s).  Device-resident inputs; each
    RLC call is synchronous (it reads every round's result on the host), so it
    is timed by wall clock around the call, after one untimed call."""
    (d_m, d_x, d_s, d_out), (msgs, xs, sigs), _ = make_schnorr_batch(ctx, torch, n, seed=64, invalid=False)
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        ctx.schnorr_verify_device(d_m.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        ctx.schnorr_verify_device(d_m.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    b.record(st)
    torch.cuda.synchronize()
    plain = n * reps / (a.elapsed_time(b) * 1e-3)
    rng = np.random.default_rng(65)
    rows = []
    for bs in (64, 512, 4096, 16384):
        for bad in (0, 1):
            expect = np.ones(n, np.uint8)
            d_sig = d_s
            if bad:
                s_bad = sigs.copy()
                for start in range(0, n, bs):
                    i = start + int(rng.integers(0, min(bs, n - start)))
                    bit = int(rng.integers(0, 256))
                    s_bad[i, 32 + bit // 8] ^= 1 << (bit % 8)
                    expect[i] = 0
                d_sig = torch.from_numpy(s_bad).cuda()
            torch.cuda.synchronize()
            seed = rng.bytes(32)
            ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_x.data_ptr(), d_sig.data_ptr(), n, d_out.data_ptr(),
                                          batch_size=bs, seed32=seed, stream=st.cuda_stream)
            t0 = time.perf_counter()
            for _ in range(reps):
                ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_x.data_ptr(), d_sig.data_ptr(), n, d_out.data_ptr(),
                                              batch_size=bs, seed32=seed, stream=st.cuda_stream)
            dt = (time.perf_counter() - t0) / reps
            stats = ctx.rlc_stats()
            agree = float((d_out.cpu().numpy() == expect).mean())
            rows.append({"batch": bs, "invalid_per_batch": bad, "sigs_per_s": n / dt, "ms_per_call": dt * 1e3,
                         "over_plain": n / dt / plain, "window_bits": stats["window_bits"],
                         "msm_rounds": stats["rounds"], "leaf_items": stats["leaf_items"],
                         "verdict_agreement": agree})
            del d_sig
    return {"workload": f"{n} valid BIP-340 signatures in batches of 64/512/4096/16384, 0 or 1 invalid per batch",
            "plain_sigs_per_s": plain,
            "plain": "ufsecp_gpu_ext_schnorr_verify_device, one launch over all items, CUDA events",
            "rlc": "ufsecp_gpu_ext_schnorr_verify_rlc_device (device buffers, wall clock per call)",
            "rows": rows}


def serving_pools(ctx, torch, n_s=300_000, n_e=130_000, pool=100_000, seed=5):
    """Signed item pools for the serving workload: keys drawn Zipf(1.1) from a
    seeded 100k-key pool, 0.5% one-bit tampering.  Signed on the GPU."""
    rng = np.random.default_rng(seed)
    pool_sk = rng.integers(1, 255, (pool, 32), dtype=np.uint8)
    w = 1.0 / np.arange(1, pool + 1) ** 1.1
    w /= w.sum()
    out = {}
    for kind, n, ps in ((1, n_s, 32), (0, n_e, 33)):
        sks = pool_sk[rng.choice(pool, size=n, p=w)]
        msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
        aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        d_m, d_k, d_a = dev(msgs), dev(sks), dev(aux)
        d_p = torch.empty(n * ps, dtype=torch.uint8, device="cuda")
        d_s = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
        d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        ctx.sign_device(kind, d_m.data_ptr(), d_k.data_ptr(), d_a.data_ptr(), n, d_p.data_ptr(), d_s.data_ptr(),
                        d_ok.data_ptr(), 0)
        torch.cuda.ExternalStream(ctx.stream()).synchronize()
        sigs = d_s.cpu().numpy().reshape(n, 64)
        expect = np.ones(n, np.uint8)
        bad = rng.choice(n, size=n // 200, replace=False)
        for i in bad:
            bit = int(rng.integers(0, 512))
            sigs[i, bit // 8] ^= 1 << (bit % 8)
        expect[bad] = 0
        out[kind] = (msgs, d_p.cpu().numpy().reshape(n, ps), sigs, expect)
    return out


def serving_requests(pools, rate, duration, seed, fixed_size=None):
    """Poisson arrivals offering `rate` sigs/s for `duration` s; sizes log-uniform
    in [1, 4096] (or fixed), 70/30 BIP-340 / ECDSA items per request."""
    rng = np.random.default_rng(seed)
    mean_size = 4095 / np.log(4096) if fixed_size is None else fixed_size
    lam = rate / mean_size
    t, reqs, off = 0.0, [], {0: 0, 1: 0}
    while True:
        t += rng.exponential(1.0 / lam)
        if t > duration:
            break
        size = fixed_size or int(np.clip(np.exp(rng.uniform(0, np.log(4096))), 1, 4096))
        n_e = int(rng.binomial(size, 0.3))
        jobs, exp = [], []
        for kind, n in ((0, n_e), (1, size - n_e)):
            if n == 0:
                continue
            m, p, s, e = pools[kind]
            lo = off[kind] % (len(m) - 4096)
            off[kind] += n
            jobs.append((kind, m[lo:lo + n], p[lo:lo + n], s[lo:lo + n]))
            exp.append(e[lo:lo + n])
        reqs.append((t, jobs, exp))
    return reqs


def _pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(q * (len(v) - 1) + 0.5))] if v else None


def run_served(uf, reqs, budget=8 << 30, slots=8, key_cache_log2=18, closed=False):
    """Submit at the arrival times from one thread (closed: all at once), wait
    from another; the verdicts are compared after the run, so the waiter holds
    the GIL only around its wait calls."""
    import threading
    sctx = uf.GpuContext(0)
    srv = uf.Server(sctx, slots=slots, max_launch_items=1 << 16, memory_budget_bytes=budget,
                    key_cache_log2=key_cache_log2)
    # warm the graph buckets
    for t, jobs, exp in reqs[:8]:
        srv.wait(srv.submit(jobs))
    srv.stats(reset=True)
    ids = [None] * len(reqs)
    got = [None] * len(reqs)
    ready = threading.Semaphore(0)

    def waiter():
        for k in range(len(reqs)):
            ready.acquire()
            got[k] = srv.wait(ids[k], 120_000)

    th = threading.Thread(target=waiter)
    # the Python collector off while requests arrive: its pauses (tens of ms
    # over thousands of requests' arrays) would hold back the submitting thread
    gc.collect()
    gc.disable()
    try:
        th.start()
        t0 = time.perf_counter()
        lag = 0.0
        for k, (t, jobs, exp) in enumerate(reqs):
            while not closed and time.perf_counter() - t0 < t:
                pass
            lag = max(lag, time.perf_counter() - t0 - t)
            ids[k] = srv.submit(jobs)
            ready.release()
        th.join()
    finally:
        gc.enable()
    st = srv.stats()
    srv.close()
    sctx.close()
    agree = [sum(int((o == e).sum()) for o, e in zip(outs, r[2])) for outs, r in zip(got, reqs)]
    agree = [sum(agree)]
    items = sum(len(j[1]) for _, jobs, _ in reqs for j in jobs)
    return {"sigs_per_s": st["items_done"] / st["span_s"] if st["span_s"] else None,
            "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3, "max_ms": st["max_us"] / 1e3,
            "requests": int(st["requests_done"]), "launches": int(st["launches"]),
            "peak_slots_in_flight": int(st["peak_slots_in_flight"]),
            "peak_budget_mb": st["peak_budget_bytes"] / 2**20, "max_submit_lag_ms": lag * 1e3,
            "key_table_hits": (st["cache_hits"] / st["cache_lookups"]) if st["cache_lookups"] else None,
            "verdict_agreement": agree[0] / items}


def run_plain(ctx, reqs, limit_s):
    """The plain kernel under the same arrivals: one synchronous per-kind ABI call
    per request, in arrival order (a queue, no batching)."""
    lat, done_items, agree = [], 0, 0
    gc.collect()
    gc.disable()            # as in run_served
    try:
        t0 = time.perf_counter()
        t_last = t0
        for t, jobs, exp in reqs:
            now = time.perf_counter() - t0
            if now > limit_s:
                break
            while now < t:
                now = time.perf_counter() - t0
            for (kind, m, p, s), e in zip(jobs, exp):
                o = ctx.ecdsa_verify_batch(m, p, s) if kind == 0 else ctx.schnorr_verify_batch(m, p, s)
                agree += int((o == e).sum())
                done_items += len(m)
            t_last = time.perf_counter()
            lat.append((t_last - t0 - t) * 1e3)
    finally:
        gc.enable()
    span = t_last - t0
    return {"sigs_per_s": done_items / span if span > 0 else None, "p50_ms": _pct(lat, 0.5),
            "p99_ms": _pct(lat, 0.99), "max_ms": max(lat) if lat else None, "requests": len(lat),
            "requests_offered": len(reqs), "verdict_agreement": agree / max(done_items, 1)}


def bench_serving(ctx, torch):
    import ultrafastsecp256k1_b200 as uf
    pools = serving_pools(ctx, torch)
    rows = []
    for rate, dur in ((10_000, 3.0), (100_000, 3.0), (1_000_000, 2.0), (10_000_000, 1.0)):
        reqs = serving_requests(pools, rate, dur, seed=rate)
        row = {"offered_sigs_per_s": rate, "duration_s": dur, "requests": len(reqs), "served": run_served(uf, reqs)}
        # the plain calls fall behind from 1 M sigs/s offered; at 10 M they are not run
        if rate <= 1_000_000:
            row["plain"] = run_plain(ctx, reqs, limit_s=dur + 8.0)
        rows.append(row)
    reqs = serving_requests(pools, 1_000_000, 2.0, seed=4096, fixed_size=4096)
    fixed = {"offered_sigs_per_s": 1_000_000, "request_size": 4096, "requests": len(reqs),
             "served": run_served(uf, reqs)}
    # closed loop: the 10 M sigs/s request set submitted all at once, with and
    # without the resident key table (each run on a fresh server: the table
    # starts empty)
    reqs = serving_requests(pools, 10_000_000, 1.0, seed=10_000_000)
    closed = {"requests": len(reqs),
              "key_table_on": run_served(uf, reqs, closed=True, key_cache_log2=18),
              "key_table_off": run_served(uf, reqs, closed=True, key_cache_log2=0)}
    return {"workload": "Poisson arrivals, request sizes log-uniform [1, 4096], 70/30 BIP-340/ECDSA items, "
                        "Zipf(1.1) keys from a 100k pool, 0.5% invalid, 8 GiB admission budget",
            "served": "ufsecp_gpu_ext_server_* (8 slots, continuous batching); latency submit -> verdicts, "
                      "measured by the server; Python's collector off while requests arrive (both forms)",
            "plain": "one synchronous ufsecp_gpu_{ecdsa,schnorr}_verify_batch call per request and kind, FIFO; "
                     "latency arrival -> verdicts (wall clock)",
            "rates": rows, "fixed_4096": fixed, "closed_loop": closed}


def ecdsa_plain_rate(ctx, torch, n=1 << 20, reps=3):
    """Plain ECDSA over n signatures in one call (all valid, keys from a seed),
    device-resident inputs, CUDA events around `reps` calls."""
    rng = np.random.default_rng(n)
    sks = rng.integers(1, 255, (n, 32), dtype=np.uint8)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_m, d_k = dev(msgs), dev(sks)
    d_p = torch.empty(n * 33, dtype=torch.uint8, device="cuda")
    d_s = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
    d_out = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    ctx.sign_device(0, d_m.data_ptr(), d_k.data_ptr(), 0, n, d_p.data_ptr(), d_s.data_ptr(), d_ok.data_ptr(),
                    st.cuda_stream)
    for _ in range(3):
        ctx.ecdsa_verify_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        ctx.ecdsa_verify_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    b.record(st)
    torch.cuda.synchronize()
    assert bool(d_out.all())
    return n * reps / (a.elapsed_time(b) * 1e-3)


def c1_corpus(n=4096, seed=4096):
    """The plain-ECDSA workload: private keys uniform in [1, n-1] from a seed
    (rejection sampling), 33-byte compressed keys, uniform 32-byte message
    hashes, RFC 6979 low-S signatures from the reference's own CPU signer
    (oracle/_ref), 10% tampered: one uniformly random bit flipped in the
    message, r or s (the field chosen uniformly).  Returns the arrays and the
    verdict each item must get by construction."""
    from oracle import RefDriver
    rng = np.random.default_rng(seed)
    sks = np.zeros((n, 32), np.uint8)
    for i in range(n):
        while True:
            k = rng.integers(0, 256, 32, dtype=np.uint8)
            if 0 < int.from_bytes(k.tobytes(), "big") < N_ORDER:
                sks[i] = k
                break
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    drv = RefDriver()
    pubs, sigs, ok = drv.sign(0, msgs, sks, None, os.cpu_count() or 1)
    assert ok.all()
    expect = np.ones(n, np.uint8)
    for i in rng.choice(n, size=n // 10, replace=False):
        field = int(rng.integers(0, 3))
        bit = int(rng.integers(0, 256))
        if field == 0:
            msgs[i, bit // 8] ^= 1 << (bit % 8)
        else:
            sigs[i, 32 * (field - 1) + bit // 8] ^= 1 << (bit % 8)
        expect[i] = 0
    return np.ascontiguousarray(msgs), np.ascontiguousarray(pubs), np.ascontiguousarray(sigs), expect


def bench_c1(ctx, torch, reps=50):
    """Plain ECDSA, 4096 signatures in one call (the workload above).  value:
    inputs on the device, CUDA events around `reps` back-to-back calls; e2e:
    ufsecp_gpu_ecdsa_verify_batch with host buffers, wall clock around `reps`
    synchronous calls (copies in and out inside); verdicts of every item against
    the reference library and the construction."""
    import time as _t
    from oracle import RefDriver
    msgs, pubs, sigs, expect = c1_corpus()
    n = len(msgs)
    ref = RefDriver().verify(0, msgs, pubs, sigs, os.cpu_count() or 1)
    dev = lambda a: torch.from_numpy(a.reshape(-1)).cuda()
    d_m, d_p, d_s = dev(msgs), dev(pubs), dev(sigs)
    d_out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(3):
        ctx.ecdsa_verify_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        ctx.ecdsa_verify_device(d_m.data_ptr(), d_p.data_ptr(), d_s.data_ptr(), n, d_out.data_ptr(), st.cuda_stream)
    b.record(st)
    torch.cuda.synchronize()
    value = n * reps / (a.elapsed_time(b) * 1e-3)
    dev_verdicts = d_out.cpu().numpy()
    for _ in range(3):
        ctx.ecdsa_verify_batch(msgs, pubs, sigs)
    t0 = _t.perf_counter()
    for _ in range(reps):
        host_verdicts = ctx.ecdsa_verify_batch(msgs, pubs, sigs)
    e2e = n * reps / (_t.perf_counter() - t0)
    return {"workload": "plain ECDSA, 4096 signatures per call: keys uniform in [1, n-1] from a seed, compressed keys, "
                        "uniform message hashes, RFC 6979 low-S signatures from the reference's CPU signer, 10% "
                        "tampered (one bit of the message, r or s)",
            "value_sigs_per_s": value, "value": "ufsecp_gpu_ext_ecdsa_verify_device, inputs on the device, CUDA events, "
                                                f"{reps} calls",
            "e2e_sigs_per_s": e2e, "e2e": f"ufsecp_gpu_ecdsa_verify_batch, host buffers, wall clock, {reps} calls",
            "e2e_ms_per_call": n / e2e * 1e3,
            "verdict_agreement": {"reference_library_device": float((dev_verdicts == ref).mean()),
                                  "reference_library_e2e": float((host_verdicts == ref).mean()),
                                  "construction": float((host_verdicts == expect).mean())},
            "valid": int(ref.sum())}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
