"""Small, self-checking GPU cases to run under a profiler.

    python -m ultrafastsecp256k1_b200.profile_cases verify [--n N] [--reps R]
    python -m ultrafastsecp256k1_b200.profile_cases rlc    [--n N] [--batch B] [--reps R] [--warmup W] [--one-per-batch]
    python -m ultrafastsecp256k1_b200.profile_cases queue  [--n N] [--reps R]

Each case signs its own seeded BIP-340 / ECDSA corpus on the GPU, runs the
named path R times on device-resident inputs (the plain per-signature kernel,
the RLC batch verifier, or the mixed-job work-queue kernel), checks every
verdict against the construction (valid signatures, plus one flipped bit in a
known set) and prints one line of timings.  The cases hold well under 1 GB on
the device, so a profiler capture of them stays small.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

import ultrafastsecp256k1_b200 as uf

N_ORDER = 0xFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFFEBAAEDCE6AF48A03BBFD25E8CD0364141


def _keys(rng, n):
    sks = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    sks[:, 0] &= 0x7F          # below n by construction
    sks[:, 31] |= 1            # never zero
    return sks


def _signed(ctx, torch, kind, n, seed, n_bad, bad_idx=None):
    rng = np.random.default_rng(seed)
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    aux = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_m, d_k, d_a = dev(msgs), dev(_keys(rng, n)), dev(aux)
    ps = 33 if kind == 0 else 32
    d_p = torch.empty(n * ps, dtype=torch.uint8, device="cuda")
    d_s = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    d_ok = torch.empty(n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.sign_device(kind, d_m.data_ptr(), d_k.data_ptr(), d_a.data_ptr(), n, d_p.data_ptr(), d_s.data_ptr(),
                    d_ok.data_ptr(), 0)
    torch.cuda.ExternalStream(ctx.stream()).synchronize()
    assert bool(d_ok.all())
    sigs = d_s.cpu().numpy().reshape(n, 64)
    expect = np.ones(n, np.uint8)
    bad = np.asarray(bad_idx) if bad_idx is not None else rng.choice(n, size=n_bad, replace=False)
    for i in bad:
        sigs[i, 40] ^= 0x04
    expect[bad] = 0
    return d_m, d_p, dev(sigs), expect, (msgs, d_p.cpu().numpy().reshape(n, ps), sigs)


def case_verify(ctx, torch, a):
    d_m, d_x, d_s, expect, _ = _signed(ctx, torch, 1, a.n, 1, a.n // 100)
    d_o = torch.zeros(a.n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(st)
    for _ in range(a.reps):
        ctx.schnorr_verify_device(d_m.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), a.n, d_o.data_ptr(), st.cuda_stream)
    ev[1].record(st)
    torch.cuda.synchronize()
    assert (d_o.cpu().numpy() == expect).all()
    ms = ev[0].elapsed_time(ev[1]) / a.reps
    print(f"verify n={a.n} ms/launch={ms:.3f} sigs/s={a.n / ms * 1e3:.4g}")


def case_rlc(ctx, torch, a):
    if a.one_per_batch:
        # exactly one invalid signature in every batch, at a seeded position
        rng = np.random.default_rng(65)
        bad_idx = [b + int(rng.integers(0, min(a.batch, a.n - b))) for b in range(0, a.n, a.batch)]
        n_bad = len(bad_idx)
    else:
        bad_idx = None
        n_bad = (a.n // a.batch) // a.bad_every if a.bad_every else 0
    d_m, d_x, d_s, expect, _ = _signed(ctx, torch, 1, a.n, 2, n_bad, bad_idx)
    d_o = torch.zeros(a.n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    for k in range(a.warmup):
        ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), a.n, d_o.data_ptr(),
                                      batch_size=a.batch, seed32=bytes([255 - k]) * 32, stream=st.cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(a.reps):
        ctx.schnorr_verify_rlc_device(d_m.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), a.n, d_o.data_ptr(),
                                      batch_size=a.batch, seed32=bytes([k]) * 32, stream=st.cuda_stream)
    dt = (time.perf_counter() - t0) / a.reps
    assert (d_o.cpu().numpy() == expect).all()
    print(f"rlc n={a.n} batch={a.batch} invalid={n_bad} ms/call={dt * 1e3:.3f} sigs/s={a.n / dt:.4g} "
          f"stats={ctx.rlc_stats()}")


def case_queue(ctx, torch, a):
    n_e, n_s = a.n * 3 // 10, a.n - a.n * 3 // 10
    *_, e_exp, e_host = _signed(ctx, torch, 0, n_e, 3, n_e // 200)
    *_, s_exp, s_host = _signed(ctx, torch, 1, n_s, 4, n_s // 200)
    jobs, exps = [], []
    rng = np.random.default_rng(5)
    oe = os_ = 0
    while oe < n_e or os_ < n_s:
        size = int(np.clip(np.exp(rng.uniform(0, np.log(8192))), 1, 8192))
        ke = min(int(size * 0.3), n_e - oe)
        ks = min(size - int(size * 0.3), n_s - os_)
        if ke:
            jobs.append((0,) + tuple(x[oe:oe + ke] for x in e_host))
            exps.append(e_exp[oe:oe + ke])
            oe += ke
        if ks:
            jobs.append((1,) + tuple(x[os_:os_ + ks] for x in s_host))
            exps.append(s_exp[os_:os_ + ks])
            os_ += ks
        if not ke and not ks:
            break
    t0 = time.perf_counter()
    for _ in range(a.reps):
        outs = ctx.verify_jobs(jobs)
    dt = (time.perf_counter() - t0) / a.reps
    assert all((o == e).all() for o, e in zip(outs, exps))
    print(f"queue n={a.n} jobs={len(jobs)} ms/call={dt * 1e3:.3f} sigs/s={a.n / dt:.4g}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["verify", "rlc", "queue"])
    ap.add_argument("--n", type=int, default=1 << 18)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=0, help="rlc: untimed calls before the timed ones")
    ap.add_argument("--bad-every", type=int, default=8, help="rlc: one invalid signature per this many batches (0: none)")
    ap.add_argument("--one-per-batch", action="store_true", help="rlc: exactly one invalid signature in every batch")
    a = ap.parse_args()
    import torch
    with uf.GpuContext(0) as ctx:
        {"verify": case_verify, "rlc": case_rlc, "queue": case_queue}[a.case](ctx, torch, a)


if __name__ == "__main__":
    main()
