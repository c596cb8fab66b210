"""Building-block throughput on the current GPU.

    python -m ultrafastsecp256k1_b200.perfprobe [variant ...]

Prints, per operation of the verify path, the device-wide rate (ops / s) and
the cost of one operation in field-multiplication equivalents, next to the
measured 32-bit IMAD issue rate.  Used to check the kernel design against the
integer-pipe roofline.
"""
import json
import sys

import ultrafastsecp256k1_b200 as uf

OPS = {1: ("fe_mul", 2), 2: ("fe_sqr", 2), 3: ("fe_inv", 1), 4: ("fe_sqrt", 1), 5: ("jac_dbl", 1),
       6: ("jac_add_aff", 1), 7: ("sc_inv", 1), 8: ("glv_split", 1), 9: ("bip340_challenge", 1)}
ITERS = {1: 2048, 2: 2048, 3: 16, 4: 4, 5: 512, 6: 512, 7: 16, 8: 64, 9: 128}


def main():
    variants = [int(v) for v in sys.argv[1:]] or [None]
    with uf.GpuContext(0) as ctx:
        props = ctx.device_props()
        sms = props["sm_count"]
        imad = ctx.imad_peak()
        result = {"sm_count": sms, "imad_ops_per_s": imad, "variants": {}}
        for variant in variants:
            if variant is not None:
                ctx.set_variant(1, variant)
            result["variants"][str(ctx.get_variant(1)[0])] = measure(ctx, sms, imad)
        json.dump(result, sys.stdout, indent=1)
        print()


def measure(ctx, sms, imad):
    if True:
        out = {"ops": {}}
        mul_rate = None
        for op, (name, per_iter) in OPS.items():
            best = None
            for threads, bps in ((128, 4), (256, 4), (128, 8), (256, 8)):
                blocks = sms * bps
                ms = ctx.probe(op, blocks, threads, ITERS[op])
                rate = blocks * threads * ITERS[op] * per_iter / (ms * 1e-3)
                if best is None or rate > best[0]:
                    best = (rate, threads, bps)
            rate, threads, bps = best
            if op == 1:
                mul_rate = rate
            out["ops"][name] = {"ops_per_s": rate, "threads": threads, "blocks_per_sm": bps,
                                "fe_mul_equiv": mul_rate / rate if mul_rate else None,
                                "imad_per_op_if_bound": imad / rate}
        return out


if __name__ == "__main__":
    main()
