"""Decoder cost per code: microseconds of the whole GPU per frame-iteration,
for the frame-pair kernel and the one-frame kernel.

    python -m dvbrx_b200.ratebench [--rates 3_5 4_5 ...] [--short]

Each code decodes several full waves of frames (6 per SM for normal frames,
24 for short ones: every CTA of either kernel busy) generated far below its
threshold, so that no frame converges and every frame runs its iterations;
the cost per iteration is the difference between a 30- and a 10-iteration
launch over 20, timed with CUDA events (best of five).
"""
import argparse

import dvbrx_b200 as D

NORMAL = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10"]


def frame_iteration_us(dec, variant, n, seed=7):
    import torch

    dec.set_variant(variant)
    llr, _, _ = dec.generate(n, -6.0, seed=seed)
    t = {}
    for it in (10, 30):
        best = float("inf")
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            _, _, ok = dec.decode_device(llr, it)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        t[it] = best
    assert int(ok.sum()) == 0, "a frame converged: the case must stay below threshold"
    return (t[30] - t[10]) / 20 * 1e3 / n


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", nargs="*", default=NORMAL)
    ap.add_argument("--short", action="store_true")
    a = ap.parse_args()
    n = (24 if a.short else 6) * torch.cuda.get_device_properties(0).multi_processor_count
    print("%-6s %-6s %12s %12s %8s" % ("frame", "rate", "pair us", "frame us", "ratio"))
    for rate in a.rates:
        if a.short and rate == "9_10":
            continue
        dec = D.Ldpc(D.fec_lookup(int(a.short), rate), rate)
        pair = frame_iteration_us(dec, D.VARIANT_PAIR, n)
        one = frame_iteration_us(dec, D.VARIANT_FRAME, n)
        print("%-6s %-6s %12.3f %12.3f %8.2f" % ("short" if a.short else "normal", rate, pair, one, one / pair))
        dec.close()


if __name__ == "__main__":
    main()
