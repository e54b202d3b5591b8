"""The headline workload checked against the reference at its full size.

DVB-S2 normal 3/5, 8PSK over AWGN, Es/N0 5.0 - 6.5 dB in 0.25 dB steps,
4096 frames per point (28,672 frames), at most 30 iterations: the very
batches `bench.py` times (the same generator and seeds), decoded by the
GPU with per-frame stopping, and every frame compared bit for bit with the
reference decoder compiled from its own sources, called once per frame
(nframes = 1, the reference's per-frame semantics: ldpc.c:614-638): hard
bits, iteration count and syndrome flag.  The reference calls run on every
host core, one decoder handle per thread (oracle/refbench.c).

Then one 4096-frame batch of the bench's frames (half from the 5.0 dB
point, half from the 6.5 dB one, so that groups both fail and pass) with
group stopping in groups of 64 frames (the reference's batch semantics,
drx_ldpc_decode on 64 lanes: tests/test_ldpc.c:78-94 decodes that way)
against one reference call per group: hard bits and each group's return
value.
"""
import numpy as np
import pytest

import bench
import dvbrx_b200 as D
import oracle

pytestmark = pytest.mark.gpu

FRAMES = 4096


@pytest.fixture(scope="module")
def dec():
    d = D.Ldpc(D.fec_lookup(bench.SHORT, bench.RATE), bench.RATE)
    yield d
    d.close()


def bench_batch(dec, k):
    """Es/N0 point k of the bench (rank 0): device LLRs and info bits."""
    return dec.generate(FRAMES, bench.ESN0[k], seed=bench.rank_seed(0, k), constellation=bench.CONST, info=True)


@pytest.mark.skipif(not oracle.ref_available("avx2"), reason="reference build missing")
@pytest.mark.parametrize("k", range(len(bench.ESN0)))
def test_bench_batch_per_frame_vs_reference(dec, k):
    import torch

    llr, info, _ = bench_batch(dec, k)
    bits, it, ok = (t.cpu().numpy() for t in dec.decode_device(llr, bench.MAX_ITER))
    torch.cuda.synchronize()
    assert dec.device_error() == 0
    host = llr.cpu().numpy()
    # the 32-lane build: a one-frame call pads half as many lanes as the 64-lane one
    ref = oracle.RefCode(bench.SHORT, bench.RATE, flavour="avx2")
    rb, ri, ro = ref.decode_frames_mt(host, bench.MAX_ITER)
    bad = np.nonzero((bits != rb).any(axis=1) | (it != ri) | (ok != ro))[0]
    assert bad.size == 0, "Es/N0 %.2f dB: %d of %d frames differ (first %s)" % (
        bench.ESN0[k], bad.size, FRAMES, bad[:8].tolist())
    # the sweep spans the waterfall: failing and converging frames alike
    fer = float((bits != info.cpu().numpy()).any(axis=1).mean())
    print("Es/N0 %.2f dB: %d frames bit-exact, FER %.4f, mean iterations %.2f"
          % (bench.ESN0[k], FRAMES, fer, float(it.mean())))


@pytest.mark.skipif(not oracle.ref_available("avx512"), reason="64-lane reference build missing")
def test_bench_batch_group64_vs_reference(dec):
    # the waterfall is steep: every 64-frame group of the 5.0 dB batch fails and every one of the
    # 6.5 dB batch passes, so the batch takes half of each (4096 frames, 64 groups of both kinds)
    lo, _, _ = bench_batch(dec, 0)
    hi, _, _ = bench_batch(dec, len(bench.ESN0) - 1)
    host = np.concatenate([lo[: FRAMES // 2].cpu().numpy(), hi[: FRAMES // 2].cpu().numpy()])
    bits, it, ok = dec.decode_host(host, bench.MAX_ITER, stop=64)
    ref = oracle.RefCode(bench.SHORT, bench.RATE, flavour="avx512")
    assert ref.lanes == 64
    rb, rets = ref.decode_groups_mt(host, bench.MAX_ITER, group=64)
    gpu_rets = np.array([int(it[g]) if ok[g:g + 64].all() else -1 for g in range(0, FRAMES, 64)])
    assert np.array_equal(gpu_rets, rets)
    assert np.array_equal(bits, rb)
    assert (rets >= 0).any() and (rets < 0).any(), "the batch should hold passing and failing groups"
