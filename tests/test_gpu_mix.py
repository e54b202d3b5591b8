"""Mixed batches (several MODCODs, normal and short frames, one batch) through
drx_ldpc_mix_*: every tiling, and the autotuner's choice, give the results
of one-code decodes, which are themselves bit-exact to the reference."""
import numpy as np
import pytest

import dvbrx_b200 as D
from helpers import check_frames, checker

pytestmark = pytest.mark.gpu

# (short, rate, constellation, Es/N0): all kernel classes, levelled and not
CODES = [
    (0, "3_5", "8PSK", 6.0),
    (0, "2_3", "8PSK", 6.8),
    (1, "1_2", "QPSK", 1.6),
    (0, "9_10", "QPSK", 7.0),   # degree 30: 16-byte message records
    (1, "8_9", "QPSK", 6.9),    # degree 27, shared links up to slot 13
    (0, "13_45", "QPSK", -0.6),
    (1, "11_45", "QPSK", 0.2),
]


def make_batch(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    code = rng.integers(0, len(CODES), size=n).astype(np.int32)
    llr = torch.zeros((n, 64800), dtype=torch.int8, device="cuda")
    handles = []
    for c, (short, rate, const, es) in enumerate(CODES):
        h = D.Ldpc(D.fec_lookup(short, rate), rate)
        handles.append(h)
        rows = np.nonzero(code == c)[0]
        if len(rows):
            l, _, _ = h.generate(len(rows), es, seed=seed * 100 + c, constellation=const)
            llr[torch.from_numpy(rows).cuda().long(), : h.N] = l
    return code, llr, handles


def test_mixed_batch_tilings_and_tuner():
    import torch
    n = 700
    code, llr, handles = make_batch(n, 3)
    mix = D.LdpcMix([(s, r) for s, r, _, _ in CODES])
    out = torch.zeros((n, 7290), dtype=torch.uint8, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    mix.plan(code, llr, out, it, ok, 30)

    # expected: each code's frames decoded on their own
    want_bits = {}
    want_it = np.zeros(n, np.int32)
    want_ok = np.zeros(n, np.uint8)
    for c, h in enumerate(handles):
        rows = np.nonzero(code == c)[0]
        if not len(rows):
            continue
        sub = llr[torch.from_numpy(rows).cuda().long(), : h.N].contiguous()
        b, i, o = h.decode_device(sub, 30)
        torch.cuda.synchronize()
        want_bits[c] = (rows, b.cpu().numpy())
        want_it[rows] = i.cpu().numpy()
        want_ok[rows] = o.cpu().numpy()

    def check():
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for c, (rows, b) in want_bits.items():
            nb = handles[c].nbytes
            assert (got[rows, :nb] == b).all(), CODES[c]
        assert (it.cpu().numpy() == want_it).all()
        assert (ok.cpu().numpy() == want_ok).all()

    for tiling in (D.TILING_ONE_LAUNCH, D.TILING_PER_CODE):
        out.zero_()
        it.fill_(-1)
        mix.set_tiling(tiling)
        mix.run()
        check()
    # S2X codes have no shape in the two-frames-per-CTA one-launch kernel: the plan lacks that tiling
    with pytest.raises(ValueError):
        mix.set_tiling(D.TILING_ONE_LAUNCH_PAIR)
    assert mix.tuned_ms(D.TILING_ONE_LAUNCH_PAIR) is None
    choice, t1, t2 = mix.tune()
    assert choice in (D.TILING_ONE_LAUNCH, D.TILING_PER_CODE) and t1 > 0 and t2 > 0
    out.zero_()
    mix.run()
    check()

    # a sample of frames against the reference decoder itself
    for c, (short, rate, _, _) in enumerate(CODES[:3]):
        rows = np.nonzero(code == c)[0][:3]
        h = handles[c]
        host = llr[torch.from_numpy(rows).cuda().long(), : h.N].cpu().numpy()
        rb, ri, ro = check_frames(checker(short, rate), host, 30)
        assert (out.cpu().numpy()[rows, : h.nbytes] == rb).all()
        assert (it.cpu().numpy()[rows] == ri).all()
    mix.close()


def test_mixed_batch_learned_with_fallback():
    """drx_ldpc_mix_plan_learned: every row equals its code's own learned
    decode with fallback (drx_ldpc_decode_learned_device), in both tilings."""
    import torch

    from dvbrx_b200 import learned as Lm

    n = 500
    code, llr, handles = make_batch(n, 5)
    mix = D.LdpcMix([(s, r) for s, r, _, _ in CODES])
    L = 8
    for c, (short, rate, _, _) in enumerate(CODES):
        degs, cod = Lm.degree_classes(short, rate)
        rng = np.random.default_rng(c)
        scale = rng.uniform(0.8, 1.0, size=(L, len(degs)))
        offset = rng.uniform(0.0, 1.0, size=(L, len(degs)))
        mix.set_learned(c, scale, offset, cod)
        handles[c].set_learned(scale, offset, cod)
    out = torch.zeros((n, 7290), dtype=torch.uint8, device="cuda")
    it = torch.zeros(n, dtype=torch.int32, device="cuda")
    ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
    fb = torch.zeros(n, dtype=torch.uint8, device="cuda")
    mix.plan_learned(code, llr, out, it, ok, fb, L, 30)

    want = {}
    for c, h in enumerate(handles):
        rows = np.nonzero(code == c)[0]
        if not len(rows):
            continue
        sub = llr[torch.from_numpy(rows).cuda().long(), : h.N].contiguous()
        b, i, o, f = h.decode_learned(sub, L, 30)
        torch.cuda.synchronize()
        want[c] = (rows, b.cpu().numpy(), i.cpu().numpy(), o.cpu().numpy(), f.cpu().numpy())
    nfb = sum(int(w[4].sum()) for w in want.values())
    assert 0 < nfb < n, "the batch should mix learned successes and fallbacks"
    for tiling in (D.TILING_ONE_LAUNCH, D.TILING_PER_CODE):
        out.zero_()
        it.fill_(-1)
        fb.fill_(7)
        mix.set_tiling(tiling)
        mix.run()
        torch.cuda.synchronize()
        got_b, got_i, got_o, got_f = out.cpu().numpy(), it.cpu().numpy(), ok.cpu().numpy(), fb.cpu().numpy()
        for c, (rows, b, i, o, f) in want.items():
            nb = handles[c].nbytes
            assert (got_b[rows, :nb] == b).all(), (CODES[c], tiling)
            assert (got_i[rows] == i).all(), (CODES[c], tiling)
            assert (got_o[rows] == o).all(), (CODES[c], tiling)
            assert (got_f[rows] == f).all(), (CODES[c], tiling)


# DVB-S2 codes of every shape of the two-frames-per-CTA one-launch kernel
S2_CODES = [(0, r, "QPSK", es) for r, es in (("1_4", -1.9), ("1_3", -0.9), ("2_5", -0.1), ("1_2", 1.2),
                                               ("3_5", 2.4), ("2_3", 3.3), ("3_4", 4.2), ("4_5", 4.8),
                                               ("5_6", 5.3), ("8_9", 6.5), ("9_10", 6.8))] + \
           [(1, r, "QPSK", es) for r, es in (("1_4", -1.2), ("1_2", 1.8), ("3_5", 2.9), ("2_3", 3.8),
                                               ("3_4", 4.6), ("5_6", 5.8), ("8_9", 6.9))]


def test_mixed_batch_one_launch_two_frames_per_cta():
    """The one-launch tiling with two frames per CTA (CTAs taking one code at
    a time, moving to the code with the most work left) gives the per-code
    results exactly, and the tuner times all three tilings."""
    import torch
    n = 900
    rng = np.random.default_rng(11)
    code = rng.integers(0, len(S2_CODES), size=n).astype(np.int32)
    llr = torch.zeros((n, 64800), dtype=torch.int8, device="cuda")
    for c, (short, rate, const, es) in enumerate(S2_CODES):
        rows = np.nonzero(code == c)[0]
        if len(rows):
            h = D.Ldpc(D.fec_lookup(short, rate), rate)
            l, _, _ = h.generate(len(rows), es, seed=700 + c, constellation=const)
            llr[torch.from_numpy(rows).cuda().long(), : h.N] = l
            h.close()
    mix = D.LdpcMix([(s, r) for s, r, _, _ in S2_CODES])
    res = {}
    out = torch.zeros((n, 7290), dtype=torch.uint8, device="cuda")
    it = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    ok = torch.full((n,), 9, dtype=torch.uint8, device="cuda")
    mix.plan(code, llr, out, it, ok, 30)
    for tiling in (D.TILING_PER_CODE, D.TILING_ONE_LAUNCH_PAIR, D.TILING_ONE_LAUNCH):
        out.zero_()
        it.fill_(-1)
        ok.fill_(9)
        mix.set_tiling(tiling)
        mix.run()
        torch.cuda.synchronize()
        res[tiling] = (out.cpu().numpy(), it.cpu().numpy(), ok.cpu().numpy())
    for a, b in zip(res[D.TILING_PER_CODE], res[D.TILING_ONE_LAUNCH_PAIR]):
        assert np.array_equal(a, b)
    for a, b in zip(res[D.TILING_PER_CODE], res[D.TILING_ONE_LAUNCH]):
        assert np.array_equal(a, b)
    its = res[D.TILING_PER_CODE][1]
    assert its.min() < its.max() and 0 < res[D.TILING_PER_CODE][2].sum() < n, "uneven iterations expected"
    choice, t1, t2 = mix.tune()
    t3 = mix.tuned_ms(D.TILING_ONE_LAUNCH_PAIR)
    assert t1 > 0 and t2 > 0 and t3 is not None and t3 > 0
    assert choice in (D.TILING_ONE_LAUNCH, D.TILING_PER_CODE, D.TILING_ONE_LAUNCH_PAIR)
    mix.close()
