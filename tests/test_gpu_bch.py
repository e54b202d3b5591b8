"""The GPU BCH decoder (drx_bch_*) against the reference's bch.c compiled
from its sources: identical corrected words and return values (corrected
bit count or -1) for every DVB-S2 code, error weights 0 .. t + 3, random
words, and behind the LDPC decoder on the device."""
import zlib

import numpy as np
import pytest
import torch

import dvbrx_b200 as D
import oracle

pytestmark = pytest.mark.gpu

NORMAL = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10"]
SHORT = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9"]


def words_with_errors(short, rate, seed, per_weight=3):
    p = oracle.fec_params(short, rate)
    rng = np.random.default_rng(seed)
    weights = [0, 1, 2, p.t // 2, p.t - 1, p.t, p.t + 1, p.t + 2, p.t + 3]
    msgs = np.packbits(rng.integers(0, 2, (len(weights) * per_weight, p.kbch), dtype=np.uint8), axis=1)
    cw = oracle.bch_encode(short, rate, msgs)
    k = 0
    for wgt in weights:
        for _ in range(per_weight):
            for b in rng.choice(p.kldpc, wgt, replace=False):
                cw[k, b // 8] ^= 0x80 >> (b % 8)
            k += 1
    garbage = rng.integers(0, 256, (4, p.kldpc // 8), dtype=np.uint8)
    return np.concatenate([cw, garbage])


@pytest.mark.parametrize("short,rate", [(0, r) for r in NORMAL] + [(1, r) for r in SHORT])
def test_bch_matches_reference(short, rate):
    words = words_with_errors(short, rate, seed=zlib.crc32(("%d%s" % (short, rate)).encode()) % 1000)
    want_w, want_r = oracle.RefBch(short, rate).decode(words)
    bch = D.Bch(D.fec_lookup(short, rate))
    dev = torch.from_numpy(words).cuda()
    res = bch.decode_device(dev)
    torch.cuda.synchronize()
    assert np.array_equal(res.cpu().numpy(), want_r), (rate, res.cpu().numpy(), want_r)
    assert np.array_equal(dev.cpu().numpy(), want_w), rate
    assert (want_r == 0).any() and (want_r > 0).any() and (want_r < 0).any()


def test_bch_single_word_dropin():
    short, rate = 0, "3_5"
    words = words_with_errors(short, rate, seed=7, per_weight=1)
    want_w, want_r = oracle.RefBch(short, rate).decode(words)
    bch = D.Bch(D.fec_lookup(short, rate))
    for f in range(words.shape[0]):
        w = words[f].copy()
        assert bch.decode(w) == want_r[f]
        assert np.array_equal(w, want_w[f])


def test_bch_after_ldpc_on_device():
    """LDPC hard bits straight into the BCH decoder on the same stream,
    against the reference BCH on the same bits (the generator's information
    bits are random words, so BCH sees arbitrary codewords)."""
    short, rate = 1, "1_2"
    p = D.fec_lookup(short, rate)
    dec = D.Ldpc(p, rate)
    llr, _, _ = dec.generate(300, 1.2, seed=3)
    bits, _, _ = dec.decode_device(llr, 50)
    host = bits.cpu().numpy().copy()
    res = D.Bch(p).decode_device(bits)
    torch.cuda.synchronize()
    want_w, want_r = oracle.RefBch(short, rate).decode(host)
    assert np.array_equal(res.cpu().numpy(), want_r)
    assert np.array_equal(bits.cpu().numpy(), want_w)


@pytest.mark.parametrize("short,rate", [(0, "1_4"), (0, "2_3"), (0, "9_10"), (1, "1_2"), (1, "8_9")])
def test_bch_encoder_matches_oracle(short, rate):
    p = D.fec_lookup(short, rate)
    rng = np.random.default_rng(5)
    msgs = np.packbits(rng.integers(0, 2, (16, p.kbch), dtype=np.uint8), axis=1)
    want = oracle.bch_encode(short, rate, msgs)
    dev = torch.zeros((16, p.kldpc // 8), dtype=torch.uint8, device="cuda")
    dev[:, : msgs.shape[1]] = torch.from_numpy(msgs).cuda()
    D.Bch(p).encode_device(dev)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), want)
