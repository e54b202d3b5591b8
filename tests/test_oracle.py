"""The checker itself: the C restatement against the reference's golden
vectors and, where it is built, against the reference compiled from its own
sources.  CPU only."""
import numpy as np
import pytest

import oracle
from helpers import golden_llr, sha

NORMAL_S2 = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10"]
SHORT_S2 = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9"]


def test_golden_cases_restatement(golden):
    """The restatement reproduces every golden case of the reference:
    per-frame bits, iterations and flags, and the batch return value."""
    for c in golden:
        llr = golden_llr(c)
        code = oracle.OrcCode(c["short"], c["rate"], c["kldpc"])
        bits, it, ok = code.decode_frames(llr, c["max_iter"])
        assert [sha(bits[f]) for f in range(c["frames"])] == c["frame_bits_sha256"], c["rate"]
        assert it.tolist() == c["frame_iterations"], c["rate"]
        assert ok.tolist() == c["frame_ok"], c["rate"]
        gbits, gret = code.decode_group(llr, c["max_iter"])
        assert gret == c["batch_return"], c["rate"]
        assert sha(gbits) == c["batch_bits_sha256"], c["rate"]


@pytest.mark.parametrize("short,rates", [(0, NORMAL_S2), (1, SHORT_S2)])
def test_encoder_zero_iterations(short, rates):
    """A noiseless encoded frame satisfies every check: 0 iterations."""
    rng = np.random.default_rng(5)
    for rate in rates:
        code = oracle.OrcCode(short, rate)
        info = rng.integers(0, 2, size=(1, code.K), dtype=np.uint8)
        llr = np.where(code.encode(info) == 0, 100, -100).astype(np.int8)
        bits, it, ok = code.decode_frames(llr, 10)
        assert it[0] == 0 and ok[0] == 1, rate
        assert (bits[0] == np.packbits(info[0, : code.kldpc])[: code.nbytes]).all()


def test_all_rates_compile():
    """Every rate string of the tables builds a code (normal and short maps)."""
    for short, rates in ((0, NORMAL_S2 + ["13_45", "154_180", "2_9_VLSNR", "2_3_t2"]),
                         (1, SHORT_S2 + ["11_45", "32_45", "1_5_VLSNR_SF2", "3_5_t2"])):
        for rate in rates:
            code = oracle.OrcCode(short, rate)
            assert code.N == (16200 if short else 64800)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")


@needs_ref
@pytest.mark.parametrize("short", [0, 1])
def test_restatement_matches_reference(short):
    """Seeded AWGN frames on every DVB-S2 rate: identical per-frame and batch
    results from the restatement and the reference build."""
    from helpers import awgn_frames
    rates = NORMAL_S2 if not short else SHORT_S2
    snr = {"1_4": -1.0, "1_3": 0.0, "2_5": 0.5, "1_2": 1.6, "3_5": 2.8, "2_3": 3.6, "3_4": 4.4,
           "4_5": 5.0, "5_6": 5.6, "8_9": 6.8, "9_10": 7.2}
    n = 2 if not short else 6
    for k, rate in enumerate(rates):
        llr = awgn_frames(short, rate, n, snr[rate], seed=1000 + k)
        ref = oracle.RefCode(short, rate)
        orc = oracle.OrcCode(short, rate)
        b1, i1, o1 = ref.decode_frames(llr, 25)
        b2, i2, o2 = orc.decode_frames(llr, 25)
        assert (b1 == b2).all() and (i1 == i2).all() and (o1 == o2).all(), rate
        g1, r1 = ref.decode_call(llr, 25)
        g2, r2 = orc.decode_group(llr, 25)
        assert r1 == r2 and (g1 == g2).all(), rate


@needs_ref
def test_reference_flavours_agree():
    """The reference's SIMD builds give the same results (its own claim,
    doc/optimisation/README.md:85-86): the checker does not depend on the
    host's ISA."""
    from helpers import awgn_frames
    llr = awgn_frames(1, "1_2", 8, 1.5, seed=77)
    outs = []
    for fl in ("avx2", "sse2") + (("avx512",) if oracle.best_ref_flavour() == "avx512" else ()):
        if not oracle.ref_available(fl):
            continue
        outs.append(oracle.RefCode(1, "1_2", fl).decode_frames(llr, 30))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert (a == b).all()


@needs_ref
def test_demapper_matches_reference():
    """The test channel's max-log demapper against the reference's
    drx_demap_frame on the same symbols (8PSK 3/5): equal up to one unit of
    float rounding at .5 boundaries."""
    import ctypes
    from oracle import datagen
    lib = oracle.load_ref()
    d = lib.ref_demap_new(b"8PSK", b"3_5", 0)
    nsym = lib.ref_demap_symbols(d)
    code = oracle.OrcCode(0, "3_5")
    rng = np.random.default_rng(3)
    cw = code.encode(rng.integers(0, 2, size=(1, code.K), dtype=np.uint8))
    sym = datagen.modulate(cw, "8PSK", "3_5", 0)
    n0 = 10 ** (-6.0 / 10)
    y = (sym + (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0 / 2)).astype(np.complex64)
    mine = datagen.demap(y, n0, "8PSK", "3_5", 0, code.N)[0]
    iq = np.empty(2 * nsym, np.float32)
    iq[0::2], iq[1::2] = y[0].real, y[0].imag
    theirs = np.empty(code.N, np.int8)
    lib.ref_demap_frame(d, iq.ctypes.data, ctypes.c_float(n0), theirs.ctypes.data)
    lib.ref_demap_free(d)
    diff = np.abs(mine.astype(int) - theirs.astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() > 0.99


def test_learned_model_unit_table_is_plain():
    """The CPU model of the learned int8 decoder with scale 1 and offset 1
    in every class and iteration is the plain decoder, bit for bit."""
    code = oracle.OrcCode(1, "1_2")
    fr = oracle.datagen.make_frames(1, "1_2", 24, 1.4, seed=21, code=code)
    cls = np.zeros(33, np.int8)
    ones = np.ones((50, 1), np.float32)
    want = code.decode_frames(fr["llr"], 50)
    got = code.decode_frames_learned(fr["llr"], 50, ones[:32], ones[:32], cls)
    for w, g in zip(want, got):
        assert np.array_equal(w, g)


def test_learned_words_rounding():
    """Q8 words: round half to even, clamped scale and offset."""
    w = oracle.learned_words([[1.0, 0.5 / 256, 300.0, -1.0]], [[1.0, -0.5, 200.0, -200.0]])
    assert w.shape == (1, 8)
    assert w[0, 0] == (256 | 256 << 16)
    assert w[0, 1] & 0xFFFF == 0 and (w[0, 1] >> 16) == (0x10000 - 128)  # 0.5 -> 0 (half-even), -0.5 -> -128
    assert w[0, 2] & 0xFFFF == 65535 and (w[0, 2] >> 16) == 32767
    assert w[0, 3] & 0xFFFF == 0 and (w[0, 3] >> 16) == 0x8000


@needs_ref
@pytest.mark.parametrize("short,rates", [(0, ["1_4", "3_5", "9_10"]), (1, ["1_4", "1_2", "8_9"])])
def test_bch_encoder_matches_reference_decoder(short, rates):
    """The oracle's BCH encoder (both fields, every t) makes words the
    reference's bch.c accepts with no correction; with t errors planted it
    corrects exactly t bits back to the codeword, and with t + 1 it never
    returns the codeword."""
    rng = np.random.default_rng(17 + short)
    for rate in rates:
        p = oracle.fec_params(short, rate)
        msgs = np.packbits(rng.integers(0, 2, (3, p.kbch), dtype=np.uint8), axis=1)
        cw = oracle.bch_encode(short, rate, msgs)
        assert np.array_equal(np.unpackbits(cw, axis=1)[:, : p.kbch], np.unpackbits(msgs, axis=1)[:, : p.kbch])
        ref = oracle.RefBch(short, rate)
        w, r = ref.decode(cw)
        assert (r == 0).all() and np.array_equal(w, cw), rate
        for wgt in (p.t, p.t + 1):
            bad = cw.copy()
            for f in range(bad.shape[0]):
                for b in rng.choice(p.kldpc, wgt, replace=False):
                    bad[f, b // 8] ^= 0x80 >> (b % 8)
            w, r = ref.decode(bad)
            if wgt == p.t:
                assert (r == p.t).all() and np.array_equal(w, cw), rate
            else:
                assert not any(np.array_equal(w[f], cw[f]) for f in range(w.shape[0])), rate
