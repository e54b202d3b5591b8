"""Parity of the sm_100a decoder with the reference, through the C ABI.

Bit-exact on every output: hard bits, per-frame iteration counts and syndrome
flags (per-frame stopping), and the reference's batch return value and bits
(group stopping and the drop-in drx_ldpc_decode)."""
import zlib

import numpy as np
import pytest

import dvbrx_b200 as D
from helpers import awgn_frames, check_frames, check_group, checker, golden_llr, sha

pytestmark = pytest.mark.gpu

_handles = {}


def fec_params(short, rate):
    try:
        return D.fec_lookup(short, rate)
    except KeyError:  # T2 codes: no BCH row, nbch = K
        info = D.code_info(short, rate)
        return D.FecParams(short, info.nldpc, info.K, info.K, 0)


def handle(short, rate, kldpc=None):
    key = (short, rate, kldpc)
    if key not in _handles:
        p = fec_params(short, rate)
        if kldpc is not None:
            p.kldpc = kldpc
        _handles[key] = D.Ldpc(p, rate)
    return _handles[key]


def test_golden_cases_per_frame(golden):
    for c in golden:
        llr = golden_llr(c)
        d = handle(c["short"], c["rate"], c["kldpc"])
        bits, it, ok = d.decode_host(llr, c["max_iter"])
        assert [sha(bits[f]) for f in range(c["frames"])] == c["frame_bits_sha256"], c["rate"]
        assert it.tolist() == c["frame_iterations"], c["rate"]
        assert ok.tolist() == c["frame_ok"], c["rate"]
        assert d.device_error() == 0


def test_golden_cases_group(golden):
    for c in golden:
        llr = golden_llr(c)
        d = handle(c["short"], c["rate"], c["kldpc"])
        bits, it, ok = d.decode_host(llr, c["max_iter"], stop=c["frames"])
        ret = int(it[0]) if ok.all() else -1
        assert ret == c["batch_return"], c["rate"]
        assert sha(bits) == c["batch_bits_sha256"], c["rate"]
        assert (it == it[0]).all() and (ok == ok[0]).all()


def test_golden_cases_dropin(golden):
    """drx_ldpc_decode itself: per-frame host pointers, reference return."""
    for c in golden:
        llr = golden_llr(c)
        d = handle(c["short"], c["rate"], c["kldpc"])
        rows = [np.ascontiguousarray(llr[f]) for f in range(c["frames"])]
        out = [np.zeros(d.nbytes, np.uint8) for _ in rows]
        ret = d.decode(rows, out, c["max_iter"])
        assert ret == c["batch_return"], c["rate"]
        assert sha(np.stack(out)) == c["batch_bits_sha256"], c["rate"]


def test_small_config_short_half_1024():
    """Short 1/2, QPSK, Es/N0 1.5 dB, 1024 frames, 50 iterations."""
    llr = awgn_frames(1, "1_2", 1024, 1.5, seed=2024)
    d = handle(1, "1_2")
    bits, it, ok = d.decode_host(llr, 50)
    rb, ri, ro = check_frames(checker(1, "1_2"), llr, 50)
    assert (bits == rb).all() and (it == ri).all() and (ok == ro).all()


@pytest.mark.parametrize("esn0", [5.0, 5.25, 5.5, 5.75, 6.0, 6.25, 6.5])
def test_normal_3_5_8psk_sweep(esn0):
    """Normal 3/5, 8PSK, the Es/N0 sweep, 30 iterations (sampled frames)."""
    llr = awgn_frames(0, "3_5", 12, esn0, seed=int(esn0 * 100), constellation="8PSK")
    d = handle(0, "3_5")
    bits, it, ok = d.decode_host(llr, 30)
    rb, ri, ro = check_frames(checker(0, "3_5"), llr, 30)
    assert (bits == rb).all() and (it == ri).all() and (ok == ro).all()


def test_normal_3_5_group_semantics():
    """128 frames in groups of the reference's lane count, reference batch
    semantics (each group's frames iterate until all pass)."""
    import oracle
    llr = awgn_frames(0, "3_5", 128, 5.9, seed=7, constellation="8PSK")
    chk = checker(0, "3_5")
    G = chk.lanes if isinstance(chk, oracle.RefCode) else 64
    d = handle(0, "3_5")
    bits, it, ok = d.decode_host(llr, 30, stop=G)
    for g0 in range(0, 128, G):
        rb, rr = check_group(chk, llr[g0:g0 + G], 30)
        ret = int(it[g0]) if ok[g0:g0 + G].all() else -1
        assert ret == rr and (bits[g0:g0 + G] == rb).all()


RATES = [(0, r) for r in ("1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10",
                          "2_9_VLSNR", "13_45", "9_20", "90_180", "11_20", "26_45", "28_45", "116_180",
                          "20_30", "22_30", "135_180", "7_9", "154_180", "2_3_t2")] + \
        [(1, r) for r in ("1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9",
                          "11_45", "4_15", "14_45", "7_15", "8_15", "26_45", "32_45", "1_5_VLSNR_SF2",
                          "3_5_t2")]

# Es/N0 near each code's waterfall (QPSK unless the MODCOD exists in 8PSK only)
SNR = {"1_4": -1.0, "1_3": 0.0, "2_5": 0.5, "1_2": 1.6, "3_5": 2.8, "2_3": 3.6, "3_4": 4.4, "4_5": 5.0,
       "5_6": 5.6, "8_9": 6.8, "9_10": 7.2}


@pytest.mark.parametrize("short,rate", RATES)
def test_every_rate(short, rate):
    import re
    if rate in SNR:
        es = SNR[rate]
    else:
        m = re.match(r"(\d+)_(\d+)", rate)
        r = int(m.group(1)) / int(m.group(2))
        es = 10 * np.log10(2 ** (2 * r) - 1) + 1.0
    n = 6 if short else 3
    llr = awgn_frames(short, rate, n, es, seed=zlib.crc32(rate.encode()) + short)
    d = handle(short, rate)
    chk = checker(short, rate)
    bits, it, ok = d.decode_host(llr, 20)
    rb, ri, ro = check_frames(chk, llr, 20)
    assert (bits == rb).all() and (it == ri).all() and (ok == ro).all()


@pytest.mark.parametrize("short,rate", [(1, "1_2"), (0, "3_5"), (1, "8_9"), (0, "9_10"), (0, "13_45")])
def test_uniform_random_llrs(short, rate):
    """Uniform int8 inputs, -128 included: the saturation corners."""
    N = 16200 if short else 64800
    llr = np.random.default_rng(11).integers(-128, 128, size=(4, N)).astype(np.int8)
    d = handle(short, rate)
    bits, it, ok = d.decode_host(llr, 4)
    rb, ri, ro = check_frames(checker(short, rate), llr, 4)
    assert (bits == rb).all() and (it == ri).all() and (ok == ro).all()


@pytest.mark.parametrize("short,rate,es,n,G", [(1, "1_2", 1.6, 37, 5), (1, "1_2", 1.6, 37, 1), (0, "9_10", 6.6, 11, 3),
                                             (0, "3_5", 5.8, 70, 64), (1, "8_9", 6.5, 20, 8)])
def test_group_stopping_pair_matches_frame(short, rate, es, n, G):
    """Group stopping on the frame-pair kernel (teams of ceil(G / 2) CTAs, an
    odd G leaving the last lane empty, a partial last group) gives the
    one-frame kernel's results, and the first group the reference's."""
    llr = awgn_frames(short, rate, n, es, seed=zlib.crc32(rate.encode()) + 31 * G)
    d = D.Ldpc(D.fec_lookup(short, rate), rate)
    res = {}
    for v in (D.VARIANT_FRAME, D.VARIANT_PAIR):
        assert d.set_variant(v) == v
        res[v] = d.decode_host(llr, 30, stop=G)
    for a, b in zip(res[D.VARIANT_FRAME], res[D.VARIANT_PAIR]):
        assert np.array_equal(a, b), (rate, G)
    bits, it, ok = res[D.VARIANT_PAIR]
    rb, rr = check_group(checker(short, rate), llr[:G], 30)
    assert (int(it[0]) if ok[:G].all() else -1) == rr and (bits[:G] == rb).all()
    d.close()


def test_edge_cases():
    d = handle(1, "1_2")
    N = 16200
    # max_iter 0: syndrome only
    llr = awgn_frames(1, "1_2", 4, 1.5, seed=3)
    bits, it, ok = d.decode_host(llr, 0)
    rb, ri, ro = check_frames(checker(1, "1_2"), llr, 0)
    assert (bits == rb).all() and (it == 0).all() and (ok == ro).all()
    # all-zero codeword at full confidence: passes at once
    bits, it, ok = d.decode_host(np.full((2, N), 127, np.int8), 10)
    assert (it == 0).all() and (ok == 1).all() and (bits == 0).all()
    # drop-in call limits (ldpc.c:620-621): more than 64 frames, no frames
    rows = [np.zeros(N, np.int8)] * 65
    out = [np.zeros(d.nbytes, np.uint8)] * 65
    assert d.decode(rows, out, 5) == -1
    assert d.decode([], [], 5) == 0


def test_device_batch_strided():
    """drx_ldpc_decode_device on padded rows gives the host call's results."""
    import torch
    llr = awgn_frames(1, "1_2", 32, 1.6, seed=9)
    d = handle(1, "1_2")
    ref = d.decode_host(llr, 30)
    big = np.zeros((32, 16200 + 64), np.int8)
    big[:, :16200] = llr
    t = torch.from_numpy(big).cuda()
    out = torch.zeros((32, d.nbytes + 16), dtype=torch.uint8, device="cuda")
    bits, it, ok = d.decode_device(t, 30, out=out[:, : d.nbytes])
    torch.cuda.synchronize()
    assert (out[:, : d.nbytes].cpu().numpy() == ref[0]).all()
    assert (it.cpu().numpy() == ref[1]).all() and (ok.cpu().numpy() == ref[2]).all()
    assert (out[:, d.nbytes:].cpu().numpy() == 0).all()


@pytest.mark.parametrize("short,rate,const,es,n,max_iter", [
    (1, "1_2", "QPSK", 1.5, 41, 50),
    (0, "3_5", "8PSK", 5.6, 17, 30),
    (0, "2_3", "8PSK", 6.4, 9, 20),
    (1, "3_5", "QPSK", 2.8, 33, 25),
    (0, "13_45", "QPSK", -0.8, 5, 30),
    (0, "1_4", "QPSK", -1.0, 5, 30),
    (1, "8_15", "QPSK", 2.4, 31, 30),
    (0, "3_5", "8PSK", 6.0, 3, 0),
    # check degrees above 16: 16-byte message records, four to six late slots
    (0, "4_5", "QPSK", 4.9, 7, 30),
    (0, "5_6", "QPSK", 5.4, 7, 30),
    (0, "8_9", "QPSK", 6.4, 5, 30),
    (0, "9_10", "QPSK", 6.6, 5, 30),
    (1, "5_6", "QPSK", 5.5, 13, 30),
    (1, "8_9", "QPSK", 6.6, 13, 30),
])
def test_kernel_variants_agree(short, rate, const, es, n, max_iter):
    """The one-frame kernel and the frame-pair kernel (odd frame counts leave
    a lane empty at the end) both reproduce the reference."""
    llr = awgn_frames(short, rate, n, es, seed=zlib.crc32(rate.encode()) + 17 * n, constellation=const)
    rb, ri, ro = check_frames(checker(short, rate), llr, max_iter)
    p = D.fec_lookup(short, rate)
    d = D.Ldpc(p, rate)
    for v in (D.VARIANT_FRAME, D.VARIANT_PAIR):
        assert d.set_variant(v) == v
        bits, it, ok = d.decode_host(llr, max_iter)
        assert (bits == rb).all() and (it == ri).all() and (ok == ro).all(), "variant %d" % v
    d.close()


def test_variant_auto_choice():
    """Every code, up to check degree 30 (normal 9/10), runs on the frame-pair
    kernel by default; the one-frame kernel can still be chosen."""
    for short, rate in ((0, "3_5"), (0, "9_10"), (1, "8_9"), (0, "2_3_t2")):
        d = handle(short, rate)
        assert d.set_variant(D.VARIANT_AUTO) == D.VARIANT_PAIR, rate
        assert d.set_variant(D.VARIANT_FRAME) == D.VARIANT_FRAME
        assert d.set_variant(D.VARIANT_PAIR) == D.VARIANT_PAIR
        d.set_variant(D.VARIANT_AUTO)


@pytest.mark.parametrize("short,rate,n", [(1, "1_2", 1500), (0, "3_5", 777), (0, "9_10", 600)])
def test_host_call_pipelined_matches_device(short, rate, n):
    """drx_ldpc_decode_host with per-frame stopping on 512 frames or more runs
    in chunks on two streams; it returns the device call's results exactly."""
    import torch

    d = handle(short, rate)
    llr = awgn_frames(short, rate, n, 1.5 if short else (2.6 if rate == "3_5" else 6.6), seed=31)
    bits, it, ok = d.decode_host(llr, 30)
    tb, ti, to = d.decode_device(torch.from_numpy(llr).cuda(), 30)
    torch.cuda.synchronize()
    assert np.array_equal(bits, tb.cpu().numpy())
    assert np.array_equal(it, ti.cpu().numpy())
    assert np.array_equal(ok, to.cpu().numpy())
    # page-locked rows in and out: the copy engines read and write the caller's arrays directly
    pin = [torch.from_numpy(llr).pin_memory(), torch.zeros((n, d.nbytes), dtype=torch.uint8).pin_memory(),
           torch.zeros(n, dtype=torch.int32).pin_memory(), torch.zeros(n, dtype=torch.uint8).pin_memory()]
    pb, pi, po = d.decode_host(pin[0].numpy(), 30, out=pin[1].numpy(), iters=pin[2].numpy(), ok=pin[3].numpy())
    assert np.array_equal(pb, bits) and np.array_equal(pi, it) and np.array_equal(po, ok)
    # pinned input, pageable outputs
    qb, qi, qo = d.decode_host(pin[0].numpy(), 30)
    assert np.array_equal(qb, bits) and np.array_equal(qi, it) and np.array_equal(qo, ok)


@pytest.mark.parametrize("short,rate,es,crate", [(0, "4_5", 4.7, None), (0, "5_6", 5.2, None), (0, "8_9", 6.2, None),
                                                 (0, "9_10", 6.45, None), (1, "5_6", 5.3, None),
                                                 (1, "8_9", 6.3, None), (0, "154_180", 5.6, "8_9"),
                                                 (0, "135_180", 4.6, "3_4")])
def test_pair_matches_frame_high_degree(short, rate, es, crate):
    """Above check degree 16 the frame-pair kernel keeps 16-byte message
    records and carries up to six late slots: on a few hundred frames around
    the waterfall it gives the one-frame kernel's bits, iterations and flags."""
    import torch

    d = D.Ldpc(D.fec_lookup(short, rate), rate)
    llr, _, _ = d.generate(300, es, seed=zlib.crc32(rate.encode()) + short, const_rate=crate)
    out = {}
    for v in (D.VARIANT_FRAME, D.VARIANT_PAIR):
        assert d.set_variant(v) == v
        out[v] = [t.cpu().numpy() for t in d.decode_device(llr, 30)]
    torch.cuda.synchronize()
    for a, b in zip(out[D.VARIANT_FRAME], out[D.VARIANT_PAIR]):
        assert np.array_equal(a, b), rate
    it, ok = out[D.VARIANT_PAIR][1], out[D.VARIANT_PAIR][2]
    assert 0 < ok.sum() and it.max() > 3, "the case should have converging frames that need iterations"
    d.close()


@pytest.mark.parametrize("short,rate", RATES)
def test_pair_matches_frame_every_code(short, rate):
    """Every code of both frame sizes: on 256 frames near the waterfall the
    frame-pair kernel gives the one-frame kernel's bits, iterations and flags,
    with per-frame stopping and with group stopping (64-frame groups), and
    both give the reference's: each of the 256 frames decoded on its own and
    two 64-frame calls (reference batch semantics)."""
    import re

    import torch

    d = D.Ldpc(fec_params(short, rate), rate)
    if rate in SNR:
        es = SNR[rate]
    else:
        m = re.match(r"(\d+)_(\d+)", rate)
        es = 10 * np.log10(2 ** (2 * int(m.group(1)) / int(m.group(2))) - 1) + 0.8
    try:
        llr, _, _ = d.generate(256, float(es), seed=zlib.crc32(rate.encode()) + 7 * short, constellation="QPSK")
    except RuntimeError:
        # no QPSK MODCOD of this code: QPSK with the 1/2 mapping stands in
        llr, _, _ = d.generate(256, float(es), seed=zlib.crc32(rate.encode()) + 7 * short, constellation="QPSK",
                               const_rate="1_2")
    host = llr.cpu().numpy()[:128]
    res = {}
    for v in (D.VARIANT_FRAME, D.VARIANT_PAIR):
        assert d.set_variant(v) == v
        res[v] = [t.cpu().numpy() for t in d.decode_device(llr, 30)] + list(d.decode_host(host, 30, stop=64))
    torch.cuda.synchronize()
    for a, b in zip(res[D.VARIANT_FRAME], res[D.VARIANT_PAIR]):
        assert np.array_equal(a, b), rate
    d.close()
    # and the reference itself: all 256 frames one call each, the first 128 in two 64-frame calls
    import oracle
    if oracle.ref_available("avx2"):
        rb, ri, ro = oracle.RefCode(short, rate, flavour="avx2").decode_frames_mt(llr.cpu().numpy(), 30)
        bits, it, ok = res[D.VARIANT_PAIR][:3]
        assert np.array_equal(bits, rb) and np.array_equal(it, ri) and np.array_equal(ok, ro), rate
    if oracle.ref_available("avx512"):
        gb, rets = oracle.RefCode(short, rate, flavour="avx512").decode_groups_mt(host, 30, group=64)
        bits, it, ok = res[D.VARIANT_PAIR][3:]
        assert np.array_equal(bits, gb), rate
        assert [int(it[g]) if ok[g:g + 64].all() else -1 for g in (0, 64)] == rets.tolist(), rate
