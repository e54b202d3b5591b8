"""The GPU soft demapper (drx_demapper_*) against the reference's
drx_demap_frame (demap.c) compiled from its sources: identical int8 LLRs for
the DVB-S2 and S2X constellations on normal and short frames, at saturating
and noisy Es/N0, and chained into the LDPC decoder.  Exactness holds for the
reference's builds with fused multiply-adds (AVX2, AVX-512); its SSE2 build
may differ by one unit on rare ties."""
import ctypes

import numpy as np
import pytest
import torch

import dvbrx_b200 as D
import oracle
from oracle import datagen

pytestmark = pytest.mark.gpu

CASES = [("QPSK", "1_2", 0), ("QPSK", "8_9", 1), ("8PSK", "3_5", 0), ("8PSK", "2_3", 1), ("16APSK", "2_3", 0),
         ("16APSK", "8_9", 1), ("32APSK", "3_4", 0), ("32APSK", "9_10", 0), ("32APSK", "5_6", 1),
         # DVB-S2X: 8 to 256 points; 128APSK pads 6 bits; the 256APSK tables made of 8 rings of the
         # same 32 phases take the reference's ring metric, the others the full search
         ("8APSK", "100_180", 0), ("8_8APSK", "90_180", 0), ("4_12_16APSK", "32_45", 1),
         ("4_8_4_16APSK", "128_180", 0), ("64APSK", "128_180", 0), ("8_16_20_20APSK", "7_9", 0),
         ("4_12_20_28APSK", "132_180", 0), ("128APSK", "135_180", 0), ("256APSK", "116_180", 0),
         ("256APSK", "135_180", 0), ("256APSK", "20_30", 0), ("256APSK", "22_30", 0)]


def ref_demap(const, rate, short, sym_iq, n0):
    lib = oracle.load_ref()
    lib.ref_demap_new.restype = ctypes.c_void_p
    lib.ref_demap_new.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    lib.ref_demap_free.argtypes = [ctypes.c_void_p]
    lib.ref_demap_frame.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p]
    d = lib.ref_demap_new(const.encode(), rate.encode(), short)
    N = 16200 if short else 64800
    out = np.zeros((sym_iq.shape[0], N), np.int8)
    for f in range(sym_iq.shape[0]):
        row = np.ascontiguousarray(sym_iq[f])
        lib.ref_demap_frame(d, row.ctypes.data, ctypes.c_float(n0[f]), out[f].ctypes.data)
    lib.ref_demap_free(d)
    return out


def noisy_symbols(const, rate, short, esn0_list, seed):
    code = oracle.OrcCode(short, rate)
    rng = np.random.default_rng(seed)
    cw = code.encode(rng.integers(0, 2, size=(len(esn0_list), code.K), dtype=np.uint8))
    sym = datagen.modulate(cw, const, rate, short)
    n0 = np.array([10 ** (-e / 10) for e in esn0_list], np.float32)
    noise = (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0[:, None] / 2)
    y = (sym + noise).astype(np.complex64)
    iq = np.empty((y.shape[0], 2 * y.shape[1]), np.float32)
    iq[:, 0::2], iq[:, 1::2] = y.real, y.imag
    return iq, n0, code


def exact_reference():
    return oracle.best_ref_flavour() in ("avx512", "avx2")


@pytest.mark.parametrize("const,rate,short", CASES)
def test_demapper_matches_reference(const, rate, short):
    iq, n0, _ = noisy_symbols(const, rate, short, [-2.0, 3.0, 8.0, 14.0, 25.0], seed=len(const) + len(rate))
    want = ref_demap(const, rate, short, iq, n0)
    m = D.Demapper(const, rate, short)
    assert iq.shape[1] == 2 * m.nsym
    got = m.run(torch.from_numpy(iq).cuda(), torch.from_numpy(n0).cuda()).cpu().numpy()
    diff = np.abs(got.astype(int) - want.astype(int))
    if exact_reference():
        assert diff.max() == 0, (const, rate, short, int((diff > 0).sum()))
    else:
        assert diff.max() <= 1 and (diff == 0).mean() > 0.999
    one = m.frame(iq[2], float(n0[2]))
    assert np.array_equal(one, got[2])


def test_demapper_into_decoder():
    """Symbols -> GPU LLRs -> GPU decoder equals the reference decoder on the
    reference demapper's LLRs."""
    const, rate, short = "8PSK", "3_5", 0
    iq, n0, _ = noisy_symbols(const, rate, short, [5.6] * 6, seed=77)
    m = D.Demapper(const, rate, short)
    llr = m.run(torch.from_numpy(iq).cuda(), torch.from_numpy(n0).cuda())
    dec = D.Ldpc(D.fec_lookup(short, rate), rate)
    bits, it, ok = dec.decode_device(llr, 30)
    ref_llr = ref_demap(const, rate, short, iq, n0)
    if exact_reference():
        assert np.array_equal(llr.cpu().numpy(), ref_llr)
    rb, ri, ro = oracle.RefCode(short, rate).decode_frames(llr.cpu().numpy(), 30)
    assert np.array_equal(bits.cpu().numpy(), rb) and np.array_equal(it.cpu().numpy(), ri)
    assert np.array_equal(ok.cpu().numpy(), ro)
