"""The receiver's FEC stage on the GPU against the reference's receivers.

* drx_fec_decode_device on the DVB-T2 FEC path (libdvbrx/src/dvbt2.c:
  2386-2396): the T2 codes (normal 2/3 with its own table "2_3_t2", short
  3/5 with "3_5_t2", both with the DVB-S2 BCH code of their rate), blocks
  LDPC-decoded in batches of 64 and every block BCH-decoded: corrected
  codewords, BCH results and batch return values equal the reference's
  decoders (ldpc.c, bch.c) called the same way.
* drx_rxq, the queue that replaces the LDPC worker pool and output thread of
  libdvbrx/src/rxmt.c: frames of five codes pushed in a mixed order come
  back in arrival order, batched exactly as batch_for / on_plframe batch
  them (one open batch per code, at most four open, a batch sent when full):
  the model below restates that rule, and every frame's corrected codeword,
  LDPC iterations and flag, and BCH result equal the reference decoding the
  model's batches with drx_ldpc_decode and drx_bch_decode.
"""
import numpy as np
import pytest

import dvbrx_b200 as D
import oracle
from oracle import datagen

pytestmark = pytest.mark.gpu


def coded_frames(short, s2rate, ldpc_rate, n, esn0, seed, constellation="QPSK"):
    """n frames: random BBFRAME bits, the BCH code of s2rate, the LDPC code
    ldpc_rate, the constellation over AWGN, int8 LLRs."""
    p = oracle.fec_params(short, s2rate)
    rng = np.random.default_rng(seed)
    msg = rng.integers(0, 256, size=(n, p.kbch // 8), dtype=np.uint8)
    cw = oracle.bch_encode(short, s2rate, msg)
    code = oracle.OrcCode(short, ldpc_rate)
    info = np.unpackbits(cw, axis=1)[:, : code.K]
    word = code.encode(info)
    crate = s2rate if (constellation, s2rate, int(short)) in datagen.constellations() else "1_2"
    sym = datagen.modulate(word, constellation, crate, short)
    n0 = 10.0 ** (-esn0 / 10.0)
    noise = (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0 / 2)
    return datagen.demap((sym + noise).astype(np.complex64), n0, constellation, crate, short, code.N)


def reference_batch(short, s2rate, ldpc_rate, llr, max_iter):
    """The reference receiver on one batch: drx_ldpc_decode on the batch,
    then drx_bch_decode of every codeword."""
    ref = oracle.RefCode(short, ldpc_rate, flavour="avx512", params=oracle.fec_params(short, s2rate))
    bits, ret = ref.decode_call(llr, max_iter)
    words, res = oracle.RefBch(short, s2rate).decode(bits)
    return words, res, ret


needs_ref = pytest.mark.skipif(not oracle.ref_available("avx512"), reason="64-lane reference build missing")


def t2_chain(short, s2rate, ldpc_rate, n, es):
    """The chain on n frames against the reference batch by batch; returns
    the BCH results."""
    import torch

    llr = coded_frames(short, s2rate, ldpc_rate, n, es, seed=n + short)
    p = D.fec_lookup(short, s2rate)
    dec, bch = D.Ldpc(p, ldpc_rate), D.Bch(p)
    cw, it, ok, res = (t.cpu().numpy() for t in D.fec_decode_device(dec, bch, torch.from_numpy(llr).cuda(), 30,
                                                                      stop=64))
    dec.close()
    bch.close()
    for g0 in range(0, n, 64):
        words, rres, ret = reference_batch(short, s2rate, ldpc_rate, llr[g0:g0 + 64], 30)
        assert (int(it[g0]) if ok[g0:g0 + 64].all() else -1) == ret
        assert np.array_equal(cw[g0:g0 + 64], words)
        assert np.array_equal(res[g0:g0 + 64], rres)
    return res


@needs_ref
@pytest.mark.parametrize("short,s2rate,ldpc_rate,n,es", [(0, "2_3", "2_3_t2", 192, 3.0),
                                                          (0, "2_3", "2_3_t2", 128, 3.3),
                                                          (1, "3_5", "3_5_t2", 256, 2.2),
                                                          (1, "3_5", "3_5_t2", 192, 2.6)])
def test_t2_fec_chain_matches_reference(short, s2rate, ldpc_rate, n, es):
    t2_chain(short, s2rate, ldpc_rate, n, es)


@needs_ref
def test_t2_fec_chain_exercises_bch():
    """Below the LDPC waterfall the BCH decoder both corrects residual errors
    and gives up on blocks, and the chain still equals the reference."""
    res = np.concatenate([t2_chain(0, "2_3", "2_3_t2", 256, 2.9), t2_chain(1, "3_5", "3_5_t2", 256, 2.1)])
    assert (res > 0).any() or (res < 0).any(), "no block reached the BCH decoder with errors"


# (short, S2 rate, LDPC table, Es/N0, constellation)
CODES = [(0, "3_5", "3_5", 5.9, "8PSK"), (1, "1_2", "1_2", 1.6, "QPSK"), (0, "2_3", "2_3", 3.3, "QPSK"),
         (1, "8_9", "8_9", 6.6, "QPSK"), (1, "1_4", "1_4", -1.6, "QPSK")]


def model_batches(codes_seq, batch_frames, max_open):
    """rxmt.c's batching (batch_for / on_plframe / send_all at the end):
    the frames of each sent batch, in send order."""
    open_, sent = [], []
    for f, c in enumerate(codes_seq):
        b = next((o for o in open_ if o[0] == c), None)
        if b is None:
            if len(open_) == max_open:
                sent.append(open_.pop(0))
            b = (c, [])
            open_.append(b)
        b[1].append(f)
        if len(b[1]) == batch_frames:
            open_.remove(b)
            sent.append(b)
    return sent + open_


@needs_ref
@pytest.mark.parametrize("group", [True, False])
def test_rxq_matches_reference_receiver(group):
    rng = np.random.default_rng(2024)
    # runs of frames of one code, as a VCM/ACM stream delivers them
    seq = []
    while len(seq) < 420:
        seq += [int(rng.integers(0, len(CODES)))] * int(rng.integers(1, 40))
    seq = seq[:420]
    frames = {}
    for c, (short, s2, lr, es, const) in enumerate(CODES):
        n = seq.count(c)
        frames[c] = iter(coded_frames(short, s2, lr, n, es, seed=77 + c, constellation=const)) if n else iter(())
    llrs = [next(frames[c]) for c in seq]
    q = D.RxQueue([(D.fec_lookup(s, r), lr) for s, r, lr, _, _ in CODES], batch_frames=64, max_open=4,
                  max_iter=30, group=group)
    for f, c in enumerate(seq):
        assert q.push(c, llrs[f]) == f
    assert q.pending() == len(seq)
    out = []
    while True:
        r = q.pop(wait=True)
        if r is None:
            break
        out.append(r)
    assert q.pending() == 0
    assert [r[0] for r in out] == list(range(len(seq))), "frames must leave in arrival order"
    assert [r[1] for r in out] == seq
    batches = model_batches(seq, 64, 4)
    assert any(len(b[1]) < 64 for b in batches[:-4]), "the case should send batches early (max_open)"
    for c, idx in batches:
        short, s2, lr, _, _ = CODES[c]
        llr = np.stack([llrs[f] for f in idx])
        if group:
            words, res, ret = reference_batch(short, s2, lr, llr, 30)
            for k, f in enumerate(idx):
                _, _, cw, it, ok, bres = out[f]
                assert (it if ok else -1) == ret, (c, f)
                assert np.array_equal(cw, words[k]) and bres == res[k], (c, f)
        else:
            ref = oracle.RefCode(short, lr, flavour="avx512", params=oracle.fec_params(short, s2))
            bits, it_r, ok_r = ref.decode_frames_mt(llr, 30)
            words, res = oracle.RefBch(short, s2).decode(bits)
            for k, f in enumerate(idx):
                _, _, cw, it, ok, bres = out[f]
                assert it == it_r[k] and ok == ok_r[k], (c, f)
                assert np.array_equal(cw, words[k]) and bres == res[k], (c, f)
    q.close()


def test_rxq_rejects_oversized_groups():
    with pytest.raises(RuntimeError, match="at most"):
        D.RxQueue([(D.fec_lookup(1, "1_2"), "1_2")], batch_frames=65, group=True)
    q = D.RxQueue([(D.fec_lookup(1, "1_2"), "1_2")], batch_frames=1024, group=False)
    assert q.pop(wait=False) is None and q.pending() == 0
    q.close()
