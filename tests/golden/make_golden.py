"""Generate tests/golden/cases.json from the reference decoder.

Run in a container where the reference tree is mounted and the oracle is
built (``make -C oracle ref``):

    python tests/golden/make_golden.py

Each case fixes a code, a channel and a seed.  The inputs are regenerated at
test time by ``oracle.datagen`` (their SHA-256 is stored to prove the bytes
are the same); the outputs stored are those of the reference's own
``drx_ldpc_decode`` compiled from its sources: per frame (one call with
nframes = 1) the SHA-256 of the hard bits, the iteration count and the
syndrome flag, and for the whole set decoded as one batch (reference batch
semantics) the return value and the SHA-256 of all hard bits.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import RefCode, datagen  # noqa: E402

# (short, rate, constellation, constellation rate, EsN0 dB, frames, max_iter, seed, kind)
CASES = [
    (1, "1_2", "QPSK", "1_2", 1.5, 32, 50, 101, "awgn"),       # small config: short 1/2, QPSK
    (0, "3_5", "8PSK", "3_5", 6.0, 8, 30, 102, "awgn"),        # config at size: normal 3/5, 8PSK
    (0, "3_5", "8PSK", "3_5", 5.0, 4, 30, 103, "awgn"),        # below threshold: failures
    (0, "2_3", "8PSK", "2_3", 6.6, 6, 20, 104, "awgn"),        # learned-decoder code
    (1, "8_9", "QPSK", "8_9", 7.0, 16, 30, 105, "awgn"),       # degree 27, levelled
    (0, "9_10", "QPSK", "9_10", 7.0, 6, 30, 106, "awgn"),      # degree 30, levelled
    (0, "1_4", "QPSK", "1_4", -1.0, 6, 30, 107, "awgn"),       # degree 4, 135 layers
    (0, "13_45", "QPSK", "13_45", -0.8, 4, 30, 108, "awgn"),   # S2X, single level
    (0, "154_180", "QPSK", "1_2", 10.0, 4, 30, 109, "awgn"),   # S2X degree 30
    (1, "32_45", "8PSK", "32_45", 8.0, 8, 30, 110, "awgn"),    # S2X short
    (0, "2_3_t2", "QPSK", "1_2", 3.4, 4, 30, 111, "awgn"),     # T2 64K
    (1, "3_5_t2", "QPSK", "1_2", 2.8, 8, 30, 112, "awgn"),     # T2 16K
    (1, "1_2", "QPSK", "1_2", 0.0, 8, 3, 113, "random"),       # uniform int8, saturation
    (1, "2_5", "QPSK", "2_5", 0.0, 4, 5, 114, "zero"),         # all-zero LLRs: never passes
    (0, "3_5", "8PSK", "3_5", 0.0, 2, 30, 115, "clean"),       # noiseless: 0 iterations
]


def case_frames(case, code=None):
    short, rate, cons, crate, es, n, max_iter, seed, kind = case
    if kind == "awgn" or kind == "clean":
        if code is None:
            from oracle import OrcCode
            code = OrcCode(short, rate)
        rng = np.random.default_rng(seed)
        info = rng.integers(0, 2, size=(n, code.K), dtype=np.uint8)
        cw = code.encode(info)
        if kind == "clean":
            return np.where(cw == 0, 127, -127).astype(np.int8)
        sym = datagen.modulate(cw, cons, crate, short)
        n0 = 10.0 ** (-es / 10.0)
        noise = (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0 / 2)
        return datagen.demap((sym + noise).astype(np.complex64), n0, cons, crate, short, code.N)
    N = 16200 if short else 64800
    if kind == "random":
        return np.random.default_rng(seed).integers(-128, 128, size=(n, N)).astype(np.int8)
    if kind == "zero":
        return np.zeros((n, N), np.int8)
    raise ValueError(kind)


def sha(b):
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()


def main():
    out = []
    for case in CASES:
        short, rate, cons, crate, es, n, max_iter, seed, kind = case
        ref = RefCode(short, rate, "avx2")
        llr = case_frames(case)
        bits, it, ok = ref.decode_frames(llr, max_iter)
        gbits, gret = ref.decode_call(llr, max_iter)
        out.append(dict(
            short=short, rate=rate, constellation=cons, constellation_rate=crate, esn0_db=es,
            frames=n, max_iter=max_iter, seed=seed, kind=kind, kldpc=ref.params.kldpc,
            llr_sha256=sha(llr),
            frame_bits_sha256=[sha(bits[f]) for f in range(n)],
            frame_iterations=[int(v) for v in it], frame_ok=[int(v) for v in ok],
            batch_return=int(gret), batch_bits_sha256=sha(gbits),
        ))
        print(rate, short, kind, "iters", list(it), "batch", gret)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "cases.json"), "w") as f:
        json.dump(dict(generator="tests/golden/make_golden.py",
                       reference="TrusterBSW/DVB-Rx 0.1.3 libdvbrx/src/ldpc.c built by oracle/Makefile (avx2)",
                       cases=out), f, indent=1)


if __name__ == "__main__":
    main()
