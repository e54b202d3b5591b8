"""Shared helpers of the tests: golden-case inputs and the checker choice."""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import oracle  # noqa: E402
from make_golden import case_frames  # noqa: E402


def sha(b):
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()


def golden_case_tuple(c):
    return (c["short"], c["rate"], c["constellation"], c["constellation_rate"], c["esn0_db"],
            c["frames"], c["max_iter"], c["seed"], c["kind"])


def golden_llr(c):
    llr = case_frames(golden_case_tuple(c))
    assert sha(llr) == c["llr_sha256"], "test input generator drifted from the fixture"
    return llr


def checker(short, rate):
    """The reference build when present (it travels as a built file), else
    the restatement; both expose decode_frames / decode_call-like calls."""
    if oracle.ref_available():
        return oracle.RefCode(short, rate)
    return oracle.OrcCode(short, rate)


def check_frames(chk, llr, max_iter):
    """Per-frame results of the checker."""
    return chk.decode_frames(llr, max_iter)


def check_group(chk, llr, max_iter):
    """The frames decoded together (reference batch semantics)."""
    if isinstance(chk, oracle.RefCode):
        return chk.decode_call(llr, max_iter)
    return chk.decode_group(llr, max_iter)


def awgn_frames(short, rate, n, esn0_db, seed, constellation="QPSK", crate=None):
    """Seeded frames of a code over AWGN; the constellation row of `crate`
    (default: the code's own rate, or 1/2 where the MODCOD has none)."""
    from oracle import datagen
    crate = crate or rate
    if (constellation, crate, int(short)) not in datagen.constellations():
        crate = "1_2"
    code = oracle.OrcCode(short, rate)
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, size=(n, code.K), dtype=np.uint8)
    cw = code.encode(info)
    sym = datagen.modulate(cw, constellation, crate, short)
    n0 = 10.0 ** (-esn0_db / 10.0)
    noise = (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0 / 2)
    return datagen.demap((sym + noise).astype(np.complex64), n0, constellation, crate, short, code.N)
