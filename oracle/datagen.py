"""ORACLE — test infrastructure only (see ``oracle/__init__.py``).

Seeded test frames in numpy: random information bits, the project's encoder
(accumulator rule, restated in ``ldpc_oracle.c``), the DVB-S2 bit interleaver
and constellation of the MODCOD, complex AWGN at a given Es/N0 and the max-log
demapper with the reference's int8 scale and quantiser:

* LLR = quantise(LLR_SCALE / n0 * (min_{bit=1} |y-p|^2 - min_{bit=0} |y-p|^2)),
  LLR_SCALE = 2 (``libdvbrx/src/demap.c:32-34,491-533``);
* QPSK in closed form, bit 2j -> I, bit 2j+1 -> Q (``demap.c:496-500``);
* bit b of symbol j <-> codeword position order[b] * nsym + j
  (``demap.c:259-268``);
* quantise: clamp to +-127, round half to even (``demap.c:225-229``).
"""
import os
import re

import numpy as np

from . import OrcCode

_HERE = os.path.dirname(os.path.abspath(__file__))
_CONSTS = None


def constellations():
    """{(name, rate, short): (bits, order, points[complex])} parsed from the
    generated table header the product compiles."""
    global _CONSTS
    if _CONSTS is None:
        path = os.path.join(_HERE, "..", "dvbrx_b200", "csrc", "codes_gen.h")
        text = open(path).read()
        body = text[text.index("cg_consts[]"):]
        rows = {}
        for m in re.finditer(
            r'\{ 0x([0-9a-f]+), "(\w+)", "(\w+)", (\d), (\d), \{ ([^}]*) \},\s*\{ ([^}]*) \} \}', body
        ):
            bits = int(m.group(5))
            order = [int(v) for v in m.group(6).split(",")]
            vals = np.array([float(v.strip().rstrip("f")) for v in m.group(7).split(",")], np.float64)
            pts = vals[0::2] + 1j * vals[1::2]
            rows[(m.group(2), m.group(3), int(m.group(4)))] = (bits, order, pts[: 1 << bits])
        _CONSTS = rows
    return _CONSTS


def quantise(v):
    v = np.clip(v, -127.0, 127.0)
    return np.rint(v).astype(np.int8)  # numpy rint: round half to even, like lrintf


def modulate(cw, constellation, rate, short_frame):
    """Codeword bits [n, N] -> unit-energy symbols [n, nsym] (complex64)."""
    bits, order, pts = constellations()[(constellation, rate, int(short_frame))]
    pts = pts / np.sqrt(np.mean(np.abs(pts) ** 2))
    n, N = cw.shape
    nsym = (N + bits - 1) // bits
    if order[0] < 0:
        labels = cw[:, 0::2].astype(np.int64) * 2 + cw[:, 1::2]
    else:
        labels = np.zeros((n, nsym), np.int64)
        for b in range(bits):
            lo = order[b] * nsym
            col = np.zeros((n, nsym), np.int64)
            seg = cw[:, lo:lo + nsym]
            col[:, : seg.shape[1]] = seg
            labels = labels * 2 + col
    return pts[labels].astype(np.complex64)


def demap(sym, n0, constellation, rate, short_frame, N):
    """Max-log int8 LLRs [n, N] in codeword order."""
    bits, order, pts = constellations()[(constellation, rate, int(short_frame))]
    pts = (pts / np.sqrt(np.mean(np.abs(pts) ** 2))).astype(np.complex64)
    k = np.float32(2.0) / np.float32(n0)
    n, nsym = sym.shape
    llr = np.zeros((n, N), np.int8)
    if order[0] < 0:
        kq = k * np.float32(4.0) * np.float32(np.sqrt(0.5))
        llr[:, 0::2] = quantise(kq * sym.real.astype(np.float32))
        llr[:, 1::2] = quantise(kq * sym.imag.astype(np.float32))
        return llr
    d = np.abs(sym[:, :, None] - pts[None, None, :]).astype(np.float32) ** 2
    lab = np.arange(1 << bits)
    for b in range(bits):
        one = ((lab >> (bits - 1 - b)) & 1) == 1
        m1 = d[:, :, one].min(axis=2)
        m0 = d[:, :, ~one].min(axis=2)
        v = quantise(k * (m1 - m0))
        lo = order[b] * nsym
        take = min(nsym, N - lo)
        llr[:, lo:lo + take] = v[:, :take]
    return llr


def make_frames(short_frame, rate, nframes, esn0_db, constellation="QPSK", seed=0, code=None):
    """Seeded frames: dict(info [n,K] u8, cw [n,N] u8, llr [n,N] i8, n0)."""
    code = code or OrcCode(short_frame, rate)
    rng = np.random.default_rng(seed)
    info = rng.integers(0, 2, size=(nframes, code.K), dtype=np.uint8)
    cw = code.encode(info)
    sym = modulate(cw, constellation, rate, short_frame)
    n0 = 10.0 ** (-esn0_db / 10.0)
    noise = (rng.standard_normal(sym.shape) + 1j * rng.standard_normal(sym.shape)) * np.sqrt(n0 / 2)
    y = (sym + noise).astype(np.complex64)
    llr = demap(y, n0, constellation, rate, short_frame, code.N)
    return dict(info=info, cw=cw, llr=llr, n0=n0, sym=y)


def pack_bits(bits):
    """[n, k] 0/1 -> [n, ceil(k/8)] packed MSB first (the decoder's output)."""
    return np.packbits(bits.astype(np.uint8), axis=-1, bitorder="big")
