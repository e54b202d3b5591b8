"""DVB-S2 MODCODs (EN 302 307-1): constellation, code rate, frame sizes, and
the Es/N0 of quasi-error-free decoding of the standard's Table 13 (the
reference receiver's copy: libdvbrx/src/pl.c:70-74, indexed by MODCOD
number).  Used to build mixed-MODCOD workloads and training ranges.

The table gives normal-frame thresholds only; short frames use the same
value (the reference has no short-frame table either)."""
import numpy as np

RATES = ["1_4", "1_3", "2_5", "1_2", "3_5", "2_3", "3_4", "4_5", "5_6", "8_9", "9_10"]

# (MODCOD number, constellation, rate, QEF Es/N0 dB)
MODCODS = [
    (1, "QPSK", "1_4", -2.35), (2, "QPSK", "1_3", -1.24), (3, "QPSK", "2_5", -0.30),
    (4, "QPSK", "1_2", 1.00), (5, "QPSK", "3_5", 2.23), (6, "QPSK", "2_3", 3.10),
    (7, "QPSK", "3_4", 4.03), (8, "QPSK", "4_5", 4.68), (9, "QPSK", "5_6", 5.18),
    (10, "QPSK", "8_9", 6.20), (11, "QPSK", "9_10", 6.42),
    (12, "8PSK", "3_5", 5.50), (13, "8PSK", "2_3", 6.62), (14, "8PSK", "3_4", 7.91),
    (15, "8PSK", "5_6", 9.35), (16, "8PSK", "8_9", 10.69), (17, "8PSK", "9_10", 10.98),
    (18, "16APSK", "2_3", 8.97), (19, "16APSK", "3_4", 10.21), (20, "16APSK", "4_5", 11.03),
    (21, "16APSK", "5_6", 11.61), (22, "16APSK", "8_9", 12.89), (23, "16APSK", "9_10", 13.13),
    (24, "32APSK", "3_4", 12.73), (25, "32APSK", "4_5", 13.64), (26, "32APSK", "5_6", 14.28),
    (27, "32APSK", "8_9", 15.69), (28, "32APSK", "9_10", 16.05),
]


def qef_db(constellation, rate):
    for _, c, r, q in MODCODS:
        if c == constellation and r == rate:
            return q
    raise KeyError((constellation, rate))


def modcods_of_rate(rate, short_frame):
    """Valid MODCODs of a rate (no 9/10 in short frames)."""
    if short_frame and rate == "9_10":
        return []
    return [(c, q) for _, c, r, q in MODCODS if r == rate]


def mixed_batch(n, seed, normal_share=0.8, margin_db=0.5):
    """A mixed-MODCOD batch: per frame (short_frame, rate, constellation,
    Es/N0): normal frames with probability normal_share, the rate uniform
    over the eleven DVB-S2 rates (redrawn for short 9/10, which does not
    exist), the constellation uniform over that rate's MODCODs, Es/N0 the
    MODCOD's QEF value plus margin_db."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        short = int(rng.random() >= normal_share)
        while True:
            rate = RATES[int(rng.integers(len(RATES)))]
            mcs = modcods_of_rate(rate, short)
            if mcs:
                break
        const, q = mcs[int(rng.integers(len(mcs)))]
        out.append((short, rate, const, q + margin_db))
    return out
