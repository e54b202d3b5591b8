"""The GPU baseband layer (drx_bb_descramble_device,
drx_bbheader_check_device) against the reference's bb.c compiled from its
sources: identical descrambled frames and header verdicts (valid, valid in
High Efficiency Mode, invalid)."""
import ctypes

import numpy as np
import pytest
import torch

import dvbrx_b200 as D
import oracle

pytestmark = pytest.mark.gpu


class RefHeader(ctypes.Structure):
    _fields_ = [("ts_gs", ctypes.c_uint8), ("sis", ctypes.c_uint8), ("ccm", ctypes.c_uint8),
                ("issyi", ctypes.c_uint8), ("npd", ctypes.c_uint8), ("ro", ctypes.c_uint8), ("isi", ctypes.c_uint8),
                ("upl", ctypes.c_uint16), ("dfl", ctypes.c_uint16), ("sync", ctypes.c_uint8),
                ("syncd", ctypes.c_uint16), ("hem", ctypes.c_uint8)]


def ref_lib():
    lib = oracle.load_ref()
    lib.ref_bb_descramble.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_crc8.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.ref_crc8.restype = ctypes.c_uint8
    lib.ref_bbheader_parse.argtypes = [ctypes.c_void_p, ctypes.POINTER(RefHeader)]
    lib.ref_bbheader_parse.restype = ctypes.c_int
    return lib


@pytest.mark.parametrize("kbytes,stride", [(7274, 7274), (4836, 4860), (2001, 2025), (879, 901), (1, 3)])
def test_descramble_matches_reference(kbytes, stride):
    lib = ref_lib()
    rng = np.random.default_rng(kbytes)
    frames = rng.integers(0, 256, (37, stride), dtype=np.uint8)
    want = frames.copy()
    for f in range(want.shape[0]):
        row = np.ascontiguousarray(want[f])
        lib.ref_bb_descramble(row.ctypes.data, kbytes)
        want[f] = row
    dev = torch.from_numpy(frames).cuda()
    D.bb_descramble(dev, kbytes)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), want)


def headers(lib, rng, n):
    out = []
    for k in range(n):
        kind = k % 6
        h = rng.integers(0, 256, 10, dtype=np.uint8)
        if kind in (0, 1, 2):  # plausible header, valid CRC
            h[0] = (3 << 6) | (rng.integers(0, 64) & 0x37)
            dfl = int(rng.integers(0, 7264)) * 8
            syncd = int(rng.integers(0, dfl // 8 + 2)) * 8
            h[4], h[5], h[7], h[8] = dfl >> 8, dfl & 255, syncd >> 8, syncd & 255
            if kind == 2:  # generic stream or out-of-range fields
                h[0] = (rng.integers(0, 3) << 6) | (h[0] & 0x3F)
                h[4] = rng.integers(0, 256)
        if kind == 3:  # High Efficiency Mode: TS, no ISSY, UPL and SYNC zero, CRC xor 1
            h[0] = (3 << 6) | (rng.integers(0, 64) & 0x37)
            h[2] = h[3] = h[6] = 0
            dfl = int(rng.integers(0, 7000)) * 8
            syncd = int(rng.integers(0, dfl // 8 + 1)) * 8
            h[4], h[5], h[7], h[8] = dfl >> 8, dfl & 255, syncd >> 8, syncd & 255
        c = lib.ref_crc8(np.ascontiguousarray(h[:9]).ctypes.data, 9)
        if kind in (0, 1, 2):
            h[9] = c
        elif kind == 3:
            h[9] = c ^ 1
        elif kind == 4:
            h[9] = c ^ (1 << int(rng.integers(1, 8)))  # damaged CRC
        out.append(h)
    return np.stack(out)


def test_header_check_matches_reference():
    lib = ref_lib()
    rng = np.random.default_rng(12)
    hs = headers(lib, rng, 600)
    want = np.zeros(hs.shape[0], np.int8)
    for f in range(hs.shape[0]):
        r = RefHeader()
        row = np.ascontiguousarray(hs[f])
        ret = lib.ref_bbheader_parse(row.ctypes.data, ctypes.byref(r))
        want[f] = -1 if ret < 0 else (1 if r.hem else 0)
    frames = np.zeros((hs.shape[0], 24), np.uint8)
    frames[:, :10] = hs
    got = D.bbheader_check(torch.from_numpy(frames).cuda()).cpu().numpy()
    assert np.array_equal(got, want)
    assert (want == 0).any() and (want == 1).any() and (want == -1).any()
