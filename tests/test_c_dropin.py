"""The drop-in boundary from C: a C program written against the reference's
own headers (libdvbrx/include/dvbrx/ldpc.h, fec.h), compiled with gcc and
linked against libdvbrx_b200.so, no ctypes on the way (tests/c/).

CPU: the program compiles and links against this project's header and
against the reference's headers, and without a GPU drx_ldpc_new fails
loudly (exit status 2), no CPU fallback.  GPU: the program decodes frames in
batches of drx_ldpc_lanes() and its bits and return values equal the
reference decoder's on the same batches (libdvbrx/tests/test_ldpc.c:78-94).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "c"))
import build as cbuild  # noqa: E402

REF_BIN = os.path.join(HERE, "c", "_bin", "dropin_ref_headers")


def binaries(tmp):
    """The caller built against our header (now) and against the
    reference's headers (now if the tree is given, else the prebuilt one)."""
    out = {"own_header": cbuild.build(os.path.join(tmp, "dropin_own_header"))}
    inc = cbuild.reference_include()
    if inc:
        out["ref_headers"] = cbuild.build(os.path.join(tmp, "dropin_ref_headers"), inc)
    elif os.path.exists(REF_BIN):
        out["ref_headers"] = REF_BIN
    return out


def run(binary, short, rate, max_iter, llr, tmp):
    src, dst = os.path.join(tmp, "llr.bin"), os.path.join(tmp, "out.bin")
    np.ascontiguousarray(llr, dtype=np.int8).tofile(src)
    r = subprocess.run([binary, str(short), rate, str(max_iter), src, dst], capture_output=True, text=True)
    return r, dst


def test_c_caller_builds_and_fails_loudly_without_gpu(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the decode itself is checked by the gpu test")
    bins = binaries(str(tmp_path))
    assert "ref_headers" in bins, "no build against the reference's headers (tests/c/build.py <tree>)"
    for name, b in bins.items():
        r, _ = run(b, 1, "1_2", 10, np.zeros((2, 16200), np.int8), str(tmp_path))
        assert r.returncode == 2, (name, r.stdout, r.stderr)
        assert "drx_ldpc_new" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("short,rate,n,es,const", [(1, "1_2", 200, 1.6, "QPSK"), (0, "3_5", 100, 5.9, "8PSK")])
def test_c_caller_matches_reference(tmp_path, short, rate, n, es, const):
    import oracle
    from helpers import awgn_frames
    llr = awgn_frames(short, rate, n, es, seed=424242 + n, constellation=const)
    ref = oracle.RefCode(short, rate, flavour="avx512") if oracle.ref_available("avx512") else None
    if ref is None or ref.lanes != 64:
        pytest.skip("the 64-lane reference build is needed for 64-frame batches")
    rb, rets = ref.decode_groups_mt(llr, 30, group=64)
    bins = binaries(str(tmp_path))
    for name, b in bins.items():
        r, dst = run(b, short, rate, 30, llr, str(tmp_path))
        assert r.returncode == 0, (name, r.stderr)
        raw = np.fromfile(dst, np.uint8)
        nb = rb.shape[1]
        bits = raw[: n * nb].reshape(n, nb)
        got = raw[n * nb:].view(np.int32)
        assert np.array_equal(got, rets), name
        assert np.array_equal(bits, rb), name
