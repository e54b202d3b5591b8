"""Failure paths, made without faulting the GPU.

* A group barrier that gives up.  Group stopping (the reference's batch
  semantics, libdvbrx/src/ldpc.c:614-638) makes the CTAs of a team wait for
  each other after every syndrome check.  Every such wait is bounded: after
  the handle's wait limit the CTA sets the device error word to 2 and ends
  its group.  Here one CTA of each team never arrives (a testing hook, not a
  fault), the limit is short, and the call must come back with the frames
  flagged as failed, drx_ldpc_device_error() == 2, and the handle and stream
  usable: the next decode gives the reference's results.
* A device allocation that fails.  The reference returns NULL from
  drx_ldpc_new when an allocation fails (ldpc.c:201-206, 229-233) and its
  callers treat a -1 decode as a failed batch (rx.c:134-139).  A testing
  hook makes the library's next cudaMalloc fail as an out-of-memory would:
  drx_ldpc_new must return NULL with drx_ldpc_last_error() set, and a decode
  whose scratch cannot be allocated must return -1, and work again once the
  allocation succeeds.
"""
import numpy as np
import pytest

import dvbrx_b200 as D
from helpers import awgn_frames, check_frames, check_group, checker

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["pair", "frame"])
def test_group_barrier_times_out_and_recovers(variant):
    d = D.Ldpc(D.fec_lookup(1, "1_2"), "1_2")
    assert d.set_variant(D.VARIANT_PAIR if variant == "pair" else D.VARIANT_FRAME) >= 0
    llr = awgn_frames(1, "1_2", 16, 1.4, seed=77)
    d.set_wait_limit(2000)          # about 0.4 ms per wait
    d.test_skip_vote(0)             # CTA 0 never votes: its team's waits run out
    bits, it, ok = d.decode_host(llr, 30, stop=8)
    assert d.device_error() == 2
    assert not ok[:8].any(), "the first group's barrier gave up: its frames are flagged as failed"
    # hook off, default limit: the same handle and stream decode correctly again
    d.test_skip_vote(-1)
    d.set_wait_limit(0)
    bits, it, ok = d.decode_host(llr, 30, stop=8)
    assert d.device_error() == 0
    chk = checker(1, "1_2")
    for g0 in (0, 8):
        rb, rr = check_group(chk, llr[g0:g0 + 8], 30)
        assert (int(it[g0]) if ok[g0:g0 + 8].all() else -1) == rr and (bits[g0:g0 + 8] == rb).all()
    # per-frame stopping has no barrier and is untouched by the hook
    d.test_skip_vote(0)
    pb, pi, po = d.decode_host(llr, 30)
    rb, ri, ro = check_frames(chk, llr, 30)
    assert (pb == rb).all() and (pi == ri).all() and (po == ro).all()
    assert d.device_error() == 0
    d.close()


def test_dropin_call_reports_timeout_as_failed_batch():
    """drx_ldpc_decode (64 lanes, one group) with a barrier that gives up
    returns -1, as a batch that did not converge does."""
    d = D.Ldpc(D.fec_lookup(1, "1_2"), "1_2")
    llr = awgn_frames(1, "1_2", 10, 3.0, seed=5)   # frames that converge
    rows = [np.ascontiguousarray(llr[f]) for f in range(10)]
    out = [np.zeros(d.nbytes, np.uint8) for _ in rows]
    assert d.decode(rows, out, 30) >= 0
    d.set_wait_limit(2000)
    d.test_skip_vote(0)
    assert d.decode(rows, out, 30) == -1
    assert d.device_error() == 2
    d.test_skip_vote(-1)
    assert d.decode(rows, out, 30) >= 0
    d.close()


def test_failed_allocation_in_new_returns_null():
    p = D.fec_lookup(0, "3_5")
    try:
        D.test_fail_device_alloc(0)      # the very next device allocation fails
        with pytest.raises(RuntimeError, match="out of memory|memory allocation"):
            D.Ldpc(p, "3_5")
    finally:
        D.test_fail_device_alloc(-1)
    d = D.Ldpc(p, "3_5")                 # allocations succeed again
    d.close()


def test_failed_scratch_allocation_fails_the_decode():
    import torch

    d = D.Ldpc(D.fec_lookup(1, "1_2"), "1_2")
    llr = torch.from_numpy(awgn_frames(1, "1_2", 64, 1.6, seed=3)).cuda()
    try:
        D.test_fail_device_alloc(0)      # the handle's first scratch allocation
        with pytest.raises(RuntimeError, match="out of memory|memory allocation"):
            d.decode_device(llr, 30)
    finally:
        D.test_fail_device_alloc(-1)
    bits, it, ok = d.decode_device(llr, 30)
    torch.cuda.synchronize()
    rb, ri, ro = check_frames(checker(1, "1_2"), llr.cpu().numpy(), 30)
    assert (bits.cpu().numpy() == rb).all() and (it.cpu().numpy() == ri).all()
    assert d.device_error() == 0
    d.close()
