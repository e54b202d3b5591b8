"""drx_ldpc_decode_device_noalloc: the decoder entry point that allocates no
GPU memory, for callers that cannot call cudaMalloc while they decode (a
real-time receiver thread, where an allocation can stall on a device-wide
synchronisation; a program whose GPU memory is owned by another allocator).
Its scratch is a fixed array compiled into the library.

Its results must equal those of the regular device entry point,
drx_ldpc_decode_device, bit for bit (the decoder's outputs are integers),
on two calls in a row: the second call sees the scratch the first one left.
A call must not lower the device's free memory: after the regular decodes
and a zero-frame set-up call, the free bytes before and after the two calls
are the same.  The file is named to be collected last; it passes alone in a
fresh process and after the other tests.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _entry():
    import dvbrx_b200 as D
    lib = ctypes.CDLL(D.LIB_PATH)
    f = lib.drx_ldpc_decode_device_noalloc
    vp, sz, ip = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    f.argtypes = [vp, vp, sz, vp, sz, vp, vp, ip, ip, vp]
    f.restype = ip
    return f


def _free_bytes():
    """Free device memory (cudaMemGetInfo: device-wide, whoever allocates)."""
    import torch
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("short,rate,const,esn0,nframes", [
    (0, "3_5", "8PSK", 5.8, 300),   # more frames than the array has CTA slabs (64 frame-pair CTAs)
    (1, "1_2", "QPSK", 1.6, 700),   # more frames than slabs (233)
])
def test_noalloc_matches_device_entry_point(short, rate, const, esn0, nframes):
    import torch

    import dvbrx_b200 as D

    torch.cuda.set_device(0)
    noalloc = _entry()
    d = D.Ldpc(D.fec_lookup(short, rate), rate)
    stream = torch.cuda.current_stream()
    # the inputs and the regular entry point's results first: those allocate
    cases = []
    for call in range(2):
        llr, _, _ = d.generate(nframes, esn0, seed=1234 + call, constellation=const)
        want = d.decode_device(llr, 30)
        got = (torch.full_like(want[0], 0xA5), torch.full_like(want[1], -7), torch.full_like(want[2], 9))
        cases.append((llr, want, got))
    # the per-device set-up: a call with no frames decodes nothing
    assert noalloc(d.h, None, d.N, None, d.nbytes, None, None, 0, 30, D.stream_handle(stream)) == 0, D.last_error()
    torch.cuda.synchronize()
    free0 = _free_bytes()
    for llr, want, got in cases:
        bits, it, ok = got
        r = noalloc(d.h, llr.data_ptr(), llr.stride(0), bits.data_ptr(), bits.stride(0), it.data_ptr(),
                    ok.data_ptr(), nframes, 30, D.stream_handle(stream))
        assert r == 0, D.last_error()
        torch.cuda.synchronize()
    # read before any comparison, which may allocate through torch's caching allocator
    assert _free_bytes() == free0, "the calls allocated device memory"
    for call, (llr, want, got) in enumerate(cases):
        assert torch.equal(got[0], want[0]), "call %d: hard bits differ" % call
        assert torch.equal(got[1], want[1]), "call %d: iterations differ" % call
        assert torch.equal(got[2], want[2]), "call %d: syndrome flags differ" % call
    assert d.device_error() == 0
    d.close()
