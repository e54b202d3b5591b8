"""drx_ldpc_decode_device_noalloc: the decoder entry point that allocates no
GPU memory, for callers that cannot call cudaMalloc while they decode (a
real-time receiver thread, where an allocation can stall on a device-wide
synchronisation; a program whose GPU memory is owned by another allocator).
Its scratch is a fixed array compiled into the library.

Its results must equal those of the regular device entry point,
drx_ldpc_decode_device, bit for bit (the decoder's outputs are integers),
on two calls in a row: the second call sees the scratch the first one left.
The file is named to be collected last; it passes alone in a fresh process
and after the other tests.
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


@pytest.mark.parametrize("short,rate,const,esn0,nframes", [
    (0, "3_5", "8PSK", 5.8, 300),   # more frames than the array has CTA slabs (161)
    (1, "1_2", "QPSK", 1.6, 700),   # more frames than slabs (466)
])
def test_noalloc_matches_device_entry_point(short, rate, const, esn0, nframes):
    import torch

    import dvbrx_b200 as D

    torch.cuda.set_device(0)
    noalloc = _entry()
    d = D.Ldpc(D.fec_lookup(short, rate), rate)
    stream = torch.cuda.current_stream()
    for call in range(2):
        llr, _, _ = d.generate(nframes, esn0, seed=1234 + call, constellation=const)
        want_bits, want_it, want_ok = d.decode_device(llr, 30)
        bits = torch.full_like(want_bits, 0xA5)
        it = torch.full_like(want_it, -7)
        ok = torch.full_like(want_ok, 9)
        r = noalloc(d.h, llr.data_ptr(), llr.stride(0), bits.data_ptr(), bits.stride(0), it.data_ptr(),
                    ok.data_ptr(), nframes, 30, D.stream_handle(stream))
        assert r == 0, D.last_error()
        torch.cuda.synchronize()
        assert torch.equal(bits, want_bits), "call %d: hard bits differ" % call
        assert torch.equal(it, want_it), "call %d: iterations differ" % call
        assert torch.equal(ok, want_ok), "call %d: syndrome flags differ" % call
    d.close()
