"""dvbrx_b200 — DVB-S2/S2X/T2 LDPC decoding on one NVIDIA B200 (sm_100a).

Python host side of ``libdvbrx_b200.so``.  The library's C ABI
(``include/dvbrx_b200.h``) is the product: a drop-in for the reference
receiver's ``drx_fec_lookup`` / ``drx_ldpc_new`` / ``drx_ldpc_decode`` /
``drx_ldpc_free`` (TrusterBSW/DVB-Rx ``libdvbrx/include/dvbrx/ldpc.h:14-36``,
``fec.h:13-25``) plus batch entry points.  This module binds it with ctypes,
keeping the reference's names and argument meaning:

    p = fec_lookup(False, "3_5")          # drx_fec_lookup
    d = Ldpc(p, "3_5")                    # drx_ldpc_new
    it = d.decode(llr_rows, out_rows, 30) # drx_ldpc_decode: iterations or -1

There is no CPU fallback: without the built library, or without a CUDA
device, every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdvbrx_b200.so")

STOP_FRAME = 0  # DRX_STOP_FRAME
VARIANT_AUTO, VARIANT_FRAME, VARIANT_PAIR = 0, 1, 2  # DRX_VARIANT_*

_lib = None


class FecParams(ctypes.Structure):
    """``drx_fec_params`` (reference ``libdvbrx/include/dvbrx/fec.h:13-19``)."""

    _fields_ = [
        ("short_frame", ctypes.c_int),
        ("nldpc", ctypes.c_int),
        ("kldpc", ctypes.c_int),
        ("kbch", ctypes.c_int),
        ("t", ctypes.c_int),
    ]

    def __repr__(self):
        return "FecParams(short_frame=%d, nldpc=%d, kldpc=%d, kbch=%d, t=%d)" % (
            self.short_frame, self.nldpc, self.kldpc, self.kbch, self.t)


class LdpcInfo(ctypes.Structure):
    """``drx_ldpc_info``."""

    _fields_ = [(n, ctypes.c_int) for n in
                ("nldpc", "kldpc", "K", "R", "q", "edges", "steps", "deg_max", "levelled")]


EXPORTS = (
    "drx_fec_lookup", "drx_ldpc_lanes", "drx_ldpc_new", "drx_ldpc_free", "drx_ldpc_decode",
    "drx_ldpc_last_error", "drx_ldpc_get_info", "drx_ldpc_decode_device", "drx_ldpc_decode_host",
    "drx_ldpc_device_error", "drx_ldpc_code_info", "drx_channel_generate", "drx_ldpc_set_variant",
)


def test_fail_device_alloc(after):
    """``drx_test_fail_device_alloc`` (testing): the library's next device
    allocation after `after` more fails once; -1 turns it off."""
    lib().drx_test_fail_device_alloc(int(after))


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("%s is missing: build it with `python -m dvbrx_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, cp, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t
        L.drx_fec_lookup.argtypes = [ip, cp, ctypes.POINTER(FecParams)]
        L.drx_fec_lookup.restype = ip
        L.drx_ldpc_lanes.restype = ip
        L.drx_ldpc_new.argtypes = [ctypes.POINTER(FecParams), cp]
        L.drx_ldpc_new.restype = vp
        L.drx_ldpc_free.argtypes = [vp]
        L.drx_ldpc_decode.argtypes = [vp, vp, vp, ip, ip]
        L.drx_ldpc_decode.restype = ip
        L.drx_ldpc_last_error.restype = cp
        L.drx_ldpc_get_info.argtypes = [vp, ctypes.POINTER(LdpcInfo)]
        L.drx_ldpc_get_info.restype = ip
        L.drx_ldpc_decode_device.argtypes = [vp, vp, sz, vp, sz, vp, vp, ip, ip, ip, vp]
        L.drx_ldpc_decode_device.restype = ip
        L.drx_ldpc_decode_host.argtypes = [vp, vp, vp, vp, vp, ip, ip, ip]
        L.drx_ldpc_decode_host.restype = ip
        L.drx_ldpc_code_info.argtypes = [ip, cp, ctypes.POINTER(LdpcInfo)]
        L.drx_ldpc_code_info.restype = ip
        L.drx_channel_generate.argtypes = [vp, cp, cp, ip, ctypes.c_float, ctypes.c_ulonglong, vp, sz,
                                           vp, sz, vp, sz, vp]
        L.drx_channel_generate.restype = ip
        L.drx_ldpc_mix_new.argtypes = [ip, ctypes.POINTER(FecParams), ctypes.POINTER(cp)]
        L.drx_ldpc_mix_new.restype = vp
        L.drx_ldpc_mix_free.argtypes = [vp]
        L.drx_ldpc_mix_plan.argtypes = [vp, ip, vp, vp, sz, vp, sz, vp, vp, ip]
        L.drx_ldpc_mix_plan.restype = ip
        L.drx_ldpc_mix_set_tiling.argtypes = [vp, ip]
        L.drx_ldpc_mix_set_tiling.restype = ip
        L.drx_ldpc_mix_tune.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.drx_ldpc_mix_tune.restype = ip
        L.drx_ldpc_mix_tuned_ms.argtypes = [vp, ip]
        L.drx_ldpc_mix_tuned_ms.restype = ctypes.c_float
        L.drx_ldpc_mix_run.argtypes = [vp, vp]
        L.drx_ldpc_mix_run.restype = ip
        L.drx_ldpc_set_variant.argtypes = [vp, ip]
        L.drx_ldpc_set_variant.restype = ip
        L.drx_fec_decode_device.argtypes = [vp, vp, vp, sz, vp, sz, vp, vp, vp, ip, ip, ip, vp]
        L.drx_fec_decode_device.restype = ip
        L.drx_rxq_new.argtypes = [ip, ctypes.POINTER(FecParams), ctypes.POINTER(cp), ip, ip, ip, ip, ip]
        L.drx_rxq_new.restype = vp
        L.drx_rxq_free.argtypes = [vp]
        L.drx_rxq_push.argtypes = [vp, ip, vp, ctypes.POINTER(ctypes.c_uint64)]
        L.drx_rxq_push.restype = ip
        L.drx_rxq_flush.argtypes = [vp]
        L.drx_rxq_flush.restype = ip
        L.drx_rxq_pop.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ip), vp,
                                  ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                  ctypes.POINTER(ctypes.c_int32)]
        L.drx_rxq_pop.restype = ip
        L.drx_rxq_pending.argtypes = [vp]
        L.drx_rxq_pending.restype = ip
        L.drx_ldpc_set_wait_limit.argtypes = [vp, ip]
        L.drx_ldpc_set_wait_limit.restype = ip
        L.drx_ldpc_test_skip_vote.argtypes = [vp, ip]
        L.drx_ldpc_test_skip_vote.restype = ip
        L.drx_test_fail_device_alloc.argtypes = [ip]
        L.drx_test_fail_device_alloc.restype = None
        L.drx_ldpc_device_error.argtypes = [vp]
        L.drx_ldpc_device_error.restype = ip
        L.drx_bb_descramble_device.argtypes = [vp, sz, ip, ip, vp]
        L.drx_bb_descramble_device.restype = ip
        L.drx_bbheader_check_device.argtypes = [vp, sz, vp, ip, vp]
        L.drx_bbheader_check_device.restype = ip
        L.drx_demapper_new.argtypes = [cp, cp, ip]
        L.drx_demapper_new.restype = vp
        L.drx_demapper_free.argtypes = [vp]
        L.drx_demapper_symbols.argtypes = [vp]
        L.drx_demapper_symbols.restype = ip
        L.drx_demapper_run.argtypes = [vp, vp, sz, vp, vp, sz, ip, vp]
        L.drx_demapper_run.restype = ip
        L.drx_demapper_frame.argtypes = [vp, vp, ctypes.c_float, vp]
        L.drx_demapper_frame.restype = ip
        L.drx_bch_new.argtypes = [ctypes.POINTER(FecParams)]
        L.drx_bch_new.restype = vp
        L.drx_bch_free.argtypes = [vp]
        L.drx_bch_decode.argtypes = [vp, vp]
        L.drx_bch_decode.restype = ip
        L.drx_bch_decode_device.argtypes = [vp, vp, sz, vp, ip, vp]
        L.drx_bch_decode_device.restype = ip
        L.drx_bch_encode_device.argtypes = [vp, vp, sz, ip, vp]
        L.drx_bch_encode_device.restype = ip
        L.drx_ldpc_mix_set_learned.argtypes = [vp, ip, ip, ip, vp, vp, vp]
        L.drx_ldpc_mix_set_learned.restype = ip
        L.drx_ldpc_mix_plan_learned.argtypes = [vp, ip, vp, vp, sz, vp, sz, vp, vp, vp, ip, ip]
        L.drx_ldpc_mix_plan_learned.restype = ip
        L.drx_ldpc_set_learned.argtypes = [vp, ip, ip, vp, vp, vp]
        L.drx_ldpc_set_learned.restype = ip
        L.drx_ldpc_decode_learned_device.argtypes = [vp, vp, sz, vp, sz, vp, vp, vp, ip, ip, ip, vp]
        L.drx_ldpc_decode_learned_device.restype = ip
        _lib = L
    return _lib


def last_error():
    return lib().drx_ldpc_last_error().decode()


def fec_lookup(short_frame, rate):
    """``drx_fec_lookup``: FecParams of a rate string; KeyError if unknown."""
    p = FecParams()
    if lib().drx_fec_lookup(int(bool(short_frame)), rate.encode(), ctypes.byref(p)) != 0:
        raise KeyError(rate)
    return p


def lanes():
    """``drx_ldpc_lanes``: most frames per ``Ldpc.decode`` call (64)."""
    return lib().drx_ldpc_lanes()


def code_info(short_frame, rate):
    """``drx_ldpc_code_info``: geometry of a code, computed on the host."""
    info = LdpcInfo()
    if lib().drx_ldpc_code_info(int(bool(short_frame)), rate.encode(), ctypes.byref(info)) != 0:
        raise KeyError(rate)
    return info


def stream_handle(stream):
    """cudaStream_t of a torch stream as the C ABI takes it: torch's legacy
    default stream has handle 0, which the C ABI reads as "the handle's own
    stream", so it is passed as cudaStreamLegacy (1) instead."""
    h = stream.cuda_stream
    return ctypes.c_void_p(h if h else 1)


def _ptrs(rows):
    arr = (ctypes.c_void_p * len(rows))()
    for i, r in enumerate(rows):
        arr[i] = r.ctypes.data
    return arr


class Ldpc:
    """A decoder handle for one code (``drx_ldpc_new`` / ``drx_ldpc_free``)."""

    def __init__(self, params, rate):
        self._lib = lib()
        self.rate = rate
        self.params = FecParams(params.short_frame, params.nldpc, params.kldpc, params.kbch, params.t)
        self.h = self._lib.drx_ldpc_new(ctypes.byref(self.params), rate.encode())
        if not self.h:
            raise RuntimeError("drx_ldpc_new(%s): %s" % (rate, last_error()))
        info = LdpcInfo()
        self._lib.drx_ldpc_get_info(self.h, ctypes.byref(info))
        self.info = info
        self.N = info.nldpc
        self.kldpc = info.kldpc
        self.nbytes = (info.kldpc + 7) // 8

    def close(self):
        if getattr(self, "h", None):
            self._lib.drx_ldpc_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def decode(self, llr, out, max_iter):
        """``drx_ldpc_decode``: llr and out are sequences of per-frame numpy
        arrays (int8, nldpc) and (uint8, ceil(kldpc/8)); returns the
        iterations run or -1."""
        n = len(llr)
        for r in llr:
            assert r.dtype == np.int8 and r.flags.c_contiguous and r.size >= self.N
        for r in out:
            assert r.dtype == np.uint8 and r.flags.c_contiguous and r.size >= self.nbytes
        return self._lib.drx_ldpc_decode(self.h, _ptrs(list(llr)), _ptrs(list(out)), n, int(max_iter))

    def decode_host(self, llr, max_iter, stop=STOP_FRAME, out=None, iters=None, ok=None):
        """Host batch: llr [n, nldpc] int8 -> (bits [n, nbytes], iters, ok).
        out / iters / ok: optional preallocated C-contiguous arrays (uint8
        [n, nbytes], int32 [n], uint8 [n]), reused by callers that decode
        batch after batch."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8) if out is None else out
        it = np.zeros(n, np.int32) if iters is None else iters
        ok = np.zeros(n, np.uint8) if ok is None else ok
        assert out.shape == (n, self.nbytes) and out.dtype == np.uint8 and out.flags.c_contiguous
        assert it.shape == (n,) and it.dtype == np.int32 and ok.shape == (n,) and ok.dtype == np.uint8
        r = self._lib.drx_ldpc_decode_host(self.h, llr.ctypes.data, out.ctypes.data, it.ctypes.data,
                                           ok.ctypes.data, n, int(max_iter), int(stop))
        if r != 0:
            raise RuntimeError("drx_ldpc_decode_host: " + last_error())
        return out, it, ok

    def decode_device(self, llr, max_iter, stop=STOP_FRAME, out=None, iters=None, ok=None, stream=None):
        """Device batch on torch CUDA tensors (asynchronous on ``stream``,
        default the current torch stream): llr [n, stride >= nldpc] int8."""
        import torch

        assert llr.is_cuda and llr.dtype == torch.int8 and llr.dim() == 2 and llr.stride(1) == 1
        n = llr.shape[0]
        dev = llr.device
        if out is None:
            out = torch.empty((n, self.nbytes), dtype=torch.uint8, device=dev)
        if iters is None:
            iters = torch.empty(n, dtype=torch.int32, device=dev)
        if ok is None:
            ok = torch.empty(n, dtype=torch.uint8, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        r = self._lib.drx_ldpc_decode_device(
            self.h, llr.data_ptr(), llr.stride(0), out.data_ptr(), out.stride(0), iters.data_ptr(),
            ok.data_ptr(), n, int(max_iter), int(stop), stream_handle(s))
        if r != 0:
            raise RuntimeError("drx_ldpc_decode_device: " + last_error())
        return out, iters, ok

    def generate(self, nframes, esn0_db, seed, constellation="QPSK", const_rate=None, llr=True,
                 info=False, llr_f16=False, stream=None):
        """``drx_channel_generate``: seeded synthetic frames of this code on
        the GPU.  Returns (llr int8 [n, N] or None, info uint8 [n, nbytes] or
        None, llr_f16 float16 [n, N] or None) as torch CUDA tensors."""
        import torch

        dev = torch.device("cuda", torch.cuda.current_device())
        t_llr = torch.empty((nframes, self.N), dtype=torch.int8, device=dev) if llr else None
        t_info = torch.empty((nframes, self.nbytes), dtype=torch.uint8, device=dev) if info else None
        t_h = torch.empty((nframes, self.N), dtype=torch.float16, device=dev) if llr_f16 else None
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        r = self._lib.drx_channel_generate(
            self.h, constellation.encode(), (const_rate or self.rate).encode(), int(nframes),
            ctypes.c_float(esn0_db), ctypes.c_ulonglong(seed),
            t_llr.data_ptr() if t_llr is not None else None, self.N,
            t_h.data_ptr() if t_h is not None else None, self.N,
            t_info.data_ptr() if t_info is not None else None, self.nbytes,
            stream_handle(s))
        if r != 0:
            raise RuntimeError("drx_channel_generate: " + last_error())
        return t_llr, t_info, t_h

    def set_variant(self, variant):
        """``drx_ldpc_set_variant``: VARIANT_AUTO, VARIANT_FRAME or
        VARIANT_PAIR; returns the kernel per-frame batches now run."""
        r = self._lib.drx_ldpc_set_variant(self.h, int(variant))
        if r < 0:
            raise ValueError("drx_ldpc_set_variant: " + last_error())
        return r

    def device_error(self):
        """``drx_ldpc_device_error``: the device error word since the last
        call (0 fine, 2 a group barrier gave up), cleared."""
        return self._lib.drx_ldpc_device_error(self.h)

    def set_wait_limit(self, polls):
        """``drx_ldpc_set_wait_limit``: polls of a group barrier before a
        group-stopping launch gives up (0: the default)."""
        if self._lib.drx_ldpc_set_wait_limit(self.h, int(polls)) != 0:
            raise ValueError(last_error())

    def test_skip_vote(self, cta):
        """``drx_ldpc_test_skip_vote`` (testing): CTA `cta` of later
        group-stopping launches never votes; -1 turns it off."""
        if self._lib.drx_ldpc_test_skip_vote(self.h, int(cta)) != 0:
            raise ValueError(last_error())

    def set_learned(self, scale, offset, class_of_degree):
        """``drx_ldpc_set_learned``: scale and offset tables [iters, nclass]
        (anything numpy converts to float32) and the class of every check
        degree (int8[33]); ``None`` removes the table."""
        if scale is None:
            if self._lib.drx_ldpc_set_learned(self.h, 0, 0, None, None, None) != 0:
                raise RuntimeError("drx_ldpc_set_learned: " + last_error())
            return
        b = np.ascontiguousarray(np.asarray(scale, dtype=np.float32))
        a = np.ascontiguousarray(np.asarray(offset, dtype=np.float32))
        cod = np.ascontiguousarray(np.asarray(class_of_degree, dtype=np.int8))
        assert b.shape == a.shape and b.ndim == 2 and cod.size == 33
        r = self._lib.drx_ldpc_set_learned(self.h, b.shape[0], b.shape[1], cod.ctypes.data, b.ctypes.data,
                                          a.ctypes.data)
        if r != 0:
            raise RuntimeError("drx_ldpc_set_learned: " + last_error())

    def decode_learned(self, llr, learned_iters, plain_max_iter=0, out=None, iters=None, ok=None,
                       fallback=None, stream=None):
        """``drx_ldpc_decode_learned_device`` on torch CUDA tensors: the
        learned decode (at most learned_iters iterations), then, with
        plain_max_iter > 0, the plain decoder on the frames whose syndrome
        still fails.  Returns (bits, iterations, ok, fallback)."""
        import torch

        assert llr.is_cuda and llr.dtype == torch.int8 and llr.dim() == 2 and llr.stride(1) == 1
        n = llr.shape[0]
        dev = llr.device
        if out is None:
            out = torch.empty((n, self.nbytes), dtype=torch.uint8, device=dev)
        if iters is None:
            iters = torch.empty(n, dtype=torch.int32, device=dev)
        if ok is None:
            ok = torch.empty(n, dtype=torch.uint8, device=dev)
        if fallback is None:
            fallback = torch.empty(n, dtype=torch.uint8, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        r = self._lib.drx_ldpc_decode_learned_device(
            self.h, llr.data_ptr(), llr.stride(0), out.data_ptr(), out.stride(0), iters.data_ptr(),
            ok.data_ptr(), fallback.data_ptr(), n, int(learned_iters), int(plain_max_iter), stream_handle(s))
        if r != 0:
            raise RuntimeError("drx_ldpc_decode_learned_device: " + last_error())
        return out, iters, ok, fallback


def bb_descramble(frames, kbch_bytes, stream=None):
    """``drx_bb_descramble_device`` on torch CUDA rows [n, >= kbch_bytes]
    uint8, in place."""
    import torch

    assert frames.is_cuda and frames.dtype == torch.uint8 and frames.dim() == 2 and frames.stride(1) == 1
    s = stream if stream is not None else torch.cuda.current_stream(frames.device)
    if lib().drx_bb_descramble_device(frames.data_ptr(), frames.stride(0), int(kbch_bytes), frames.shape[0],
                                      stream_handle(s)) != 0:
        raise RuntimeError("drx_bb_descramble_device: " + last_error())
    return frames


def bbheader_check(frames, stream=None):
    """``drx_bbheader_check_device``: int8 status per row (0 valid, 1 valid
    in High Efficiency Mode, -1 invalid)."""
    import torch

    assert frames.is_cuda and frames.dtype == torch.uint8 and frames.dim() == 2 and frames.stride(1) == 1
    st = torch.empty(frames.shape[0], dtype=torch.int8, device=frames.device)
    s = stream if stream is not None else torch.cuda.current_stream(frames.device)
    if lib().drx_bbheader_check_device(frames.data_ptr(), frames.stride(0), st.data_ptr(), frames.shape[0],
                                       stream_handle(s)) != 0:
        raise RuntimeError("drx_bbheader_check_device: " + last_error())
    return st


class Demapper:
    """The reference receiver's soft demapper on the GPU (``drx_demapper_*``)."""

    def __init__(self, constellation, rate, short_frame=0):
        self._lib = lib()
        self.h = self._lib.drx_demapper_new(constellation.encode(), rate.encode(), int(short_frame))
        if not self.h:
            raise RuntimeError("drx_demapper_new: " + last_error())
        self.nsym = self._lib.drx_demapper_symbols(self.h)
        self.nldpc = 16200 if short_frame else 64800

    def close(self):
        if getattr(self, "h", None):
            self._lib.drx_demapper_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def run(self, sym, n0, llr=None, stream=None):
        """Device batch: sym float32 [n, >= 2 nsym] (I/Q interleaved), n0
        float32 [n]; returns int8 LLRs [n, nldpc]."""
        import torch

        assert sym.is_cuda and sym.dtype == torch.float32 and sym.dim() == 2 and sym.stride(1) == 1
        n = sym.shape[0]
        if llr is None:
            llr = torch.empty((n, self.nldpc), dtype=torch.int8, device=sym.device)
        n0 = n0.contiguous()
        s = stream if stream is not None else torch.cuda.current_stream(sym.device)
        r = self._lib.drx_demapper_run(self.h, sym.data_ptr(), sym.stride(0), n0.data_ptr(), llr.data_ptr(),
                                       llr.stride(0), n, stream_handle(s))
        if r != 0:
            raise RuntimeError("drx_demapper_run: " + last_error())
        return llr

    def frame(self, sym, n0):
        """One host frame (numpy float32 [2 nsym]) -> int8 LLRs [nldpc]."""
        sym = np.ascontiguousarray(sym, dtype=np.float32)
        out = np.zeros(self.nldpc, np.int8)
        if self._lib.drx_demapper_frame(self.h, sym.ctypes.data, ctypes.c_float(n0), out.ctypes.data) != 0:
            raise RuntimeError("drx_demapper_frame: " + last_error())
        return out


class Bch:
    """The BCH outer code of one FEC configuration (``drx_bch_new`` /
    ``drx_bch_free``), decoded on the GPU."""

    def __init__(self, params):
        self._lib = lib()
        self.params = FecParams(params.short_frame, params.nldpc, params.kldpc, params.kbch, params.t)
        self.h = self._lib.drx_bch_new(ctypes.byref(self.params))
        if not self.h:
            raise RuntimeError("drx_bch_new: " + last_error())
        self.nbytes = self.params.kldpc // 8

    def close(self):
        if getattr(self, "h", None):
            self._lib.drx_bch_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def decode(self, word):
        """``drx_bch_decode`` on one packed codeword (numpy uint8, corrected in
        place); returns the corrected bit count or -1."""
        assert word.dtype == np.uint8 and word.flags.c_contiguous and word.size >= self.nbytes
        return self._lib.drx_bch_decode(self.h, word.ctypes.data)

    def encode_device(self, cw, stream=None):
        """``drx_bch_encode_device``: rows [n, >= nbytes] uint8 holding the
        message in their first kbch bits get their parity bits, in place."""
        import torch

        assert cw.is_cuda and cw.dtype == torch.uint8 and cw.dim() == 2 and cw.stride(1) == 1
        s = stream if stream is not None else torch.cuda.current_stream(cw.device)
        if self._lib.drx_bch_encode_device(self.h, cw.data_ptr(), cw.stride(0), cw.shape[0], stream_handle(s)) != 0:
            raise RuntimeError("drx_bch_encode_device: " + last_error())
        return cw

    def decode_device(self, cw, result=None, stream=None):
        """``drx_bch_decode_device`` on torch CUDA rows [n, >= nbytes] uint8
        (in place); returns the int32 results [n]."""
        import torch

        assert cw.is_cuda and cw.dtype == torch.uint8 and cw.dim() == 2 and cw.stride(1) == 1
        n = cw.shape[0]
        if result is None:
            result = torch.empty(n, dtype=torch.int32, device=cw.device)
        s = stream if stream is not None else torch.cuda.current_stream(cw.device)
        r = self._lib.drx_bch_decode_device(self.h, cw.data_ptr(), cw.stride(0), result.data_ptr(), n,
                                            stream_handle(s))
        if r != 0:
            raise RuntimeError("drx_bch_decode_device: " + last_error())
        return result


TILING_ONE_LAUNCH, TILING_PER_CODE, TILING_ONE_LAUNCH_PAIR = 1, 2, 3  # DRX_TILING_*


class LdpcMix:
    """A set of codes decoded together in mixed device batches
    (``drx_ldpc_mix_*``): plan a batch once (captured as CUDA graphs), tune
    the tiling on real frames, then replay it on new data in the same
    buffers."""

    def __init__(self, codes):
        """codes: sequence of (short_frame, rate) or (FecParams, rate)."""
        self._lib = lib()
        params, rates = [], []
        for a, rate in codes:
            if isinstance(a, FecParams):
                params.append(FecParams(a.short_frame, a.nldpc, a.kldpc, a.kbch, a.t))
            else:
                try:
                    params.append(fec_lookup(a, rate))
                except KeyError:  # codes without a BCH row (T2): nbch = K
                    info = code_info(a, rate)
                    params.append(FecParams(int(bool(a)), info.nldpc, info.K, info.K, 0))
            rates.append(rate)
        n = len(codes)
        self.params = (FecParams * n)(*params)
        self._rates = [r.encode() for r in rates]
        self.rates = (ctypes.c_char_p * n)(*self._rates)
        self.h = self._lib.drx_ldpc_mix_new(n, self.params, self.rates)
        if not self.h:
            raise RuntimeError("drx_ldpc_mix_new: " + last_error())
        self.ncodes = n
        self.nldpc = [p.nldpc for p in params]
        self.nbytes = [(p.kldpc + 7) // 8 for p in params]
        self._keep = None

    def close(self):
        if getattr(self, "h", None):
            self._lib.drx_ldpc_mix_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def plan(self, code, llr, out, iters, ok, max_iter):
        """code: host int32 [n] code indexes; llr, out, iters, ok: torch CUDA
        tensors [n, >= max nldpc] int8, [n, >= max bytes] uint8, [n] int32,
        [n] uint8."""
        code = np.ascontiguousarray(code, dtype=np.int32)
        n = code.shape[0]
        r = self._lib.drx_ldpc_mix_plan(self.h, n, code.ctypes.data, llr.data_ptr(), llr.stride(0),
                                        out.data_ptr(), out.stride(0), iters.data_ptr(), ok.data_ptr(),
                                        int(max_iter))
        if r != 0:
            raise RuntimeError("drx_ldpc_mix_plan: " + last_error())
        self._keep = (llr, out, iters, ok)

    def set_learned(self, code_index, scale, offset, class_of_degree):
        """``drx_ldpc_mix_set_learned``: learned tables of one code of the set."""
        b = np.ascontiguousarray(np.asarray(scale, dtype=np.float32))
        a = np.ascontiguousarray(np.asarray(offset, dtype=np.float32))
        cod = np.ascontiguousarray(np.asarray(class_of_degree, dtype=np.int8))
        r = self._lib.drx_ldpc_mix_set_learned(self.h, int(code_index), b.shape[0], b.shape[1], cod.ctypes.data,
                                              b.ctypes.data, a.ctypes.data)
        if r != 0:
            raise RuntimeError("drx_ldpc_mix_set_learned: " + last_error())

    def plan_learned(self, code, llr, out, iters, ok, fallback, learned_iters, plain_max_iter):
        """``drx_ldpc_mix_plan_learned``: as plan, learned decode with the
        plain decoder as fallback; fallback: torch CUDA uint8 [n] or None."""
        code = np.ascontiguousarray(code, dtype=np.int32)
        n = code.shape[0]
        r = self._lib.drx_ldpc_mix_plan_learned(
            self.h, n, code.ctypes.data, llr.data_ptr(), llr.stride(0), out.data_ptr(), out.stride(0),
            iters.data_ptr(), ok.data_ptr(), fallback.data_ptr() if fallback is not None else None,
            int(learned_iters), int(plain_max_iter))
        if r != 0:
            raise RuntimeError("drx_ldpc_mix_plan_learned: " + last_error())
        self._keep = (llr, out, iters, ok, fallback)

    def set_tiling(self, tiling):
        if self._lib.drx_ldpc_mix_set_tiling(self.h, int(tiling)) < 0:
            raise ValueError(last_error())

    def tuned_ms(self, tiling):
        """``drx_ldpc_mix_tuned_ms``: the tuner's time of a tiling (None if the
        plan lacks it)."""
        v = self._lib.drx_ldpc_mix_tuned_ms(self.h, int(tiling))
        return None if v < 0 else v

    def tune(self, stream=None):
        """Times every tiling of the plan on the planned batch; returns
        (choice, ms_one_launch, ms_per_code); tuned_ms gives the rest."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        a, b = ctypes.c_float(), ctypes.c_float()
        r = self._lib.drx_ldpc_mix_tune(self.h, stream_handle(s), ctypes.byref(a), ctypes.byref(b))
        if r < 0:
            raise RuntimeError("drx_ldpc_mix_tune: " + last_error())
        return r, a.value, b.value

    def run(self, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        if self._lib.drx_ldpc_mix_run(self.h, stream_handle(s)) != 0:
            raise RuntimeError("drx_ldpc_mix_run: " + last_error())


def fec_decode_device(dec, bch, llr, max_iter, stop=STOP_FRAME, stream=None):
    """``drx_fec_decode_device``: LDPC then BCH of device rows (torch CUDA
    int8 [n, >= nldpc]); returns (codewords uint8 [n, kldpc/8] corrected in
    place by the BCH decoder, LDPC iterations, LDPC flags, BCH results)."""
    import torch

    n = llr.shape[0]
    dev = llr.device
    cw = torch.empty((n, dec.nbytes), dtype=torch.uint8, device=dev)
    it = torch.empty(n, dtype=torch.int32, device=dev)
    ok = torch.empty(n, dtype=torch.uint8, device=dev)
    res = torch.empty(n, dtype=torch.int32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    r = lib().drx_fec_decode_device(dec.h, bch.h, llr.data_ptr(), llr.stride(0), cw.data_ptr(), cw.stride(0),
                                    it.data_ptr(), ok.data_ptr(), res.data_ptr(), n, int(max_iter), int(stop),
                                    stream_handle(s))
    if r != 0:
        raise RuntimeError("drx_fec_decode_device: " + last_error())
    return cw, it, ok, res


class RxQueue:
    """``drx_rxq_*``: the receiver's frame queue in front of the GPU.  codes:
    sequence of (FecParams, rate); frames pushed with a code index come back
    in arrival order, LDPC- and BCH-decoded."""

    def __init__(self, codes, batch_frames=64, max_open=4, max_iter=30, group=False, max_latency_ms=0):
        self._lib = lib()
        params = (FecParams * len(codes))(*[FecParams(p.short_frame, p.nldpc, p.kldpc, p.kbch, p.t)
                                             for p, _ in codes])
        rates = (ctypes.c_char_p * len(codes))(*[r.encode() for _, r in codes])
        self.nbytes = [(p.kldpc + 7) // 8 for p, _ in codes]
        self.h = self._lib.drx_rxq_new(len(codes), params, rates, int(batch_frames), int(max_open), int(max_iter),
                                       1 if group else 0, int(max_latency_ms))
        if not self.h:
            raise RuntimeError("drx_rxq_new: " + last_error())
        self._buf = np.zeros(64800 // 8, np.uint8)

    def push(self, code, llr):
        """Queue one frame (host int8 [nldpc]); returns its sequence number."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        f = ctypes.c_uint64()
        if self._lib.drx_rxq_push(self.h, int(code), llr.ctypes.data, ctypes.byref(f)) != 0:
            raise RuntimeError("drx_rxq_push: " + last_error())
        return f.value

    def flush(self):
        if self._lib.drx_rxq_flush(self.h) != 0:
            raise RuntimeError("drx_rxq_flush: " + last_error())

    def pop(self, wait=True):
        """The next frame in arrival order: (fseq, code, codeword bytes,
        LDPC iterations, LDPC flag, BCH result), or None."""
        f, c = ctypes.c_uint64(), ctypes.c_int()
        it, ok, bch = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        r = self._lib.drx_rxq_pop(self.h, 1 if wait else 0, ctypes.byref(f), ctypes.byref(c), self._buf.ctypes.data,
                                  ctypes.byref(it), ctypes.byref(ok), ctypes.byref(bch))
        if r < 0:
            raise RuntimeError("drx_rxq_pop: " + last_error())
        if r == 0:
            return None
        return f.value, c.value, self._buf[: self.nbytes[c.value]].copy(), it.value, ok.value, bch.value

    def pending(self):
        return self._lib.drx_rxq_pending(self.h)

    def close(self):
        if getattr(self, "h", None):
            self._lib.drx_rxq_free(self.h)
            self.h = None

    def __del__(self):
        self.close()
