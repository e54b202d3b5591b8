"""Learned (neural offset / scaled) min-sum decoder: training through the
hand-written CUDA forward and backward kernels.

The decoder is the plain decoder's layered schedule with the check node's
offset 1 replaced by a learned scale and offset per unrolled iteration t and
check-degree class k::

    mag = max(beta[t][k] * min(min_other, 127) - alpha[t][k], 0)

on the int8 decoder's scale (2 x LLR) with its saturations, evaluated in fp32
(the parameters are FP16, as the int8 decoder consumes them).  Loss: the mean
binary cross-entropy of the information bits after every iteration.

``LearnedMinSum`` is the ``torch.autograd.Function``: its forward runs
``drx_learned_forward`` keeping one checkpoint of the decoder state per
iteration, its backward runs ``drx_learned_backward``, which re-runs each
iteration from its checkpoint and walks it in reverse.  ``LearnedDecoder`` is
the module with fp32 master parameters.
"""
import ctypes

import numpy as np
import torch

from . import Ldpc, last_error, lib, stream_handle

_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    L = lib()
    vp, ip, sz, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_float
    L.drx_learned_workspace_bytes.argtypes = [vp, ip, ip, ip]
    L.drx_learned_workspace_bytes.restype = sz
    L.drx_learned_forward.argtypes = [vp, ip, vp, sz, vp, sz, ip, vp, vp, ip, vp, vp, vp, vp, sz, ip, vp]
    L.drx_learned_forward.restype = ip
    L.drx_learned_backward.argtypes = [vp, ip, vp, sz, vp, sz, ip, vp, vp, ip, vp, fp, vp, vp, vp, vp, vp, sz, vp]
    L.drx_learned_backward.restype = ip
    L.drx_ldpc_schedule.argtypes = [ip, ctypes.c_char_p, ctypes.POINTER(ip), ctypes.POINTER(ip), vp, vp]
    L.drx_ldpc_schedule.restype = ip
    _bound = True
    return L


def schedule(short_frame, rate):
    """(check_step [R] int32, links [R, deg_max] int32) of a code: the step
    of every check (layer order) and its links as codeword bit indexes
    (parity, previous parity or -1, information bits, -1 padding)."""
    L = _bind()
    ns, dm = ctypes.c_int(), ctypes.c_int()
    if L.drx_ldpc_schedule(int(short_frame), rate.encode(), ctypes.byref(ns), ctypes.byref(dm), None, None):
        raise KeyError(rate)
    from . import code_info
    R = code_info(short_frame, rate).R
    step = np.zeros(R, np.int32)
    links = np.zeros((R, dm.value), np.int32)
    L.drx_ldpc_schedule(int(short_frame), rate.encode(), ctypes.byref(ns), ctypes.byref(dm),
                        step.ctypes.data, links.ctypes.data)
    return step, links


def degree_classes(short_frame, rate):
    """Check-degree classes of a code: (degrees, class_of_degree int8[33])."""
    _, links = schedule(short_frame, rate)
    degs = sorted(set(int(d) for d in (links >= 0).sum(axis=1)))
    cod = np.zeros(33, np.int8)
    for k, d in enumerate(degs):
        cod[d] = k
    return degs, cod


class _Work:
    """Workspace, class table and per-iteration loss weights of one
    (decoder, batch size, iterations); weights None: all ones."""

    def __init__(self, dec, nframes, iters, cod, weights=None):
        L = _bind()
        self.bytes = L.drx_learned_workspace_bytes(dec.h, nframes, iters, 1)
        self.ws = torch.empty(self.bytes, dtype=torch.uint8, device="cuda")
        self.cod = np.ascontiguousarray(cod, dtype=np.int8)
        w = np.ones(iters, np.float32) if weights is None else np.asarray(weights, np.float32)
        assert w.shape == (iters,)
        self.w = torch.from_numpy(w).cuda()
        self.wsum = float(w.sum())


class LearnedMinSum(torch.autograd.Function):
    """Weighted mean of the per-iteration BCE of the learned decoder over a
    batch (weights from the workspace, all ones by default); gradients for
    the scale and offset tables through the hand-written backward."""

    @staticmethod
    def forward(ctx, beta, alpha, dec, llr16, bits, iters, cod, work):
        L = _bind()
        n = llr16.shape[0]
        nclass = beta.shape[1]
        b16 = beta.detach().to(torch.float16).contiguous()
        a16 = alpha.detach().to(torch.float16).contiguous()
        loss = torch.zeros(iters, dtype=torch.float32, device=llr16.device)
        s = torch.cuda.current_stream()
        r = L.drx_learned_forward(dec.h, n, llr16.data_ptr(), llr16.stride(0), bits.data_ptr(), bits.stride(0),
                                  iters, b16.data_ptr(), a16.data_ptr(), nclass, work.cod.ctypes.data,
                                  loss.data_ptr(), None, work.ws.data_ptr(), work.bytes, 1, stream_handle(s))
        if r:
            raise RuntimeError("drx_learned_forward: " + last_error())
        ctx.args = (dec, llr16, bits, iters, work, b16, a16, nclass, n)
        denom = work.wsum * n * dec.kldpc
        ctx.denom = denom
        return (loss * work.w).sum() / denom

    @staticmethod
    def backward(ctx, g):
        L = _bind()
        dec, llr16, bits, iters, work, b16, a16, nclass, n = ctx.args
        dbeta = torch.zeros((iters, nclass), dtype=torch.float32, device=llr16.device)
        dalpha = torch.zeros_like(dbeta)
        scratch = torch.zeros(iters, dtype=torch.float32, device=llr16.device)
        scale = float(g) / ctx.denom
        s = torch.cuda.current_stream()
        r = L.drx_learned_backward(dec.h, n, llr16.data_ptr(), llr16.stride(0), bits.data_ptr(), bits.stride(0),
                                   iters, b16.data_ptr(), a16.data_ptr(), nclass, work.cod.ctypes.data,
                                   ctypes.c_float(scale), work.w.data_ptr(), dbeta.data_ptr(), dalpha.data_ptr(),
                                   scratch.data_ptr(),
                                   work.ws.data_ptr(), work.bytes, stream_handle(s))
        if r:
            raise RuntimeError("drx_learned_backward: " + last_error())
        return dbeta, dalpha, None, None, None, None, None, None


def learned_posteriors(dec, beta, alpha, cod, llr16, bits, iters):
    """Forward only: (per-iteration BCE sums [iters], final information-bit
    posteriors [n, kldpc])."""
    L = _bind()
    n = llr16.shape[0]
    b16 = beta.detach().to(torch.float16).contiguous()
    a16 = alpha.detach().to(torch.float16).contiguous()
    ws_bytes = L.drx_learned_workspace_bytes(dec.h, n, iters, 0)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    loss = torch.zeros(iters, dtype=torch.float32, device="cuda")
    post = torch.empty((n, dec.kldpc), dtype=torch.float32, device="cuda")
    cod = np.ascontiguousarray(cod, dtype=np.int8)
    r = L.drx_learned_forward(dec.h, n, llr16.data_ptr(), llr16.stride(0), bits.data_ptr(), bits.stride(0), iters,
                              b16.data_ptr(), a16.data_ptr(), b16.shape[1], cod.ctypes.data, loss.data_ptr(),
                              post.data_ptr(), ws.data_ptr(), ws_bytes, 0, stream_handle(torch.cuda.current_stream()))
    if r:
        raise RuntimeError("drx_learned_forward: " + last_error())
    return loss, post


class LearnedDecoder(torch.nn.Module):
    """Scale and offset tables (iters x check-degree classes) of one code,
    fp32 masters of the FP16 values the decoder uses; initialised to the
    plain decoder (scale 1, offset 1)."""

    def __init__(self, short_frame, rate, iters=20, params=None, weights=None):
        super().__init__()
        from . import FecParams, code_info, fec_lookup
        try:
            p = params or fec_lookup(short_frame, rate)
        except KeyError:
            info = code_info(short_frame, rate)
            p = FecParams(int(bool(short_frame)), info.nldpc, info.K, info.K, 0)
        self.dec = Ldpc(p, rate)
        self.iters = iters
        self.degrees, self.cod = degree_classes(short_frame, rate)
        nclass = len(self.degrees)
        self.beta = torch.nn.Parameter(torch.ones(iters, nclass, device="cuda"))
        self.alpha = torch.nn.Parameter(torch.ones(iters, nclass, device="cuda"))
        self._work = {}
        self.weights = weights

    def forward(self, llr16, bits):
        n = llr16.shape[0]
        key = n
        if key not in self._work:
            self._work[key] = _Work(self.dec, n, self.iters, self.cod, self.weights)
        return LearnedMinSum.apply(self.beta, self.alpha, self.dec, llr16, bits, self.iters, self.cod,
                                   self._work[key])

    def fp16_tables(self):
        return self.beta.detach().half(), self.alpha.detach().half()
