"""ORACLE — test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker: the product library
(``dvbrx_b200``) never loads anything from here.

Two checkers live here:

* ``liborc.so`` (``ldpc_oracle.c``): this project's scalar C restatement of the
  reference decoder ``libdvbrx/src/ldpc.c`` (see that file's header).
* ``_ref/libref_<isa>.so``: the reference's own ``ldpc.c`` / ``bch.c`` /
  ``demap.c`` compiled from its sources by ``oracle/Makefile`` (exported
  ``drx_*`` names renamed ``ref_*``).  Built where the reference tree exists and
  carried, as a built file, to machines where it does not.

``datagen`` makes seeded test frames: the project's encoder (accumulator rule),
the DVB-S2 bit interleaver and constellations, AWGN and the max-log int8 LLR
quantiser of ``libdvbrx/src/demap.c:225-229,491-533``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")


class FecParams(ctypes.Structure):
    """``drx_fec_params`` (reference ``libdvbrx/include/dvbrx/fec.h:13-19``)."""

    _fields_ = [
        ("short_frame", ctypes.c_int),
        ("nldpc", ctypes.c_int),
        ("kldpc", ctypes.c_int),
        ("kbch", ctypes.c_int),
        ("t", ctypes.c_int),
    ]


def cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def cpu_info():
    """The host CPU: model name, vendor family/model, logical CPUs this
    process may use and physical cores (distinct (package, core) pairs)."""
    model, vendor, family, mnum = "unknown", "", -1, -1
    cores = set()
    pkg = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model == "unknown":
                    model = v
                elif k == "vendor_id" and not vendor:
                    vendor = v
                elif k == "cpu family" and family < 0:
                    family = int(v)
                elif k == "model" and mnum < 0:
                    mnum = int(v)
                elif k == "physical id":
                    pkg = v
                elif k == "core id":
                    core = v
                elif not k and pkg is not None:
                    cores.add((pkg, core))
                    pkg = core = None
        if pkg is not None:
            cores.add((pkg, core))
    except OSError:
        pass
    try:
        logical = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        logical = os.cpu_count() or 1
    return {"model": model, "vendor": vendor, "family": family, "model_number": mnum,
            "logical_cpus": logical, "physical_cores": len(cores) or None}


def native_arch():
    """The gcc -march name of this host's CPU among the oracle's native
    builds (oracle/Makefile NATIVE_ARCHS), or None."""
    c = cpu_info()
    if c["vendor"] == "GenuineIntel" and c["family"] == 6:
        return {143: "sapphirerapids", 207: "emeraldrapids", 173: "graniterapids",
                174: "graniterapids"}.get(c["model_number"])
    if c["vendor"] == "AuthenticAMD":
        if c["family"] == 25 and (0x10 <= c["model_number"] <= 0x1F or 0xA0 <= c["model_number"] <= 0xAF):
            return "znver4"
        if c["family"] == 26:
            return "znver5"
    return None


def best_ref_flavour():
    """The reference build for this host: the one compiled for its CPU
    (what -march=native gives) if present, else the widest portable one
    its instruction set runs."""
    arch = native_arch()
    if arch and os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % arch)):
        return arch
    flags = cpu_flags()
    if "avx512bw" in flags and "avx512vl" in flags and "avx512dq" in flags:
        return "avx512"
    if "avx2" in flags and "fma" in flags:
        return "avx2"
    return "sse2"


MARCH = {"avx512": "x86-64-v4", "avx2": "x86-64-v3", "sse2": "x86-64-v2"}


def flavour_march(flavour):
    """The -march a reference build was compiled with."""
    return MARCH.get(flavour, flavour)


_orc = None
_ref = {}


def load_orc():
    """The restatement library (built by ``make -C oracle``)."""
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_PATH):
            raise FileNotFoundError(ORC_PATH + " missing: run `make -C oracle`")
        lib = ctypes.CDLL(ORC_PATH)
        vp, ip, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p
        lib.orc_new.restype = vp
        lib.orc_new.argtypes = [ip, cp, ip]
        lib.orc_free.argtypes = [vp]
        for f in ("orc_n", "orc_k", "orc_q", "orc_cnl", "orc_comp"):
            getattr(lib, f).argtypes = [vp]
            getattr(lib, f).restype = ip
        lib.orc_fec_lookup.argtypes = [ip, cp] + [ctypes.POINTER(ctypes.c_int)] * 4
        lib.orc_decode_group.argtypes = [vp, vp, vp, ip, ip]
        lib.orc_decode_frame.argtypes = [vp, vp, vp, ip, ctypes.POINTER(ctypes.c_int)]
        lib.orc_decode_frames.argtypes = [vp, vp, vp, vp, vp, ip, ip]
        lib.orc_encode.argtypes = [vp, vp, vp]
        lib.orc_decode_frame_learned.argtypes = [vp, vp, vp, ip, vp, vp, ip, vp]
        lib.orc_decode_frame_learned.restype = ip
        lib.orc_bch_encode.argtypes = [ip, ip, ip, ip, vp, vp]
        lib.orc_bch_encode.restype = ip
        _orc = lib
    return _orc


def ref_available(flavour=None):
    flavour = flavour or best_ref_flavour()
    return os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % flavour))


def load_ref(flavour=None):
    """The reference compiled from its own sources, or None if not built."""
    flavour = flavour or best_ref_flavour()
    if flavour in _ref:
        return _ref[flavour]
    path = os.path.join(REF_DIR, "libref_%s.so" % flavour)
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    vp, ip, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p
    lib.ref_ldpc_lanes.restype = ip
    lib.ref_ldpc_new.restype = vp
    lib.ref_ldpc_new.argtypes = [ctypes.POINTER(FecParams), cp]
    lib.ref_ldpc_free.argtypes = [vp]
    lib.ref_ldpc_decode.argtypes = [vp, vp, vp, ip, ip]
    lib.ref_ldpc_decode.restype = ip
    lib.ref_fec_lookup.argtypes = [ip, cp, ctypes.POINTER(FecParams)]
    lib.ref_fec_lookup.restype = ip
    lib.ref_demap_new.restype = vp
    lib.ref_demap_new.argtypes = [cp, cp, ip]
    lib.ref_demap_free.argtypes = [vp]
    lib.ref_demap_frame.argtypes = [vp, vp, ctypes.c_float, vp]
    lib.ref_demap_symbols.argtypes = [vp]
    lib.ref_demap_symbols.restype = ip
    sz, dp = ctypes.c_size_t, ctypes.c_double
    if hasattr(lib, "refx_bench"):
        fp = ctypes.POINTER(FecParams)
        lib.refx_decode_frames_mt.argtypes = [fp, cp, vp, sz, ip, ip, vp, sz, vp, vp, ip]
        lib.refx_decode_frames_mt.restype = ip
        lib.refx_decode_groups_mt.argtypes = [fp, cp, vp, sz, ip, ip, ip, vp, sz, vp, ip]
        lib.refx_decode_groups_mt.restype = ip
        lib.refx_bench.argtypes = [fp, cp, vp, sz, ip, ip, ip, ip, ip, ip, dp, vp,
                                   ctypes.POINTER(ctypes.c_longlong)]
        lib.refx_bench.restype = ip
    _ref[flavour] = lib
    return lib


def host_threads():
    """Threads for the reference's CPU work: every logical CPU this process
    may use."""
    return cpu_info()["logical_cpus"]


def fec_params(short_frame, rate):
    """FEC parameters of a rate as the restatement's lookup gives them; the
    T2 codes (absent from the BCH table) get nbch = K of their LDPC table."""
    lib = load_orc()
    n, k, kb, t = (ctypes.c_int() for _ in range(4))
    if lib.orc_fec_lookup(int(short_frame), rate.encode(), ctypes.byref(n), ctypes.byref(k),
                          ctypes.byref(kb), ctypes.byref(t)) == 0:
        return FecParams(int(short_frame), n.value, k.value, kb.value, t.value)
    h = lib.orc_new(int(short_frame), rate.encode(), 0)
    if not h:
        raise KeyError(rate)
    N, K = lib.orc_n(h), lib.orc_k(h)
    lib.orc_free(h)
    return FecParams(int(short_frame), N, K, K, 0)


def _ptr_array(rows):
    arr = (ctypes.c_void_p * len(rows))()
    for i, r in enumerate(rows):
        arr[i] = r.ctypes.data
    return arr


def bch_encode(short_frame, rate, msgs):
    """DVB-S2 BCH codewords of packed kbch-bit messages [n, >= ceil(kbch/8)]:
    [n, kldpc/8] packed, MSB first (the oracle's encoder, checked by the
    reference's decoder finding no error)."""
    p = fec_params(short_frame, rate)
    lib = load_orc()
    msgs = np.ascontiguousarray(msgs, dtype=np.uint8)
    out = np.zeros((msgs.shape[0], p.kldpc // 8), np.uint8)
    for f in range(msgs.shape[0]):
        row = np.concatenate([msgs[f], np.zeros(8, np.uint8)])
        if lib.orc_bch_encode(int(short_frame), p.t, p.kbch, p.kldpc, row.ctypes.data, out[f].ctypes.data) < 0:
            raise ValueError(rate)
    return out


class RefBch:
    """The reference's BCH decoder (bch.c) compiled from its sources."""

    def __init__(self, short_frame, rate):
        self.lib = load_ref()
        if self.lib is None:
            raise RuntimeError("reference build missing")
        vp = ctypes.c_void_p
        self.lib.ref_bch_new.restype = vp
        self.lib.ref_bch_new.argtypes = [ctypes.POINTER(FecParams)]
        self.lib.ref_bch_free.argtypes = [vp]
        self.lib.ref_bch_decode.argtypes = [vp, vp]
        self.lib.ref_bch_decode.restype = ctypes.c_int
        self.params = fec_params(short_frame, rate)
        self.h = self.lib.ref_bch_new(ctypes.byref(self.params))

    def decode(self, words):
        """In a copy: (corrected words, results)."""
        w = np.ascontiguousarray(words, dtype=np.uint8).copy()
        res = np.zeros(w.shape[0], np.int32)
        for f in range(w.shape[0]):
            res[f] = self.lib.ref_bch_decode(self.h, w[f].ctypes.data)
        return w, res

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_bch_free(self.h)


def learned_words(scale, offset):
    """Learned tables [iters, nclass] as the decoder's Q8 words
    [iters, 8]: round-half-even(256 scale) clamped to [0, 65535] in the low
    half, round-half-even(256 offset) clamped to [-32768, 32767] in the high
    half."""
    b = np.asarray(scale, dtype=np.float32)
    a = np.asarray(offset, dtype=np.float32)
    bq = np.clip(np.rint(b * np.float32(256)), 0, 65535).astype(np.int64)
    aq = np.clip(np.rint(a * np.float32(256)), -32768, 32767).astype(np.int64)
    w = np.zeros((b.shape[0], 8), np.uint32)
    w[:, : b.shape[1]] = (bq | ((aq & 0xFFFF) << 16)).astype(np.uint32)
    return np.ascontiguousarray(w)


class OrcCode:
    """The restatement for one code."""

    def __init__(self, short_frame, rate, kldpc=None):
        self.lib = load_orc()
        self.params = fec_params(short_frame, rate)
        if kldpc is None:
            kldpc = self.params.kldpc
        self.kldpc = kldpc
        self.h = self.lib.orc_new(int(short_frame), rate.encode(), int(kldpc))
        if not self.h:
            raise KeyError(rate)
        self.N = self.lib.orc_n(self.h)
        self.K = self.lib.orc_k(self.h)
        self.q = self.lib.orc_q(self.h)
        self.cnl = self.lib.orc_cnl(self.h)
        self.comp = self.lib.orc_comp(self.h)
        self.nbytes = (kldpc + 7) // 8

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_free(self.h)
            self.h = None

    def encode(self, info):
        info = np.ascontiguousarray(info, dtype=np.uint8)
        out = np.empty(info.shape[:-1] + (self.N,), np.uint8)
        for f in range(info.shape[0]):
            self.lib.orc_encode(self.h, info[f].ctypes.data, out[f].ctypes.data)
        return out

    def decode_frames(self, llr, max_iter):
        """Each frame on its own: hard bits, iterations, syndrome flags."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        it = np.zeros(n, np.int32)
        ok = np.zeros(n, np.uint8)
        self.lib.orc_decode_frames(self.h, llr.ctypes.data, out.ctypes.data, it.ctypes.data,
                                   ok.ctypes.data, n, max_iter)
        return out, it, ok

    def decode_frames_learned(self, llr, max_iter, scale, offset, class_of_degree):
        """This project's learned decoder at int8 (each frame on its own):
        the scale / offset tables [iters, nclass] are rounded to Q8 as the
        library does.  Hard bits, iterations, syndrome flags."""
        words = learned_words(scale, offset)
        cls = np.ascontiguousarray(np.asarray(class_of_degree, dtype=np.int8))
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        it = np.zeros(n, np.int32)
        ok = np.zeros(n, np.uint8)
        for f in range(n):
            itf = ctypes.c_int()
            ok[f] = self.lib.orc_decode_frame_learned(self.h, llr[f].ctypes.data, out[f].ctypes.data, max_iter,
                                                      ctypes.byref(itf), words.ctypes.data, words.shape[0],
                                                      cls.ctypes.data)
            it[f] = itf.value
        return out, it, ok

    def decode_group(self, llr, max_iter):
        """The frames decoded together, reference batch semantics."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        rows_in = [llr[f] for f in range(n)]
        rows_out = [out[f] for f in range(n)]
        r = self.lib.orc_decode_group(self.h, _ptr_array(rows_in), _ptr_array(rows_out), n, max_iter)
        return out, r


class RefCode:
    """The reference decoder compiled from its own sources."""

    def bench(self, pool, max_iter, threads, steps=1, calls_per_step=1, seconds=0.0, lanes=None):
        """The reference's production mode on `pool` (int8 frames): worker
        threads with their own handles decoding `lanes`-frame calls
        (refbench.c).  Returns (seconds of every step, calls made)."""
        lanes = lanes or self.lanes
        pool = np.ascontiguousarray(pool, dtype=np.int8)
        nsteps = 1 if seconds > 0 else steps
        step_s = np.zeros(nsteps, np.float64)
        calls = ctypes.c_longlong()
        if self.lib.refx_bench(ctypes.byref(self.params), self.rate.encode(), pool.ctypes.data, pool.strides[0],
                               pool.shape[0], max_iter, lanes, threads, steps, calls_per_step, float(seconds),
                               step_s.ctypes.data, ctypes.byref(calls)):
            raise RuntimeError("reference benchmark failed")
        return step_s, calls.value

    def __init__(self, short_frame, rate, flavour=None, params=None):
        self.lib = load_ref(flavour)
        if self.lib is None:
            raise FileNotFoundError("reference oracle not built (make -C oracle ref)")
        self.lanes = self.lib.ref_ldpc_lanes()
        p = params if params is not None else fec_params(short_frame, rate)
        self.params = FecParams(p.short_frame, p.nldpc, p.kldpc, p.kbch, p.t)
        self.h = self.lib.ref_ldpc_new(ctypes.byref(self.params), rate.encode())
        if not self.h:
            raise KeyError(rate)
        self.rate = rate
        self.flavour = flavour or best_ref_flavour()
        self.N = self.params.nldpc
        self.nbytes = (self.params.kldpc + 7) // 8

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_ldpc_free(self.h)
            self.h = None

    def decode_call(self, llr, max_iter):
        """One drx_ldpc_decode call (n <= lanes frames)."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        r = self.lib.ref_ldpc_decode(self.h, _ptr_array([llr[f] for f in range(n)]),
                                     _ptr_array([out[f] for f in range(n)]), n, max_iter)
        return out, r

    def decode_frames(self, llr, max_iter):
        """Per-frame semantics: one call per frame (nframes = 1)."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        it = np.zeros(n, np.int32)
        ok = np.zeros(n, np.uint8)
        for f in range(n):
            o, r = self.decode_call(llr[f:f + 1], max_iter)
            out[f] = o[0]
            it[f] = max_iter if r < 0 else r
            ok[f] = r >= 0
        return out, it, ok

    def decode_frames_mt(self, llr, max_iter, threads=None):
        """Per-frame semantics (one call per frame) on host threads, each
        with its own handle (refbench.c): hard bits, iterations, flags."""
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        it = np.zeros(n, np.int32)
        ok = np.zeros(n, np.uint8)
        if n and self.lib.refx_decode_frames_mt(ctypes.byref(self.params), self.rate.encode(), llr.ctypes.data,
                                                llr.strides[0], n, max_iter, out.ctypes.data, out.strides[0],
                                                it.ctypes.data, ok.ctypes.data, threads or host_threads()):
            raise RuntimeError("reference per-frame decode failed")
        return out, it, ok

    def decode_groups_mt(self, llr, max_iter, group=None, threads=None):
        """Consecutive groups of ``group`` frames (default: lanes), one call
        each, on host threads: hard bits and the per-group return values."""
        group = group or self.lanes
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        rets = np.zeros((n + group - 1) // group, np.int32)
        if n and self.lib.refx_decode_groups_mt(ctypes.byref(self.params), self.rate.encode(), llr.ctypes.data,
                                                llr.strides[0], n, group, max_iter, out.ctypes.data,
                                                out.strides[0], rets.ctypes.data, threads or host_threads()):
            raise RuntimeError("reference group decode failed")
        return out, rets

    def decode_groups(self, llr, max_iter, group=None):
        """Consecutive groups of ``group`` (default: lanes) frames, one call
        each: hard bits and the per-group return values."""
        group = group or self.lanes
        llr = np.ascontiguousarray(llr, dtype=np.int8)
        n = llr.shape[0]
        out = np.zeros((n, self.nbytes), np.uint8)
        rets = []
        for f0 in range(0, n, group):
            o, r = self.decode_call(llr[f0:f0 + group], max_iter)
            out[f0:f0 + group] = o
            rets.append(r)
        return out, np.array(rets, np.int32)
