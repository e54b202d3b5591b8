"""The C-ABI library on the CPU: it loads, exports every declared symbol, and
its host-side logic (FEC lookup, code compiler) matches the reference.  No
kernel runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

import dvbrx_b200 as D
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dvbrx_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(drx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(D.LIB_PATH)
    syms = declared_symbols()
    assert "drx_ldpc_decode" in syms and "drx_fec_lookup" in syms
    for s in syms:
        assert hasattr(lib, s), s
    assert set(D.EXPORTS) <= set(syms)


def fec_rates(short):
    text = open(os.path.join(ROOT, "dvbrx_b200", "csrc", "codes_gen.h")).read()
    body = text[text.index("cg_fec_%s[]" % ("short" if short else "normal")):]
    body = body[: body.index("};")]
    return re.findall(r'\{ "(\w+)",', body)


@pytest.mark.parametrize("short", [0, 1])
def test_fec_lookup_matches_reference(short):
    rates = fec_rates(short)
    assert len(rates) == (22 if short else 35)
    ref = oracle.load_ref() if oracle.ref_available() else None
    for rate in rates:
        p = D.fec_lookup(short, rate)
        assert p.nldpc == (16200 if short else 64800) and p.short_frame == short
        if ref is not None:
            q = oracle.FecParams()
            assert ref.ref_fec_lookup(short, rate.encode(), ctypes.byref(q)) == 0
            assert (p.nldpc, p.kldpc, p.kbch, p.t) == (q.nldpc, q.kldpc, q.kbch, q.t), rate
    with pytest.raises(KeyError):
        D.fec_lookup(short, "7_7")


def test_lanes():
    assert D.lanes() == 64


# steps per iteration from the wavefront analysis of the tables
LEVELS = {(0, "3_5"): 293, (1, "1_2"): 84, (0, "1_3"): 420, (0, "3_4"): 349, (0, "2_3"): 262,
          (0, "9_10"): 197, (1, "3_5"): 235, (0, "2_3_t2"): 147}


def test_code_compiler_levels():
    for (short, rate), n in LEVELS.items():
        info = D.code_info(short, rate)
        assert info.steps == n and info.levelled == 1, rate
    # S2X tables have no intra-layer conflicts: one step per layer
    for short, rate in ((0, "13_45"), (0, "154_180"), (1, "32_45"), (0, "18_30"), (1, "3_5_t2")):
        info = D.code_info(short, rate)
        assert info.steps == info.q and info.levelled == 0, rate


def test_code_compiler_geometry_matches_restatement():
    """N, K, q and the check degree of the compiled code agree with the
    restatement's walk of the same table (ldpc.c:199-260)."""
    for short, rate in ((0, "3_5"), (1, "1_2"), (0, "9_10"), (1, "8_9"), (0, "1_4"), (0, "22_30")):
        info = D.code_info(short, rate)
        o = oracle.OrcCode(short, rate)
        assert (info.nldpc, info.K, info.q, info.deg_max) == (o.N, o.K, o.q, o.cnl + 2), rate


def test_unknown_rate():
    with pytest.raises(KeyError):
        D.code_info(0, "1_1")


def _cuda_device_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_device_present(), reason="checks the no-device error path")
def test_new_without_device_fails_loudly():
    p = D.fec_lookup(0, "3_5")
    with pytest.raises(RuntimeError):
        D.Ldpc(p, "3_5")
    assert D.last_error() != ""


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "dvbrx_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "from oracle" not in text, f
                assert "liborc" not in text and "libref_" not in text, f
