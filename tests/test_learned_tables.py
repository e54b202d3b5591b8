"""The committed learned tables (dvbrx_b200/learned_tables/*.json), on the
CPU: each one loads into the layout drx_ldpc_set_learned takes (iterations x
degree classes, at most 32 iterations and 8 classes), its Q8 words fit the
kernel's 16-bit scale and signed 16-bit offset, its degree classes are the
code's own check degrees (the schedule of the compiled code), and the tables
bench.py runs are there."""
import glob
import json
import os

import numpy as np
import pytest

from dvbrx_b200 import learned as Lm
from dvbrx_b200 import train

TABLES = sorted(glob.glob(os.path.join(train.TABLES, "*.json")))


def test_tables_present():
    names = {os.path.basename(p) for p in TABLES}
    # the bench's learned lines: 12 iterations with fallback, 30 in one pass
    assert "normal_3_5_8psk_12it.json" in names
    assert "normal_3_5_8psk_30it.json" in names
    # the config-4 table
    assert "normal_2_3_8psk_20it.json" in names


@pytest.mark.parametrize("path", TABLES, ids=[os.path.basename(p) for p in TABLES])
def test_table_layout(path):
    t = json.load(open(path))
    scale = np.asarray(t["scale"], np.float64)
    offset = np.asarray(t["offset"], np.float64)
    cod = np.asarray(t["class_of_degree"])
    iters = int(t["iters"])
    assert 1 <= iters <= 32
    assert scale.shape == offset.shape == (iters, len(t["degrees"]))
    assert 1 <= scale.shape[1] <= 8
    assert np.isfinite(scale).all() and np.isfinite(offset).all()
    # Q8 words: scale unsigned 16 bits, offset signed 16 bits
    assert (np.round(scale * 256) >= 0).all() and (np.round(scale * 256) < 65536).all()
    assert (np.abs(np.round(offset * 256)) < 32768).all()
    assert cod.shape == (33,) and cod.min() >= 0 and cod.max() < scale.shape[1]
    # the classes are the code's check degrees, in order
    degs, want = Lm.degree_classes(int(t["short"]), t["rate"])
    assert list(t["degrees"]) == degs
    assert np.array_equal(cod, want)
    # the file name is the one train.load_table looks for
    assert os.path.basename(path) == os.path.basename(
        train.table_path(int(t["short"]), t["rate"], t["constellation"], iters))
