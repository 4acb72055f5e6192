"""The oracle reproduces the committed golden fixtures bit for bit (guards
the restatement against drift; tests/golden/make_golden.py made them)."""
import os
import sys

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

import make_golden  # noqa: E402


def test_cornell_golden():
    gold = np.load(os.path.join(HERE, "cornell_64x64.npz"))
    got = make_golden.cornell_samples()
    assert np.array_equal(got.view(np.uint32), gold["samples"].view(np.uint32))
    assert np.isfinite(got).all() and got.mean() > 0.01


def test_soup_golden():
    gold = np.load(os.path.join(HERE, "soup_trace.npz"))
    _, closest, anyh = make_golden.soup_records()
    assert np.array_equal(closest, gold["closest"])
    assert np.array_equal(anyh, gold["any"])
    assert (closest[:, 3] != 0xFFFFFFFF).sum() > 20
