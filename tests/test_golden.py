"""The oracle reproduces the committed golden fixtures bit for bit.  The
fixtures come from the reference's own shader code compiled on the host
(tests/golden/make_golden.py); samples whose value the reference leaves
undefined (an out-of-range buffer read) are left out."""
import os
import sys

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

import make_golden  # noqa: E402


def test_cornell_golden():
    gold = np.load(os.path.join(HERE, "cornell_64x64.npz"))
    got = make_golden.cornell_oracle().reshape(-1, 3)
    ref = gold["samples"].reshape(-1, 3)
    defined = ~gold["undefined"]
    assert defined.mean() > 0.9
    assert np.array_equal(got[defined].view(np.uint32), ref[defined].view(np.uint32))
    assert np.isfinite(got).all() and got.mean() > 0.01


def test_soup_golden():
    gold = np.load(os.path.join(HERE, "soup_trace.npz"))
    closest, anyh = make_golden.soup_oracle()
    assert np.array_equal(closest, gold["closest"])
    assert np.array_equal(anyh, gold["any"])
    assert (closest[:, 3] != 0xFFFFFFFF).sum() > 20
