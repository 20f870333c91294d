"""The CPU oracle's restated device math against golden vectors produced by
sundog's own device headers (tests/golden/make_golden.py): bit-exact."""

import glob
import os

import numpy as np
import pytest

from oracle import items, oracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "fnvec_*.npz")))


def load_golden(path):
    z = np.load(path)
    which, n = int(z["which"]), int(z["n"])
    _, din, dout = items.ITEMS[which]
    return which, n, z["input"].tobytes(), np.frombuffer(z["output"].tobytes(), dout)


def test_golden_files_present():
    names = {os.path.basename(p) for p in GOLDEN}
    for k in ("pcg", "bsdf_eval", "bsdf_draw", "quadric", "light", "flame", "noise", "cdf_search"):
        assert "fnvec_%s.npz" % k in names


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[6:-4] for p in GOLDEN])
def test_oracle_matches_reference_bit_exact(oracle_lib, path):
    which, n, payload, ref = load_golden(path)
    got = oracle.fn(which, payload, n, ref.dtype)
    assert got.tobytes() == ref.tobytes()


def test_pcg_stream_known_answers():
    # PCG32 reference implementation (pcg_basic.c): pcg32_srandom_r(42, 54)
    # yields 0xa15c02b7 0x7b47f409 0xba1d3330 0x83d2f293 0xbfa4784b 0xcbed606e.
    a = np.zeros(1, items.ITEMS[1][1])
    a["seed"], a["seq"] = 42, 54
    out = oracle.fn(1, a.tobytes(), 1, items.ITEMS[1][2])
    assert list(out["next"][0][:6]) == [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293,
                                        0xbfa4784b, 0xcbed606e]
