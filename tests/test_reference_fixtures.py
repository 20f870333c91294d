"""The reference-image fixtures on the CPU: each recorded C-ABI call stream
(tests/golden/abi_<scene>.json, from sundog's own scene library) replays
through this library with every call returning what it returned when
recorded, and builds a scene that validates; the decoded goldens are
256x256 RGB; the PQ restatement maps linear 1.0 to the BT.2408 reference
white (203 cd/m^2 -> PQ 0.5807 -> 12-bit code 2378)."""

import json
import os

import numpy as np
import pytest
from PIL import Image

from oracle import film_pq

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("scene", ["smoke", "01-marble-run", "02-cornell-lume"])
def test_call_stream_replays(lib, scene):
    from test_gpu_reference_images import replay
    with open(os.path.join(GOLDEN, "abi_%s.json" % scene)) as f:
        calls = json.load(f)["calls"]
    h = replay(lib, calls)
    try:
        assert lib.sundog_scene_validate(h) == 0
    finally:
        lib.sundog_scene_destroy(h)
    img = np.array(Image.open(os.path.join(GOLDEN, "ref_%s.png" % scene)))
    assert img.shape == (256, 256, 3) and img.dtype == np.uint8


def test_pq_reference_white():
    assert film_pq.pq_codes12(np.ones((1, 1, 3), np.float32))[0, 0, 0] == 2378
    assert film_pq.pq_codes12(np.zeros((1, 1, 3), np.float32))[0, 0, 0] == 0
    assert film_pq.pq_codes12(np.full((1, 1, 3), 1e6, np.float32))[0, 0, 0] == 4095
