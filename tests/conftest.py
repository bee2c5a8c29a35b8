import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gsplat-rs_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(GOLDEN, "kats.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def minimal_scene():
    import gsplat_scenes
    with open(os.path.join(GOLDEN, "minimal_ascii_scene.json")) as f:
        return gsplat_scenes.scene_from_json(json.load(f))


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.lib()
    return oracle_py


def lcg_seq(seed, n, mul=1664525, inc=1013904223):
    out = []
    s = seed & 0xFFFFFFFF
    for _ in range(n):
        s = (s * mul + inc) & 0xFFFFFFFF
        out.append(s)
    return out


def assert_fp32_image(img, ref, label=""):
    """The CUDA FP32 raster's RGBA8 image against the oracle's FP32 tile
    model. The device takes 2^t from the hardware base-2 exponential, the
    model from a degree-6 polynomial (both within a few 1e-7 of e^x), and
    every other operation is the same, so the images differ only where a
    weight sits on the 1/256 threshold or a channel on a rounding boundary:
    at most 2 steps, on at most 1e-4 of the channels."""
    img = np.asarray(img)
    ref = np.asarray(ref)
    assert img.shape == ref.shape, (label, img.shape, ref.shape)
    d = np.abs(img.astype(np.int16) - ref.astype(np.int16))
    assert int(d.max(initial=0)) <= 2, (label, int(d.max()))
    changed = int(np.count_nonzero(d))
    assert changed <= max(16, 1e-4 * d.size), (label, changed, d.size)
