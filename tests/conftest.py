import json
import os
import sys

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
