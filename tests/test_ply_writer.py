"""The scene module's PLY writer inverts the loader's RDF -> RUF conversion:
a written scene loads back bit for bit through the host PLY path (CPU)."""

import numpy as np
import pytest

import gsplat_ffi as ffi
import gsplat_scenes


@pytest.mark.parametrize("degree,big", [(0, False), (1, True), (3, False), (4, True)])
def test_written_scene_loads_back_bit_for_bit(tmp_path, degree, big):
    rng = np.random.default_rng(degree)
    scene = gsplat_scenes.make_scene(rng, gsplat_scenes.gmm_means(rng, 777), -4.5, 0.7, 0.5, 1.5,
                                     degree)
    path = str(tmp_path / "s.ply")
    gsplat_scenes.write_ply(path, scene, big_endian=big)
    back = ffi.ply_load(path)
    assert back["sh_degree"] == degree
    for k in ("positions", "opacity", "scale_xyz", "rotation_xyzw", "color_dc", "sh_rest"):
        if scene.get(k) is None:
            continue
        a = np.asarray(scene[k], np.float32).reshape(-1)
        b = np.asarray(back[k], np.float32).reshape(-1)
        assert a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
