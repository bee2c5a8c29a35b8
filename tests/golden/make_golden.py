"""Regenerates the golden fixtures under tests/golden/ from the reference tree.

Run with REFERENCE_ROOT naming a checkout of the reference project (read
only; the variable is required):

    REFERENCE_ROOT=/path/to/gsplat-rs python tests/golden/make_golden.py

What it writes (all small, committed):
  minimal_ascii.ply, minimal_binary.ply  byte copies of the reference's
      tests/datasets fixtures, so scene-loading tests run where the reference
      tree is absent.
  minimal_ascii_scene.json  minimal_ascii.ply decoded into SceneBuffers the way
      crates/gsplat-io-ply/src/lib.rs:76-113 does (wxyz -> xyzw, then the
      RDF -> RUF y flip, quaternion x/z negation).
  kats.json  known-answer values quoted from the reference's own tests; every
      quoted value is checked to appear verbatim in the cited source file, so a
      drifting reference makes this script fail instead of silently writing
      stale expectations.
"""

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE_ROOT", "")
if not REF or not os.path.isdir(REF):
    raise SystemExit("REFERENCE_ROOT must name a checkout of the reference project "
                     "(misotofu0525/gsplat-rs); got " + repr(REF))


def ref_text(rel):
    with open(os.path.join(REF, rel), "r", encoding="utf-8") as f:
        return f.read()


def require(rel, *snippets):
    text = ref_text(rel)
    for s in snippets:
        if s not in text:
            raise SystemExit(f"reference drift: {rel} no longer contains {s!r}")


def parse_ascii_ply(path):
    with open(path, "r", encoding="utf-8") as f:
        lines = [ln.strip() for ln in f]
    props, count, i = [], 0, 0
    while lines[i] != "end_header":
        parts = lines[i].split()
        if parts[:2] == ["element", "vertex"]:
            count = int(parts[2])
        elif parts and parts[0] == "property":
            props.append(parts[2])
        i += 1
    rows = [ln for ln in lines[i + 1:] if ln and not ln.startswith("comment")][:count]
    return props, [[float(x) for x in r.split()] for r in rows]


def decode_scene(props, rows):
    idx = {p: k for k, p in enumerate(props)}
    scene = {"positions": [], "opacity": [], "scale_xyz": [], "rotation_xyzw": [],
             "color_dc": [], "sh_degree": 0, "sh_rest": None}
    for r in rows:
        x, y, z = r[idx["x"]], r[idx["y"]], r[idx["z"]]
        scene["positions"].append([x, -y, z])  # RDF -> RUF
        scene["opacity"].append(r[idx["opacity"]])
        scene["scale_xyz"].append([r[idx[f"scale_{k}"]] for k in range(3)])
        w, qx, qy, qz = (r[idx[f"rot_{k}"]] for k in range(4))
        scene["rotation_xyzw"].append([-qx, qy, -qz, w])
        scene["color_dc"].append([r[idx[f"f_dc_{k}"]] for k in range(3)])
    return scene


def main():
    if not os.path.isdir(REF):
        raise SystemExit(f"reference tree not found at {REF}")
    for name in ("minimal_ascii.ply", "minimal_binary.ply"):
        with open(os.path.join(REF, "tests/datasets", name), "rb") as f:
            data = f.read()
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)

    props, rows = parse_ascii_ply(os.path.join(REF, "tests/datasets/minimal_ascii.ply"))
    with open(os.path.join(HERE, "minimal_ascii_scene.json"), "w") as f:
        json.dump(decode_scene(props, rows), f, indent=1)

    conf = "crates/gsplat-render-wgpu/tests/conformance_sorted_alpha.rs"
    require(conf, "width: 64", "height: 64", "assert_eq!(stats.visible_count, 2);",
            "assert_eq!(stats.drawn_count, 2);",
            "let expected_means = [0.4194_f32, 0.3234, 0.3073, 0.5712];",
            "(actual - expected).abs() <= 0.035")
    sort = "crates/gsplat-sort/src/lib.rs"
    require(sort, "let mut keys = [20_u32, 5, 12];", "assert_eq!(keys, [20, 12, 5]);",
            "assert_eq!(values, [0, 2, 1]);", "let keys = [20_u32, 5, 12, 12];",
            "assert_eq!(values, [0, 2, 3, 1]);",
            "let mut keys = [10_u32, 2, 7, 7, 100, 1];",
            "assert_eq!(keys, [100, 10, 7, 7, 2, 1]);",
            "assert_eq!(values, [4, 0, 2, 3, 1, 5]);",
            "for &len in &[0_usize, 1, 2, 255, 256, 257, 1024, 65537]",
            "let mut seed = 42_u32.wrapping_add(len as u32);", "let len = 4099;",
            "state.wrapping_mul(1664525).wrapping_add(1013904223)")
    order = "crates/gsplat-render-wgpu/src/direct_gpu_order.rs"
    require(order, "for count in [255_usize, 256, 257, 4099]", "0 => 0,", "1 => u32::MAX,",
            "_ => ((index * 2_654_435_761_usize) as u32) & 0x00ff_ffff,",
            "id: (count - index) as u32,", "(0..257).map(|id| GpuSortPair { key: 42, id })")
    render = "crates/gsplat-render-wgpu/src/lib.rs"
    require(render, "Vec3f::new(0.0, 0.0, 2000.0),",
            "assert_eq!(renderer.current_sorted_indices(), &[1, 2, 0]);",
            "Vec3f::new(0.2, -0.1, 2.0)", "scale_xyz: vec![[0.8, -0.4, -0.4]],",
            "positions: vec![Vec3f::new(2.3, 0.0, 1.0)],", "scale_xyz: vec![[2.0, 2.0, 2.0]],")
    ply = "crates/gsplat-io-ply/src/lib.rs"
    require(ply, "assert_eq!(result.scene.rotation_xyzw[0], [-0.2, 0.3, -0.4, 0.9]);",
            "assert_eq!(sh[0], -0.01);", "assert_eq!(sh[3], -0.04);",
            "-1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0, 1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0,",
            "const OPACITY_LOGIT_LIMIT: f32 = 16.0;")
    core = "crates/gsplat-core/src/lib.rs"
    require(core, "const CAMERA_ROTATION_NORM2_TOLERANCE: f32 = 1.0e-3;",
            "camera.pose.rotation_xyzw = [0.0, 0.0, 0.0, 2.0];",
            "camera.intrinsics.near_plane = 10.0;")

    kats = {
        "conformance": {
            "source": conf + ":14-77",
            "size": [64, 64],
            "visible": 2,
            "drawn": 2,
            "channel_means": [0.4194, 0.3234, 0.3073, 0.5712],
            "tolerance": 0.035,
        },
        "sort_pairs_small": {"source": sort + ":602-612", "keys": [20, 5, 12],
                             "values": [0, 1, 2], "keys_out": [20, 12, 5],
                             "values_out": [0, 2, 1]},
        "sort_values_immutable": {"source": sort + ":678-688", "keys": [20, 5, 12, 12],
                                  "values": [0, 1, 2, 3], "values_out": [0, 2, 3, 1]},
        "sort_gpu_small": {"source": sort + ":750-763", "keys": [10, 2, 7, 7, 100, 1],
                           "values": [0, 1, 2, 3, 4, 5], "keys_out": [100, 10, 7, 7, 2, 1],
                           "values_out": [4, 0, 2, 3, 1, 5]},
        "sort_lcg": {"source": sort + ":597-647", "multiplier": 1664525,
                     "increment": 1013904223, "large_len": 4099, "large_seed": 1,
                     "edge_lengths": [0, 1, 2, 255, 256, 257, 1024, 65537],
                     "edge_seed_base": 42},
        "gpu_radix_cases": {"source": order + ":557-584", "counts": [255, 256, 257, 4099],
                            "hash_multiplier": 2654435761, "key_mask": 16777215,
                            "equal_keys": {"count": 257, "key": 42}},
        "back_to_front": {"source": render + ":4062-4089",
                          "positions": [[0, 0, 0.5], [0, 0, 2.0], [0, 0, 1.0], [0, 0, -1.0],
                                        [0, 0, 2000.0]],
                          "visible": 3, "order": [1, 2, 0]},
        "ply_quat": {"source": ply + ":1031-1037",
                     "ply": "ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nproperty float z\nproperty float opacity\nproperty float scale_0\nproperty float scale_1\nproperty float scale_2\nproperty float rot_0\nproperty float rot_1\nproperty float rot_2\nproperty float rot_3\nproperty float f_dc_0\nproperty float f_dc_1\nproperty float f_dc_2\nend_header\n0.0 0.1 1.0 0.9 1.0 1.1 1.2 0.9 0.2 0.3 0.4 0.2 0.3 0.4\n",
                     "rotation_xyzw": [-0.2, 0.3, -0.4, 0.9]},
        "ply_sh_deg1": {"source": ply + ":1049-1062",
                        "rest_in": [0.01, 0.02, 0.03, 0.04, 0.05, 0.06, 0.07, 0.08, 0.09],
                        "rest_out": [-0.01, 0.02, 0.03, -0.04, 0.05, 0.06, -0.07, 0.08, 0.09]},
        "sh_flip_rdf_to_ruf": {"source": ply + ":54-56",
                               "signs": [-1, 1, 1, -1, -1, 1, 1, 1, -1, -1, -1, 1, 1, 1, 1]},
        "opacity_logit_limit": {"source": ply + ":18", "value": 16.0},
    }
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, indent=1)

    # Benchmark artifact v1 (tests/perf/benchmark-artifact-v1.md): the
    # product's producer writes the fixture, the reference's own validator
    # must accept it.
    import subprocess

    import artifact_fixture

    art = os.path.join(HERE, "artifact_v1")
    artifact_fixture.write(art)
    subprocess.run([sys.executable, os.path.join(REF, "tests/perf/validate-benchmark-artifacts.py"),
                    art], check=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.exit(main())
