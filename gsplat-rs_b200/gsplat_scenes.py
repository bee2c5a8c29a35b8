"""Seeded synthetic Gaussian-splat scenes and cameras for the benchmark configs.

Scenes are generated directly in the reference's SceneBuffers layout
(crates/gsplat-core/src/lib.rs:201-213): RUF positions, opacity as a logit,
log-scales, xyzw rotations, DC coefficients and channel-major `sh_rest`
(`[R c1..cK, G c1..cK, B c1..cK]` per splat). They stand in for Kitsune-class
captured scenes, which cannot be fetched here; only their sizes and parameter
distributions are modelled.

Cameras are GsplatCamera-shaped dicts (position, rotation_xyzw,
vertical_fov_radians, near_plane, far_plane).
"""

import math

import numpy as np


def sh_rest_width(degree):
    return 3 * ((degree + 1) ** 2 - 1)


def _uniform_quats(rng, n):
    q = rng.normal(size=(n, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def make_scene(rng, means, log_scale_mu, log_scale_sd, logit_mu, logit_sd, degree,
               dc_sd=0.5, rest_sd=0.1):
    n = means.shape[0]
    scene = {
        "positions": np.ascontiguousarray(means, np.float32),
        "opacity": rng.normal(logit_mu, logit_sd, n).astype(np.float32),
        "scale_xyz": rng.normal(log_scale_mu, log_scale_sd, (n, 3)).astype(np.float32),
        "rotation_xyzw": _uniform_quats(rng, n),
        "color_dc": rng.normal(0.0, dc_sd, (n, 3)).astype(np.float32),
        "sh_degree": int(degree),
        "sh_rest": None,
    }
    if degree > 0:
        scene["sh_rest"] = rng.normal(0.0, rest_sd, (n, sh_rest_width(degree))).astype(np.float32)
    return scene


def gmm_means(rng, n, sigmas=(0.3, 0.6, 0.9, 1.2), center_sd=0.5):
    k = rng.integers(0, len(sigmas), n)
    centers = rng.normal(0.0, center_sd, (len(sigmas), 3))
    sig = np.asarray(sigmas)[k][:, None]
    return (centers[k] + rng.normal(size=(n, 3)) * sig).astype(np.float32)


def look_at(position, target):
    """Rotation (xyzw) of a camera at `position` looking at `target`.

    Same construction as camera_rotation_looking_at in
    crates/gsplat-ffi-c/src/lib.rs:1677-1733: forward = normalize(target - pos),
    world up +Y (or +Z when looking nearly straight up/down), right =
    up x forward, then the quaternion of the basis matrix [right up forward].
    """
    p = np.asarray(position, np.float64)
    t = np.asarray(target, np.float64)
    f = t - p
    n = np.linalg.norm(f)
    f = f / n if n > 1e-6 else np.array([0.0, 0.0, 1.0])
    up = np.array([0.0, 0.0, 1.0]) if abs(f[1]) > 0.98 else np.array([0.0, 1.0, 0.0])
    r = np.cross(up, f)
    rn = np.linalg.norm(r)
    r = r / rn if rn > 1e-6 else np.array([1.0, 0.0, 0.0])
    u = np.cross(f, r)
    m00, m01, m02 = r[0], u[0], f[0]
    m10, m11, m12 = r[1], u[1], f[1]
    m20, m21, m22 = r[2], u[2], f[2]
    tr = m00 + m11 + m22
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2
        q = ((m21 - m12) / s, (m02 - m20) / s, (m10 - m01) / s, 0.25 * s)
    elif m00 > m11 and m00 > m22:
        s = math.sqrt(1.0 + m00 - m11 - m22) * 2
        q = (0.25 * s, (m01 + m10) / s, (m02 + m20) / s, (m21 - m12) / s)
    elif m11 > m22:
        s = math.sqrt(1.0 + m11 - m00 - m22) * 2
        q = ((m01 + m10) / s, 0.25 * s, (m12 + m21) / s, (m02 - m20) / s)
    else:
        s = math.sqrt(1.0 + m22 - m00 - m11) * 2
        q = ((m02 + m20) / s, (m12 + m21) / s, 0.25 * s, (m10 - m01) / s)
    q = np.asarray(q)
    q /= max(np.linalg.norm(q), 1e-6)
    return [float(v) for v in q.astype(np.float32)]


def camera(position, target=(0.0, 0.0, 0.0), fov_deg=60.0, near=0.01, far=1000.0):
    return {
        "position": [float(v) for v in np.asarray(position, np.float32)],
        "rotation_xyzw": look_at(position, target),
        "vertical_fov_radians": float(np.float32(math.radians(fov_deg))),
        "near_plane": float(np.float32(near)),
        "far_plane": float(np.float32(far)),
    }


def orbit_camera(rng, radius_range=(3.0, 8.0), fov_range=(40.0, 70.0), target=(0, 0, 0)):
    r = rng.uniform(*radius_range)
    yaw = rng.uniform(0, 2 * math.pi)
    pitch = rng.uniform(-0.6, 0.6)
    pos = (r * math.sin(yaw) * math.cos(pitch), r * math.sin(pitch),
           -r * math.cos(yaw) * math.cos(pitch))
    return camera(pos, target, rng.uniform(*fov_range))


def config1(seed=0):
    """16,384 splats, SH0, camera at (0,0,-5) looking at the origin, fov 50, 256x256."""
    rng = np.random.default_rng(seed)
    n = 16384
    scene = make_scene(rng, rng.normal(0.0, 1.0, (n, 3)), -4.0, 0.5, 0.0, 1.5, 0)
    cam = camera((0.0, 0.0, -5.0), (0.0, 0.0, 0.0), 50.0)
    return scene, cam, 256, 256


def config2(seed=1, n=279199):
    """279,199 splats, SH3, 4-component GMM, orbit radius 4, fov 45, 1920x1080."""
    rng = np.random.default_rng(seed)
    scene = make_scene(rng, gmm_means(rng, n), -4.5, 0.7, 0.5, 1.5, 3)
    yaw = 0.7
    cam = camera((4.0 * math.sin(yaw), 0.5, -4.0 * math.cos(yaw)), (0.0, 0.0, 0.0), 45.0)
    return scene, cam, 1920, 1080


def config3(seed=2, n=3_000_000):
    """3M splats, SH3, uniform 10^3 box plus a GMM core, camera inside, fov 60, 3840x2160."""
    rng = np.random.default_rng(seed)
    half = n // 2
    means = np.concatenate([rng.uniform(-5.0, 5.0, (half, 3)),
                            rng.normal(0.0, 0.7, (n - half, 3))]).astype(np.float32)
    scene = make_scene(rng, means, -3.5, 0.8, 1.0, 1.0, 3)
    cam = camera((0.5, 0.3, -3.0), (0.0, 0.0, 0.0), 60.0)
    return scene, cam, 3840, 2160


RESOLUTIONS = ((512, 512), (1280, 720), (1920, 1080))


def config4(seed=3, sizes=(50_000, 279_199, 1_000_000, 3_000_000), cameras_per_scene=64):
    """Resident scenes of uneven sizes (SH3) with seeded orbit cameras and mixed resolutions."""
    rng = np.random.default_rng(seed)
    scenes = []
    for k, n in enumerate(sizes):
        srng = np.random.default_rng(seed * 100 + k)
        scenes.append(make_scene(srng, gmm_means(srng, n), -4.5, 0.7, 0.5, 1.5, 3))
    views = []
    for s in range(len(scenes)):
        for _ in range(cameras_per_scene):
            w, h = RESOLUTIONS[rng.integers(0, len(RESOLUTIONS))]
            views.append({"scene": s, "camera": orbit_camera(rng), "width": w, "height": h})
    return scenes, views


def config5_scenes(seed=4, count=8, lo=50_000, hi=3_000_000):
    """Served-stream scenes: sizes log-uniform in [lo, hi], SH degree 0-3 mixed."""
    rng = np.random.default_rng(seed)
    scenes = []
    for k in range(count):
        n = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        degree = int(rng.integers(0, 4))
        srng = np.random.default_rng(seed * 100 + k)
        scenes.append(make_scene(srng, gmm_means(srng, n), -4.5, 0.7, 0.5, 1.5, degree))
    return scenes


def config5_requests(seed, rate_per_s, count, num_scenes):
    """Poisson arrivals: (arrival_s, scene, camera, width, height) tuples."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, count))
    reqs = []
    for i in range(count):
        w, h = RESOLUTIONS[rng.integers(0, len(RESOLUTIONS))]
        reqs.append({"arrival_s": float(t[i]), "scene": int(rng.integers(0, num_scenes)),
                     "camera": orbit_camera(rng), "width": w, "height": h})
    return reqs


def scene_from_json(obj):
    scene = {
        "positions": np.asarray(obj["positions"], np.float32).reshape(-1, 3),
        "opacity": np.asarray(obj["opacity"], np.float32),
        "scale_xyz": np.asarray(obj["scale_xyz"], np.float32).reshape(-1, 3),
        "rotation_xyzw": np.asarray(obj["rotation_xyzw"], np.float32).reshape(-1, 4),
        "color_dc": np.asarray(obj["color_dc"], np.float32).reshape(-1, 3),
        "sh_degree": int(obj["sh_degree"]),
        "sh_rest": None,
    }
    if obj.get("sh_rest") is not None:
        scene["sh_rest"] = np.asarray(obj["sh_rest"], np.float32).reshape(scene["positions"].shape[0], -1)
    return scene


# SH rest sign flips of the RDF <-> RUF reflection per coefficient (an
# involution: the loader applies the same signs).
_SH_FLIP = np.array([-1, 1, 1, -1, -1, 1, 1, 1, -1, -1, -1, 1, 1, 1, 1], np.float32)


def write_ply(path, scene, big_endian=False):
    """Writes a SceneBuffers-shaped dict (RUF) as a standard 3DGS binary PLY
    (RDF, rot_0..3 = w x y z, f_rest_* channel-major), so that loading the
    file gives back the same scene bit for bit: every conversion is a sign
    flip or a permutation."""
    pos = np.asarray(scene["positions"], np.float32).reshape(-1, 3)
    n = pos.shape[0]
    q = np.asarray(scene["rotation_xyzw"], np.float32).reshape(-1, 4)
    degree = int(scene.get("sh_degree", 0))
    per_channel = (degree + 1) ** 2 - 1
    rest = scene.get("sh_rest")
    cols = [("x", pos[:, 0]), ("y", -pos[:, 1]), ("z", pos[:, 2])]
    dc = np.asarray(scene["color_dc"], np.float32).reshape(-1, 3)
    cols += [(f"f_dc_{c}", dc[:, c]) for c in range(3)]
    if degree > 0 and rest is not None:
        r = np.asarray(rest, np.float32).reshape(n, 3, per_channel)
        flip = np.ones(per_channel, np.float32)
        flip[:min(15, per_channel)] = _SH_FLIP[:min(15, per_channel)]
        r = r * flip
        cols += [(f"f_rest_{ch * per_channel + k}", r[:, ch, k])
                 for ch in range(3) for k in range(per_channel)]
    cols += [("opacity", np.asarray(scene["opacity"], np.float32).reshape(-1))]
    sc = np.asarray(scene["scale_xyz"], np.float32).reshape(-1, 3)
    cols += [(f"scale_{k}", sc[:, k]) for k in range(3)]
    cols += [("rot_0", q[:, 3]), ("rot_1", -q[:, 0]), ("rot_2", q[:, 1]), ("rot_3", -q[:, 2])]
    order = ">" if big_endian else "<"
    body = np.empty((n, len(cols)), np.dtype(order + "f4"))
    for k, (_, v) in enumerate(cols):
        body[:, k] = v
    fmt = "binary_big_endian" if big_endian else "binary_little_endian"
    head = f"ply\nformat {fmt} 1.0\nelement vertex {n}\n"
    head += "".join(f"property float {name}\n" for name, _ in cols) + "end_header\n"
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(body.tobytes())


def default_camera():
    """gsplat_camera_default(): origin, identity rotation, fov 60, near 0.01, far 1000."""
    return {"position": [0.0, 0.0, 0.0], "rotation_xyzw": [0.0, 0.0, 0.0, 1.0],
            "vertical_fov_radians": float(np.float32(math.radians(60.0))),
            "near_plane": float(np.float32(0.01)), "far_plane": 1000.0}
