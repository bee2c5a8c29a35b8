"""FP64 evaluation of the reference's per-splat outputs (test infrastructure).

The reference's vertex stage, project_splat and eval_color
(crates/gsplat-render-wgpu/shaders/splat_surface_direct.wgsl:131-334), and
the load-time precomputes it reads (precompute_alpha_values and
precompute_world_covariances, crates/gsplat-render-wgpu/src/lib.rs:1251-1261,
1654-1674; the view rotation quat_to_mat3(quat_inverse(q)), lib.rs:1374-1407)
restated in float64 with numpy, from the scene's own SceneBuffers arrays
(positions, logit opacity, log scales, quaternions, SH coefficients). It is
the exact-arithmetic yardstick for the float32 outputs of the CUDA kernels:
means2d (the NDC centre), the clamped ellipse axes, the conic they imply and
the premultiplied SH colour. Nothing in the product imports it.
"""

import numpy as np

C0 = 0.28209479177387814
C1 = 0.4886025119029199
C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792,
      0.5462742152960396)
C3 = (-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
      -0.4570457994644658, 1.445305721320277, -0.5900435899266435)
C4 = (2.5033429417967046, -1.7701307697799304, 0.9461746957575601, -0.6690465435572892,
      0.10578554691520431, -0.6690465435572892, 0.47308734787878004, -1.7701307697799304,
      0.6258357354491761)


def quat_to_mat3(q):
    """Rotation matrices of (..., 4) xyzw quaternions, normalised first."""
    q = np.asarray(q, np.float64)
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def sh_rgb(dc, rest, d, degree):
    """eval_sh_rgb in float64; rest is (n, 3, k) channel-major."""
    x, y, z = d[:, 0:1], d[:, 1:2], d[:, 2:3]
    out = C0 * dc
    if degree == 0:
        return out
    r = lambda k: rest[:, :, k]  # noqa: E731
    out = out - C1 * y * r(0) + C1 * z * r(1) - C1 * x * r(2)
    if degree == 1:
        return out
    xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
    out = (out + C2[0] * xy * r(3) + C2[1] * yz * r(4) + C2[2] * (2 * zz - xx - yy) * r(5)
           + C2[3] * xz * r(6) + C2[4] * (xx - yy) * r(7))
    if degree == 2:
        return out
    out = (out + C3[0] * y * (3 * xx - yy) * r(8) + C3[1] * xy * z * r(9)
           + C3[2] * y * (4 * zz - xx - yy) * r(10) + C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * r(11)
           + C3[4] * x * (4 * zz - xx - yy) * r(12) + C3[5] * z * (xx - yy) * r(13)
           + C3[6] * x * (xx - 3 * yy) * r(14))
    if degree == 3:
        return out
    return (out + C4[0] * xy * (xx - yy) * r(15) + C4[1] * yz * (3 * xx - yy) * r(16)
            + C4[2] * xy * (7 * zz - 1) * r(17) + C4[3] * yz * (7 * zz - 3) * r(18)
            + C4[4] * (zz * (35 * zz - 30) + 3) * r(19) + C4[5] * xz * (7 * zz - 3) * r(20)
            + C4[6] * (xx - yy) * (7 * zz - 1) * r(21) + C4[7] * xz * (xx - 3 * yy) * r(22)
            + C4[8] * (xx * (xx - 3 * yy) - yy * (3 * xx - yy)) * r(23))


def project(scene, cam, width, height):
    """Per-splat float64 outputs of the vertex stage for every splat:
    dict of center_ndc (n, 2), axis_u, axis_v (n, 2), color (n, 4: rgb *
    alpha, alpha), conic (n, 3: the quadratic form |local|^2 = a x^2 + 2b xy
    + c y^2 of NDC offsets, from the clamped axes) and drawn (n,) bool."""
    pos = np.asarray(scene["positions"], np.float64).reshape(-1, 3)
    n = pos.shape[0]
    alpha = np.clip(1.0 / (1.0 + np.exp(-np.asarray(scene["opacity"], np.float64))), 0.0, 1.0)
    s = np.maximum(np.exp(np.asarray(scene["scale_xyz"], np.float64).reshape(-1, 3)), 1e-6)
    R = quat_to_mat3(np.asarray(scene["rotation_xyzw"], np.float64).reshape(-1, 4))
    cov = np.einsum("nij,nj,nkj->nik", R, s * s, R)
    q = np.asarray(cam["rotation_xyzw"], np.float64)
    V = quat_to_mat3(q * np.array([-1.0, -1.0, -1.0, 1.0]))  # R(q^-1)
    campos = np.asarray(cam["position"], np.float64)
    rel = pos - campos
    p = rel @ V.T
    near, far = float(cam["near_plane"]), float(cam["far_plane"])
    fov = float(cam["vertical_fov_radians"])
    aspect = max(width / max(height, 1), 1e-6)
    f = 1.0 / np.tan(0.5 * fov)
    z = p[:, 2]
    valid = (z >= near) & (z <= far) & (z > 1e-6)
    zs = np.where(valid, z, 1.0)
    x_ndc = p[:, 0] * f / zs / aspect
    y_ndc = p[:, 1] * f / zs
    cc = np.einsum("ij,njk,lk->nil", V, cov, V)
    tanh = np.tan(0.5 * fov)
    lim_x, lim_y = 1.3 * tanh * aspect, 1.3 * tanh
    xc = np.clip(p[:, 0] / zs, -lim_x, lim_x) * zs
    yc = np.clip(p[:, 1] / zs, -lim_y, lim_y) * zs
    fx, fy = f / aspect, f
    j00, j11 = fx / zs, fy / zs
    j02 = -fx * xc / zs ** 2
    j12 = -fy * yc / zs ** 2
    a = j00 * j00 * cc[:, 0, 0] + 2 * j00 * j02 * cc[:, 0, 2] + j02 * j02 * cc[:, 2, 2]
    b = (j00 * j11 * cc[:, 0, 1] + j00 * j12 * cc[:, 0, 2] + j02 * j11 * cc[:, 1, 2]
         + j02 * j12 * cc[:, 2, 2])
    c = j11 * j11 * cc[:, 1, 1] + 2 * j11 * j12 * cc[:, 1, 2] + j12 * j12 * cc[:, 2, 2]
    a = a + (0.3 * 2.0 / max(width, 1)) ** 2
    c = c + (0.3 * 2.0 / max(height, 1)) ** 2
    apc, amc = 0.5 * (a + c), 0.5 * (a - c)
    term = np.sqrt(np.maximum(amc * amc + b * b, 0.0))
    major = np.maximum(apc + term, 1e-10)
    minor = np.maximum(apc - term, 1e-10)
    ux, uy = np.ones(n), np.zeros(n)
    use_b = np.abs(b) > 1e-8
    vx, vy = b, major - a
    l2 = vx * vx + vy * vy
    ok = use_b & (l2 > 1e-20)
    inv = 1.0 / np.sqrt(np.where(ok, l2, 1.0))
    ux = np.where(ok, vx * inv, ux)
    uy = np.where(ok, vy * inv, uy)
    swap = ~use_b & (a < c)
    ux = np.where(swap, 0.0, ux)
    uy = np.where(swap, 1.0, uy)
    major_r = np.clip(np.sqrt(major) * 3.0, 1e-4, 2.0)
    minor_r = np.clip(np.sqrt(minor) * 3.0, 1e-4, 2.0)
    major_r = np.minimum(major_r, minor_r * 64.0)
    axis_u = np.stack([ux * major_r, uy * major_r], -1)
    axis_v = np.stack([-uy * minor_r, ux * minor_r], -1)
    ex = np.abs(axis_u[:, 0]) + np.abs(axis_v[:, 0])
    ey = np.abs(axis_u[:, 1]) + np.abs(axis_v[:, 1])
    onscreen = ~((x_ndc + ex < -1) | (x_ndc - ex > 1) | (y_ndc + ey < -1) | (y_ndc - ey > 1))
    drawn = valid & onscreen
    # colour
    d = rel.copy()
    l2d = (d * d).sum(-1, keepdims=True)
    d = np.where(l2d > 1e-20, d / np.sqrt(np.maximum(l2d, 1e-300)), np.array([0.0, 0.0, 1.0]))
    degree = int(scene.get("sh_degree", 0) or 0)
    dc = np.asarray(scene["color_dc"], np.float64).reshape(-1, 3)
    rest = scene.get("sh_rest")
    k = (degree + 1) ** 2 - 1
    rest = (np.asarray(rest, np.float64).reshape(n, 3, k) if degree > 0 and rest is not None
            else np.zeros((n, 3, 0)))
    rgb = np.clip(sh_rgb(dc, rest, d, min(degree, 4)) + 0.5, 0.0, 1.0)
    color = np.concatenate([rgb * alpha[:, None], alpha[:, None]], -1)
    # conic of the clamped axes: local = M^-1 (x - c), M = [axis_u axis_v]
    det = axis_u[:, 0] * axis_v[:, 1] - axis_u[:, 1] * axis_v[:, 0]
    det = np.where(det == 0.0, 1.0, det)
    i00, i01 = axis_v[:, 1] / det, -axis_v[:, 0] / det
    i10, i11 = -axis_u[:, 1] / det, axis_u[:, 0] / det
    conic = np.stack([i00 * i00 + i10 * i10, i00 * i01 + i10 * i11, i01 * i01 + i11 * i11], -1)
    return {"center_ndc": np.stack([x_ndc, y_ndc], -1), "axis_u": axis_u, "axis_v": axis_v,
            "color": color, "conic": conic, "drawn": drawn}


def conic_from_axes(axis_u, axis_v):
    """The same conic from (float32) axes, evaluated in float64."""
    u = np.asarray(axis_u, np.float64)
    v = np.asarray(axis_v, np.float64)
    det = u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]
    det = np.where(det == 0.0, 1.0, det)
    i00, i01 = v[:, 1] / det, -v[:, 0] / det
    i10, i11 = -u[:, 1] / det, u[:, 0] / det
    return np.stack([i00 * i00 + i10 * i10, i00 * i01 + i10 * i11, i01 * i01 + i11 * i11], -1)


def output_errors(proj32, ref64):
    """Max and mean error of float32 per-splat outputs (a GsplatProjectedSplat
    array) against project(): absolute, and relative to the norm of the
    output vector, over the splats both draw; also how many splats one draws
    and the other does not (a clamp or a cull decided differently at its
    boundary)."""
    drawn32 = (np.asarray(proj32["flags"]) & 2) != 0
    both = drawn32 & ref64["drawn"]
    out = {"drawn_both": int(both.sum()),
           "drawn_disagree": int((drawn32 != ref64["drawn"]).sum())}
    gpu = {"center_ndc": proj32["center_ndc"], "axis_u": proj32["axis_u"],
           "axis_v": proj32["axis_v"], "color": proj32["color"],
           "conic": conic_from_axes(proj32["axis_u"], proj32["axis_v"])}
    for k, g in gpu.items():
        g = np.asarray(g, np.float64)[both]
        r = np.asarray(ref64[k], np.float64)[both]
        if g.size == 0:
            out[k] = None
            continue
        err = np.abs(g - r).max(axis=-1)
        rel = err / np.maximum(np.abs(r).max(axis=-1), 1e-30)
        out[k] = {"max_abs": float(err.max()), "mean_abs": float(err.mean()),
                  "max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                  "p999_rel": float(np.quantile(rel, 0.999))}
    return out
