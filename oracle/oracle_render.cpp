// CPU oracle, part 2: the WGSL vertex stage (projection + SH colour), the
// reference's CPU instance builder, the tile-key contract of the CUDA design,
// and three compositors.
//
// TEST INFRASTRUCTURE ONLY (see gsplat_oracle.h).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "gsplat_oracle.h"
#include "oracle_internal.h"

namespace orc {

struct Cov6 {
  float xx, xy, xz, yy, yz, zz;
};

// splat_surface_direct.wgsl:96-103 (covariance_quadratic)
static inline float cov_quadratic(const Cov6 &c, const float r[3]) {
  return r[0] * r[0] * c.xx + 2.0f * r[0] * r[1] * c.xy + 2.0f * r[0] * r[2] * c.xz +
         r[1] * r[1] * c.yy + 2.0f * r[1] * r[2] * c.yz + r[2] * r[2] * c.zz;
}

// splat_surface_direct.wgsl:105-110 (covariance_bilinear)
static inline float cov_bilinear(const Cov6 &c, const float a[3], const float b[3]) {
  float bx = c.xx * b[0] + c.xy * b[1] + c.xz * b[2];
  float by = c.xy * b[0] + c.yy * b[1] + c.yz * b[2];
  float bz = c.xz * b[0] + c.yz * b[1] + c.zz * b[2];
  return a[0] * bx + a[1] * by + a[2] * bz;
}

// splat_surface_direct.wgsl:233-326 (eval_sh_rgb) for one channel; the
// coefficient reader takes rest index k (0-based, excluding DC).
template <typename Rest>
static inline float eval_sh_channel(float dc, float x, float y, float z, uint32_t degree,
                                    Rest rest) {
  const float c0 = 0.28209479177387814f;
  const float c1 = 0.4886025119029199f;
  const float c2_0 = 1.0925484305920792f, c2_1 = -1.0925484305920792f,
              c2_2 = 0.31539156525252005f, c2_3 = -1.0925484305920792f,
              c2_4 = 0.5462742152960396f;
  const float c3_0 = -0.5900435899266435f, c3_1 = 2.890611442640554f,
              c3_2 = -0.4570457994644658f, c3_3 = 0.3731763325901154f,
              c3_4 = -0.4570457994644658f, c3_5 = 1.445305721320277f,
              c3_6 = -0.5900435899266435f;
  const float c4_0 = 2.5033429417967046f, c4_1 = -1.7701307697799304f,
              c4_2 = 0.9461746957575601f, c4_3 = -0.6690465435572892f,
              c4_4 = 0.10578554691520431f, c4_5 = -0.6690465435572892f,
              c4_6 = 0.47308734787878004f, c4_7 = -1.7701307697799304f,
              c4_8 = 0.6258357354491761f;
  float result = c0 * dc;
  if (degree == 0) return result;
  result = result - c1 * y * rest(0) + c1 * z * rest(1) - c1 * x * rest(2);
  if (degree == 1) return result;
  float xx = x * x, yy = y * y, zz = z * z;
  float xy = x * y, yz = y * z, xz = x * z;
  result = result + c2_0 * xy * rest(3) + c2_1 * yz * rest(4) +
           c2_2 * (2.0f * zz - xx - yy) * rest(5) + c2_3 * xz * rest(6) +
           c2_4 * (xx - yy) * rest(7);
  if (degree == 2) return result;
  result = result + c3_0 * y * (3.0f * xx - yy) * rest(8) + c3_1 * xy * z * rest(9) +
           c3_2 * y * (4.0f * zz - xx - yy) * rest(10) +
           c3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * rest(11) +
           c3_4 * x * (4.0f * zz - xx - yy) * rest(12) + c3_5 * z * (xx - yy) * rest(13) +
           c3_6 * x * (xx - 3.0f * yy) * rest(14);
  if (degree == 3) return result;
  result = result + c4_0 * xy * (xx - yy) * rest(15) + c4_1 * yz * (3.0f * xx - yy) * rest(16) +
           c4_2 * xy * (7.0f * zz - 1.0f) * rest(17) + c4_3 * yz * (7.0f * zz - 3.0f) * rest(18) +
           c4_4 * (zz * (35.0f * zz - 30.0f) + 3.0f) * rest(19) +
           c4_5 * xz * (7.0f * zz - 3.0f) * rest(20) +
           c4_6 * (xx - yy) * (7.0f * zz - 1.0f) * rest(21) +
           c4_7 * xz * (xx - 3.0f * yy) * rest(22) +
           c4_8 * (xx * (xx - 3.0f * yy) - yy * (3.0f * xx - yy)) * rest(23);
  return result;
}

static inline float clamp01(float x) { return std::fmin(std::fmax(x, 0.0f), 1.0f); }

// One splat through project_splat (splat_surface_direct.wgsl:131-217),
// eval_color (328-334) and alpha_extent_scale (74-77, precomputed per splat at
// load), then the tile rect and pixel-space record of the CUDA design.
static void project_one(const OrcScene &sc, const float *alpha, const float *extent,
                        const float *cov6, const OrcFrameParams &p, uint64_t i,
                        OrcProjected &out, OrcRecord &rec) {
  std::memset(&out, 0, sizeof(out));
  std::memset(&rec, 0, sizeof(rec));
  const float *pos = &sc.positions[3 * i];
  float rel[3] = {pos[0] - p.cam[0], pos[1] - p.cam[1], pos[2] - p.cam[2]};
  const float *r0 = &p.view_rot[0], *r1 = &p.view_rot[3], *r2 = &p.view_rot[6];
  // Depth as preprocess_visible_into computes it (lib.rs:1346-1354); the
  // vertex stage's dot(r2, rel) is the same expression.
  float depth = r2[0] * rel[0] + r2[1] * rel[1] + r2[2] * rel[2];
  out.depth = depth;
  bool visible = depth >= p.near_plane && depth <= p.far_plane;
  if (!visible) return;
  out.flags = 1u;
  float px = r0[0] * rel[0] + r0[1] * rel[1] + r0[2] * rel[2];
  float py = r1[0] * rel[0] + r1[1] * rel[1] + r1[2] * rel[2];
  float z = depth;
  if (z < p.near_plane || z > p.far_plane || z <= 1e-6f) return;
  float inv_z = 1.0f / z;
  float x_ndc = (px * p.f) * inv_z / p.aspect;
  float y_ndc = (py * p.f) * inv_z;

  Cov6 wc{cov6[6 * i + 0], cov6[6 * i + 1], cov6[6 * i + 2],
          cov6[6 * i + 3], cov6[6 * i + 4], cov6[6 * i + 5]};
  Cov6 cc{cov_quadratic(wc, r0),    cov_bilinear(wc, r0, r1), cov_bilinear(wc, r0, r2),
          cov_quadratic(wc, r1),    cov_bilinear(wc, r1, r2), cov_quadratic(wc, r2)};
  float x_cl = clamp_f(px / z, -p.lim_x, p.lim_x) * z;
  float y_cl = clamp_f(py / z, -p.lim_y, p.lim_y) * z;
  float inv_z2 = inv_z * inv_z;
  float j00 = p.fx * inv_z;
  float j02 = -p.fx * x_cl * inv_z2;
  float j11 = p.fy * inv_z;
  float j12 = -p.fy * y_cl * inv_z2;
  float cov01 = j00 * j11 * cc.xy + j00 * j12 * cc.xz + j02 * j11 * cc.yz + j02 * j12 * cc.zz;
  float a = j00 * j00 * cc.xx + 2.0f * j00 * j02 * cc.xz + j02 * j02 * cc.zz;
  float b = cov01;
  float c = j11 * j11 * cc.yy + 2.0f * j11 * j12 * cc.yz + j12 * j12 * cc.zz;
  a = a + p.blur_x;
  c = c + p.blur_y;
  float apco2 = (a + c) * 0.5f;
  float amco2 = (a - c) * 0.5f;
  float term = std::sqrt(std::fmax(amco2 * amco2 + b * b, 0.0f));
  float major = std::fmax(apco2 + term, 1e-10f);
  float minor = std::fmax(apco2 - term, 1e-10f);
  float ux = 1.0f, uy = 0.0f;
  if (std::fabs(b) > 1e-8f) {
    float vx = b, vy = major - a;
    float len2 = vx * vx + vy * vy;
    if (len2 <= 1e-20f) {
      ux = 1.0f; uy = 0.0f;
    } else {
      float inv = 1.0f / std::sqrt(len2);
      ux = vx * inv; uy = vy * inv;
    }
  } else if (a < c) {
    ux = 0.0f; uy = 1.0f;
  }
  float vdx = -uy, vdy = ux;
  float major_r = clamp_f(std::sqrt(major) * 3.0f, 1e-4f, 2.0f);
  float minor_r = clamp_f(std::sqrt(minor) * 3.0f, 1e-4f, 2.0f);
  major_r = std::fmin(major_r, minor_r * 64.0f);
  float au0 = ux * major_r, au1 = uy * major_r;
  float av0 = vdx * minor_r, av1 = vdy * minor_r;
  float ext_x = std::fabs(au0) + std::fabs(av0);
  float ext_y = std::fabs(au1) + std::fabs(av1);
  if (x_ndc + ext_x < -1.0f || x_ndc - ext_x > 1.0f || y_ndc + ext_y < -1.0f ||
      y_ndc - ext_y > 1.0f)
    return;
  out.flags |= 2u;
  float al = alpha[i];
  float s = extent[i];
  out.center_ndc[0] = x_ndc; out.center_ndc[1] = y_ndc;
  out.axis_u[0] = au0; out.axis_u[1] = au1;
  out.axis_v[0] = av0; out.axis_v[1] = av1;
  out.extent_scale = s;

  // eval_color: dir = normalize3_or_default(pos - cam, (0,0,1)).
  float len2 = rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2];
  float dx = 0.0f, dy = 0.0f, dz = 1.0f;
  if (!(len2 <= 1e-20f)) {
    float inv = 1.0f / std::sqrt(len2);
    dx = rel[0] * inv; dy = rel[1] * inv; dz = rel[2] * inv;
  }
  uint32_t degree = std::min<uint32_t>(p.sh_degree, 4u);
  uint32_t per_channel = (degree + 1) * (degree + 1) - 1;
  float rgb[3];
  for (int ch = 0; ch < 3; ++ch) {
    const float *base = sc.sh_rest ? &sc.sh_rest[i * per_channel * 3 + ch * per_channel] : nullptr;
    float v = eval_sh_channel(sc.color_dc[3 * i + ch], dx, dy, dz, degree,
                              [base](uint32_t k) { return base[k]; });
    rgb[ch] = clamp01(v + 0.5f);
  }
  out.color[0] = rgb[0] * al; out.color[1] = rgb[1] * al; out.color[2] = rgb[2] * al;
  out.color[3] = al;

  // Pixel-space record: centre in pixel-centre coordinates and the inverse of
  // the axis matrix, so that local = (ax*dx + ay*dy, bx*dx + by*dy).
  float cxp = (x_ndc + 1.0f) * p.half_w - 0.5f;
  float cyp = (1.0f - y_ndc) * p.half_h - 0.5f;
  float uu = au0 * au0 + au1 * au1;
  float vv = av0 * av0 + av1 * av1;
  rec.cx = cxp; rec.cy = cyp;
  rec.ax = (au0 * p.sx) / uu; rec.ay = (au1 * p.sy) / uu;
  rec.bx = (av0 * p.sx) / vv; rec.by = (av1 * p.sy) / vv;
  rec.s = s; rec.alpha = al;
  rec.cr = rgb[0]; rec.cg = rgb[1]; rec.cb = rgb[2];
  rec.log2a = std::log2(al);

  // Tile rect: pixel bbox of the ellipse |local| <= s, widened by a small
  // margin, clamped to the image. Splats with alpha <= 1/256 never pass the
  // fragment threshold and get no tiles.
  if (!(al > 1.0f / 256.0f)) return;
  float ex = s * std::sqrt(au0 * au0 + av0 * av0) * p.half_w;
  float ey = s * std::sqrt(au1 * au1 + av1 * av1) * p.half_h;
  ex = ex * 1.00001f + 0.001f;
  ey = ey * 1.00001f + 0.001f;
  float fx0 = std::fmax(std::ceil(cxp - ex), 0.0f);
  float fx1 = std::fmin(std::floor(cxp + ex), (float)(p.width - 1));
  float fy0 = std::fmax(std::ceil(cyp - ey), 0.0f);
  float fy1 = std::fmin(std::floor(cyp + ey), (float)(p.height - 1));
  if (!(fx0 <= fx1) || !(fy0 <= fy1)) return;
  out.tile_x0 = (uint16_t)((uint32_t)fx0 / p.tile);
  out.tile_x1 = (uint16_t)((uint32_t)fx1 / p.tile + 1);
  out.tile_y0 = (uint16_t)((uint32_t)fy0 / p.tile);
  out.tile_y1 = (uint16_t)((uint32_t)fy1 / p.tile + 1);
}

// ---- reference CPU instance builder (lib.rs:1134-1194 and helpers) ----

static bool cpu_project_cov(const float pc[3], const Cov6 &cc, const float lim_x,
                            const float lim_y, const float fx, const float fy, const float bx,
                            const float by, float cov2[3]) {
  // lib.rs:1456-1506 (project_camera_covariance_to_ndc)
  float z = pc[2];
  if (z <= 1e-6f || !std::isfinite(z)) return false;
  float x_cl = clamp_f(pc[0] / z, -lim_x, lim_x) * z;
  float y_cl = clamp_f(pc[1] / z, -lim_y, lim_y) * z;
  float inv_z = 1.0f / z;
  float inv_z2 = inv_z * inv_z;
  float j00 = fx * inv_z, j02 = -fx * x_cl * inv_z2;
  float j11 = fy * inv_z, j12 = -fy * y_cl * inv_z2;
  float cov01 = j00 * j11 * cc.xy + j00 * j12 * cc.xz + j02 * j11 * cc.yz + j02 * j12 * cc.zz;
  cov2[0] = j00 * j00 * cc.xx + 2.0f * j00 * j02 * cc.xz + j02 * j02 * cc.zz;
  cov2[1] = cov01;
  cov2[2] = j11 * j11 * cc.yy + 2.0f * j11 * j12 * cc.yz + j12 * j12 * cc.zz;
  cov2[0] += bx;
  cov2[2] += by;
  return std::isfinite(cov2[0]) && std::isfinite(cov2[1]) && std::isfinite(cov2[2]);
}

static bool cpu_ellipse_axes(const float cov2[3], float u[2], float v[2]) {
  // lib.rs:1589-1634 (ellipse_axes_from_covariance)
  float a = cov2[0], b = cov2[1], c = cov2[2];
  float apco2 = (a + c) * 0.5f, amco2 = (a - c) * 0.5f;
  float term = std::sqrt(amco2 * amco2 + b * b);
  float major = std::fmax(apco2 + term, 1e-10f);
  float minor = std::fmax(apco2 - term, 1e-10f);
  float d0, d1;
  if (std::fabs(b) > 1e-8f) {
    float len2 = b * b + (major - a) * (major - a);
    if (len2 <= 0.0f) {
      d0 = 1.0f; d1 = 0.0f;
    } else {
      float inv = 1.0f / std::sqrt(len2);
      d0 = b * inv; d1 = (major - a) * inv;
    }
  } else if (a >= c) {
    d0 = 1.0f; d1 = 0.0f;
  } else {
    d0 = 0.0f; d1 = 1.0f;
  }
  float e0 = -d1, e1 = d0;
  float major_r = clamp_f(std::sqrt(major) * 3.0f, 1e-4f, 2.0f);
  float minor_r = clamp_f(std::sqrt(minor) * 3.0f, 1e-4f, 2.0f);
  if (major_r > minor_r * 64.0f) major_r = minor_r * 64.0f;
  u[0] = d0 * major_r; u[1] = d1 * major_r;
  v[0] = e0 * minor_r; v[1] = e1 * minor_r;
  return std::isfinite(u[0]) && std::isfinite(u[1]) && std::isfinite(v[0]) && std::isfinite(v[1]);
}

// lib.rs:2066-2155 (sh_basis, dot_sh_terms) and 1945-2039 (degree-3 fast path):
// DC term first, the rest summed separately, then +0.5 and max(0).
static void cpu_sh_color(const OrcScene &sc, uint64_t i, const float dir[3], float rgb[3]) {
  const float C0 = 0.2820948f;
  const float C1 = 0.48860252f;
  const float C2[5] = {1.0925485f, -1.0925485f, 0.31539157f, -1.0925485f, 0.54627424f};
  const float C3[7] = {-0.5900436f, 2.8906114f, -0.4570458f, 0.37317634f,
                       -0.4570458f, 1.4453057f,  -0.5900436f};
  const float C4[9] = {2.5033429f,  -1.7701308f, 0.9461747f,  -0.6690465f, 0.10578555f,
                       -0.6690465f, 0.47308734f, -1.7701308f, 0.6258357f};
  const float *dc = &sc.color_dc[3 * i];
  rgb[0] = C0 * dc[0]; rgb[1] = C0 * dc[1]; rgb[2] = C0 * dc[2];
  uint32_t deg = sc.sh_rest ? sc.sh_degree : 0;
  if (deg > 0) {
    float x = dir[0], y = dir[1], z = dir[2];
    float basis[24] = {0};
    uint32_t len = 0;
    basis[0] = -C1 * y; basis[1] = C1 * z; basis[2] = -C1 * x; len = 3;
    if (deg >= 2) {
      float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
      basis[3] = C2[0] * xy; basis[4] = C2[1] * yz; basis[5] = C2[2] * (2.0f * zz - xx - yy);
      basis[6] = C2[3] * xz; basis[7] = C2[4] * (xx - yy); len = 8;
      if (deg >= 3) {
        basis[8] = C3[0] * y * (3.0f * xx - yy); basis[9] = C3[1] * xy * z;
        basis[10] = C3[2] * y * (4.0f * zz - xx - yy);
        basis[11] = C3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
        basis[12] = C3[4] * x * (4.0f * zz - xx - yy); basis[13] = C3[5] * z * (xx - yy);
        basis[14] = C3[6] * x * (xx - 3.0f * yy); len = 15;
      }
      if (deg >= 4) {
        basis[15] = C4[0] * xy * (xx - yy); basis[16] = C4[1] * yz * (3.0f * xx - yy);
        basis[17] = C4[2] * xy * (7.0f * zz - 1.0f); basis[18] = C4[3] * yz * (7.0f * zz - 3.0f);
        basis[19] = C4[4] * (zz * (35.0f * zz - 30.0f) + 3.0f);
        basis[20] = C4[5] * xz * (7.0f * zz - 3.0f);
        basis[21] = C4[6] * (xx - yy) * (7.0f * zz - 1.0f);
        basis[22] = C4[7] * xz * (xx - 3.0f * yy);
        basis[23] = C4[8] * (xx * (xx - 3.0f * yy) - yy * (3.0f * xx - yy)); len = 24;
      }
    }
    uint32_t per_channel = (deg + 1) * (deg + 1) - 1;
    for (int ch = 0; ch < 3; ++ch) {
      const float *rest = &sc.sh_rest[i * per_channel * 3 + ch * per_channel];
      float acc = 0.0f;
      for (uint32_t k = 0; k < len && k < per_channel; ++k) acc += basis[k] * rest[k];
      rgb[ch] = rgb[ch] + acc;
    }
  }
  for (int ch = 0; ch < 3; ++ch) rgb[ch] = std::fmax(rgb[ch] + 0.5f, 0.0f);
}

// Exact f32 quotients d / 255 for d in 0..255 (the same correctly rounded
// values a division produces).
static float g_inv255[256];
static bool init_inv255() {
  for (int d = 0; d < 256; ++d) g_inv255[d] = (float)d / 255.0f;
  return true;
}
static const bool g_inv255_ready = init_inv255();

static void parallel_rows(uint32_t height, int threads,
                          const std::function<void(uint32_t, uint32_t)> &fn) {
  if (threads <= 1 || height < 2) {
    fn(0, height);
    return;
  }
  std::vector<std::thread> pool;
  uint32_t chunk = (height + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    uint32_t y0 = t * chunk, y1 = std::min(height, y0 + chunk);
    if (y0 >= y1) break;
    pool.emplace_back(fn, y0, y1);
  }
  for (auto &th : pool) th.join();
}

static inline void quad_pixel_bbox(const OrcProjected &p, const OrcRecord &r, uint32_t w,
                                   uint32_t h, int &x0, int &x1, int &y0, int &y1) {
  // Bounding box of the drawn quad c +- s*u +- s*v in pixel coordinates, one
  // pixel wider on each side; the per-pixel test decides coverage.
  double hx = (double)p.extent_scale * (std::fabs((double)p.axis_u[0]) + std::fabs((double)p.axis_v[0]));
  double hy = (double)p.extent_scale * (std::fabs((double)p.axis_u[1]) + std::fabs((double)p.axis_v[1]));
  double rx = hx * 0.5 * w + 1.0, ry = hy * 0.5 * h + 1.0;
  x0 = (int)std::max(0.0, std::floor(r.cx - rx));
  x1 = (int)std::min((double)w - 1, std::ceil(r.cx + rx));
  y0 = (int)std::max(0.0, std::floor(r.cy - ry));
  y1 = (int)std::min((double)h - 1, std::ceil(r.cy + ry));
}

// Band workers of the compositors. target_clones builds an FMA version
// (explicit fmaf becomes one instruction) and a portable one, picked at load
// time; both compute identical values.
__attribute__((target_clones("fma", "default"))) static void unorm8_band(
    const OrcRecord *records, const OrcProjected *proj, const uint32_t *order, uint64_t v,
    uint32_t width, uint32_t height, uint8_t *rgba, uint32_t ya, uint32_t yb) {
  for (uint64_t j = 0; j < v; ++j) {
    uint32_t s = order[j];
    const OrcProjected &p = proj[s];
    if (!(p.flags & 2u)) continue;
    const OrcRecord &r = records[s];
    int x0, x1, y0, y1;
    quad_pixel_bbox(p, r, width, height, x0, x1, y0, y1);
    y0 = std::max<int>(y0, (int)ya);
    y1 = std::min<int>(y1, (int)yb - 1);
    for (int py = y0; py <= y1; ++py)
      for (int px = x0; px <= x1; ++px) {
        float g, w;
        if (!pixel_weight(r, px, py, g, w)) continue;
        uint8_t *d = &rgba[((size_t)py * width + px) * 4];
        float one_minus = 1.0f - w;
        // premultiplied colour: the vertex stage's rgb * alpha
        float src[3] = {(r.cr * r.alpha) * g, (r.cg * r.alpha) * g, (r.cb * r.alpha) * g};
        for (int ch = 0; ch < 3; ++ch) d[ch] = to_unorm8(std::fma(g_inv255[d[ch]], one_minus, src[ch]));
        d[3] = to_unorm8(std::fma(g_inv255[d[3]], one_minus, w));
      }
  }
}

// The CUDA FP32 tile raster, pixel by pixel: per (splat, 16-pixel grid cell)
// the local offsets ox, oy and s^2; per pixel local = (ax*lx + ay*ly + ox,
// bx*lx + by*ly + oy) in pixel coordinates relative to the cell corner,
// coverage r^2 <= s^2 and w = alpha e^(-4.5 r^2) > 1/256 (the latter as a
// bound on r^2), C += rgb * (w T), T -= w T, stop once T < 1e-4.
__attribute__((target_clones("fma", "default"))) static void tiles_fp32_band(
    const OrcRecord *records, const uint32_t *ranges, const uint32_t *sorted_ids, uint32_t width,
    uint32_t tile, uint32_t tiles_x, uint8_t *rgba, uint32_t ya, uint32_t yb) {
  for (uint32_t py = ya; py < yb; ++py)
    for (uint32_t px = 0; px < width; ++px) {
      uint32_t tx = px / tile, ty = py / tile;
      uint32_t t = ty * tiles_x + tx;
      // local coordinates from the 16-pixel grid corner at or before the tile
      const uint32_t ax0 = (tx * tile) & ~15u, ay0 = (ty * tile) & ~15u;
      const float ftx = (float)ax0, fty = (float)ay0;
      const float fx = (float)(px - ax0), fy = (float)(py - ay0);
      uint32_t start = ranges[2 * t], end = ranges[2 * t + 1];
      float T = 1.0f, c[3] = {0.0f, 0.0f, 0.0f};
      for (uint32_t k = end; k > start; --k) {
        const OrcRecord &r = records[sorted_ids[k - 1]];
        float cxl = r.cx - ftx, cyl = r.cy - fty;
        float ox = -std::fma(r.ax, cxl, r.ay * cyl);
        float oy = -std::fma(r.bx, cxl, r.by * cyl);
        float s2 = r.s * r.s;
        // w > 1/256 exactly when r2 < (log2 alpha + 8) / (4.5 log2 e): covered
        // when r2 <= the largest float below that bound, capped at s^2
        float wlim = (r.log2a + 8.0f) / 6.49212768f;
        float thr = wlim > 0.0f ? std::fmin(s2, std::nextafterf(wlim, 0.0f)) : -1.0f;
        float lx = std::fma(r.ax, fx, std::fma(r.ay, fy, ox));
        float ly = std::fma(r.bx, fx, std::fma(r.by, fy, oy));
        float r2 = std::fma(lx, lx, ly * ly);
        if (!(r2 <= thr)) continue;
        float w = blend_weight(r2, r.log2a);
        float wT = w * T;
        c[0] = std::fma(r.cr, wT, c[0]);
        c[1] = std::fma(r.cg, wT, c[1]);
        c[2] = std::fma(r.cb, wT, c[2]);
        T = T - wT;
        if (T < 1e-4f) break;
      }
      uint8_t *d = &rgba[((size_t)py * width + px) * 4];
      d[0] = to_unorm8(c[0]); d[1] = to_unorm8(c[1]); d[2] = to_unorm8(c[2]);
      d[3] = to_unorm8(1.0f - T);
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

void orc_project_all(const OrcScene *scene, const float *alpha, const float *extent_scale,
                     const float *cov6, const OrcFrameParams *params, OrcProjected *out,
                     OrcRecord *records) {
  for (uint64_t i = 0; i < scene->count; ++i)
    project_one(*scene, alpha, extent_scale, cov6, *params, i, out[i], records[i]);
}

// lib.rs:1134-1194 (build_instance_unchecked) with InstanceBuildParams
// (lib.rs:1217-1249). out12 per kept instance: center_and_axis_u[4],
// axis_v_and_pad[4], color_rgba[4]. Returns the number kept.
uint64_t orc_build_instances(const OrcScene *sc, const float *alpha, const float *cov6,
                             const OrcCamera *cam, uint32_t width, uint32_t height,
                             const uint32_t *indices, uint64_t m, float *out12,
                             uint32_t *out_index) {
  if (width == 0 || height == 0) return 0;
  float tan_half = std::tan(cam->vertical_fov_radians * 0.5f);
  if (tan_half <= 0.0f || !std::isfinite(tan_half)) return 0;
  float aspect = (float)width / (float)height;
  float f = 1.0f / tan_half;
  float fx = f / aspect, fy = f;
  float lim_x = 1.3f * (tan_half * aspect), lim_y = 1.3f * tan_half;
  float pxx = 2.0f / (float)width, pxy = 2.0f / (float)height;
  float bx = (0.3f * pxx) * (0.3f * pxx), by = (0.3f * pxy) * (0.3f * pxy);
  float view[9];
  orc_view_rotation(cam->rotation_xyzw, view);
  uint64_t kept = 0;
  for (uint64_t j = 0; j < m; ++j) {
    uint64_t i = indices[j];
    if (i >= sc->count) continue;
    const float *pos = &sc->positions[3 * i];
    float p[3] = {pos[0] - cam->position[0], pos[1] - cam->position[1], pos[2] - cam->position[2]};
    float pc[3];
    for (int r = 0; r < 3; ++r)
      pc[r] = view[3 * r + 0] * p[0] + view[3 * r + 1] * p[1] + view[3 * r + 2] * p[2];
    if (!(pc[2] >= cam->near_plane && pc[2] <= cam->far_plane)) continue;
    float inv_z = 1.0f / std::fmax(pc[2], 1e-6f);
    float x_ndc = (pc[0] * f) * inv_z / aspect;
    float y_ndc = (pc[1] * f) * inv_z;
    Cov6 wc{cov6[6 * i + 0], cov6[6 * i + 1], cov6[6 * i + 2],
            cov6[6 * i + 3], cov6[6 * i + 4], cov6[6 * i + 5]};
    const float *r0 = &view[0], *r1 = &view[3], *r2 = &view[6];
    Cov6 cc{cov_quadratic(wc, r0), cov_bilinear(wc, r0, r1), cov_bilinear(wc, r0, r2),
            cov_quadratic(wc, r1), cov_bilinear(wc, r1, r2), cov_quadratic(wc, r2)};
    float cov2[3], u[2], v[2];
    if (!cpu_project_cov(pc, cc, lim_x, lim_y, fx, fy, bx, by, cov2)) continue;
    if (!cpu_ellipse_axes(cov2, u, v)) continue;
    float ext_x = std::fabs(u[0]) + std::fabs(v[0]);
    float ext_y = std::fabs(u[1]) + std::fabs(v[1]);
    if (x_ndc + ext_x < -1.0f || x_ndc - ext_x > 1.0f || y_ndc + ext_y < -1.0f ||
        y_ndc - ext_y > 1.0f)
      continue;
    float al = alpha[i];
    // lib.rs:1161-1166: normalize3 (len2 <= 0 -> (0,0,1)).
    float len2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    float dir[3] = {0.0f, 0.0f, 1.0f};
    if (!(len2 <= 0.0f)) {
      float inv = 1.0f / std::sqrt(len2);
      dir[0] = p[0] * inv; dir[1] = p[1] * inv; dir[2] = p[2] * inv;
    }
    float rgb[3];
    cpu_sh_color(*sc, i, dir, rgb);
    for (int ch = 0; ch < 3; ++ch) rgb[ch] = clamp01(rgb[ch]);
    float *o = &out12[12 * kept];
    o[0] = x_ndc; o[1] = y_ndc; o[2] = u[0]; o[3] = u[1];
    o[4] = v[0]; o[5] = v[1]; o[6] = 0.0f; o[7] = 0.0f;
    o[8] = clamp01(rgb[0] * al); o[9] = clamp01(rgb[1] * al); o[10] = clamp01(rgb[2] * al);
    o[11] = al;
    if (out_index) out_index[kept] = (uint32_t)i;
    ++kept;
  }
  return kept;
}

// Tile-key contract of the CUDA design: walking the depth-sorted visible ids
// in order, each drawn splat emits one (tile, id) pair per tile it covers,
// rows outer, columns inner: per row of its tile rect the exact span
// (orc::row_span), or with exact = 0 the whole rect. Returns the pair count
// (may exceed capacity; only the first `capacity` pairs are written).
uint64_t orc_emit_tile_pairs(const OrcProjected *proj, const OrcRecord *rec, const uint32_t *order,
                             uint64_t v, uint32_t tiles_x, uint32_t tile, uint32_t exact,
                             uint32_t *tile_out, uint32_t *id_out, uint64_t capacity) {
  uint64_t k = 0;
  for (uint64_t j = 0; j < v; ++j) {
    uint32_t s = order[j];
    const OrcProjected &p = proj[s];
    if (!(p.flags & 2u) || p.tile_x1 <= p.tile_x0 || p.tile_y1 <= p.tile_y0) continue;
    const orc::SpanPre pre = orc::span_pre(rec[s]);
    const float inv_tile = 1.0f / (float)tile;
    for (uint32_t ty = p.tile_y0; ty < p.tile_y1; ++ty) {
      uint32_t c0 = p.tile_x0, c1 = p.tile_x1;
      if (exact) orc::row_span(rec[s], pre, ty, tile, inv_tile, p.tile_x0, p.tile_x1, c0, c1);
      for (uint32_t tx = c0; tx < c1; ++tx) {
        if (k < capacity) {
          tile_out[k] = ty * tiles_x + tx;
          id_out[k] = s;
        }
        ++k;
      }
    }
  }
  return k;
}

// Stable counting sort of the pairs by tile: ranges[2*t] = start,
// ranges[2*t+1] = end; sorted_ids holds each tile's ids in emission order.
void orc_tile_lists(const uint32_t *tiles, const uint32_t *ids, uint64_t k, uint32_t num_tiles,
                    uint32_t *ranges, uint32_t *sorted_ids) {
  std::vector<uint64_t> count(num_tiles + 1, 0);
  for (uint64_t i = 0; i < k; ++i) count[tiles[i] + 1]++;
  for (uint32_t t = 0; t < num_tiles; ++t) count[t + 1] += count[t];
  for (uint32_t t = 0; t < num_tiles; ++t) {
    ranges[2 * t] = (uint32_t)count[t];
    ranges[2 * t + 1] = (uint32_t)count[t + 1];
  }
  std::vector<uint64_t> cursor(count.begin(), count.end() - 1);
  for (uint64_t i = 0; i < k; ++i) sorted_ids[cursor[tiles[i]]++] = ids[i];
}

// Reference formulation of the per-tile order: a stable ascending sort of
// 64-bit keys (tile << 32) | ~depth_bits with values in id order.
void orc_sort_u64_pairs_stable(uint64_t *keys, uint32_t *values, uint64_t n) {
  std::vector<std::pair<uint64_t, uint32_t>> v(n);
  for (uint64_t i = 0; i < n; ++i) v[i] = {keys[i], values[i]};
  std::stable_sort(v.begin(), v.end(),
                   [](const auto &a, const auto &b) { return a.first < b.first; });
  for (uint64_t i = 0; i < n; ++i) {
    keys[i] = v[i].first;
    values[i] = v[i].second;
  }
}

float orc_exp_neg(float x) { return exp_neg(x); }

// The reference image model: instanced quads in sorted (back-to-front) order,
// fs_main coverage and weight, PREMULTIPLIED_ALPHA_BLENDING
// (draw_pass.rs:75: dst = src + dst * (1 - src.a)) into an Rgba8Unorm target
// cleared to zero (lib.rs:53, 2746). Each blend result is rounded to the
// nearest UNORM8 value; the source is blended in f32. The exact rounding of a
// given GPU's blender is not specified by the reference; round-to-nearest is
// assumed.
void orc_raster_unorm8(const OrcRecord *records, const OrcProjected *proj,
                       const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                       uint8_t *rgba, int32_t threads) {
  std::memset(rgba, 0, (size_t)width * height * 4);
  parallel_rows(height, threads, [&](uint32_t ya, uint32_t yb) {
    unorm8_band(records, proj, order, v, width, height, rgba, ya, yb);
  });
}

// Rows [y0, y1) of the reference image model; the other rows stay zero. A
// band of a large frame (the 3M-splat 4K stress frame) finishes in seconds.
void orc_raster_unorm8_rows(const OrcRecord *records, const OrcProjected *proj,
                            const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                            uint8_t *rgba, int32_t threads, uint32_t y0, uint32_t y1) {
  std::memset(rgba, 0, (size_t)width * height * 4);
  y1 = std::min(y1, height);
  if (y0 >= y1) return;
  parallel_rows(y1 - y0, threads, [&](uint32_t ya, uint32_t yb) {
    unorm8_band(records, proj, order, v, width, height, rgba, y0 + ya, y0 + yb);
  });
}

// FP64 evaluation of the same image: local coordinates, coverage, weights and
// blending in double precision, one rounding to UNORM8 at the end.
void orc_raster_f64(const OrcRecord *records, const OrcProjected *proj, const uint32_t *order,
                    uint64_t v, uint32_t width, uint32_t height, uint8_t *rgba,
                    double *rgba_f64, int32_t threads) {
  orc_raster_f64_rows(records, proj, order, v, width, height, rgba, rgba_f64, threads, 0, height);
}

void orc_raster_f64_rows(const OrcRecord *records, const OrcProjected *proj,
                         const uint32_t *order, uint64_t v, uint32_t width, uint32_t height,
                         uint8_t *rgba, double *rgba_f64, int32_t threads, uint32_t row0,
                         uint32_t row1) {
  std::vector<double> acc((size_t)width * height * 4, 0.0);
  row1 = std::min(row1, height);
  parallel_rows(row1 > row0 ? row1 - row0 : 0, threads, [&](uint32_t ra, uint32_t rb) {
    const uint32_t ya = row0 + ra, yb = row0 + rb;
    for (uint64_t j = 0; j < v; ++j) {
      uint32_t s = order[j];
      const OrcProjected &p = proj[s];
      if (!(p.flags & 2u)) continue;
      const OrcRecord &r = records[s];
      int x0, x1, y0, y1;
      quad_pixel_bbox(p, r, width, height, x0, x1, y0, y1);
      y0 = std::max<int>(y0, (int)ya);
      y1 = std::min<int>(y1, (int)yb - 1);
      double uu = (double)p.axis_u[0] * p.axis_u[0] + (double)p.axis_u[1] * p.axis_u[1];
      double vv = (double)p.axis_v[0] * p.axis_v[0] + (double)p.axis_v[1] * p.axis_v[1];
      for (int py = y0; py <= y1; ++py)
        for (int px = x0; px <= x1; ++px) {
          double xn = ((double)px + 0.5) * 2.0 / width - 1.0 - p.center_ndc[0];
          double yn = 1.0 - ((double)py + 0.5) * 2.0 / height - p.center_ndc[1];
          double lx = (p.axis_u[0] * xn + p.axis_u[1] * yn) / uu;
          double ly = (p.axis_v[0] * xn + p.axis_v[1] * yn) / vv;
          double sd = p.extent_scale;
          if (!(std::fabs(lx) <= sd && std::fabs(ly) <= sd)) continue;
          double r2 = lx * lx + ly * ly;
          if (!(r2 <= 1.0)) continue;
          double g = std::exp(-4.5 * r2);
          double w = (double)p.color[3] * g;
          if (!(w > 1.0 / 256.0)) continue;
          double *d = &acc[((size_t)py * width + px) * 4];
          for (int ch = 0; ch < 3; ++ch) d[ch] = (double)p.color[ch] * g + d[ch] * (1.0 - w);
          d[3] = w + d[3] * (1.0 - w);
        }
    }
  });
  for (size_t i = 0; i < acc.size(); ++i) {
    double c = std::min(std::max(acc[i], 0.0), 1.0);
    if (rgba) rgba[i] = (uint8_t)std::nearbyint(c * 255.0);
    if (rgba_f64) rgba_f64[i] = acc[i];
  }
}

// Restatement of the CUDA FP32 front-to-back tile raster: each pixel walks its
// tile's list from the back (nearest) to the front (see tiles_fp32_band).
void orc_raster_tiles_fp32(const OrcRecord *records, const uint32_t *ranges,
                           const uint32_t *sorted_ids, uint32_t width, uint32_t height,
                           uint32_t tile, uint32_t tiles_x, uint8_t *rgba, int32_t threads) {
  parallel_rows(height, threads, [&](uint32_t ya, uint32_t yb) {
    tiles_fp32_band(records, ranges, sorted_ids, width, tile, tiles_x, rgba, ya, yb);
  });
}

void orc_raster_tiles_fp32_rows(const OrcRecord *records, const uint32_t *ranges,
                                const uint32_t *sorted_ids, uint32_t width, uint32_t height,
                                uint32_t tile, uint32_t tiles_x, uint8_t *rgba, int32_t threads,
                                uint32_t y0, uint32_t y1) {
  std::memset(rgba, 0, (size_t)width * height * 4);
  y1 = std::min(y1, height);
  if (y0 >= y1) return;
  parallel_rows(y1 - y0, threads, [&](uint32_t ya, uint32_t yb) {
    tiles_fp32_band(records, ranges, sorted_ids, width, tile, tiles_x, rgba, y0 + ya, y0 + yb);
  });
}

// The reference's SortedAlpha frame on the CPU: preprocess and sort on one
// thread (as Renderer::render_frame does, lib.rs:723-742), then the vertex
// stage and the UNORM8 raster on `threads` host threads.
int32_t orc_render_reference_frame(const OrcScene *scene, const float *alpha,
                                   const float *extent_scale, const float *cov6,
                                   const OrcCamera *camera, uint32_t width, uint32_t height,
                                   uint32_t raster_rows, uint8_t *rgba, int32_t threads,
                                   OrcFrameTiming *timing) {
  using clk = std::chrono::steady_clock;
  auto ms = [](clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  auto t0 = clk::now();
  uint64_t n = scene->count;
  std::vector<uint32_t> keys(n ? n : 1), order(n ? n : 1);
  uint64_t v = orc_preprocess_visible(scene->positions, n, camera, keys.data(), order.data());
  if (v == UINT64_MAX) return 1;
  auto t1 = clk::now();
  orc_sort_values_by_keys(keys.data(), order.data(), v);
  auto t2 = clk::now();
  OrcFrameParams p;
  frame_params(*camera, width, height, 16, scene->sh_degree, p);
  std::vector<OrcProjected> proj(n ? n : 1);
  std::vector<OrcRecord> rec(n ? n : 1);
  uint64_t drawn = 0;
  {
    int nt = std::max(1, threads);
    std::vector<std::thread> pool;
    std::vector<uint64_t> drawn_t(nt, 0);
    for (int t = 0; t < nt; ++t)
      pool.emplace_back([&, t]() {
        for (uint64_t j = t; j < v; j += nt) {
          uint32_t s = order[j];
          project_one(*scene, alpha, extent_scale, cov6, p, s, proj[s], rec[s]);
          if (proj[s].flags & 2u) drawn_t[t]++;
        }
      });
    for (auto &th : pool) th.join();
    for (int t = 0; t < nt; ++t) drawn += drawn_t[t];
  }
  auto t3 = clk::now();
  // raster_rows < height composites only the top rows (a bounded sample).
  uint32_t rows = raster_rows && raster_rows < height ? raster_rows : height;
  std::memset(rgba, 0, (size_t)width * height * 4);
  parallel_rows(rows, threads, [&](uint32_t ya, uint32_t yb) {
    unorm8_band(rec.data(), proj.data(), order.data(), v, width, height, rgba, ya, yb);
  });
  auto t4 = clk::now();
  if (timing) {
    timing->preprocess_ms = ms(t0, t1);
    timing->sort_ms = ms(t1, t2);
    timing->project_ms = ms(t2, t3);
    timing->raster_ms = ms(t3, t4);
    timing->total_ms = ms(t0, t4);
    timing->visible = v;
    timing->drawn = drawn;
  }
  return 0;
}

}  // extern "C"
