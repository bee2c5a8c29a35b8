// K1: per-splat preprocess. Built with --fmad=false: every f32 expression
// rounds after each operation, as the reference's f32 code does, so depth
// keys, projected records and tile rects match the CPU restatement bit for
// bit (division and sqrt are IEEE-rounded; there are no transcendental calls
// per frame — alpha, extent scale and covariance are precomputed at load).
//
// One thread per splat:
//   1. depth = row2 . (p - cam); visible iff near <= depth <= far
//      (preprocess_visible_into, crates/gsplat-render-wgpu/src/lib.rs:1263-1296);
//   2. project_splat + eval_color (splat_surface_direct.wgsl:131-217, 233-334),
//      tile rect of the ellipse |local| <= s and the pixel-space record;
//   3. digit histograms of the depth keys for the radix sort;
//   4. visible splats are compacted in id order with a block scan and a
//      decoupled look-back, emitting (~bits(max(depth, 0)), id) so that an
//      ascending stable sort yields the reference's descending-depth order.

#include "device_common.cuh"
#include "kernels.h"

namespace gsr {

namespace {

__device__ __forceinline__ float clampf(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}

struct Cov6 {
  float xx, xy, xz, yy, yz, zz;
};

// splat_surface_direct.wgsl:96-103
__device__ __forceinline__ float cov_quadratic(const Cov6 &c, float r0, float r1, float r2) {
  return r0 * r0 * c.xx + 2.0f * r0 * r1 * c.xy + 2.0f * r0 * r2 * c.xz + r1 * r1 * c.yy +
         2.0f * r1 * r2 * c.yz + r2 * r2 * c.zz;
}

// splat_surface_direct.wgsl:105-110
__device__ __forceinline__ float cov_bilinear(const Cov6 &c, const float *a, const float *b) {
  float bx = c.xx * b[0] + c.xy * b[1] + c.xz * b[2];
  float by = c.xy * b[0] + c.yy * b[1] + c.yz * b[2];
  float bz = c.xz * b[0] + c.yz * b[1] + c.zz * b[2];
  return a[0] * bx + a[1] * by + a[2] * bz;
}

constexpr int kK1Threads = 256;

// Float k of a splat's colour data; plane q of the splat is planes[q * kK1Threads]
// (the block's shared-memory stage, one float4 per splat and plane).
__device__ __forceinline__ float plane_float(const float4 *planes, int k) {
  const float4 v = planes[(k >> 2) * kK1Threads];
  switch (k & 3) {
    case 0: return v.x;
    case 1: return v.y;
    case 2: return v.z;
    default: return v.w;
  }
}

// eval_sh_rgb (splat_surface_direct.wgsl:233-326): the basis scalars are the
// left-associated prefixes of each WGSL term, so each channel accumulates
// exactly the WGSL sequence. `f` holds (DC rgb, rest 1 rgb, rest 2 rgb, ...).
template <int kPlanes>
__device__ __forceinline__ void eval_sh(const float4 *f, uint32_t degree, float x, float y,
                                        float z, float rgb[3]) {
  const float c0 = 0.28209479177387814f;
  const float c1 = 0.4886025119029199f;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) rgb[ch] = c0 * plane_float(f, ch);
  if (degree == 0) return;
  {
    float b0 = c1 * y, b1 = c1 * z, b2 = c1 * x;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
      rgb[ch] = rgb[ch] - b0 * plane_float(f, 3 + ch) + b1 * plane_float(f, 6 + ch) -
                b2 * plane_float(f, 9 + ch);
  }
  if (degree == 1 || kPlanes < 7) return;
  float xx = x * x, yy = y * y, zz = z * z;
  float xy = x * y, yz = y * z, xz = x * z;
  {
    float b[5] = {1.0925484305920792f * xy, -1.0925484305920792f * yz,
                  0.31539156525252005f * (2.0f * zz - xx - yy), -1.0925484305920792f * xz,
                  0.5462742152960396f * (xx - yy)};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float r = rgb[ch];
#pragma unroll
      for (int k = 0; k < 5; ++k) r = r + b[k] * plane_float(f, 3 * (4 + k) + ch);
      rgb[ch] = r;
    }
  }
  if (degree == 2 || kPlanes < 12) return;
  {
    float b[7] = {-0.5900435899266435f * y * (3.0f * xx - yy),
                  2.890611442640554f * xy * z,
                  -0.4570457994644658f * y * (4.0f * zz - xx - yy),
                  0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
                  -0.4570457994644658f * x * (4.0f * zz - xx - yy),
                  1.445305721320277f * z * (xx - yy),
                  -0.5900435899266435f * x * (xx - 3.0f * yy)};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float r = rgb[ch];
#pragma unroll
      for (int k = 0; k < 7; ++k) r = r + b[k] * plane_float(f, 3 * (9 + k) + ch);
      rgb[ch] = r;
    }
  }
  if (degree == 3 || kPlanes < 19) return;
  {
    float b[9] = {2.5033429417967046f * xy * (xx - yy),
                  -1.7701307697799304f * yz * (3.0f * xx - yy),
                  0.9461746957575601f * xy * (7.0f * zz - 1.0f),
                  -0.6690465435572892f * yz * (7.0f * zz - 3.0f),
                  0.10578554691520431f * (zz * (35.0f * zz - 30.0f) + 3.0f),
                  -0.6690465435572892f * xz * (7.0f * zz - 3.0f),
                  0.47308734787878004f * (xx - yy) * (7.0f * zz - 1.0f),
                  -1.7701307697799304f * xz * (xx - 3.0f * yy),
                  0.6258357354491761f * (xx * (xx - 3.0f * yy) - yy * (3.0f * xx - yy))};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      float r = rgb[ch];
#pragma unroll
      for (int k = 0; k < 9; ++k) r = r + b[k] * plane_float(f, 3 * (16 + k) + ch);
      rgb[ch] = r;
    }
  }
}

// The per-splat vertex stage for a depth-visible splat. Returns false when
// project_splat marks the splat invalid (behind near, beyond far, or outside
// the frustum by its axis extents).
// `ca`, `cb` are the splat's covariance planes and `col` its first colour
// plane in the block's stage (planes kK1Threads float4 apart).
template <int kPlanes>
__device__ __forceinline__ bool project(const FrameParams &p, const float4 &pa, const float4 &ca,
                                        const float4 &cb, const float4 *col, const float rel[3],
                                        float depth, Record &rec, uint2 &rect, ProjectedDev *dbg) {
  float px = p.r0[0] * rel[0] + p.r0[1] * rel[1] + p.r0[2] * rel[2];
  float py = p.r1[0] * rel[0] + p.r1[1] * rel[1] + p.r1[2] * rel[2];
  float z = depth;
  if (z < p.near_plane || z > p.far_plane || z <= 1e-6f) return false;
  float inv_z = 1.0f / z;
  float x_ndc = (px * p.f) * inv_z / p.aspect;
  float y_ndc = (py * p.f) * inv_z;

  Cov6 wc{ca.x, ca.y, ca.z, ca.w, cb.x, cb.y};
  Cov6 cc{cov_quadratic(wc, p.r0[0], p.r0[1], p.r0[2]), cov_bilinear(wc, p.r0, p.r1),
          cov_bilinear(wc, p.r0, p.r2),                 cov_quadratic(wc, p.r1[0], p.r1[1], p.r1[2]),
          cov_bilinear(wc, p.r1, p.r2),                 cov_quadratic(wc, p.r2[0], p.r2[1], p.r2[2])};
  float x_cl = clampf(px / z, -p.lim_x, p.lim_x) * z;
  float y_cl = clampf(py / z, -p.lim_y, p.lim_y) * z;
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
  float term = sqrtf(fmaxf(amco2 * amco2 + b * b, 0.0f));
  float major = fmaxf(apco2 + term, 1e-10f);
  float minor = fmaxf(apco2 - term, 1e-10f);
  float ux = 1.0f, uy = 0.0f;
  if (fabsf(b) > 1e-8f) {
    float vx = b, vy = major - a;
    float len2 = vx * vx + vy * vy;
    if (!(len2 <= 1e-20f)) {
      float inv = 1.0f / sqrtf(len2);
      ux = vx * inv;
      uy = vy * inv;
    }
  } else if (a < c) {
    ux = 0.0f;
    uy = 1.0f;
  }
  float major_r = clampf(sqrtf(major) * 3.0f, 1e-4f, 2.0f);
  float minor_r = clampf(sqrtf(minor) * 3.0f, 1e-4f, 2.0f);
  major_r = fminf(major_r, minor_r * 64.0f);
  float au0 = ux * major_r, au1 = uy * major_r;
  float av0 = -uy * minor_r, av1 = ux * minor_r;
  float ext_x = fabsf(au0) + fabsf(av0);
  float ext_y = fabsf(au1) + fabsf(av1);
  if (x_ndc + ext_x < -1.0f || x_ndc - ext_x > 1.0f || y_ndc + ext_y < -1.0f ||
      y_ndc - ext_y > 1.0f)
    return false;

  const float al = pa.w;
  const float s = cb.z;
  // eval_color: dir = normalize3_or_default(pos - cam, (0,0,1))
  float len2 = rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2];
  float dx = 0.0f, dy = 0.0f, dz = 1.0f;
  if (!(len2 <= 1e-20f)) {
    float inv = 1.0f / sqrtf(len2);
    dx = rel[0] * inv;
    dy = rel[1] * inv;
    dz = rel[2] * inv;
  }
  float rgb[3];
  eval_sh<kPlanes>(col, p.sh_degree, dx, dy, dz, rgb);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) rgb[ch] = clampf(rgb[ch] + 0.5f, 0.0f, 1.0f);
  float pr = rgb[0] * al, pg = rgb[1] * al, pb = rgb[2] * al;

  float cxp = (x_ndc + 1.0f) * p.half_w - 0.5f;
  float cyp = (1.0f - y_ndc) * p.half_h - 0.5f;
  float uu = au0 * au0 + au1 * au1;
  float vv = av0 * av0 + av1 * av1;
  rec.a = make_float4(cxp, cyp, (au0 * p.sx) / uu, (au1 * p.sy) / uu);
  rec.b = make_float4((av0 * p.sx) / vv, (av1 * p.sy) / vv, s, al);
  // colour before alpha and log2(alpha) (hardware logarithm): the FP32
  // raster's weight is 2^(log2 alpha - 4.5 log2(e) r2)
  rec.c = make_float4(rgb[0], rgb[1], rgb[2], __log2f(al));

  rect = make_uint2(0u, 0u);
  if (al > 1.0f / 256.0f) {
    float ex = s * sqrtf(au0 * au0 + av0 * av0) * p.half_w;
    float ey = s * sqrtf(au1 * au1 + av1 * av1) * p.half_h;
    ex = ex * 1.00001f + 0.001f;
    ey = ey * 1.00001f + 0.001f;
    float fx0 = fmaxf(ceilf(cxp - ex), 0.0f);
    float fx1 = fminf(floorf(cxp + ex), (float)(p.width - 1));
    float fy0 = fmaxf(ceilf(cyp - ey), 0.0f);
    float fy1 = fminf(floorf(cyp + ey), (float)(p.height - 1));
    if (fx0 <= fx1 && fy0 <= fy1) {
      uint32_t tx0 = (uint32_t)fx0 / p.tile, tx1 = (uint32_t)fx1 / p.tile + 1;
      uint32_t ty0 = (uint32_t)fy0 / p.tile, ty1 = (uint32_t)fy1 / p.tile + 1;
      rect = make_uint2(tx0 | (ty0 << 16), tx1 | (ty1 << 16));
    }
  }
  if (dbg) {
    dbg->center_ndc[0] = x_ndc;
    dbg->center_ndc[1] = y_ndc;
    dbg->axis_u[0] = au0;
    dbg->axis_u[1] = au1;
    dbg->axis_v[0] = av0;
    dbg->axis_v[1] = av1;
    dbg->color[0] = pr;
    dbg->color[1] = pg;
    dbg->color[2] = pb;
    dbg->color[3] = al;
    dbg->extent_scale = s;
    dbg->flags |= 2u;
    dbg->tile_x0 = (uint16_t)(rect.x & 0xffffu);
    dbg->tile_y0 = (uint16_t)(rect.x >> 16);
    dbg->tile_x1 = (uint16_t)(rect.y & 0xffffu);
    dbg->tile_y1 = (uint16_t)(rect.y >> 16);
  }
  return true;
}

constexpr int kK1Warps = kK1Threads / 32;
constexpr uint32_t kPackedHotBytes = 20u * kK1Threads;   // one slice of hot records
constexpr uint32_t kPackedSideBytes = 48u * kK1Threads;  // one slice of SH sidecars
constexpr uint32_t kPackedTableBytes = 4u * kPackedFloats;  // header and tables
static_assert(kPackedTableBytes % 16 == 0, "the table is one bulk copy");
// Resident blocks per SM the register allocation must allow (tuning knob).
#ifndef GSR_K1_MIN_BLOCKS
#define GSR_K1_MIN_BLOCKS 3
#endif

// The block's slice of the scene planes in shared memory: 256 splats of
// position/alpha, both covariance planes and kPlanes colour planes.
template <int kPlanes>
struct K1Stage {
  float4 pos[kK1Threads];
  float4 cov_a[kK1Threads];
  float4 cov_b[kK1Threads];
  float4 color[kPlanes][kK1Threads];
  uint64_t bar[2];  // [0]: positions, [1]: covariance and colour
};

// Decode of a packed splat into the thread's column of the stage, the values
// a plane-format scene would hold there: position + alpha, the covariance
// terms + extent scale, and the colour planes (the DC as (rgb10 - 0.5) / C0,
// rest coefficients i8 / 127 * scale). Follows splat_surface_packed.wgsl:
// 128-241 (position, opacity, smallest-three quaternion, rotation and
// covariance from log scales); the axis variances exp(2 log_scale) and the
// extent scales come from the scene's tables (computed on the host, staged
// in shared memory with the slice).
// x / d for the values the packed decode divides by a constant (integers in
// [-127, 127], [0, 255], [0, 1023], [0, 65535] and the 1,024 RGB10 levels
// less one half over C0): the product with RN(1/d) and one fma correction,
// equal to the IEEE quotient for every such x (checked exhaustively by the
// tests), three instructions instead of a division.
__device__ __forceinline__ float div_const(float x, float d, float r) {
  const float q = __fmul_rn(x, r);
  return __fmaf_rn(__fmaf_rn(-q, d, x), r, q);
}

struct PackedIn {
  uint32_t w[5];      // hot record
  uint32_t side[12];  // SH sidecar (zero without one)
  float h[11];        // bounds min, span, log-scale min, extent, SH scales
  float var[3];       // the axis variances of the three scale codes
  float ext;          // the extent scale of the opacity code
};

template <int kPlanes>
__device__ __forceinline__ void decode_packed(uint32_t planes, const PackedIn &in,
                                              K1Stage<kPlanes> &st) {
  const uint32_t *w = in.w;
  const uint32_t *side = in.side;
  const float *h = in.h;
  const uint32_t t = threadIdx.x;
  const uint32_t pu[3] = {w[0] & 0xffffu, w[0] >> 16, w[1] & 0xffffu};
  float pos[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    pos[a] = h[a] + div_const((float)pu[a], 65535.0f, 1.0f / 65535.0f) * h[3 + a];
  const uint32_t op = (w[1] >> 16) & 0xffu;
  const float alpha = fminf(fmaxf(div_const((float)op, 255.0f, 1.0f / 255.0f), 1e-4f), 1.0f - 1e-4f);
  st.pos[t] = make_float4(pos[0], pos[1], pos[2], alpha);
  const float sx2 = in.var[0], sy2 = in.var[1], sz2 = in.var[2];
  const uint32_t mi = w[3] & 3u;
  const float inv_sqrt2 = 0.70710678118654752440f;
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
    c[k] = (div_const((float)((w[3] >> (2 + 10 * k)) & 0x3ffu), 1023.0f, 1.0f / 1023.0f) * 2.0f -
            1.0f) * inv_sqrt2;
  const float sum_sq = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
  const float dropped = sqrtf(fmaxf(1.0f - sum_sq, 0.0f));
  float q[4];
  q[0] = mi == 0 ? dropped : c[0];
  q[1] = mi == 0 ? c[0] : (mi == 1 ? dropped : c[1]);
  q[2] = mi <= 1 ? c[1] : (mi == 2 ? dropped : c[2]);
  q[3] = mi <= 2 ? c[2] : dropped;
  const float len = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const float x = q[0] / len, y = q[1] / len, z = q[2] / len, ww = q[3] / len;
  const float x2 = x + x, y2 = y + y, z2 = z + z;
  const float xx = x * x2, yy = y * y2, zz = z * z2;
  const float xy = x * y2, xz = x * z2, yz = y * z2;
  const float wx = ww * x2, wy = ww * y2, wz = ww * z2;
  const float r[9] = {1.0f - (yy + zz), xy - wz, xz + wy,
                      xy + wz, 1.0f - (xx + zz), yz - wx,
                      xz - wy, yz + wx, 1.0f - (xx + yy)};
  auto term = [&](int a, int b) {
    return sx2 * r[3 * a] * r[3 * b] + sy2 * r[3 * a + 1] * r[3 * b + 1] +
           sz2 * r[3 * a + 2] * r[3 * b + 2];
  };
  st.cov_a[t] = make_float4(term(0, 0), term(0, 1), term(0, 2), term(1, 1));
  st.cov_b[t] = make_float4(term(1, 2), term(2, 2), in.ext, 0.0f);
  // Colour: float f = 3 c + ch is coefficient c (0 = DC) of channel ch.
  const uint32_t pc = planes == 1 ? 0u : planes == 3 ? 3u : planes == 7 ? 8u : 15u;
  auto coeff = [&](uint32_t f) {
    constexpr float kC0 = 0.28209479177387814f;
    if (f < 3) {
      const float v = div_const((float)((w[4] >> (10 * f)) & 0x3ffu), 1023.0f, 1.0f / 1023.0f);
      return div_const(v - 0.5f, kC0, 1.0f / kC0);
    }
    const uint32_t k = f / 3 - 1, ch = f % 3;
    if (k >= pc) return 0.0f;
    const uint32_t byte = ch * 15 + k;
    const int8_t v = (int8_t)((side[byte >> 2] >> (8 * (byte & 3))) & 0xffu);
    return div_const((float)v, 127.0f, 1.0f / 127.0f) * h[8 + ch];
  };
#pragma unroll
  for (int pl = 0; pl < kPlanes; ++pl)
    if ((uint32_t)pl < planes)
      st.color[pl][t] = make_float4(coeff(4 * pl), coeff(4 * pl + 1), coeff(4 * pl + 2),
                                    coeff(4 * pl + 3));
}

// One block covers 256 consecutive splats of one scene for every view of a
// view set (up to kMaxSetViews views of that scene). One thread stages the
// block's slice of every scene plane into shared memory with bulk copies
// (cp.async.bulk, completion on an mbarrier), so all of the block's HBM
// reads are in flight at once and every view of the set reads the slice
// from shared memory: the scene is read from HBM once per set. Positions
// arrive on their own barrier, so the depth tests start while covariance and
// colour are still in flight. Per view, the arithmetic is exactly the
// single-view sequence. Visible entries are compacted in (block, view, id)
// order, which keeps every view's entries in ascending id order.
template <int kPlanes, bool kDebug>
__global__ void __launch_bounds__(kK1Threads, GSR_K1_MIN_BLOCKS)
    preprocess_kernel(const ViewDev *__restrict__ views, const ViewSetDev *__restrict__ sets,
                      uint32_t num_sets, uint32_t total_blocks, K1Buffers b) {
  extern __shared__ __align__(128) unsigned char k1_dyn[];
  K1Stage<kPlanes> &st = *reinterpret_cast<K1Stage<kPlanes> *>(k1_dyn);
  __shared__ uint32_t s_block;
  __shared__ uint32_t s_set;
  __shared__ uint32_t s_lost;  // a stage wait expired twice: copies may still land
  __shared__ uint32_t s_cnt[kMaxSetViews][kK1Warps];  // visible per view and warp
  __shared__ uint32_t s_hist[4][256];
  __shared__ FrameParams s_params[kMaxSetViews];  // the set's per-view uniforms
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    const uint32_t blk = atomicAdd(&b.counters->k1_ticket, 1u);
    s_block = blk;
    s_lost = 0;
    const uint32_t si = find_view(num_sets, blk, [&](uint32_t v) { return sets[v].block_base; });
    s_set = si;
    const ViewSetDev set0 = sets[si];
    const SceneDev sc0 = views[set0.first_view].sc;
    const uint32_t i0 = (blk - set0.block_base) * kK1Threads;
    const uint32_t bytes = min((uint32_t)kK1Threads, sc0.n - i0) * 16u;  // >= 16: i0 < n
    mbar_init(&st.bar[0], 1);
    mbar_init(&st.bar[1], 1);
    fence_barrier_init();
    if (sc0.hot) {
      // Packed scene: the slice's hot records and SH sidecars (whole slices;
      // the arrays are padded), staged at the start of the block's stage.
      // The scene's header and tables follow them.
      unsigned char *raw = reinterpret_cast<unsigned char *>(&st);
      const uint32_t side = sc0.sidecar ? kPackedSideBytes : 0u;
      mbar_arrive_expect_tx(&st.bar[0], kPackedHotBytes + kPackedTableBytes);
      bulk_copy_g2s(raw, sc0.hot + (size_t)i0 * 5, kPackedHotBytes, &st.bar[0]);
      bulk_copy_g2s(raw + kPackedHotBytes + side, sc0.packed, kPackedTableBytes, &st.bar[0]);
      mbar_arrive_expect_tx(&st.bar[1], side);
      if (side) bulk_copy_g2s(raw + kPackedHotBytes, sc0.sidecar + (size_t)i0 * 48, side, &st.bar[1]);
    } else {
      mbar_arrive_expect_tx(&st.bar[0], bytes);
      bulk_copy_g2s(st.pos, sc0.pos_alpha + i0, bytes, &st.bar[0]);
      mbar_arrive_expect_tx(&st.bar[1], bytes * (2u + sc0.planes));
      bulk_copy_g2s(st.cov_a, sc0.cov_a + i0, bytes, &st.bar[1]);
      bulk_copy_g2s(st.cov_b, sc0.cov_b + i0, bytes, &st.bar[1]);
      for (uint32_t q = 0; q < sc0.planes && q < (uint32_t)kPlanes; ++q)
        bulk_copy_g2s(st.color[q], sc0.color + (size_t)q * sc0.n + i0, bytes, &st.bar[1]);
    }
  }
  for (uint32_t k = threadIdx.x; k < 4 * 256; k += kK1Threads) (&s_hist[0][0])[k] = 0;
  __syncthreads();
  const uint32_t block = s_block;
  const ViewSetDev set = sets[s_set];
  {
    constexpr uint32_t kWords = sizeof(FrameParams) / 4;
    static_assert(sizeof(FrameParams) % 4 == 0, "FrameParams is copied as words");
    for (uint32_t w = threadIdx.x; w < set.count * kWords; w += kK1Threads) {
      const uint32_t v = w / kWords, o = w % kWords;
      reinterpret_cast<uint32_t *>(&s_params[v])[o] =
          reinterpret_cast<const uint32_t *>(&views[set.first_view + v].p)[o];
    }
  }
  __syncthreads();
  const SceneDev sc = views[set.first_view].sc;
  const uint32_t i = (block - set.block_base) * kK1Threads + threadIdx.x;
  const bool valid = i < sc.n;
  // Stage waits: a wait that expires sets the error bit (the frame reports an
  // internal error) and is retried once, bounded, for the copies in flight.
  // When the retry expires too, this thread reads nothing of that stage (its
  // splat counts as not visible, or as not drawn), the block never writes
  // into the stage and does not retire its barriers; the block may then exit
  // while copies still land in its shared memory, which only a faulting
  // device can cause.
  bool ok0 = true, ok1 = true;
  if (sc.hot) {
    // Every thread takes its packed record, the scene constants and its table
    // entries into registers, then the block overwrites the stage with the
    // decoded planes (not at all if any thread's wait expired twice).
    ok0 = mbar_wait(&st.bar[0], 0, &b.counters->error) || mbar_wait(&st.bar[0], 0, &b.counters->error);
    ok1 = mbar_wait(&st.bar[1], 0, &b.counters->error) || mbar_wait(&st.bar[1], 0, &b.counters->error);
    const uint32_t *raw = reinterpret_cast<const uint32_t *>(&st);
    PackedIn in;
#pragma unroll
    for (int k = 0; k < 5; ++k) in.w[k] = raw[5 * threadIdx.x + k];
    const uint32_t side_words = sc.sidecar ? kPackedSideBytes / 4 : 0u;
#pragma unroll
    for (int k = 0; k < 12; ++k)
      in.side[k] = side_words ? raw[kPackedHotBytes / 4 + 12 * threadIdx.x + k] : 0u;
    const float *table = reinterpret_cast<const float *>(raw + kPackedHotBytes / 4 + side_words);
#pragma unroll
    for (int k = 0; k < 11; ++k) in.h[k] = table[k];
    const float *var = table + kPackedHeaderFloats;
    in.var[0] = var[in.w[2] & 0x3ffu];
    in.var[1] = var[(in.w[2] >> 10) & 0x3ffu];
    in.var[2] = var[(in.w[2] >> 20) & 0x3ffu];
    in.ext = table[kPackedHeaderFloats + kPackedVarLut + ((in.w[1] >> 16) & 0xffu)];
    if (__syncthreads_or(!(ok0 && ok1))) {
      ok0 = ok1 = false;
      if (threadIdx.x == 0) s_lost = 1;
    } else {
      decode_packed<kPlanes>(sc.planes, in, st);
    }
    __syncthreads();
  } else {
    ok0 = mbar_wait(&st.bar[0], 0, &b.counters->error) || mbar_wait(&st.bar[0], 0, &b.counters->error);
    if (!ok0) s_lost = 1;
  }
  const float4 pa = valid && ok0 ? st.pos[threadIdx.x] : make_float4(0.f, 0.f, 0.f, 0.f);

  // Depth test for every view of the set. The block's visible count is
  // known right after it: publish it for the successors' look-back before
  // doing the heavy vertex stage.
  uint32_t vis_bits = 0;
  for (uint32_t k = 0; k < set.count; ++k) {
    const FrameParams &p = s_params[k];
    const float rx = pa.x - p.cam[0], ry = pa.y - p.cam[1], rz = pa.z - p.cam[2];
    const float depth = p.r2[0] * rx + p.r2[1] * ry + p.r2[2] * rz;
    const bool vis = valid && ok0 && depth >= p.near_plane && depth <= p.far_plane;
    const uint32_t ballot = __ballot_sync(0xffffffffu, vis);
    if (lane == 0) s_cnt[k][warp] = __popc(ballot);
    vis_bits |= (vis ? 1u : 0u) << k;
  }
  __syncthreads();
  uint32_t block_total = 0;
  for (uint32_t k = 0; k < set.count; ++k)
#pragma unroll
    for (int w = 0; w < kK1Warps; ++w) block_total += s_cnt[k][w];
  if (threadIdx.x == 0) lookback_publish_aggregate(b.status, block, block_total);
  if (threadIdx.x < set.count) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kK1Warps; ++w) c += s_cnt[threadIdx.x][w];
    if (c) atomicAdd(&b.view_counters[set.first_view + threadIdx.x].visible, c);
  }

  if (!sc.hot) {
    ok1 = mbar_wait(&st.bar[1], 0, &b.counters->error) || mbar_wait(&st.bar[1], 0, &b.counters->error);
    if (!ok1) s_lost = 1;
  }
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 ca = ok1 ? st.cov_a[threadIdx.x] : zero4;
  const float4 cb = ok1 ? st.cov_b[threadIdx.x] : zero4;
  const float4 *col = &st.color[0][threadIdx.x];
  for (uint32_t k = 0; k < set.count; ++k) {
    const uint32_t view = set.first_view + k;
    const FrameParams &p = s_params[k];
    const uint32_t gid = views[view].splat_base + i;
    const bool vis = (vis_bits >> k) & 1u;
    float rel[3] = {pa.x - p.cam[0], pa.y - p.cam[1], pa.z - p.cam[2]};
    const float depth = p.r2[0] * rel[0] + p.r2[1] * rel[1] + p.r2[2] * rel[2];
    ProjectedDev *dbg = nullptr;
    if (kDebug && valid) {
      dbg = &b.projected[gid];
      ProjectedDev z = {};
      z.depth = depth;
      z.flags = vis ? 1u : 0u;
      *dbg = z;
    }
    bool drawn = false;
    // Digit histograms of the depth keys for every radix pass (every
    // compacted key is counted).
    if (vis && !b.reuse_order) {
      const uint32_t key = ~__float_as_uint(fmaxf(depth, 0.0f));
#pragma unroll
      for (int d = 0; d < 4; ++d) atomicAdd(&s_hist[d][(key >> (8 * d)) & 255u], 1u);
    }
    if (vis && ok1) {
      Record rec;
      uint2 rect = make_uint2(0u, 0u);
      drawn = project<kPlanes>(p, pa, ca, cb, col, rel, depth, rec, rect, dbg);
      b.rects[gid] = rect;
      if (drawn) b.records[gid] = rec;
    } else if ((b.reuse_order || vis) && valid) {
      // The reused order may list this splat (or its stage was lost): it
      // emits no tile this frame.
      b.rects[gid] = make_uint2(0u, 0u);
    }
    const uint32_t dmask = __ballot_sync(0xffffffffu, drawn);
    if (lane == 0 && dmask) {
      atomicAdd(&b.counters->drawn, __popc(dmask));
      atomicAdd(&b.view_counters[view].drawn, __popc(dmask));
    }
  }

  // Every warp resolves the block's offset on its own (no second block
  // barrier); warp 0 publishes the inclusive prefix.
  const unsigned long long prefix = lookback_resolve(b.status, block, &b.counters->error);
  if (warp == 0 && lane == 0) {
    lookback_publish_inclusive(b.status, block, prefix + block_total);
    if (block == total_blocks - 1) b.counters->visible = (uint32_t)(prefix + block_total);
  }
  uint32_t slot = (uint32_t)prefix;
  for (uint32_t k = 0; k < set.count; ++k) {
    uint32_t warp_prefix = 0, view_total = 0;
#pragma unroll
    for (int w = 0; w < kK1Warps; ++w) {
      const uint32_t c = s_cnt[k][w];
      warp_prefix += (w < (int)warp) ? c : 0u;
      view_total += c;
    }
    const bool vis = (vis_bits >> k) & 1u;
    const uint32_t bal = __ballot_sync(0xffffffffu, vis);
    if (vis && !b.reuse_order) {
      const uint32_t view = set.first_view + k;
      const FrameParams &p = s_params[k];
      const float rx = pa.x - p.cam[0], ry = pa.y - p.cam[1], rz = pa.z - p.cam[2];
      const float depth = p.r2[0] * rx + p.r2[1] * ry + p.r2[2] * rz;
      const uint32_t at = slot + warp_prefix + __popc(bal & lanemask_lt());
      b.vis_keys[at] = ~__float_as_uint(fmaxf(depth, 0.0f));
      b.vis_ids[at] = views[view].splat_base + i;
    }
    slot += view_total;
  }
  __syncthreads();
  if (threadIdx.x == 0 && !s_lost) {  // every thread has passed both waits
    mbar_inval(&st.bar[0]);
    mbar_inval(&st.bar[1]);
  }
  for (uint32_t k = threadIdx.x; k < 4 * 256; k += kK1Threads) {
    uint32_t c = (&s_hist[0][0])[k];
    if (c) atomicAdd(&b.key_hist[k], c);
  }
}

template <int kPlanes, bool kDebug>
void launch_k1_t(const ViewDev *views, const ViewSetDev *sets, uint32_t num_sets,
                 uint32_t total_blocks, const K1Buffers &b, cudaStream_t stream) {
  constexpr size_t kSmem = sizeof(K1Stage<kPlanes>);
  static const bool configured = [] {
    cudaFuncSetAttribute(preprocess_kernel<kPlanes, kDebug>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    return true;
  }();
  (void)configured;
  preprocess_kernel<kPlanes, kDebug>
      <<<total_blocks, kK1Threads, kSmem, stream>>>(views, sets, num_sets, total_blocks, b);
}

template <int kPlanes>
void launch_k1(const ViewDev *views, const ViewSetDev *sets, uint32_t num_sets,
               uint32_t total_blocks, const K1Buffers &b, bool debug, cudaStream_t stream) {
  if (total_blocks == 0) return;
  if (debug)
    launch_k1_t<kPlanes, true>(views, sets, num_sets, total_blocks, b, stream);
  else
    launch_k1_t<kPlanes, false>(views, sets, num_sets, total_blocks, b, stream);
}

}  // namespace

uint32_t preprocess_blocks(uint32_t splats) { return (splats + kK1Threads - 1) / kK1Threads; }

void launch_preprocess(const ViewDev *views, const ViewSetDev *sets, uint32_t num_sets,
                       uint32_t total_blocks, uint32_t max_planes, const K1Buffers &b, bool debug,
                       cudaStream_t stream) {
  if (max_planes <= 1) launch_k1<1>(views, sets, num_sets, total_blocks, b, debug, stream);
  else if (max_planes <= 3) launch_k1<3>(views, sets, num_sets, total_blocks, b, debug, stream);
  else if (max_planes <= 7) launch_k1<7>(views, sets, num_sets, total_blocks, b, debug, stream);
  else if (max_planes <= 12) launch_k1<12>(views, sets, num_sets, total_blocks, b, debug, stream);
  else launch_k1<19>(views, sets, num_sets, total_blocks, b, debug, stream);
}

}  // namespace gsr
