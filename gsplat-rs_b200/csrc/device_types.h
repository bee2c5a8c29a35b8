// Plain data structures shared by the kernels and the host orchestration.
#pragma once

#include <cstdint>
#include <vector_types.h>

#include "gsr_host.h"

namespace gsr {

// Scene resident in HBM, structure of arrays of float4 planes (16-byte
// aligned, one 128-bit load per plane and splat):
//   pos_alpha[i] = (x, y, z, alpha)         alpha = clamp(sigmoid(opacity))
//   cov_a[i]     = (xx, xy, xz, yy)         world covariance
//   cov_b[i]     = (yz, zz, extent_scale, 0)
//   color[p*n+i] = floats 4p..4p+3 of (DC rgb, rest coefficient 1 rgb, ...)
//
// A packed scene (packed_atlas.rs: the 20-byte hot record, an i8 SH sidecar)
// has no planes; the preprocess kernel decodes it into the same per-block
// values instead:
//   hot[5i .. 5i+4]  = u16 x, y | u16 z, u8 opacity | 3 x u10 log scale |
//                      smallest-three quaternion | RGB10 baked colour
//   sidecar[48i ..]  = 45 i8 rest coefficients (channel-major, 15 per channel)
//   packed           = bounds min (3), span (3), log-scale min, extent, SH
//                      scales (3), pad, then the 1,024 axis variances
//                      exp(2 log_scale(u)) and the 256 extent scales
// Both arrays are padded to whole 256-splat slices.
struct SceneDev {
  const float4 *pos_alpha;
  const float4 *cov_a;
  const float4 *cov_b;
  const float4 *color;
  uint32_t n;
  uint32_t planes;
  const uint32_t *hot;     // packed scenes only (else null)
  const int8_t *sidecar;   // packed scenes of SH degree >= 1
  const float *packed;     // header and tables of a packed scene
};
constexpr uint32_t kPackedHeaderFloats = 12;
constexpr uint32_t kPackedVarLut = 1024;
constexpr uint32_t kPackedExtLut = 256;
constexpr uint32_t kPackedFloats = kPackedHeaderFloats + kPackedVarLut + kPackedExtLut;

// Pixel-space raster record of a drawn splat (48 bytes):
//   a = (cx, cy, ax, ay)  centre in pixel-centre coordinates, first row of
//                         the inverse axis matrix (local x = ax*dx + ay*dy)
//   b = (bx, by, s, alpha) second row, quad extent scale, opacity
//   c = (r, g, b, log2(alpha))  colour before alpha (premultiplied: r*alpha)
struct Record {
  float4 a, b, c;
};

// Same layout as GsplatProjectedSplat.
struct ProjectedDev {
  float center_ndc[2];
  float axis_u[2];
  float axis_v[2];
  float color[4];
  float extent_scale;
  float depth;
  uint32_t flags;
  uint16_t tile_x0, tile_y0, tile_x1, tile_y1;
  uint32_t reserved;
};
static_assert(sizeof(ProjectedDev) == 64, "projected splat layout");

// Error bits reported through FrameCounters::error.
enum : uint32_t {
  kErrLookbackTimeout = 1u,  // a decoupled look-back wait hit its iteration limit
  kErrSortTooLarge = 2u,
  kErrStageTimeout = 4u,     // a bulk-copy (TMA) completion wait hit its iteration limit
};

// Per-frame device counters; zeroed before each frame.
struct FrameCounters {
  uint32_t k1_ticket;
  uint32_t emit_ticket;
  uint32_t visible;
  uint32_t drawn;
  uint32_t error;
  uint32_t overflow;
  uint32_t pairs;  // pairs written: min(keys, capacity)
  uint32_t raster_ticket;  // persistent raster tile queue
  unsigned long long keys;  // pairs emitted (may exceed the capacity)
  uint32_t sort_tickets[16];
};

// One view of a frame batch (a plain frame is a batch of one view). Splats
// of all views share one index space: view v's splat i is gid = splat_base+i.
struct ViewDev {
  FrameParams p;       // per-view uniforms (camera, image size, tile grid)
  SceneDev sc;         // the view's scene
  uint32_t splat_base; // first gid of the view
  uint32_t set;        // the view set (views of one scene) the view belongs to
  uint32_t tile_base;  // first global tile id of the view
  uint32_t pad;
  unsigned long long image_base;  // first pixel of the view's image
};

// Consecutive views of one scene that the preprocess kernel handles together
// (one read of the scene planes for all of them).
struct ViewSetDev {
  uint32_t first_view;  // index into the view table
  uint32_t count;       // 1..kMaxSetViews
  uint32_t block_base;  // first preprocess block of the set
  uint32_t pad;
};
constexpr uint32_t kMaxSetViews = 16;

// Per-view counters of a batch (zeroed per batch).
struct ViewCounters {
  uint32_t visible;  // depth-visible splats
  uint32_t drawn;    // splats with a raster record
  uint32_t pairs;    // tile pairs the view emits (its splats' exact row-span counts)
  uint32_t pad;
};

// Plan of one radix sort, computed on the device from the global histogram.
struct SortPlan {
  uint32_t n;
  uint32_t passes;
  uint32_t final_buffer;  // 0: the input buffers, 1: the alternate buffers
  uint32_t pad;
  uint32_t skip[8];
  uint32_t src[8];
  uint32_t digit_offset[8][256];
};

}  // namespace gsr
