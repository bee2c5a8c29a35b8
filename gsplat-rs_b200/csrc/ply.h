// Binary PLY bodies as the reference loader reads them
// (crates/gsplat-io-ply/src/lib.rs:843-907), described for a decode that
// runs on the device.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gsr {

enum class PlyType : uint8_t { I8, U8, I16, U16, I32, U32, F32, F64 };

// One vertex property: byte offset within the record and scalar type.
struct PlyField {
  uint32_t offset;
  PlyType type;
};

struct PlyBinaryLayout {
  bool big_endian = false;
  uint64_t vertices = 0;
  uint64_t stride = 0;       // bytes per vertex record
  uint64_t body_offset = 0;  // first body byte in the file
  uint32_t sh_degree = 0;    // inferred from the f_rest_* properties
  bool has_rest = false;
  bool rot_xyzw = false;     // GSPLAT_ROT_LAYOUT=xyzw (lib.rs:63-74); else rot_0 is w
  PlyField pos[3], opacity, scale[3], rot[4], dc[3];
  std::vector<PlyField> rest;  // rest coefficient k of the channel-major list -> property
};

// The checks load_ply makes before it decodes the body (file access, limits,
// header, required fields, SH layout, body length, decoded size), with the
// same error codes and messages, reading only the header. Fills `out` and
// returns true for a binary body; returns false for an ASCII one.
bool inspect_binary_ply(const std::string &path, PlyBinaryLayout &out);

// Value rules of the body decode (lib.rs:843-907, 993-1004): every field must
// be finite, except that an infinite opacity logit becomes +-16.
bool ply_value_finite(float v);
float ply_read_scalar(const unsigned char *p, PlyType t, bool big);  // one property value as f32
float ply_opacity_logit(float v);  // throws PARSE_FAILED for NaN
// Sign flips of rest coefficients 0..14 for the RDF -> RUF reflection (lib.rs:54-56).
const float *ply_sh_flip();

}  // namespace gsr
