// PLY scene loader with the behaviour of crates/gsplat-io-ply/src/lib.rs:
// ascii / binary_little_endian / binary_big_endian 1.0, the same resource
// limits, field inference, error codes and RDF -> RUF conversion.

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "gsr_host.h"
#include "ply.h"

namespace gsr {
namespace {

// lib.rs:28-47 (PlyLoadLimits::default)
constexpr uint64_t kMiB = 1024ull * 1024ull;
constexpr uint64_t kGiB = 1024ull * kMiB;
constexpr uint64_t kMaxInputBytes = kGiB;
constexpr uint64_t kMaxHeaderBytes = kMiB;
constexpr uint64_t kMaxVertices = 5000000;
constexpr uint64_t kMaxVertexProperties = 128;
constexpr uint64_t kMaxSceneBytes = kGiB;
// lib.rs:18: infinite opacity logits are clamped to +-16.
constexpr float kOpacityLogitLimit = 16.0f;
// lib.rs:54-56: SH sign flips for the RDF -> RUF y reflection, per rest coefficient.
constexpr float kShFlip[15] = {-1.0f, 1.0f, 1.0f,  -1.0f, -1.0f, 1.0f, 1.0f, 1.0f,
                               -1.0f, -1.0f, -1.0f, 1.0f, 1.0f,  1.0f, 1.0f};

enum class Fmt { Ascii, BinLE, BinBE };
enum class Ty { I8, U8, I16, U16, I32, U32, F32, F64 };

struct Prop {
  std::string name;
  Ty ty;
};

struct Header {
  Fmt format;
  uint64_t vertex_count;
  std::vector<Prop> props;
};

[[noreturn]] void fail(Code c, const std::string &what) { throw Error(c, what); }
void limit(const char *resource, uint64_t requested, uint64_t lim) {
  // lib.rs:306-321 (ensure_limit) -> ResourceLimit -> Unsupported
  if (requested > lim)
    fail(Code::Unsupported, std::string("PLY resource limit exceeded for ") + resource +
                                ": requested " + std::to_string(requested) + ", limit " +
                                std::to_string(lim));
}

size_t ty_size(Ty t) {
  switch (t) {
    case Ty::I8: case Ty::U8: return 1;
    case Ty::I16: case Ty::U16: return 2;
    case Ty::I32: case Ty::U32: case Ty::F32: return 4;
    case Ty::F64: return 8;
  }
  return 0;
}

bool parse_ty(const std::string &s, Ty &t) {
  // lib.rs:634-646
  if (s == "char" || s == "int8") t = Ty::I8;
  else if (s == "uchar" || s == "uint8") t = Ty::U8;
  else if (s == "short" || s == "int16") t = Ty::I16;
  else if (s == "ushort" || s == "uint16") t = Ty::U16;
  else if (s == "int" || s == "int32") t = Ty::I32;
  else if (s == "uint" || s == "uint32") t = Ty::U32;
  else if (s == "float" || s == "float32") t = Ty::F32;
  else if (s == "double" || s == "float64") t = Ty::F64;
  else return false;
  return true;
}

std::string trim(const std::string &s) {
  size_t b = s.find_first_not_of(" \t\r\n\f\v");
  if (b == std::string::npos) return "";
  size_t e = s.find_last_not_of(" \t\r\n\f\v");
  return s.substr(b, e - b + 1);
}

std::vector<std::string> split_ws(const std::string &s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string tok;
  while (is >> tok) out.push_back(tok);
  return out;
}

bool valid_utf8(const unsigned char *p, size_t n) {
  size_t i = 0;
  while (i < n) {
    unsigned char c = p[i];
    size_t len = c < 0x80 ? 1 : (c >> 5) == 6 ? 2 : (c >> 4) == 14 ? 3 : (c >> 3) == 30 ? 4 : 0;
    if (len == 0 || i + len > n) return false;
    for (size_t k = 1; k < len; ++k)
      if ((p[i + k] & 0xC0) != 0x80) return false;
    i += len;
  }
  return true;
}

// lib.rs:539-605 (parse_header_text)
Header parse_header_text(const std::string &text) {
  std::istringstream is(text);
  std::string line;
  if (!std::getline(is, line) || trim(line) != "ply") fail(Code::ParseFailed, "malformed PLY header");
  bool have_format = false, have_count = false, saw_end = false, in_vertex = false;
  Header h{Fmt::Ascii, 0, {}};
  while (std::getline(is, line)) {
    std::string t = trim(line);
    if (t.empty() || t.rfind("comment", 0) == 0) continue;
    if (t == "end_header") {
      saw_end = true;
      break;
    }
    auto parts = split_ws(t);
    if (parts[0] == "format") {
      have_format = false;
      if (parts.size() >= 3 && parts[2] == "1.0") {
        if (parts[1] == "ascii") { h.format = Fmt::Ascii; have_format = true; }
        else if (parts[1] == "binary_little_endian") { h.format = Fmt::BinLE; have_format = true; }
        else if (parts[1] == "binary_big_endian") { h.format = Fmt::BinBE; have_format = true; }
      }
    } else if (parts[0] == "element") {
      in_vertex = parts.size() >= 2 && parts[1] == "vertex";
      if (in_vertex) {
        if (parts.size() < 3) fail(Code::ParseFailed, "malformed PLY header");
        const std::string &c = parts[2];
        if (c.empty() || c.find_first_not_of("0123456789") != std::string::npos ||
            c.size() > 19)
          fail(Code::ParseFailed, "malformed PLY header");
        uint64_t count = std::strtoull(c.c_str(), nullptr, 10);
        limit("vertices", count, kMaxVertices);
        h.vertex_count = count;
        have_count = true;
      }
    } else if (parts[0] == "property" && in_vertex) {
      if (parts.size() < 2) fail(Code::ParseFailed, "malformed PLY header");
      if (parts[1] == "list")
        fail(Code::Unsupported,
             "unsupported PLY format; supported: ascii 1.0, binary_little_endian 1.0, "
             "binary_big_endian 1.0");
      if (parts.size() < 3) fail(Code::ParseFailed, "malformed PLY header");
      Ty ty;
      if (!parse_ty(parts[1], ty)) fail(Code::ParseFailed, "malformed PLY header");
      limit("vertex properties", h.props.size() + 1, kMaxVertexProperties);
      h.props.push_back({parts[2], ty});
    }
  }
  if (!have_format)
    fail(Code::Unsupported,
         "unsupported PLY format; supported: ascii 1.0, binary_little_endian 1.0, "
         "binary_big_endian 1.0");
  if (!saw_end || !have_count) fail(Code::ParseFailed, "malformed PLY header");
  return h;
}

// lib.rs:486-537 (split_header_body)
Header split_header(const std::vector<unsigned char> &in, size_t &body_off) {
  size_t cursor = 0;
  bool found = false;
  size_t header_end = 0;
  while (cursor < in.size()) {
    size_t scan_end = std::min<size_t>(in.size(), kMaxHeaderBytes + 1);
    if (cursor >= scan_end) limit("header bytes", cursor + 1, kMaxHeaderBytes);
    size_t line_end = cursor;
    while (line_end < scan_end && in[line_end] != '\n') ++line_end;
    size_t next = line_end < in.size() ? line_end + 1 : line_end;
    limit("header bytes", next, kMaxHeaderBytes);
    if (!valid_utf8(&in[cursor], line_end - cursor)) fail(Code::ParseFailed, "malformed PLY header");
    std::string line(reinterpret_cast<const char *>(&in[cursor]), line_end - cursor);
    while (!line.empty() && line.back() == '\r') line.pop_back();
    if (trim(line) == "end_header") {
      header_end = next;
      found = true;
      break;
    }
    cursor = line_end + 1;
  }
  if (!found) fail(Code::ParseFailed, "malformed PLY header");
  body_off = header_end;
  return parse_header_text(std::string(reinterpret_cast<const char *>(in.data()), header_end));
}

// lib.rs:662-730 (infer_sh_rest_layout, infer_sh_degree)
uint32_t infer_sh(const Header &h, std::vector<size_t> &rest_props) {
  std::vector<std::pair<uint64_t, size_t>> pairs;
  for (size_t k = 0; k < h.props.size(); ++k) {
    const std::string &n = h.props[k].name;
    if (n.rfind("f_rest_", 0) != 0) continue;
    std::string digits = n.substr(7);
    if (digits.empty() || digits.find_first_not_of("0123456789") != std::string::npos ||
        digits.size() > 18)
      continue;
    pairs.push_back({std::strtoull(digits.c_str(), nullptr, 10), k});
  }
  rest_props.clear();
  if (pairs.empty()) return 0;
  std::stable_sort(pairs.begin(), pairs.end(),
                   [](const auto &a, const auto &b) { return a.first < b.first; });
  if (pairs.size() != pairs.back().first + 1) return 0;
  for (size_t k = 0; k < pairs.size(); ++k)
    if (pairs[k].first != k) return 0;
  uint64_t total = pairs.size();
  if (total % 3 != 0) return 0;
  uint64_t coeff_total = total / 3 + 1;
  uint64_t root = (uint64_t)std::sqrt((double)coeff_total);
  while (root * root > coeff_total) --root;
  while ((root + 1) * (root + 1) <= coeff_total) ++root;
  if (root * root != coeff_total) return 0;
  uint64_t degree = root - 1;
  if (degree == 0 || degree > 4) return 0;
  for (auto &p : pairs) rest_props.push_back(p.second);
  return (uint32_t)degree;
}

// Rust's str::parse::<f32>: decimal only, whole token, correctly rounded.
bool parse_f32(const std::string &tok, float &out) {
  if (tok.empty()) return false;
  const char *s = tok.c_str();
  const char *d = s + ((*s == '+' || *s == '-') ? 1 : 0);
  if ((d[0] == '0') && (d[1] == 'x' || d[1] == 'X')) return false;
  char *end = nullptr;
  errno = 0;
  float v = std::strtof(s, &end);
  if (end == s || *end != '\0') return false;
  out = v;
  return true;
}

float read_scalar(const unsigned char *p, Ty ty, bool big) {
  unsigned char b[8];
  size_t n = ty_size(ty);
  for (size_t k = 0; k < n; ++k) b[k] = big ? p[n - 1 - k] : p[k];
  switch (ty) {
    case Ty::I8: return (float)(int8_t)b[0];
    case Ty::U8: return (float)b[0];
    case Ty::I16: { int16_t v; std::memcpy(&v, b, 2); return (float)v; }
    case Ty::U16: { uint16_t v; std::memcpy(&v, b, 2); return (float)v; }
    case Ty::I32: { int32_t v; std::memcpy(&v, b, 4); return (float)v; }
    case Ty::U32: { uint32_t v; std::memcpy(&v, b, 4); return (float)v; }
    case Ty::F32: { float v; std::memcpy(&v, b, 4); return v; }
    case Ty::F64: { double v; std::memcpy(&v, b, 8); return (float)v; }
  }
  return 0.0f;
}

// lib.rs:993-1004 (normalize_opacity_logit)
float opacity_logit(float v) {
  if (std::isfinite(v)) return v;
  if (std::isinf(v)) return v > 0 ? kOpacityLogitLimit : -kOpacityLogitLimit;
  fail(Code::ParseFailed, "failed to parse numeric value");
}

float finite_or_fail(float v) {
  if (!std::isfinite(v)) fail(Code::ParseFailed, "failed to parse numeric value");
  return v;
}

bool rot_layout_xyzw() {
  // lib.rs:63-74: GSPLAT_ROT_LAYOUT=xyzw keeps rot_0..3 as xyzw.
  const char *e = std::getenv("GSPLAT_ROT_LAYOUT");
  return e && (std::strcmp(e, "xyzw") == 0 || std::strcmp(e, "XYZW") == 0);
}

// What the body decode needs from a parsed header: the property index by
// name (a later duplicate name overrides the earlier one, as a HashMap
// insert does), the SH layout and the record layout of a binary body.
struct Analysis {
  std::map<std::string, size_t> idx;
  std::vector<size_t> rest_props;
  uint32_t degree = 0;
  bool has_rest = false;
  uint64_t rest_stride = 0;
  std::vector<size_t> offsets;
  size_t stride = 0;
};

Analysis analyze(const Header &h) {
  Analysis a;
  for (size_t k = 0; k < h.props.size(); ++k) a.idx.emplace(h.props[k].name, k);
  static const char *kRequired[14] = {"x", "y", "z", "opacity", "scale_0", "scale_1", "scale_2",
                                      "rot_0", "rot_1", "rot_2", "rot_3", "f_dc_0", "f_dc_1",
                                      "f_dc_2"};
  for (const char *r : kRequired)
    if (!a.idx.count(r)) fail(Code::ParseFailed, std::string("missing required field `") + r + "`");
  for (size_t k = 0; k < h.props.size(); ++k) a.idx[h.props[k].name] = k;
  a.degree = infer_sh(h, a.rest_props);
  a.has_rest = a.degree > 0 && !a.rest_props.empty();
  a.rest_stride = a.has_rest ? sh_rest_stride(a.degree) : 0;
  a.offsets.resize(h.props.size());
  for (size_t k = 0; k < h.props.size(); ++k) {
    a.offsets[k] = a.stride;
    a.stride += ty_size(h.props[k].ty);
  }
  return a;
}

// lib.rs:376-404 (validate_body_before_allocation), binary bodies.
void check_binary_body(uint64_t n, size_t stride, uint64_t body_len) {
  if (stride != 0 && n > (uint64_t)-1 / stride)
    fail(Code::Unsupported, "PLY resource size overflow while computing binary body bytes");
  if (body_len < n * stride) fail(Code::ParseFailed, "vertex rows do not match declared vertex count");
}

// lib.rs:323-374 (allocate_scene): decoded bytes limit.
void check_scene_bytes(uint64_t n, uint64_t rest_stride) {
  uint64_t scene_bytes = n * (12 + 4 + 12 + 12 + 16) + n * rest_stride * 4;
  limit("decoded scene bytes", scene_bytes, kMaxSceneBytes);
}

PlyType ply_type(Ty t) {
  switch (t) {
    case Ty::I8: return PlyType::I8;
    case Ty::U8: return PlyType::U8;
    case Ty::I16: return PlyType::I16;
    case Ty::U16: return PlyType::U16;
    case Ty::I32: return PlyType::I32;
    case Ty::U32: return PlyType::U32;
    case Ty::F32: return PlyType::F32;
    case Ty::F64: return PlyType::F64;
  }
  return PlyType::F32;
}

}  // namespace

bool ply_value_finite(float v) { return std::isfinite(v); }

float ply_read_scalar(const unsigned char *p, PlyType t, bool big) {
  static const Ty kTy[8] = {Ty::I8, Ty::U8, Ty::I16, Ty::U16, Ty::I32, Ty::U32, Ty::F32, Ty::F64};
  return read_scalar(p, kTy[(int)t], big);
}

float ply_opacity_logit(float v) { return opacity_logit(v); }

const float *ply_sh_flip() { return kShFlip; }

// The checks of load_ply that precede the body decode, on the header alone
// (the file's first bytes and its size).
bool inspect_binary_ply(const std::string &path, PlyBinaryLayout &out) {
  struct stat st;
  if (::stat(path.c_str(), &st) != 0) fail(Code::NotFound, "I/O error while reading PLY");
  limit("input bytes", (uint64_t)st.st_size, kMaxInputBytes);
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(Code::NotFound, "I/O error while reading PLY");
  const uint64_t file_size = (uint64_t)st.st_size;
  std::vector<unsigned char> head((size_t)std::min<uint64_t>(file_size, kMaxHeaderBytes + 2));
  f.read(reinterpret_cast<char *>(head.data()), (std::streamsize)head.size());
  if (f.bad() || (uint64_t)f.gcount() != head.size()) fail(Code::NotFound, "I/O error while reading PLY");
  size_t body_off = 0;
  Header h = split_header(head, body_off);
  Analysis a = analyze(h);
  if (h.format == Fmt::Ascii) return false;
  const uint64_t n = h.vertex_count;
  check_binary_body(n, a.stride, file_size - body_off);
  check_scene_bytes(n, a.rest_stride);
  auto field = [&](const char *name) {
    const size_t k = a.idx.at(name);
    return PlyField{(uint32_t)a.offsets[k], ply_type(h.props[k].ty)};
  };
  out = PlyBinaryLayout{};
  out.big_endian = h.format == Fmt::BinBE;
  out.vertices = n;
  out.stride = a.stride;
  out.body_offset = body_off;
  out.sh_degree = a.degree;
  out.has_rest = a.has_rest;
  out.rot_xyzw = rot_layout_xyzw();
  const char *pos[3] = {"x", "y", "z"}, *scale[3] = {"scale_0", "scale_1", "scale_2"};
  const char *rot[4] = {"rot_0", "rot_1", "rot_2", "rot_3"};
  const char *dc[3] = {"f_dc_0", "f_dc_1", "f_dc_2"};
  for (int k = 0; k < 3; ++k) {
    out.pos[k] = field(pos[k]);
    out.scale[k] = field(scale[k]);
    out.dc[k] = field(dc[k]);
  }
  for (int k = 0; k < 4; ++k) out.rot[k] = field(rot[k]);
  out.opacity = field("opacity");
  if (a.has_rest)
    for (size_t k : a.rest_props) out.rest.push_back({(uint32_t)a.offsets[k], ply_type(h.props[k].ty)});
  return true;
}

// lib.rs:178-181, 199-288 (load_ply, parse_ply_bytes_with_limits)
HostScene load_ply(const std::string &path) {
  struct stat st;
  if (::stat(path.c_str(), &st) != 0) fail(Code::NotFound, "I/O error while reading PLY");
  limit("input bytes", (uint64_t)st.st_size, kMaxInputBytes);
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(Code::NotFound, "I/O error while reading PLY");
  std::vector<unsigned char> in((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  if (f.bad()) fail(Code::NotFound, "I/O error while reading PLY");
  limit("input bytes", in.size(), kMaxInputBytes);

  size_t body_off = 0;
  Header h = split_header(in, body_off);
  Analysis an = analyze(h);
  std::map<std::string, size_t> &idx = an.idx;
  const std::vector<size_t> &rest_props = an.rest_props;
  const uint32_t degree = an.degree;
  const bool has_rest = an.has_rest;
  const uint64_t rest_stride = an.rest_stride;
  const std::vector<size_t> &offsets = an.offsets;
  const size_t stride = an.stride;
  const uint64_t n = h.vertex_count;
  const unsigned char *body = in.data() + body_off;
  const size_t body_len = in.size() - body_off;

  std::vector<std::string> rows;
  if (h.format == Fmt::Ascii) {
    if (!valid_utf8(body, body_len))
      fail(Code::Unsupported,
           "unsupported PLY format; supported: ascii 1.0, binary_little_endian 1.0, "
           "binary_big_endian 1.0");
    std::string text(reinterpret_cast<const char *>(body), body_len);
    std::istringstream is(text);
    std::string line;
    while (rows.size() < n && std::getline(is, line)) {
      std::string t = trim(line);
      if (t.empty() || t.rfind("comment", 0) == 0) continue;
      rows.push_back(t);
    }
    if (rows.size() < n) fail(Code::ParseFailed, "vertex rows do not match declared vertex count");
  } else {
    check_binary_body(n, stride, body_len);
  }
  check_scene_bytes(n, rest_stride);

  HostScene s;
  s.sh_degree = degree;
  s.has_sh_rest = has_rest;
  s.positions.resize(3 * n);
  s.opacity.resize(n);
  s.scale_xyz.resize(3 * n);
  s.rotation_xyzw.resize(4 * n);
  s.color_dc.resize(3 * n);
  if (has_rest) s.sh_rest.resize(n * rest_stride);
  const bool xyzw = rot_layout_xyzw();
  const size_t ix = idx["x"], iy = idx["y"], iz = idx["z"], io = idx["opacity"];
  const size_t is0 = idx["scale_0"], is1 = idx["scale_1"], is2 = idx["scale_2"];
  const size_t ir[4] = {idx["rot_0"], idx["rot_1"], idx["rot_2"], idx["rot_3"]};
  const size_t idc[3] = {idx["f_dc_0"], idx["f_dc_1"], idx["f_dc_2"]};

  auto store = [&](uint64_t i, auto get, auto get_raw) {
    s.positions[3 * i + 0] = get(ix);
    s.positions[3 * i + 1] = get(iy);
    s.positions[3 * i + 2] = get(iz);
    s.opacity[i] = opacity_logit(get_raw(io));
    s.scale_xyz[3 * i + 0] = get(is0);
    s.scale_xyz[3 * i + 1] = get(is1);
    s.scale_xyz[3 * i + 2] = get(is2);
    float r[4] = {get(ir[0]), get(ir[1]), get(ir[2]), get(ir[3])};
    float *q = &s.rotation_xyzw[4 * i];
    if (xyzw) { q[0] = r[0]; q[1] = r[1]; q[2] = r[2]; q[3] = r[3]; }
    else { q[0] = r[1]; q[1] = r[2]; q[2] = r[3]; q[3] = r[0]; }  // wxyz -> xyzw
    for (int c = 0; c < 3; ++c) s.color_dc[3 * i + c] = get(idc[c]);
    if (has_rest)
      for (size_t k = 0; k < rest_props.size(); ++k) s.sh_rest[i * rest_stride + k] = get(rest_props[k]);
  };

  if (h.format == Fmt::Ascii) {
    // lib.rs:732-806 (parse_ascii_body)
    for (uint64_t i = 0; i < n; ++i) {
      auto vals = split_ws(rows[i]);
      if (vals.size() < h.props.size())
        fail(Code::ParseFailed, "vertex row does not match declared property count");
      auto raw = [&](size_t k) {
        if (k >= vals.size()) fail(Code::ParseFailed, "vertex row does not match declared property count");
        float v;
        if (!parse_f32(vals[k], v)) fail(Code::ParseFailed, "failed to parse numeric value");
        return v;
      };
      auto get = [&](size_t k) { return finite_or_fail(raw(k)); };
      store(i, get, raw);
    }
  } else {
    // lib.rs:843-907 (parse_binary_body)
    const bool big = h.format == Fmt::BinBE;
    for (uint64_t i = 0; i < n; ++i) {
      const unsigned char *rec = body + i * stride;
      auto raw = [&](size_t k) { return read_scalar(rec + offsets[k], h.props[k].ty, big); };
      auto get = [&](size_t k) { return finite_or_fail(raw(k)); };
      store(i, get, raw);
    }
  }

  // lib.rs:76-113 (convert_scene_rdf_to_ruf)
  for (uint64_t i = 0; i < n; ++i) {
    s.positions[3 * i + 1] = -s.positions[3 * i + 1];
    s.rotation_xyzw[4 * i + 0] = -s.rotation_xyzw[4 * i + 0];
    s.rotation_xyzw[4 * i + 2] = -s.rotation_xyzw[4 * i + 2];
  }
  if (has_rest) {
    const uint32_t per_channel = (degree + 1) * (degree + 1) - 1;
    for (uint64_t i = 0; i < n; ++i)
      for (int ch = 0; ch < 3; ++ch)
        for (uint32_t k = 0; k < per_channel; ++k) {
          float sign = k < 15 ? kShFlip[k] : 1.0f;
          float &c = s.sh_rest[i * rest_stride + ch * per_channel + k];
          c = c * sign;
        }
  }
  if (scene_validate(s) != Code::Ok) fail(Code::ParseFailed, "parsed scene buffers are inconsistent");
  return s;
}

}  // namespace gsr
