// Scene ingestion from PLY files (crates/gsplat-io-ply/src/lib.rs:178-288,
// 843-907, 76-113, then the renderer's load-time precompute,
// crates/gsplat-render-wgpu/src/lib.rs:499-527).
//
// A binary body is decoded on the device. Host threads read the file in
// chunks into pinned memory and, per vertex, compute the scalars that need
// the C library's exp/log (alpha, extent scale, axis scales; splat_scalars,
// the same code the host path runs), so that every plane equals the host
// path's bit for bit; each chunk and its scalars are copied to the device
// while the next chunk is read, and one thread per vertex decodes its record
// (any PLY scalar type, either byte order), checks every value is finite,
// converts RDF -> RUF (y and the rotation's x, z negated; rest coefficients
// sign-flipped), builds the world covariance from the normalised quaternion
// and writes the scene planes. Built with --fmad=false: the covariance is
// the host's f32 expression sequence, rounded after every operation.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fcntl.h>
#include <thread>
#include <unistd.h>

#include "cuda_check.h"
#include "pipeline.h"
#include "ply.h"

namespace gsr {
namespace {

constexpr uint64_t kChunkBytes = 32ull << 20;  // file bytes per chunk
constexpr uint32_t kMaxRest = 72;              // rest coefficients of SH degree 4

struct DecodeArgs {
  const unsigned char *body;  // the chunk's records
  const float *scalars;       // per record: alpha, extent scale, sx, sy, sz
  uint64_t first;             // scene index of the chunk's first vertex
  uint64_t n;                 // scene size (plane length)
  uint32_t count, stride;
  uint32_t big_endian, rot_xyzw, per_channel, planes, rest_count;
  PlyField pos[3], rot[4], dc[3];
  PlyField rest[kMaxRest];
  float flip[15];
  float4 *pos_alpha, *cov_a, *cov_b, *color;
  uint32_t *error;
};

__device__ float read_field(const unsigned char *rec, PlyField f, bool big) {
  const unsigned char *p = rec + f.offset;
  uint32_t n = 4;
  switch (f.type) {
    case PlyType::I8: case PlyType::U8: n = 1; break;
    case PlyType::I16: case PlyType::U16: n = 2; break;
    case PlyType::F64: n = 8; break;
    default: break;
  }
  unsigned long long bits = 0;
  for (uint32_t k = 0; k < n; ++k)
    bits |= (unsigned long long)p[big ? n - 1 - k : k] << (8 * k);
  switch (f.type) {
    case PlyType::I8: return (float)(int8_t)bits;
    case PlyType::U8: return (float)(uint8_t)bits;
    case PlyType::I16: return (float)(int16_t)bits;
    case PlyType::U16: return (float)(uint16_t)bits;
    case PlyType::I32: return (float)(int32_t)bits;
    case PlyType::U32: return (float)(uint32_t)bits;
    case PlyType::F64: return (float)__longlong_as_double((long long)bits);
    default: return __uint_as_float((uint32_t)bits);
  }
}

// lib.rs:1390-1417, as gsr_host.cpp states them.
__device__ void quat_normalize_d(const float q[4], float out[4]) {
  float norm2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (norm2 <= 0.0f) {
    out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; out[3] = 1.0f;
    return;
  }
  float inv = 1.0f / sqrtf(norm2);
  out[0] = q[0] * inv; out[1] = q[1] * inv; out[2] = q[2] * inv; out[3] = q[3] * inv;
}

__device__ void quat_to_mat3_d(const float qin[4], float m[9]) {
  float q[4];
  quat_normalize_d(qin, q);
  float x = q[0], y = q[1], z = q[2], w = q[3];
  float xx = x * x, yy = y * y, zz = z * z;
  float xy = x * y, xz = x * z, yz = y * z;
  float wx = w * x, wy = w * y, wz = w * z;
  m[0] = 1.0f - 2.0f * (yy + zz); m[1] = 2.0f * (xy - wz);        m[2] = 2.0f * (xz + wy);
  m[3] = 2.0f * (xy + wz);        m[4] = 1.0f - 2.0f * (xx + zz); m[5] = 2.0f * (yz - wx);
  m[6] = 2.0f * (xz - wy);        m[7] = 2.0f * (yz + wx);        m[8] = 1.0f - 2.0f * (xx + yy);
}

__device__ void mat3_mul_d(const float a[9], const float b[9], float out[9]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out[3 * r + c] = a[3 * r + 0] * b[0 + c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}

__global__ void __launch_bounds__(256) decode_kernel(DecodeArgs a) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.count) return;
  const unsigned char *rec = a.body + (uint64_t)j * a.stride;
  const uint64_t i = a.first + j;
  const bool big = a.big_endian != 0;
  bool bad = false;
  auto get = [&](PlyField f) {
    const float v = read_field(rec, f, big);
    bad |= !isfinite(v);
    return v;
  };
  const float x = get(a.pos[0]), y = get(a.pos[1]), z = get(a.pos[2]);
  const float r[4] = {get(a.rot[0]), get(a.rot[1]), get(a.rot[2]), get(a.rot[3])};
  // rot_0..3 as wxyz (or xyzw), stored xyzw; RDF -> RUF negates x and z.
  float q[4];
  if (a.rot_xyzw) {
    q[0] = r[0]; q[1] = r[1]; q[2] = r[2]; q[3] = r[3];
  } else {
    q[0] = r[1]; q[1] = r[2]; q[2] = r[3]; q[3] = r[0];
  }
  q[0] = -q[0];
  q[2] = -q[2];
  const float *sc = a.scalars + 5 * (uint64_t)j;
  const float sx = sc[2], sy = sc[3], sz = sc[4];
  float obj[9] = {sx * sx, 0.0f, 0.0f, 0.0f, sy * sy, 0.0f, 0.0f, 0.0f, sz * sz};
  float qn[4], rot[9], rt[9], tmp[9], w[9];
  quat_normalize_d(q, qn);
  quat_to_mat3_d(qn, rot);
  mat3_mul_d(rot, obj, tmp);
  for (int rr = 0; rr < 3; ++rr)
    for (int c = 0; c < 3; ++c) rt[3 * rr + c] = rot[3 * c + rr];
  mat3_mul_d(tmp, rt, w);
  a.pos_alpha[i] = make_float4(x, -y, z, sc[0]);
  a.cov_a[i] = make_float4(w[0], w[1], w[2], w[4]);
  a.cov_b[i] = make_float4(w[5], w[8], sc[1], 0.0f);
  // Colour planes: float 3c + ch is coefficient c (0 = DC) of channel ch;
  // rest coefficient k of channel ch is property ch * per_channel + k.
  auto coeff = [&](uint32_t f) {
    if (f < 3) return get(a.dc[f]);
    const uint32_t k = f / 3 - 1, ch = f % 3;
    if (k >= a.per_channel || a.rest_count == 0) return 0.0f;
    const float v = get(a.rest[ch * a.per_channel + k]);
    return v * (k < 15 ? a.flip[k] : 1.0f);
  };
  for (uint32_t pl = 0; pl < a.planes; ++pl)
    a.color[(uint64_t)pl * a.n + i] =
        make_float4(coeff(4 * pl), coeff(4 * pl + 1), coeff(4 * pl + 2), coeff(4 * pl + 3));
  if (bad) atomicOr(a.error, 1u);
}

// Pinned host memory, released after the stream it was used on is idle.
struct PinnedBlock {
  void *p = nullptr;
  cudaStream_t stream = nullptr;
  PinnedBlock(uint64_t bytes, cudaStream_t s) : stream(s) {
    GSR_CUDA(cudaMallocHost(&p, std::max<uint64_t>(bytes, 16)));
  }
  ~PinnedBlock() {
    cudaStreamSynchronize(stream);
    cudaFreeHost(p);
  }
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
};

struct FileHandle {
  int fd = -1;
  ~FileHandle() {
    if (fd >= 0) ::close(fd);
  }
};

// Reads [offset, offset + bytes) of the file with `threads` parallel preads.
void read_range(int fd, unsigned char *dst, uint64_t offset, uint64_t bytes, unsigned threads) {
  std::vector<std::thread> pool;
  std::vector<int> ok(threads, 1);
  const uint64_t part = (bytes + threads - 1) / threads;
  for (unsigned t = 0; t < threads; ++t) {
    const uint64_t b = t * part, e = std::min(bytes, b + part);
    if (b >= e) break;
    pool.emplace_back([&, t, b, e] {
      uint64_t done = b;
      while (done < e) {
        const ssize_t r = ::pread(fd, dst + done, e - done, (off_t)(offset + done));
        if (r <= 0) {
          ok[t] = 0;
          return;
        }
        done += (uint64_t)r;
      }
    });
  }
  for (auto &th : pool) th.join();
  for (int o : ok)
    if (!o) throw Error(Code::NotFound, "I/O error while reading PLY");
}

std::unique_ptr<DeviceScene> load_binary(const std::string &path, const PlyBinaryLayout &L,
                                         cudaStream_t stream) {
  const uint64_t n = L.vertices;
  if (L.rest.size() > kMaxRest) throw Error(Code::Unsupported, "too many SH rest coefficients");
  auto sc = alloc_scene(n, L.sh_degree);
  sc->positions.resize(3 * n);
  if (n == 0) return sc;
  FileHandle file;
  file.fd = ::open(path.c_str(), O_RDONLY);
  if (file.fd < 0) throw Error(Code::NotFound, "I/O error while reading PLY");

  const uint64_t stride = L.stride;
  const uint64_t per_chunk = std::max<uint64_t>(1, kChunkBytes / stride);
  const unsigned threads = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  DeviceBuffer dev_body, dev_scalars, dev_error;
  dev_body.reset(2 * per_chunk * stride);
  dev_scalars.reset(2 * per_chunk * 5 * sizeof(float));
  dev_error.reset(sizeof(uint32_t));
  GSR_CUDA(cudaMemsetAsync(dev_error.get(), 0, sizeof(uint32_t), stream));
  PinnedBlock host_body(2 * per_chunk * stride, stream);
  PinnedBlock host_scalars(2 * per_chunk * 5 * sizeof(float), stream);
  PinnedBlock host_error(sizeof(uint32_t), stream);
  cudaEvent_t done[2];
  for (auto &e : done) GSR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  struct Events {
    cudaEvent_t *e;
    ~Events() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } events{done};

  DecodeArgs a{};
  a.n = n;
  a.stride = (uint32_t)stride;
  a.big_endian = L.big_endian;
  a.rot_xyzw = L.rot_xyzw;
  a.per_channel = L.has_rest ? (L.sh_degree + 1) * (L.sh_degree + 1) - 1 : 0;
  a.planes = sc->dev.planes;
  a.rest_count = (uint32_t)L.rest.size();
  for (int k = 0; k < 3; ++k) {
    a.pos[k] = L.pos[k];
    a.dc[k] = L.dc[k];
  }
  for (int k = 0; k < 4; ++k) a.rot[k] = L.rot[k];
  for (size_t k = 0; k < L.rest.size(); ++k) a.rest[k] = L.rest[k];
  std::memcpy(a.flip, ply_sh_flip(), sizeof(a.flip));
  a.pos_alpha = const_cast<float4 *>(sc->dev.pos_alpha);
  a.cov_a = const_cast<float4 *>(sc->dev.cov_a);
  a.cov_b = const_cast<float4 *>(sc->dev.cov_b);
  a.color = const_cast<float4 *>(sc->dev.color);
  a.error = dev_error.as<uint32_t>();

  const uint64_t chunks = (n + per_chunk - 1) / per_chunk;
  for (uint64_t c = 0; c < chunks; ++c) {
    const int slot = (int)(c & 1);
    if (c >= 2) GSR_CUDA(cudaEventSynchronize(done[slot]));
    const uint64_t first = c * per_chunk;
    const uint64_t count = std::min(per_chunk, n - first);
    unsigned char *body = host_body.as<unsigned char>() + slot * per_chunk * stride;
    float *scal = host_scalars.as<float>() + slot * per_chunk * 5;
    read_range(file.fd, body, L.body_offset + first * stride, count * stride, threads);
    // Host part of the decode: positions (for automatic framing) and the
    // scalars that need exp/log, with the finite-value rules of the loader.
    std::vector<std::thread> pool;
    std::vector<int> valid(threads, 1);
    const uint64_t part = (count + threads - 1) / threads;
    for (unsigned t = 0; t < threads; ++t) {
      const uint64_t b = t * part, e = std::min(count, b + part);
      if (b >= e) break;
      pool.emplace_back([&, t, b, e] {
        for (uint64_t j = b; j < e; ++j) {
          const unsigned char *rec = body + j * stride;
          float p[3], ls[3];
          bool ok = true;
          for (int k = 0; k < 3; ++k) {
            p[k] = ply_read_scalar(rec + L.pos[k].offset, L.pos[k].type, L.big_endian);
            ls[k] = ply_read_scalar(rec + L.scale[k].offset, L.scale[k].type, L.big_endian);
            ok = ok && ply_value_finite(p[k]) && ply_value_finite(ls[k]);
          }
          float o = ply_read_scalar(rec + L.opacity.offset, L.opacity.type, L.big_endian);
          if (std::isnan(o)) ok = false;
          if (!ok) {
            valid[t] = 0;
            return;
          }
          o = ply_opacity_logit(o);
          float *pos = &sc->positions[3 * (first + j)];
          pos[0] = p[0];
          pos[1] = -p[1];
          pos[2] = p[2];
          splat_scalars(o, ls, scal + 5 * j);
        }
      });
    }
    for (auto &th : pool) th.join();
    for (int v : valid)
      if (!v) throw Error(Code::ParseFailed, "failed to parse numeric value");
    GSR_CUDA(cudaMemcpyAsync(dev_body.as<unsigned char>() + slot * per_chunk * stride, body,
                             count * stride, cudaMemcpyHostToDevice, stream));
    GSR_CUDA(cudaMemcpyAsync(dev_scalars.as<float>() + slot * per_chunk * 5, scal,
                             count * 5 * sizeof(float), cudaMemcpyHostToDevice, stream));
    a.body = dev_body.as<unsigned char>() + slot * per_chunk * stride;
    a.scalars = dev_scalars.as<float>() + slot * per_chunk * 5;
    a.first = first;
    a.count = (uint32_t)count;
    decode_kernel<<<(uint32_t)((count + 255) / 256), 256, 0, stream>>>(a);
    GSR_CUDA(cudaGetLastError());
    GSR_CUDA(cudaEventRecord(done[slot], stream));
  }
  GSR_CUDA(cudaMemcpyAsync(host_error.p, dev_error.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           stream));
  GSR_CUDA(cudaStreamSynchronize(stream));
  if (*host_error.as<uint32_t>()) throw Error(Code::ParseFailed, "failed to parse numeric value");
  return sc;
}

}  // namespace

std::unique_ptr<DeviceScene> load_scene_file(const std::string &path, cudaStream_t stream,
                                             const std::function<void(uint64_t)> &admit) {
  PlyBinaryLayout layout;
  if (!inspect_binary_ply(path, layout)) {
    HostScene s = load_ply(path);
    if (admit) admit(scene_device_bytes(s));
    return upload_scene(s, stream);
  }
  if (admit) admit(scene_device_bytes(layout.vertices, layout.sh_degree));
  return load_binary(path, layout, stream);
}

}  // namespace gsr
