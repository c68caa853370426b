// On-disk scene files: the device records of a built scene (node records, triangle and
// shading records, id map, Morton codes and order, materials, lights) and its build
// settings, so that another process can render the scene without building it again.
// The reference rebuilds its CPU tree in Scene::flush on every run (src/Scene.cpp:204-209).
//
// Layout, in the host's byte order: a 104-byte header (magic "EOSSCN01", a format
// version, the sizes and settings of Header, a checksum of the payload), then the
// payload: node records (128 B each), triangle records and shading records (48 B per
// triangle each), triangle id -> position, sorted Morton codes, sorted triangle ids
// (4 B per triangle each), materials (eos_material), lights (eos_light).
//
// Both directions stream the payload through two pinned chunks of the context, so that
// the file read / write and the checksum of one chunk overlap the copy of the other.
// eos_scene_load checks magic, version and sizes before it allocates anything on the
// device and the checksum once the last chunk is read; on a mismatch it frees the scene.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "eos_internal.cuh"

namespace {

constexpr char kMagic[8] = {'E', 'O', 'S', 'S', 'C', 'N', '0', '1'};
constexpr uint32_t kVersion = 2;  // 2: unused child slots hold lo = +inf, hi = -inf
constexpr size_t kChunk = 8u << 20;  // bytes per pinned chunk (a multiple of 32)

struct Header {
  char magic[8];
  uint32_t version;
  uint32_t n_tris, n_nodes, n_obj, n_lights;
  int32_t leaf_size, layout, width, builder, levels;
  float sah_cost, ambient_index, build_ms;
  uint64_t payload_bytes;
  uint64_t checksum;
  uint32_t reserved[6];
};
static_assert(sizeof(Header) == 104, "header layout");

// FNV-1a (64-bit basis and prime) in four lanes over consecutive 8-byte words, so that
// the four multiply chains run side by side; bytes after the last 32-byte block go to a
// fifth lane, and the lanes are folded into one value in order.  Every update but the
// last must be a multiple of 32 bytes.
struct Checksum {
  static constexpr uint64_t kBasis = 1469598103934665603ull;
  static constexpr uint64_t kPrime = 1099511628211ull;
  uint64_t lane[4] = {kBasis, kBasis, kBasis, kBasis};
  uint64_t tail = kBasis;
  void update(const unsigned char* p, size_t n) {
    size_t i = 0;
    for (; i + 32 <= n; i += 32) {
      uint64_t w[4];
      memcpy(w, p + i, 32);
      for (int j = 0; j < 4; ++j) lane[j] = (lane[j] ^ w[j]) * kPrime;
    }
    for (; i < n; ++i) tail = (tail ^ p[i]) * kPrime;
  }
  uint64_t value() const {
    uint64_t h = tail;
    for (int j = 0; j < 4; ++j) h = (h ^ lane[j]) * kPrime;
    return h;
  }
};

struct Part {
  void** dev;
  size_t bytes;
};

// The payload arrays of a flat scene of n triangles and the given node count.
std::vector<Part> parts(eos_scene* sc, size_t n, size_t n_nodes, size_t n_obj, size_t n_lights) {
  return {{&sc->d_nodes, 128 * n_nodes},         {&sc->d_tris, 48 * n},  {&sc->d_shade, 48 * n},
          {&sc->d_pos_of_id, 4 * n},             {&sc->d_codes, 4 * n},  {&sc->d_order, 4 * n},
          {&sc->d_mats, sizeof(eos_material) * n_obj}, {&sc->d_lights, sizeof(eos_light) * n_lights}};
}

// One async copy per part overlapping payload bytes [at, at + len) between the parts'
// device arrays and host (pinned chunk starting at payload offset `at`).
cudaError_t copy_range(const std::vector<Part>& ps, size_t at, size_t len, unsigned char* host, bool to_device,
                       cudaStream_t st) {
  size_t base = 0;
  for (const Part& p : ps) {
    const size_t lo = std::max(at, base), hi = std::min(at + len, base + p.bytes);
    if (lo < hi) {
      unsigned char* d = (unsigned char*)*p.dev + (lo - base);
      unsigned char* h = host + (lo - at);
      const cudaError_t e = to_device ? cudaMemcpyAsync(d, h, hi - lo, cudaMemcpyHostToDevice, st)
                                      : cudaMemcpyAsync(h, d, hi - lo, cudaMemcpyDeviceToHost, st);
      if (e != cudaSuccess) return e;
    }
    base += p.bytes;
  }
  return cudaSuccess;
}

// Two pinned chunks of the context (grown once) and one event per chunk.
struct Staging {
  unsigned char* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  ~Staging() {
    for (cudaEvent_t e : done)
      if (e) cudaEventDestroy(e);
  }
  eos_status init(eos_ctx* ctx) {
    if (ctx->pinned_bytes < 2 * kChunk) {
      if (ctx->pinned) cudaFreeHost(ctx->pinned);
      ctx->pinned = nullptr;
      ctx->pinned_bytes = 0;
      if (cudaHostAlloc(&ctx->pinned, 2 * kChunk, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        ctx->pinned = nullptr;
        return EOS_ERR_OOM;
      }
      ctx->pinned_bytes = 2 * kChunk;
    }
    for (int k = 0; k < 2; ++k) {
      buf[k] = (unsigned char*)ctx->pinned + k * kChunk;
      EOS_CUDA(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
    }
    return EOS_OK;
  }
};

}  // namespace

extern "C" eos_status eos_scene_save(const eos_scene* scene, const char* path) {
  if (!scene || !path) return EOS_ERR_INVALID_ARG;
  if (scene->instanced) return EOS_ERR_UNSUPPORTED;  // it refers to other scenes
  eos_scene* sc = const_cast<eos_scene*>(scene);
  eos_ctx* ctx = sc->ctx;
  EOS_CUDA(cudaSetDevice(ctx->device));
  EOS_CUDA(cudaStreamSynchronize(ctx->stream));
  const size_t n = std::max<size_t>(1, sc->dev.n_tris);
  const std::vector<Part> ps = parts(sc, n, sc->n_nodes, sc->dev.n_obj, sc->dev.n_lights);
  size_t total = 0;
  for (const Part& p : ps) total += p.bytes;
  Header h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.n_tris = (uint32_t)sc->dev.n_tris;
  h.n_nodes = sc->n_nodes;
  h.n_obj = (uint32_t)sc->dev.n_obj;
  h.n_lights = (uint32_t)sc->dev.n_lights;
  h.leaf_size = sc->leaf_size;
  h.layout = sc->layout;
  h.width = sc->width;
  h.builder = sc->builder;
  h.levels = sc->levels;
  h.sah_cost = sc->sah_cost;
  h.ambient_index = sc->dev.ambient_index;
  h.build_ms = sc->build_ms;
  h.payload_bytes = total;
  Staging sg;
  eos_status st = sg.init(ctx);
  if (st != EOS_OK) return st;
  FILE* f = std::fopen(path, "wb");
  if (!f) return EOS_ERR_IO;
  bool ok = std::fwrite(&h, sizeof h, 1, f) == 1;  // checksum filled in at the end
  Checksum cs;
  const size_t n_chunks = (total + kChunk - 1) / kChunk;
  // copy chunk i + 1 while chunk i is hashed and written
  auto issue = [&](size_t i) {
    const size_t at = i * kChunk, len = std::min(kChunk, total - at);
    return copy_range(ps, at, len, sg.buf[i & 1], false, ctx->stream) == cudaSuccess &&
           cudaEventRecord(sg.done[i & 1], ctx->stream) == cudaSuccess;
  };
  bool cuda_ok = n_chunks == 0 || issue(0);
  for (size_t i = 0; ok && cuda_ok && i < n_chunks; ++i) {
    if (i + 1 < n_chunks) cuda_ok = issue(i + 1);
    cuda_ok = cuda_ok && cudaEventSynchronize(sg.done[i & 1]) == cudaSuccess;
    if (!cuda_ok) break;
    const size_t len = std::min(kChunk, total - i * kChunk);
    cs.update(sg.buf[i & 1], len);
    ok = std::fwrite(sg.buf[i & 1], 1, len, f) == len;
  }
  cudaStreamSynchronize(ctx->stream);  // no copy into the chunks outlives the call
  h.checksum = cs.value();
  ok = ok && cuda_ok && std::fseek(f, 0, SEEK_SET) == 0 && std::fwrite(&h, sizeof h, 1, f) == 1;
  const bool closed = std::fclose(f) == 0;
  if (!cuda_ok) return EOS_ERR_CUDA;
  return ok && closed ? EOS_OK : EOS_ERR_IO;
}

extern "C" eos_status eos_scene_load(eos_ctx* ctx, const char* path, eos_scene** out) {
  if (!ctx || !path || !out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return EOS_ERR_IO;
  Header h;
  bool ok = std::fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, kMagic, 8) == 0 && h.version == kVersion;
  size_t n = 0, expect = 0;
  if (ok) {
    n = std::max<size_t>(1, h.n_tris);
    expect = 128 * (size_t)h.n_nodes + (48 + 48 + 4 + 4 + 4) * n + sizeof(eos_material) * h.n_obj +
             sizeof(eos_light) * h.n_lights;
    ok = h.payload_bytes == expect && h.n_tris < (1u << 25) && h.n_nodes >= 1 && h.n_nodes <= n &&
         h.n_obj >= 1 && h.n_obj < (1u << 24) && h.n_lights <= EOS_MAX_LIGHTS && (h.width == 2 || h.width == 4) &&
         h.levels >= 1 && (h.width - 1) * h.levels <= eos::kStackMax;
  }
  if (ok) {  // the payload must be all there before anything is allocated
    const long here = std::ftell(f);
    ok = here >= 0 && std::fseek(f, 0, SEEK_END) == 0 && std::ftell(f) - here == (long)expect &&
         std::fseek(f, here, SEEK_SET) == 0;
  }
  if (!ok) {
    std::fclose(f);
    return EOS_ERR_PARSE;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    std::fclose(f);
    return EOS_ERR_CUDA;
  }
  eos_scene* sc = new eos_scene();
  sc->ctx = ctx;
  auto fail = [&](eos_status s) {
    std::fclose(f);
    eos_scene_destroy(sc);  // syncs the stream first: no copy from the chunks is left
    return s;
  };
  const std::vector<Part> ps = parts(sc, n, h.n_nodes, h.n_obj, h.n_lights);
  for (const Part& p : ps) {
    const size_t bytes = std::max<size_t>(p.bytes, 16);
    if (cudaMalloc(p.dev, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(EOS_ERR_OOM);
    }
    sc->device_bytes += bytes;
  }
  Staging sg;
  eos_status st = sg.init(ctx);
  if (st != EOS_OK) return fail(st);
  Checksum cs;
  bool used[2] = {false, false};
  for (size_t at = 0, i = 0; at < expect; at += kChunk, ++i) {
    const size_t len = std::min(kChunk, expect - at);
    const int k = (int)(i & 1);
    if (used[k] && cudaEventSynchronize(sg.done[k]) != cudaSuccess) return fail(EOS_ERR_CUDA);
    if (std::fread(sg.buf[k], 1, len, f) != len) return fail(EOS_ERR_PARSE);
    cs.update(sg.buf[k], len);
    if (copy_range(ps, at, len, sg.buf[k], true, ctx->stream) != cudaSuccess ||
        cudaEventRecord(sg.done[k], ctx->stream) != cudaSuccess)
      return fail(EOS_ERR_CUDA);
    used[k] = true;
  }
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(EOS_ERR_CUDA);
  if (cs.value() != h.checksum) return fail(EOS_ERR_PARSE);
  std::fclose(f);
  sc->n_nodes = h.n_nodes;
  sc->leaf_size = h.leaf_size;
  sc->layout = h.layout;
  sc->width = h.width;
  sc->builder = h.builder;
  sc->levels = h.levels;
  sc->sah_cost = h.sah_cost;
  sc->build_ms = 0.0f;  // nothing was built
  sc->dev.n_tris = (int)h.n_tris;
  sc->dev.n_obj = (int)h.n_obj;
  sc->dev.n_lights = (int)h.n_lights;
  sc->dev.ambient_index = h.ambient_index;
  sc->dev.nodes = (const float4*)sc->d_nodes;
  sc->dev.tris = (const float4*)sc->d_tris;
  sc->dev.shade = (const float4*)sc->d_shade;
  sc->dev.pos_of_id = (const int32_t*)sc->d_pos_of_id;
  sc->dev.mats = (const float*)sc->d_mats;
  sc->dev.lights = (const float*)sc->d_lights;
  std::vector<eos_material> mats(h.n_obj);
  if (h.n_obj && cudaMemcpy(mats.data(), sc->d_mats, sizeof(eos_material) * h.n_obj, cudaMemcpyDeviceToHost) !=
                     cudaSuccess) {
    eos_scene_destroy(sc);  // the file is closed already
    return EOS_ERR_CUDA;
  }
  sc->branching = eos::has_branching(mats.data(), h.n_obj);
  *out = sc;
  return EOS_OK;
}
