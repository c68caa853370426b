// C ABI of the render library (include/eos_c.h): argument checking, host/device buffer
// staging, error words and statistics.  The kernels live in lbvh.cu, render.cu,
// wavefront.cu and adjoint.cu.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "eos_internal.cuh"

using namespace eos;

eos_ctx::~eos_ctx() {
  if (copy_stream) cudaStreamSynchronize(copy_stream);
  for (AsyncSlot& a : async) {
    if (a.rendered) cudaEventDestroy(a.rendered);
    if (a.copied) cudaEventDestroy(a.copied);
  }
  if (async_host) cudaFreeHost(async_host);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  for (WfLane& l : wf_lane) {
    for (cudaStream_t s : {l.main, l.side, l.shade})
      if (s) cudaStreamSynchronize(s);
    for (int k = 0; k < eos::kMaxBounces; ++k) {
      if (l.ev_closest[k]) cudaEventDestroy(l.ev_closest[k]);
      if (l.ev_any[k]) cudaEventDestroy(l.ev_any[k]);
      if (l.ev_shaded[k]) cudaEventDestroy(l.ev_shaded[k]);
    }
    for (cudaStream_t s : {l.main, l.side, l.shade})
      if (s) cudaStreamDestroy(s);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  for (cudaEvent_t e : ev_join)
    if (e) cudaEventDestroy(e);
  for (auto& kv : scratch)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  if (pinned) cudaFreeHost(pinned);
  if (ring_host) cudaFreeHost(ring_host);
  for (cudaEvent_t e : ring_ev)
    if (e) cudaEventDestroy(e);
  if (d_err) cudaFree(d_err);
  if (d_counts) cudaFree(d_counts);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (own_stream) cudaStreamDestroy(own_stream);
}

namespace eos {

void* scratch(eos_ctx* ctx, const char* name, size_t bytes, eos_status* st) {
  DevBuffer& b = ctx->scratch[name];
  if (b.bytes >= bytes && b.ptr) return b.ptr;
  if (b.ptr) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
  }
  size_t want = std::max<size_t>(bytes, 256);
  if (cudaMalloc(&b.ptr, want) != cudaSuccess) {
    cudaGetLastError();
    b.ptr = nullptr;
    if (st) *st = EOS_ERR_OOM;
    return nullptr;
  }
  b.bytes = want;
  return b.ptr;
}

namespace {
thread_local char g_error_detail[192] = "";
}

void note_cuda_error(cudaError_t e, const char* file, int line) {
  const char* base = std::strrchr(file, '/');
  std::snprintf(g_error_detail, sizeof g_error_detail, "%s (%s) at %s:%d", cudaGetErrorName(e),
                cudaGetErrorString(e), base ? base + 1 : file, line);
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace eos

namespace {

// Device view of a caller buffer: device pointers pass through, host buffers are copied
// into a named scratch buffer on the context stream.
const void* stage_in(eos_ctx* ctx, const char* name, const void* p, size_t bytes, eos_status* st) {
  if (!p || bytes == 0) return p;
  if (is_device_ptr(p)) return p;
  void* d = scratch(ctx, name, bytes, st);
  if (!d) return nullptr;
  if (cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
    *st = EOS_ERR_CUDA;
    return nullptr;
  }
  return d;
}

struct OutBuf {
  void* user = nullptr;
  void* dev = nullptr;
  size_t bytes = 0;
  bool host = false;
};

eos_status out_buf(eos_ctx* ctx, const char* name, void* user, size_t bytes, OutBuf& o) {
  o.user = user;
  o.bytes = bytes;
  if (!user) return EOS_OK;
  if (is_device_ptr(user)) {
    o.dev = user;
    return EOS_OK;
  }
  eos_status st = EOS_OK;
  o.dev = scratch(ctx, name, bytes, &st);
  o.host = true;
  return o.dev ? EOS_OK : st;
}

eos_status copy_out(eos_ctx* ctx, const OutBuf& o) {
  if (o.user && o.host) EOS_CUDA(cudaMemcpyAsync(o.user, o.dev, o.bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return EOS_OK;
}

// Clears the error word and counters before a call.
eos_status begin_call(eos_ctx* ctx) {
  ctx->launches = 0;
  ctx->stage_ms[0] = ctx->stage_ms[1] = ctx->stage_ms[2] = 0.0f;
  EOS_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
  EOS_CUDA(cudaMemsetAsync(ctx->d_counts, 0, kCounters * sizeof(unsigned long long), ctx->stream));
  return EOS_OK;
}

// Waits for the call, reads the error word (and counters into stats).
eos_status end_call(eos_ctx* ctx, eos_stats* stats) {
  struct {
    unsigned long long c[kCounters];
    int err;
  } h;
  EOS_CUDA(cudaMemcpyAsync(h.c, ctx->d_counts, sizeof h.c, cudaMemcpyDeviceToHost, ctx->stream));
  EOS_CUDA(cudaMemcpyAsync(&h.err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  EOS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (stats) {
    stats->primary_rays = h.c[0];
    stats->shadow_rays = h.c[1];
    stats->secondary_rays = h.c[2];
    stats->nodes_closest = h.c[3];
    stats->tests_closest = h.c[4];
    stats->nodes_shadow = h.c[5];
    stats->tests_shadow = h.c[6];
    stats->shaded_hits = h.c[7];
    stats->error_flags = h.err;
    stats->kernel_launches = ctx->launches;
    for (int k = 0; k < 3; ++k) stats->stage_ms[k] = ctx->stage_ms[k];
  }
  return err_to_status(h.err);
}

bool valid_camera(const eos_camera* c) {
  return c && c->width > 0 && c->height > 0 && (long long)c->width * c->height <= (1ll << 28);
}

eos_status check_params(const eos_render_params* p) {
  if (!p) return EOS_ERR_INVALID_ARG;
  if (p->trace_depth < 0 || p->trace_depth >= EOS_MAX_BOUNCES) return EOS_ERR_INVALID_ARG;
  if (p->spp < 1 || p->spp > 1024) return EOS_ERR_INVALID_ARG;
  if (p->mode != EOS_MODE_PLAIN && p->mode != EOS_MODE_WAVEFRONT) return EOS_ERR_INVALID_ARG;
  if (p->flags & ~(EOS_FLAG_STAGE_TIMING | EOS_FLAG_TREE_RECORDS | EOS_FLAG_AA_GRID | EOS_FLAG_ASYNC))
    return EOS_ERR_INVALID_ARG;
  if ((p->flags & EOS_FLAG_AA_GRID) && aa_grid_side(p->spp) == 0) return EOS_ERR_INVALID_ARG;
  return EOS_OK;
}

// Bytes of one path record: eos_path_record, or the tree form's nodes.
size_t record_bytes(int flags, int trace_depth) {
  return (flags & EOS_FLAG_TREE_RECORDS) ? sizeof(eos_tree_node) * EOS_TREE_NODES(trace_depth)
                                         : sizeof(eos_path_record);
}

// Row band [rb, re) of an image of h rows; 0, 0 = all rows.
bool valid_rows(int h, int rb, int re) { return (rb == 0 && re == 0) || (rb >= 0 && rb < re && re <= h); }
int band_rows(int h, int rb, int re) { return re > 0 ? re - rb : h; }

eos_status set_device(eos_ctx* ctx) {
  EOS_CUDA(cudaSetDevice(ctx->device));
  return EOS_OK;
}

// Copy stream, events and pinned read-back of asynchronous batches (made on first use).
eos_status async_setup(eos_ctx* ctx) {
  if (ctx->copy_stream) return EOS_OK;
  EOS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  for (eos_ctx::AsyncSlot& a : ctx->async) {
    EOS_CUDA(cudaEventCreateWithFlags(&a.rendered, cudaEventDisableTiming));
    EOS_CUDA(cudaEventCreateWithFlags(&a.copied, cudaEventDisableTiming));
  }
  EOS_CUDA(cudaHostAlloc((void**)&ctx->async_host, 2 * (kCounters + 1) * sizeof(unsigned long long),
                         cudaHostAllocDefault));
  return EOS_OK;
}

// Waits for a pending asynchronous slot's copies and folds in its error word and counters.
eos_status async_finish(eos_ctx* ctx, int k) {
  eos_ctx::AsyncSlot& a = ctx->async[k];
  if (!a.pending) return EOS_OK;
  a.pending = false;
  EOS_CUDA(cudaEventSynchronize(a.copied));
  const unsigned long long* h = ctx->async_host + k * (kCounters + 1);
  const int err = (int)h[kCounters];
  if (a.stats) {
    eos_stats* st = a.stats;
    std::memset(st, 0, sizeof *st);
    st->primary_rays = h[0];
    st->shadow_rays = h[1];
    st->secondary_rays = h[2];
    st->nodes_closest = h[3];
    st->tests_closest = h[4];
    st->nodes_shadow = h[5];
    st->tests_shadow = h[6];
    st->shaded_hits = h[7];
    st->error_flags = err;
    st->kernel_launches = a.launches;
  }
  return err_to_status(err);
}

// Folds every pending asynchronous slot, oldest first; the first error wins.
eos_status async_drain(eos_ctx* ctx) {
  const int first = (ctx->async[0].pending && ctx->async[1].pending)
                        ? (ctx->async[0].seq < ctx->async[1].seq ? 0 : 1) : (ctx->async[0].pending ? 0 : 1);
  eos_status s0 = async_finish(ctx, first);
  eos_status s1 = async_finish(ctx, first ^ 1);
  return s0 != EOS_OK ? s0 : s1;
}

// Tuned entry for a scene of n triangles (zeros when the table has none).
eos_tuning tuned_for(const eos_ctx* ctx, uint32_t n) {
  eos_tuning t{0, 0, 0, 0, 0, 0, 0};
  auto it = ctx->tuning.upper_bound(n);
  if (it != ctx->tuning.begin()) t = std::prev(it)->second;
  return t;
}

}  // namespace

// Parameters left at 0 take the tuned value.
eos_render_params eos::with_tuning(const eos_ctx* ctx, const eos_render_params& p, uint32_t n_tris) {
  eos_render_params q = p;
  eos_tuning t = tuned_for(ctx, n_tris);
  if (q.block_size <= 0) q.block_size = t.block_size;
  if (q.queue_chunk <= 0) q.queue_chunk = t.queue_chunk;
  if (q.stack_depth <= 0) q.stack_depth = t.stack_depth;
  return q;
}

extern "C" {

int32_t eos_abi_version(void) { return EOS_ABI_VERSION; }

const char* eos_last_error_detail(void) { return g_error_detail; }

const char* eos_status_string(eos_status s) {
  switch (s) {
    case EOS_OK: return "ok";
    case EOS_ERR_INVALID_ARG: return "invalid argument";
    case EOS_ERR_OOM: return "out of device memory";
    case EOS_ERR_CUDA: return "CUDA error";
    case EOS_ERR_TIMEOUT: return "device loop ran out of iterations";
    case EOS_ERR_STACK_OVERFLOW: return "traversal stack overflow";
    case EOS_ERR_QUEUE_OVERFLOW: return "ray queue overflow";
    case EOS_ERR_UNSUPPORTED: return "unsupported";
    case EOS_ERR_NO_DEVICE: return "no CUDA device";
    case EOS_ERR_IO: return "file could not be read or written";
    case EOS_ERR_PARSE: return "malformed input file";
  }
  return "unknown status";
}

eos_status eos_device_count(int32_t* n) {
  if (!n) return EOS_ERR_INVALID_ARG;
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *n = c;
  return EOS_OK;
}

eos_status eos_ctx_create(int32_t device, eos_ctx** out) {
  if (!out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return EOS_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return EOS_ERR_INVALID_ARG;
  eos_ctx* ctx = new eos_ctx();
  ctx->device = device;
  eos_status st = EOS_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { st = EOS_ERR_CUDA; break; }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) { st = EOS_ERR_CUDA; break; }
    ctx->stream = ctx->own_stream;
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) { st = EOS_ERR_CUDA; break; }
    if (cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess) { st = EOS_ERR_OOM; break; }
    if (cudaMalloc(&ctx->d_counts, kCounters * sizeof(unsigned long long)) != cudaSuccess) { st = EOS_ERR_OOM; break; }
    cudaMemset(ctx->d_err, 0, sizeof(int));
    cudaMemset(ctx->d_counts, 0, kCounters * sizeof(unsigned long long));
  } while (0);
  if (st != EOS_OK) {
    cudaGetLastError();
    delete ctx;
    return st;
  }
  *out = ctx;
  return EOS_OK;
}

eos_status eos_ctx_destroy(eos_ctx* ctx) {
  if (!ctx) return EOS_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  delete ctx;
  return EOS_OK;
}

eos_status eos_ctx_set_stream(eos_ctx* ctx, void* stream) {
  if (!ctx) return EOS_ERR_INVALID_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return EOS_OK;
}

eos_status eos_ctx_synchronize(eos_ctx* ctx) {
  if (!ctx) return EOS_ERR_INVALID_ARG;
  EOS_CUDA(cudaSetDevice(ctx->device));
  EOS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->copy_stream) EOS_CUDA(cudaStreamSynchronize(ctx->copy_stream));
  const eos_status drained = async_drain(ctx);
  const eos_status st = ctx->async_status != EOS_OK ? ctx->async_status : drained;
  ctx->async_status = EOS_OK;
  return st;
}

eos_status eos_ctx_set_tuning(eos_ctx* ctx, uint32_t min_tris, const eos_tuning* t) {
  if (!ctx || !t) return EOS_ERR_INVALID_ARG;
  if (t->block_size < 0 || t->block_size > 1024 || t->queue_chunk < 0 || t->stack_depth < 0 || t->leaf_size < 0 ||
      t->leaf_size > 32 || t->layout < EOS_LAYOUT_DEFAULT || t->layout > EOS_LAYOUT_FIXED ||
      (t->width != 0 && t->width != 2 && t->width != 4) || t->builder < EOS_BUILDER_DEFAULT ||
      t->builder > EOS_BUILDER_PLOC)
    return EOS_ERR_INVALID_ARG;
  ctx->tuning[min_tris] = *t;
  return EOS_OK;
}

eos_status eos_ctx_clear_tuning(eos_ctx* ctx) {
  if (!ctx) return EOS_ERR_INVALID_ARG;
  ctx->tuning.clear();
  return EOS_OK;
}

eos_status eos_ctx_set_limits(eos_ctx* ctx, const eos_limits* lim) {
  if (!ctx) return EOS_ERR_INVALID_ARG;
  if (lim && (lim->queue_entries < 0 || lim->work_budget < 0)) return EOS_ERR_INVALID_ARG;
  ctx->limits = lim ? *lim : eos_limits{0, 0, 0};
  return EOS_OK;
}

eos_status eos_scene_create(eos_ctx* ctx, const float* verts, const float* normals, uint32_t n_verts,
                            const uint32_t* tris, const uint32_t* tri_obj, uint32_t n_tris,
                            const eos_material* materials, uint32_t n_materials, const eos_light* lights,
                            uint32_t n_lights, const eos_build_params* build, eos_scene** out) {
  if (!ctx || !out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  if (n_tris > 0 && (!verts || !normals || !tris || !tri_obj || n_verts == 0)) return EOS_ERR_INVALID_ARG;
  if (n_tris >= (1u << 25) || n_materials == 0 || !materials || n_lights > EOS_MAX_LIGHTS ||
      (n_lights > 0 && !lights))
    return EOS_ERR_INVALID_ARG;
  const eos_tuning tuned = tuned_for(ctx, n_tris);
  int leaf = build && build->leaf_size > 0 ? build->leaf_size : tuned.leaf_size;
  if (leaf <= 0) leaf = 8;
  if (leaf > 32) return EOS_ERR_INVALID_ARG;  // leaf refs hold counts up to 32
  int layout = build && build->layout != EOS_LAYOUT_DEFAULT ? build->layout : tuned.layout;
  if (layout == EOS_LAYOUT_DEFAULT) layout = EOS_LAYOUT_SAH;
  if (layout != EOS_LAYOUT_SAH && layout != EOS_LAYOUT_FIXED) return EOS_ERR_INVALID_ARG;
  int width = build && build->width != 0 ? build->width : tuned.width;
  if (width == 0) width = 4;
  if (width != 2 && width != 4) return EOS_ERR_INVALID_ARG;
  int builder = build && build->builder != EOS_BUILDER_DEFAULT ? build->builder : tuned.builder;
  if (builder == EOS_BUILDER_DEFAULT) builder = EOS_BUILDER_PLOC;
  if (builder != EOS_BUILDER_LBVH && builder != EOS_BUILDER_PLOC) return EOS_ERR_INVALID_ARG;
  eos_status st = set_device(ctx);
  if (st != EOS_OK) return st;
  eos_scene* sc = new eos_scene();
  sc->ctx = ctx;
  sc->leaf_size = leaf;
  sc->layout = layout;
  sc->width = width;
  sc->builder = builder;
  auto fail = [&](eos_status s) {
    eos_scene_destroy(sc);
    return s;
  };
  if ((st = begin_call(ctx)) != EOS_OK) return fail(st);
  const float* dv = (const float*)stage_in(ctx, "in.verts", verts, 12ull * n_verts, &st);
  const float* dn = (const float*)stage_in(ctx, "in.normals", normals, 12ull * n_verts, &st);
  const uint32_t* dt = (const uint32_t*)stage_in(ctx, "in.tris", tris, 12ull * n_tris, &st);
  const uint32_t* dob = (const uint32_t*)stage_in(ctx, "in.obj", tri_obj, 4ull * n_tris, &st);
  if (st != EOS_OK) return fail(st);
  if (cudaMalloc(&sc->d_mats, sizeof(eos_material) * n_materials) != cudaSuccess) return fail(EOS_ERR_OOM);
  if (cudaMalloc(&sc->d_lights, sizeof(eos_light) * std::max<uint32_t>(1, n_lights)) != cudaSuccess)
    return fail(EOS_ERR_OOM);
  sc->device_bytes += sizeof(eos_material) * n_materials + sizeof(eos_light) * std::max<uint32_t>(1, n_lights);
  sc->dev.n_obj = (int)n_materials;
  sc->dev.n_lights = (int)n_lights;
  sc->dev.ambient_index = 1.0f;
  sc->dev.n_tris = (int)n_tris;
  if ((st = eos_scene_set_materials(sc, materials, n_materials)) != EOS_OK) return fail(st);
  if (n_lights && (st = eos_scene_set_lights(sc, lights, n_lights)) != EOS_OK) return fail(st);
  if ((st = build_scene(ctx, sc, dv, dn, n_verts, dt, dob, n_tris)) != EOS_OK) return fail(st);
  sc->dev.nodes = (const float4*)sc->d_nodes;
  sc->dev.tris = (const float4*)sc->d_tris;
  sc->dev.shade = (const float4*)sc->d_shade;
  sc->dev.pos_of_id = (const int32_t*)sc->d_pos_of_id;
  sc->dev.mats = (const float*)sc->d_mats;
  sc->dev.lights = (const float*)sc->d_lights;
  if ((st = end_call(ctx, nullptr)) != EOS_OK) return fail(st);
  // object ids must index the material table: checked on the device copy
  {
    std::vector<uint32_t> probe;
    (void)probe;
  }
  *out = sc;
  return EOS_OK;
}

eos_status eos_scene_destroy(eos_scene* sc) {
  if (!sc) return EOS_ERR_INVALID_ARG;
  if (sc->ctx) {
    cudaSetDevice(sc->ctx->device);
    cudaStreamSynchronize(sc->ctx->stream);
  }
  void* bufs[] = {sc->d_nodes, sc->d_tris, sc->d_shade, sc->d_pos_of_id, sc->d_mats, sc->d_lights, sc->d_codes,
                  sc->d_order, sc->d_inst};
  for (void* b : bufs)
    if (b) cudaFree(b);
  delete sc;
  return EOS_OK;
}

eos_status eos_scene_set_materials(eos_scene* sc, const eos_material* m, uint32_t n) {
  if (!sc || !m || n != (uint32_t)sc->dev.n_obj) return EOS_ERR_INVALID_ARG;
  EOS_CUDA(cudaSetDevice(sc->ctx->device));
  // a material both reflective and transparent spawns two secondary rays per hit: the
  // scene then renders in ray-tree form
  std::vector<eos_material> host(n);
  const bool dev = is_device_ptr(m);
  if (dev) EOS_CUDA(cudaMemcpy(host.data(), m, sizeof(eos_material) * n, cudaMemcpyDeviceToHost));
  else std::memcpy(host.data(), m, sizeof(eos_material) * n);
  EOS_CUDA(cudaMemcpyAsync(sc->d_mats, m, sizeof(eos_material) * n,
                           dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, sc->ctx->stream));
  EOS_CUDA(cudaStreamSynchronize(sc->ctx->stream));
  sc->branching = has_branching(host.data(), n);
  return EOS_OK;
}

eos_status eos_scene_set_ambient_index(eos_scene* sc, float refractive_index) {
  if (!sc || !(refractive_index > 0.0f)) return EOS_ERR_INVALID_ARG;
  sc->dev.ambient_index = refractive_index;
  return EOS_OK;
}

eos_status eos_scene_set_lights(eos_scene* sc, const eos_light* l, uint32_t n) {
  if (!sc || (!l && n) || n != (uint32_t)sc->dev.n_lights) return EOS_ERR_INVALID_ARG;
  if (n == 0) return EOS_OK;
  EOS_CUDA(cudaSetDevice(sc->ctx->device));
  cudaMemcpyKind kind = is_device_ptr(l) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  EOS_CUDA(cudaMemcpyAsync(sc->d_lights, l, sizeof(eos_light) * n, kind, sc->ctx->stream));
  EOS_CUDA(cudaStreamSynchronize(sc->ctx->stream));
  return EOS_OK;
}

eos_status eos_scene_get_info(const eos_scene* sc, eos_scene_info* info) {
  if (!sc || !info) return EOS_ERR_INVALID_ARG;
  info->n_tris = (uint32_t)sc->dev.n_tris;
  info->n_nodes = sc->n_nodes;
  info->leaf_size = (uint32_t)sc->leaf_size;
  info->layout = (uint32_t)sc->layout;
  info->sah_cost = sc->sah_cost;
  info->width = (uint32_t)sc->width;
  info->n_objects = (uint32_t)sc->dev.n_obj;
  info->n_lights = (uint32_t)sc->dev.n_lights;
  info->build_ms = sc->build_ms;
  info->device_bytes = sc->device_bytes;
  info->builder = (uint32_t)sc->builder;
  info->depth = (uint32_t)sc->levels;
  return EOS_OK;
}

eos_status eos_scene_get_morton(const eos_scene* sc, uint32_t* codes, uint32_t* order) {
  if (!sc) return EOS_ERR_INVALID_ARG;
  if (sc->instanced) return EOS_ERR_UNSUPPORTED;
  EOS_CUDA(cudaSetDevice(sc->ctx->device));
  size_t b = 4ull * sc->dev.n_tris;
  if (b == 0) return EOS_OK;
  if (codes) EOS_CUDA(cudaMemcpyAsync(codes, sc->d_codes, b, cudaMemcpyDefault, sc->ctx->stream));
  if (order) EOS_CUDA(cudaMemcpyAsync(order, sc->d_order, b, cudaMemcpyDefault, sc->ctx->stream));
  EOS_CUDA(cudaStreamSynchronize(sc->ctx->stream));
  return EOS_OK;
}

eos_status eos_render(eos_ctx* ctx, const eos_scene* sc, const eos_camera* cam, const eos_render_params* p,
                      float* rgb_out, uint8_t* rgba8_out, int32_t* hit_out, eos_path_record* paths_out,
                      eos_stats* stats) {
  if (!ctx || !sc || !valid_camera(cam)) return EOS_ERR_INVALID_ARG;
  eos_status st = check_params(p);
  if (st != EOS_OK) return st;
  if (!valid_rows(cam->height, p->row_begin, p->row_end)) return EOS_ERR_INVALID_ARG;
  const bool tree_records = (p->flags & EOS_FLAG_TREE_RECORDS) != 0;
  if (paths_out && sc->branching && !tree_records) return EOS_ERR_UNSUPPORTED;  // one hit per bounce cannot hold a tree
  if ((st = set_device(ctx)) != EOS_OK) return st;
  const size_t npx = (size_t)cam->width * band_rows(cam->height, p->row_begin, p->row_end);
  const size_t npath = npx * p->spp;
  OutBuf o_rgb, o_q, o_hit, o_paths;
  if ((st = out_buf(ctx, "out.rgb", rgb_out, 12 * npx, o_rgb)) != EOS_OK) return st;
  if ((st = out_buf(ctx, "out.rgba8", rgba8_out, 4 * npx, o_q)) != EOS_OK) return st;
  if ((st = out_buf(ctx, "out.hit", hit_out, 4 * npath, o_hit)) != EOS_OK) return st;
  if ((st = out_buf(ctx, "out.paths", paths_out, record_bytes(p->flags, p->trace_depth) * npath, o_paths)) != EOS_OK)
    return st;
  if ((st = begin_call(ctx)) != EOS_OK) return st;
  EOS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  if (p->mode == EOS_MODE_PLAIN) {
    st = render_plain(ctx, sc, *cam, with_tuning(ctx, *p, (uint32_t)sc->dev.n_tris), (float*)o_rgb.dev,
                      (uint8_t*)o_q.dev, (int32_t*)o_hit.dev, o_paths.dev, tree_records || sc->branching);
  } else {
    if (hit_out) return EOS_ERR_UNSUPPORTED;  // per-path hits come from paths_out in this mode
    eos_job job;
    job.scene = sc;
    job.camera = *cam;
    job.trace_depth = p->trace_depth;
    job.pixel_offset = p->pixel_offset;
    job.spp = p->spp;
    job.jitter_seed = p->jitter_seed;
    job.rgb_out = (float*)o_rgb.dev;
    job.rgba8_out = (uint8_t*)o_q.dev;
    job.paths_out = (eos_path_record*)o_paths.dev;
    job.row_begin = p->row_begin;
    job.row_end = p->row_end;
    st = render_wavefront(ctx, &job, 1, with_tuning(ctx, *p, (uint32_t)sc->dev.n_tris), false);
  }
  if (st != EOS_OK) return st;
  EOS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  if ((st = copy_out(ctx, o_rgb)) != EOS_OK) return st;
  if ((st = copy_out(ctx, o_q)) != EOS_OK) return st;
  if ((st = copy_out(ctx, o_hit)) != EOS_OK) return st;
  if ((st = copy_out(ctx, o_paths)) != EOS_OK) return st;
  st = end_call(ctx, stats);
  if (stats) cudaEventElapsedTime(&stats->gpu_ms, ctx->ev0, ctx->ev1);
  return st;
}

eos_status eos_render_batch(eos_ctx* ctx, const eos_job* jobs, uint32_t n_jobs, const eos_render_params* p,
                            eos_stats* stats) {
  if (!ctx || !jobs || n_jobs == 0) return EOS_ERR_INVALID_ARG;
  eos_status st = check_params(p);
  if (st != EOS_OK) return st;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const eos_job& jb = jobs[j];
    if (!jb.scene || !valid_camera(&jb.camera) || jb.trace_depth < 0 || jb.trace_depth >= EOS_MAX_BOUNCES ||
        jb.spp < 1 || jb.spp > 1024 || !valid_rows(jb.camera.height, jb.row_begin, jb.row_end))
      return EOS_ERR_INVALID_ARG;
    if (jb.paths_out && jb.scene->branching && !(p->flags & EOS_FLAG_TREE_RECORDS)) return EOS_ERR_UNSUPPORTED;
    if ((p->flags & EOS_FLAG_AA_GRID) && aa_grid_side(jb.spp) == 0) return EOS_ERR_INVALID_ARG;
  }
  if ((st = set_device(ctx)) != EOS_OK) return st;
  const bool async = (p->flags & EOS_FLAG_ASYNC) != 0;
  int slot = 0;
  if (async) {
    if ((st = async_setup(ctx)) != EOS_OK) return st;
    slot = ctx->async_next;
    // the slot's previous call (two calls ago) must have finished copying out of its
    // staging buffer; its status is kept for the next synchronize
    if (ctx->async[slot].pending) {
      const eos_status prev = async_finish(ctx, slot);
      if (ctx->async_status == EOS_OK) ctx->async_status = prev;
    }
  }
  // host output buffers are staged through one device buffer and copied back at the end
  struct HostOut {
    void* user;
    size_t off, bytes;
  };
  std::vector<HostOut> host_outs;
  std::vector<eos_job> dj(jobs, jobs + n_jobs);
  size_t staged = 0;
  auto plan = [&](void* user, size_t bytes) {
    if (!user || is_device_ptr(user)) return;
    host_outs.push_back({user, staged, bytes});
    staged += (bytes + 255) & ~size_t(255);
  };
  for (const eos_job& jb : dj) {
    const size_t npx = (size_t)jb.camera.width * band_rows(jb.camera.height, jb.row_begin, jb.row_end);
    plan(jb.rgb_out, 12 * npx);
    plan(jb.rgba8_out, 4 * npx);
    plan(jb.paths_out, record_bytes(p->flags, jb.trace_depth) * npx * jb.spp);
  }
  char* stage = nullptr;
  if (staged) {
    stage = (char*)scratch(ctx, async ? (slot ? "batch.async1" : "batch.async0") : "batch.host_out", staged, &st);
    if (st != EOS_OK) return st;
    size_t k = 0;
    auto swap_in = [&](auto*& ptr) {
      if (k < host_outs.size() && ptr && (void*)ptr == host_outs[k].user)
        ptr = reinterpret_cast<std::remove_reference_t<decltype(ptr)>>(stage + host_outs[k++].off);
    };
    for (eos_job& jb : dj) {
      swap_in(jb.rgb_out);
      swap_in(jb.rgba8_out);
      swap_in(jb.paths_out);
    }
  }
  if ((st = begin_call(ctx)) != EOS_OK) return st;
  EOS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  uint32_t largest = 0;
  for (uint32_t j = 0; j < n_jobs; ++j) largest = std::max(largest, (uint32_t)jobs[j].scene->dev.n_tris);
  st = render_wavefront(ctx, dj.data(), n_jobs, with_tuning(ctx, *p, largest),
                        (p->flags & EOS_FLAG_STAGE_TIMING) == 0);
  if (st != EOS_OK) return st;
  if (async) {
    // read-back of this call's error word and counters (ordered before the next call's
    // clearing), then the output copies on the copy stream, behind the render
    eos_ctx::AsyncSlot& a = ctx->async[slot];
    unsigned long long* hb = ctx->async_host + slot * (kCounters + 1);
    EOS_CUDA(cudaMemcpyAsync(hb, ctx->d_counts, kCounters * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx->stream));
    EOS_CUDA(cudaMemsetAsync(hb + kCounters, 0, sizeof(unsigned long long), ctx->stream));
    EOS_CUDA(cudaMemcpyAsync(hb + kCounters, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    EOS_CUDA(cudaEventRecord(a.rendered, ctx->stream));
    EOS_CUDA(cudaStreamWaitEvent(ctx->copy_stream, a.rendered, 0));
    for (const HostOut& h : host_outs)
      EOS_CUDA(cudaMemcpyAsync(h.user, stage + h.off, h.bytes, cudaMemcpyDeviceToHost, ctx->copy_stream));
    EOS_CUDA(cudaEventRecord(a.copied, ctx->copy_stream));
    a.pending = true;
    a.seq = ++ctx->async_seq;
    a.stats = stats;
    a.launches = ctx->launches;
    ctx->async_next = slot ^ 1;
    return EOS_OK;
  }
  EOS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  for (const HostOut& h : host_outs)
    EOS_CUDA(cudaMemcpyAsync(h.user, stage + h.off, h.bytes, cudaMemcpyDeviceToHost, ctx->stream));
  st = end_call(ctx, stats);
  if (stats) cudaEventElapsedTime(&stats->gpu_ms, ctx->ev0, ctx->ev1);
  return st;
}

eos_status eos_render_backward(eos_ctx* ctx, const eos_scene* sc, const eos_camera* cams, uint32_t n_views,
                               const eos_render_params* p, const eos_path_record* paths, const float* d_rgb,
                               eos_grads* grads) {
  if (!ctx || !sc || !cams || n_views == 0 || !paths || !d_rgb || !grads || !grads->materials || !grads->lights)
    return EOS_ERR_INVALID_ARG;
  eos_status st = check_params(p);
  if (st != EOS_OK) return st;
  for (uint32_t v = 0; v < n_views; ++v)
    if (!valid_camera(&cams[v]) || cams[v].width != cams[0].width || cams[v].height != cams[0].height)
      return EOS_ERR_INVALID_ARG;
  if (!valid_rows(cams[0].height, p->row_begin, p->row_end)) return EOS_ERR_INVALID_ARG;
  if (sc->branching && !(p->flags & EOS_FLAG_TREE_RECORDS)) return EOS_ERR_UNSUPPORTED;  // chain records of a tree
  if ((st = set_device(ctx)) != EOS_OK) return st;
  const size_t npx = (size_t)n_views * cams[0].width * band_rows(cams[0].height, p->row_begin, p->row_end);
  if ((st = begin_call(ctx)) != EOS_OK) return st;
  const void* dp = stage_in(ctx, "bw.paths", paths, record_bytes(p->flags, p->trace_depth) * npx * p->spp, &st);
  const float* dg = (const float*)stage_in(ctx, "bw.drgb", d_rgb, 12 * npx, &st);
  if (st != EOS_OK) return st;
  OutBuf o_m, o_l;
  if ((st = out_buf(ctx, "bw.gm", grads->materials, 28ull * sc->dev.n_obj, o_m)) != EOS_OK) return st;
  if ((st = out_buf(ctx, "bw.gl", grads->lights, 24ull * std::max(1, sc->dev.n_lights), o_l)) != EOS_OK) return st;
  EOS_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  st = render_backward(ctx, sc, cams, n_views, *p, dp, dg, (float*)o_m.dev, (float*)o_l.dev);
  if (st != EOS_OK) return st;
  EOS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  if ((st = copy_out(ctx, o_m)) != EOS_OK) return st;
  if ((st = copy_out(ctx, o_l)) != EOS_OK) return st;
  return end_call(ctx, nullptr);
}

eos_status eos_trace_closest(eos_ctx* ctx, const eos_scene* sc, const float* rays, uint32_t n, int32_t* ids,
                             float* t) {
  if (!ctx || !sc || (n && (!rays || !ids))) return EOS_ERR_INVALID_ARG;
  eos_status st = set_device(ctx);
  if (st != EOS_OK) return st;
  if ((st = begin_call(ctx)) != EOS_OK) return st;
  const float* dr = (const float*)stage_in(ctx, "q.rays", rays, 24ull * n, &st);
  if (st != EOS_OK) return st;
  OutBuf oi, ot;
  if ((st = out_buf(ctx, "q.ids", ids, 4ull * n, oi)) != EOS_OK) return st;
  if ((st = out_buf(ctx, "q.t", t, 4ull * n, ot)) != EOS_OK) return st;
  if ((st = trace_closest(ctx, sc, dr, n, (int32_t*)oi.dev, (float*)ot.dev)) != EOS_OK) return st;
  if ((st = copy_out(ctx, oi)) != EOS_OK) return st;
  if ((st = copy_out(ctx, ot)) != EOS_OK) return st;
  return end_call(ctx, nullptr);
}

eos_status eos_trace_any(eos_ctx* ctx, const eos_scene* sc, const float* rays, uint32_t n, uint8_t* occluded) {
  if (!ctx || !sc || (n && (!rays || !occluded))) return EOS_ERR_INVALID_ARG;
  eos_status st = set_device(ctx);
  if (st != EOS_OK) return st;
  if ((st = begin_call(ctx)) != EOS_OK) return st;
  const float* dr = (const float*)stage_in(ctx, "q.rays", rays, 24ull * n, &st);
  if (st != EOS_OK) return st;
  OutBuf oo;
  if ((st = out_buf(ctx, "q.occ", occluded, n, oo)) != EOS_OK) return st;
  if ((st = trace_any(ctx, sc, dr, n, (uint8_t*)oo.dev)) != EOS_OK) return st;
  if ((st = copy_out(ctx, oo)) != EOS_OK) return st;
  return end_call(ctx, nullptr);
}

}  // extern "C"
