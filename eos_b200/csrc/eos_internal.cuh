// Internal types of the render library: device scene layout, context and error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/eos_c.h"
#include "eos_math.cuh"

namespace eos {

constexpr int kMaxBounces = EOS_MAX_BOUNCES;
constexpr int kMaxLights = EOS_MAX_LIGHTS;
// Traversal stack entries: >= the binary LBVH depth bound (30 code bits + 32 index bits + 2)
// and >= 3 per level of the 4-wide layout (which is used only when its depth allows).
constexpr int kStackMax = 96;
constexpr float kInf = __builtin_huge_valf();
constexpr int kCounters = 8;  // ray / traversal counters per call (see trace.cuh)
constexpr int kMatStride = 10;  // floats per material (sizeof(eos_material) / 4)

// Device error word bits (atomicOr'ed by kernels, read back by the host).
enum : int {
  kErrStack = 1 << 0,
  kErrQueue = 1 << 1,
  kErrIndex = 1 << 2,
  kErrTimeout = 1 << 3,
  kErrDepth = 1 << 4,
};

// Status of a call from its device error word; every entry point maps it the same way.
inline eos_status err_to_status(int e) {
  if (e & (kErrStack | kErrDepth)) return EOS_ERR_STACK_OVERFLOW;
  if (e & kErrQueue) return EOS_ERR_QUEUE_OVERFLOW;
  if (e & kErrIndex) return EOS_ERR_INVALID_ARG;
  if (e & kErrTimeout) return EOS_ERR_TIMEOUT;
  return EOS_OK;
}

// ---------------------------------------------------------------------------------
// HBM layout of a scene (all 16-byte aligned, read with 128-bit loads):
//
//  Node record, 128 B = 8 x float4, the boxes of up to four children in the parent,
//  structure of arrays over the four slots (written by lbvh.cu, read by trace.cuh):
//    [0] lo.x[4]  [1] lo.y[4]  [2] lo.z[4]  [3] hi.x[4]  [4] hi.y[4]  [5] hi.z[4]
//    [6] ref[4]   [7] count[4]                (int)
//  ref: interior record index; leaf 0x80000000 | (count-1) << 25 | first (sorted positions
//  [first, first + count), count <= 32, first < 2^25); 0xC0000000 for an unused slot,
//  whose box is lo = +inf, hi = -inf.  count: triangles of a leaf, 0 interior, -1 unused.
//  A binary tree (width 2) fills two slots per record.
//
//  Triangle record (intersection), 48 B = 3 x float4, sorted (Morton) order:
//    [0] v1.x v1.y v1.z e1.x   [1] e1.y e1.z e2.x e2.y   [2] e2.z id(int) - -
//  Shading record, 48 B = 3 x float4, same order:
//    [0] n1.x n1.y n1.z n2.x   [1] n2.y n2.z n3.x n3.y   [2] n3.z obj(int) - -
// ---------------------------------------------------------------------------------
// One instance of a mesh in a two-level scene (eos_scene_create_instanced), 96 B with its
// padding: 16-byte aligned, because the traversal reads minv as three float4.
struct __align__(16) DevInstance {
  float minv[12];       // object-from-world affine, row-major 3x4 (the inverse of the transform)
  const float4* nodes;  // the mesh's node records, triangle and shading records
  const float4* tris;
  const float4* shade;
  int32_t id_offset;    // global id of the mesh's triangle 0 in this instance
  int32_t mat_base;     // added to the mesh's object ids
  const int32_t* pos_of_id;  // the mesh's triangle id -> sorted position (the adjoint's replay)
};
static_assert(sizeof(DevInstance) % 16 == 0 && alignof(DevInstance) == 16, "minv is read as float4");

struct DevScene {
  const float4* nodes;
  const float4* tris;
  const float4* shade;
  const int32_t* pos_of_id;  // triangle id -> sorted position
  const float* mats;         // n_obj x kMatStride: kd rgb, ks rgb, shininess, reflectivity,
                             // transparency, refractive index (eos_material)
  const float* lights;       // n_lights x 6: position xyz, colour rgb
  int32_t n_tris;
  int32_t n_obj;
  int32_t n_lights;
  float ambient_index;       // refractive index outside transparent objects
  const DevInstance* inst;   // two-level scene: nodes = tree over instances (leaf = one
  int32_t n_inst;            // instance), tris / shade / pos_of_id unused; else nullptr, 0
};

struct DevBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace eos

struct eos_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int* d_err = nullptr;                   // device error word
  unsigned long long* d_counts = nullptr; // ray / traversal counters [kCounters]
  std::map<std::string, eos::DevBuffer> scratch;
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  // PLOC round read-back ring (made on first use): mapped pinned slots the merge kernel
  // writes, and one event per slot
  int* ring_host = nullptr;
  int* ring_dev = nullptr;
  cudaEvent_t ring_ev[4] = {};
  // autotuner table: min triangle count -> tuned parameters
  std::map<uint32_t, eos_tuning> tuning;
  // test limits of the wavefront kernels (eos_ctx_set_limits); zeros = none
  eos_limits limits{0, 0, 0};
  // asynchronous batches (EOS_FLAG_ASYNC): two slots used in turn, each with its staging
  // buffer ("batch.async<k>"), the events that order its copies, and a pinned read-back of
  // its error word and counters; eos_ctx_synchronize folds pending slots in issue order
  struct AsyncSlot {
    cudaEvent_t rendered = nullptr;  // recorded on the render stream after the read-back
    cudaEvent_t copied = nullptr;    // recorded on copy_stream after the output copies
    bool pending = false;
    long long seq = 0;               // issue order
    eos_stats* stats = nullptr;      // caller's stats, filled at synchronize
    uint32_t launches = 0;
  };
  cudaStream_t copy_stream = nullptr;
  AsyncSlot async[2];
  // batched renders run as up to kWfLanes lanes (parts of the paths) at once; a lane's
  // nearest-hit stages run on its main stream (lane 0: the context's stream), its shadow
  // and shading stages on two more streams, ordered by events (all made on first use)
  struct WfLane {
    cudaStream_t main = nullptr;  // lane 1 only
    cudaStream_t side = nullptr;
    cudaStream_t shade = nullptr;
    cudaEvent_t ev_closest[eos::kMaxBounces] = {};
    cudaEvent_t ev_any[eos::kMaxBounces] = {};
    cudaEvent_t ev_shaded[eos::kMaxBounces] = {};
  };
  static constexpr int kWfLanes = 4;
  WfLane wf_lane[kWfLanes];
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kWfLanes] = {};
  int async_next = 0;
  long long async_seq = 0;
  unsigned long long* async_host = nullptr;  // pinned [2][kCounters + 1] (counters, error word)
  eos_status async_status = EOS_OK;          // first error of slots folded before a synchronize
  // per-call bookkeeping reported in eos_stats
  uint32_t launches = 0;
  float stage_ms[3] = {0, 0, 0};
  // batched-render graph cache: one instantiated graph per batch shape
  struct BatchGraph {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;  // kernel nodes in the graph
    ~BatchGraph() {
      if (exec) cudaGraphExecDestroy(exec);
    }
  };
  std::vector<std::unique_ptr<BatchGraph>> graphs;
  ~eos_ctx();
};

struct eos_scene {
  eos_ctx* ctx = nullptr;
  eos::DevScene dev{};
  void* d_nodes = nullptr;
  void* d_tris = nullptr;
  void* d_shade = nullptr;
  void* d_pos_of_id = nullptr;
  void* d_mats = nullptr;
  void* d_lights = nullptr;
  void* d_codes = nullptr;  // sorted Morton codes (kept for the test hook)
  void* d_order = nullptr;  // sorted triangle ids
  void* d_inst = nullptr;   // DevInstance array of a two-level scene
  bool instanced = false;
  bool branching = false;   // some material is both reflective and transparent: ray trees
  int mesh_levels = 0;      // deepest mesh tree of a two-level scene (stack bound)
  uint32_t n_nodes = 0;
  int leaf_size = 8;
  int layout = EOS_LAYOUT_SAH;
  int width = 4;   // children per 128-B node record: 4, or 2 (binary tree)
  int builder = EOS_BUILDER_PLOC;
  int levels = 0;  // depth of the tree of records
  float sah_cost = 0.0f;
  float build_ms = 0.0f;
  size_t device_bytes = 0;
};

namespace eos {

// Scratch buffers owned by the context, grown on demand and reused across calls.
void* scratch(eos_ctx* ctx, const char* name, size_t bytes, eos_status* st);
// Pointer classification (cudaPointerGetAttributes): true for device/managed memory.
bool is_device_ptr(const void* p);

// Scene build (lbvh.cu).  verts/normals/tris/tri_obj are device pointers.
eos_status build_scene(eos_ctx* ctx, eos_scene* sc, const float* d_verts, const float* d_normals,
                       uint32_t n_verts, const uint32_t* d_tris, const uint32_t* d_obj, uint32_t n_tris);

// PLOC hierarchy over n >= 2 leaves with boxes at blo / bhi[n-1+p] in Morton order
// (ploc.cu): child / range / parent in the refit's layout, perm[p] = record position of
// Morton position p, *depth = tree depth (above 4 * kStackMax nothing is written).
eos_status build_ploc(eos_ctx* ctx, int n, const float4* blo, const float4* bhi, int2* child, int2* range,
                      int* parent, uint32_t* perm, int* depth);

// True when some material is both reflective and transparent (the scene renders ray trees).
inline bool has_branching(const eos_material* m, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i)
    if (m[i].reflectivity > 0.0f && m[i].transparency > 0.0f) return true;
  return false;
}

// Parameters left at 0 take the context's tuned values for a scene of n_tris triangles.
eos_render_params with_tuning(const eos_ctx* ctx, const eos_render_params& p, uint32_t n_tris);

// Renderers (render.cu).
struct RenderArgs {
  const float* cam;  // 12 floats, device-visible via kernel params copy
  int width, height;
  int trace_depth;
  float pixel_offset;
  int spp;
  uint32_t jitter_seed;
  float* rgb;
  uint8_t* rgba8;
  int32_t* hit;
  eos_path_record* paths;
};
eos_status render_plain(eos_ctx* ctx, const eos_scene* sc, const eos_camera& cam,
                        const eos_render_params& p, float* rgb, uint8_t* rgba8, int32_t* hit,
                        void* paths, bool tree);
eos_status render_wavefront(eos_ctx* ctx, const eos_job* jobs, uint32_t n_jobs,
                            const eos_render_params& p, bool use_graph);
eos_status trace_closest(eos_ctx* ctx, const eos_scene* sc, const float* d_rays, uint32_t n,
                         int32_t* d_ids, float* d_t);
eos_status trace_any(eos_ctx* ctx, const eos_scene* sc, const float* d_rays, uint32_t n,
                     uint8_t* d_occ);
eos_status render_backward(eos_ctx* ctx, const eos_scene* sc, const eos_camera* cams, uint32_t n_views,
                           const eos_render_params& p, const void* d_paths,
                           const float* d_rgb, float* d_gmat, float* d_glight);

}  // namespace eos

namespace eos {
// Records a failing CUDA call for eos_last_error_detail (per host thread).
void note_cuda_error(cudaError_t e, const char* file, int line);
}  // namespace eos

#define EOS_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) {                             \
      eos::note_cuda_error(e_, __FILE__, __LINE__);      \
      if (e_ == cudaErrorMemoryAllocation) return EOS_ERR_OOM; \
      return EOS_ERR_CUDA;                               \
    }                                                    \
  } while (0)
