/*
 * eos_c.h -- C ABI of the B200-native Eos render path (sm_100a).
 *
 * Plain C: pointers, sizes and POD structs only.  Every function returns an eos_status
 * and never calls exit() or traps; the reference reports errors by printing and exit()
 * (src/cudaQualifiers.h:35-45).
 *
 * Each entry point replaces a reference interface:
 *   eos_device_count,            cudaGetDeviceCount + cudaSetDevice + per-renderer setup
 *   eos_ctx_create / destroy     (src/MultiDeviceRenderer.cu:31-110)
 *   eos_scene_create             Scene::flush + createCudaScene
 *                                (src/Scene.cpp:204-209, src/cudaStructures.cu:483-543):
 *                                uploads the triangles once and builds a Morton-code LBVH
 *                                on the GPU instead of the CPU top-down BVH
 *                                (src/BVH.cpp:97-111)
 *   eos_scene_set_materials      Scene::addMaterial + copyMaterials (src/Scene.cpp:85-91,
 *                                src/cudaStructures.cu:407-481)
 *   eos_scene_set_lights         Scene::addLightSource + copyLights (src/Scene.cpp:77-83,
 *                                src/cudaStructures.cu:177-218)
 *   eos_scene_set_ambient_index  Scene::setAmbientRefractiveIndex (src/Scene.cpp:134-136)
 *   eos_render                   DeviceRenderer::renderCudaSceneToHostBufferMegaKernel and
 *                                the C wrapper rayTrace_MegaKernel (src/DeviceRenderer.cu:61-109,
 *                                src/kernelWrapper.h:30), with the CPU RayTracer's full
 *                                Whitted semantics (src/RayTracer.cpp:85-458)
 *   eos_render_batch             (no reference counterpart: many views / scenes per launch)
 *   eos_render_backward          (no reference counterpart: adjoint of the shading)
 *   eos_trace_closest / any      Scene::findMinDistanceIntersectionBVH /
 *                                shadowRayVisibilityBVH (src/Scene.cpp:145-158)
 *   eos_mesh_load_obj            TriangleMesh::loadFromFile (src/triangleMesh.cpp:79-160)
 *   eos_scene_create_instanced   per-object transformations (src/Scene.cpp:96-106,
 *                                src/kernelInvocations.h:158-163) with shared meshes
 *   eos_scene_save / load        (no reference counterpart: the reference rebuilds its
 *                                tree in Scene::flush on every run, src/Scene.cpp:204-209)
 *
 * Buffers are owned by the caller.  A pointer argument may be host or device memory; the
 * library tells them apart with cudaPointerGetAttributes and stages host buffers through
 * its own device memory.  Calls on one context are serialised on its stream.
 */
#ifndef EOS_C_H
#define EOS_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EOS_ABI_VERSION 1
#define EOS_MAX_BOUNCES 8   /* trace_depth <= EOS_MAX_BOUNCES - 1 */
#define EOS_MAX_LIGHTS 32
#define EOS_HIT_NONE (-1)     /* ray traced, nothing hit */
#define EOS_HIT_UNTRACED (-2) /* bounce not reached */

typedef enum eos_status {
  EOS_OK = 0,
  EOS_ERR_INVALID_ARG = 1,
  EOS_ERR_OOM = 2,
  EOS_ERR_CUDA = 3,
  EOS_ERR_TIMEOUT = 4,        /* a bounded device loop ran out of iterations */
  EOS_ERR_STACK_OVERFLOW = 5, /* traversal stack exhausted (tree deeper than supported) */
  EOS_ERR_QUEUE_OVERFLOW = 6,
  EOS_ERR_UNSUPPORTED = 7,
  EOS_ERR_NO_DEVICE = 8,
  EOS_ERR_IO = 9,             /* a file could not be opened, read or written */
  EOS_ERR_PARSE = 10          /* malformed input file */
} eos_status;

typedef struct eos_ctx eos_ctx;
typedef struct eos_scene eos_scene;

/* Material of one object (src/Material.h:46-78).  The reference's diffuse/specular are
 * vec4 with an unused alpha and its shininess is an int; reflective = reflectivity > 0,
 * transparent = transparency > 0 (the reference's m_Transparent flag; its value is not
 * used otherwise).  A material that is both reflective and transparent makes a hit spawn
 * two secondary rays, as the reference traces them (src/RayTracer.cpp:339-407): the path
 * becomes a binary tree of rays, whose records need the tree form (EOS_FLAG_TREE_RECORDS).
 * The ambient term is unused by the reference renderer (src/RayTracer.cpp:412-413). */
typedef struct eos_material {
  float kd[3];
  float ks[3];
  float shininess;
  float reflectivity;
  float transparency;
  float refractive_index;
} eos_material;

/* Point light (src/LightSource.h:27-39); the position's w is 1. */
typedef struct eos_light {
  float position[3];
  float color[3];
} eos_light;

/* Pinhole camera, the reference's POD Camera (src/Camera.h:30-64): no fov, the lengths of
 * right and up set it.  Primary ray of pixel (x, y):
 *   d = normalize(aa*right + bb*up + view),  aa = ((x + ox) - W/2) * (1/(W/2)),
 *   bb = ((y + oy) - H/2) * (1/(H/2)),  row 0 = bottom  (src/RayTracer.cpp:119-145). */
typedef struct eos_camera {
  float position[3];
  float view[3];
  float right[3];
  float up[3];
  int32_t width;
  int32_t height;
} eos_camera;

enum { EOS_MODE_PLAIN = 0, EOS_MODE_WAVEFRONT = 1 };

typedef struct eos_render_params {
  int32_t trace_depth;  /* RayTracer::setTracedDepth: deepest bounce index (depth 2 -> 1) */
  float pixel_offset;   /* sub-pixel sample position: 0 = reference corners, 0.5 = centres */
  int32_t spp;          /* samples per pixel: 1, or >1 with hashed jitter */
  uint32_t jitter_seed;
  int32_t mode;         /* EOS_MODE_PLAIN (one launch per frame) or EOS_MODE_WAVEFRONT */
  int32_t block_size;   /* 0 = autotuned / default */
  int32_t queue_chunk;  /* rays taken per queue grab in the persistent kernels; 0 = default */
  int32_t stack_depth;  /* shared-memory part of the traversal stack; 0 = default */
  int32_t flags;        /* EOS_FLAG_* */
  int32_t row_begin;    /* render image rows [row_begin, row_end) only (split-frame, as */
  int32_t row_end;      /* src/MultiDeviceRenderer.cu:126-200 does per GPU); 0, 0 = the
                           whole image.  Outputs then hold those rows only. */
} eos_render_params;

/* Wavefront only: run the stages eagerly (no graph) with CUDA events between them and
 * report per-stage device time in eos_stats.stage_ms. */
#define EOS_FLAG_STAGE_TIMING 1
/* Path records in tree form: paths_out (eos_render, eos_job, eos_render_backward) holds
 * EOS_TREE_NODES(trace_depth) eos_tree_node entries per path instead of one
 * eos_path_record.  Required for path records of a scene with a material that is both
 * reflective and transparent (chain records of such a scene: EOS_ERR_UNSUPPORTED); any
 * scene may use it. */
#define EOS_FLAG_TREE_RECORDS 2
/* Samples on the reference's anti-aliasing grid (RayTracer::setAASamples / renderWithAA,
 * src/RayTracer.cpp:176-265): spp = n * n samples per pixel at offsets (p, q) / n,
 * p, q = 0..n-1, row by row, and the pixel is their sum times (1/n)^2 in the reference's
 * float order; pixel_offset and jitter_seed are not used.  spp must be a square
 * (EOS_ERR_INVALID_ARG otherwise).  Without the flag, spp > 1 samples at hashed jitter. */
#define EOS_FLAG_AA_GRID 4
/* eos_render_batch only: return once the batch is queued.  Host output buffers are copied on
 * a second stream of the context from one of two staging buffers, so one call's copy to the
 * host overlaps the next call's rendering; they are complete, and the call's device errors
 * and stats (when stats is not NULL; the pointer must stay valid) are known, when
 * eos_ctx_synchronize returns, which reports the first error of the pending calls.  At
 * most two calls are in flight: a third waits for the first one's copies.  Host outputs
 * should be pinned memory (pageable copies do not overlap). */
#define EOS_FLAG_ASYNC 8
/* Other flag bits are refused (EOS_ERR_INVALID_ARG). */

/* Tuned launch / layout parameters of one scene-size bucket (see eos_ctx_set_tuning). */
typedef struct eos_tuning {
  int32_t block_size;
  int32_t queue_chunk;
  int32_t stack_depth;
  int32_t leaf_size;
  int32_t layout;
  int32_t width;
  int32_t builder;
} eos_tuning;

/* Node layout of the LBVH: which subtrees become leaves. */
enum {
  EOS_LAYOUT_DEFAULT = 0, /* tuned value, else SAH */
  EOS_LAYOUT_SAH = 1,     /* leaf when n <= leaf_size and its SAH cost is not above the split's */
  EOS_LAYOUT_FIXED = 2    /* leaf whenever n <= leaf_size */
};

/* Hierarchy builder (both start from the Morton-sorted triangles). */
enum {
  EOS_BUILDER_DEFAULT = 0, /* tuned value, else PLOC */
  EOS_BUILDER_LBVH = 1,    /* Karras 2012 radix tree over the Morton codes */
  EOS_BUILDER_PLOC = 2     /* locally-ordered agglomerative clustering (Meister & Bittner 2018);
                              falls back to LBVH for a tree deeper than the traversal allows */
};

typedef struct eos_build_params {
  int32_t leaf_size;    /* largest leaf, 1..32 triangles; 0 = tuned value, else 8 */
  int32_t layout;       /* EOS_LAYOUT_* */
  int32_t width;        /* children per 128-B node record: 4, or 2 (binary tree);
                           0 = tuned value, else 4 */
  int32_t builder;      /* EOS_BUILDER_* */
} eos_build_params;

/* Per-path record of the bounce path: hit triangle id per bounce and, per bounce, the
 * bit mask of lights whose shadow ray was blocked.  It is also the forward record that
 * eos_render_backward replays (visibility frozen). */
typedef struct eos_path_record {
  int32_t hit[EOS_MAX_BOUNCES];
  uint32_t shadow[EOS_MAX_BOUNCES];
} eos_path_record;

/* One node of a tree-form path record.  Nodes in heap order: node 0 the primary ray; node
 * j's mirror ray is node 2j + 1, its transparent bounce's ray node 2j + 2; node j lies at
 * bounce floor(log2(j + 1)).  hit: triangle id, EOS_HIT_NONE or EOS_HIT_UNTRACED; shadow:
 * the blocked-light mask of the node's hit. */
typedef struct eos_tree_node {
  int32_t hit;
  uint32_t shadow;
} eos_tree_node;
#define EOS_TREE_NODES(trace_depth) ((1 << ((trace_depth) + 1)) - 1)

typedef struct eos_stats {
  uint64_t primary_rays;
  uint64_t shadow_rays;
  uint64_t secondary_rays;
  uint64_t nodes_closest;  /* BVH nodes fetched by nearest-hit (primary + mirror) rays */
  uint64_t tests_closest;  /* ray-triangle tests of nearest-hit rays */
  uint64_t nodes_shadow;   /* BVH nodes fetched by shadow rays */
  uint64_t tests_shadow;   /* ray-triangle tests of shadow rays */
  uint64_t shaded_hits;    /* hits shaded (each fetches normals + material) */
  float gpu_ms;            /* device time of the render, CUDA events on the context stream */
  int32_t error_flags;     /* device-side error bits raised during the call */
  uint32_t kernel_launches;/* kernels launched by the call (graph kernel nodes included) */
  float stage_ms[3];       /* with EOS_FLAG_STAGE_TIMING: nearest-hit, shadow, other stages */
} eos_stats;

typedef struct eos_scene_info {
  uint32_t n_tris;
  uint32_t n_nodes;       /* node records (128 B each) */
  uint32_t leaf_size;
  uint32_t layout;        /* EOS_LAYOUT_SAH or EOS_LAYOUT_FIXED */
  uint32_t width;         /* 2 or 4 (a 4-wide request too deep for the stack stays 2) */
  float sah_cost;         /* SAH cost of the tree, in triangle-test units */
  uint32_t n_objects;
  uint32_t n_lights;
  float build_ms;         /* device time of the build */
  uint64_t device_bytes;  /* device memory held by the scene */
  uint32_t builder;       /* EOS_BUILDER_LBVH or EOS_BUILDER_PLOC (the one used) */
  uint32_t depth;         /* levels of the tree of node records */
} eos_scene_info;

/* One view of one scene for eos_render_batch.  Outputs follow eos_render. */
typedef struct eos_job {
  const eos_scene* scene;
  eos_camera camera;
  int32_t trace_depth;
  float pixel_offset;
  int32_t spp;
  uint32_t jitter_seed;
  float* rgb_out;              /* [H*W*3], nullable */
  uint8_t* rgba8_out;          /* [H*W*4], nullable */
  eos_path_record* paths_out;  /* [H*W*spp], nullable */
  int32_t row_begin;           /* rows [row_begin, row_end) only; 0, 0 = whole image */
  int32_t row_end;             /* (outputs then hold (row_end - row_begin) rows) */
} eos_job;

/* Gradients of an image loss L; d_rgb = dL/drgb per pixel. */
typedef struct eos_grads {
  float* materials;  /* [n_objects * 7]: dL/dkd rgb, dL/dks rgb, dL/dlog(shininess) */
  float* lights;     /* [n_lights * 6]:  dL/dcolor rgb, dL/dposition xyz */
} eos_grads;

/* ---------------------------------------------------------------------------- context */
int32_t eos_abi_version(void);
const char* eos_status_string(eos_status s);
/* The CUDA error behind the calling thread's last EOS_ERR_CUDA / EOS_ERR_OOM: its name,
 * text and the library source line ("" when none).  No reference counterpart: the
 * reference prints the error and exits (src/cudaQualifiers.h:35-45). */
const char* eos_last_error_detail(void);
/* Number of CUDA devices visible to the process (0 when none). */
eos_status eos_device_count(int32_t* n);
eos_status eos_ctx_create(int32_t device, eos_ctx** out);
eos_status eos_ctx_destroy(eos_ctx* ctx);
/* Use a caller stream (a cudaStream_t) instead of the context's own; NULL restores it. */
eos_status eos_ctx_set_stream(eos_ctx* ctx, void* stream);
/* Waits for all work of the context, the copies of asynchronous batches included; returns
 * the first device error of the asynchronous calls since the last synchronize (EOS_OK if
 * none) and fills their stats. */
eos_status eos_ctx_synchronize(eos_ctx* ctx);
/* Autotuner table (no reference counterpart): parameters for scenes of at least min_tris
 * triangles.  A render / scene-create parameter left at 0 takes the entry with the largest
 * min_tris not above the scene's triangle count (for a batch: its largest scene). */
eos_status eos_ctx_set_tuning(eos_ctx* ctx, uint32_t min_tris, const eos_tuning* tuning);
eos_status eos_ctx_clear_tuning(eos_ctx* ctx);

/* Test limits of the wavefront kernels (no reference counterpart; the reference exits on
 * any error, src/cudaQualifiers.h:35-45).  They make the device error paths reachable on
 * ordinary scenes without faulting anything: a call that runs into a limit stops the work
 * it cannot do, returns the status below and leaves the context usable.  All zero (or
 * limits NULL) = no limits, the default.
 *   queue_entries  > 0: each secondary-ray and shadow-ray queue holds at most this many
 *                  entries; a bounce that emits more -> EOS_ERR_QUEUE_OVERFLOW
 *   work_budget    > 0: queue entries one persistent launch traces; the loop over the
 *                  queue leaves the entries beyond untraced -> EOS_ERR_TIMEOUT
 *   small_stack    != 0: traversal stacks of flat scenes hold 8 entries (the shared-memory
 *                  part only, no spill); a deeper traversal -> EOS_ERR_STACK_OVERFLOW
 * eos_render in wavefront mode and eos_render_batch apply them; eos_render_noalloc does not. */
typedef struct eos_limits {
  int32_t queue_entries;
  int32_t work_budget;
  int32_t small_stack;
} eos_limits;
eos_status eos_ctx_set_limits(eos_ctx* ctx, const eos_limits* limits);

/* ---------------------------------------------------------------------------- scenes */
/* verts / normals [n_verts*3], tris [n_tris*3] vertex indices, tri_obj [n_tris] material
 * rows.  Limits (EOS_ERR_INVALID_ARG, checked before any device work): n_tris < 2^25
 * (leaf references hold 25-bit positions), 1 <= n_materials, n_lights <= EOS_MAX_LIGHTS,
 * leaf_size <= 32; vertex indices < n_verts and material rows < n_materials are checked
 * on the device and fail the call the same way.  build may be NULL (tuned values). */
eos_status eos_scene_create(eos_ctx* ctx, const float* verts, const float* normals, uint32_t n_verts,
                            const uint32_t* tris, const uint32_t* tri_obj, uint32_t n_tris,
                            const eos_material* materials, uint32_t n_materials,
                            const eos_light* lights, uint32_t n_lights,
                            const eos_build_params* build, eos_scene** out);
/* Destroy every scene before the context it was created on (it syncs that context's stream). */
eos_status eos_scene_destroy(eos_scene* scene);
eos_status eos_scene_set_materials(eos_scene* scene, const eos_material* materials, uint32_t n);
eos_status eos_scene_set_lights(eos_scene* scene, const eos_light* lights, uint32_t n);
/* Scene::setAmbientRefractiveIndex (src/Scene.cpp:134-136): the index outside every
 * transparent object; 1 when never set. */
eos_status eos_scene_set_ambient_index(eos_scene* scene, float refractive_index);
eos_status eos_scene_get_info(const eos_scene* scene, eos_scene_info* info);
/* One placement of a mesh scene in an instanced scene. */
typedef struct eos_instance {
  const eos_scene* mesh;     /* a scene from eos_scene_create, used as geometry only (its tree,
                                triangles and object ids); it must outlive the instanced scene */
  float transform[12];       /* world-from-object affine, row-major 3x4 [A | t] */
  uint32_t material_base;    /* added to the mesh's triangle object ids */
} eos_instance;

/* A two-level scene: a tree over the instances' world boxes (built on the host), each
 * instance's mesh traversed with the ray moved into its object space -- what the
 * reference's GPU kernel does per triangle with the inverse of its transformation
 * (src/kernelInvocations.h:158-163, src/Scene.cpp:96-106).  Ray r in object space:
 * o' = A^-1 (o - t) evaluated as Minv [o, 1] (Minv = the inverse affine, computed in
 * double from the adjugate and rounded to float), d' = Minv [d, 0], not renormalised,
 * so t is the same parameter in both spaces.  The shading normal is
 * normalize(Minv^T n) of the mesh's interpolated unit normal; hit ids are global:
 * instance k's triangles are numbered after those of instances 0..k-1.  A mesh shared by
 * many instances is stored once.  eos_render / eos_render_batch / eos_trace_* and
 * eos_render_backward accept the scene; eos_scene_get_morton and eos_scene_save return
 * EOS_ERR_UNSUPPORTED. */
eos_status eos_scene_create_instanced(eos_ctx* ctx, const eos_instance* instances, uint32_t n_instances,
                                      const eos_material* materials, uint32_t n_materials,
                                      const eos_light* lights, uint32_t n_lights, eos_scene** out);

/* On-disk scene file: the built scene's device records (tree, triangle and shading
 * records, id map, Morton order), materials, lights and build settings, with a checksum
 * (FNV-1a over 8-byte words).  eos_scene_load uploads them into a new scene on ctx's
 * device without building anything; it renders exactly as the saved scene did (the
 * file's materials and lights; set_materials / set_lights change them as on any scene).
 * It needs no input mesh.  Errors: EOS_ERR_IO (the
 * file cannot be opened, read or written), EOS_ERR_PARSE (wrong magic or version, sizes
 * out of range, truncated, checksum mismatch), EOS_ERR_UNSUPPORTED (saving an instanced
 * scene, which refers to other scenes).  The file holds the host's byte order; it is
 * meant for the machine that wrote it. */
eos_status eos_scene_save(const eos_scene* scene, const char* path);
eos_status eos_scene_load(eos_ctx* ctx, const char* path, eos_scene** out);

/* Test hook: Morton codes of the triangles in sorted order and the sorted triangle ids. */
eos_status eos_scene_get_morton(const eos_scene* scene, uint32_t* codes, uint32_t* order);

/* ---------------------------------------------------------------------------- render */
/* rgb_out [H*W*3] float, rgba8_out [H*W*4] (src/RayTracer.cpp:150-153 quantisation),
 * hit_out [H*W*spp] primary hit triangle id, paths_out [H*W*spp]; all nullable. */
eos_status eos_render(eos_ctx* ctx, const eos_scene* scene, const eos_camera* camera,
                      const eos_render_params* params, float* rgb_out, uint8_t* rgba8_out,
                      int32_t* hit_out, eos_path_record* paths_out, eos_stats* stats);

/* Many views of one or several resident scenes through one wavefront pass (persistent
 * kernels over a global ray queue, replayed as a CUDA graph when the batch repeats).
 * Output buffers may be device or host memory; host buffers (pinned ones copy fastest)
 * are filled before the call returns. */
eos_status eos_render_batch(eos_ctx* ctx, const eos_job* jobs, uint32_t n_jobs,
                            const eos_render_params* params, eos_stats* stats);

/* Adjoint of the shading with visibility frozen from the forward records.  Views are
 * n_views cameras of equal size rendered with params' spp, jitter_seed and pixel_offset
 * (the same as the forward call's); paths are [n_views*H*W*spp] (the forward's order),
 * d_rgb is [n_views*H*W*3]: a pixel is the mean of its samples.  With a row band in
 * params (the forward's), paths and d_rgb hold those rows only and the gradients are the
 * band's share: the bands of a frame sum to its gradients. */
eos_status eos_render_backward(eos_ctx* ctx, const eos_scene* scene, const eos_camera* cameras,
                               uint32_t n_views, const eos_render_params* params,
                               const eos_path_record* paths, const float* d_rgb, eos_grads* grads);

/* ---------------------------------------------------------------------------- queries */
/* rays [n*6] (origin, direction).  Nearest hit: ids (EOS_HIT_NONE on a miss), t (may be
 * NULL).  Any hit: occluded[i] = 1 when some triangle is hit at t >= 0. */
eos_status eos_trace_closest(eos_ctx* ctx, const eos_scene* scene, const float* rays, uint32_t n,
                             int32_t* ids, float* t);
eos_status eos_trace_any(eos_ctx* ctx, const eos_scene* scene, const float* rays, uint32_t n,
                         uint8_t* occluded);

/* ---------------------------------------------------------------------------- meshes */
/* A triangle mesh read from a Wavefront OBJ file on the host; replaces
 * TriangleMesh::loadFromFile (src/triangleMesh.cpp:79-160), which imports through assimp
 * with aiProcess_Triangulate | aiProcess_GenSmoothNormals | aiProcess_JoinIdenticalVertices.
 * The same three steps are applied: polygons triangulated (a quad from its concave corner),
 * the file's vertex normals used when every face corner names one, otherwise smooth
 * normals generated (normalised sum of the unit face normals of all corners within
 * 1e-4 x the bounding-box diagonal), identical vertices joined.  Unlike the reference,
 * which keeps assimp's first mesh only, all faces of the file are loaded.  The arrays feed
 * eos_scene_create directly (verts, normals, tris). */
typedef struct eos_mesh eos_mesh;
typedef struct eos_mesh_info {
  uint32_t n_verts;
  uint32_t n_tris;
  uint32_t normals_from_file; /* 1: 'vn' normals of the file, 0: generated smooth normals */
  uint32_t n_faces;           /* 'f' statements read (before triangulation) */
  float bounds[6];            /* min xyz, max xyz of the triangles' vertices */
} eos_mesh_info;
eos_status eos_mesh_load_obj(const char* path, eos_mesh** out);
/* The same from OBJ text in memory (len bytes, need not be NUL-terminated). */
eos_status eos_mesh_parse_obj(const char* text, size_t len, eos_mesh** out);
eos_status eos_mesh_get_info(const eos_mesh* mesh, eos_mesh_info* info);
/* Host arrays: verts / normals [n_verts*3] float, tris [n_tris*3] vertex indices; any may
 * be NULL. */
eos_status eos_mesh_get_data(const eos_mesh* mesh, float* verts, float* normals, uint32_t* tris);
eos_status eos_mesh_destroy(eos_mesh* mesh);

/* ---------------------------------------------------------------------------- no-alloc */
/* Renders one view without allocating any device memory.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc while rendering -- code
 * that runs under another framework's allocator or memory pool, real-time loops that
 * forbid allocation after start-up, processes whose device memory belongs to another
 * owner.  The wavefront renderer's queues live in one fixed device array inside the
 * library (about 7.6 MB, held on every GPU that loads the library until the process
 * exits); scene, camera, stream and device output buffers come from the caller.
 *
 * Limits: at most EOS_NOALLOC_MAX_PATHS paths counted in 8x4-pixel tiles times spp
 * (128x128 at 1 spp) and at most EOS_NOALLOC_MAX_LIGHTS lights; larger requests return
 * EOS_ERR_INVALID_ARG without touching the GPU.  rgb_out [H*W*3] and paths_out [H*W*spp]
 * must be device memory (either may be NULL); stats may be NULL.  params->mode is not
 * read: the call always renders with the wavefront kernels (the same image as either
 * mode); block size, queue chunk and stack depth left at 0 take the scene context's tuned
 * values, as in eos_render; EOS_FLAG_STAGE_TIMING is ignored, EOS_FLAG_AA_GRID applies,
 * EOS_FLAG_TREE_RECORDS and scenes with a material both reflective and transparent (ray
 * trees need more than one ray per path and bounce) give EOS_ERR_UNSUPPORTED, other flags
 * EOS_ERR_INVALID_ARG.  The call waits for its stream.  The first call on a device looks up the
 * array's device address (make that first call before any stream capture).  All calls
 * share the one array: calls that overlap on the GPU race, so serialise them. */
#define EOS_NOALLOC_MAX_PATHS 16384
#define EOS_NOALLOC_MAX_LIGHTS 8
eos_status eos_render_noalloc(const eos_scene* scene, const eos_camera* camera,
                              const eos_render_params* params, void* stream, float* rgb_out,
                              eos_path_record* paths_out, eos_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* EOS_C_H */
