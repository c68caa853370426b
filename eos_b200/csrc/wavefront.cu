// Wavefront renderer: many views of one or several resident scenes through one global
// ray queue, per bounce:
//
//   closest  (persistent)  nearest hit of every ray in R_k; writes a hit record; emits
//                          one shadow ray per light into S_k and the mirror ray into
//                          R_k+1, both compacted with warp ballot / popc and one atomic
//                          per warp
//   any      (persistent)  any-hit of every shadow ray in S_k; blocked -> bit in the hit's
//                          light mask
//   shade                  Phong over the unblocked lights, in light order, per hit; for a
//                          one-sample job, the colour and pixel of each path ending here
//   resolve                colour fold c_k = phong_k + refl_k c_k+1 per path, sample mean,
//                          RGB / RGBA8 to each job's buffers (jobs of several samples, trees)
//
// The semantics are those of the reference's CPU renderer (src/RayTracer.cpp:268-458),
// identical to the plain renderer (render.cu) bit for bit: the same hits, masks and
// colours.  Persistent kernels take `queue_chunk` rays per warp from a work counter, so
// rays of uneven cost balance across the SMs.  Paths are processed in chunks of at most
// kChunkPathsMax, fewer when the queues of a chunk would exceed kQueueBudget bytes: one
// large chunk keeps the persistent kernels' tails short (8.3M paths in one chunk ran the
// config-2 batch 25 % faster than four chunks of 2M).  Bounce k's shadow and shading stages
// run beside bounce k+1's nearest-hit stage (Overlap), and a large chunk runs as kLanes
// parts side by side (render_wavefront), so that stages fill each other's tails.  The whole
// sequence for a batch is captured once as a CUDA graph and replayed; the job table is
// uploaded before each replay.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "trace.cuh"

namespace eos {
namespace {

constexpr long long kChunkPathsMax = 1ll << 24;
constexpr long long kQueueBudget = 16ll << 30;  // bytes of queues and accumulators per chunk
constexpr long long kLaneSplitMin = 1ll << 20;  // paths of a chunk from which it runs as several lanes
constexpr int kLanes = 2;                       // lanes of such a chunk (<= eos_ctx::kWfLanes)
constexpr int kTileW = 8, kTileH = 4;  // one warp = 8 x 4 pixels

struct DevJob {
  DevScene s;
  float cam[12];
  int w, h, trace_depth, spp;
  int y0, rows;  // image rows [y0, y0 + rows) are rendered; outputs hold those rows
  float off;
  uint32_t seed;
  int grid;  // side of the reference's AA grid (EOS_FLAG_AA_GRID), 0 = jitter
  float* rgb;
  uint8_t* rgba8;
  eos_path_record* paths;
  eos_tree_node* tree;  // tree-form records instead of paths (EOS_FLAG_TREE_RECORDS)
  int tree_nn;          // nodes per tree record: EOS_TREE_NODES(trace_depth)
  long long path_off;  // first global path index of this job
  long long n_paths;   // tiled, padded path count
  int tiles_x;
  int pad;
};

struct RayQ {
  float4 a;  // origin xyz, path (int)
  float4 b;  // direction xyz, ray-tree node (int; tree mode)
};
struct HitQ {
  float4 a;  // P xyz, path (int; tree mode: path | node << 24, all ones = padding)
  float4 b;  // N xyz, obj (int; -1 = miss)
};

// Ray-tree mode (materials both reflective and transparent, or tree-form records): a hit
// may emit a mirror ray (node 2j + 1) and a transparent one (node 2j + 2); accumulators
// hold one entry per node (phong rgb, weight of the edge into the node: reflectivity, or
// -K for a transparent ray with its sign marking the mix) and k_wf_resolve folds each
// path's tree bottom-up.  Paths of a chunk are < 2^24 and nodes < 2^8, so a hit record
// packs both into one word.
constexpr uint32_t kTreePad = 0xFFFFFFFFu;
// Chain mode: object id bit of a hit record whose path ends at this bounce (no secondary
// ray follows); a miss (object id -1) ends its path too.
constexpr int kEndsBit = 1 << 30;
__device__ __forceinline__ uint32_t tree_pack(int path, int node) { return (uint32_t)path | ((uint32_t)node << 24); }
struct ShadowQ {
  float4 a;  // origin xyz, hit index (int)
  float4 b;  // direction xyz, light (int)
};

// Per-bounce counters: [1] tail of R_k+1 (the input count of bounce k+1), [2] tail of
// S_k, [3] closest work, [4] any work.
constexpr int kCtr = 8;

struct WfArgs {
  const DevJob* jobs;
  int n_jobs;
  long long c0;   // first path of the chunk
  int n_chunk;    // paths in the chunk
  int k;          // bounce
  int depth;      // max trace depth over jobs
  const RayQ* rin;
  RayQ* rout;
  HitQ* hits;
  uint32_t* masks;
  ShadowQ* sq;
  float4* acc;   // [n_chunk][depth+1] phong rgb, reflectivity (tree mode: [n_chunk][nn], see above)
  int* ctr;      // [depth+1][kCtr]
  int cap_r, cap_s;
  int nn;         // tree mode: nodes per path (EOS_TREE_NODES of the deepest job)
  int qchunk;
  int work_limit;  // queue entries a persistent launch traces (test limit; INT_MAX = all)
  int init_in_primary;  // chain mode without a work budget: the primary nearest-hit stage
                        // does k_wf_init's clearing for its own paths (no init launch), and
                        // the shading stage writes the pixel of a one-sample path when the
                        // path ends (k_wf_resolve skips those jobs)
  int resolve;          // host side: some job needs k_wf_resolve
  int* err;
  unsigned long long* counts;
};

__device__ __forceinline__ int find_job(const DevJob* jobs, int n, long long path) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(&jobs[mid].path_off) <= path) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Tiled path order: warp-sized 8x4 pixel tiles, samples of a pixel consecutive.
// y is the row within the job's band (output row); the image row is j.y0 + y.
__device__ __forceinline__ bool path_pixel(const DevJob& j, long long local, int& x, int& y, int& smp) {
  smp = (int)(local % j.spp);
  long long tp = local / j.spp;
  long long tile = tp >> 5;
  int lane = (int)(tp & 31);
  x = (int)(tile % j.tiles_x) * kTileW + (lane & (kTileW - 1));
  y = (int)(tile / j.tiles_x) * kTileH + (lane >> 3);
  return x < j.w && y < j.rows;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-wide work grab: lane 0 takes `qchunk` items, broadcast to the warp.
__device__ __forceinline__ int grab(int* ctr, int qchunk) {
  int s = 0;
  if ((threadIdx.x & 31) == 0) s = atomicAdd(ctr, qchunk);
  return __shfl_sync(0xffffffffu, s, 0);
}

// Work budget of a persistent launch (eos_limits.work_budget): its loop over the queue
// stops after work_limit entries and raises the timeout bit when entries are left.  The
// entries beyond stay untraced and the shading stage reads no further than the budget
// either: their path records keep EOS_HIT_UNTRACED and no stale queue entry is read.
__device__ __forceinline__ int budget(int n, int work_limit, int* err) {
  if (n <= work_limit) return n;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, kErrTimeout);
  return work_limit;
}

// The wavefront traversal kernels are capped at 64 registers (blocks up to 256, 4 per SM):
// measured faster than no cap (77 registers) and than caps of 56 or 48 (spills).  CAP is
// the traversal stack's size (TraversalStack): kStackMax, or SH for the small-stack test
// limit.
// Appends the secondary rays of the lanes with `want` to R_k+1 (ballot / popc compaction,
// one atomic per warp); node = the ray-tree node of the ray (0 outside tree mode).
// Warp-uniform: every lane calls it.
__device__ __forceinline__ void emit_secondary(const WfArgs& A, int* ctr, bool want, int path, int node, f3 ro,
                                               f3 rd) {
  const int lane = threadIdx.x & 31;
  const uint32_t rb = __ballot_sync(0xffffffffu, want);
  if (!rb) return;
  int rbase = 0;
  if (lane == 0) rbase = atomicAdd(&ctr[1], __popc(rb));
  rbase = __shfl_sync(0xffffffffu, rbase, 0);
  if (want) {
    const int pos = rbase + __popc(rb & lanemask_lt());
    if (pos >= A.cap_r) {
      atomicOr(A.err, kErrQueue);
    } else {
      RayQ r;
      r.a = make_float4(ro.x, ro.y, ro.z, __int_as_float(path));
      r.b = make_float4(rd.x, rd.y, rd.z, __int_as_float(node));
      A.rout[pos] = r;
    }
  }
}

template <bool PRIMARY, int SH, int CAP = kStackMax, bool TREE = false>
__global__ void __launch_bounds__(256, 4) k_wf_closest(WfArgs A) {
  extern __shared__ uint2 shstack[];
  uint2* shs = shstack + threadIdx.x;
  const int stride = blockDim.x;
  int* ctr = A.ctr + A.k * kCtr;
  // primary rays of the chunk, or the secondary rays of bounce k-1
  const int n_in = budget(PRIMARY ? A.n_chunk : min(ctr[1 - kCtr], A.cap_r), A.work_limit, A.err);
  const int lane = threadIdx.x & 31;
  unsigned nrays = 0, nshadow = 0, nhits = 0;
  unsigned long long nodes = 0, tests = 0;
  for (;;) {
    int start = grab(&ctr[3], A.qchunk);
    if (start >= n_in) break;
    int end = min(start + A.qchunk, n_in);
    for (int base = start; base < end; base += 32) {
      int i = base + lane;
      bool valid = i < end;
      bool hit = false, refl = false, transp = false;
      int path = -1, jb = 0, obj = -1, node = 0;
      f3 o = mk3(0, 0, 0), d = mk3(0, 0, 1), P = o, N = o, ro = o, rd = d, to = o, td = d;
      if (valid) {
        if (PRIMARY) {
          long long gp = A.c0 + i;
          jb = find_job(A.jobs, A.n_jobs, gp);
          const DevJob& J = A.jobs[jb];
          int x, y, smp;
          if (path_pixel(J, gp - J.path_off, x, y, smp)) {
            float ox, oy;
            sample_offset((uint32_t)((J.y0 + y) * J.w + x), smp, J.spp, J.seed, J.off, ox, oy, J.grid);
            d = primary_direction(J.cam, J.w, J.h, x, J.y0 + y, ox, oy);
            o = mk3(J.cam[0], J.cam[1], J.cam[2]);
            path = i;
          } else {
            valid = false;
            if (!TREE && A.init_in_primary) {  // tile padding: the mark k_wf_init writes
              HitQ hq;
              hq.a = make_float4(0, 0, 0, __int_as_float(-1));
              hq.b = make_float4(0, 0, 0, __int_as_float(-1));
              A.hits[i] = hq;
            }
          }
        } else {
          RayQ r = A.rin[i];
          o = mk3(r.a.x, r.a.y, r.a.z);
          d = mk3(r.b.x, r.b.y, r.b.z);
          path = __float_as_int(r.a.w);
          if constexpr (TREE) node = __float_as_int(r.b.w);
          jb = find_job(A.jobs, A.n_jobs, A.c0 + path);
        }
      }
      const DevJob& J = A.jobs[jb];
      if (valid) {
        ++nrays;
        Hit h = closest_hit<SH, true, CAP>(J.s, o, d, shs, stride, A.err);
        nodes += h.nodes;
        tests += h.tests;
        hit = h.pos >= 0;
        nhits += hit;
        if constexpr (TREE) {
          if (J.tree) {
            int x, y, smp;
            path_pixel(J, A.c0 + path - J.path_off, x, y, smp);
            J.tree[(((size_t)y * J.w + x) * J.spp + smp) * J.tree_nn + node].hit = hit ? h.id : EOS_HIT_NONE;
          }
          if (hit) {
            hit_geometry(J.s, o, d, h, P, N, obj);
            const float* m = J.s.mats + kMatStride * obj;
            if (A.k < J.trace_depth) {  // children only within the trace depth: nodes < tree_nn
              float* row = reinterpret_cast<float*>(A.acc + (size_t)path * A.nn);
              if (m[7] > 0.0f) {
                mirror_ray(d, P, N, ro, rd);
                refl = true;
                row[4 * (2 * node + 1) + 3] = m[7];
              }
              if (m[8] > 0.0f) {
                row[4 * (2 * node + 2) + 3] = -transparent_ray(m, J.s.ambient_index, d, P, N, to, td);
                transp = true;
              }
            }
          }
        } else {
          const bool whole = PRIMARY && A.init_in_primary;  // this stage writes the whole record / row
          if (J.paths) {
            int x, y, smp;
            path_pixel(J, A.c0 + path - J.path_off, x, y, smp);
            eos_path_record* rec = J.paths + ((size_t)y * J.w + x) * J.spp + smp;
            if (whole) {
              eos_path_record r;
              for (int k = 0; k < kMaxBounces; ++k) {
                r.hit[k] = EOS_HIT_UNTRACED;
                r.shadow[k] = 0u;
              }
              r.hit[0] = hit ? h.id : EOS_HIT_NONE;
              *rec = r;
            } else {
              rec->hit[A.k] = hit ? h.id : EOS_HIT_NONE;
            }
          }
          float w = 0.0f;
          if (hit) {
            hit_geometry(J.s, o, d, h, P, N, obj);
            refl = secondary_ray(J.s.mats + kMatStride * obj, J.s.ambient_index, d, P, N, ro, rd, w);
            refl = refl && A.k < J.trace_depth;
          }
          float4* row = A.acc + (size_t)path * (A.depth + 1);
          if (whole) {
            row[0] = make_float4(0, 0, 0, w);
            for (int k = 1; k <= A.depth; ++k) row[k] = make_float4(0, 0, 0, 0);
          } else if (hit) {
            reinterpret_cast<float*>(row + A.k)[3] = w;
          }
        }
        HitQ hq;
        hq.a = make_float4(P.x, P.y, P.z, TREE ? __uint_as_float(tree_pack(path, node)) : __int_as_float(path));
        hq.b = make_float4(N.x, N.y, N.z, __int_as_float(hit ? (TREE || refl ? obj : obj | kEndsBit) : -1));
        A.hits[i] = hq;
        A.masks[i] = 0u;
      }
      // shadow rays, compacted light-major inside the warp's block of the queue so that a
      // warp of the any-hit kernel mostly traces rays towards one light
      int nl = hit ? J.s.n_lights : 0;
      int maxl = nl;
      for (int off = 16; off > 0; off >>= 1) maxl = max(maxl, __shfl_xor_sync(0xffffffffu, maxl, off));
      if (maxl > 0) {
        int total = nl;
        for (int off = 16; off > 0; off >>= 1) total += __shfl_xor_sync(0xffffffffu, total, off);
        int wbase = 0;
        if (lane == 0) wbase = atomicAdd(&ctr[2], total);
        wbase = __shfl_sync(0xffffffffu, wbase, 0);
        // past the capacity the queue overflows (error bit); the entries below it are all
        // written, also those of a block that only partly fits, because the shadow stage
        // reads every entry below min(count, capacity)
        if (wbase + total > A.cap_s && lane == 0) atomicOr(A.err, kErrQueue);
        int prefix = 0;
        for (int l = 0; l < maxl; ++l) {
          uint32_t bl = __ballot_sync(0xffffffffu, l < nl);
          const int pos = wbase + prefix + __popc(bl & lanemask_lt());
          if (l < nl && pos < A.cap_s) {
            const float* lp = J.s.lights + 6 * l;
            f3 sd = norm3(sub3(mk3(lp[0], lp[1], lp[2]), P));
            f3 so = add3(P, scale3(kRayEps, sd));
            ShadowQ s;
            s.a = make_float4(so.x, so.y, so.z, __int_as_float(i));
            s.b = make_float4(sd.x, sd.y, sd.z, __int_as_float((jb << 5) | l));
            A.sq[pos] = s;
          }
          prefix += __popc(bl);
        }
        nshadow += nl;
      }
      // secondary rays (mirror, or the transparent bounce's ray; both in tree mode)
      if constexpr (TREE) {
        emit_secondary(A, ctr, refl, path, 2 * node + 1, ro, rd);
        emit_secondary(A, ctr, transp, path, 2 * node + 2, to, td);
      } else {
        emit_secondary(A, ctr, refl, path, 0, ro, rd);
      }
    }
  }
  warp_add_count(&A.counts[A.k == 0 ? kCntPrimary : kCntSecondary], nrays);
  warp_add_count(&A.counts[kCntShadow], nshadow);
  warp_add_count(&A.counts[kCntHits], nhits);
  warp_add_count(&A.counts[kCntNodesC], nodes);
  warp_add_count(&A.counts[kCntTestsC], tests);
}

template <int SH, int CAP = kStackMax>
__global__ void __launch_bounds__(256, 4) k_wf_any(WfArgs A) {
  extern __shared__ uint2 shstack[];
  uint2* shs = shstack + threadIdx.x;
  const int stride = blockDim.x;
  int* ctr = A.ctr + A.k * kCtr;
  const int n = budget(min(ctr[2], A.cap_s), A.work_limit, A.err);
  unsigned long long nodes = 0, tests = 0;
  for (;;) {
    int start = grab(&ctr[4], A.qchunk);
    if (start >= n) break;
    int end = min(start + A.qchunk, n);
    for (int i = start + (threadIdx.x & 31); i < end; i += 32) {
      ShadowQ s = A.sq[i];
      int hi = __float_as_int(s.a.w);
      int key = __float_as_int(s.b.w);
      const DevJob& J = A.jobs[key >> 5];
      AnyResult ar =
          any_hit<SH, true, CAP>(J.s, mk3(s.a.x, s.a.y, s.a.z), mk3(s.b.x, s.b.y, s.b.z), shs, stride, A.err);
      nodes += ar.nodes;
      tests += ar.tests;
      if (ar.hit) atomicOr(&A.masks[hi], 1u << (key & 31));
    }
  }
  warp_add_count(&A.counts[kCntNodesA], nodes);
  warp_add_count(&A.counts[kCntTestsA], tests);
}

// The output pixel of path gp (its first sample): FP32 RGB and / or RGBA8.
__device__ __forceinline__ void write_pixel(const DevJob& J, long long gp, f3 c) {
  int x, y, smp;
  path_pixel(J, gp - J.path_off, x, y, smp);
  const size_t pix = (size_t)y * J.w + x;
  if (J.rgb) {
    J.rgb[3 * pix] = c.x;
    J.rgb[3 * pix + 1] = c.y;
    J.rgb[3 * pix + 2] = c.z;
  }
  if (J.rgba8)
    reinterpret_cast<uchar4*>(J.rgba8)[pix] = make_uchar4(quantize(c.x), quantize(c.y), quantize(c.z), 255);
}

template <bool TREE = false>
__global__ void k_wf_shade(WfArgs A) {
  int* ctr = A.ctr + A.k * kCtr;
  // primary hit records beyond the work budget keep k_wf_init's padding marks
  const int n = A.k == 0 ? A.n_chunk : min(min(ctr[1 - kCtr], A.cap_r), A.work_limit);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    HitQ hq = A.hits[i];
    int path, node = 0;
    if constexpr (TREE) {
      const uint32_t w = __float_as_uint(hq.a.w);
      if (w == kTreePad) continue;  // tile padding (primary only)
      path = (int)(w & 0xFFFFFFu);
      node = (int)(w >> 24);
    } else {
      path = __float_as_int(hq.a.w);
      if (path < 0) continue;  // tile padding (primary only)
    }
    int obj = __float_as_int(hq.b.w);
    bool ends = false;
    if constexpr (!TREE) {
      ends = obj < 0 || (obj & kEndsBit) != 0;
      if (obj >= 0) obj &= ~kEndsBit;
    }
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, A.c0 + path)];
    if (obj >= 0) {
      f3 P = mk3(hq.a.x, hq.a.y, hq.a.z), N = mk3(hq.b.x, hq.b.y, hq.b.z);
      f3 cam = mk3(J.cam[0], J.cam[1], J.cam[2]);
      const float* m = J.s.mats + kMatStride * obj;
      uint32_t mask = A.masks[i];
      f3 acc = mk3(0, 0, 0);
      for (int l = 0; l < J.s.n_lights; ++l)
        if (!(mask & (1u << l))) acc = add3(acc, phong_light(m, J.s.lights + 6 * l, P, N, cam));
      // .w: the bounce weight (tree mode: the weight of the edge into the node), set by the hit stage
      float4* e = TREE ? A.acc + (size_t)path * A.nn + node : A.acc + (size_t)path * (A.depth + 1) + A.k;
      *e = make_float4(acc.x, acc.y, acc.z, e->w);
      if (J.paths || (TREE && J.tree)) {
        int x, y, smp;
        path_pixel(J, A.c0 + path - J.path_off, x, y, smp);
        const size_t rec = ((size_t)y * J.w + x) * J.spp + smp;
        if (TREE) J.tree[rec * J.tree_nn + node].shadow = mask;
        else J.paths[rec].shadow[A.k] = mask;
      }
    }
    if constexpr (!TREE) {
      // the path's colour is final: slots beyond this bounce hold zeros, which the fold of
      // k_wf_resolve passes through unchanged (0 + 0 * 0 = +0), so folding from here gives
      // its colour bit for bit
      if (ends && A.init_in_primary && J.spp == 1 && J.grid == 0) {
        const float4* a = A.acc + (size_t)path * (A.depth + 1);
        f3 c = mk3(0, 0, 0);
        for (int k = A.k; k >= 0; --k) {
          const float4 e = a[k];
          c = fold_colour(mk3(e.x, e.y, e.z), e.w, c);
        }
        write_pixel(J, A.c0 + path, c);
      }
    }
  }
}

// Marks every padding entry of the primary hit queue and clears path records / acc.
template <bool TREE = false>
__global__ void k_wf_init(WfArgs A) {
  const int slots = TREE ? A.nn : A.depth + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_chunk; i += gridDim.x * blockDim.x) {
    long long gp = A.c0 + i;
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, gp)];
    for (int k = 0; k < slots; ++k) A.acc[(size_t)i * slots + k] = make_float4(0, 0, 0, 0);
    HitQ hq;
    hq.a = make_float4(0, 0, 0, TREE ? __uint_as_float(kTreePad) : __int_as_float(-1));
    hq.b = make_float4(0, 0, 0, __int_as_float(-1));
    A.hits[i] = hq;
    int x, y, smp;
    if (TREE && J.tree && path_pixel(J, gp - J.path_off, x, y, smp)) {
      eos_tree_node* rec = J.tree + (((size_t)y * J.w + x) * J.spp + smp) * J.tree_nn;
      for (int k = 0; k < J.tree_nn; ++k) rec[k] = eos_tree_node{EOS_HIT_UNTRACED, 0u};
    }
    if (!TREE && J.paths && path_pixel(J, gp - J.path_off, x, y, smp)) {
      eos_path_record rec;
      for (int k = 0; k < kMaxBounces; ++k) {
        rec.hit[k] = EOS_HIT_UNTRACED;
        rec.shadow[k] = 0u;
      }
      J.paths[((size_t)y * J.w + x) * J.spp + smp] = rec;
    }
  }
}

// Colour of one path: the chain fold c_k = fold_colour(phong_k, w_k, c_k+1), or in tree
// mode the bottom-up fold of its nodes in place (children 2j + 1 and 2j + 2 come after j).
template <bool TREE>
__device__ __forceinline__ f3 path_colour(const WfArgs& A, long long path) {
  if constexpr (TREE) {
    float4* a = A.acc + (size_t)path * A.nn;
    for (int j = A.nn - 1; j >= 0; --j) {
      const float4 e = a[j];
      f3 c = mk3(e.x, e.y, e.z);
      if (2 * j + 1 < A.nn) {
        const float4 r = a[2 * j + 1], t = a[2 * j + 2];
        // r.w = reflectivity of the mirror ray (0: none); t.w = -K of the transparent one
        // (+0: none; the sign bit marks it, -0 for K = 0)
        c = tree_colour(c, r.w, mk3(r.x, r.y, r.z), signbit(t.w), -t.w, mk3(t.x, t.y, t.z));
      } else {
        c = tree_colour(c, 0.0f, mk3(0, 0, 0), false, 0.0f, mk3(0, 0, 0));
      }
      a[j] = make_float4(c.x, c.y, c.z, e.w);
    }
    return mk3(a[0].x, a[0].y, a[0].z);
  } else {
    const float4* a = A.acc + (size_t)path * (A.depth + 1);
    f3 c = mk3(0, 0, 0);
    for (int k = A.depth; k >= 0; --k) {
      float4 e = a[k];
      c = fold_colour(mk3(e.x, e.y, e.z), e.w, c);
    }
    return c;
  }
}

template <bool TREE = false>
__global__ void k_wf_resolve(WfArgs A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_chunk; i += gridDim.x * blockDim.x) {
    long long gp = A.c0 + i;
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, gp)];
    if (!TREE && A.init_in_primary && J.spp == 1 && J.grid == 0) continue;  // written by k_wf_shade
    int x, y, smp;
    if (!path_pixel(J, gp - J.path_off, x, y, smp) || smp != 0) continue;
    f3 sum = mk3(0, 0, 0);
    for (int s = 0; s < J.spp; ++s) sum = add3(sum, path_colour<TREE>(A, i + s));
    if (J.spp > 1 || J.grid > 0) sum = scale3(sample_weight(J.spp, J.grid), sum);
    write_pixel(J, gp, sum);
  }
}

struct Chunk {
  long long c0;
  int n;
};

}  // namespace
}  // namespace eos

namespace eos {
namespace {

// Device time per stage when the caller asks for it (eager launches only): events around
// each kernel, waited for right away.
struct StageTimer {
  bool on;
  cudaStream_t st;
  cudaEvent_t e0, e1;
  float* acc;  // [3] milliseconds per stage
  eos_status begin() { return on ? (cudaEventRecord(e0, st) == cudaSuccess ? EOS_OK : EOS_ERR_CUDA) : EOS_OK; }
  eos_status end(int stage) {
    if (!on) return EOS_OK;
    EOS_CUDA(cudaEventRecord(e1, st));
    EOS_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    EOS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    acc[stage] += ms;
    return EOS_OK;
  }
};

#define EOS_TRY(x)                  \
  do {                              \
    eos_status s_ = (x);            \
    if (s_ != EOS_OK) return s_;    \
  } while (0)

// The kernels of one configuration: a warp of the nearest-hit / shadow kernels takes
// `queue_chunk` rays and finishes all before taking more.  small_stack selects the test
// instantiation whose traversal stack is its SH shared-memory entries only (launch_config
// pins SH = 8 then); tree the ray-tree mode.
template <int SH>
struct StageKernels {
  void (*closest_primary)(WfArgs);
  void (*closest)(WfArgs);
  void (*any)(WfArgs);
  void (*shade)(WfArgs);
  void (*init)(WfArgs);
  void (*resolve)(WfArgs);
  static StageKernels get(bool small_stack, bool tree) {
    if (tree)
      return {k_wf_closest<true, SH, kStackMax, true>, k_wf_closest<false, SH, kStackMax, true>, k_wf_any<SH>,
              k_wf_shade<true>, k_wf_init<true>, k_wf_resolve<true>};
    if constexpr (SH == 8) {
      if (small_stack)
        return {k_wf_closest<true, 8, 8>, k_wf_closest<false, 8, 8>, k_wf_any<8, 8>,
                k_wf_shade<false>, k_wf_init<false>, k_wf_resolve<false>};
    }
    return {k_wf_closest<true, SH>, k_wf_closest<false, SH>, k_wf_any<SH>,
            k_wf_shade<false>, k_wf_init<false>, k_wf_resolve<false>};
  }
};

// Overlapped bounces: bounce k's shadow stage depends on its nearest-hit stage only, its
// shading stage on its shadow stage, and bounce k+1's nearest-hit stage on bounce k's
// nearest-hit stage only (its rays and counters).  So the nearest-hit stages run in order
// on the render stream, the shadow stages on `side` and the shading stages on `shade`, each
// as soon as its inputs are there; the stages fill each other's tails of straggling warps.
// Bounces alternate between two sets of hit records, shadow masks and shadow queues (set
// k & 1; `hits1` etc. is the second), and the nearest-hit stage of bounce k+2, which reuses
// bounce k's set, waits for bounce k's shading (ev_shaded[k]), which followed its shadow
// stage.  side == nullptr: one stream, strictly in order.
struct Overlap {
  cudaStream_t side = nullptr;
  cudaStream_t shade = nullptr;
  cudaEvent_t* ev_closest = nullptr;  // [kMaxBounces]
  cudaEvent_t* ev_any = nullptr;      // [kMaxBounces]
  cudaEvent_t* ev_shaded = nullptr;   // [kMaxBounces]
  HitQ* hits1 = nullptr;
  uint32_t* masks1 = nullptr;
  ShadowQ* sq1 = nullptr;
};

template <int SH>
eos_status launch_sequence(cudaStream_t st, int num_sms, const WfArgs& base, const Chunk* chunks, int n_chunks,
                           int depth, int block, int grid_closest, int grid_any, int* ctr, size_t smem,
                           bool small_stack, bool tree, StageTimer tm, const Overlap& ov, uint32_t& launches) {
  const int grid_lin = num_sms * 8;
  const StageKernels<SH> K = StageKernels<SH>::get(small_stack, tree);
  const bool split = ov.side != nullptr && !tm.on;  // stage timing times the stages one by one
  cudaStream_t st2 = split ? ov.side : st, st3 = split ? ov.shade : st;
  for (int ci = 0; ci < n_chunks; ++ci) {
    const Chunk& c = chunks[ci];
    WfArgs A = base;
    A.c0 = c.c0;
    A.n_chunk = c.n;
    EOS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int) * kCtr * (depth + 1), st));
    if (!A.init_in_primary) {
      EOS_TRY(tm.begin());
      K.init<<<grid_lin, 256, 0, st>>>(A);
      EOS_TRY(tm.end(2));
      ++launches;
    }
    const RayQ* rin = nullptr;
    RayQ* bufs[2] = {base.rout, const_cast<RayQ*>(base.rin)};
    for (int k = 0; k <= depth; ++k) {
      A.k = k;
      A.rin = rin;
      A.rout = bufs[k & 1];
      const bool second = split && (k & 1);
      A.hits = second ? ov.hits1 : base.hits;
      A.masks = second ? ov.masks1 : base.masks;
      A.sq = second ? ov.sq1 : base.sq;
      if (split && k >= 2) EOS_CUDA(cudaStreamWaitEvent(st, ov.ev_shaded[k - 2], 0));
      EOS_TRY(tm.begin());
      (k == 0 ? K.closest_primary : K.closest)<<<grid_closest, block, smem, st>>>(A);
      EOS_TRY(tm.end(0));
      if (split) {
        EOS_CUDA(cudaEventRecord(ov.ev_closest[k], st));
        EOS_CUDA(cudaStreamWaitEvent(st2, ov.ev_closest[k], 0));
      }
      EOS_TRY(tm.begin());
      K.any<<<grid_any, block, smem, st2>>>(A);
      EOS_TRY(tm.end(1));
      if (split) {
        EOS_CUDA(cudaEventRecord(ov.ev_any[k], st2));
        EOS_CUDA(cudaStreamWaitEvent(st3, ov.ev_any[k], 0));
      }
      EOS_TRY(tm.begin());
      K.shade<<<grid_lin, 256, 0, st3>>>(A);
      EOS_TRY(tm.end(2));
      if (split) EOS_CUDA(cudaEventRecord(ov.ev_shaded[k], st3));
      launches += 3;
      rin = A.rout;
    }
    // both side streams end with this chunk's last bounce (each ran its stages in order)
    // and join the render stream
    if (split) {
      EOS_CUDA(cudaStreamWaitEvent(st, ov.ev_any[depth], 0));
      EOS_CUDA(cudaStreamWaitEvent(st, ov.ev_shaded[depth], 0));
    }
    if (A.resolve) {
      EOS_TRY(tm.begin());
      K.resolve<<<grid_lin, 256, 0, st>>>(A);
      EOS_TRY(tm.end(2));
      ++launches;
    }
  }
  EOS_CUDA(cudaGetLastError());
  return EOS_OK;
}

// Device job record of one view (tiled, padded path count).  tree_records: paths_out holds
// tree-form records (EOS_FLAG_TREE_RECORDS).
void fill_job(const eos_job& J, long long path_off, bool tree_records, bool aa_grid, DevJob& d) {
  memset(&d, 0, sizeof d);
  d.s = J.scene->dev;
  for (int k = 0; k < 3; ++k) {
    d.cam[k] = J.camera.position[k];
    d.cam[3 + k] = J.camera.view[k];
    d.cam[6 + k] = J.camera.right[k];
    d.cam[9 + k] = J.camera.up[k];
  }
  d.w = J.camera.width;
  d.h = J.camera.height;
  d.trace_depth = J.trace_depth;
  d.spp = J.spp;
  d.off = J.pixel_offset;
  d.seed = J.jitter_seed;
  d.grid = aa_grid ? aa_grid_side(J.spp) : 0;
  d.rgb = J.rgb_out;
  d.rgba8 = J.rgba8_out;
  d.paths = tree_records ? nullptr : J.paths_out;
  d.tree = tree_records ? reinterpret_cast<eos_tree_node*>(J.paths_out) : nullptr;
  d.tree_nn = EOS_TREE_NODES(J.trace_depth);
  d.y0 = J.row_end > 0 ? J.row_begin : 0;
  d.rows = J.row_end > 0 ? J.row_end - J.row_begin : d.h;
  d.tiles_x = (d.w + kTileW - 1) / kTileW;
  long long tiles_y = (d.rows + kTileH - 1) / kTileH;
  d.n_paths = (long long)d.tiles_x * tiles_y * 32 * d.spp;
  d.path_off = path_off;
}

struct LaunchConfig {
  int block, sh, qchunk, grid_c, grid_a;
  bool small_stack;  // test limit: 8-entry traversal stacks (chain mode)
  bool tree;         // ray-tree mode
  size_t smem;
};

template <int SH>
void configure(LaunchConfig& c, int num_sms) {
  const StageKernels<SH> K = StageKernels<SH>::get(c.small_stack, c.tree);
  if (c.smem > 48 * 1024) {  // opt in to more than the default 48 KB of dynamic shared memory
    cudaFuncSetAttribute(K.closest_primary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
    cudaFuncSetAttribute(K.closest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
    cudaFuncSetAttribute(K.any, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
  }
  int occ_c = 0, occ_a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, K.closest, c.block, c.smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, K.any, c.block, c.smem);
  c.grid_c = num_sms * std::max(1, occ_c);
  c.grid_a = num_sms * std::max(1, occ_a);
}

LaunchConfig launch_config(const eos_render_params& p, int num_sms, bool small_stack, bool tree) {
  LaunchConfig c;
  c.block = p.block_size > 0 ? std::min(512, std::max(32, (p.block_size / 32) * 32)) : 128;
  c.sh = p.stack_depth <= 0 ? 16 : (p.stack_depth <= 8 ? 8 : (p.stack_depth <= 16 ? 16 : 32));
  c.qchunk = p.queue_chunk > 0 ? std::max(32, (p.queue_chunk / 32) * 32) : 64;
  c.tree = tree;
  c.small_stack = small_stack && !tree;
  if (c.small_stack) c.sh = 8;
  c.smem = (size_t)c.sh * c.block * sizeof(uint2);
  if (c.sh == 8) configure<8>(c, num_sms);
  else if (c.sh == 16) configure<16>(c, num_sms);
  else configure<32>(c, num_sms);
  return c;
}

eos_status run_sequence(cudaStream_t st, int num_sms, const LaunchConfig& lc, const WfArgs& A, const Chunk* chunks,
                        int n_chunks, int depth, StageTimer tm, const Overlap& ov, uint32_t& launches) {
  if (lc.sh == 8)
    return launch_sequence<8>(st, num_sms, A, chunks, n_chunks, depth, lc.block, lc.grid_c, lc.grid_a, A.ctr, lc.smem,
                              lc.small_stack, lc.tree, tm, ov, launches);
  if (lc.sh == 16)
    return launch_sequence<16>(st, num_sms, A, chunks, n_chunks, depth, lc.block, lc.grid_c, lc.grid_a, A.ctr,
                               lc.smem, false, lc.tree, tm, ov, launches);
  return launch_sequence<32>(st, num_sms, A, chunks, n_chunks, depth, lc.block, lc.grid_c, lc.grid_a, A.ctr, lc.smem,
                             false, lc.tree, tm, ov, launches);
}

}  // namespace

eos_status render_wavefront(eos_ctx* ctx, const eos_job* jobs, uint32_t n_jobs, const eos_render_params& p,
                            bool use_graph) {
  // host job table + chunk plan
  std::vector<DevJob> dj(n_jobs);
  long long total = 0;
  int depth = 0, max_lights = 0;
  std::vector<Chunk> chunks;
  const bool tree_records = (p.flags & EOS_FLAG_TREE_RECORDS) != 0;
  bool tree = tree_records;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    depth = std::max(depth, jobs[j].trace_depth);
    max_lights = std::max(max_lights, (int)jobs[j].scene->dev.n_lights);
    tree = tree || jobs[j].scene->branching;
  }
  // Per path: rays per bounce (1, or up to 2^depth in tree mode) x (two ray queues, two
  // sets of hit record, mask and shadow queue: Overlap) + accumulators (one per bounce, or
  // per tree node).
  const long long width = tree ? 1ll << depth : 1;
  const int nn = EOS_TREE_NODES(depth);
  const long long per_path =
      width * (2ll * 32 + 2 * (32 + 4 + 32ll * std::max(1, max_lights))) + 16ll * (tree ? nn : depth + 1);
  const long long chunk_paths = std::max(1ll << 16, std::min(kChunkPathsMax, kQueueBudget / per_path));
  for (uint32_t j = 0; j < n_jobs; ++j) {
    DevJob& d = dj[j];
    fill_job(jobs[j], total, tree_records, (p.flags & EOS_FLAG_AA_GRID) != 0, d);
    // chunks aligned to whole pixels of this job
    long long unit = 32ll * d.spp;
    long long per = std::max(unit, (chunk_paths / unit) * unit);
    for (long long s = 0; s < d.n_paths; s += per) chunks.push_back({total + s, (int)std::min(per, d.n_paths - s)});
    total += d.n_paths;
  }
  // merge small consecutive chunks (many small views share one pass)
  std::vector<Chunk> merged;
  for (const Chunk& c : chunks) {
    if (!merged.empty() && merged.back().c0 + merged.back().n == c.c0 && merged.back().n + (long long)c.n <= chunk_paths)
      merged.back().n += c.n;
    else
      merged.push_back(c);
  }
  // Lanes: the paths of a large pass are split in kLanes parts (at whole pixels) that run
  // at the same time, each on its own streams and buffers, so that one part's start and its
  // tails of straggling warps overlap the other parts' busy stages.
  static_assert(kLanes >= 1 && kLanes <= eos_ctx::kWfLanes, "lane count");
  const bool timing = (p.flags & EOS_FLAG_STAGE_TIMING) != 0;
  long long biggest = 0;
  for (const Chunk& c : merged) biggest = std::max<long long>(biggest, c.n);
  std::vector<Chunk> lane_chunks[kLanes];
  if (timing || depth == 0 || !use_graph || biggest < kLaneSplitMin) {
    lane_chunks[0] = merged;
  } else {
    for (const Chunk& c : merged) {
      std::vector<long long> cuts = {c.c0};
      for (int part = 1; part < kLanes; ++part) {
        const long long at = c.c0 + (long long)c.n * part / kLanes;
        int j = 0;  // the job holding path `at`
        for (int lo = 0, hi = (int)n_jobs - 1; lo <= hi;) {
          const int m = (lo + hi) / 2;
          if (dj[m].path_off <= at) {
            j = m;
            lo = m + 1;
          } else {
            hi = m - 1;
          }
        }
        const long long unit = 32ll * dj[j].spp;
        const long long cut = dj[j].path_off + ((at - dj[j].path_off) / unit) * unit;
        if (cut > cuts.back() && cut < c.c0 + c.n) cuts.push_back(cut);
      }
      cuts.push_back(c.c0 + c.n);
      for (size_t l = 0; l + 1 < cuts.size(); ++l) lane_chunks[l].push_back({cuts[l], (int)(cuts[l + 1] - cuts[l])});
    }
  }
  int n_lanes = 1;
  while (n_lanes < kLanes && !lane_chunks[n_lanes].empty()) ++n_lanes;

  eos_status es = EOS_OK;
  DevJob* d_jobs = (DevJob*)scratch(ctx, "wf.jobs", sizeof(DevJob) * n_jobs, &es);
  const eos_limits& lim = ctx->limits;
  const LaunchConfig lc = launch_config(p, ctx->num_sms, lim.small_stack != 0, tree);
  const int block = lc.block, sh = lc.sh, qchunk = lc.qchunk;

  WfArgs A[kLanes];
  Overlap ov[kLanes];
  std::vector<long long> key = {(long long)n_jobs, depth, max_lights, block, sh, qchunk, (long long)lc.small_stack,
                                (long long)lc.tree, n_lanes, (long long)(size_t)d_jobs};
  for (int l = 0; l < n_lanes; ++l) {
    int max_chunk = 0;
    for (const Chunk& c : lane_chunks[l]) max_chunk = std::max(max_chunk, c.n);
    const std::string tag = l == 0 ? std::string("wf.") : "wf." + std::to_string(l) + ".";
    auto buf = [&](const char* name, size_t bytes) { return scratch(ctx, (tag + name).c_str(), bytes, &es); };
    const size_t cap_q = (size_t)max_chunk * width;  // rays of one bounce
    const size_t cap_s = cap_q * std::max(1, max_lights);
    WfArgs& a = A[l];
    memset(&a, 0, sizeof a);
    a.jobs = d_jobs;
    a.n_jobs = (int)n_jobs;
    a.depth = depth;
    a.rout = (RayQ*)buf("r0", sizeof(RayQ) * cap_q);
    a.rin = (RayQ*)buf("r1", sizeof(RayQ) * cap_q);
    a.hits = (HitQ*)buf("hits", sizeof(HitQ) * cap_q);
    a.masks = (uint32_t*)buf("masks", 4 * cap_q);
    a.sq = (ShadowQ*)buf("sq", sizeof(ShadowQ) * cap_s);
    a.acc = (float4*)buf("acc", 16 * (size_t)max_chunk * (tree ? nn : depth + 1));
    a.ctr = (int*)buf("ctr", sizeof(int) * kCtr * (depth + 1));
    a.cap_r = (int)std::min<size_t>(cap_q, 0x7fffffff);
    a.cap_s = (int)std::min<size_t>(cap_s, 0x7fffffff);
    a.nn = nn;
    if (lim.queue_entries > 0) {
      a.cap_r = std::min(a.cap_r, (int)lim.queue_entries);
      a.cap_s = std::min(a.cap_s, (int)lim.queue_entries);
    }
    a.qchunk = qchunk;
    a.work_limit = lim.work_budget > 0 ? lim.work_budget : 0x7fffffff;
    a.init_in_primary = !tree && lim.work_budget <= 0;  // a budget leaves primary entries untraced
    a.resolve = !a.init_in_primary;
    for (uint32_t j = 0; j < n_jobs; ++j) a.resolve |= dj[j].spp > 1 || dj[j].grid > 0;
    a.err = ctx->d_err;
    a.counts = ctx->d_counts;
    eos_ctx::WfLane& ln = ctx->wf_lane[l];
    if (depth > 0 && !timing) {  // the second set of per-bounce buffers, the side streams and their events
      ov[l].hits1 = (HitQ*)buf("hits1", sizeof(HitQ) * cap_q);
      ov[l].masks1 = (uint32_t*)buf("masks1", 4 * cap_q);
      ov[l].sq1 = (ShadowQ*)buf("sq1", sizeof(ShadowQ) * cap_s);
      if (l > 0 && !ln.main) EOS_CUDA(cudaStreamCreateWithFlags(&ln.main, cudaStreamNonBlocking));
      if (!ln.side) EOS_CUDA(cudaStreamCreateWithFlags(&ln.side, cudaStreamNonBlocking));
      if (!ln.shade) EOS_CUDA(cudaStreamCreateWithFlags(&ln.shade, cudaStreamNonBlocking));
      for (int k = 0; k < kMaxBounces; ++k) {
        if (!ln.ev_closest[k]) EOS_CUDA(cudaEventCreateWithFlags(&ln.ev_closest[k], cudaEventDisableTiming));
        if (!ln.ev_any[k]) EOS_CUDA(cudaEventCreateWithFlags(&ln.ev_any[k], cudaEventDisableTiming));
        if (!ln.ev_shaded[k]) EOS_CUDA(cudaEventCreateWithFlags(&ln.ev_shaded[k], cudaEventDisableTiming));
      }
      ov[l].side = ln.side;
      ov[l].shade = ln.shade;
      ov[l].ev_closest = ln.ev_closest;
      ov[l].ev_any = ln.ev_any;
      ov[l].ev_shaded = ln.ev_shaded;
    }
    if (es != EOS_OK) return es;
    for (long long v : {(long long)a.cap_r, (long long)a.cap_s, (long long)a.work_limit, (long long)a.init_in_primary,
                        (long long)a.resolve, (long long)(size_t)a.rout, (long long)(size_t)a.rin,
                        (long long)(size_t)a.hits, (long long)(size_t)a.masks, (long long)(size_t)a.sq,
                        (long long)(size_t)a.acc, (long long)(size_t)a.ctr, (long long)(size_t)ov[l].hits1,
                        (long long)(size_t)ov[l].masks1, (long long)(size_t)ov[l].sq1})
      key.push_back(v);
    for (const Chunk& c : lane_chunks[l]) {
      key.push_back(c.c0);
      key.push_back(c.n);
    }
  }
  if (n_lanes > 1 && !ctx->ev_fork) EOS_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  for (int l = 1; l < n_lanes; ++l)
    if (!ctx->ev_join[l]) EOS_CUDA(cudaEventCreateWithFlags(&ctx->ev_join[l], cudaEventDisableTiming));
  EOS_CUDA(cudaMemcpyAsync(d_jobs, dj.data(), sizeof(DevJob) * n_jobs, cudaMemcpyHostToDevice, ctx->stream));

  uint32_t launches = 0;
  StageTimer tm{!use_graph && timing, ctx->stream, ctx->ev0, ctx->ev1, ctx->stage_ms};
  auto run = [&]() -> eos_status {
    // lanes 1.. fork from the context's stream and join it at the end
    if (n_lanes > 1) EOS_CUDA(cudaEventRecord(ctx->ev_fork, ctx->stream));
    for (int l = 1; l < n_lanes; ++l) EOS_CUDA(cudaStreamWaitEvent(ctx->wf_lane[l].main, ctx->ev_fork, 0));
    for (int l = 0; l < n_lanes; ++l) {
      cudaStream_t s_l = l == 0 ? ctx->stream : ctx->wf_lane[l].main;
      EOS_TRY(run_sequence(s_l, ctx->num_sms, lc, A[l], lane_chunks[l].data(), (int)lane_chunks[l].size(), depth, tm,
                           ov[l], launches));
    }
    for (int l = 1; l < n_lanes; ++l) {
      EOS_CUDA(cudaEventRecord(ctx->ev_join[l], ctx->wf_lane[l].main));
      EOS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_join[l], 0));
    }
    return EOS_OK;
  };
  if (!use_graph) {
    eos_status rs = run();
    ctx->launches += launches;
    return rs;
  }

  // graph cache: the sequence depends on the lanes' chunk plans, depth, buffers and tuning only
  for (auto& g : ctx->graphs)
    if (g->key == key) {
      EOS_CUDA(cudaGraphLaunch(g->exec, ctx->stream));
      ctx->launches += g->launches;
      return EOS_OK;
    }
  cudaGraph_t graph = nullptr;
  EOS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  eos_status rs = run();
  cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
  if (rs != EOS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rs;
  }
  EOS_CUDA(ce);
  auto bg = std::make_unique<eos_ctx::BatchGraph>();
  bg->key = key;
  bg->launches = launches;
  cudaError_t ie = cudaGraphInstantiate(&bg->exec, graph, 0);
  cudaGraphDestroy(graph);
  EOS_CUDA(ie);
  EOS_CUDA(cudaGraphLaunch(bg->exec, ctx->stream));
  ctx->launches += launches;
  if (ctx->graphs.size() >= 8) ctx->graphs.erase(ctx->graphs.begin());
  ctx->graphs.push_back(std::move(bg));
  return EOS_OK;
}

}  // namespace eos

// ---------------------------------------------------------------------------------
// Allocation-free render (eos_render_noalloc).
//
// For callers that must not allocate device memory at render time: code running inside
// another framework's memory pool or allocator, real-time loops that forbid allocation
// after start-up, or processes that hand all device memory to another owner.  The
// wavefront's queues live in one fixed, file-scope device array instead of context
// scratch; the caller passes the scene, the camera and device output buffers.
//
// Capacity: kNoAllocMaxPaths padded paths (8x4-pixel tiles x spp; 16,384 = 128x128 at
// 1 spp) and kNoAllocMaxLights lights.  The array (about 7.6 MB) is held on every GPU that
// loads this library until the process exits.  Every call shares it and it keeps the last
// call's contents, so calls that overlap on the GPU (two streams, two threads) race; the
// counters, error word and colour accumulators are cleared at the start of each call.
// ---------------------------------------------------------------------------------
namespace eos {
namespace {

constexpr int kNoAllocMaxPaths = EOS_NOALLOC_MAX_PATHS;
constexpr int kNoAllocMaxLights = EOS_NOALLOC_MAX_LIGHTS;
constexpr size_t kNaJob = 0;
constexpr size_t kNaCtr = 256;
constexpr size_t kNaErr = 512;
constexpr size_t kNaCounts = 768;
constexpr size_t kNaR0 = 1024;
constexpr size_t kNaR1 = kNaR0 + sizeof(RayQ) * (size_t)kNoAllocMaxPaths;
constexpr size_t kNaHits = kNaR1 + sizeof(RayQ) * (size_t)kNoAllocMaxPaths;
constexpr size_t kNaMasks = kNaHits + sizeof(HitQ) * (size_t)kNoAllocMaxPaths;
constexpr size_t kNaSq = kNaMasks + 4 * (size_t)kNoAllocMaxPaths;
constexpr size_t kNaAcc = kNaSq + sizeof(ShadowQ) * (size_t)kNoAllocMaxPaths * kNoAllocMaxLights;
constexpr size_t kNaBytes = kNaAcc + sizeof(float4) * (size_t)kNoAllocMaxPaths * kMaxBounces;
static_assert(sizeof(DevJob) <= kNaCtr - kNaJob, "job record does not fit its slot");
static_assert(sizeof(int) * kCtr * kMaxBounces <= kNaErr - kNaCtr, "counters do not fit their slot");
static_assert(sizeof(unsigned long long) * kCounters <= kNaR0 - kNaCounts, "ray counters do not fit their slot");
static_assert(kNaSq % 256 == 0 && kNaAcc % 256 == 0, "queues must stay 256-byte aligned");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// The job record travels as a kernel argument, so no host staging buffer is involved.
__global__ void k_na_put_job(DevJob j, DevJob* dst) { *dst = j; }

// Device address of g_noalloc_scratch per device.  In host code the symbol names a host
// stand-in, not device memory, so the address is looked up once per device, with that
// device current, and cached.
std::mutex g_na_mutex;
unsigned char* g_na_base[64] = {};

eos_status noalloc_base(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 64) return EOS_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_base[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return EOS_ERR_CUDA;
    }
    g_na_base[dev] = (unsigned char*)p;
  }
  *out = g_na_base[dev];
  return EOS_OK;
}

}  // namespace
}  // namespace eos

extern "C" eos_status eos_render_noalloc(const eos_scene* scene, const eos_camera* camera,
                                         const eos_render_params* params, void* stream, float* rgb_out,
                                         eos_path_record* paths_out, eos_stats* stats) {
  using namespace eos;
  if (!scene || !camera || !params || !scene->ctx) return EOS_ERR_INVALID_ARG;
  if (camera->width <= 0 || camera->height <= 0 || camera->width > kNoAllocMaxPaths ||
      camera->height > kNoAllocMaxPaths)
    return EOS_ERR_INVALID_ARG;
  if (params->trace_depth < 0 || params->trace_depth >= EOS_MAX_BOUNCES || params->spp < 1 ||
      params->spp > kNoAllocMaxPaths ||
      (params->flags & ~(EOS_FLAG_STAGE_TIMING | EOS_FLAG_TREE_RECORDS | EOS_FLAG_AA_GRID)))
    return EOS_ERR_INVALID_ARG;
  // the fixed array holds the one-ray-per-bounce queues only
  if ((params->flags & EOS_FLAG_TREE_RECORDS) || scene->branching) return EOS_ERR_UNSUPPORTED;
  if (scene->dev.n_lights > kNoAllocMaxLights) return EOS_ERR_INVALID_ARG;
  if ((rgb_out && !is_device_ptr(rgb_out)) || (paths_out && !is_device_ptr(paths_out))) return EOS_ERR_INVALID_ARG;
  const int dev = scene->ctx->device;
  EOS_CUDA(cudaSetDevice(dev));
  unsigned char* base = nullptr;
  eos_status st = noalloc_base(dev, &base);
  if (st != EOS_OK) return st;
  int num_sms = 0;
  EOS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));

  eos_job J;
  memset(&J, 0, sizeof J);
  J.scene = scene;
  J.camera = *camera;
  J.trace_depth = params->trace_depth;
  J.pixel_offset = params->pixel_offset;
  J.spp = params->spp;
  J.jitter_seed = params->jitter_seed;
  J.rgb_out = rgb_out;
  J.paths_out = paths_out;
  const bool rows_ok = (params->row_begin == 0 && params->row_end == 0) ||
                       (params->row_begin >= 0 && params->row_begin < params->row_end &&
                        params->row_end <= camera->height);
  if (!rows_ok) return EOS_ERR_INVALID_ARG;
  J.row_begin = params->row_begin;
  J.row_end = params->row_end;
  DevJob job;
  if ((params->flags & EOS_FLAG_AA_GRID) && aa_grid_side(params->spp) == 0) return EOS_ERR_INVALID_ARG;
  fill_job(J, 0, false, (params->flags & EOS_FLAG_AA_GRID) != 0, job);
  if (job.n_paths > kNoAllocMaxPaths) return EOS_ERR_INVALID_ARG;  // beyond the fixed scratch capacity

  cudaStream_t s = (cudaStream_t)stream;
  k_na_put_job<<<1, 1, 0, s>>>(job, (DevJob*)(base + kNaJob));
  EOS_CUDA(cudaMemsetAsync(base + kNaErr, 0, sizeof(int), s));
  EOS_CUDA(cudaMemsetAsync(base + kNaCounts, 0, sizeof(unsigned long long) * kCounters, s));

  WfArgs A;
  memset(&A, 0, sizeof A);
  A.jobs = (const DevJob*)(base + kNaJob);
  A.n_jobs = 1;
  A.depth = params->trace_depth;
  A.rin = (const RayQ*)(base + kNaR1);
  A.rout = (RayQ*)(base + kNaR0);
  A.hits = (HitQ*)(base + kNaHits);
  A.masks = (uint32_t*)(base + kNaMasks);
  A.sq = (ShadowQ*)(base + kNaSq);
  A.acc = (float4*)(base + kNaAcc);
  A.ctr = (int*)(base + kNaCtr);
  A.cap_r = kNoAllocMaxPaths;
  A.cap_s = kNoAllocMaxPaths * kNoAllocMaxLights;
  // the scene context's tuning table, as eos_render applies it (the table is read here
  // only; it is changed by eos_ctx_set_tuning calls, which callers serialise with renders)
  const LaunchConfig lc =
      launch_config(with_tuning(scene->ctx, *params, (uint32_t)scene->dev.n_tris), num_sms, false, false);
  A.qchunk = lc.qchunk;
  A.work_limit = 0x7fffffff;
  A.init_in_primary = 1;
  A.resolve = job.spp > 1 || job.grid > 0;
  A.err = (int*)(base + kNaErr);
  A.counts = (unsigned long long*)(base + kNaCounts);
  Chunk ch{0, (int)job.n_paths};
  StageTimer tm{false, s, nullptr, nullptr, nullptr};
  uint32_t launches = 1;
  st = run_sequence(s, num_sms, lc, A, &ch, 1, A.depth, tm, Overlap{}, launches);
  if (st != EOS_OK) return st;

  struct {
    unsigned long long c[kCounters];
    int err;
  } h;
  EOS_CUDA(cudaMemcpyAsync(h.c, base + kNaCounts, sizeof h.c, cudaMemcpyDeviceToHost, s));
  EOS_CUDA(cudaMemcpyAsync(&h.err, base + kNaErr, sizeof(int), cudaMemcpyDeviceToHost, s));
  EOS_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->primary_rays = h.c[kCntPrimary];
    stats->shadow_rays = h.c[kCntShadow];
    stats->secondary_rays = h.c[kCntSecondary];
    stats->nodes_closest = h.c[kCntNodesC];
    stats->tests_closest = h.c[kCntTestsC];
    stats->nodes_shadow = h.c[kCntNodesA];
    stats->tests_shadow = h.c[kCntTestsA];
    stats->shaded_hits = h.c[kCntHits];
    stats->error_flags = h.err;
    stats->kernel_launches = launches;
  }
  return err_to_status(h.err);
}
