// Wavefront renderer: many views of one or several resident scenes through one global
// ray queue, per bounce:
//
//   closest  (persistent)  nearest hit of every ray in R_k; writes a hit record; emits
//                          one shadow ray per light into S_k and the mirror ray into
//                          R_k+1, both compacted with warp ballot / popc and one atomic
//                          per warp
//   any      (persistent)  any-hit of every shadow ray in S_k; blocked -> bit in the hit's
//                          light mask
//   shade                  Phong over the unblocked lights, in light order, per hit
//   resolve                colour fold c_k = phong_k + refl_k c_k+1 per path, sample mean,
//                          RGB / RGBA8 / path records to each job's buffers
//
// The semantics are those of the reference's CPU renderer (src/RayTracer.cpp:268-458),
// identical to the plain renderer (render.cu) bit for bit: the same hits, masks and
// colours.  Persistent kernels take `queue_chunk` rays per warp from a work counter, so
// rays of uneven cost balance across the SMs.  Paths are processed in chunks of at most
// kChunkPaths to bound the queues.  The whole sequence for a batch is captured once as a
// CUDA graph and replayed; the job table is uploaded before each replay.
#include <algorithm>
#include <cstring>
#include <vector>

#include "trace.cuh"

namespace eos {
namespace {

constexpr long long kChunkPaths = 1ll << 21;
constexpr int kTileW = 8, kTileH = 4;  // one warp = 8 x 4 pixels

struct DevJob {
  DevScene s;
  float cam[12];
  int w, h, trace_depth, spp;
  float off;
  uint32_t seed;
  float* rgb;
  uint8_t* rgba8;
  eos_path_record* paths;
  long long path_off;  // first global path index of this job
  long long n_paths;   // tiled, padded path count
  int tiles_x;
  int pad;
};

struct RayQ {
  float4 a;  // origin xyz, path (int)
  float4 b;  // direction xyz, -
};
struct HitQ {
  float4 a;  // P xyz, path (int)
  float4 b;  // N xyz, obj (int; -1 = miss)
};
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
  float4* acc;   // [n_chunk][depth+1] phong rgb, reflectivity
  int* ctr;      // [depth+1][kCtr]
  int cap_r, cap_s;
  int qchunk;
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
__device__ __forceinline__ bool path_pixel(const DevJob& j, long long local, int& x, int& y, int& smp) {
  smp = (int)(local % j.spp);
  long long tp = local / j.spp;
  long long tile = tp >> 5;
  int lane = (int)(tp & 31);
  x = (int)(tile % j.tiles_x) * kTileW + (lane & (kTileW - 1));
  y = (int)(tile / j.tiles_x) * kTileH + (lane >> 3);
  return x < j.w && y < j.h;
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

template <bool PRIMARY, int SH>
__global__ void k_wf_closest(WfArgs A) {
  extern __shared__ uint2 shstack[];
  uint2* shs = shstack + threadIdx.x;
  const int stride = blockDim.x;
  int* ctr = A.ctr + A.k * kCtr;
  const int n_in = PRIMARY ? A.n_chunk : min(ctr[1 - kCtr], A.cap_r);  // mirror rays of bounce k-1
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
      bool hit = false, refl = false;
      int path = -1, jb = 0, obj = -1;
      f3 o = mk3(0, 0, 0), d = mk3(0, 0, 1), P = o, N = o;
      if (valid) {
        if (PRIMARY) {
          long long gp = A.c0 + i;
          jb = find_job(A.jobs, A.n_jobs, gp);
          const DevJob& J = A.jobs[jb];
          int x, y, smp;
          if (path_pixel(J, gp - J.path_off, x, y, smp)) {
            float ox, oy;
            sample_offset((uint32_t)(y * J.w + x), smp, J.spp, J.seed, J.off, ox, oy);
            d = primary_direction(J.cam, J.w, J.h, x, y, ox, oy);
            o = mk3(J.cam[0], J.cam[1], J.cam[2]);
            path = i;
          } else {
            valid = false;
          }
        } else {
          RayQ r = A.rin[i];
          o = mk3(r.a.x, r.a.y, r.a.z);
          d = mk3(r.b.x, r.b.y, r.b.z);
          path = __float_as_int(r.a.w);
          jb = find_job(A.jobs, A.n_jobs, A.c0 + path);
        }
      }
      const DevJob& J = A.jobs[jb];
      if (valid) {
        ++nrays;
        Hit h = closest_hit<SH>(J.s, o, d, shs, stride, A.err);
        nodes += h.nodes;
        tests += h.tests;
        hit = h.pos >= 0;
        nhits += hit;
        if (J.paths) {
          int x, y, smp;
          path_pixel(J, A.c0 + path - J.path_off, x, y, smp);
          J.paths[((size_t)y * J.w + x) * J.spp + smp].hit[A.k] = hit ? h.id : EOS_HIT_NONE;
        }
        if (hit) {
          hit_geometry(J.s, o, d, h, P, N, obj);
          refl = J.s.mats[8 * obj + 7] > 0.0f && A.k < J.trace_depth;
        }
        HitQ hq;
        hq.a = make_float4(P.x, P.y, P.z, __int_as_float(path));
        hq.b = make_float4(N.x, N.y, N.z, __int_as_float(hit ? obj : -1));
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
        bool fits = wbase + total <= A.cap_s;
        if (!fits && lane == 0) atomicOr(A.err, kErrQueue);
        int prefix = 0;
        for (int l = 0; l < maxl; ++l) {
          uint32_t bl = __ballot_sync(0xffffffffu, l < nl);
          if (l < nl && fits) {
            const float* lp = J.s.lights + 6 * l;
            f3 sd = norm3(sub3(mk3(lp[0], lp[1], lp[2]), P));
            f3 so = add3(P, scale3(kRayEps, sd));
            ShadowQ s;
            s.a = make_float4(so.x, so.y, so.z, __int_as_float(i));
            s.b = make_float4(sd.x, sd.y, sd.z, __int_as_float((jb << 5) | l));
            A.sq[wbase + prefix + __popc(bl & lanemask_lt())] = s;
          }
          prefix += __popc(bl);
        }
        nshadow += nl;
      }
      // mirror rays
      uint32_t rb = __ballot_sync(0xffffffffu, refl);
      if (rb) {
        int rbase = 0;
        if (lane == 0) rbase = atomicAdd(&ctr[1], __popc(rb));
        rbase = __shfl_sync(0xffffffffu, rbase, 0);
        if (refl) {
          int pos = rbase + __popc(rb & lanemask_lt());
          if (pos >= A.cap_r) {
            atomicOr(A.err, kErrQueue);
          } else {
            f3 rd = norm3(reflect3(d, N));
            f3 ro = add3(P, scale3(kRayEps, rd));
            RayQ r;
            r.a = make_float4(ro.x, ro.y, ro.z, __int_as_float(path));
            r.b = make_float4(rd.x, rd.y, rd.z, 0.0f);
            A.rout[pos] = r;
          }
        }
      }
    }
  }
  warp_add_count(&A.counts[A.k == 0 ? kCntPrimary : kCntSecondary], nrays);
  warp_add_count(&A.counts[kCntShadow], nshadow);
  warp_add_count(&A.counts[kCntHits], nhits);
  warp_add_count(&A.counts[kCntNodesC], nodes);
  warp_add_count(&A.counts[kCntTestsC], tests);
}

template <int SH>
__global__ void k_wf_any(WfArgs A) {
  extern __shared__ uint2 shstack[];
  uint2* shs = shstack + threadIdx.x;
  const int stride = blockDim.x;
  int* ctr = A.ctr + A.k * kCtr;
  const int n = min(ctr[2], A.cap_s);
  const int lane = threadIdx.x & 31;
  unsigned long long nodes = 0, tests = 0;
  for (;;) {
    int start = grab(&ctr[4], A.qchunk);
    if (start >= n) break;
    int end = min(start + A.qchunk, n);
    for (int i = start + lane; i < end; i += 32) {
      ShadowQ s = A.sq[i];
      int hi = __float_as_int(s.a.w);
      int key = __float_as_int(s.b.w);
      const DevJob& J = A.jobs[key >> 5];
      AnyResult ar = any_hit<SH>(J.s, mk3(s.a.x, s.a.y, s.a.z), mk3(s.b.x, s.b.y, s.b.z), shs, stride, A.err);
      nodes += ar.nodes;
      tests += ar.tests;
      if (ar.hit) atomicOr(&A.masks[hi], 1u << (key & 31));
    }
  }
  warp_add_count(&A.counts[kCntNodesA], nodes);
  warp_add_count(&A.counts[kCntTestsA], tests);
}

__global__ void k_wf_shade(WfArgs A) {
  int* ctr = A.ctr + A.k * kCtr;
  const int n = A.k == 0 ? A.n_chunk : min(ctr[1 - kCtr], A.cap_r);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    HitQ hq = A.hits[i];
    int path = __float_as_int(hq.a.w);
    int obj = __float_as_int(hq.b.w);
    if (path < 0) continue;  // tile padding (primary only)
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, A.c0 + path)];
    if (obj < 0) continue;
    f3 P = mk3(hq.a.x, hq.a.y, hq.a.z), N = mk3(hq.b.x, hq.b.y, hq.b.z);
    f3 cam = mk3(J.cam[0], J.cam[1], J.cam[2]);
    const float* m = J.s.mats + 8 * obj;
    uint32_t mask = A.masks[i];
    f3 acc = mk3(0, 0, 0);
    for (int l = 0; l < J.s.n_lights; ++l)
      if (!(mask & (1u << l))) acc = add3(acc, phong_light(m, J.s.lights + 6 * l, P, N, cam));
    float r = m[7] > 0.0f ? m[7] : 0.0f;
    A.acc[(size_t)path * (A.depth + 1) + A.k] = make_float4(acc.x, acc.y, acc.z, r);
    if (J.paths) {
      int x, y, smp;
      path_pixel(J, A.c0 + path - J.path_off, x, y, smp);
      J.paths[((size_t)y * J.w + x) * J.spp + smp].shadow[A.k] = mask;
    }
  }
}

// Marks every padding entry of the primary hit queue and clears path records / acc.
__global__ void k_wf_init(WfArgs A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_chunk; i += gridDim.x * blockDim.x) {
    long long gp = A.c0 + i;
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, gp)];
    for (int k = 0; k <= A.depth; ++k) A.acc[(size_t)i * (A.depth + 1) + k] = make_float4(0, 0, 0, 0);
    HitQ hq;
    hq.a = make_float4(0, 0, 0, __int_as_float(-1));
    hq.b = make_float4(0, 0, 0, __int_as_float(-1));
    A.hits[i] = hq;
    int x, y, smp;
    if (J.paths && path_pixel(J, gp - J.path_off, x, y, smp)) {
      eos_path_record rec;
      for (int k = 0; k < kMaxBounces; ++k) {
        rec.hit[k] = EOS_HIT_UNTRACED;
        rec.shadow[k] = 0u;
      }
      J.paths[((size_t)y * J.w + x) * J.spp + smp] = rec;
    }
  }
}

__global__ void k_wf_resolve(WfArgs A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_chunk; i += gridDim.x * blockDim.x) {
    long long gp = A.c0 + i;
    const DevJob& J = A.jobs[find_job(A.jobs, A.n_jobs, gp)];
    int x, y, smp;
    if (!path_pixel(J, gp - J.path_off, x, y, smp) || smp != 0) continue;
    f3 sum = mk3(0, 0, 0);
    for (int s = 0; s < J.spp; ++s) {
      const float4* a = A.acc + (size_t)(i + s) * (A.depth + 1);
      f3 c = mk3(0, 0, 0);
      for (int k = A.depth; k >= 0; --k) {
        float4 e = a[k];
        c = add3(mk3(e.x, e.y, e.z), scale3(e.w, c));
      }
      sum = add3(sum, c);
    }
    if (J.spp > 1) sum = scale3(1.0f / (float)J.spp, sum);
    size_t pix = (size_t)y * J.w + x;
    if (J.rgb) {
      J.rgb[3 * pix] = sum.x;
      J.rgb[3 * pix + 1] = sum.y;
      J.rgb[3 * pix + 2] = sum.z;
    }
    if (J.rgba8)
      reinterpret_cast<uchar4*>(J.rgba8)[pix] = make_uchar4(quantize(sum.x), quantize(sum.y), quantize(sum.z), 255);
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
  eos_ctx* ctx;
  bool on;
  eos_status begin() { return on ? (cudaEventRecord(ctx->ev0, ctx->stream) == cudaSuccess ? EOS_OK : EOS_ERR_CUDA) : EOS_OK; }
  eos_status end(int stage) {
    if (!on) return EOS_OK;
    EOS_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    EOS_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0.0f;
    EOS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->stage_ms[stage] += ms;
    return EOS_OK;
  }
};

#define EOS_TRY(x)                  \
  do {                              \
    eos_status s_ = (x);            \
    if (s_ != EOS_OK) return s_;    \
  } while (0)

template <int SH>
eos_status launch_sequence(eos_ctx* ctx, const WfArgs& base, const std::vector<Chunk>& chunks, int depth,
                           int block, int grid_closest, int grid_any, int* ctr, size_t smem, StageTimer tm,
                           uint32_t& launches) {
  cudaStream_t st = ctx->stream;
  const int grid_lin = ctx->num_sms * 8;
  for (const Chunk& c : chunks) {
    WfArgs A = base;
    A.c0 = c.c0;
    A.n_chunk = c.n;
    EOS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int) * kCtr * (depth + 1), st));
    EOS_TRY(tm.begin());
    k_wf_init<<<grid_lin, 256, 0, st>>>(A);
    EOS_TRY(tm.end(2));
    ++launches;
    const RayQ* rin = nullptr;
    RayQ* bufs[2] = {base.rout, const_cast<RayQ*>(base.rin)};
    for (int k = 0; k <= depth; ++k) {
      A.k = k;
      A.rin = rin;
      A.rout = bufs[k & 1];
      EOS_TRY(tm.begin());
      if (k == 0)
        k_wf_closest<true, SH><<<grid_closest, block, smem, st>>>(A);
      else
        k_wf_closest<false, SH><<<grid_closest, block, smem, st>>>(A);
      EOS_TRY(tm.end(0));
      EOS_TRY(tm.begin());
      k_wf_any<SH><<<grid_any, block, smem, st>>>(A);
      EOS_TRY(tm.end(1));
      EOS_TRY(tm.begin());
      k_wf_shade<<<grid_lin, 256, 0, st>>>(A);
      EOS_TRY(tm.end(2));
      launches += 3;
      rin = A.rout;
    }
    EOS_TRY(tm.begin());
    k_wf_resolve<<<grid_lin, 256, 0, st>>>(A);
    EOS_TRY(tm.end(2));
    ++launches;
  }
  EOS_CUDA(cudaGetLastError());
  return EOS_OK;
}

}  // namespace

eos_status render_wavefront(eos_ctx* ctx, const eos_job* jobs, uint32_t n_jobs, const eos_render_params& p,
                            bool use_graph) {
  // host job table + chunk plan
  std::vector<DevJob> dj(n_jobs);
  long long total = 0;
  int depth = 0, max_lights = 0;
  std::vector<Chunk> chunks;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const eos_job& J = jobs[j];
    DevJob& d = dj[j];
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
    d.rgb = J.rgb_out;
    d.rgba8 = J.rgba8_out;
    d.paths = J.paths_out;
    d.tiles_x = (d.w + kTileW - 1) / kTileW;
    long long tiles_y = (d.h + kTileH - 1) / kTileH;
    d.n_paths = (long long)d.tiles_x * tiles_y * 32 * d.spp;
    d.path_off = total;
    // chunks aligned to whole pixels of this job
    long long unit = 32ll * d.spp;
    long long per = std::max(unit, (kChunkPaths / unit) * unit);
    for (long long s = 0; s < d.n_paths; s += per) chunks.push_back({total + s, (int)std::min(per, d.n_paths - s)});
    total += d.n_paths;
    depth = std::max(depth, J.trace_depth);
    max_lights = std::max(max_lights, d.s.n_lights);
  }
  // merge small consecutive chunks (many small views share one pass)
  std::vector<Chunk> merged;
  for (const Chunk& c : chunks) {
    if (!merged.empty() && merged.back().c0 + merged.back().n == c.c0 && merged.back().n + (long long)c.n <= kChunkPaths)
      merged.back().n += c.n;
    else
      merged.push_back(c);
  }
  int max_chunk = 0;
  for (const Chunk& c : merged) max_chunk = std::max(max_chunk, c.n);

  eos_status es = EOS_OK;
  DevJob* d_jobs = (DevJob*)scratch(ctx, "wf.jobs", sizeof(DevJob) * n_jobs, &es);
  RayQ* r0 = (RayQ*)scratch(ctx, "wf.r0", sizeof(RayQ) * (size_t)max_chunk, &es);
  RayQ* r1 = (RayQ*)scratch(ctx, "wf.r1", sizeof(RayQ) * (size_t)max_chunk, &es);
  HitQ* hits = (HitQ*)scratch(ctx, "wf.hits", sizeof(HitQ) * (size_t)max_chunk, &es);
  uint32_t* masks = (uint32_t*)scratch(ctx, "wf.masks", 4 * (size_t)max_chunk, &es);
  size_t cap_s = (size_t)max_chunk * std::max(1, max_lights);
  ShadowQ* sq = (ShadowQ*)scratch(ctx, "wf.sq", sizeof(ShadowQ) * cap_s, &es);
  float4* acc = (float4*)scratch(ctx, "wf.acc", 16 * (size_t)max_chunk * (depth + 1), &es);
  int* ctr = (int*)scratch(ctx, "wf.ctr", sizeof(int) * kCtr * (depth + 1), &es);
  if (es != EOS_OK) return es;
  EOS_CUDA(cudaMemcpyAsync(d_jobs, dj.data(), sizeof(DevJob) * n_jobs, cudaMemcpyHostToDevice, ctx->stream));

  const int block = p.block_size > 0 ? std::min(512, std::max(32, (p.block_size / 32) * 32)) : 128;
  const int sh = p.stack_depth <= 0 ? 16 : (p.stack_depth <= 8 ? 8 : (p.stack_depth <= 16 ? 16 : 32));
  const int qchunk = p.queue_chunk > 0 ? std::max(32, (p.queue_chunk / 32) * 32) : 64;
  const size_t smem = (size_t)sh * block * sizeof(uint2);

  WfArgs A;
  memset(&A, 0, sizeof A);
  A.jobs = d_jobs;
  A.n_jobs = (int)n_jobs;
  A.depth = depth;
  A.rin = r1;
  A.rout = r0;
  A.hits = hits;
  A.masks = masks;
  A.sq = sq;
  A.acc = acc;
  A.ctr = ctr;
  A.cap_r = max_chunk;
  A.cap_s = (int)std::min<size_t>(cap_s, 0x7fffffff);
  A.qchunk = qchunk;
  A.err = ctx->d_err;
  A.counts = ctx->d_counts;

  int occ_c = 0, occ_a = 0;
  if (sh == 8) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k_wf_closest<false, 8>, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_wf_any<8>, block, smem);
  } else if (sh == 16) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k_wf_closest<false, 16>, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_wf_any<16>, block, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k_wf_closest<false, 32>, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_wf_any<32>, block, smem);
  }
  const int grid_c = ctx->num_sms * std::max(1, occ_c);
  const int grid_a = ctx->num_sms * std::max(1, occ_a);

  uint32_t launches = 0;
  StageTimer tm{ctx, !use_graph && (p.flags & EOS_FLAG_STAGE_TIMING) != 0};
  auto run = [&]() -> eos_status {
    if (sh == 8) return launch_sequence<8>(ctx, A, merged, depth, block, grid_c, grid_a, ctr, smem, tm, launches);
    if (sh == 16) return launch_sequence<16>(ctx, A, merged, depth, block, grid_c, grid_a, ctr, smem, tm, launches);
    return launch_sequence<32>(ctx, A, merged, depth, block, grid_c, grid_a, ctr, smem, tm, launches);
  };
  if (!use_graph) {
    eos_status rs = run();
    ctx->launches += launches;
    return rs;
  }

  // graph cache: the sequence depends on the chunk plan, depth, buffers and tuning only
  std::vector<long long> key = {(long long)n_jobs, depth, max_lights, block, sh, qchunk, (long long)(size_t)d_jobs,
                                (long long)(size_t)r0, (long long)(size_t)r1, (long long)(size_t)sq,
                                (long long)(size_t)acc};
  for (const Chunk& c : merged) {
    key.push_back(c.c0);
    key.push_back(c.n);
  }
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
