// Plain renderer: one launch per frame, one thread per pixel (all its samples), the whole
// Whitted path of that pixel in the thread: nearest hit, one shadow ray per light, Phong,
// mirror bounce up to trace_depth (src/RayTracer.cpp:99-174,268-458).  This is the
// B200 replacement of the reference's primary-only __rayTrace_MegaKernel
// (src/kernelInvocations.cu:172-310) with the CPU renderer's full semantics.
//
// Also the ray-query kernels behind eos_trace_closest / eos_trace_any.
#include <algorithm>

#include "trace.cuh"

namespace eos {
namespace {

struct PlainParams {
  DevScene s;
  float cam[12];
  int width, height, trace_depth, spp;
  int y0, rows;  // image rows [y0, y0 + rows) are rendered; outputs hold those rows
  float pixel_offset;
  uint32_t jitter_seed;
  float* rgb;
  uint8_t* rgba8;
  int32_t* hit;
  eos_path_record* paths;
  int* err;
  unsigned long long* counts;  // kNumCounts traversal counters
};

// One path: colour with the reference's fold c_k = phong_k + w_k c_{k+1} (fold_colour).
template <int SH>
__device__ f3 trace_path(const PlainParams& P, f3 o, f3 d, int32_t* hits, uint32_t* masks, unsigned* cnt,
                         uint2* shs, int stride) {
  const DevScene& s = P.s;
  f3 phong[kMaxBounces];
  float weight[kMaxBounces];
  int nb = 0;
  const f3 campos = mk3(P.cam[0], P.cam[1], P.cam[2]);
  for (int k = 0; k <= P.trace_depth; ++k) {
    cnt[k == 0 ? kCntPrimary : kCntSecondary]++;
    Hit h = closest_hit<SH>(s, o, d, shs, stride, P.err);
    cnt[kCntNodesC] += h.nodes;
    cnt[kCntTestsC] += h.tests;
    if (h.pos < 0) {
      hits[k] = EOS_HIT_NONE;
      break;
    }
    hits[k] = h.id;
    cnt[kCntHits]++;
    f3 Pp, N;
    int obj;
    hit_geometry(s, o, d, h, Pp, N, obj);
    const float* m = s.mats + kMatStride * obj;
    f3 acc = mk3(0.0f, 0.0f, 0.0f);
    uint32_t mask = 0;
    for (int li = 0; li < s.n_lights; ++li) {
      const float* l = s.lights + 6 * li;
      f3 sd = norm3(sub3(mk3(l[0], l[1], l[2]), Pp));
      f3 so = add3(Pp, scale3(kRayEps, sd));
      cnt[kCntShadow]++;
      AnyResult ar = any_hit<SH>(s, so, sd, shs, stride, P.err);
      cnt[kCntNodesA] += ar.nodes;
      cnt[kCntTestsA] += ar.tests;
      if (ar.hit)
        mask |= 1u << li;
      else
        acc = add3(acc, phong_light(m, l, Pp, N, campos));
    }
    masks[k] = mask;
    phong[k] = acc;
    nb = k + 1;
    f3 ro, rd;
    if (!secondary_ray(m, s.ambient_index, d, Pp, N, ro, rd, weight[k])) break;
    o = ro;
    d = rd;
  }
  f3 c = mk3(0.0f, 0.0f, 0.0f);
  for (int k = nb - 1; k >= 0; --k) c = fold_colour(phong[k], weight[k], c);
  return c;
}

// Registers capped at 64 (32 warps per SM with blocks of 128): the megakernel is latency-
// bound and gains more from resident warps than it loses to spills (measured on config 2:
// 112 registers 2,580 Mrays/s, 96 2,794, 80 2,913, 64 3,076, 56 2,987, 48 2,481).
template <int SH>
__global__ void __maxnreg__(64) k_render_plain(PlainParams P) {
  extern __shared__ uint2 shstack[];
  uint2* shs = shstack + threadIdx.x;
  const int stride = blockDim.x;
  unsigned cnt[kNumCounts] = {0, 0, 0, 0, 0, 0, 0, 0};
  // one warp = one 8x4 pixel tile (coherent primary rays)
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int tiles_x = (P.width + 7) >> 3;
  const int tile = g >> 5, lane = g & 31;
  const int x = (tile % tiles_x) * 8 + (lane & 7);
  const int ly = (tile / tiles_x) * 4 + (lane >> 3);  // row within the rendered band
  const int y = P.y0 + ly;
  const int img_pix = y * P.width + x;  // pixel of the whole image: its sample hash
  const int pix = ly * P.width + x;     // pixel of the outputs
  if (x < P.width && ly < P.rows) {
    f3 sum = mk3(0.0f, 0.0f, 0.0f);
    for (int smp = 0; smp < P.spp; ++smp) {
      int32_t hits[kMaxBounces];
      uint32_t masks[kMaxBounces];
#pragma unroll
      for (int k = 0; k < kMaxBounces; ++k) {
        hits[k] = EOS_HIT_UNTRACED;
        masks[k] = 0;
      }
      float ox, oy;
      sample_offset((uint32_t)img_pix, smp, P.spp, P.jitter_seed, P.pixel_offset, ox, oy);
      f3 d = primary_direction(P.cam, P.width, P.height, x, y, ox, oy);
      f3 o = mk3(P.cam[0], P.cam[1], P.cam[2]);
      f3 c = trace_path<SH>(P, o, d, hits, masks, cnt, shs, stride);
      sum = add3(sum, c);
      size_t path = (size_t)pix * P.spp + smp;
      if (P.hit) P.hit[path] = hits[0];
      if (P.paths) {
        eos_path_record rec;
#pragma unroll
        for (int k = 0; k < kMaxBounces; ++k) {
          rec.hit[k] = hits[k];
          rec.shadow[k] = masks[k];
        }
        P.paths[path] = rec;
      }
    }
    if (P.spp > 1) sum = scale3(1.0f / (float)P.spp, sum);
    if (P.rgb) {
      P.rgb[3 * (size_t)pix] = sum.x;
      P.rgb[3 * (size_t)pix + 1] = sum.y;
      P.rgb[3 * (size_t)pix + 2] = sum.z;
    }
    if (P.rgba8) {
      uchar4 q = make_uchar4(quantize(sum.x), quantize(sum.y), quantize(sum.z), 255);
      reinterpret_cast<uchar4*>(P.rgba8)[pix] = q;
    }
  }
#pragma unroll
  for (int c = 0; c < kNumCounts; ++c) warp_add_count(&P.counts[c], cnt[c]);
}

template <int SH>
__global__ void k_trace_closest(DevScene s, const float* __restrict__ rays, int n, int32_t* ids, float* ts, int* err) {
  extern __shared__ uint2 shstack[];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + 6 * (size_t)i;
  Hit h = closest_hit<SH>(s, mk3(r[0], r[1], r[2]), mk3(r[3], r[4], r[5]), shstack + threadIdx.x, blockDim.x, err);
  ids[i] = h.pos < 0 ? EOS_HIT_NONE : h.id;
  if (ts) ts[i] = h.t;
}

template <int SH>
__global__ void k_trace_any(DevScene s, const float* __restrict__ rays, int n, uint8_t* occ, int* err) {
  extern __shared__ uint2 shstack[];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + 6 * (size_t)i;
  occ[i] = any_hit<SH>(s, mk3(r[0], r[1], r[2]), mk3(r[3], r[4], r[5]), shstack + threadIdx.x, blockDim.x, err).hit
               ? 1
               : 0;
}

inline int clamp_block(int b) { return b <= 0 ? 128 : std::min(512, std::max(32, (b / 32) * 32)); }
inline int pick_stack(int d) { return d <= 0 ? 16 : (d <= 8 ? 8 : (d <= 16 ? 16 : 32)); }

}  // namespace

eos_status render_plain(eos_ctx* ctx, const eos_scene* sc, const eos_camera& cam, const eos_render_params& p,
                        float* rgb, uint8_t* rgba8, int32_t* hit, eos_path_record* paths) {
  PlainParams P;
  P.s = sc->dev;
  for (int k = 0; k < 3; ++k) {
    P.cam[k] = cam.position[k];
    P.cam[3 + k] = cam.view[k];
    P.cam[6 + k] = cam.right[k];
    P.cam[9 + k] = cam.up[k];
  }
  P.width = cam.width;
  P.height = cam.height;
  P.y0 = p.row_end > 0 ? p.row_begin : 0;
  P.rows = p.row_end > 0 ? p.row_end - p.row_begin : cam.height;
  P.trace_depth = p.trace_depth;
  P.spp = p.spp;
  P.pixel_offset = p.pixel_offset;
  P.jitter_seed = p.jitter_seed;
  P.rgb = rgb;
  P.rgba8 = rgba8;
  P.hit = hit;
  P.paths = paths;
  P.err = ctx->d_err;
  P.counts = ctx->d_counts;
  const int block = clamp_block(p.block_size);
  const int sh = pick_stack(p.stack_depth);
  const long long n_threads = (long long)((cam.width + 7) / 8) * ((P.rows + 3) / 4) * 32;
  const int grid = (int)std::max<long long>(1, (n_threads + block - 1) / block);
  const size_t smem = (size_t)sh * block * sizeof(uint2);
  cudaStream_t st = ctx->stream;
  if (smem > 48 * 1024) {  // opt in to more than the default 48 KB of dynamic shared memory
    if (sh == 8) cudaFuncSetAttribute(k_render_plain<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    else if (sh == 16) cudaFuncSetAttribute(k_render_plain<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    else cudaFuncSetAttribute(k_render_plain<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  if (sh == 8) k_render_plain<8><<<grid, block, smem, st>>>(P);
  else if (sh == 16) k_render_plain<16><<<grid, block, smem, st>>>(P);
  else k_render_plain<32><<<grid, block, smem, st>>>(P);
  EOS_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return EOS_OK;
}

eos_status trace_closest(eos_ctx* ctx, const eos_scene* sc, const float* d_rays, uint32_t n, int32_t* d_ids,
                         float* d_t) {
  if (n == 0) return EOS_OK;
  const int block = 128;
  const int grid = (int)((n + block - 1) / block);
  k_trace_closest<16><<<grid, block, 16 * block * sizeof(uint2), ctx->stream>>>(sc->dev, d_rays, (int)n, d_ids, d_t,
                                                                               ctx->d_err);
  EOS_CUDA(cudaGetLastError());
  return EOS_OK;
}

eos_status trace_any(eos_ctx* ctx, const eos_scene* sc, const float* d_rays, uint32_t n, uint8_t* d_occ) {
  if (n == 0) return EOS_OK;
  const int block = 128;
  const int grid = (int)((n + block - 1) / block);
  k_trace_any<16><<<grid, block, 16 * block * sizeof(uint2), ctx->stream>>>(sc->dev, d_rays, (int)n, d_occ,
                                                                           ctx->d_err);
  EOS_CUDA(cudaGetLastError());
  return EOS_OK;
}

}  // namespace eos
