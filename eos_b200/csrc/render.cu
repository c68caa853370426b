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
  int grid;  // side of the reference's AA grid (EOS_FLAG_AA_GRID), 0 = jitter
  float* rgb;
  uint8_t* rgba8;
  int32_t* hit;
  eos_path_record* paths;
  eos_tree_node* tree;         // tree-form records (TREE kernel): EOS_TREE_NODES(trace_depth) per path
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

// One shaded node of a ray tree waiting for its children (trace_tree).
struct TreeFrame {
  f3 phong, cR;   // the node's Phong sum; its mirror child's colour once known
  f3 to, td;      // its transparent child's ray
  float wR, K;    // reflectivity (0: no mirror ray), Fresnel weight of the transparent ray
  int node, depth;
  bool has_t;     // transparent ray present
  bool in_t;      // the child being traced is the transparent one
};

// A path as a ray tree (materials both reflective and transparent trace both secondary
// rays, src/RayTracer.cpp:339-407): a post-order walk with an explicit stack of shaded
// nodes (at most one per bounce), mirror child first as the reference recurses; node
// colours by tree_colour.  rec (nullable): the path's tree record, heap order.
template <int SH>
__device__ f3 trace_tree(const PlainParams& P, f3 o, f3 d, eos_tree_node* rec, int& root_hit, unsigned* cnt,
                         uint2* shs, int stride) {
  const DevScene& s = P.s;
  const f3 campos = mk3(P.cam[0], P.cam[1], P.cam[2]);
  const f3 zero = mk3(0.0f, 0.0f, 0.0f);
  TreeFrame st[kMaxBounces];
  int sp = 0, node = 0, depth = 0;
  for (;;) {
    // trace the ray of (node, depth <= trace_depth) and shade its hit
    f3 c = zero;
    cnt[depth == 0 ? kCntPrimary : kCntSecondary]++;
    Hit h = closest_hit<SH>(s, o, d, shs, stride, P.err);
    cnt[kCntNodesC] += h.nodes;
    cnt[kCntTestsC] += h.tests;
    if (node == 0) root_hit = h.pos < 0 ? EOS_HIT_NONE : h.id;
    if (h.pos < 0) {
      if (rec) rec[node].hit = EOS_HIT_NONE;
    } else {
      cnt[kCntHits]++;
      f3 Pp, N;
      int obj;
      hit_geometry(s, o, d, h, Pp, N, obj);
      const float* m = s.mats + kMatStride * obj;
      TreeFrame F;
      F.phong = zero;
      uint32_t mask = 0;
      for (int li = 0; li < s.n_lights; ++li) {
        const float* l = s.lights + 6 * li;
        f3 sd = norm3(sub3(mk3(l[0], l[1], l[2]), Pp));
        f3 so = add3(Pp, scale3(kRayEps, sd));
        cnt[kCntShadow]++;
        AnyResult ar = any_hit<SH>(s, so, sd, shs, stride, P.err);
        cnt[kCntNodesA] += ar.nodes;
        cnt[kCntTestsA] += ar.tests;
        if (ar.hit) mask |= 1u << li;
        else F.phong = add3(F.phong, phong_light(m, l, Pp, N, campos));
      }
      if (rec) {
        rec[node].hit = h.id;
        rec[node].shadow = mask;
      }
      f3 ro = zero, rd = zero;
      const bool has_r = m[7] > 0.0f;
      F.wR = has_r ? m[7] : 0.0f;
      if (has_r) mirror_ray(d, Pp, N, ro, rd);
      F.has_t = m[8] > 0.0f;
      F.K = F.has_t ? transparent_ray(m, s.ambient_index, d, Pp, N, F.to, F.td) : 0.0f;
      F.cR = zero;
      F.node = node;
      F.depth = depth;
      if (depth < P.trace_depth && (has_r || F.has_t)) {
        F.in_t = !has_r;
        st[sp++] = F;
        if (has_r) {
          o = ro;
          d = rd;
          node = 2 * node + 1;
        } else {
          o = F.to;
          d = F.td;
          node = 2 * node + 2;
        }
        ++depth;
        continue;
      }
      c = tree_colour(F.phong, F.wR, zero, F.has_t, F.K, zero);  // children beyond the trace depth
    }
    // hand the colour up until a node still has its transparent child to trace
    bool next = false;
    while (sp > 0) {
      TreeFrame& F = st[sp - 1];
      if (!F.in_t) {
        F.cR = c;
        if (F.has_t) {
          F.in_t = true;
          o = F.to;
          d = F.td;
          node = 2 * F.node + 2;
          depth = F.depth + 1;
          next = true;
          break;
        }
        c = tree_colour(F.phong, F.wR, F.cR, false, 0.0f, zero);
      } else {
        c = tree_colour(F.phong, F.wR, F.cR, true, F.K, c);
      }
      --sp;
    }
    if (!next) return c;
  }
}

// Registers capped at 64 (32 warps per SM with blocks of 128): the megakernel is latency-
// bound and gains more from resident warps than it loses to spills (measured on config 2:
// 112 registers 2,580 Mrays/s, 96 2,794, 80 2,913, 64 3,076, 56 2,987, 48 2,481).
template <int SH, bool TREE = false>
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
      float ox, oy;
      sample_offset((uint32_t)img_pix, smp, P.spp, P.jitter_seed, P.pixel_offset, ox, oy, P.grid);
      f3 d = primary_direction(P.cam, P.width, P.height, x, y, ox, oy);
      f3 o = mk3(P.cam[0], P.cam[1], P.cam[2]);
      size_t path = (size_t)pix * P.spp + smp;
      if constexpr (TREE) {
        const int nn = EOS_TREE_NODES(P.trace_depth);
        eos_tree_node* rec = P.tree ? P.tree + path * nn : nullptr;
        if (rec)
          for (int k = 0; k < nn; ++k) rec[k] = eos_tree_node{EOS_HIT_UNTRACED, 0u};
        int root_hit = EOS_HIT_NONE;
        f3 c = trace_tree<SH>(P, o, d, rec, root_hit, cnt, shs, stride);
        sum = add3(sum, c);
        if (P.hit) P.hit[path] = root_hit;
      } else {
        int32_t hits[kMaxBounces];
        uint32_t masks[kMaxBounces];
#pragma unroll
        for (int k = 0; k < kMaxBounces; ++k) {
          hits[k] = EOS_HIT_UNTRACED;
          masks[k] = 0;
        }
        f3 c = trace_path<SH>(P, o, d, hits, masks, cnt, shs, stride);
        sum = add3(sum, c);
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
    }
    if (P.spp > 1 || P.grid > 0) sum = scale3(sample_weight(P.spp, P.grid), sum);
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

namespace {

template <bool TREE>
void launch_plain(const PlainParams& P, int sh, int grid, int block, size_t smem, cudaStream_t st) {
  if (smem > 48 * 1024) {  // opt in to more than the default 48 KB of dynamic shared memory
    if (sh == 8) cudaFuncSetAttribute(k_render_plain<8, TREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    else if (sh == 16)
      cudaFuncSetAttribute(k_render_plain<16, TREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    else cudaFuncSetAttribute(k_render_plain<32, TREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  if (sh == 8) k_render_plain<8, TREE><<<grid, block, smem, st>>>(P);
  else if (sh == 16) k_render_plain<16, TREE><<<grid, block, smem, st>>>(P);
  else k_render_plain<32, TREE><<<grid, block, smem, st>>>(P);
}

}  // namespace

// tree: ray-tree kernel (scenes with materials both reflective and transparent, or tree
// records asked for); paths then points at tree-form records.
eos_status render_plain(eos_ctx* ctx, const eos_scene* sc, const eos_camera& cam, const eos_render_params& p,
                        float* rgb, uint8_t* rgba8, int32_t* hit, void* paths, bool tree) {
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
  P.grid = (p.flags & EOS_FLAG_AA_GRID) ? aa_grid_side(p.spp) : 0;
  P.rgb = rgb;
  P.rgba8 = rgba8;
  P.hit = hit;
  P.paths = tree ? nullptr : (eos_path_record*)paths;
  P.tree = tree ? (eos_tree_node*)paths : nullptr;
  P.err = ctx->d_err;
  P.counts = ctx->d_counts;
  const int block = clamp_block(p.block_size);
  const int sh = pick_stack(p.stack_depth);
  const long long n_threads = (long long)((cam.width + 7) / 8) * ((P.rows + 3) / 4) * 32;
  const int grid = (int)std::max<long long>(1, (n_threads + block - 1) / block);
  const size_t smem = (size_t)sh * block * sizeof(uint2);
  if (tree) launch_plain<true>(P, sh, grid, block, smem, ctx->stream);
  else launch_plain<false>(P, sh, grid, block, smem, ctx->stream);
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
