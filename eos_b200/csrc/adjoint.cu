// Adjoint of the shading (no reference counterpart): gradients of an image loss L with
// respect to per-object kd, ks, log(shininess) and per-light colour and position, with
// visibility frozen from the forward pass's path records (hit triangle per bounce and
// blocked-light masks).  Nothing else of the forward pass is stored: each bounce's hit is
// re-derived from its triangle id with the same exact-order Moller-Trumbore, hit point,
// normal and secondary ray as the forward kernels (in the instance's object space for a
// two-level scene), so the geometry matches the forward pass bit for bit.
//
// Forward model per path (src/RayTracer.cpp:302-458): c = sum_k T_k phong_k with
// T_k = prod_{j<k} w_j, w = reflectivity for a mirror bounce and K + (1 - K) for a
// transparent one (its Fresnel mix of one colour); for a ray tree the sum runs over its
// nodes, T the product of the edge weights from the primary ray.  Per unblocked light l,
//   phong = max(0, N.L) kd*C_l + [V.R > 0] (V.R)^s C_l*ks,  L = (p_l - P)/|p_l - P|,
//   R = w/|w|, w = 2 (N.L) N - L,  V = normalize(camera - P),  s = shininess.
// Gradients with g = dL/dc * T_k:
//   dkd_c += g_c max(0,N.L) C_c          dks_c += g_c (V.R)^s C_c
//   dlog s += sum_c g_c ks_c C_c (V.R)^s ln(V.R) s
//   dC_c  += g_c (max(0,N.L) kd_c + (V.R)^s ks_c)
//   dp_l  += a (N - (N.L) L)/|u|  [N.L > 0]
//          + b s (V.R)^(s-1) (I - L L^T)/|u| (2 N N^T - I) (V - (V.R) R)/|w|  [V.R > 0]
//   with a = sum_c g_c C_c kd_c, b = sum_c g_c C_c ks_c.
// Per-object sums use a warp segmented reduction (peers by object id) and one atomic per
// object per warp; per-light sums are reduced over the warp first (every lane takes part,
// with zeros for blocked lights and finished paths), then one shared-memory atomic per
// warp and component, and one global atomic per block and component.
#include <algorithm>

#include "trace.cuh"

namespace eos {
namespace {

struct BwArgs {
  DevScene s;
  const float* cams;  // n_views x 12
  int w, h, n_views, trace_depth, spp;
  int y0, rows;   // image rows [y0, y0 + rows) of the forward records (a row band, or all)
  float off;
  uint32_t seed;  // sample jitter (spp > 1), as in the forward pass
  int grid;       // side of the reference's AA grid (EOS_FLAG_AA_GRID), 0 = jitter
  const eos_path_record* paths;  // chain records, or
  const eos_tree_node* tree;     // tree records, nn nodes per path
  int nn;
  const float* drgb;
  float* gmat;    // n_obj x 7
  float* glight;  // n_lights x 6
  int* err;
};

__device__ __forceinline__ float warp_sum(float v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Primary ray and weighted dL/dc of path i (pixel-major, samples consecutive).
__device__ __forceinline__ void path_start(const BwArgs& A, long long i, f3& o, f3& d, f3& campos, float* g) {
  const long long npx = (long long)A.w * A.rows;
  const long long px = i / A.spp;  // view * npx + pixel
  const int smp = (int)(i % A.spp);
  int view = (int)(px / npx);
  int pix = (int)(px % npx);
  const float* cam = A.cams + 12 * view;
  const int x = pix % A.w, y = A.y0 + pix / A.w;  // image row
  float ox, oy;
  sample_offset((uint32_t)(y * A.w + x), smp, A.spp, A.seed, A.off, ox, oy, A.grid);
  d = primary_direction(cam, A.w, A.h, x, y, ox, oy);
  campos = mk3(cam[0], cam[1], cam[2]);
  o = campos;
  // the pixel is the weighted sum of its samples (the mean, or the reference grid's (1/n)^2)
  const float ws = (A.spp > 1 || A.grid > 0) ? sample_weight(A.spp, A.grid) : 1.0f;
  g[0] = A.drgb[3 * px] * ws;
  g[1] = A.drgb[3 * px + 1] * ws;
  g[2] = A.drgb[3 * px + 2] * ws;
}

// Re-derives the recorded hit `id` of ray (o, d): false (and *alive cleared) when the
// record does not match this scene / camera or holds no hit.
__device__ __forceinline__ bool replay_hit(const BwArgs& A, int id, f3 o, f3 d, f3& P, f3& N, int& obj,
                                           const float*& m) {
  const DevScene& s = A.s;
  if (id < 0 || id >= s.n_tris) return false;
  Hit h;
  if (!hit_of_id(s, o, d, id, h)) {
    atomicOr(A.err, kErrIndex);  // record does not match this scene / camera
    return false;
  }
  hit_geometry(s, o, d, h, P, N, obj);
  m = s.mats + kMatStride * obj;
  return true;
}

// Adjoint of one shaded hit per lane (alive lanes; the others take part with zeros):
// per-light terms reduced over the warp into sl, per-object terms by a warp segmented
// reduction into A.gmat.  gT = dL/dc times the hit's throughput.  Warp-uniform.
__device__ __forceinline__ void hit_adjoint(const BwArgs& A, float* sl, bool alive, f3 P, f3 N, int obj,
                                            const float* m, uint32_t mask, f3 campos, const float* gT) {
  const DevScene& s = A.s;
  const int lane = threadIdx.x & 31;
  float gm[7] = {0, 0, 0, 0, 0, 0, 0};
  {
    const float shin = alive ? m[6] : 0.0f;
    f3 V = alive ? norm3(sub3(campos, P)) : mk3(0, 0, 1);
    if (!alive) mask = 0xffffffffu;
    for (int l = 0; l < s.n_lights; ++l) {
      float gl[6] = {0, 0, 0, 0, 0, 0};
      if (!(mask & (1u << l))) {
        const float* lp = s.lights + 6 * l;
        f3 u = sub3(mk3(lp[0], lp[1], lp[2]), P);
        float ul = sqrtf(dot3(u, u));
        f3 L = scale3(1.0f / ul, u);
        float ndl = dot3(N, L);
        f3 wv = sub3(scale3(2.0f * ndl, N), L);
        float wl = sqrtf(dot3(wv, wv));
        f3 R = scale3(1.0f / wl, wv);
        float fd = ndl > 0.0f ? ndl : 0.0f;
        float vr = dot3(V, R);
        float fs = vr > 0.0f ? powf(vr, shin) : 0.0f;
        float C[3] = {lp[3], lp[4], lp[5]};
        float a = 0.0f, b = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          gm[c] += gT[c] * fd * C[c];
          gm[3 + c] += gT[c] * fs * C[c];
          gl[c] = gT[c] * (fd * m[c] + fs * m[3 + c]);
          a += gT[c] * C[c] * m[c];
          b += gT[c] * C[c] * m[3 + c];
        }
        if (vr > 0.0f) gm[6] += b * fs * logf(vr) * shin;
        f3 gp = mk3(0, 0, 0);
        if (ndl > 0.0f) gp = add3(gp, scale3(a / ul, sub3(N, scale3(ndl, L))));
        if (vr > 0.0f) {
          f3 q = scale3(1.0f / wl, sub3(V, scale3(vr, R)));
          f3 q2 = sub3(scale3(2.0f * dot3(N, q), N), q);
          f3 gs = scale3(1.0f / ul, sub3(q2, scale3(dot3(L, q2), L)));
          float dfs = shin * powf(vr, shin - 1.0f);
          gp = add3(gp, scale3(b * dfs, gs));
        }
        gl[3] = gp.x;
        gl[4] = gp.y;
        gl[5] = gp.z;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const float v = warp_sum(gl[c]);
        if (lane == 0 && v != 0.0f) atomicAdd(&sl[6 * l + c], v);
      }
    }
  }
  // per-object segmented reduction: one leader per distinct object in the warp
  int key = alive ? obj : -1;
  uint32_t pending = __ballot_sync(0xffffffffu, key >= 0);
  while (pending) {
    int leader = __ffs(pending) - 1;
    int lk = __shfl_sync(0xffffffffu, key, leader);
    bool mine = key == lk;
    uint32_t peers = __ballot_sync(0xffffffffu, mine);
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      float v = warp_sum(mine ? gm[c] : 0.0f);
      if (lane == leader && v != 0.0f) atomicAdd(&A.gmat[7 * lk + c], v);
    }
    pending &= ~peers;
  }
}

__device__ __forceinline__ void flush_lights(const BwArgs& A, const float* sl) {
  __syncthreads();
  for (int c = threadIdx.x; c < A.s.n_lights * 6; c += blockDim.x)
    if (sl[c] != 0.0f) atomicAdd(&A.glight[c], sl[c]);
}

// Chain records: one secondary ray per hit, T_k+1 = T_k fold_weight(w_k).
__global__ void __launch_bounds__(128) k_backward(BwArgs A) {
  __shared__ float sl[kMaxLights * 6];
  for (int i = threadIdx.x; i < kMaxLights * 6; i += blockDim.x) sl[i] = 0.0f;
  __syncthreads();
  const long long total = (long long)A.w * A.rows * A.spp * A.n_views;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < total;
  const DevScene& s = A.s;
  eos_path_record rec;
  f3 o = mk3(0, 0, 0), d = mk3(0, 0, 1), campos = o;
  float g[3] = {0, 0, 0};
  if (active) {
    rec = A.paths[i];
    path_start(A, i, o, d, campos, g);
  }
  float T = 1.0f;
  bool alive = active;
  for (int k = 0; k <= A.trace_depth; ++k) {
    int obj = -1;
    f3 P = o, N = o;
    const float* m = nullptr;
    if (alive) alive = replay_hit(A, rec.hit[k], o, d, P, N, obj, m);
    const float gT[3] = {g[0] * T, g[1] * T, g[2] * T};
    hit_adjoint(A, sl, alive, P, N, obj, m, alive ? rec.shadow[k] : 0u, campos, gT);
    if (alive) {
      f3 ro, rd;
      float w;
      if (!secondary_ray(m, s.ambient_index, d, P, N, ro, rd, w) || k + 1 > A.trace_depth) {
        alive = false;
      } else {
        T *= fold_weight(w);
        o = ro;
        d = rd;
      }
    }
    if (!__any_sync(0xffffffffu, alive)) break;
  }
  flush_lights(A, sl);
}

// Tree records: a walk over each path's ray tree with a stack of pending rays (mirror
// child 2j + 1 with weight reflectivity, transparent child 2j + 2 with K + (1 - K)); one
// node per lane per step, so the warp reductions stay warp-uniform.
__global__ void __launch_bounds__(128) k_backward_tree(BwArgs A) {
  __shared__ float sl[kMaxLights * 6];
  for (int i = threadIdx.x; i < kMaxLights * 6; i += blockDim.x) sl[i] = 0.0f;
  __syncthreads();
  struct Pending {
    f3 o, d;
    float T;
    int node, k;
  };
  const long long total = (long long)A.w * A.rows * A.spp * A.n_views;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const DevScene& s = A.s;
  Pending st[kMaxBounces + 1];  // depth-first: at most one waiting sibling per bounce, plus the current
  int sp = 0;
  f3 campos = mk3(0, 0, 0);
  float g[3] = {0, 0, 0};
  const eos_tree_node* rec = nullptr;
  if (i < total) {
    f3 o, d;
    path_start(A, i, o, d, campos, g);
    rec = A.tree + (size_t)i * A.nn;
    st[sp++] = Pending{o, d, 1.0f, 0, 0};
  }
  while (__any_sync(0xffffffffu, sp > 0)) {
    bool alive = sp > 0;
    Pending q;
    if (alive) q = st[--sp];
    int obj = -1;
    f3 P = q.o, N = q.o;
    const float* m = nullptr;
    if (alive) alive = replay_hit(A, rec[q.node].hit, q.o, q.d, P, N, obj, m);
    const float gT[3] = {g[0] * q.T, g[1] * q.T, g[2] * q.T};
    hit_adjoint(A, sl, alive, P, N, obj, m, alive ? rec[q.node].shadow : 0u, campos, gT);
    if (alive && q.k + 1 <= A.trace_depth) {
      if (m[8] > 0.0f) {
        Pending c;
        const float K = transparent_ray(m, s.ambient_index, q.d, P, N, c.o, c.d);
        c.T = q.T * fold_weight(-K);
        c.node = 2 * q.node + 2;
        c.k = q.k + 1;
        st[sp++] = c;
      }
      if (m[7] > 0.0f) {
        Pending c;
        mirror_ray(q.d, P, N, c.o, c.d);
        c.T = q.T * m[7];
        c.node = 2 * q.node + 1;
        c.k = q.k + 1;
        st[sp++] = c;
      }
    }
  }
  flush_lights(A, sl);
}

}  // namespace

eos_status render_backward(eos_ctx* ctx, const eos_scene* sc, const eos_camera* cams, uint32_t n_views,
                           const eos_render_params& p, const void* d_paths, const float* d_rgb,
                           float* d_gmat, float* d_glight) {
  eos_status es = EOS_OK;
  float* d_cams = (float*)scratch(ctx, "bw.cams", 48ull * n_views, &es);
  if (es != EOS_OK) return es;
  std::vector<float> hc(12 * (size_t)n_views);
  for (uint32_t v = 0; v < n_views; ++v)
    for (int k = 0; k < 3; ++k) {
      hc[12 * v + k] = cams[v].position[k];
      hc[12 * v + 3 + k] = cams[v].view[k];
      hc[12 * v + 6 + k] = cams[v].right[k];
      hc[12 * v + 9 + k] = cams[v].up[k];
    }
  EOS_CUDA(cudaMemcpyAsync(d_cams, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  EOS_CUDA(cudaMemsetAsync(d_gmat, 0, 28ull * sc->dev.n_obj, ctx->stream));
  EOS_CUDA(cudaMemsetAsync(d_glight, 0, 24ull * std::max(1, sc->dev.n_lights), ctx->stream));
  BwArgs A;
  A.s = sc->dev;
  A.cams = d_cams;
  A.w = cams[0].width;
  A.h = cams[0].height;
  A.n_views = (int)n_views;
  A.trace_depth = p.trace_depth;
  A.y0 = p.row_end > 0 ? p.row_begin : 0;
  A.rows = p.row_end > 0 ? p.row_end - p.row_begin : A.h;
  A.spp = p.spp;
  A.seed = p.jitter_seed;
  A.grid = (p.flags & EOS_FLAG_AA_GRID) ? aa_grid_side(p.spp) : 0;
  A.off = p.pixel_offset;
  const bool tree = (p.flags & EOS_FLAG_TREE_RECORDS) != 0;
  A.paths = tree ? nullptr : (const eos_path_record*)d_paths;
  A.tree = tree ? (const eos_tree_node*)d_paths : nullptr;
  A.nn = EOS_TREE_NODES(p.trace_depth);
  A.drgb = d_rgb;
  A.gmat = d_gmat;
  A.glight = d_glight;
  A.err = ctx->d_err;
  long long total = (long long)A.w * A.rows * p.spp * n_views;
  int grid = (int)((total + 127) / 128);
  if (tree) k_backward_tree<<<grid, 128, 0, ctx->stream>>>(A);
  else k_backward<<<grid, 128, 0, ctx->stream>>>(A);
  EOS_CUDA(cudaGetLastError());
  // the hc vector must outlive the async copy: wait for it
  EOS_CUDA(cudaStreamSynchronize(ctx->stream));
  return EOS_OK;
}

}  // namespace eos
