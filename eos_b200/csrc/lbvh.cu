// GPU BVH build: Morton codes -> stable radix sort -> hierarchy (Karras radix tree, or
// PLOC clustering in ploc.cu) -> atomic refit -> 128-byte node records (4-wide, or 2
// children per record) / 48-byte triangle records.
//
// Replaces the reference's CPU top-down median/SAH build (src/BVH.cpp:97-111,549-606) and
// its SoA upload (src/cudaStructures.cu:36-174,274-405).  The Morton encoder is the
// reference's 30-bit EncodeMorton3 (src/morton.h:45-48); the centroid is the reference
// triangle centroid ((v1 + v2) + v3) / 3 (src/Triangle.h:37), quantised per axis over the
// centroid bounds as q = min(1023, (uint)((1024 * (c - lo)) / (hi - lo))).
// Primitive order = stable sort by (code, triangle id).
#include <algorithm>


#include "eos_internal.cuh"
#include "scan.cuh"

namespace eos {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per block
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

__device__ __forceinline__ uint32_t float_to_ordered(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ f3 load_vert(const float* v, uint32_t i) {
  return mk3(v[3 * (size_t)i], v[3 * (size_t)i + 1], v[3 * (size_t)i + 2]);
}

// Centroids and their bounds.  bounds: [6] ordered uints (min xyz, max xyz).
__global__ void k_centroids(const float* __restrict__ verts, uint32_t n_verts,
                            const uint32_t* __restrict__ tris, int n, float4* __restrict__ cent,
                            uint32_t* __restrict__ bounds, int* err) {
  float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t a = tris[3 * (size_t)i], b = tris[3 * (size_t)i + 1], c = tris[3 * (size_t)i + 2];
    if (a >= n_verts || b >= n_verts || c >= n_verts) {
      atomicOr(err, kErrIndex);
      a = b = c = 0;
    }
    f3 s = add3(add3(load_vert(verts, a), load_vert(verts, b)), load_vert(verts, c));
    f3 m = mk3(s.x / 3.0f, s.y / 3.0f, s.z / 3.0f);
    cent[i] = make_float4(m.x, m.y, m.z, 0.0f);
    lo[0] = fminf(lo[0], m.x); lo[1] = fminf(lo[1], m.y); lo[2] = fminf(lo[2], m.z);
    hi[0] = fmaxf(hi[0], m.x); hi[1] = fmaxf(hi[1], m.y); hi[2] = fmaxf(hi[2], m.z);
  }
  for (int k = 0; k < 3; ++k) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int k = 0; k < 3; ++k) {
      if (lo[k] <= hi[k]) {
        atomicMin(&bounds[k], float_to_ordered(lo[k]));
        atomicMax(&bounds[3 + k], float_to_ordered(hi[k]));
      }
    }
  }
}

__global__ void k_morton(const float4* __restrict__ cent, int n, const uint32_t* __restrict__ bounds,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 c = cent[i];
  float cc[3] = {c.x, c.y, c.z};
  uint32_t q[3];
  for (int k = 0; k < 3; ++k) {
    float lo = ordered_to_float(bounds[k]);
    float hi = ordered_to_float(bounds[3 + k]);
    float ext = hi - lo;
    if (ext > 0.0f) {
      float f = (1024.0f * (cc[k] - lo)) / ext;
      uint32_t u = (uint32_t)f;
      q[k] = u > 1023u ? 1023u : u;
    } else {
      q[k] = 0u;
    }
  }
  keys[i] = morton3(q[0], q[1], q[2]);
  vals[i] = (uint32_t)i;
}

// ------------------------------------------------------------------ stable LSD radix sort
// Per pass: per-tile digit histogram -> per-digit exclusive scan over tiles -> scan of the
// digit totals -> stable scatter.  Inside a tile, warp w owns keys [w*256, w*256+256) in
// 8 rounds of 32; peers with the same digit are found with __match_any_sync and ranked
// with popc, so the scatter keeps the input order (stability gives the (code, id) order).
__global__ void k_sort_hist(const uint32_t* __restrict__ keys, int n, int shift, uint32_t* __restrict__ counts,
                            int n_tiles) {
  __shared__ uint32_t h[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int base = blockIdx.x * kSortTile;
  for (int j = threadIdx.x; j < kSortTile; j += blockDim.x) {
    int idx = base + j;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) counts[(size_t)d * n_tiles + blockIdx.x] = h[d];
}

// One block per digit: exclusive scan of that digit's per-tile counts (in place).
__global__ void k_sort_scan_rows(uint32_t* __restrict__ counts, int n_tiles, uint32_t* __restrict__ totals) {
  __shared__ uint32_t s[kSortThreads];
  __shared__ uint32_t carry;
  uint32_t* row = counts + (size_t)blockIdx.x * n_tiles;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b = 0; b < n_tiles; b += blockDim.x) {
    int i = b + threadIdx.x;
    uint32_t v = i < n_tiles ? row[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < blockDim.x; off <<= 1) {
      uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    uint32_t incl = s[threadIdx.x];
    if (i < n_tiles) row[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

__global__ void k_sort_scan_digits(uint32_t* __restrict__ totals) {
  __shared__ uint32_t s[kRadix];
  uint32_t v = totals[threadIdx.x];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < kRadix; off <<= 1) {
    uint32_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  totals[threadIdx.x] = s[threadIdx.x] - v;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ counts, int n_tiles,
    const uint32_t* __restrict__ digit_base) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t wh[kWarps][kRadix];
  __shared__ uint32_t tile_base[kRadix];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWarps * kRadix; i += blockDim.x) (&wh[0][0])[i] = 0;
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x)
    tile_base[d] = digit_base[d] + counts[(size_t)d * n_tiles + blockIdx.x];
  __syncthreads();
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t key[kSortItems], val[kSortItems], local[kSortItems];
  int base = blockIdx.x * kSortTile + w * 32 * kSortItems;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    int idx = base + r * 32 + lane;
    bool valid = idx < n;
    key[r] = valid ? kin[idx] : 0u;
    val[r] = valid ? vin[idx] : 0u;
    uint32_t digit = valid ? ((key[r] >> shift) & (kRadix - 1)) : (uint32_t)kRadix + lane;
    uint32_t peers = __match_any_sync(0xffffffffu, digit);
    uint32_t rank = __popc(peers & lt_mask);
    uint32_t pre = valid ? wh[w][digit] : 0u;
    __syncwarp();
    if (valid && rank == 0) wh[w][digit] = pre + __popc(peers);
    __syncwarp();
    local[r] = pre + rank;
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    uint32_t s = 0;
    for (int ww = 0; ww < kWarps; ++ww) {
      uint32_t t = wh[ww][d];
      wh[ww][d] = s;
      s += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    int idx = base + r * 32 + lane;
    if (idx < n) {
      uint32_t digit = (key[r] >> shift) & (kRadix - 1);
      uint32_t pos = tile_base[digit] + wh[w][digit] + local[r];
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
  }
}

// ------------------------------------------------------------------ Karras hierarchy
__device__ __forceinline__ int common_prefix(const uint32_t* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = k[i], b = k[j];
  if (a == b) return 32 + __clz((uint32_t)(i ^ j));
  return __clz(a ^ b);
}

// Internal node i of n-1 (Karras 2012, "Maximizing parallelism in the construction of
// BVHs, octrees and k-d trees").  Node numbering: interior 0..n-2, leaf p -> n-1+p.
__global__ void k_karras(const uint32_t* __restrict__ k, int n, int2* __restrict__ child,
                         int2* __restrict__ range, int* __restrict__ parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (common_prefix(k, n, i, i + 1) - common_prefix(k, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = common_prefix(k, n, i, i - d);
  int lmax = 2;
  while (common_prefix(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (common_prefix(k, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = common_prefix(k, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (common_prefix(k, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int gamma = i + s * d + min(d, 0);
  int first = min(i, j), last = max(i, j);
  int left = (first == gamma) ? (n - 1 + gamma) : gamma;
  int right = (last == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
  child[i] = make_int2(left, right);
  range[i] = make_int2(first, last);
  parent[left] = i;
  parent[right] = i;
}

// Triangle records, leaf boxes, id -> position map.  The triangle at Morton position m
// goes to record position p = perm[m] (perm NULL: p = m).
__global__ void k_records(const float* __restrict__ verts, const float* __restrict__ normals, uint32_t n_verts,
                          const uint32_t* __restrict__ tris, const uint32_t* __restrict__ obj,
                          const uint32_t* __restrict__ order, const uint32_t* __restrict__ perm, int n, uint32_t n_obj,
                          float4* __restrict__ trec, float4* __restrict__ srec, int32_t* __restrict__ pos_of_id,
                          float4* __restrict__ blo, float4* __restrict__ bhi, int* err) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  uint32_t id = order[m];
  const int p = perm ? (int)perm[m] : m;
  uint32_t a = tris[3 * (size_t)id], b = tris[3 * (size_t)id + 1], c = tris[3 * (size_t)id + 2];
  if (a >= n_verts || b >= n_verts || c >= n_verts) a = b = c = 0;  // flagged in k_centroids
  f3 v1 = load_vert(verts, a), v2 = load_vert(verts, b), v3 = load_vert(verts, c);
  f3 e1 = sub3(v2, v1), e2 = sub3(v3, v1);
  trec[3 * (size_t)p] = make_float4(v1.x, v1.y, v1.z, e1.x);
  trec[3 * (size_t)p + 1] = make_float4(e1.y, e1.z, e2.x, e2.y);
  trec[3 * (size_t)p + 2] = make_float4(e2.z, __int_as_float((int)id), 0.0f, 0.0f);
  f3 n1 = load_vert(normals, a), n2 = load_vert(normals, b), n3 = load_vert(normals, c);
  srec[3 * (size_t)p] = make_float4(n1.x, n1.y, n1.z, n2.x);
  srec[3 * (size_t)p + 1] = make_float4(n2.y, n2.z, n3.x, n3.y);
  uint32_t ob = obj[id];
  if (ob >= n_obj) {
    atomicOr(err, kErrIndex);
    ob = 0;
  }
  srec[3 * (size_t)p + 2] = make_float4(n3.z, __int_as_float((int)ob), 0.0f, 0.0f);
  pos_of_id[id] = p;
  size_t leaf = (size_t)(n - 1) + p;  // .w: SAH cost of one triangle, leaf flag
  blo[leaf] = make_float4(fminf(fminf(v1.x, v2.x), v3.x), fminf(fminf(v1.y, v2.y), v3.y),
                          fminf(fminf(v1.z, v2.z), v3.z), 1.0f);
  bhi[leaf] = make_float4(fmaxf(fmaxf(v1.x, v2.x), v3.x), fmaxf(fmaxf(v1.y, v2.y), v3.y),
                          fmaxf(fmaxf(v1.z, v2.z), v3.z), 1.0f);
}

// Leaf reference: 0x80000000 | (count - 1) << 25 | first  (count <= 32, first < 2^25).
__host__ __device__ __forceinline__ int pack_leaf(int first, int count) {
  return (int)(0x80000000u | ((uint32_t)(count - 1) << 25) | (uint32_t)first);
}

constexpr float kCostNode = 1.0f;  // SAH cost of visiting one node (two box tests)
constexpr float kCostTri = 1.0f;   // SAH cost of one triangle test

__device__ __forceinline__ float half_area(float4 l, float4 h) {
  float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
  return dx * dy + dy * dz + dz * dx;
}

// Bottom-up refit: one thread per leaf walks to the root; the second thread to reach an
// interior node merges the two child boxes and decides whether the subtree becomes one
// leaf (node records are written afterwards by the wide conversion).  Leaf decision: fixed layout -> the range has at most
// max_leaf triangles; SAH layout -> additionally the leaf's cost kCostTri * n is not above
// kCostNode + (A_l cost_l + A_r cost_r) / A.  Box .w carries the subtree cost (lo) and the
// leaf decision (hi).  Bounded walk: the tree depth is at most kStackMax.
__global__ void k_refit(int n, const int2* __restrict__ child, const int2* __restrict__ range,
                        const int* __restrict__ parent, float4* blo, float4* bhi, int* __restrict__ arrive,
                        int max_leaf, int sah, int* err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int node = parent[n - 1 + p];
  for (int step = 0; node >= 0; ++step) {
    if (step > kStackMax) {
      atomicOr(err, kErrDepth);
      return;
    }
    __threadfence();
    if (atomicAdd(&arrive[node], 1) == 0) return;
    __threadfence();
    int2 c = child[node];
    float4 l0 = __ldcg(&blo[c.x]), h0 = __ldcg(&bhi[c.x]);
    float4 l1 = __ldcg(&blo[c.y]), h1 = __ldcg(&bhi[c.y]);
    float4 lo = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
    float4 hi = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
    int2 rg = range[node];
    int size = rg.y - rg.x + 1;
    float a = half_area(lo, hi);
    float inner = kCostNode + (a > 0.0f ? (half_area(l0, h0) * l0.w + half_area(l1, h1) * l1.w) / a : l0.w + l1.w);
    float as_leaf = size <= max_leaf ? kCostTri * (float)size : kInf;
    bool collapse = sah ? (as_leaf <= inner) : (size <= max_leaf);
    lo.w = collapse ? as_leaf : inner;
    hi.w = collapse ? 1.0f : 0.0f;
    blo[node] = lo;
    bhi[node] = hi;
    node = parent[node];
  }
}

// ------------------------------------------------------------------ node records
// Every node record has four child slots.  A node is made from one binary node by
// replacing its interior child of largest surface area by that child's two children until
// it has `max_children` children (4 for the 4-wide layout, 2 for the binary one) or only
// leaves (one-triangle leaves and collapsed subtrees stay leaves).  Top-down, one launch
// per level; frontier entries are (binary node, record) pairs.
//
// Record, 128 B = 8 x float4 (structure of arrays over the four slots):
//   [0] lo.x[4] [1] lo.y[4] [2] lo.z[4] [3] hi.x[4] [4] hi.y[4] [5] hi.z[4]
//   [6] ref[4]: interior record index, packed leaf, or kEmptyRef for an unused slot
//       (whose box is lo = +inf, hi = -inf: every slab test misses it, so the traversal
//       needs no per-slot check)
//   [7] count[4]: triangles of a leaf, 0 for an interior child, -1 for an unused slot
constexpr int kEmptyRef = (int)0xC0000000;

__device__ __forceinline__ void write_record(float4* o, const float (&v)[6][4], const int (&ref)[4],
                                             const int (&cnt)[4]) {
  for (int a = 0; a < 6; ++a) o[a] = make_float4(v[a][0], v[a][1], v[a][2], v[a][3]);
  o[6] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
  o[7] = make_float4(__int_as_float(cnt[0]), __int_as_float(cnt[1]), __int_as_float(cnt[2]), __int_as_float(cnt[3]));
}

// One level of the wide records, in two passes over the frontier (binary node, record):
// k_wide_select opens each frontier node's children greedily (the largest-area interior
// child is replaced by its two children until max_children) and counts those that get a
// record of their own; after an exclusive scan of the counts, k_wide_write numbers them
// base + scan[t] + j and writes the record.  Records come out level by level, each node's
// children in consecutive records, the same on every run.
// Greedy opening of one frontier node (k_wide_select): its children, then the children of
// the largest-area interior child until max_children are reached; returns how many of
// them get records of their own.
__device__ __forceinline__ int wide_select_one(int n, const int2* __restrict__ child, const float4* __restrict__ blo,
                                               const float4* __restrict__ bhi, int node, int max_children,
                                               int4& sel) {
  int c[4] = {-1, -1, -1, -1};
  const int2 ch = child[node];
  c[0] = ch.x;
  c[1] = ch.y;
  int k = 2;
  while (k < max_children) {
    int best = -1;
    float best_area = -1.0f;
    for (int i = 0; i < k; ++i) {
      const int ci = c[i];
      if (ci >= n - 1 || bhi[ci].w != 0.0f) continue;  // triangle or collapsed subtree: a leaf
      const float a = half_area(blo[ci], bhi[ci]);
      if (a > best_area) {
        best_area = a;
        best = i;
      }
    }
    if (best < 0) break;
    const int2 g = child[c[best]];
    c[best] = g.x;
    c[k++] = g.y;
  }
  int m = 0;
  for (int i = 0; i < k; ++i) m += c[i] < n - 1 && bhi[c[i]].w == 0.0f;
  sel = make_int4(c[0], c[1], c[2], c[3]);
  return m;
}

__global__ void __launch_bounds__(kScanBlock) k_wide_select(int n, const int2* __restrict__ child,
                                                            const float4* __restrict__ blo,
                                                            const float4* __restrict__ bhi,
                                                            const int2* __restrict__ frontier_in, int n_in,
                                                            int max_children, int4* __restrict__ sel,
                                                            int* __restrict__ n_interior, int* __restrict__ bsum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = t < n_in ? wide_select_one(n, child, blo, bhi, frontier_in[t].x, max_children, sel[t]) : 0;
  if (t < n_in) n_interior[t] = m;
  block_total(m, bsum);  // the scan's first step (scan.cuh)
}

// The first record number of frontier node t's children: its block's exclusive scan of n_interior
// plus the block's scanned sum (bsum after k_scan_totals); same grid as k_wide_select.
__global__ void __launch_bounds__(kScanBlock) k_wide_write(int n, const int2* __restrict__ range,
                                                           const float4* __restrict__ blo,
                                                           const float4* __restrict__ bhi,
                                                           const int2* __restrict__ frontier_in, int n_in,
                                                           const int4* __restrict__ sel,
                                                           const int* __restrict__ n_interior,
                                                           const int* __restrict__ bsum, int base,
                                                           int2* __restrict__ frontier_out,
                                                           float4* __restrict__ wnodes, int max_nodes, int* err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int block_sum;
  int next = bsum[blockIdx.x] + block_exclusive_scan(t < n_in ? n_interior[t] : 0, block_sum);
  if (t >= n_in) return;
  const int4 s4 = sel[t];
  const int c[4] = {s4.x, s4.y, s4.z, s4.w};
  float v[6][4];
  int ref[4], cnt[4];
  for (int i = 0; i < 4; ++i) {
    const int ci = c[i];
    if (ci < 0) {
      for (int a = 0; a < 6; ++a) v[a][i] = a < 3 ? kInf : -kInf;  // a box no ray enters
      ref[i] = kEmptyRef;
      cnt[i] = -1;
      continue;
    }
    const float4 l = blo[ci], h = bhi[ci];
    v[0][i] = l.x; v[1][i] = l.y; v[2][i] = l.z;
    v[3][i] = h.x; v[4][i] = h.y; v[5][i] = h.z;
    if (ci >= n - 1) {
      cnt[i] = 1;
      ref[i] = pack_leaf(ci - (n - 1), 1);
    } else if (h.w != 0.0f) {
      const int2 r = range[ci];
      cnt[i] = r.y - r.x + 1;
      ref[i] = pack_leaf(r.x, cnt[i]);
    } else {
      const int w = base + next;
      if (w >= max_nodes) {  // cannot happen: the tree has at most n - 1 records (the host stops)
        atomicOr(err, kErrQueue);
        for (int a = 0; a < 6; ++a) v[a][i] = a < 3 ? kInf : -kInf;
        ref[i] = kEmptyRef;
        cnt[i] = -1;
        ++next;
        continue;
      }
      frontier_out[next++] = make_int2(ci, w);
      ref[i] = w;
      cnt[i] = 0;
    }
  }
  write_record(wnodes + 8 * (size_t)frontier_in[t].y, v, ref, cnt);
}

// Root record of a scene with 0 or 1 triangle (no binary interior node exists).
__global__ void k_small_root(int n, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                             float4* __restrict__ nodes) {
  float v[6][4];
  for (int a = 0; a < 6; ++a)
    for (int i = 0; i < 4; ++i) v[a][i] = a < 3 ? kInf : -kInf;
  int ref[4] = {kEmptyRef, kEmptyRef, kEmptyRef, kEmptyRef};
  int cnt[4] = {-1, -1, -1, -1};
  if (n == 1) {
    const float4 l = blo[0], h = bhi[0];
    v[0][0] = l.x; v[1][0] = l.y; v[2][0] = l.z;
    v[3][0] = h.x; v[4][0] = h.y; v[5][0] = h.z;
    ref[0] = pack_leaf(0, 1);
    cnt[0] = 1;
  }
  write_record(nodes, v, ref, cnt);
}

inline int grid_for(size_t n, int block) { return (int)std::max<size_t>(1, (n + block - 1) / block); }

// Writes the node records of the binary tree in the given width (top-down, one select /
// scan / write per level).  Returns the number of levels through *levels (kStackMax * 4 + 1 when the walk
// did not end, which cannot happen for a tree of depth <= kStackMax).
eos_status write_records(eos_ctx* ctx, int n, const int2* child, const int2* range, const float4* blo,
                         const float4* bhi, int width, float4* out, int max_nodes, int* levels, int* n_records) {
  cudaStream_t st = ctx->stream;
  eos_status es = EOS_OK;
  const size_t nn = (size_t)n;
  int2* fa = (int2*)scratch(ctx, "lbvh.wide.fa", 8 * nn, &es);
  int2* fb = (int2*)scratch(ctx, "lbvh.wide.fb", 8 * nn, &es);
  int4* sel = (int4*)scratch(ctx, "lbvh.wide.sel", 16 * nn, &es);
  int* m = (int*)scratch(ctx, "lbvh.wide.m", 4 * (nn + 1), &es);
  int* bsum = (int*)scratch(ctx, "lbvh.wide.bsum", 4 * ((size_t)scan_blocks(n + 1) + 1), &es);
  if (es != EOS_OK) return es;
  const int2 root = make_int2(0, 0);  // the binary root becomes record 0
  EOS_CUDA(cudaMemcpyAsync(fa, &root, sizeof root, cudaMemcpyHostToDevice, st));
  int n_in = 1, base = 1, lv = 0;
  while (n_in > 0 && lv <= 4 * kStackMax) {  // bounded: the depth is at most the binary depth
    const int nb = scan_blocks(n_in);
    k_wide_select<<<nb, kScanBlock, 0, st>>>(n, child, blo, bhi, fa, n_in, width, sel, m, bsum);
    k_scan_totals<<<1, 1024, 0, st>>>(bsum, nb);
    k_wide_write<<<nb, kScanBlock, 0, st>>>(n, range, blo, bhi, fa, n_in, sel, m, bsum, base, fb, out, max_nodes,
                                            ctx->d_err);
    EOS_CUDA(cudaGetLastError());
    ++lv;
    int n_out = 0;
    EOS_CUDA(cudaMemcpyAsync(&n_out, bsum + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
    EOS_CUDA(cudaStreamSynchronize(st));
    if ((long long)base + n_out > max_nodes) return EOS_ERR_QUEUE_OVERFLOW;  // cannot happen, as above
    base += n_out;
    n_in = n_out;
    std::swap(fa, fb);
  }
  *n_records = std::min(base, max_nodes);
  *levels = n_in > 0 ? 4 * kStackMax + 1 : lv;
  return EOS_OK;
}

// Node records of the scene.  The traversal stack holds at most width - 1 entries per
// level, so a 4-wide tree deeper than kStackMax / 3 levels (degenerate geometry) is written
// with two children per record instead; a binary tree's depth is at most 62 <= kStackMax.
eos_status build_records(eos_ctx* ctx, eos_scene* sc, int n, const int2* child, const int2* range,
                         const float4* blo, const float4* bhi) {
  const int max_nodes = n - 1;
  EOS_CUDA(cudaMalloc(&sc->d_nodes, 128 * (size_t)max_nodes));
  sc->device_bytes += 128 * (size_t)max_nodes;
  int levels = 0, records = 0;
  eos_status es = write_records(ctx, n, child, range, blo, bhi, sc->width, (float4*)sc->d_nodes, max_nodes, &levels,
                                &records);
  if (es != EOS_OK) return es;
  if (sc->width == 4 && 3 * levels > kStackMax) {
    sc->width = 2;
    es = write_records(ctx, n, child, range, blo, bhi, 2, (float4*)sc->d_nodes, max_nodes, &levels, &records);
    if (es != EOS_OK) return es;
  }
  if ((sc->width - 1) * levels > kStackMax) return EOS_ERR_STACK_OVERFLOW;
  sc->n_nodes = (uint32_t)records;
  sc->levels = levels;
  return EOS_OK;
}

}  // namespace

eos_status build_scene(eos_ctx* ctx, eos_scene* sc, const float* d_verts, const float* d_normals,
                       uint32_t n_verts, const uint32_t* d_tris, const uint32_t* d_obj, uint32_t n_tris) {
  cudaStream_t st = ctx->stream;
  const int n = (int)n_tris;
  const size_t nn = std::max<size_t>(1, n);
  eos_status es = EOS_OK;
  const size_t n_nodes = std::max<size_t>(1, nn - 1);
  // persistent scene buffers (node records: build_records, or one root record below)
  EOS_CUDA(cudaMalloc(&sc->d_tris, 48 * nn));
  EOS_CUDA(cudaMalloc(&sc->d_shade, 48 * nn));
  EOS_CUDA(cudaMalloc(&sc->d_pos_of_id, 4 * nn));
  EOS_CUDA(cudaMalloc(&sc->d_codes, 4 * nn));
  EOS_CUDA(cudaMalloc(&sc->d_order, 4 * nn));
  sc->device_bytes += 48 * nn * 2 + 4 * nn * 3;
  // temporaries
  float4* cent = (float4*)scratch(ctx, "lbvh.cent", 16 * nn, &es);
  uint32_t* bounds = (uint32_t*)scratch(ctx, "lbvh.bounds", 64, &es);
  uint32_t* k2 = (uint32_t*)scratch(ctx, "lbvh.k2", 4 * nn, &es);
  uint32_t* v2 = (uint32_t*)scratch(ctx, "lbvh.v2", 4 * nn, &es);
  const int n_tiles = (int)((nn + kSortTile - 1) / kSortTile);
  uint32_t* counts = (uint32_t*)scratch(ctx, "lbvh.counts", 4 * (size_t)kRadix * n_tiles, &es);
  uint32_t* totals = (uint32_t*)scratch(ctx, "lbvh.totals", 4 * kRadix, &es);
  int2* child = (int2*)scratch(ctx, "lbvh.child", 8 * n_nodes, &es);
  int2* range = (int2*)scratch(ctx, "lbvh.range", 8 * n_nodes, &es);
  int* parent = (int*)scratch(ctx, "lbvh.parent", 4 * (2 * nn), &es);
  int* arrive = (int*)scratch(ctx, "lbvh.arrive", 4 * n_nodes, &es);
  float4* blo = (float4*)scratch(ctx, "lbvh.blo", 16 * (2 * nn), &es);
  float4* bhi = (float4*)scratch(ctx, "lbvh.bhi", 16 * (2 * nn), &es);
  if (es != EOS_OK) return es;

  uint32_t* keys = (uint32_t*)sc->d_codes;
  uint32_t* vals = (uint32_t*)sc->d_order;
  EOS_CUDA(cudaEventRecord(ctx->ev0, st));
  if (n > 0) {
    uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    EOS_CUDA(cudaMemcpyAsync(bounds, init, sizeof init, cudaMemcpyHostToDevice, st));
    int g = std::min(grid_for(nn, 256), ctx->num_sms * 8);
    k_centroids<<<g, 256, 0, st>>>(d_verts, n_verts, d_tris, n, cent, bounds, ctx->d_err);
    k_morton<<<grid_for(nn, 256), 256, 0, st>>>(cent, n, bounds, keys, vals);
    uint32_t *ki = keys, *vi = vals, *ko = k2, *vo = v2;
    for (int shift = 0; shift < 30; shift += kRadixBits) {
      k_sort_hist<<<n_tiles, kSortThreads, 0, st>>>(ki, n, shift, counts, n_tiles);
      k_sort_scan_rows<<<kRadix, kSortThreads, 0, st>>>(counts, n_tiles, totals);
      k_sort_scan_digits<<<1, kRadix, 0, st>>>(totals);
      k_sort_scatter<<<n_tiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n, shift, counts, n_tiles, totals);
      std::swap(ki, ko);
      std::swap(vi, vo);
    }
    // 4 passes: the sorted result is back in (keys, vals)
    k_records<<<grid_for(nn, 256), 256, 0, st>>>(d_verts, d_normals, n_verts, d_tris, d_obj, vals, nullptr, n,
                                                 (uint32_t)sc->dev.n_obj, (float4*)sc->d_tris, (float4*)sc->d_shade,
                                                 (int32_t*)sc->d_pos_of_id, blo, bhi, ctx->d_err);
  }
  if (n >= 2) {
    bool ploc = sc->builder == EOS_BUILDER_PLOC;
    if (ploc) {
      // PLOC over the leaf boxes in Morton order, then the records again in the tree's
      // depth-first leaf order (every subtree a contiguous range)
      uint32_t* perm = (uint32_t*)scratch(ctx, "lbvh.perm", 4 * nn, &es);
      if (es != EOS_OK) return es;
      int depth = 0;
      if ((es = build_ploc(ctx, n, blo, bhi, child, range, parent, perm, &depth)) != EOS_OK) return es;
      ploc = depth + 2 <= kStackMax;  // the refit walks at most kStackMax levels
      if (ploc)
        k_records<<<grid_for(nn, 256), 256, 0, st>>>(d_verts, d_normals, n_verts, d_tris, d_obj, vals, perm, n,
                                                     (uint32_t)sc->dev.n_obj, (float4*)sc->d_tris,
                                                     (float4*)sc->d_shade, (int32_t*)sc->d_pos_of_id, blo, bhi,
                                                     ctx->d_err);
      else
        sc->builder = EOS_BUILDER_LBVH;
    }
    EOS_CUDA(cudaMemsetAsync(arrive, 0, 4 * n_nodes, st));
    if (!ploc) {
      EOS_CUDA(cudaMemsetAsync(parent, 0xff, 4 * (2 * nn), st));
      k_karras<<<grid_for(n - 1, 256), 256, 0, st>>>(keys, n, child, range, parent);
    }
    k_refit<<<grid_for(nn, 256), 256, 0, st>>>(n, child, range, parent, blo, bhi, arrive, sc->leaf_size,
                                              sc->layout == EOS_LAYOUT_SAH, ctx->d_err);
    // SAH cost of the tree (subtree cost of the root, in triangle-test units)
    EOS_CUDA(cudaMemcpyAsync(&sc->sah_cost, &blo[0].w, sizeof(float), cudaMemcpyDeviceToHost, st));
    eos_status ws = build_records(ctx, sc, n, child, range, blo, bhi);
    if (ws != EOS_OK) return ws;
  } else {
    EOS_CUDA(cudaMalloc(&sc->d_nodes, 128));
    sc->device_bytes += 128;
    k_small_root<<<1, 1, 0, st>>>(n, blo, bhi, (float4*)sc->d_nodes);
    sc->n_nodes = 1;
    sc->levels = 1;
  }
  EOS_CUDA(cudaGetLastError());
  EOS_CUDA(cudaEventRecord(ctx->ev1, st));
  EOS_CUDA(cudaEventSynchronize(ctx->ev1));
  EOS_CUDA(cudaEventElapsedTime(&sc->build_ms, ctx->ev0, ctx->ev1));
  return EOS_OK;
}

}  // namespace eos
