// BVH traversal and shading device functions (header-only; included by the kernel TUs).
//
// Nearest hit = the smallest t >= 0 over all triangles, exact ties resolved to the larger
// triangle id.  This is the reference's result (src/BVH.cpp:609-659 keeps t <= best
// through Triangle::hit, src/Triangle.cpp:37-38) without its dependence on one particular
// tree: the reference keeps the later of two equal hits in its own traversal order.
// Shadow rays = any triangle hit at t >= 0 (src/BVH.cpp:661-716 with the uninitialised
// distance at :703 read as FLT_MAX).
//
// Box tests are conservative so that culling never removes the exact answer:
//  * slab far distances are widened by 1 + 2*gamma(3) (rounding of (b - o) * (1/d));
//    the traversals use a one-instruction-per-plane form that accepts a superset of those
//    boxes (FmaSlabRay);
//  * a box is culled against the current best t only beyond best * (1 + 2^-12), a margin
//    for the rounding of the triangle test's own t;
//  * a direction component with |d| < 1e-30 is treated as parallel: its slab is the whole
//    line when the origin lies inside the closed slab and empty otherwise (the
//    reference's (b - o) * inf turns into NaN there, src/Box.cu:234-255).
#pragma once
#include "eos_internal.cuh"

namespace eos {

constexpr float kSlack = 1.0000004f;           // 1 + 2*gamma(3)
constexpr float kCull = 1.000244140625f;       // 1 + 2^-12
constexpr float kParallelEps = 1e-30f;
constexpr float kRayEps = 1e-3f;               // shadow / mirror ray offset, src/RayTracer.cpp:305

// Ray prepared for box tests.  sx / sy / sz select the near plane of each axis in a node
// record ([0..2] = lo.xyz, [3..5] = hi.xyz): 0 (lo) for a direction component >= 0 or a
// parallel axis, 3 (hi) otherwise; the far plane is the other one.  The near and far
// distances are then (near - o) / d and (far - o) / d directly, the same values the
// min / max of the two plane distances would give.
struct SlabRay {
  float ox, oy, oz, ix, iy, iz;
  int sx, sy, sz;
  bool par;
};

__device__ __forceinline__ SlabRay make_slab(f3 o, f3 d) {
  SlabRay r;
  r.ox = o.x; r.oy = o.y; r.oz = o.z;
  bool px = fabsf(d.x) < kParallelEps, py = fabsf(d.y) < kParallelEps, pz = fabsf(d.z) < kParallelEps;
  r.ix = px ? 0.0f : 1.0f / d.x;
  r.iy = py ? 0.0f : 1.0f / d.y;
  r.iz = pz ? 0.0f : 1.0f / d.z;
  r.sx = (px || d.x >= 0.0f) ? 0 : 3;
  r.sy = (py || d.y >= 0.0f) ? 0 : 3;
  r.sz = (pz || d.z >= 0.0f) ? 0 : 3;
  r.par = px || py || pz;
  return r;
}

// Three-input min / max (sm_100): exact, like two fminf / fmaxf.
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Entry and exit distances of a box from its near planes (nx, ny, nz) and far planes
// (fx, fy, fz).  Rays with a (near-)zero direction component take the containment branch
// (near = lo, far = hi there); it is warp-uniform in practice (whole pixel columns share it).
__device__ __forceinline__ void slab_range(const SlabRay& r, float nx, float ny, float nz, float fx, float fy,
                                           float fz, float& tn, float& tf) {
  float tnx = (nx - r.ox) * r.ix, tfx = (fx - r.ox) * r.ix;
  float tny = (ny - r.oy) * r.iy, tfy = (fy - r.oy) * r.iy;
  float tnz = (nz - r.oz) * r.iz, tfz = (fz - r.oz) * r.iz;
  if (r.par) {
    if (r.ix == 0.0f) { tnx = -kInf; tfx = (r.ox >= nx && r.ox <= fx) ? kInf : -kInf; }
    if (r.iy == 0.0f) { tny = -kInf; tfy = (r.oy >= ny && r.oy <= fy) ? kInf : -kInf; }
    if (r.iz == 0.0f) { tnz = -kInf; tfz = (r.oz >= nz && r.oz <= fz) ? kInf : -kInf; }
  }
  tn = fmaxf(max3f(tnx, tny, tnz), 0.0f);
  tf = min3f(tfx, tfy, tfz) * kSlack;
}

// Entry distance of a box, or kInf when the box is missed or starts beyond `limit`.
__device__ __forceinline__ float slab(const SlabRay& r, float nx, float ny, float nz, float fx, float fy, float fz,
                                      float limit) {
  float tn, tf;
  slab_range(r, nx, ny, nz, fx, fy, fz, tn, tf);
  return tn <= fminf(tf, limit) ? tn : kInf;
}

// Hit test of a box for shadow rays (no distance limit, no entry distance needed).
__device__ __forceinline__ bool slab_hit(const SlabRay& r, float nx, float ny, float nz, float fx, float fy,
                                         float fz) {
  float tn, tf;
  slab_range(r, nx, ny, nz, fx, fy, fz, tn, tf);
  return tn <= tf;
}

// Box test in the form b = fma(p, i, c) per plane (i = 1/d), one instruction where
// (p - o) * i takes two; used by both traversals.  c is offset per axis: c_near = fl(c - eps),
// c_far = fl(c + eps), c = fl(-(o i)), eps = 2^-20 |c| + 2^-126.  With u = 2^-24 and
// x = (p - o) i: p i + c_near = x - o i d3 - eps' <= x - eps / 4 (the rounding of c is
// <= 1.0001u|c| <= eps / 16), so b_near <= x + u|x|, and likewise b_far >= x - u|x|;
// the (p - o) * i value a satisfies |a - x| <= 2.0001u|x|.  Hence max(b_near) <=
// max(a_near)(1 + 3.0002u) when that is >= 0 (both entries clamp to 0 otherwise) and
// min(b_far) >= min(a_far)(1 - 3.0002u) when min(a_far) >= 0, and the exit distance
// times 1 + 2^-19 (>= kSlack (1 + 8u) / (1 - u)) accepts every box that slab_hit accepts.
// The entry distance exceeds the exact form's by at most 3.0002u relative, so nearest-hit
// culling compares it with best * (kCull + 2^-19) (RayCull), which keeps every box and
// stack entry the exact form keeps.  Rays with a parallel axis or |o / d| above 1e30 keep
// the exact form (fma_slab_ok).
struct FmaSlabRay {
  float ix, iy, iz, nx, ny, nz, fx, fy, fz;
  int sx, sy, sz;
};

__device__ __forceinline__ bool fma_slab_ok(const SlabRay& r) {
  return !r.par && fabsf(r.ox * r.ix) <= 1e30f && fabsf(r.oy * r.iy) <= 1e30f && fabsf(r.oz * r.iz) <= 1e30f;
}

__device__ __forceinline__ void fma_axis(float o, float i, float& cn, float& cf) {
  const float c = -(o * i);
  const float eps = fabsf(c) * 0x1p-20f + 0x1p-126f;
  cn = c - eps;
  cf = c + eps;
}

__device__ __forceinline__ FmaSlabRay make_fma_slab(const SlabRay& r) {
  FmaSlabRay q;
  q.ix = r.ix; q.iy = r.iy; q.iz = r.iz;
  q.sx = r.sx; q.sy = r.sy; q.sz = r.sz;
  fma_axis(r.ox, r.ix, q.nx, q.fx);
  fma_axis(r.oy, r.iy, q.ny, q.fy);
  fma_axis(r.oz, r.iz, q.nz, q.fz);
  return q;
}

__device__ __forceinline__ bool slab_hit(const FmaSlabRay& r, float nx, float ny, float nz, float fx, float fy,
                                         float fz) {
  const float tn = fmaxf(max3f(fmaf(nx, r.ix, r.nx), fmaf(ny, r.iy, r.ny), fmaf(nz, r.iz, r.nz)), 0.0f);
  const float tf = min3f(fmaf(fx, r.ix, r.fx), fmaf(fy, r.iy, r.fy), fmaf(fz, r.iz, r.fz)) * (1.0f + 0x1p-19f);
  return tn <= tf;
}

__device__ __forceinline__ float slab(const FmaSlabRay& r, float nx, float ny, float nz, float fx, float fy, float fz,
                                      float limit) {
  const float tn = fmaxf(max3f(fmaf(nx, r.ix, r.nx), fmaf(ny, r.iy, r.ny), fmaf(nz, r.iz, r.nz)), 0.0f);
  const float tf = min3f(fmaf(fx, r.ix, r.fx), fmaf(fy, r.iy, r.fy), fmaf(fz, r.iz, r.fz)) * (1.0f + 0x1p-19f);
  return tn <= fminf(tf, limit) ? tn : kInf;
}

// Culling factor on the best hit distance per ray form: the fma form's entry distance can
// exceed the exact form's by 3.0002u relative, which 2^-19 more covers.
template <class Ray>
struct RayCull {
  static constexpr float k = kCull;
};
template <>
struct RayCull<FmaSlabRay> {
  static constexpr float k = 1.0f + 0x1p-12f + 0x1p-19f;
};

struct Hit {
  float t, u, v;
  int pos;  // sorted position, -1 on a miss
  int id;   // triangle id
  unsigned nodes, tests;  // interior nodes fetched, triangles tested
};

struct AnyResult {
  int hit;
  unsigned nodes, tests;
};

// Child references in a node record (written by the LBVH build):
//   >= 0          interior node index
//   leaf          0x80000000 | (count - 1) << 25 | first   (count <= 32, first < 2^25)
//   kDone (-1)    end of traversal (never stored in a node; bit 30 distinguishes it)
constexpr int kDone = -1;
__device__ __forceinline__ bool is_leaf_ref(int r) { return ((uint32_t)r & 0xC0000000u) == 0x80000000u; }
__device__ __forceinline__ int leaf_first(int r) { return r & 0x01ffffff; }
__device__ __forceinline__ int leaf_count(int r) { return ((r >> 25) & 31) + 1; }

// Per-thread traversal stack of (child ref, entry distance): the first SH entries live in
// shared memory (column threadIdx.x of a [SH][blockDim] array), deeper entries spill to
// local memory, CAP in total (kStackMax; CAP = SH, no spill, is the small stack of the
// error-path test limit, eos_limits.small_stack).
template <int SH, int CAP = kStackMax>
struct TraversalStack {
  static_assert(CAP >= SH, "the shared part is the bottom of the stack");
  static constexpr int kShared = SH;
  uint2* sh;
  int stride;
  int sp;
  uint2 spill[CAP > SH ? CAP - SH : 1];
  __device__ __forceinline__ TraversalStack(uint2* base, int str) : sh(base), stride(str), sp(0) {}
  __device__ __forceinline__ bool push(int ref, float t) {
    uint2 v = make_uint2((uint32_t)ref, __float_as_uint(t));
    if (sp < SH) sh[sp * stride] = v;
    else if (sp < CAP) spill[sp - SH] = v;
    else return false;
    ++sp;
    return true;
  }
  __device__ __forceinline__ void push_shared(int ref, float t) {
    sh[sp * stride] = make_uint2((uint32_t)ref, __float_as_uint(t));
    ++sp;
  }
  __device__ __forceinline__ uint2 pop() {
    --sp;
    return sp < SH ? sh[sp * stride] : spill[sp - SH];
  }
  // Next entry whose box starts no later than `limit`, or kDone.
  __device__ __forceinline__ int next(float limit) {
    while (sp > 0) {
      uint2 e = pop();
      if (__uint_as_float(e.y) <= limit) return (int)e.x;
    }
    return kDone;
  }
  // Next entry, any distance (shadow rays), or kDone.
  __device__ __forceinline__ int next_any() { return sp > 0 ? (int)pop().x : kDone; }
  // Entries without a distance (any-hit traversal).
  __device__ __forceinline__ bool push_ref(int ref) { return push(ref, 0.0f); }
  __device__ __forceinline__ void push_ref_shared(int ref) { push_shared(ref, 0.0f); }
};


__device__ __forceinline__ void load_tri(const float4* __restrict__ tris, int p, f3& v1, f3& e1, f3& e2, int& id) {
  float4 a = __ldg(tris + 3 * (size_t)p);
  float4 b = __ldg(tris + 3 * (size_t)p + 1);
  float4 c = __ldg(tris + 3 * (size_t)p + 2);
  v1 = mk3(a.x, a.y, a.z);
  e1 = mk3(a.w, b.x, b.y);
  e2 = mk3(b.z, b.w, c.x);
  id = __float_as_int(c.y);
}

// One fetch of a node record (128 B, four child slots; a binary tree leaves two of them
// unused): the child boxes are tested; with SORT the hit children are ordered by entry
// distance (five compare-exchanges), the nearest becomes `cur` and the others are pushed
// farthest first; without SORT (shadow rays: no distance limit) only hit / miss is
// computed and the first hit in slot order is taken, which measured faster for shadow
// rays than nearest-first.  An unused slot holds the box
// lo = +inf, hi = -inf: on every axis the near plane gives an entry of +inf and the far
// plane an exit of -inf, whatever the direction's sign (parallel axes fail the containment
// test), so both box tests reject it and no per-slot check is needed.  With three free
// shared-memory stack entries (the most one node pushes) the pushes skip their bound
// checks.  Returns false on stack overflow.

template <bool SORT, class Ray, class Stack>
__device__ __forceinline__ bool visit_node4(const float4* __restrict__ node_base, const Ray& r, int& cur,
                                            float limit, Stack& st, unsigned& nodes) {
  constexpr int SH = Stack::kShared;
  const float4* nd = node_base + 8 * (size_t)cur;
  const float4 lx = __ldg(nd + r.sx), ly = __ldg(nd + 1 + r.sy), lz = __ldg(nd + 2 + r.sz);  // near planes
  const float4 hx = __ldg(nd + 3 - r.sx), hy = __ldg(nd + 4 - r.sy), hz = __ldg(nd + 5 - r.sz);  // far planes
  const int4 ref = __ldg(reinterpret_cast<const int4*>(nd) + 6);
  ++nodes;
  int c[4] = {ref.x, ref.y, ref.z, ref.w};
  if constexpr (SORT) {
    float t[4];
    t[0] = slab(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, limit);
    t[1] = slab(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, limit);
    t[2] = slab(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, limit);
    t[3] = slab(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, limit);
#define EOS_CX(a, b)                 \
  if (t[b] < t[a]) {                 \
    float tt = t[a]; t[a] = t[b]; t[b] = tt; \
    int cc = c[a]; c[a] = c[b]; c[b] = cc;   \
  }
    EOS_CX(0, 1) EOS_CX(2, 3) EOS_CX(0, 2) EOS_CX(1, 3) EOS_CX(1, 2)
#undef EOS_CX
    if (t[0] == kInf) {
      cur = st.next(limit);
      return true;
    }
    if (st.sp + 3 <= SH) {
#pragma unroll
      for (int i = 3; i >= 1; --i)
        if (t[i] != kInf) st.push_shared(c[i], t[i]);
    } else {
#pragma unroll
      for (int i = 3; i >= 1; --i)
        if (t[i] != kInf && !st.push(c[i], t[i])) return false;
    }
    cur = c[0];
    return true;
  } else {
    bool h[4];
    h[0] = slab_hit(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x);
    h[1] = slab_hit(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y);
    h[2] = slab_hit(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z);
    h[3] = slab_hit(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w);
    int first = -1;
    if (st.sp + 3 <= SH) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (!h[i]) continue;
        if (first < 0) first = i;
        else st.push_ref_shared(c[i]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (!h[i]) continue;
        if (first < 0) first = i;
        else if (!st.push_ref(c[i])) return false;
      }
    }
    cur = first < 0 ? st.next_any() : c[first];
    return true;
  }
}

// Nearest hit.  Traversal in the two-loop form of Aila & Laine ("Understanding the
// efficiency of ray traversal on GPUs", HPG 2009): a lane that reaches a leaf parks it and
// keeps descending until every lane of the warp holds a leaf, then the lanes intersect
// their leaves together, so triangle tests run with full warps.
template <int SH, int CAP, class Ray>
__device__ __forceinline__ Hit closest_traverse(const DevScene& s, f3 o, f3 d, const Ray& r, uint2* shs, int stride,
                                               int* err) {
  constexpr float kCullR = RayCull<Ray>::k;
  Hit h;
  h.t = kInf; h.u = h.v = 0.0f; h.pos = -1; h.id = -1; h.nodes = 0; h.tests = 0;
  TraversalStack<SH, CAP> st(shs, stride);
  int cur = 0;   // interior node, leaf ref or kDone
  int leaf = 0;  // parked leaf (0 = none)
  for (;;) {
    while (cur >= 0) {
      if (!visit_node4<true>(s.nodes, r, cur, h.t * kCullR, st, h.nodes)) {
        atomicOr(err, kErrStack);
        return h;
      }
      if (cur != kDone && cur < 0 && leaf == 0) {
        leaf = cur;
        cur = st.next(h.t * kCullR);
      }
      if (!__any_sync(__activemask(), leaf == 0)) break;
    }
    while (leaf != 0) {
      const int first = leaf_first(leaf), cnt = leaf_count(leaf);
      h.tests += cnt;
      for (int p = first; p < first + cnt; ++p) {
        f3 v1, e1, e2;
        int id;
        load_tri(s.tris, p, v1, e1, e2, id);
        float t, u, v;
        if (mt_intersect_fast(o, d, v1, e1, e2, t, u, v) && (t < h.t || (t == h.t && id > h.id))) {
          h.t = t; h.u = u; h.v = v; h.pos = p; h.id = id;
        }
      }
      leaf = 0;
      if (cur != kDone && cur < 0) {
        leaf = cur;
        cur = st.next(h.t * kCullR);
      }
    }
    if (cur == kDone) return h;
  }
}

template <int SH, int CAP = kStackMax>
__device__ __forceinline__ Hit closest_hit_body(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  const SlabRay r = make_slab(o, d);
  if (fma_slab_ok(r)) return closest_traverse<SH, CAP>(s, o, d, make_fma_slab(r), shs, stride, err);
  return closest_traverse<SH, CAP>(s, o, d, r, shs, stride, err);
}

// Any hit at t >= 0 (shadow rays), same two-loop form; returns at the first hit.
template <int SH, int CAP, class Ray>
__device__ __forceinline__ AnyResult any_traverse(const DevScene& s, f3 o, f3 d, const Ray& r, uint2* shs,
                                                  int stride, int* err) {
  AnyResult res{0, 0u, 0u};
  TraversalStack<SH, CAP> st(shs, stride);
  int cur = 0;
  int leaf = 0;
  for (;;) {
    while (cur >= 0) {
      if (!visit_node4<false>(s.nodes, r, cur, kInf, st, res.nodes)) {
        atomicOr(err, kErrStack);
        return res;
      }
      if (cur != kDone && cur < 0 && leaf == 0) {
        leaf = cur;
        cur = st.next_any();
      }
      if (!__any_sync(__activemask(), leaf == 0)) break;
    }
    while (leaf != 0) {
      const int first = leaf_first(leaf), cnt = leaf_count(leaf);
      for (int p = first; p < first + cnt; ++p) {
        f3 v1, e1, e2;
        int id;
        load_tri(s.tris, p, v1, e1, e2, id);
        float t, u, v;
        ++res.tests;
        if (mt_intersect_fast(o, d, v1, e1, e2, t, u, v)) {
          res.hit = 1;
          return res;
        }
      }
      leaf = 0;
      if (cur != kDone && cur < 0) {
        leaf = cur;
        cur = st.next_any();
      }
    }
    if (cur == kDone) return res;
  }
}

template <int SH, int CAP = kStackMax>
__device__ __forceinline__ AnyResult any_hit_body(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  const SlabRay r = make_slab(o, d);
  if (fma_slab_ok(r)) return any_traverse<SH, CAP>(s, o, d, make_fma_slab(r), shs, stride, err);
  return any_traverse<SH, CAP>(s, o, d, r, shs, stride, err);
}

// Out-of-line copies for the plain megakernel, which calls both traversals: keeping them
// out of line bounds its register allocation.  The specialised wavefront kernels inline.
template <int SH>
__device__ __noinline__ Hit closest_hit_call(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  return closest_hit_body<SH>(s, o, d, shs, stride, err);
}
template <int SH>
__device__ __noinline__ AnyResult any_hit_call(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  return any_hit_body<SH>(s, o, d, shs, stride, err);
}

// ------------------------------------------------------------------ two-level scenes
// A scene of instances (eos_scene_create_instanced): s.nodes is a tree over the instances'
// world boxes whose leaves each hold one instance; reaching one moves the ray into the
// instance's object space and continues in its mesh's tree.  A marker entry below the
// mesh's entries on the stack (t = -inf, so no limit drops it) brings the ray back.  t is
// the same parameter in both spaces (the direction is not renormalised), so one limit
// culls both levels.  Nearest-hit semantics as for a flat scene, with global ids.
constexpr int kExitMesh = (int)0xC0000001;

// o' = Minv [o, 1], d' = Minv [d, 0]; row r: ((m_r0 x + m_r1 y) + m_r2 z) (+ m_r3).
__device__ __forceinline__ void to_object(const DevInstance* I, f3 o, f3 d, f3& oo, f3& od) {
  const float4* m = reinterpret_cast<const float4*>(I->minv);
  const float4 a = __ldg(m), b = __ldg(m + 1), c = __ldg(m + 2);
  oo = mk3(((a.x * o.x + a.y * o.y) + a.z * o.z) + a.w, ((b.x * o.x + b.y * o.y) + b.z * o.z) + b.w,
           ((c.x * o.x + c.y * o.y) + c.z * o.z) + c.w);
  od = mk3((a.x * d.x + a.y * d.y) + a.z * d.z, (b.x * d.x + b.y * d.y) + b.z * d.z,
           (c.x * d.x + c.y * d.y) + c.z * d.z);
}

// ANY: returns at the first hit (h.pos >= 0 then); otherwise the nearest hit.
template <int SH, bool ANY>
__device__ __noinline__ Hit traverse_instanced(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  Hit h;
  h.t = kInf; h.u = h.v = 0.0f; h.pos = -1; h.id = -1; h.nodes = 0; h.tests = 0;
  const SlabRay rw = make_slab(o, d);
  SlabRay r = rw;
  f3 oo = o, od = d;
  const float4* nodes = s.nodes;
  const float4* tris = nullptr;
  int id_off = 0;
  bool in_mesh = false;
  TraversalStack<SH> st(shs, stride);
  int cur = 0;
  for (;;) {
    const float limit = ANY ? kInf : h.t * kCull;
    if (cur >= 0) {
      if (!visit_node4<!ANY>(nodes, r, cur, limit, st, h.nodes)) {
        atomicOr(err, kErrStack);
        return h;
      }
      continue;
    }
    if (cur == kDone) return h;
    if (cur == kExitMesh) {  // back to the instance tree
      r = rw;
      nodes = s.nodes;
      in_mesh = false;
    } else if (!in_mesh) {  // an instance: continue in its mesh, in object space
      const DevInstance* I = s.inst + leaf_first(cur);
      to_object(I, o, d, oo, od);
      r = make_slab(oo, od);
      nodes = I->nodes;
      tris = I->tris;
      id_off = I->id_offset;
      if (!st.push(kExitMesh, -kInf)) {
        atomicOr(err, kErrStack);
        return h;
      }
      in_mesh = true;
      cur = 0;
      continue;
    } else {  // a leaf of the mesh
      const int first = leaf_first(cur), cnt = leaf_count(cur);
      for (int p = first; p < first + cnt; ++p) {
        f3 v1, e1, e2;
        int id;
        load_tri(tris, p, v1, e1, e2, id);
        float t, u, v;
        ++h.tests;
        if (!mt_intersect_fast(oo, od, v1, e1, e2, t, u, v)) continue;
        const int gid = id_off + id;
        if (ANY) {
          h.t = t; h.u = u; h.v = v; h.pos = p; h.id = gid;
          return h;
        }
        if (t < h.t || (t == h.t && gid > h.id)) {
          h.t = t; h.u = u; h.v = v; h.pos = p; h.id = gid;
        }
      }
    }
    cur = ANY ? st.next_any() : st.next(h.t * kCull);
  }
}

// Instance holding global triangle id `gid` (instances in id order).
__device__ __forceinline__ const DevInstance* instance_of(const DevScene& s, int gid) {
  int lo = 0, hi = s.n_inst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&s.inst[mid].id_offset) <= gid) lo = mid;
    else hi = mid - 1;
  }
  return s.inst + lo;
}

// CAP (inline traversals of flat scenes only): total stack entries, see TraversalStack.
template <int SH, bool INLINE = false, int CAP = kStackMax>
__device__ __forceinline__ Hit closest_hit(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  if (s.inst) return traverse_instanced<SH, false>(s, o, d, shs, stride, err);
  if (INLINE) return closest_hit_body<SH, CAP>(s, o, d, shs, stride, err);
  return closest_hit_call<SH>(s, o, d, shs, stride, err);
}

template <int SH, bool INLINE = false, int CAP = kStackMax>
__device__ __forceinline__ AnyResult any_hit(const DevScene& s, f3 o, f3 d, uint2* shs, int stride, int* err) {
  if (s.inst) {
    const Hit h = traverse_instanced<SH, true>(s, o, d, shs, stride, err);
    return AnyResult{h.pos >= 0 ? 1 : 0, h.nodes, h.tests};
  }
  if (INLINE) return any_hit_body<SH, CAP>(s, o, d, shs, stride, err);
  return any_hit_call<SH>(s, o, d, shs, stride, err);
}

// Traversal work counters, reduced per warp into the context's counter block:
// [3] interior nodes fetched by nearest-hit rays, [4] their triangle tests,
// [5] nodes fetched by shadow rays, [6] their triangle tests, [7] shaded hits.
enum { kCntPrimary = 0, kCntShadow = 1, kCntSecondary = 2, kCntNodesC = 3, kCntTestsC = 4, kCntNodesA = 5,
       kCntTestsA = 6, kCntHits = 7, kNumCounts = 8 };

__device__ __forceinline__ void warp_add_count(unsigned long long* dst, unsigned long long v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// ------------------------------------------------------------------ shading
// Hit point o + t*d and the shading normal normalize(n1(1-u-v) + n2 u + n3 v), normalised
// once more as the reference does after its (identity) world transform
// (src/Triangle.cpp:41-46, src/BVH.cpp:373-380).
__device__ __forceinline__ void hit_geometry(const DevScene& s, f3 o, f3 d, const Hit& h, f3& P, f3& N, int& obj) {
  P = add3(o, scale3(h.t, d));
  const DevInstance* I = s.inst ? instance_of(s, h.id) : nullptr;
  const float4* sr = (I ? I->shade : s.shade) + 3 * (size_t)h.pos;
  float4 a = __ldg(sr), b = __ldg(sr + 1), c = __ldg(sr + 2);
  f3 n1 = mk3(a.x, a.y, a.z), n2 = mk3(a.w, b.x, b.y), n3 = mk3(b.z, b.w, c.x);
  obj = __float_as_int(c.y);
  float w = (1.0f - h.u) - h.v;
  f3 n = norm3(add3(add3(scale3(w, n1), scale3(h.u, n2)), scale3(h.v, n3)));
  if (I) {  // normal to world space: Minv^T n, column c of Minv: ((m_0c n.x + m_1c n.y) + m_2c n.z)
    const float* m = I->minv;
    n = mk3((__ldg(m + 0) * n.x + __ldg(m + 4) * n.y) + __ldg(m + 8) * n.z,
            (__ldg(m + 1) * n.x + __ldg(m + 5) * n.y) + __ldg(m + 9) * n.z,
            (__ldg(m + 2) * n.x + __ldg(m + 6) * n.y) + __ldg(m + 10) * n.z);
    obj += I->mat_base;
  }
  N = norm3(n);
}

// Replay of a recorded hit (the adjoint): the hit of global triangle `id` for ray (o, d),
// through the same exact-order test as the traversal (in the instance's object space for a
// two-level scene), so t, u, v and the sorted position equal the forward pass's.  False if
// the triangle does not take the ray (a record from another scene or camera).
__device__ __forceinline__ bool hit_of_id(const DevScene& s, f3 o, f3 d, int id, Hit& h) {
  const float4* tris = s.tris;
  const int32_t* pos = s.pos_of_id;
  int local = id;
  f3 oo = o, od = d;
  if (s.inst) {
    const DevInstance* I = instance_of(s, id);
    to_object(I, o, d, oo, od);
    tris = I->tris;
    pos = I->pos_of_id;
    local = id - I->id_offset;
  }
  h.id = id;
  h.pos = pos[local];
  f3 v1, e1, e2;
  int rid;
  load_tri(tris, h.pos, v1, e1, e2, rid);
  return mt_intersect(oo, od, v1, e1, e2, h.t, h.u, h.v);
}

// RayTracer::calcPhong + findDiffuseColor for one light (src/RayTracer.cpp:418-458):
// diffuse max(0, L.N) kd Lc, specular [V.R > 0] pow(V.R, shininess) Lc ks with
// R = normalize(2 (N.L) N - L) and V towards the camera position.
__device__ __forceinline__ f3 phong_light(const float* m, const float* l, f3 P, f3 N, f3 cam) {
  f3 L = norm3(sub3(mk3(l[0], l[1], l[2]), P));
  f3 V = norm3(sub3(cam, P));
  float ndl = dot3(N, L);
  float two = 2.0f * ndl;
  f3 R = norm3(sub3(scale3(two, N), L));
  float dd = dot3(L, N);
  dd = dd > 0.0f ? dd : 0.0f;
  f3 diff = mk3((dd * m[0]) * l[3], (dd * m[1]) * l[4], (dd * m[2]) * l[5]);
  float vr = dot3(V, R);
  if (vr > 0.0f) {
    float st = powf(vr, m[6]);
    return add3(diff, mk3((st * l[3]) * m[3], (st * l[4]) * m[4], (st * l[5]) * m[5]));
  }
  return diff;
}

// RayTracer::fresnel (src/RayTracer.cpp:52-64, after Bram de Greve 2006), in its float
// order: reflectance of an interface n1 -> n2 for a unit incident direction and the normal
// on the incident side; 1 under total internal reflection.
__device__ __forceinline__ float fresnel(f3 incident, f3 normal, float n1, float n2) {
  const float n = n1 / n2;
  const float cos_i = -dot3(normal, incident);
  const float sin_t2 = (n * n) * (1.0f - cos_i * cos_i);
  if (sin_t2 > 1.0f) return 1.0f;
  const float cos_t = sqrtf(1.0f - sin_t2);
  const float r_orth = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
  const float r_par = (n2 * cos_i - n1 * cos_t) / (n2 * cos_i + n1 * cos_t);
  return (r_orth * r_orth + r_par * r_par) / 2.0f;
}

// Secondary ray of a hit with material m (RayTracer::shadeIntersection,
// src/RayTracer.cpp:329-407).  Reflective: the mirror ray from P + 1e-3 R, weight =
// reflectivity.  Transparent: the reference computes the Fresnel weight K and traces the
// mirror ray about the incident-side normal from P + 1e-3 n -- twice, as "reflected" and,
// by a slip at :403, again as "refracted" -- and mixes K c + (1 - K) c; the refracted ray
// itself is never traced.  That ray once, with w = -K: the sign bit marks the mix.
// Returns false when the material spawns no ray.
// The mirror ray of a reflective hit: normalize(reflect(d, N)) from P + 1e-3 of it (:339-351).
__device__ __forceinline__ void mirror_ray(f3 d, f3 P, f3 N, f3& ro, f3& rd) {
  rd = norm3(reflect3(d, N));
  ro = add3(P, scale3(kRayEps, rd));
}

// The ray of a transparent hit (:353-407) and its Fresnel weight K.
__device__ __forceinline__ float transparent_ray(const float* m, float ambient, f3 d, f3 P, f3 N, f3& ro, f3& rd) {
  const f3 inc = norm3(d);
  f3 n = N;
  float n1 = ambient, n2 = m[9];
  if (!(dot3(inc, N) < 0.0f)) {  // leaving the material: normal flipped as 0 - N
    n1 = m[9];
    n2 = ambient;
    n = sub3(mk3(0.0f, 0.0f, 0.0f), N);
  }
  const float K = fresnel(inc, n, n1, n2);
  rd = norm3(reflect3(d, n));
  ro = add3(P, scale3(kRayEps, n));
  return K;
}

__device__ __forceinline__ bool secondary_ray(const float* m, float ambient, f3 d, f3 P, f3 N, f3& ro, f3& rd,
                                              float& w) {
  if (m[7] > 0.0f) {
    mirror_ray(d, P, N, ro, rd);
    w = m[7];
    return true;
  }
  if (m[8] > 0.0f) {
    w = -transparent_ray(m, ambient, d, P, N, ro, rd);
    return true;
  }
  w = 0.0f;
  return false;
}

// Colour of a ray-tree node (a material that is both reflective and transparent traces
// both rays, src/RayTracer.cpp:339-407) as :410 sums it: (phong + wR c_mirror) +
// (K c_t + (1 - K) c_t); a term the material lacks is 0 (wR = 0, has_t false), a child not
// traced (beyond the trace depth, or a miss) has colour 0.  For a node with one secondary
// ray this equals fold_colour bit for bit (x + 0 = x for the non-negative sums here).
__device__ __forceinline__ f3 tree_colour(f3 phong, float wR, f3 cR, bool has_t, float K, f3 cT) {
  const f3 refr = has_t ? add3(scale3(K, cT), scale3(1.0f - K, cT)) : mk3(0.0f, 0.0f, 0.0f);
  return add3(add3(phong, scale3(wR, cR)), refr);
}

// Colour fold of one bounce: phong + w c for a mirror (or no) bounce; for a transparent
// one (sign bit of w set, K = -w) (phong + 0) + (K c + (1 - K) c) as the reference sums it.
__device__ __forceinline__ f3 fold_colour(f3 phong, float w, f3 c) {
  if (signbit(w)) {
    const float K = -w, L = 1.0f - K;
    return add3(phong, add3(scale3(K, c), scale3(L, c)));
  }
  return add3(phong, scale3(w, c));
}

// Weight of the next bounce's colour in the adjoint: d(fold)/dc.
__device__ __forceinline__ float fold_weight(float w) { return signbit(w) ? (-w) + (1.0f - (-w)) : w; }

// 8-bit quantisation of src/RayTracer.cpp:150-153: floor(c == 1 ? 255 : min(256 c, 255)).
// 256*c, the min and the floor are exact in float, so the float form matches the
// reference's double arithmetic bit for bit.
__device__ __forceinline__ uint8_t quantize(float c) {
  float q = c == 1.0f ? 255.0f : fminf(c * 256.0f, 255.0f);
  q = floorf(q);
  return (uint8_t)(q > 0.0f ? q : 0.0f);
}

}  // namespace eos
