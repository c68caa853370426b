/*
 * eos_oracle.c -- CPU restatement of the Eos render path.  TEST INFRASTRUCTURE ONLY:
 * loaded by tests/, by the smoke check and by the CPU-baseline leg of bench.py as the
 * checker; the product never links or calls it.
 *
 * What is restated, with the reference lines each part follows:
 *   - Moller-Trumbore with the |det| < 1e-5 rejection and t < 0 / u / v bounds, in the
 *     reference's operation order                        src/Triangle.cpp:57-91
 *   - hit point o + t*d and the normal normalize(n1(1-u-v) + n2 u + n3 v), normalised a
 *     second time after the identity world transform    src/Triangle.cpp:26-55,
 *                                                        src/BVH.cpp:369-381
 *   - primary rays  normalize(aa*right + bb*up + view)   src/RayTracer.cpp:119-145
 *   - per-light shadow ray P + 1e-3*L, Phong diffuse + specular with V from the camera,
 *     mirror ray normalize(reflect(d, N)) from P + 1e-3*r, colour fold
 *     phong + reflectivity * trace(next), depth rule     src/RayTracer.cpp:268-458
 *   - glm 0.9.6 arithmetic: dot = (x0y0 + x1y1) + x2y2, normalize = v * (1/sqrt(dot)),
 *     reflect = I - (N*dot(N,I))*2                        glm/detail/func_geometric.inl:65-72,
 *                                                        :154-173; func_exponential.inl:150-153
 *   - 30-bit Morton codes: EncodeMorton3 / Part1By2      src/morton.h:30-48
 *
 * Semantics that differ on purpose from the reference's traversal, so that the result
 * does not depend on a particular tree:
 *   - nearest hit = the smallest t >= 0 over ALL triangles (exact ties: the larger
 *     triangle id wins).  The reference walks its own tree and keeps the later of equal
 *     hits; its interior boxes are tested against [0.001, 999] (src/BVH.cpp:609-659).
 *   - shadow ray = any triangle with t >= 0 (the reference, with its uninitialised
 *     distance at src/BVH.cpp:703 fixed to FLT_MAX, accepts every t >= 0 in the leaves
 *     its box tests reach, src/BVH.cpp:661-716).
 * Paths where these differences can matter are flagged per path (near ties within
 * 2 ulp; hits closer than 1e-3 to a ray origin), so parity tests can count them.
 *
 * The FP64 section re-renders with frozen visibility (given hit ids and shadow masks)
 * and evaluates the analytic adjoint of an image loss with respect to per-object
 * kd / ks / log-shininess and per-light colour / position.
 *
 * Built with -ffp-contract=off and without -ffast-math (oracle/Makefile).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#define MAXB 8
#define HIT_NONE (-1)
#define HIT_UNTRACED (-2)
#define FLAG_TIE 1u
#define FLAG_NEAR_ORIGIN 2u
#define FLAG_OUT_OF_RANGE 4u
#define FLAG_AXIS_PARALLEL 8u
#define LEAF_MAX 4

typedef struct { float x, y, z; } v3f;

static inline v3f V3(float x, float y, float z) { v3f r = {x, y, z}; return r; }
static inline v3f vadd(v3f a, v3f b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3f vsub(v3f a, v3f b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3f vscale(float s, v3f a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline float vdot(v3f a, v3f b) { float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z; return (x + y) + z; }
static inline v3f vcross(v3f a, v3f b) {
  return V3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline v3f vnorm(v3f a) { float s = 1.0f / sqrtf(vdot(a, a)); return V3(a.x * s, a.y * s, a.z * s); }
static inline float fget(v3f a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

/* Material record: kd rgb, ks rgb, shininess, reflectivity, transparency, refractive index. */
#define OMAT 10

typedef struct {
  float lo[3], hi[3];
  int left, right;   /* children (interior) */
  int start, count;  /* triangle range in sorted order (leaf when count > 0) */
} onode;

typedef struct {
  int nt, nobj, nl;
  v3f *v1, *v2, *v3, *e1, *e2, *n1, *n2, *n3; /* sorted (Morton) order */
  int32_t *id;                                 /* sorted position -> triangle id */
  uint32_t *obj;                               /* sorted position -> object */
  float *mats;                                 /* nobj x OMAT (eos_material) */
  float ambient;                               /* refractive index outside objects */
  /* two-level scene (oracle_instanced_create): ninst > 0, the arrays above unused */
  int ninst;
  const void** inst_mesh;                      /* per instance: its mesh (an oscene) */
  float* inst_minv;                            /* ninst x 12: object-from-world affine */
  int32_t* inst_id_off;                        /* global id of the mesh's triangle 0 */
  int32_t* inst_mat_base;
  float *lights;                               /* nl x 6 */
  onode *nodes;
  int nnodes;
  /* by triangle id, for the frozen-visibility FP64 path */
  int32_t *pos_of_id;
} oscene;

/* ---------------------------------------------------------------- Morton codes */
static inline uint32_t part1by2(uint32_t x) {
  x &= 0x000003ffu;
  x = (x ^ (x << 16)) & 0xff0000ffu;
  x = (x ^ (x << 8)) & 0x0300f00fu;
  x = (x ^ (x << 4)) & 0x030c30c3u;
  x = (x ^ (x << 2)) & 0x09249249u;
  return x;
}
static inline uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return (part1by2(z) << 2) + (part1by2(y) << 1) + part1by2(x);
}

typedef struct { uint32_t code; int32_t idx; } keyidx;
static int cmp_keyidx(const void* a, const void* b) {
  const keyidx* x = (const keyidx*)a; const keyidx* y = (const keyidx*)b;
  if (x->code != y->code) return x->code < y->code ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static inline v3f load3(const float* p, uint32_t i) { return V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

/* Centroid ((v1 + v2) + v3) / 3 (src/Triangle.h:37), quantised per axis over the
 * centroid bounds: q = min(1023, (uint)((1024 * (c - lo)) / (hi - lo))), 0 for a flat axis. */
void oracle_morton(const float* verts, const uint32_t* tris, int nt, uint32_t* codes,
                   int32_t* order) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  v3f* c = (v3f*)malloc(sizeof(v3f) * (size_t)(nt > 0 ? nt : 1));
  for (int i = 0; i < nt; ++i) {
    v3f a = load3(verts, tris[3 * i]), b = load3(verts, tris[3 * i + 1]), d = load3(verts, tris[3 * i + 2]);
    v3f s = vadd(vadd(a, b), d);
    c[i] = V3(s.x / 3.0f, s.y / 3.0f, s.z / 3.0f);
    for (int k = 0; k < 3; ++k) {
      float v = fget(c[i], k);
      if (v < lo[k]) lo[k] = v;
      if (v > hi[k]) hi[k] = v;
    }
  }
  keyidx* ki = (keyidx*)malloc(sizeof(keyidx) * (size_t)(nt > 0 ? nt : 1));
  for (int i = 0; i < nt; ++i) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      float ext = hi[k] - lo[k];
      if (ext > 0.0f) {
        float f = (1024.0f * (fget(c[i], k) - lo[k])) / ext;
        uint32_t u = (uint32_t)f;
        q[k] = u > 1023u ? 1023u : u;
      } else {
        q[k] = 0;
      }
    }
    codes[i] = morton3(q[0], q[1], q[2]);
    ki[i].code = codes[i];
    ki[i].idx = i;
  }
  qsort(ki, (size_t)nt, sizeof(keyidx), cmp_keyidx);
  for (int i = 0; i < nt; ++i) order[i] = ki[i].idx;
  free(ki);
  free(c);
}

/* ---------------------------------------------------------------- scene + BVH */
static void box_of_range(const oscene* s, int a, int b, float lo[3], float hi[3]) {
  for (int k = 0; k < 3; ++k) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
  for (int i = a; i < b; ++i) {
    v3f p[3] = {s->v1[i], s->v2[i], s->v3[i]};
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        float v = fget(p[j], k);
        if (v < lo[k]) lo[k] = v;
        if (v > hi[k]) hi[k] = v;
      }
  }
}

static int build_rec(oscene* s, int a, int b) {
  int me = s->nnodes++;
  onode* n = &s->nodes[me];
  box_of_range(s, a, b, n->lo, n->hi);
  if (b - a <= LEAF_MAX) {
    n->start = a; n->count = b - a; n->left = n->right = -1;
    return me;
  }
  int mid = a + (b - a) / 2;
  n->count = 0; n->start = a;
  int l = build_rec(s, a, mid);
  int r = build_rec(s, mid, b);
  s->nodes[me].left = l;
  s->nodes[me].right = r;
  return me;
}

void* oracle_scene_create(const float* verts, const float* normals, int nv, const uint32_t* tris,
                          const uint32_t* tri_obj, int nt, const float* mats, int nobj,
                          const float* lights, int nl) {
  (void)nv;
  oscene* s = (oscene*)calloc(1, sizeof(oscene));
  s->nt = nt; s->nobj = nobj; s->nl = nl;
  size_t n = (size_t)(nt > 0 ? nt : 1);
  s->v1 = malloc(sizeof(v3f) * n); s->v2 = malloc(sizeof(v3f) * n); s->v3 = malloc(sizeof(v3f) * n);
  s->e1 = malloc(sizeof(v3f) * n); s->e2 = malloc(sizeof(v3f) * n);
  s->n1 = malloc(sizeof(v3f) * n); s->n2 = malloc(sizeof(v3f) * n); s->n3 = malloc(sizeof(v3f) * n);
  s->id = malloc(sizeof(int32_t) * n); s->obj = malloc(sizeof(uint32_t) * n);
  s->pos_of_id = malloc(sizeof(int32_t) * n);
  uint32_t* codes = malloc(sizeof(uint32_t) * n);
  int32_t* order = malloc(sizeof(int32_t) * n);
  oracle_morton(verts, tris, nt, codes, order);
  for (int p = 0; p < nt; ++p) {
    int i = order[p];
    const uint32_t* t = tris + 3 * i;
    s->v1[p] = load3(verts, t[0]); s->v2[p] = load3(verts, t[1]); s->v3[p] = load3(verts, t[2]);
    s->n1[p] = load3(normals, t[0]); s->n2[p] = load3(normals, t[1]); s->n3[p] = load3(normals, t[2]);
    s->e1[p] = vsub(s->v2[p], s->v1[p]);
    s->e2[p] = vsub(s->v3[p], s->v1[p]);
    s->id[p] = i;
    s->obj[p] = tri_obj[i];
    s->pos_of_id[i] = p;
  }
  free(codes); free(order);
  s->mats = malloc(sizeof(float) * OMAT * (size_t)(nobj > 0 ? nobj : 1));
  memcpy(s->mats, mats, sizeof(float) * OMAT * (size_t)nobj);
  s->ambient = 1.0f;
  s->lights = malloc(sizeof(float) * 6 * (size_t)(nl > 0 ? nl : 1));
  memcpy(s->lights, lights, sizeof(float) * 6 * (size_t)nl);
  s->nodes = malloc(sizeof(onode) * (2 * n + 1));
  s->nnodes = 0;
  if (nt > 0) build_rec(s, 0, nt);
  return s;
}

/* Scene::setAmbientRefractiveIndex (src/Scene.cpp:134-136). */
void oracle_scene_set_ambient(void* h, float ambient) { ((oscene*)h)->ambient = ambient; }

void oracle_scene_destroy(void* h) {
  oscene* s = (oscene*)h;
  if (!s) return;
  free(s->v1); free(s->v2); free(s->v3); free(s->e1); free(s->e2);
  free(s->n1); free(s->n2); free(s->n3); free(s->id); free(s->obj); free(s->pos_of_id);
  free(s->mats); free(s->lights); free(s->nodes);
  free((void*)s->inst_mesh); free(s->inst_minv); free(s->inst_id_off); free(s->inst_mat_base); free(s);
}

/* ---------------------------------------------------------------- intersection */
/* Triangle::RayTriangleIntersection, src/Triangle.cpp:57-91 (e1, e2 precomputed with the
 * same subtraction). Returns 1 and t,u,v on a hit. */
static inline int mt_hit(v3f o, v3f d, v3f v1, v3f e1, v3f e2, float* t, float* u, float* v) {
  v3f P = vcross(d, e2);
  float det = vdot(e1, P);
  if (det > -0.00001f && det < 0.00001f) return 0;
  float inv_det = 1.0f / det;
  v3f T = vsub(o, v1);
  v3f Q = vcross(T, e1);
  float tt = vdot(e2, Q) * inv_det;
  if (tt < 0.0f) return 0;
  float uu = vdot(T, P) * inv_det;
  if (uu < 0.0f || uu > 1.0f) return 0;
  float vv = vdot(d, Q) * inv_det;
  if (vv < 0.0f || uu + vv > 1.0f) return 0;
  *t = tt; *u = uu; *v = vv;
  return 1;
}

/* Conservative slab test: the float interval is widened by 1 + 2*gamma(3) so that no box
 * that contains a hit with t in [0, tlimit] is rejected by rounding. */
static const float kSlack = 1.0000004f;          /* 1 + 2 * gamma(3), gamma(n) = n u / (1 - n u) */
static const float kCullSlack = 1.000244140625f; /* 1 + 2^-12: margin against MT's own t error */

/* A direction component that is exactly zero makes the slab of that axis either the
 * whole line (origin inside the closed slab) or empty; it is tested by containment
 * instead of by 0 * inf products (the reference's test yields NaN there,
 * src/Box.cu:234-255). */
typedef struct { v3f o, inv; int par[3]; } bray;

static inline bray make_bray(v3f o, v3f d) {
  bray r; r.o = o;
  float dd[3] = {d.x, d.y, d.z}, iv[3];
  for (int k = 0; k < 3; ++k) { r.par[k] = fabsf(dd[k]) < 1e-30f; iv[k] = r.par[k] ? 0.0f : 1.0f / dd[k]; }
  r.inv = V3(iv[0], iv[1], iv[2]);
  return r;
}

static inline int box_test(const onode* n, const bray* r, float tlimit) {
  float tmin = -FLT_MAX, tmax = FLT_MAX;
  float oo[3] = {r->o.x, r->o.y, r->o.z}, ii[3] = {r->inv.x, r->inv.y, r->inv.z};
  for (int k = 0; k < 3; ++k) {
    if (r->par[k]) {
      if (oo[k] < n->lo[k] || oo[k] > n->hi[k]) return 0;
      continue;
    }
    float a = (n->lo[k] - oo[k]) * ii[k];
    float b = (n->hi[k] - oo[k]) * ii[k];
    float lo = a < b ? a : b, hi = a < b ? b : a;
    if (lo > tmin) tmin = lo;
    if (hi < tmax) tmax = hi;
  }
  tmax *= kSlack;
  return tmin <= tmax && tmax >= 0.0f && tmin <= tlimit;
}

static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

typedef struct { int pos; float t, u, v; float t2; int gid, inst; } chit;

/* Nearest hit with the larger-id tie rule; also tracks the second-nearest distinct hit
 * (culling by it) so near ties can be flagged. */
static chit closest_flat(const oscene* s, v3f o, v3f d) {
  chit h; h.pos = -1; h.t = FLT_MAX; h.u = h.v = 0; h.t2 = FLT_MAX; h.gid = -1; h.inst = -1;
  if (s->nt == 0) return h;
  bray br = make_bray(o, d);
  int stack[128]; int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const onode* n = &s->nodes[stack[--sp]];
    float lim = h.t2 < FLT_MAX ? h.t2 * kCullSlack : FLT_MAX;
    if (!box_test(n, &br, lim)) continue;
    if (n->count) {
      for (int p = n->start; p < n->start + n->count; ++p) {
        float t, u, v;
        if (!mt_hit(o, d, s->v1[p], s->e1[p], s->e2[p], &t, &u, &v)) continue;
        int better = h.pos < 0 || t < h.t || (t == h.t && s->id[p] > s->id[h.pos]);
        if (better) {
          if (h.pos >= 0 && h.t < h.t2) h.t2 = h.t;
          h.pos = p; h.t = t; h.u = u; h.v = v; h.gid = s->id[p];
        } else if (t < h.t2) {
          h.t2 = t;
        }
      }
    } else {
      stack[sp++] = n->left;
      stack[sp++] = n->right;
    }
  }
  return h;
}

static int any_hit_flat(const oscene* s, v3f o, v3f d) {
  if (s->nt == 0) return 0;
  bray br = make_bray(o, d);
  int stack[128]; int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const onode* n = &s->nodes[stack[--sp]];
    if (!box_test(n, &br, FLT_MAX)) continue;
    if (n->count) {
      for (int p = n->start; p < n->start + n->count; ++p) {
        float t, u, v;
        if (mt_hit(o, d, s->v1[p], s->e1[p], s->e2[p], &t, &u, &v)) return 1;
      }
    } else {
      stack[sp++] = n->left;
      stack[sp++] = n->right;
    }
  }
  return 0;
}

/* ---------------------------------------------------------------- two-level scenes */
/* A scene of instances of mesh scenes (the library's eos_scene_create_instanced): every
 * instance's mesh is tested with the ray moved into its object space,
 * o' = Minv [o, 1], d' = Minv [d, 0] with row r evaluated as ((m_r0 x + m_r1 y) + m_r2 z)
 * (+ m_r3), in float; the nearest hit over all instances with the larger global id on
 * exact ties; the normal is normalize(Minv^T n).  Minv is the inverse of the world-from-
 * object affine [A | t] computed in double from the adjugate and rounded to float. */
static void affine_inverse_d(const float* M, float* out) {
  const double a00 = M[0], a01 = M[1], a02 = M[2], a10 = M[4], a11 = M[5], a12 = M[6];
  const double a20 = M[8], a21 = M[9], a22 = M[10];
  const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  const double det = (a00 * c00 + a01 * c01) + a02 * c02;
  const double inv[3][3] = {{c00 / det, (a02 * a21 - a01 * a22) / det, (a01 * a12 - a02 * a11) / det},
                            {c01 / det, (a00 * a22 - a02 * a20) / det, (a02 * a10 - a00 * a12) / det},
                            {c02 / det, (a01 * a20 - a00 * a21) / det, (a00 * a11 - a01 * a10) / det}};
  const double t[3] = {M[3], M[7], M[11]};
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) out[4 * r + c] = (float)inv[r][c];
    out[4 * r + 3] = (float)(-((inv[r][0] * t[0] + inv[r][1] * t[1]) + inv[r][2] * t[2]));
  }
}

static inline void to_object(const float* m, v3f o, v3f d, v3f* oo, v3f* od) {
  *oo = V3(((m[0] * o.x + m[1] * o.y) + m[2] * o.z) + m[3], ((m[4] * o.x + m[5] * o.y) + m[6] * o.z) + m[7],
           ((m[8] * o.x + m[9] * o.y) + m[10] * o.z) + m[11]);
  *od = V3((m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
           (m[8] * d.x + m[9] * d.y) + m[10] * d.z);
}

static chit closest(const oscene* s, v3f o, v3f d) {
  if (!s->ninst) return closest_flat(s, o, d);
  chit best; best.pos = -1; best.t = FLT_MAX; best.u = best.v = 0; best.t2 = FLT_MAX; best.gid = -1; best.inst = -1;
  for (int i = 0; i < s->ninst; ++i) {
    const oscene* m = (const oscene*)s->inst_mesh[i];
    v3f oo, od;
    to_object(s->inst_minv + 12 * i, o, d, &oo, &od);
    chit h = closest_flat(m, oo, od);
    if (h.t2 < best.t2) best.t2 = h.t2;
    if (h.pos < 0) continue;
    int gid = s->inst_id_off[i] + m->id[h.pos];
    int better = best.pos < 0 || h.t < best.t || (h.t == best.t && gid > best.gid);
    if (better) {
      if (best.pos >= 0 && best.t < best.t2) best.t2 = best.t;
      best.pos = h.pos; best.t = h.t; best.u = h.u; best.v = h.v; best.gid = gid; best.inst = i;
    } else if (h.t < best.t2) {
      best.t2 = h.t;
    }
  }
  return best;
}

static int any_hit(const oscene* s, v3f o, v3f d) {
  if (!s->ninst) return any_hit_flat(s, o, d);
  for (int i = 0; i < s->ninst; ++i) {
    v3f oo, od;
    to_object(s->inst_minv + 12 * i, o, d, &oo, &od);
    if (any_hit_flat((const oscene*)s->inst_mesh[i], oo, od)) return 1;
  }
  return 0;
}

void* oracle_instanced_create(void* const* meshes, const int32_t* mesh_of, const float* transforms,
                              const int32_t* mat_base, int ninst, const float* mats, int nobj, const float* lights,
                              int nl) {
  oscene* s = (oscene*)calloc(1, sizeof(oscene));
  s->ninst = ninst; s->nobj = nobj; s->nl = nl; s->ambient = 1.0f;
  s->inst_mesh = malloc(sizeof(void*) * (size_t)ninst);
  s->inst_minv = malloc(sizeof(float) * 12 * (size_t)ninst);
  s->inst_id_off = malloc(sizeof(int32_t) * (size_t)ninst);
  s->inst_mat_base = malloc(sizeof(int32_t) * (size_t)ninst);
  int total = 0;
  for (int i = 0; i < ninst; ++i) {
    s->inst_mesh[i] = meshes[mesh_of[i]];
    affine_inverse_d(transforms + 12 * i, s->inst_minv + 12 * i);
    s->inst_id_off[i] = total;
    s->inst_mat_base[i] = mat_base[i];
    total += ((const oscene*)meshes[mesh_of[i]])->nt;
  }
  s->nt = total;
  s->mats = malloc(sizeof(float) * OMAT * (size_t)(nobj > 0 ? nobj : 1));
  memcpy(s->mats, mats, sizeof(float) * OMAT * (size_t)nobj);
  s->lights = malloc(sizeof(float) * 6 * (size_t)(nl > 0 ? nl : 1));
  memcpy(s->lights, lights, sizeof(float) * 6 * (size_t)nl);
  return s;
}

/* ---------------------------------------------------------------- FP32 render */
static inline uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}

/* 1 / n as RayTracer::renderWithAA computes it: `1.0 / (float) aaSamples`, a double
 * division stored as float (src/RayTracer.cpp:211). */
static inline float grid_step(int n) { return (float)(1.0 / (double)(float)n); }

/* Sub-pixel offsets of sample `s` of pixel `p`: the pixel offset for spp == 1; with grid n
 * the reference's n x n anti-aliasing grid, sample s = q n + p at (p + ksi, q + ksi) / n with
 * ksi = rand() / RAND_MAX, integer division, 0 (src/RayTracer.cpp:214-227); else a hashed
 * jitter in [0, 1). */
static inline void sample_offset(uint32_t p, int smp, int spp, uint32_t seed, float off,
                                 float* ox, float* oy, int grid) {
  if (grid > 0) {
    const float st = grid_step(grid);
    *ox = (float)(smp % grid) * st;
    *oy = (float)(smp / grid) * st;
    return;
  }
  if (spp <= 1) { *ox = off; *oy = off; return; }
  uint32_t h1 = hash32(p * 0x9E3779B9u ^ hash32((uint32_t)smp * 0x85EBCA6Bu + seed));
  uint32_t h2 = hash32(h1 ^ 0x68E31DA4u);
  *ox = (float)(h1 >> 8) * (1.0f / 16777216.0f);
  *oy = (float)(h2 >> 8) * (1.0f / 16777216.0f);
}

/* Weight of a sample in its pixel: 1 / spp, or the grid's inv_aaSamplesSquared (:212). */
static inline float sample_weight(int spp, int grid) {
  if (grid > 0) { const float st = grid_step(grid); return st * st; }
  return 1.0f / (float)spp;
}

static inline v3f primary_dir(const float* cam, int w, int hgt, int x, int y, float ox, float oy) {
  float nw = w / 2.0f, nh = hgt / 2.0f;
  float inw = 1.0f / nw, inh = 1.0f / nh;
  float bb = (((float)y + oy) - nh) * inh;
  float aa = (((float)x + ox) - nw) * inw;
  v3f right = V3(cam[6], cam[7], cam[8]), up = V3(cam[9], cam[10], cam[11]), view = V3(cam[3], cam[4], cam[5]);
  v3f d = vadd(vadd(vscale(aa, right), vscale(bb, up)), view);
  return vnorm(d);
}

/* Hit point and shading normal (src/Triangle.cpp:41-46, src/BVH.cpp:379-380). */
static inline void hit_geometry(const oscene* s, int p, v3f o, v3f d, float t, float u, float v,
                                v3f* P, v3f* N) {
  *P = vadd(o, vscale(t, d));
  float w = (1.0f - u) - v;
  v3f a = vscale(w, s->n1[p]), b = vscale(u, s->n2[p]), c = vscale(v, s->n3[p]);
  v3f n = vnorm(vadd(vadd(a, b), c));
  *N = vnorm(n);
}

/* The hit's point, normal and object (either kind of scene). */
static inline void hit_shading(const oscene* s, const chit* h, v3f o, v3f d, v3f* P, v3f* N, int* obj) {
  if (!s->ninst) {
    hit_geometry(s, h->pos, o, d, h->t, h->u, h->v, P, N);
    *obj = (int)s->obj[h->pos];
    return;
  }
  const oscene* m = (const oscene*)s->inst_mesh[h->inst];
  const float* M = s->inst_minv + 12 * h->inst;
  int p = h->pos;
  *P = vadd(o, vscale(h->t, d));
  float w = (1.0f - h->u) - h->v;
  v3f a = vscale(w, m->n1[p]), b = vscale(h->u, m->n2[p]), c = vscale(h->v, m->n3[p]);
  v3f n = vnorm(vadd(vadd(a, b), c));
  v3f nw = V3((M[0] * n.x + M[4] * n.y) + M[8] * n.z, (M[1] * n.x + M[5] * n.y) + M[9] * n.z,
              (M[2] * n.x + M[6] * n.y) + M[10] * n.z);
  *N = vnorm(nw);
  *obj = (int)m->obj[p] + s->inst_mat_base[h->inst];
}

/* RayTracer::calcPhong for one light (src/RayTracer.cpp:418-458). */
static inline v3f phong_one(const float* m, const float* l, v3f P, v3f N, v3f cam) {
  v3f L = vnorm(vsub(V3(l[0], l[1], l[2]), P));
  v3f Vv = vnorm(vsub(cam, P));
  float ndl = vdot(N, L);
  float two = 2.0f * ndl;
  v3f R = vnorm(vsub(vscale(two, N), L));
  float dd = vdot(L, N);
  dd = dd > 0.0f ? dd : 0.0f;
  v3f diff = V3((dd * m[0]) * l[3], (dd * m[1]) * l[4], (dd * m[2]) * l[5]);
  float vr = vdot(Vv, R);
  if (vr > 0.0f) {
    float st = powf(vr, m[6]);
    v3f sp = V3((st * l[3]) * m[3], (st * l[4]) * m[4], (st * l[5]) * m[5]);
    return vadd(diff, sp);
  }
  return diff;
}

/* RayTracer::fresnel (src/RayTracer.cpp:52-64). */
static inline float fresnel_f(v3f incident, v3f normal, float n1, float n2) {
  float n = n1 / n2;
  float cos_i = -vdot(normal, incident);
  float sin_t2 = (n * n) * (1.0f - cos_i * cos_i);
  if (sin_t2 > 1.0f) return 1.0f;
  float cos_t = sqrtf(1.0f - sin_t2);
  float r_orth = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
  float r_par = (n2 * cos_i - n1 * cos_t) / (n2 * cos_i + n1 * cos_t);
  return (r_orth * r_orth + r_par * r_par) / 2.0f;
}

static inline v3f reflect_f(v3f d, v3f n) {
  float dn = vdot(n, d);
  return V3(d.x - ((n.x * dn) * 2.0f), d.y - ((n.y * dn) * 2.0f), d.z - ((n.z * dn) * 2.0f));
}

/* The secondary ray of a hit (RayTracer::shadeIntersection, src/RayTracer.cpp:329-407):
 * reflective -> mirror ray from P + 1e-3 R, weight = reflectivity; transparent -> the
 * reference traces the mirror ray about the incident-side normal from P + 1e-3 n twice
 * (:401 and, instead of the refracted ray, :403) and mixes K c + (1 - K) c with the
 * Fresnel K; *K_out = K, *transp = 1 then.  Returns 0 when no ray is spawned. */
static inline int secondary_f(const float* m, float ambient, v3f d, v3f P, v3f N, v3f* ro, v3f* rd, float* w,
                              int* transp) {
  const float eps = 1e-3f;
  *transp = 0;
  if (m[7] > 0.0f) {
    *rd = vnorm(reflect_f(d, N));
    *ro = vadd(P, vscale(eps, *rd));
    *w = m[7];
    return 1;
  }
  if (m[8] > 0.0f) {
    v3f inc = vnorm(d);
    v3f n = N;
    float n1 = ambient, n2 = m[9];
    if (!(vdot(inc, N) < 0.0f)) {
      n1 = m[9];
      n2 = ambient;
      n = vsub(V3(0.0f, 0.0f, 0.0f), N);
    }
    *w = fresnel_f(inc, n, n1, n2);
    *rd = vnorm(reflect_f(d, n));
    *ro = vadd(P, vscale(eps, n));
    *transp = 1;
    return 1;
  }
  return 0;
}

typedef struct { long long prim, shadow, second; } counts_t;

static v3f trace_path(const oscene* s, const float* cam, v3f o, v3f d, int trace_depth, int32_t* hits,
                      uint32_t* shadows, uint32_t* flags, counts_t* cnt) {
  v3f phong[MAXB];
  float wgt[MAXB];
  int transp[MAXB];
  int nb = 0;
  v3f campos = V3(cam[0], cam[1], cam[2]);
  const float eps = 1e-3f;
  for (int k = 0; k < MAXB; ++k) {
    if (k > trace_depth) break;
    if (k == 0) cnt->prim++; else cnt->second++;
    if (d.x == 0.0f || d.y == 0.0f || d.z == 0.0f) *flags |= FLAG_AXIS_PARALLEL;
    chit h = closest(s, o, d);
    if (h.pos < 0) { hits[k] = HIT_NONE; break; }
    hits[k] = h.gid;
    if (h.t2 < FLT_MAX && fbits(h.t2) - fbits(h.t) <= 2u) *flags |= FLAG_TIE;
    if (h.t < 1e-3f || h.t > 999.0f) *flags |= FLAG_OUT_OF_RANGE;
    v3f P, N;
    int ob;
    hit_shading(s, &h, o, d, &P, &N, &ob);
    const float* m = s->mats + OMAT * ob;
    v3f acc = V3(0, 0, 0);
    uint32_t mask = 0;
    for (int li = 0; li < s->nl; ++li) {
      const float* l = s->lights + 6 * li;
      v3f sd = vnorm(vsub(V3(l[0], l[1], l[2]), P));
      v3f so = vadd(P, vscale(eps, sd));
      cnt->shadow++;
      if (sd.x == 0.0f || sd.y == 0.0f || sd.z == 0.0f) *flags |= FLAG_AXIS_PARALLEL;
      int occ = any_hit(s, so, sd);
      if (occ) {
        mask |= 1u << li;
        chit sh = closest(s, so, sd);
        if (sh.pos >= 0 && sh.t < 1e-3f) *flags |= FLAG_NEAR_ORIGIN;
      } else {
        acc = vadd(acc, phong_one(m, l, P, N, campos));
      }
    }
    shadows[k] = mask;
    phong[k] = acc;
    wgt[k] = 0.0f;
    transp[k] = 0;
    nb = k + 1;
    v3f ro, rd;
    if (!secondary_f(m, s->ambient, d, P, N, &ro, &rd, &wgt[k], &transp[k])) break;
    o = ro;
    d = rd;
  }
  /* c_k = (phong_k + refl_k c_{k+1}) + 0 for a mirror bounce, (phong_k + 0) +
   * (K c_{k+1} + (1 - K) c_{k+1}) for a transparent one (src/RayTracer.cpp:356-357,405,410) */
  v3f c = V3(0, 0, 0);
  for (int k = nb - 1; k >= 0; --k) {
    if (transp[k]) {
      float K = wgt[k], L1 = 1.0f - K;
      c = vadd(phong[k], vadd(vscale(K, c), vscale(L1, c)));
    } else {
      c = vadd(phong[k], vscale(wgt[k], c));
    }
  }
  return c;
}

/* ---------------------------------------------------------------- ray trees
 * A material that is both reflective and transparent makes the reference trace the
 * mirror ray (src/RayTracer.cpp:339-351) and then the transparent bounce's ray (:353-407)
 * from the same hit, so a path is a binary tree of rays.  Nodes in heap order: node 0 the
 * primary ray, node j's mirror child 2j + 1 and transparent child 2j + 2 (node j lies at
 * bounce floor(log2(j + 1))); a record holds 2^(trace_depth + 1) - 1 nodes.  Colour of a
 * node as :410 sums it: (phong + refl c_mirror) + (K c_t + (1 - K) c_t), an absent term
 * being 0; a child beyond trace_depth is not traced and contributes 0 (:275-276). */
static v3f trace_node(const oscene* s, const float* cam, v3f o, v3f d, int depth, int node, int trace_depth,
                      int32_t* hits, uint32_t* shadows, uint32_t* flags, counts_t* cnt) {
  const v3f zero = V3(0.0f, 0.0f, 0.0f);
  if (depth > trace_depth) return zero;
  const float eps = 1e-3f;
  v3f campos = V3(cam[0], cam[1], cam[2]);
  if (depth == 0) cnt->prim++; else cnt->second++;
  if (d.x == 0.0f || d.y == 0.0f || d.z == 0.0f) *flags |= FLAG_AXIS_PARALLEL;
  chit h = closest(s, o, d);
  if (h.pos < 0) { hits[node] = HIT_NONE; return zero; }
  hits[node] = h.gid;
  if (h.t2 < FLT_MAX && fbits(h.t2) - fbits(h.t) <= 2u) *flags |= FLAG_TIE;
  if (h.t < 1e-3f || h.t > 999.0f) *flags |= FLAG_OUT_OF_RANGE;
  v3f P, N;
  int ob;
  hit_shading(s, &h, o, d, &P, &N, &ob);
  const float* m = s->mats + OMAT * ob;
  v3f phong = zero;
  uint32_t mask = 0;
  for (int li = 0; li < s->nl; ++li) {
    const float* l = s->lights + 6 * li;
    v3f sd = vnorm(vsub(V3(l[0], l[1], l[2]), P));
    v3f so = vadd(P, vscale(eps, sd));
    cnt->shadow++;
    if (sd.x == 0.0f || sd.y == 0.0f || sd.z == 0.0f) *flags |= FLAG_AXIS_PARALLEL;
    if (any_hit(s, so, sd)) {
      mask |= 1u << li;
      chit sh = closest(s, so, sd);
      if (sh.pos >= 0 && sh.t < 1e-3f) *flags |= FLAG_NEAR_ORIGIN;
    } else {
      phong = vadd(phong, phong_one(m, l, P, N, campos));
    }
  }
  shadows[node] = mask;
  v3f reflected = zero, refracted = zero;
  if (m[7] > 0.0f) {  /* mirror ray (:339-351) */
    v3f rd = vnorm(reflect_f(d, N));
    v3f ro = vadd(P, vscale(eps, rd));
    v3f c = trace_node(s, cam, ro, rd, depth + 1, 2 * node + 1, trace_depth, hits, shadows, flags, cnt);
    reflected = vscale(m[7], c);
  }
  if (m[8] > 0.0f) {  /* transparent: the mirror ray about the incident-side normal, traced for both halves of the mix */
    v3f inc = vnorm(d);
    v3f n = N;
    float n1 = s->ambient, n2 = m[9];
    if (!(vdot(inc, N) < 0.0f)) {
      n1 = m[9];
      n2 = s->ambient;
      n = vsub(zero, N);
    }
    float K = fresnel_f(inc, n, n1, n2);
    v3f rd = vnorm(reflect_f(d, n));
    v3f ro = vadd(P, vscale(eps, n));
    v3f c = trace_node(s, cam, ro, rd, depth + 1, 2 * node + 2, trace_depth, hits, shadows, flags, cnt);
    refracted = vadd(vscale(K, c), vscale(1.0f - K, c));
  }
  return vadd(vadd(phong, reflected), refracted);
}

/* As oracle_render with ray trees: hits / shadows [npix*spp, 2^(trace_depth+1) - 1] in heap
 * order (nodes not reached: HIT_UNTRACED, mask 0). */
int oracle_render_tree(void* h, const float* cam, int w, int hgt, float pixel_offset, int trace_depth,
                       int spp, uint32_t jitter_seed, const int32_t* pix, int npix, int nthreads,
                       float* rgb, int32_t* hits, uint32_t* shadows, uint32_t* flags, long long* counts, int grid) {
  const oscene* s = (const oscene*)h;
  if (trace_depth < 0 || trace_depth >= MAXB) return -1;
  const int nn = (1 << (trace_depth + 1)) - 1;
  int n = pix ? npix : w * hgt;
  if (spp < 1) spp = 1;
  long long c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 32) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : c0, c1, c2)
  for (int i = 0; i < n; ++i) {
    int p = pix ? pix[i] : i;
    int x = p % w, y = p / w;
    v3f sum = V3(0, 0, 0);
    counts_t cnt = {0, 0, 0};
    int32_t hh[(1 << MAXB) - 1];
    uint32_t ss[(1 << MAXB) - 1];
    for (int smp = 0; smp < spp; ++smp) {
      size_t r = (size_t)i * spp + smp;
      uint32_t fl = 0;
      for (int k = 0; k < nn; ++k) { hh[k] = HIT_UNTRACED; ss[k] = 0; }
      float ox, oy;
      sample_offset((uint32_t)p, smp, spp, jitter_seed, pixel_offset, &ox, &oy, grid);
      v3f d = primary_dir(cam, w, hgt, x, y, ox, oy);
      v3f c = trace_node(s, cam, V3(cam[0], cam[1], cam[2]), d, 0, 0, trace_depth, hh, ss, &fl, &cnt);
      sum = vadd(sum, c);
      if (hits) memcpy(hits + r * nn, hh, sizeof(int32_t) * nn);
      if (shadows) memcpy(shadows + r * nn, ss, sizeof(uint32_t) * nn);
      if (flags) flags[r] = fl;
    }
    if (spp > 1 || grid > 0) sum = vscale(sample_weight(spp, grid), sum);
    rgb[3 * (size_t)i] = sum.x; rgb[3 * (size_t)i + 1] = sum.y; rgb[3 * (size_t)i + 2] = sum.z;
    c0 += cnt.prim; c1 += cnt.shadow; c2 += cnt.second;
  }
  if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
  return 0;
}

/* rgb [npix,3]; hits/shadows [npix*spp, 8]; flags [npix*spp]; counts [3]. */
int oracle_render(void* h, const float* cam, int w, int hgt, float pixel_offset, int trace_depth,
                  int spp, uint32_t jitter_seed, const int32_t* pix, int npix, int nthreads,
                  float* rgb, int32_t* hits, uint32_t* shadows, uint32_t* flags, long long* counts, int grid) {
  const oscene* s = (const oscene*)h;
  int n = pix ? npix : w * hgt;
  if (spp < 1) spp = 1;
  long long c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 32) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : c0, c1, c2)
  for (int i = 0; i < n; ++i) {
    int p = pix ? pix[i] : i;
    int x = p % w, y = p / w;
    v3f sum = V3(0, 0, 0);
    counts_t cnt = {0, 0, 0};
    for (int smp = 0; smp < spp; ++smp) {
      size_t r = (size_t)i * spp + smp;
      int32_t hh[MAXB]; uint32_t ss[MAXB]; uint32_t fl = 0;
      for (int k = 0; k < MAXB; ++k) { hh[k] = HIT_UNTRACED; ss[k] = 0; }
      float ox, oy;
      sample_offset((uint32_t)p, smp, spp, jitter_seed, pixel_offset, &ox, &oy, grid);
      v3f d = primary_dir(cam, w, hgt, x, y, ox, oy);
      v3f c = trace_path(s, cam, V3(cam[0], cam[1], cam[2]), d, trace_depth, hh, ss, &fl, &cnt);
      sum = vadd(sum, c);
      if (hits) memcpy(hits + r * MAXB, hh, sizeof hh);
      if (shadows) memcpy(shadows + r * MAXB, ss, sizeof ss);
      if (flags) flags[r] = fl;
    }
    if (spp > 1 || grid > 0) sum = vscale(sample_weight(spp, grid), sum);
    rgb[3 * (size_t)i] = sum.x; rgb[3 * (size_t)i + 1] = sum.y; rgb[3 * (size_t)i + 2] = sum.z;
    c0 += cnt.prim; c1 += cnt.shadow; c2 += cnt.second;
  }
  if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
  return 0;
}

/* Nearest / any hit of arbitrary rays [n,6]: ids (-1 = miss), t, near-tie flag. */
void oracle_closest(void* h, const float* rays, int n, int32_t* ids, float* ts, uint8_t* tie) {
  const oscene* s = (const oscene*)h;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 6 * (size_t)i;
    chit c = closest(s, V3(r[0], r[1], r[2]), V3(r[3], r[4], r[5]));
    ids[i] = c.pos < 0 ? HIT_NONE : c.gid;
    if (ts) ts[i] = c.pos < 0 ? FLT_MAX : c.t;
    if (tie) tie[i] = (c.pos >= 0 && c.t2 < FLT_MAX && fbits(c.t2) - fbits(c.t) <= 2u) ? 1 : 0;
  }
}

void oracle_any(void* h, const float* rays, int n, uint8_t* occ) {
  const oscene* s = (const oscene*)h;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 6 * (size_t)i;
    occ[i] = (uint8_t)any_hit(s, V3(r[0], r[1], r[2]), V3(r[3], r[4], r[5]));
  }
}

/* Brute force over every triangle (validates the BVH culling above on small scenes). */
void oracle_closest_brute(void* h, const float* rays, int n, int32_t* ids, float* ts) {
  const oscene* s = (const oscene*)h;
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 6 * (size_t)i;
    v3f o = V3(r[0], r[1], r[2]), d = V3(r[3], r[4], r[5]);
    int best = -1; float bt = FLT_MAX;
    for (int p = 0; p < s->nt; ++p) {
      float t, u, v;
      if (!mt_hit(o, d, s->v1[p], s->e1[p], s->e2[p], &t, &u, &v)) continue;
      if (best < 0 || t < bt || (t == bt && s->id[p] > s->id[best])) { best = p; bt = t; }
    }
    ids[i] = best < 0 ? HIT_NONE : s->id[best];
    if (ts) ts[i] = bt;
  }
}

/* ---------------------------------------------------------------- FP64 adjoint */
typedef struct { double x, y, z; } v3d;
static inline v3d D3(double x, double y, double z) { v3d r = {x, y, z}; return r; }
static inline v3d dadd(v3d a, v3d b) { return D3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3d dsub(v3d a, v3d b) { return D3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3d dsc(double s, v3d a) { return D3(s * a.x, s * a.y, s * a.z); }
static inline double ddot(v3d a, v3d b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3d dcross(v3d a, v3d b) { return D3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
static inline double dlen(v3d a) { return sqrt(ddot(a, a)); }
static inline v3d dnorm(v3d a) { return dsc(1.0 / dlen(a), a); }
static inline v3d f2d(v3f a) { return D3(a.x, a.y, a.z); }

/* Parameters: per object [kd r,g,b, ks r,g,b, log shininess, reflectivity, transparency,
 * refractive index] (OMAT doubles),
 * per light [position xyz, colour rgb] (6 doubles).  Gradients: per object
 * [kd rgb, ks rgb, log shininess] (7), per light [colour rgb, position xyz] (6). */
typedef struct {
  const oscene* s;
  const double* mp;  /* nobj x OMAT */
  const double* lp;  /* nl x 6 */
} f64ctx;

/* One node of a frozen path in FP64: re-derive the hit from the stored triangle id, shade
 * it and recurse into the secondary rays; when g != NULL accumulate the adjoint of
 * <g, colour>.  T = the product of the weights from the primary ray: reflectivity for a
 * mirror edge, 1 for a transparent one (its Fresnel mix K c + (1 - K) c of one colour).
 * Records: chain form (tree = 0, slot = bounce k; one secondary ray per hit, the mirror
 * ray before the transparent one as the chain renderer takes them) or tree form (tree = 1,
 * slot = heap node: mirror child 2j + 1, transparent child 2j + 2, both traced). */
static void f64_node(const f64ctx* c, v3d campos, v3d o, v3d d, int k, int node, double T, const int32_t* hits,
                     const uint32_t* shadows, int tree, int trace_depth, const double* g, double* gm, double* gl,
                     v3d* col) {
  const oscene* s = c->s;
  const int slot = tree ? node : k;
  const int id = hits[slot];
  if (id < 0) return;
  const uint32_t mask = shadows[slot];
  /* the triangle: flat scene, or (two-level) the instance holding global id `id`, its
   * mesh, the ray in object space (o' = Minv [o, 1], d' = Minv [d, 0]: t is the same
   * parameter) and the normal back through Minv^T */
  const oscene* ms = s;
  const float* minv = NULL;
  int base = 0, local = id;
  if (s->ninst) {
    int lo = 0, hi = s->ninst - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (s->inst_id_off[mid] <= id) lo = mid; else hi = mid - 1;
    }
    ms = (const oscene*)s->inst_mesh[lo];
    minv = s->inst_minv + 12 * lo;
    base = s->inst_mat_base[lo];
    local = id - s->inst_id_off[lo];
  }
  int p = ms->pos_of_id[local];
  v3d oo = o, od = d;
  if (minv) {
    oo = D3(minv[0] * o.x + minv[1] * o.y + minv[2] * o.z + minv[3],
            minv[4] * o.x + minv[5] * o.y + minv[6] * o.z + minv[7],
            minv[8] * o.x + minv[9] * o.y + minv[10] * o.z + minv[11]);
    od = D3(minv[0] * d.x + minv[1] * d.y + minv[2] * d.z, minv[4] * d.x + minv[5] * d.y + minv[6] * d.z,
            minv[8] * d.x + minv[9] * d.y + minv[10] * d.z);
  }
  v3d v1 = f2d(ms->v1[p]), e1 = f2d(ms->e1[p]), e2 = f2d(ms->e2[p]);
  v3d Pm = dcross(od, e2);
  double det = ddot(e1, Pm);
  v3d Tv = dsub(oo, v1);
  v3d Q = dcross(Tv, e1);
  double t = ddot(e2, Q) / det, u = ddot(Tv, Pm) / det, v = ddot(od, Q) / det;
  v3d P = dadd(o, dsc(t, d));
  v3d n = dadd(dadd(dsc(1.0 - u - v, f2d(ms->n1[p])), dsc(u, f2d(ms->n2[p]))), dsc(v, f2d(ms->n3[p])));
  if (minv) {
    n = dnorm(n);
    n = D3(minv[0] * n.x + minv[4] * n.y + minv[8] * n.z, minv[1] * n.x + minv[5] * n.y + minv[9] * n.z,
           minv[2] * n.x + minv[6] * n.y + minv[10] * n.z);
  }
  v3d N = dnorm(n);
  int ob = (int)ms->obj[p] + base;
  const double* m = c->mp + OMAT * ob;
  double shin = exp(m[6]);
  v3d V = dnorm(dsub(campos, P));
  for (int li = 0; li < s->nl; ++li) {
    if (mask & (1u << li)) continue;
    const double* l = c->lp + 6 * li;
    v3d uvec = dsub(D3(l[0], l[1], l[2]), P);
    double ul = dlen(uvec);
    v3d L = dsc(1.0 / ul, uvec);
    double ndl = ddot(N, L);
    v3d wv = dsub(dsc(2.0 * ndl, N), L);
    double wl = dlen(wv);
    v3d R = dsc(1.0 / wl, wv);
    double fd = ndl > 0.0 ? ndl : 0.0;
    double vr = ddot(V, R);
    double fs = vr > 0.0 ? pow(vr, shin) : 0.0;
    double C[3] = {l[3], l[4], l[5]};
    col->x += T * (fd * m[0] * C[0] + fs * C[0] * m[3]);
    col->y += T * (fd * m[1] * C[1] + fs * C[1] * m[4]);
    col->z += T * (fd * m[2] * C[2] + fs * C[2] * m[5]);
    if (!g) continue;
    double* gmo = gm + 7 * ob;
    double* glo = gl + 6 * li;
    double a = 0.0, b = 0.0, sl = 0.0;
    for (int ch = 0; ch < 3; ++ch) {
      double gc = g[ch] * T;
      gmo[ch] += gc * fd * C[ch];
      gmo[3 + ch] += gc * fs * C[ch];
      glo[ch] += gc * (fd * m[ch] + fs * m[3 + ch]);
      a += gc * C[ch] * m[ch];
      b += gc * C[ch] * m[3 + ch];
    }
    if (vr > 0.0) {
      sl = b * fs * log(vr) * shin;
      gmo[6] += sl;
    }
    v3d gp = D3(0, 0, 0);
    if (ndl > 0.0) {
      v3d gd = dsc(1.0 / ul, dsub(N, dsc(ndl, L)));
      gp = dadd(gp, dsc(a, gd));
    }
    if (vr > 0.0) {
      v3d q = dsc(1.0 / wl, dsub(V, dsc(vr, R)));
      v3d q2 = dsub(dsc(2.0 * ddot(N, q), N), q);
      v3d gs = dsc(1.0 / ul, dsub(q2, dsc(ddot(L, q2), L)));
      double dfs = shin * pow(vr, shin - 1.0);
      gp = dadd(gp, dsc(b * dfs, gs));
    }
    glo[3] += gp.x; glo[4] += gp.y; glo[5] += gp.z;
  }
  if (k + 1 > trace_depth) return;
  if (m[7] > 0.0) {
    v3d rd = dnorm(dsub(d, dsc(2.0 * ddot(N, d), N)));
    f64_node(c, campos, dadd(P, dsc(1e-3, rd)), rd, k + 1, 2 * node + 1, T * m[7], hits, shadows, tree,
             trace_depth, g, gm, gl, col);
    if (!tree) return;
  }
  if (m[8] > 0.0) {
    v3d n = ddot(dnorm(d), N) < 0.0 ? N : dsc(-1.0, N);
    v3d rd = dnorm(dsub(d, dsc(2.0 * ddot(n, d), n)));
    f64_node(c, campos, dadd(P, dsc(1e-3, n)), rd, k + 1, 2 * node + 2, T, hits, shadows, tree, trace_depth, g,
             gm, gl, col);
  }
}

/* One frozen path in FP64 from its primary ray (see f64_node). */
static v3d f64_path(const f64ctx* c, const float* cam, int w, int hgt, int x, int y, float ox,
                    float oy, const int32_t* hits, const uint32_t* shadows, int tree, int trace_depth,
                    const double* g, double* gm, double* gl) {
  double nw = w / 2.0, nh = hgt / 2.0;
  double aa = ((x + (double)ox) - nw) / nw, bb = ((y + (double)oy) - nh) / nh;
  v3d campos = D3(cam[0], cam[1], cam[2]);
  v3d d = dnorm(dadd(dadd(dsc(aa, D3(cam[6], cam[7], cam[8])), dsc(bb, D3(cam[9], cam[10], cam[11]))),
                     D3(cam[3], cam[4], cam[5])));
  v3d col = D3(0, 0, 0);
  f64_node(c, campos, campos, d, 0, 0, 1.0, hits, shadows, tree, trace_depth, g, gm, gl, &col);
  return col;
}

/* Frozen-visibility FP64 render of n_views cameras (cams: n_views x 12; every view has
 * w x hgt pixels, spp samples from seed at pixel_offset).  hits / shadows:
 * [n_views*w*hgt*spp, 8] (chain records) or [.., 2^(trace_depth+1) - 1] (tree = 1).
 * rgb_out: [n_views*w*hgt, 3].  If g is non-NULL, also writes gradients of <g, rgb>. */
int oracle_frozen_f64(void* h, const float* cams, int n_views, int w, int hgt, float pixel_offset,
                      int spp, uint32_t seed, int trace_depth, const int32_t* hits, const uint32_t* shadows,
                      const double* mat_params, const double* light_params, double* rgb_out,
                      const double* g, double* grad_mat, double* grad_light, int nthreads, int tree, int grid) {
  /* Paths are per sample (pixel-major, samples of a pixel consecutive, the forward's
   * order); a pixel's colour is the sample mean (on the reference's grid: the sum times
   * (1/n)^2), so each sample's adjoint is g times that weight. */
  const oscene* s = (const oscene*)h;
  f64ctx c = {s, mat_params, light_params};
  size_t npx = (size_t)w * hgt;
  /* record slots per path: 8 bounces (chain form) or the 2^(trace_depth+1) - 1 tree nodes */
  const long long rec = tree ? (1ll << (trace_depth + 1)) - 1 : MAXB;
  if (spp < 1) spp = 1;
  int nth = nthreads > 0 ? nthreads : 1;
  size_t gms = (size_t)7 * s->nobj, gls = (size_t)6 * s->nl;
  double* gmt = g ? calloc((size_t)nth * gms + 1, sizeof(double)) : NULL;
  double* glt = g ? calloc((size_t)nth * gls + 1, sizeof(double)) : NULL;
#pragma omp parallel num_threads(nth)
  {
    int tid = omp_get_thread_num();
#pragma omp for schedule(dynamic, 64)
    for (long long i = 0; i < (long long)(n_views * npx); ++i) {
      int view = (int)(i / (long long)npx);
      int p = (int)(i % (long long)npx);
      const float* cam = cams + 12 * view;
      double gs[3];
      const double wsmp = grid > 0 ? (double)sample_weight(spp, grid) : 1.0 / spp;
      if (g) for (int k = 0; k < 3; ++k) gs[k] = g[3 * i + k] * wsmp;
      v3d sum = D3(0, 0, 0);
      for (int smp = 0; smp < spp; ++smp) {
        float ox, oy;
        sample_offset((uint32_t)p, smp, spp, seed, pixel_offset, &ox, &oy, grid);
        long long path = i * spp + smp;
        v3d col = f64_path(&c, cam, w, hgt, p % w, p / w, ox, oy, hits + rec * path, shadows + rec * path, tree,
                           trace_depth, g ? gs : NULL, g ? gmt + gms * tid : NULL, g ? glt + gls * tid : NULL);
        sum = dadd(sum, col);
      }
      sum = dsc(wsmp, sum);
      if (rgb_out) { rgb_out[3 * i] = sum.x; rgb_out[3 * i + 1] = sum.y; rgb_out[3 * i + 2] = sum.z; }
    }
  }
  if (g) {
    memset(grad_mat, 0, sizeof(double) * gms);
    memset(grad_light, 0, sizeof(double) * gls);
    for (int t = 0; t < nth; ++t) {
      for (size_t k = 0; k < gms; ++k) grad_mat[k] += gmt[gms * t + k];
      for (size_t k = 0; k < gls; ++k) grad_light[k] += glt[gls * t + k];
    }
    free(gmt); free(glt);
  }
  return 0;
}
