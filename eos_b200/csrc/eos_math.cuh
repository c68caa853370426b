// Exact-order float3 arithmetic shared by every kernel on the render path.
//
// The reference's CPU renderer evaluates its vector math through glm 0.9.6, whose
// operation order fixes the rounding of every result (glm/detail/func_geometric.inl):
//   dot(a, b)    = (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a, b)  = (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
//   normalize(a) = a * (1 / sqrt(dot(a, a)))
//   reflect(I,N) = I - (N * dot(N, I)) * 2
// Every translation unit that includes this header is compiled with --fmad=false, so
// a*b + c is a rounded multiply followed by a rounded add, exactly as on the CPU, and
// division and sqrt are IEEE round-to-nearest (no fast-math).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define EOS_HD __host__ __device__ __forceinline__

struct f3 {
  float x, y, z;
};

EOS_HD f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
EOS_HD f3 add3(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
EOS_HD f3 sub3(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
EOS_HD f3 scale3(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
EOS_HD float dot3(f3 a, f3 b) {
  float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z;
  return (x + y) + z;
}
EOS_HD f3 cross3(f3 a, f3 b) {
  return f3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
EOS_HD f3 norm3(f3 a) {
  float s = 1.0f / sqrtf(dot3(a, a));
  return f3{a.x * s, a.y * s, a.z * s};
}
EOS_HD f3 reflect3(f3 i, f3 n) {
  float d = dot3(n, i);
  return f3{i.x - ((n.x * d) * 2.0f), i.y - ((n.y * d) * 2.0f), i.z - ((n.z * d) * 2.0f)};
}

// Moller-Trumbore in the order of Triangle::RayTriangleIntersection
// (src/Triangle.cpp:57-91); e1 = v2 - v1 and e2 = v3 - v1 are precomputed with the same
// subtraction the reference does per test.
EOS_HD bool mt_intersect(f3 o, f3 d, f3 v1, f3 e1, f3 e2, float& t, float& u, float& v) {
  f3 P = cross3(d, e2);
  float det = dot3(e1, P);
  if (det > -0.00001f && det < 0.00001f) return false;
  float inv_det = 1.0f / det;
  f3 T = sub3(o, v1);
  f3 Q = cross3(T, e1);
  float tt = dot3(e2, Q) * inv_det;
  if (tt < 0.0f) return false;
  float uu = dot3(T, P) * inv_det;
  if (uu < 0.0f || uu > 1.0f) return false;
  float vv = dot3(d, Q) * inv_det;
  if (vv < 0.0f || uu + vv > 1.0f) return false;
  t = tt;
  u = uu;
  v = vv;
  return true;
}

// The same test with the rejections evaluated cheapest first; the result (accept and the
// bits of t, u, v) is identical to mt_intersect because acceptance is the conjunction of
// the same five conditions on the same values:
//   u = (T.P) * (1/det), v = (d.Q) * (1/det), t = (e2.Q) * (1/det)
// A product of two floats rounds to a value of the product's sign (or to zero), so when
// a numerator's sign is opposite to det's and its magnitude is far from the underflow
// range, u (v, t) < 0 is decided without the division; misses mostly end there.
__device__ __forceinline__ bool opposite_sign_reject(float num, float det) {
  return (num < 0.0f) != (det < 0.0f) && fabsf(num) > 1e-30f;
}

__device__ __forceinline__ bool mt_intersect_fast(f3 o, f3 d, f3 v1, f3 e1, f3 e2, float& t, float& u, float& v) {
  f3 P = cross3(d, e2);
  float det = dot3(e1, P);
  if (det > -0.00001f && det < 0.00001f) return false;
  f3 T = sub3(o, v1);
  float nu = dot3(T, P);
  if (opposite_sign_reject(nu, det)) return false;  // u < 0
  f3 Q = cross3(T, e1);
  float nv = dot3(d, Q);
  if (opposite_sign_reject(nv, det)) return false;  // v < 0
  float nt = dot3(e2, Q);
  if (opposite_sign_reject(nt, det)) return false;  // t < 0
  float inv_det = 1.0f / det;
  float uu = nu * inv_det;
  if (uu < 0.0f || uu > 1.0f) return false;
  float vv = nv * inv_det;
  if (vv < 0.0f || uu + vv > 1.0f) return false;
  float tt = nt * inv_det;
  if (tt < 0.0f) return false;
  t = tt;
  u = uu;
  v = vv;
  return true;
}

// Primary ray direction of pixel (x, y) with sub-pixel offset (ox, oy)
// (src/RayTracer.cpp:119-145; offset 0 reproduces the reference's integer corners).
EOS_HD f3 primary_direction(const float* cam, int w, int h, int x, int y, float ox, float oy) {
  float nw = w / 2.0f, nh = h / 2.0f;
  float inw = 1.0f / nw, inh = 1.0f / nh;
  float bb = (((float)y + oy) - nh) * inh;
  float aa = (((float)x + ox) - nw) * inw;
  f3 right = mk3(cam[6], cam[7], cam[8]), up = mk3(cam[9], cam[10], cam[11]);
  f3 view = mk3(cam[3], cam[4], cam[5]);
  return norm3(add3(add3(scale3(aa, right), scale3(bb, up)), view));
}

EOS_HD uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Side of the reference's anti-aliasing grid for spp samples per pixel (EOS_FLAG_AA_GRID):
// n with n * n == spp, else 0.
EOS_HD int aa_grid_side(int spp) {
  int n = 1;
  while (n * n < spp) ++n;
  return n * n == spp ? n : 0;
}

// 1 / n as the reference computes it, `1.0 / (float) aaSamples` (double, then float).
EOS_HD float aa_grid_step(int n) { return (float)(1.0 / (double)(float)n); }

// Sub-pixel position of sample `s` of pixel `p`: the fixed offset for one sample per
// pixel; with grid = n > 0 the reference's n x n anti-aliasing grid
// (RayTracer::renderWithAA, src/RayTracer.cpp:214-233): sample s = q n + p at
// ((p + ksi) step, (q + ksi) step), ksi = rand() / RAND_MAX in integer arithmetic = 0;
// otherwise a hashed jitter in [0, 1).
EOS_HD void sample_offset(uint32_t p, int s, int spp, uint32_t seed, float off, float& ox, float& oy,
                          int grid = 0) {
  if (grid > 0) {
    const float step = aa_grid_step(grid);
    ox = (float)(s % grid) * step;
    oy = (float)(s / grid) * step;
    return;
  }
  if (spp <= 1) {
    ox = off;
    oy = off;
    return;
  }
  uint32_t h1 = hash32(p * 0x9E3779B9u ^ hash32((uint32_t)s * 0x85EBCA6Bu + seed));
  uint32_t h2 = hash32(h1 ^ 0x68E31DA4u);
  ox = (float)(h1 >> 8) * (1.0f / 16777216.0f);
  oy = (float)(h2 >> 8) * (1.0f / 16777216.0f);
}

// Weight of one sample in its pixel: 1 / spp, or on the reference's grid its
// inv_aaSamplesSquared = step * step (src/RayTracer.cpp:212,237).
EOS_HD float sample_weight(int spp, int grid) {
  if (grid > 0) {
    const float step = aa_grid_step(grid);
    return step * step;
  }
  return 1.0f / (float)spp;
}

// 30-bit Morton code: two zero bits inserted after each of the 10 low bits of x, y, z,
// code = (z' << 2) + (y' << 1) + x'  (src/morton.h:30-48).
EOS_HD uint32_t spread_bits_by_2(uint32_t x) {
  x &= 0x000003ffu;
  x = (x ^ (x << 16)) & 0xff0000ffu;
  x = (x ^ (x << 8)) & 0x0300f00fu;
  x = (x ^ (x << 4)) & 0x030c30c3u;
  x = (x ^ (x << 2)) & 0x09249249u;
  return x;
}
EOS_HD uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return (spread_bits_by_2(z) << 2) + (spread_bits_by_2(y) << 1) + spread_bits_by_2(x);
}
