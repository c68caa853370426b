// Test-only harness around the reference's own CPU renderer.
//
// This file is test infrastructure: it is linked with the reference's CPU sources
// (src/Scene.cpp, src/RayTracer.cpp, src/BVH.cpp, src/Triangle.cpp, src/Box.cu,
// src/Material.cpp, src/RayIntersection.cpp, src/LightSource.cpp, src/getTime.cpp)
// into oracle/_ref/libeosref.so by oracle/Makefile.  Only the tests, the smoke check
// and the CPU-baseline leg of the benchmark load it.  It never ships with the product.
//
// What it adds on top of the reference:
//  * builds a Scene of Triangle surfaces from flat float32 arrays with identity
//    transforms (src/Scene.cpp:47-106, src/Triangle.h:35-41);
//  * gives every triangle its own material index (a per-triangle copy of its object's
//    Material) so the hit triangle id can be read back from
//    RayIntersection::getMaterialIndex (src/RayIntersection.h:51-55, src/Triangle.cpp:50-51);
//  * evaluates the reference's private RayTracer::rayTrace per pixel to get the FP32
//    colour before the 8-bit quantisation of src/RayTracer.cpp:150-153;
//  * replays the bounce path (closest hit, per-light shadow ray, mirror ray) through the
//    public Scene queries with the ray construction of src/RayTracer.cpp:119-145,326-359.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stack>
#include <vector>
#include <omp.h>
#include <glm/glm.hpp>
#include <glm/gtx/type_aligned.hpp>

// RayTracer::rayTrace is private in the reference; the harness needs it to read the
// FP32 colour of one primary ray.  Standard headers are included above, so the macro
// only reaches the reference's own class definitions.
#define private public
#include "RayTracer.h"
#include "Scene.h"
#include "Triangle.h"
#include "morton.h"
#undef private

double getRealTime();

namespace {

constexpr int kMaxBounces = 8;
constexpr int32_t kHitNone = -1;      // ray traced, nothing hit
constexpr int32_t kHitUntraced = -2;  // bounce not reached

struct RefScene {
  Scene scene;
  glm::mat4 identity{1.0f};
  glm::mat4 identity_inv{1.0f};
  glm::mat4 identity_inv_t{1.0f};
  std::vector<Material> object_materials;
  // per-object transformations of eosref_scene_create_transformed (sized once: the
  // triangles keep pointers into them)
  std::vector<glm::mat4> xf, xf_inv, xf_inv_t;
  std::vector<Triangle*> triangles;
  std::vector<LightSource*> lights;
  int max_leaf = 0;
  int n_nodes = 0;
};

Camera make_camera(const float* c, int w, int h) {
  Camera cam;
  cam.setPosition(glm::vec3(c[0], c[1], c[2]));
  cam.setViewingDirection(glm::vec3(c[3], c[4], c[5]));
  cam.setRightVector(glm::vec3(c[6], c[7], c[8]));
  cam.setUpVector(glm::vec3(c[9], c[10], c[11]));
  cam.setWidth(w);
  cam.setHeight(h);
  return cam;
}

// Primary ray of pixel (x, y), src/RayTracer.cpp:119-145; pixel_offset 0 is the
// reference's own integer-corner convention, 0.5 samples pixel centres.
Ray primary_ray(const Camera& camera, int x, int y, float ox, float oy) {
  float norm_width = camera.getWidth() / 2.0f;
  float norm_height = camera.getHeight() / 2.0f;
  float inv_norm_width = 1.0f / norm_width;
  float inv_norm_height = 1.0f / norm_height;
  float bb = (((float)y + oy) - norm_height) * inv_norm_height;
  float aa = (((float)x + ox) - norm_width) * inv_norm_width;
  glm::vec3 d = (aa * camera.getRightVector()) + (bb * camera.getUpVector()) + camera.getViewingDirection();
  d = glm::normalize(d);
  Ray ray;
  ray.setOrigin(camera.getPosition());
  ray.setDirection(d);
  return ray;
}

// Bounce path of one primary ray: the same queries and ray construction as
// RayTracer::rayTrace / shadeIntersection (src/RayTracer.cpp:268-359).
void replay_path(const RefScene& rs, Ray ray, int trace_depth, int32_t* hits,
                 uint32_t* shadows, long long* cnt) {
  const float epsilon = 1e-3f;
  const Scene& scene = rs.scene;
  for (int depth = 0; depth < kMaxBounces; ++depth) {
    if (depth > trace_depth) return;
    RayIntersection isect;
    cnt[depth == 0 ? 0 : 2]++;
    bool hit = scene.findMinDistanceIntersectionBVH(ray, isect);
    if (!hit) {
      hits[depth] = kHitNone;
      return;
    }
    int id = isect.getMaterialIndex();
    hits[depth] = id;
    const glm::vec3& P = isect.getPoint();
    uint32_t mask = 0;
    int nl = scene.getNumLightSources();
    for (int i = 0; i < nl; ++i) {
      const LightSource* light = scene.getLightSource(i);
      glm::vec3 sd = glm::normalize(glm::vec3(light->getPosition()) - P);
      glm::vec3 so = P + epsilon * sd;
      Ray sray;
      sray.setOrigin(so);
      sray.setDirection(sd);
      cnt[1]++;
      if (scene.shadowRayVisibilityBVH(sray)) mask |= 1u << i;
    }
    shadows[depth] = mask;
    const Material& m = scene.getMaterialAtIndex(id);
    if (m.isReflective()) {  // src/RayTracer.cpp:339-351
      glm::vec3 rd = glm::normalize(glm::reflect(ray.getDirection(), isect.getNormal()));
      glm::vec3 ro = P + epsilon * rd;
      ray.setOrigin(ro);
      ray.setDirection(rd);
    } else if (m.isTransparent()) {  // src/RayTracer.cpp:353-407: the reflected ray, traced twice
      glm::vec3 incident = glm::normalize(ray.getDirection());
      glm::vec3 n = isect.getNormal();
      if (!(glm::dot(incident, n) < 0.0f)) n = glm::vec3(0.0f) - isect.getNormal();
      glm::vec3 rd = glm::normalize(glm::reflect(ray.getDirection(), n));
      glm::vec3 ro = P + epsilon * n;
      ray.setOrigin(ro);
      ray.setDirection(rd);
    } else {
      return;
    }
  }
}

// The reference Scene with its surfaces, materials and lights, before Scene::flush.
RefScene* make_scene(const float* verts, const float* normals, const uint32_t* tris, const uint32_t* tri_obj,
                     int nt, const float* mats, int nobj, const float* lights, int nl) {
  RefScene* rs = new RefScene();
  rs->object_materials.resize(nobj);
  // materials: kd rgb, ks rgb, shininess, reflectivity, transparency, refractive index
  for (int k = 0; k < nobj; ++k) {
    const float* m = mats + 10 * k;
    Material mat(0.0f, glm::vec4(m[0], m[1], m[2], 1.0f), glm::vec4(m[3], m[4], m[5], 1.0f),
                 (int)m[6]);
    mat.setReflective(m[7] > 0.0f);
    mat.setReflectionIntensity(m[7]);
    mat.setTransparent(m[8] > 0.0f);
    mat.setRefractiveIndex(m[9]);
    rs->object_materials[k] = mat;
  }
  rs->scene.setMaxTracedDepth(8);
  rs->scene.setAmbientRefractiveIndex(1.0f);
  rs->scene.useBvh(true);
  rs->scene.setAASamples(1);
  rs->triangles.resize(nt);
  for (int i = 0; i < nt; ++i) {
    const uint32_t* t = tris + 3 * i;
    glm::vec3 v[3], n[3];
    for (int j = 0; j < 3; ++j) {
      v[j] = glm::vec3(verts[3 * t[j]], verts[3 * t[j] + 1], verts[3 * t[j] + 2]);
      n[j] = glm::vec3(normals[3 * t[j]], normals[3 * t[j] + 1], normals[3 * t[j] + 2]);
    }
    Triangle* tri = new Triangle(v[0], v[1], v[2], n[0], n[1], n[2]);
    tri->setTransformation(rs->identity);
    tri->setInverseTransformation(rs->identity_inv);
    tri->setInverseTransposeTransformation(rs->identity_inv_t);
    tri->setMaterial(rs->object_materials[tri_obj[i]]);
    tri->setMaterialIndex(i);
    tri->setTransformationIndex(0);
    rs->scene.addMaterial(rs->object_materials[tri_obj[i]]);
    rs->scene.addSurface(tri);
    rs->triangles[i] = tri;
  }
  for (int i = 0; i < nl; ++i) {
    const float* l = lights + 6 * i;
    LightSource* ls = new LightSource(glm::vec4(l[0], l[1], l[2], 1.0f), glm::vec4(l[3], l[4], l[5], 1.0f));
    rs->lights.push_back(ls);
    rs->scene.addLightSource(ls);
  }
  return rs;
}

void scan_leaves(RefScene* rs) {
  const BVH& bvh = rs->scene.getBVH();
  BvhNode* nodes = bvh.getNodesBuffer();
  rs->n_nodes = bvh.getNodesBufferSize();
  rs->max_leaf = 0;
  for (int i = 0; i < rs->n_nodes; ++i)
    if (nodes[i].type == BVH_LEAF) rs->max_leaf = std::max(rs->max_leaf, nodes[i].numSurfacesEncapulated);
}

// Ray tree of one primary ray, node j's mirror child 2j + 1 and transparent child 2j + 2:
// the same queries and rays as RayTracer::rayTrace / shadeIntersection, which for a
// material that is both reflective and transparent traces the mirror ray (:339-351) and
// then the transparent bounce's ray (:353-407) from the same hit.
void replay_node(const RefScene& rs, const Ray& ray, int depth, int node, int trace_depth, int32_t* hits,
                 uint32_t* shadows, long long* cnt) {
  const float epsilon = 1e-3f;
  if (depth > trace_depth) return;
  const Scene& scene = rs.scene;
  RayIntersection isect;
  cnt[depth == 0 ? 0 : 2]++;
  if (!scene.findMinDistanceIntersectionBVH(ray, isect)) {
    hits[node] = kHitNone;
    return;
  }
  const int id = isect.getMaterialIndex();
  hits[node] = id;
  const glm::vec3& P = isect.getPoint();
  uint32_t mask = 0;
  for (int i = 0; i < scene.getNumLightSources(); ++i) {
    const LightSource* light = scene.getLightSource(i);
    glm::vec3 sd = glm::normalize(glm::vec3(light->getPosition()) - P);
    Ray sray;
    sray.setOrigin(P + epsilon * sd);
    sray.setDirection(sd);
    cnt[1]++;
    if (scene.shadowRayVisibilityBVH(sray)) mask |= 1u << i;
  }
  shadows[node] = mask;
  const Material& m = scene.getMaterialAtIndex(id);
  if (m.isReflective()) {
    glm::vec3 rd = glm::normalize(glm::reflect(ray.getDirection(), isect.getNormal()));
    Ray r;
    r.setOrigin(P + epsilon * rd);
    r.setDirection(rd);
    replay_node(rs, r, depth + 1, 2 * node + 1, trace_depth, hits, shadows, cnt);
  }
  if (m.isTransparent()) {
    glm::vec3 incident = glm::normalize(ray.getDirection());
    glm::vec3 n = isect.getNormal();
    if (!(glm::dot(incident, n) < 0.0f)) n = glm::vec3(0.0f) - isect.getNormal();
    glm::vec3 rd = glm::normalize(glm::reflect(ray.getDirection(), n));
    Ray r;
    r.setOrigin(P + epsilon * n);
    r.setDirection(rd);
    replay_node(rs, r, depth + 1, 2 * node + 2, trace_depth, hits, shadows, cnt);
  }
}

}  // namespace

extern "C" {

// Builds the reference Scene and its BVH (Scene::flush, src/Scene.cpp:204-209).
// build_threads = 1 gives a deterministic tree: the SAH sweep's OpenMP loop races on
// shared temporaries otherwise (src/BVH.cpp:454-480).
void* eosref_scene_create(const float* verts, const float* normals, int nv, const uint32_t* tris,
                          const uint32_t* tri_obj, int nt, const float* mats, int nobj,
                          const float* lights, int nl, int build_threads, double* build_seconds) {
  (void)nv;
  RefScene* rs = make_scene(verts, normals, tris, tri_obj, nt, mats, nobj, lights, nl);
  int prev = omp_get_max_threads();
  omp_set_num_threads(build_threads > 0 ? build_threads : 1);
  double t0 = getRealTime();
  rs->scene.flush();
  double t1 = getRealTime();
  omp_set_num_threads(prev);
  if (build_seconds) *build_seconds = t1 - t0;
  scan_leaves(rs);
  return rs;
}

// A scene whose triangles carry per-object transformations, built the way the reference's
// main program places a transformed mesh (src/main.cpp:388-394, src/triangleMesh.cpp:140-150):
// object-space vertices and normals, triangle i placed by transformation tri_xf[i] of
// xforms [nx][12] (world-from-object, row-major 3 x 4), each registered in order with
// Scene::addTransformation (src/Scene.cpp:96-106, which the GPU path reads) and pointed to
// by the triangle (which the builder reads: BVH::computeBoxWithSurfaces transforms every
// triangle's local box, src/BVH.cpp:144-159).  Built by the reference's builder with
// build_threads threads.  The reference's CPU renderer ignores the transformations
// (src/Triangle.cpp:26-54); only its GPU path renders such a scene.
void* eosref_scene_create_transformed(const float* verts, const float* normals, const uint32_t* tris,
                                      const uint32_t* tri_obj, int nt, const float* mats, int nobj,
                                      const float* lights, int nl, const int32_t* tri_xf, const float* xforms,
                                      int nx, int build_threads) {
  if (nx < 1) return nullptr;
  for (int i = 0; i < nt; ++i)
    if (tri_xf[i] < 0 || tri_xf[i] >= nx) return nullptr;
  RefScene* rs = make_scene(verts, normals, tris, tri_obj, nt, mats, nobj, lights, nl);
  rs->xf.assign(nx, glm::mat4(1.0f));
  rs->xf_inv.assign(nx, glm::mat4(1.0f));
  rs->xf_inv_t.assign(nx, glm::mat4(1.0f));
  for (int k = 0; k < nx; ++k) {
    const float* m = xforms + 12 * k;
    glm::mat4 M(1.0f);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) M[c][r] = m[4 * r + c];  // glm: column c, row r
    rs->xf[k] = M;
    rs->xf_inv[k] = glm::inverse(M);
    rs->xf_inv_t[k] = glm::inverse(glm::transpose(M));
    rs->scene.addTransformation(M);
  }
  for (int i = 0; i < nt; ++i) {
    Triangle* tri = rs->triangles[i];
    const int k = tri_xf[i];
    tri->setTransformation(rs->xf[k]);
    tri->setInverseTransformation(rs->xf_inv[k]);
    tri->setInverseTransposeTransformation(rs->xf_inv_t[k]);
    tri->setTransformationIndex(k);
  }
  int prev = omp_get_max_threads();
  omp_set_num_threads(build_threads > 0 ? build_threads : 1);
  rs->scene.flush();
  omp_set_num_threads(prev);
  scan_leaves(rs);
  return rs;
}

// The tree the reference's builder made, as plain arrays, so that a scene whose build
// takes minutes on one core (the 1.06M-triangle benchmark scene) is built once and
// restored afterwards.  perm [nt]: triangle id at each position of the scene's surface
// array after the build's in-place sorts.  nodes [n_nodes * 6]: per entry of the
// reference's flat node buffer (src/BVH.cpp:742-784) type, numSurfacesEncapulated,
// leftChildIndex, rightChildIndex, surfacesIndices[0] (leaves; -1 otherwise), splitAxis.
void eosref_tree_export(void* h, int32_t* perm, int32_t* nodes) {
  RefScene* rs = (RefScene*)h;
  const int nt = rs->scene.getNumSurfaces();
  Surface** surf = rs->scene.getFirstSurfaceAddress();
  for (int i = 0; i < nt; ++i) perm[i] = surf[i]->getMaterialIndex();
  const BvhNode* nb = rs->scene.getBVH().getNodesBuffer();
  for (int i = 0; i < rs->n_nodes; ++i) {
    const BvhNode& n = nb[i];
    int32_t* o = nodes + 6 * i;
    o[0] = n.type;
    o[1] = n.numSurfacesEncapulated;
    o[2] = n.type == BVH_LEAF ? -1 : n.leftChildIndex;
    o[3] = n.type == BVH_LEAF ? -1 : n.rightChildIndex;
    o[4] = n.type == BVH_LEAF ? n.surfacesIndices[0] : -1;
    o[5] = n.type == BVH_LEAF ? 0 : n.splitAxis;
  }
}

// The scene with the tree restored from eosref_tree_export's arrays instead of built:
// the surface array is put in the exported order and the flat node buffer is refilled
// (leaves as the patched createLeaf writes them, src/BVH.cpp:325-340); every node's box is
// recomputed by the builder's own BVH::computeBoxWithSurfaces over the node's surface
// range (src/BVH.cpp:144-159), a min / max union over the same surfaces and so the box the
// build computed.  Returns NULL when the arrays do not describe a tree over nt surfaces.
void* eosref_scene_create_from_tree(const float* verts, const float* normals, int nv, const uint32_t* tris,
                                    const uint32_t* tri_obj, int nt, const float* mats, int nobj,
                                    const float* lights, int nl, const int32_t* perm, const int32_t* nodes,
                                    int n_nodes) {
  (void)nv;
  if (n_nodes < 2 || nt < 1) return nullptr;
  std::vector<char> seen(nt, 0);
  for (int i = 0; i < nt; ++i) {
    if (perm[i] < 0 || perm[i] >= nt || seen[perm[i]]) return nullptr;
    seen[perm[i]] = 1;
  }
  // first surface of every node: a leaf's own, an interior node's leftmost leaf's; in the
  // preorder buffer a child comes after its parent, so one backwards pass fills them
  std::vector<int> first(n_nodes, -1);
  for (int i = n_nodes - 1; i >= 0; --i) {
    const int32_t* n = nodes + 6 * i;
    if (n[0] == BVH_LEAF) {
      first[i] = n[4];
    } else {
      if (n[2] <= i || n[2] >= n_nodes || n[3] <= i || n[3] >= n_nodes) return nullptr;
      first[i] = first[n[2]];
    }
    if (first[i] < 0 || n[1] < 1 || first[i] + n[1] > nt) return nullptr;
  }
  RefScene* rs = make_scene(verts, normals, tris, tri_obj, nt, mats, nobj, lights, nl);
  std::vector<Surface*>& so = rs->scene.m_SurfaceObjects;
  std::vector<Surface*> by_id(so.begin(), so.end());
  for (int i = 0; i < nt; ++i) so[i] = by_id[perm[i]];
  BVH& bvh = rs->scene.m_Bvh;
  bvh.m_NodesBuffer = new BvhNode[n_nodes];
  bvh.m_FlatTreePointers.assign(n_nodes, nullptr);
  bvh.m_Root = nullptr;
  for (int i = 0; i < n_nodes; ++i) {
    const int32_t* n = nodes + 6 * i;
    BvhNode& b = bvh.m_NodesBuffer[i];
    b.type = n[0];
    b.numSurfacesEncapulated = n[1];
    b.leftChild = nullptr;
    b.rightChild = nullptr;
    b.leftChildIndex = n[2];
    b.rightChildIndex = n[3];
    b.splitAxis = n[5];
    for (int k = 0; k < SURFACES_PER_LEAF; ++k) b.surfacesIndices[k] = k < n[1] ? first[i] + k : 0;
    b.aabb = bvh.computeBoxWithSurfaces(&so[0], first[i], first[i] + n[1]);
  }
  scan_leaves(rs);
  return rs;
}

// The harness scene's reference Scene (for the GPU harness, ref_gpu_harness.cu).
void* eosref_scene_ptr(void* h) { return &((RefScene*)h)->scene; }

// Boxes of the flat node buffer, [n_nodes * 6] min xyz, max xyz (to check a restore).
void eosref_tree_boxes(void* h, float* boxes) {
  RefScene* rs = (RefScene*)h;
  const BvhNode* nb = rs->scene.getBVH().getNodesBuffer();
  for (int i = 0; i < rs->n_nodes; ++i) {
    const glm::vec3 lo = nb[i].aabb.getMinVertex(), hi = nb[i].aabb.getMaxVertex();
    float* o = boxes + 6 * i;
    o[0] = lo.x; o[1] = lo.y; o[2] = lo.z;
    o[3] = hi.x; o[4] = hi.y; o[5] = hi.z;
  }
}

void eosref_scene_set_ambient(void* h, float ambient) {
  ((RefScene*)h)->scene.setAmbientRefractiveIndex(ambient);
}

void eosref_scene_stats(void* h, int* n_nodes, int* max_leaf) {
  RefScene* rs = (RefScene*)h;
  *n_nodes = rs->n_nodes;
  *max_leaf = rs->max_leaf;
}

void eosref_scene_destroy(void* h) {
  RefScene* rs = (RefScene*)h;
  for (Triangle* t : rs->triangles) delete t;
  for (LightSource* l : rs->lights) delete l;
  delete rs;
}

// FP32 colour and bounce path per pixel.  pix == NULL renders every pixel in row-major
// order (row 0 = bottom, as the reference); otherwise npix listed pixel indices.
// hits / shadows are [npix, 8]; counts gets primary, shadow and secondary ray counts.
int eosref_render(void* h, const float* cam12, int w, int hgt, float pixel_offset, int trace_depth,
                  int nthreads, const int32_t* pix, int npix, float* rgb, int32_t* hits,
                  uint32_t* shadows, long long* counts, double* seconds) {
  RefScene* rs = (RefScene*)h;
  Camera cam = make_camera(cam12, w, hgt);
  RayTracer rt;
  rt.setAASamples(RAYTRACER_NO_AA);
  rt.setTracedDepth(trace_depth);
  if (rt.getTracedDepth() != trace_depth) return -1;  // the reference cannot set depth 0
  int n = pix ? npix : w * hgt;
  long long c0 = 0, c1 = 0, c2 = 0;
  double t0 = getRealTime();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : c0, c1, c2)
  for (int i = 0; i < n; ++i) {
    int p = pix ? pix[i] : i;
    int x = p % w, y = p / w;
    Ray ray = primary_ray(cam, x, y, pixel_offset, pixel_offset);
    glm::vec4 c = rt.rayTrace(rs->scene, cam, ray, 0);
    rgb[3 * i] = c.x;
    rgb[3 * i + 1] = c.y;
    rgb[3 * i + 2] = c.z;
    if (hits) {
      int32_t* hh = hits + kMaxBounces * i;
      uint32_t* ss = shadows + kMaxBounces * i;
      for (int k = 0; k < kMaxBounces; ++k) { hh[k] = kHitUntraced; ss[k] = 0; }
      long long cnt[3] = {0, 0, 0};
      replay_path(*rs, ray, trace_depth, hh, ss, cnt);
      c0 += cnt[0];
      c1 += cnt[1];
      c2 += cnt[2];
    }
  }
  double t1 = getRealTime();
  if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
  if (seconds) *seconds = t1 - t0;
  return 0;
}

// As eosref_render with ray-tree records: hits / shadows [npix, 2^(trace_depth+1) - 1] in
// heap order (replay_node).
int eosref_render_tree(void* h, const float* cam12, int w, int hgt, float pixel_offset, int trace_depth,
                       int nthreads, const int32_t* pix, int npix, float* rgb, int32_t* hits, uint32_t* shadows,
                       long long* counts) {
  RefScene* rs = (RefScene*)h;
  Camera cam = make_camera(cam12, w, hgt);
  RayTracer rt;
  rt.setAASamples(RAYTRACER_NO_AA);
  rt.setTracedDepth(trace_depth);
  if (rt.getTracedDepth() != trace_depth || trace_depth >= kMaxBounces) return -1;
  const int nn = (1 << (trace_depth + 1)) - 1;
  int n = pix ? npix : w * hgt;
  long long c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : c0, c1, c2)
  for (int i = 0; i < n; ++i) {
    int p = pix ? pix[i] : i;
    int x = p % w, y = p / w;
    Ray ray = primary_ray(cam, x, y, pixel_offset, pixel_offset);
    glm::vec4 c = rt.rayTrace(rs->scene, cam, ray, 0);
    rgb[3 * i] = c.x;
    rgb[3 * i + 1] = c.y;
    rgb[3 * i + 2] = c.z;
    int32_t* hh = hits + (size_t)nn * i;
    uint32_t* ss = shadows + (size_t)nn * i;
    for (int k = 0; k < nn; ++k) { hh[k] = kHitUntraced; ss[k] = 0; }
    long long cnt[3] = {0, 0, 0};
    replay_node(*rs, ray, 0, 0, trace_depth, hh, ss, cnt);
    c0 += cnt[0];
    c1 += cnt[1];
    c2 += cnt[2];
  }
  if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
  return 0;
}

// Colours and paths on the reference's anti-aliasing grid (RayTracer::renderWithAA,
// src/RayTracer.cpp:176-265): per pixel aa x aa samples at ((p + ksi) / aa, (q + ksi) / aa),
// ksi = rand() / RAND_MAX = 0 in its integer arithmetic, summed in that order and scaled by
// inv_aaSamples^2.  hits / shadows [npix * aa * aa, 8], samples of a pixel consecutive.
int eosref_render_aa(void* h, const float* cam12, int w, int hgt, int trace_depth, int aa, int nthreads,
                     const int32_t* pix, int npix, float* rgb, int32_t* hits, uint32_t* shadows,
                     long long* counts) {
  RefScene* rs = (RefScene*)h;
  Camera cam = make_camera(cam12, w, hgt);
  RayTracer rt;
  rt.setAASamples(aa);
  rt.setTracedDepth(trace_depth);
  if (rt.getTracedDepth() != trace_depth || aa < 1) return -1;
  const float inv = 1.0 / (float)aa;
  const float inv2 = inv * inv;
  const int n = pix ? npix : w * hgt;
  long long c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : c0, c1, c2)
  for (int i = 0; i < n; ++i) {
    int p0 = pix ? pix[i] : i;
    int x = p0 % w, y = p0 / w;
    glm::vec4 sum(0.0f);
    for (int q = 0; q < aa; ++q) {
      for (int p = 0; p < aa; ++p) {
        const float ksi = 0.0f;
        Ray ray = primary_ray(cam, x, y, (p + ksi) * inv, (q + ksi) * inv);
        sum += rt.rayTrace(rs->scene, cam, ray, 0);
        if (hits) {
          const size_t r = (size_t)i * aa * aa + q * aa + p;
          int32_t* hh = hits + kMaxBounces * r;
          uint32_t* ss = shadows + kMaxBounces * r;
          for (int k = 0; k < kMaxBounces; ++k) { hh[k] = kHitUntraced; ss[k] = 0; }
          long long cnt[3] = {0, 0, 0};
          replay_path(*rs, ray, trace_depth, hh, ss, cnt);
          c0 += cnt[0];
          c1 += cnt[1];
          c2 += cnt[2];
        }
      }
    }
    sum = sum * inv2;
    rgb[3 * i] = sum.x;
    rgb[3 * i + 1] = sum.y;
    rgb[3 * i + 2] = sum.z;
  }
  if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
  return 0;
}

// The reference's own frame call, RayTracer::render (src/RayTracer.cpp:85-265), into a
// caller-owned RGBA8 buffer; aa > 0 = setAASamples(aa), its anti-aliasing grid.
int eosref_render_rgba8(void* h, const float* cam12, int w, int hgt, int trace_depth, int nthreads,
                        unsigned char* out, double* seconds, int aa) {
  RefScene* rs = (RefScene*)h;
  Camera cam = make_camera(cam12, w, hgt);
  RayTracer rt;
  rt.setAASamples(aa > 0 ? aa : RAYTRACER_NO_AA);
  rt.setTracedDepth(trace_depth);
  int prev = omp_get_max_threads();
  omp_set_num_threads(nthreads > 0 ? nthreads : 1);
  double t0 = getRealTime();
  rt.render(rs->scene, cam, out);
  double t1 = getRealTime();
  omp_set_num_threads(prev);
  if (seconds) *seconds = t1 - t0;
  return 0;
}

// Nearest hit / shadow visibility of arbitrary rays through the public Scene queries
// (src/Scene.cpp:145-158).  rays: [n, 6] origin, direction.
void eosref_closest_hit(void* h, const float* rays, int n, int32_t* ids, float* pts) {
  RefScene* rs = (RefScene*)h;
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 6 * i;
    Ray ray;
    ray.setOrigin(glm::vec3(r[0], r[1], r[2]));
    ray.setDirection(glm::vec3(r[3], r[4], r[5]));
    RayIntersection isect;
    bool hit = rs->scene.findMinDistanceIntersectionBVH(ray, isect);
    ids[i] = hit ? isect.getMaterialIndex() : kHitNone;
    if (pts) {
      glm::vec3 p = isect.getPoint();
      pts[3 * i] = hit ? p.x : 0.0f;
      pts[3 * i + 1] = hit ? p.y : 0.0f;
      pts[3 * i + 2] = hit ? p.z : 0.0f;
    }
  }
}

void eosref_any_hit(void* h, const float* rays, int n, uint8_t* occluded) {
  RefScene* rs = (RefScene*)h;
  for (int i = 0; i < n; ++i) {
    const float* r = rays + 6 * i;
    Ray ray;
    ray.setOrigin(glm::vec3(r[0], r[1], r[2]));
    ray.setDirection(glm::vec3(r[3], r[4], r[5]));
    occluded[i] = rs->scene.shadowRayVisibilityBVH(ray) ? 1 : 0;
  }
}

// The reference's 30-bit 3-D Morton encoder (src/morton.h:30-48), for golden vectors.
void eosref_morton3(const uint32_t* xyz, int n, uint32_t* out) {
  for (int i = 0; i < n; ++i) out[i] = EncodeMorton3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

}  // extern "C"
