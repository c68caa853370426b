// Two-level scenes (eos_scene_create_instanced): placements of mesh scenes with affine
// transforms, a tree over the instances' world boxes on top of the meshes' own trees.
//
// The reference keeps one transformation per object (Scene::addTransformation,
// src/Scene.cpp:96-106, with the inverse and inverse transpose from glm) and its GPU kernel
// moves the ray into each triangle's object space with the inverse
// (src/kernelInvocations.h:158-163); its CPU renderer ignores transformations
// (src/Triangle.cpp:26-54).  Here the ray moves once per instance (trace.cuh,
// traverse_instanced) and a mesh used by many instances is stored once.
//
// The instance tree is small (one leaf per instance) and is built on the host: median
// splits of the instance centroids along the widest axis give a binary tree, which is
// written as 4-wide node records in the device layout (lbvh.cu) by the same collapse
// rule (replace the interior child of largest surface area by its children).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include "eos_internal.cuh"

namespace eos {
namespace {

constexpr int kEmptySlot = (int)0xC0000000;

int pack_leaf_host(int first, int count) { return (int)(0x80000000u | ((uint32_t)(count - 1) << 25) | (uint32_t)first); }

// Inverse of the affine [A | t] (row-major 3x4) in double from the adjugate, rounded to
// float: [A^-1 | -A^-1 t].  Returns false for a singular A.
bool affine_inverse(const float* M, float* out) {
  const double a00 = M[0], a01 = M[1], a02 = M[2], a10 = M[4], a11 = M[5], a12 = M[6];
  const double a20 = M[8], a21 = M[9], a22 = M[10];
  const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  const double det = (a00 * c00 + a01 * c01) + a02 * c02;
  if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
  double inv[3][3] = {{c00 / det, (a02 * a21 - a01 * a22) / det, (a01 * a12 - a02 * a11) / det},
                      {c01 / det, (a00 * a22 - a02 * a20) / det, (a02 * a10 - a00 * a12) / det},
                      {c02 / det, (a01 * a20 - a00 * a21) / det, (a00 * a11 - a01 * a10) / det}};
  const double t[3] = {M[3], M[7], M[11]};
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) out[4 * r + c] = (float)inv[r][c];
    out[4 * r + 3] = (float)(-((inv[r][0] * t[0] + inv[r][1] * t[1]) + inv[r][2] * t[2]));
  }
  return true;
}

struct Box {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const Box& b) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], b.lo[k]);
      hi[k] = std::max(hi[k], b.hi[k]);
    }
  }
  double half_area() const {
    const double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1], dz = (double)hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
  }
};

// Box of a mesh scene: the union of the used slots of its root record.
eos_status mesh_root_box(const eos_scene* m, Box& b) {
  float rec[32];
  EOS_CUDA(cudaMemcpy(rec, m->d_nodes, sizeof rec, cudaMemcpyDeviceToHost));
  const int* ref = reinterpret_cast<const int*>(rec + 24);
  for (int s = 0; s < 4; ++s) {
    if (ref[s] == kEmptySlot) continue;
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = std::min(b.lo[k], rec[4 * k + s]);
      b.hi[k] = std::max(b.hi[k], rec[4 * (3 + k) + s]);
    }
  }
  return EOS_OK;
}

// World box of a transformed object box: the 8 corners through [A | t] in double, then
// widened by 1e-5 of the box's size and position and rounded outwards, so that rounding of
// the object-space ray never puts a hit outside it.
Box world_box(const Box& ob, const float* M) {
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int c = 0; c < 8; ++c) {
    const double p[3] = {(c & 1) ? ob.hi[0] : ob.lo[0], (c & 2) ? ob.hi[1] : ob.lo[1], (c & 4) ? ob.hi[2] : ob.lo[2]};
    for (int r = 0; r < 3; ++r) {
      const double w = M[4 * r] * p[0] + M[4 * r + 1] * p[1] + M[4 * r + 2] * p[2] + M[4 * r + 3];
      lo[r] = std::min(lo[r], w);
      hi[r] = std::max(hi[r], w);
    }
  }
  double size = 0.0;
  for (int r = 0; r < 3; ++r) size = std::max({size, hi[r] - lo[r], std::fabs(lo[r]), std::fabs(hi[r])});
  const double pad = 1e-5 * size + 1e-30;
  Box b;
  for (int r = 0; r < 3; ++r) {
    b.lo[r] = std::nextafter((float)(lo[r] - pad), -FLT_MAX);
    b.hi[r] = std::nextafter((float)(hi[r] + pad), FLT_MAX);
  }
  return b;
}

struct BNode {
  Box box;
  int left = -1, right = -1;  // children (interior)
  int inst = -1;              // instance (leaf)
};

int build_binary(std::vector<BNode>& nodes, std::vector<int>& ids, int a, int b, const std::vector<Box>& boxes) {
  const int me = (int)nodes.size();
  nodes.emplace_back();
  Box bb;
  for (int i = a; i < b; ++i) bb.grow(boxes[ids[i]]);
  nodes[me].box = bb;
  if (b - a == 1) {
    nodes[me].inst = ids[a];
    return me;
  }
  float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int i = a; i < b; ++i)
    for (int k = 0; k < 3; ++k) {
      const float c = 0.5f * (boxes[ids[i]].lo[k] + boxes[ids[i]].hi[k]);
      clo[k] = std::min(clo[k], c);
      chi[k] = std::max(chi[k], c);
    }
  int axis = 0;
  for (int k = 1; k < 3; ++k)
    if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
  const int mid = (a + b) / 2;
  std::nth_element(ids.begin() + a, ids.begin() + mid, ids.begin() + b, [&](int x, int y) {
    const float cx = boxes[x].lo[axis] + boxes[x].hi[axis], cy = boxes[y].lo[axis] + boxes[y].hi[axis];
    return cx < cy || (cx == cy && x < y);
  });
  const int l = build_binary(nodes, ids, a, mid, boxes);
  const int r = build_binary(nodes, ids, mid, b, boxes);
  nodes[me].left = l;
  nodes[me].right = r;
  return me;
}

// 4-wide records from the binary tree, breadth first; returns the number of levels.
int write_records_host(const std::vector<BNode>& bn, int root, std::vector<float>& out) {
  struct Item {
    int node, rec;
  };
  std::vector<Item> frontier{{root, 0}}, next;
  out.assign(32, 0.0f);
  int n_rec = 1, levels = 0;
  while (!frontier.empty()) {
    ++levels;
    next.clear();
    for (const Item& it : frontier) {
      std::vector<int> c;
      if (bn[it.node].inst >= 0) {
        c.push_back(it.node);  // a lone leaf at the root
      } else {
        c = {bn[it.node].left, bn[it.node].right};
        while (c.size() < 4) {
          int best = -1;
          double area = -1.0;
          for (size_t i = 0; i < c.size(); ++i)
            if (bn[c[i]].inst < 0 && bn[c[i]].box.half_area() > area) {
              area = bn[c[i]].box.half_area();
              best = (int)i;
            }
          if (best < 0) break;
          const int x = c[best];
          c[best] = bn[x].left;
          c.push_back(bn[x].right);
        }
      }
      float* rec = out.data() + 32 * (size_t)it.rec;
      int* ref = reinterpret_cast<int*>(rec + 24);
      int* cnt = reinterpret_cast<int*>(rec + 28);
      for (int s = 0; s < 4; ++s) {
        if (s >= (int)c.size()) {
          for (int k = 0; k < 6; ++k) rec[4 * k + s] = k < 3 ? INFINITY : -INFINITY;  // a box no ray enters
          ref[s] = kEmptySlot;
          cnt[s] = -1;
          continue;
        }
        const BNode& ch = bn[c[s]];
        for (int k = 0; k < 3; ++k) {
          rec[4 * k + s] = ch.box.lo[k];
          rec[4 * (3 + k) + s] = ch.box.hi[k];
        }
        if (ch.inst >= 0) {
          ref[s] = pack_leaf_host(ch.inst, 1);
          cnt[s] = 1;
        } else {
          ref[s] = n_rec;
          cnt[s] = 0;
          out.resize(32 * (size_t)(n_rec + 1), 0.0f);
          rec = out.data() + 32 * (size_t)it.rec;  // the resize may have moved the array
          ref = reinterpret_cast<int*>(rec + 24);
          cnt = reinterpret_cast<int*>(rec + 28);
          next.push_back({c[s], n_rec++});
        }
      }
    }
    std::swap(frontier, next);
  }
  return levels;
}

}  // namespace
}  // namespace eos

using namespace eos;

extern "C" eos_status eos_scene_create_instanced(eos_ctx* ctx, const eos_instance* instances, uint32_t n_instances,
                                                 const eos_material* materials, uint32_t n_materials,
                                                 const eos_light* lights, uint32_t n_lights, eos_scene** out) {
  if (!ctx || !out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  if (!instances || n_instances == 0 || n_instances >= (1u << 25) || !materials || n_materials == 0 ||
      n_lights > EOS_MAX_LIGHTS || (n_lights > 0 && !lights))
    return EOS_ERR_INVALID_ARG;
  EOS_CUDA(cudaSetDevice(ctx->device));
  std::vector<DevInstance> dev(n_instances);
  std::vector<Box> boxes(n_instances);
  std::map<const eos_scene*, Box> mesh_box;
  long long total = 0;
  int mesh_stack = 0;
  for (uint32_t i = 0; i < n_instances; ++i) {
    const eos_instance& I = instances[i];
    const eos_scene* m = I.mesh;
    if (!m || m->instanced || m->ctx != ctx || m->dev.n_tris == 0) return EOS_ERR_INVALID_ARG;
    if ((long long)I.material_base + m->dev.n_obj > (long long)n_materials) return EOS_ERR_INVALID_ARG;
    DevInstance& d = dev[i];
    if (!affine_inverse(I.transform, d.minv)) return EOS_ERR_INVALID_ARG;
    d.nodes = (const float4*)m->d_nodes;
    d.tris = (const float4*)m->d_tris;
    d.shade = (const float4*)m->d_shade;
    d.pos_of_id = (const int32_t*)m->d_pos_of_id;
    d.id_offset = (int32_t)total;
    d.mat_base = (int32_t)I.material_base;
    total += m->dev.n_tris;
    if (total > INT_MAX) return EOS_ERR_INVALID_ARG;
    if (!mesh_box.count(m)) {
      Box b;
      eos_status st = mesh_root_box(m, b);
      if (st != EOS_OK) return st;
      mesh_box[m] = b;
    }
    boxes[i] = world_box(mesh_box[m], I.transform);
    mesh_stack = std::max(mesh_stack, (m->width - 1) * m->levels);
  }
  std::vector<BNode> bn;
  bn.reserve(2 * (size_t)n_instances);
  std::vector<int> ids(n_instances);
  std::iota(ids.begin(), ids.end(), 0);
  const int root = build_binary(bn, ids, 0, (int)n_instances, boxes);
  std::vector<float> rec;
  const int levels = write_records_host(bn, root, rec);
  // stack: up to 3 entries per instance-tree level, the return marker, the mesh's entries
  if (3 * levels + 1 + mesh_stack > kStackMax) return EOS_ERR_UNSUPPORTED;

  eos_scene* sc = new eos_scene();
  sc->ctx = ctx;
  sc->instanced = true;
  auto fail = [&](eos_status s) {
    eos_scene_destroy(sc);
    return s;
  };
  const size_t rec_bytes = rec.size() * sizeof(float), inst_bytes = sizeof(DevInstance) * n_instances;
  if (cudaMalloc(&sc->d_nodes, rec_bytes) != cudaSuccess || cudaMalloc(&sc->d_inst, inst_bytes) != cudaSuccess ||
      cudaMalloc(&sc->d_mats, sizeof(eos_material) * n_materials) != cudaSuccess ||
      cudaMalloc(&sc->d_lights, sizeof(eos_light) * std::max<uint32_t>(1, n_lights)) != cudaSuccess) {
    cudaGetLastError();
    return fail(EOS_ERR_OOM);
  }
  if (cudaMemcpy(sc->d_nodes, rec.data(), rec_bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(sc->d_inst, dev.data(), inst_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(EOS_ERR_CUDA);
  sc->device_bytes = rec_bytes + inst_bytes + sizeof(eos_material) * n_materials +
                     sizeof(eos_light) * std::max<uint32_t>(1, n_lights);
  sc->dev.n_obj = (int)n_materials;
  sc->dev.n_lights = (int)n_lights;
  sc->dev.n_tris = (int)total;
  sc->dev.ambient_index = 1.0f;
  eos_status st = eos_scene_set_materials(sc, materials, n_materials);
  if (st == EOS_OK && n_lights) st = eos_scene_set_lights(sc, lights, n_lights);
  if (st != EOS_OK) return fail(st);
  sc->dev.nodes = (const float4*)sc->d_nodes;
  sc->dev.mats = (const float*)sc->d_mats;
  sc->dev.lights = (const float*)sc->d_lights;
  sc->dev.inst = (const DevInstance*)sc->d_inst;
  sc->dev.n_inst = (int)n_instances;
  sc->n_nodes = (uint32_t)(rec.size() / 32);
  sc->width = 4;
  sc->levels = levels;
  sc->mesh_levels = mesh_stack;
  sc->leaf_size = 1;
  *out = sc;
  return EOS_OK;
}
