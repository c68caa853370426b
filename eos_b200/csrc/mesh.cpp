// Wavefront OBJ ingestion (host C++, no GPU work).
//
// Replaces TriangleMesh::loadFromFile (src/triangleMesh.cpp:79-160), which imports the file
// with assimp 3 (src/CMakeLists.txt:11 find_package(ASSIMP); dependencies/libassimp.so ->
// libassimp.so.3) through aiImportFile(aiProcess_Triangulate | aiProcess_GenSmoothNormals |
// aiProcess_JoinIdenticalVertices) and copies positions and normals of the triangles of
// mesh 0.  Assimp is not used; the steps of its published algorithm are restated:
//
//  1. Parse (ObjFileParser / ObjFileImporter::createVertexArray): 'v x y z [w]',
//     'vn x y z', 'f c1 c2 c3 ...' with corners i, i/t, i//n, i/t/n, negative indices
//     counting back from the last element read; other statements are ignored.  Every face
//     corner becomes its own vertex.  Numbers are read with strtof (correctly rounded).
//  2. Triangulate (TriangulateProcess): triangles stay; a quad is split into the fans
//     (s, s+1, s+2), (s, s+2, s+3) from its concave corner s -- the first corner whose
//     angles to its two neighbours, measured against the diagonal, sum above pi -- or from
//     corner 0 when it is convex; a larger polygon is fanned from corner 0.  Faces with
//     fewer than three corners are dropped.
//  3. Normals: the file's when every corner of every face names one; otherwise smooth
//     normals (GenVertexNormalsProcess with its default limit of 175 degrees, i.e. no angle
//     limit): each triangle's normal normalize(cross(v2 - v1, v3 - v1)) is stored on its
//     three corners; then for every corner i in order that no group has claimed, the group
//     S of all corners j with |P_j - P_i|^2 < eps^2 (eps = 1e-4 |bbox max - bbox min|) gets
//     normalize(sum over S of the corners' face normals), summed in corner order, and every
//     member of S is claimed (a member claimed before is overwritten).
//  4. Join identical vertices (JoinVerticesProcess): a corner whose position equals that
//     of a vertex already kept and whose normal lies within 1e-5 of it maps to that vertex;
//     vertices keep first-occurrence order.
//
// normalize(v) = v / |v| with |v| = sqrt((x x + y y) + z z), a zero vector left as is.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/eos_c.h"

struct eos_mesh {
  std::vector<float> verts;    // [n_verts][3]
  std::vector<float> normals;  // [n_verts][3]
  std::vector<uint32_t> tris;  // [n_tris][3]
  uint32_t normals_from_file = 0;
  uint32_t n_faces = 0;
  float bounds[6] = {0, 0, 0, 0, 0, 0};
};

namespace {

struct V3 {
  float x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float sq_len(V3 a) { return dot(a, a); }
inline V3 normalize_safe(V3 v) {
  const float len = std::sqrt(sq_len(v));
  if (len > 0.0f) return {v.x / len, v.y / len, v.z / len};
  return v;
}

struct Corner {
  int v, n;  // 0-based position / normal index; n = -1 when absent
};

// Parses one corner token "i", "i/t", "i//n" or "i/t/n".  Returns false when malformed.
bool parse_corner(const char*& p, int nv, int nn, Corner& c) {
  char* end = nullptr;
  errno = 0;
  long vi = std::strtol(p, &end, 10);
  if (end == p || errno) return false;
  p = end;
  long ni = 0;
  if (*p == '/') {
    ++p;
    if (*p != '/') {  // texture index, read and ignored
      std::strtol(p, &end, 10);
      if (end == p) return false;
      p = end;
    }
    if (*p == '/') {
      ++p;
      ni = std::strtol(p, &end, 10);
      if (end == p) return false;
      p = end;
    }
  }
  if (vi < 0) vi = nv + vi + 1;
  if (vi < 1 || vi > nv) return false;
  c.v = (int)vi - 1;
  c.n = -1;
  if (ni != 0) {
    if (ni < 0) ni = nn + ni + 1;
    if (ni < 1 || ni > nn) return false;
    c.n = (int)ni - 1;
  }
  return *p == '\0' || *p == ' ' || *p == '\t' || *p == '\r' || *p == '\n';
}

bool read_floats(const char* p, float* out, int n) {
  for (int i = 0; i < n; ++i) {
    char* end = nullptr;
    out[i] = std::strtof(p, &end);
    if (end == p) return false;
    p = end;
  }
  return true;
}

// Index of the concave corner of a quad (TriangulateProcess), 0 when convex.
int quad_start(const V3* q) {
  for (int i = 0; i < 4; ++i) {
    const V3 v = q[i];
    V3 left = sub(q[(i + 3) % 4], v), diag = sub(q[(i + 2) % 4], v), right = sub(q[(i + 1) % 4], v);
    const float ll = std::sqrt(sq_len(left)), ld = std::sqrt(sq_len(diag)), lr = std::sqrt(sq_len(right));
    left = {left.x / ll, left.y / ll, left.z / ll};
    diag = {diag.x / ld, diag.y / ld, diag.z / ld};
    right = {right.x / lr, right.y / lr, right.z / lr};
    const float angle = std::acos(dot(left, diag)) + std::acos(dot(right, diag));
    if (angle > 3.1415926538f) return i;
  }
  return 0;
}

eos_status build_mesh(const char* text, size_t len, eos_mesh** out) {
  std::vector<V3> pos, nrm;
  std::vector<Corner> corners;  // three per triangle
  uint32_t n_faces = 0;
  bool all_normals = true;
  std::string line;
  std::vector<Corner> face;
  size_t i = 0;
  while (i < len) {
    size_t j = i;
    while (j < len && text[j] != '\n') ++j;
    line.assign(text + i, j - i);
    i = j + 1;
    // strip a comment and leading blanks
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    const char* p = line.c_str();
    while (*p == ' ' || *p == '\t') ++p;
    if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
      float f[3];
      if (!read_floats(p + 2, f, 3)) return EOS_ERR_PARSE;
      pos.push_back({f[0], f[1], f[2]});
    } else if (p[0] == 'v' && p[1] == 'n' && (p[2] == ' ' || p[2] == '\t')) {
      float f[3];
      if (!read_floats(p + 3, f, 3)) return EOS_ERR_PARSE;
      nrm.push_back({f[0], f[1], f[2]});
    } else if (p[0] == 'f' && (p[1] == ' ' || p[1] == '\t')) {
      face.clear();
      p += 2;
      for (;;) {
        while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
        if (*p == '\0') break;
        Corner c;
        if (!parse_corner(p, (int)pos.size(), (int)nrm.size(), c)) return EOS_ERR_PARSE;
        face.push_back(c);
      }
      ++n_faces;
      if (face.size() < 3) continue;
      for (const Corner& c : face) all_normals = all_normals && c.n >= 0;
      int s = 0;
      if (face.size() == 4) {
        const V3 q[4] = {pos[face[0].v], pos[face[1].v], pos[face[2].v], pos[face[3].v]};
        s = quad_start(q);
      }
      const int k = (int)face.size();
      for (int t = 1; t + 1 < k; ++t) {
        corners.push_back(face[s]);
        corners.push_back(face[(s + t) % k]);
        corners.push_back(face[(s + t + 1) % k]);
      }
    }
  }
  const size_t nc = corners.size();
  if (nc == 0) return EOS_ERR_PARSE;
  if (nc / 3 >= (1u << 25)) return EOS_ERR_INVALID_ARG;

  std::vector<V3> cp(nc), cn(nc);
  for (size_t c = 0; c < nc; ++c) cp[c] = pos[corners[c].v];
  eos_mesh* m = new eos_mesh();
  V3 lo = cp[0], hi = cp[0];
  for (const V3& v : cp) {
    lo = {std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z)};
    hi = {std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z)};
  }
  if (all_normals) {
    for (size_t c = 0; c < nc; ++c) cn[c] = nrm[corners[c].n];
    m->normals_from_file = 1;
  } else {
    std::vector<V3> fn(nc);
    for (size_t t = 0; t < nc / 3; ++t) {
      const V3 n = normalize_safe(cross(sub(cp[3 * t + 1], cp[3 * t]), sub(cp[3 * t + 2], cp[3 * t])));
      fn[3 * t] = fn[3 * t + 1] = fn[3 * t + 2] = n;
    }
    const float eps = std::sqrt(sq_len(sub(hi, lo))) * 1e-4f;
    const float eps2 = eps * eps;
    // corners sorted by x; a group lies inside the x-window [x_i - eps, x_i + eps], searched
    // with twice that width so that rounding of the window bounds never drops a member
    std::vector<uint32_t> by_x(nc);
    for (size_t c = 0; c < nc; ++c) by_x[c] = (uint32_t)c;
    std::stable_sort(by_x.begin(), by_x.end(), [&](uint32_t a, uint32_t b) { return cp[a].x < cp[b].x; });
    std::vector<uint32_t> rank(nc);
    for (size_t r = 0; r < nc; ++r) rank[by_x[r]] = (uint32_t)r;
    std::vector<char> had(nc, 0);
    std::vector<uint32_t> group;
    for (size_t c = 0; c < nc; ++c) {
      if (had[c]) continue;
      group.clear();
      const V3 pc = cp[c];
      for (long r = rank[c]; r >= 0 && cp[by_x[r]].x >= pc.x - 2.0f * eps; --r)
        if (sq_len(sub(cp[by_x[r]], pc)) < eps2) group.push_back(by_x[r]);
      for (size_t r = rank[c] + 1; r < nc && cp[by_x[r]].x <= pc.x + 2.0f * eps; ++r)
        if (sq_len(sub(cp[by_x[r]], pc)) < eps2) group.push_back(by_x[r]);
      if (eps2 == 0.0f) {  // all corners at one point: the group is the equal positions
        group.clear();
        for (size_t r = 0; r < nc; ++r)
          if (cp[r].x == pc.x && cp[r].y == pc.y && cp[r].z == pc.z) group.push_back((uint32_t)r);
      }
      std::sort(group.begin(), group.end());
      V3 sum = {0.0f, 0.0f, 0.0f};
      for (uint32_t g : group) sum = {sum.x + fn[g].x, sum.y + fn[g].y, sum.z + fn[g].z};
      sum = normalize_safe(sum);
      for (uint32_t g : group) {
        cn[g] = sum;
        had[g] = 1;
      }
    }
  }
  // join identical vertices
  struct Key {
    uint32_t x, y, z;
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return (size_t)k.x * 73856093u ^ (size_t)k.y * 19349663u ^ (size_t)k.z * 83492791u;
    }
  };
  auto bits = [](float f) {
    uint32_t u;
    f = f == 0.0f ? 0.0f : f;  // -0 and +0 are the same position
    std::memcpy(&u, &f, 4);
    return u;
  };
  std::unordered_map<Key, std::vector<uint32_t>, KeyHash> at;
  at.reserve(nc);
  std::vector<V3> uv, un;
  m->tris.resize(nc);
  for (size_t c = 0; c < nc; ++c) {
    const Key k{bits(cp[c].x), bits(cp[c].y), bits(cp[c].z)};
    std::vector<uint32_t>& cand = at[k];
    uint32_t idx = 0xffffffffu;
    for (uint32_t u : cand)
      if (sq_len(sub(un[u], cn[c])) <= 1e-5f * 1e-5f) {
        idx = u;
        break;
      }
    if (idx == 0xffffffffu) {
      idx = (uint32_t)uv.size();
      uv.push_back(cp[c]);
      un.push_back(cn[c]);
      cand.push_back(idx);
    }
    m->tris[c] = idx;
  }
  m->verts.resize(3 * uv.size());
  m->normals.resize(3 * uv.size());
  for (size_t v = 0; v < uv.size(); ++v) {
    m->verts[3 * v] = uv[v].x;
    m->verts[3 * v + 1] = uv[v].y;
    m->verts[3 * v + 2] = uv[v].z;
    m->normals[3 * v] = un[v].x;
    m->normals[3 * v + 1] = un[v].y;
    m->normals[3 * v + 2] = un[v].z;
  }
  m->n_faces = n_faces;
  const float b[6] = {lo.x, lo.y, lo.z, hi.x, hi.y, hi.z};
  std::memcpy(m->bounds, b, sizeof b);
  *out = m;
  return EOS_OK;
}

}  // namespace

extern "C" {

eos_status eos_mesh_parse_obj(const char* text, size_t len, eos_mesh** out) {
  if (!out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  if (!text) return EOS_ERR_INVALID_ARG;
  try {
    return build_mesh(text, len, out);
  } catch (const std::bad_alloc&) {
    return EOS_ERR_OOM;
  }
}

eos_status eos_mesh_load_obj(const char* path, eos_mesh** out) {
  if (!out) return EOS_ERR_INVALID_ARG;
  *out = nullptr;
  if (!path) return EOS_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return EOS_ERR_IO;
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  if (bad) return EOS_ERR_IO;
  return eos_mesh_parse_obj(text.data(), text.size(), out);
}

eos_status eos_mesh_get_info(const eos_mesh* mesh, eos_mesh_info* info) {
  if (!mesh || !info) return EOS_ERR_INVALID_ARG;
  info->n_verts = (uint32_t)(mesh->verts.size() / 3);
  info->n_tris = (uint32_t)(mesh->tris.size() / 3);
  info->normals_from_file = mesh->normals_from_file;
  info->n_faces = mesh->n_faces;
  std::memcpy(info->bounds, mesh->bounds, sizeof info->bounds);
  return EOS_OK;
}

eos_status eos_mesh_get_data(const eos_mesh* mesh, float* verts, float* normals, uint32_t* tris) {
  if (!mesh) return EOS_ERR_INVALID_ARG;
  if (verts) std::memcpy(verts, mesh->verts.data(), 4 * mesh->verts.size());
  if (normals) std::memcpy(normals, mesh->normals.data(), 4 * mesh->normals.size());
  if (tris) std::memcpy(tris, mesh->tris.data(), 4 * mesh->tris.size());
  return EOS_OK;
}

eos_status eos_mesh_destroy(eos_mesh* mesh) {
  if (!mesh) return EOS_ERR_INVALID_ARG;
  delete mesh;
  return EOS_OK;
}

}  // extern "C"
