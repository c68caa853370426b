// eos.hpp -- header-only C++ drop-in for the reference's render-frame API, over eos_c.h.
//
// Mirrors the classes a caller of the reference uses to render a frame:
//   Material, LightSource, Triangle (Surface), Scene   src/Material.h, src/LightSource.h,
//                                                      src/Triangle.h, src/Scene.h
//   TriangleMesh (OBJ files)                            src/triangleMesh.h
//   Camera                                              src/Camera.h
//   createCudaScene / cudaScene_t                       src/cudaStructures.h:86-98
//   DeviceCameraHandler                                 src/DeviceCameraHandler.h
//   DeviceRenderer::renderCudaSceneToHostBufferMegaKernel
//                                                       src/DeviceRenderer.h:33-55
//   MultiDeviceRenderer::renderSceneToHostBuffer        src/MultiDeviceRenderer.h:31-45
//   RayTracer::render (same call, run on the GPU)       src/RayTracer.h:38-68
//   rayTrace_MegaKernel, rayTrace_WarpShuffle_MegaKernel,
//   rayTrace_MultiMegaKernel (C linkage)                src/kernelWrapper.h:30-34
// with the same names, argument meaning and output layout (RGBA8, row 0 = bottom).
//
// Differences a caller sees:
//  * the frame has the CPU RayTracer's full semantics (shadow rays, mirror bounces up to
//    the traced depth, its 8-bit quantisation) instead of the reference GPU kernel's
//    primary-only shading;
//  * errors throw eos::Error (with the eos_status) instead of exit();
//  * vectors are any type with .x/.y/.z(/.w) members (glm types work unchanged);
//  * per-surface transforms are applied to the vertices (M) and normals (M^-T) once in
//    createCudaScene; with identity transforms the frame equals the reference bit for
//    bit on hit ids and paths;
//  * the scene must be triangles only, as the reference GPU upload requires
//    (src/cudaStructures.cu:342-348).
#ifndef EOS_EOS_HPP
#define EOS_EOS_HPP

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../eos_c.h"

namespace eos {

struct Error : std::runtime_error {
  eos_status status;
  Error(eos_status s, const char* where)
      : std::runtime_error(std::string(where) + ": " + eos_status_string(s)), status(s) {}
};

inline void check(eos_status s, const char* where) {
  if (s != EOS_OK) throw Error(s, where);
}

struct vec3 {
  float x = 0, y = 0, z = 0;
  vec3() = default;
  vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  template <class V>
  vec3(const V& v) : x(v.x), y(v.y), z(v.z) {}
};

struct vec4 {
  float x = 0, y = 0, z = 0, w = 0;
  vec4() = default;
  explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  template <class V>
  vec4(const V& v) : x(v.x), y(v.y), z(v.z), w(v.w) {}
};

// Column-major 4x4 (m[col][row]), the layout of glm::mat4.
struct mat4 {
  float m[4][4];
  mat4() : mat4(1.0f) {}
  explicit mat4(float d) {
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) m[c][r] = c == r ? d : 0.0f;
  }
  template <class M>
  static mat4 from(const M& g) {
    mat4 o;
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) o.m[c][r] = g[c][r];
    return o;
  }
  static mat4 from(const mat4& g) { return g; }
  bool identity() const {
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r)
        if (m[c][r] != (c == r ? 1.0f : 0.0f)) return false;
    return true;
  }
};

inline vec3 transform_point(const mat4& M, const vec3& p) {
  return vec3(M.m[0][0] * p.x + M.m[1][0] * p.y + M.m[2][0] * p.z + M.m[3][0],
              M.m[0][1] * p.x + M.m[1][1] * p.y + M.m[2][1] * p.z + M.m[3][1],
              M.m[0][2] * p.x + M.m[1][2] * p.y + M.m[2][2] * p.z + M.m[3][2]);
}

// Normal transform by the inverse transpose of the upper 3x3 of M.
inline vec3 transform_normal(const mat4& M, const vec3& n) {
  double a[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[r][c] = M.m[c][r];
  double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
               a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  double inv[3][3];
  inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
  inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
  inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
  inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
  inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
  inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
  inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
  inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
  inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
  // (M^-1)^T n
  return vec3((float)(inv[0][0] * n.x + inv[1][0] * n.y + inv[2][0] * n.z),
              (float)(inv[0][1] * n.x + inv[1][1] * n.y + inv[2][1] * n.z),
              (float)(inv[0][2] * n.x + inv[1][2] * n.y + inv[2][2] * n.z));
}

// src/Material.h:46-78 (ambient stored, unused by the renderer as in the reference).
class Material {
 public:
  Material() : m_Ambient(0.2f), m_Diffuse(1.0f), m_Specular(1.0f), m_Shininess(128) {}
  Material(float ambient, vec4 diffuse, vec4 specular, int shininess)
      : m_Ambient(ambient), m_Diffuse(diffuse), m_Specular(specular), m_Shininess(shininess) {}
  void setAmbientIntensity(float a) { m_Ambient = a; }
  void setDiffuseColor(vec4 c) { m_Diffuse = c; }
  void setSpecularColor(vec4 c) { m_Specular = c; }
  void setReflective(bool r) { m_Reflective = r; }
  void setReflectionIntensity(float i) { m_ReflectionIntensity = i; }
  void setTransparent(bool t) { m_Transparent = t; }
  void setRefractiveIndex(float n) { m_RefractiveIndex = n; }
  float getAmbientIntensity() const { return m_Ambient; }
  const vec4& getDiffuseColor() const { return m_Diffuse; }
  const vec4& getSpecularColor() const { return m_Specular; }
  int getShininess() const { return m_Shininess; }
  bool isReflective() const { return m_Reflective; }
  float getReflectiveIntensity() const { return m_ReflectionIntensity; }
  bool isTransparent() const { return m_Transparent; }
  float getRefractiveIndex() const { return m_RefractiveIndex; }

  eos_material to_c() const {
    eos_material m;
    m.kd[0] = m_Diffuse.x; m.kd[1] = m_Diffuse.y; m.kd[2] = m_Diffuse.z;
    m.ks[0] = m_Specular.x; m.ks[1] = m_Specular.y; m.ks[2] = m_Specular.z;
    m.shininess = (float)m_Shininess;
    m.reflectivity = m_Reflective ? m_ReflectionIntensity : 0.0f;
    m.transparency = m_Transparent ? 1.0f : 0.0f;
    m.refractive_index = m_RefractiveIndex;
    return m;
  }

 private:
  float m_Ambient;
  vec4 m_Diffuse, m_Specular;
  int m_Shininess;
  bool m_Reflective = false;
  float m_ReflectionIntensity = 0.0f;
  bool m_Transparent = false;
  float m_RefractiveIndex = 1.0f;
};

// src/LightSource.h:27-39
class LightSource {
 public:
  LightSource() : m_Position(0.0f), m_Color(1.0f) {}
  LightSource(const vec4& position, const vec4& color) : m_Position(position), m_Color(color) {}
  const vec4& getPosition() const { return m_Position; }
  const vec4& getLightColor() const { return m_Color; }

 private:
  vec4 m_Position, m_Color;
};

// src/surface.h + src/Triangle.h:32-99, triangles only.
class Surface {
 public:
  virtual ~Surface() = default;
};

class Triangle : public Surface {
 public:
  Triangle(const vec3& v1, const vec3& v2, const vec3& v3, const vec3& n1, const vec3& n2, const vec3& n3)
      : m_V{v1, v2, v3}, m_N{n1, n2, n3} {}
  void setTransformation(const mat4& M) { m_M = M; }
  template <class M>
  void setTransformation(M& g) { m_M = mat4::from(g); }
  void setMaterial(Material& m) { m_Material = &m; }
  Material& getMaterial() { return *m_Material; }
  void setMaterialIndex(int i) { m_MaterialIndex = i; }
  int getMaterialIndex() const { return m_MaterialIndex; }
  void setTransformationIndex(int i) { m_TransformationIndex = i; }
  int getTransformationIndex() const { return m_TransformationIndex; }
  const vec3& getV1() const { return m_V[0]; }
  const vec3& getV2() const { return m_V[1]; }
  const vec3& getV3() const { return m_V[2]; }
  const vec3& getN1() const { return m_N[0]; }
  const vec3& getN2() const { return m_N[1]; }
  const vec3& getN3() const { return m_N[2]; }
  const mat4& transformation() const { return m_M; }

 private:
  vec3 m_V[3], m_N[3];
  mat4 m_M;
  Material* m_Material = nullptr;
  int m_MaterialIndex = 0;
  int m_TransformationIndex = 0;
};

// src/triangleMesh.h:30-75.  loadFromFile reads a Wavefront OBJ through eos_mesh_load_obj
// (triangulation, smooth normals when the file has none, identical vertices joined; see
// eos_c.h) and makes one Triangle per face with the mesh's transformation, material,
// material index and transformation index at the time of the call, as the reference does
// (src/triangleMesh.cpp:79-160).  All faces of the file are loaded (the reference keeps
// assimp's first mesh).
class TriangleMesh {
 public:
  bool loadFromFile(const char* filename) {
    eos_mesh* m = nullptr;
    if (eos_mesh_load_obj(filename, &m) != EOS_OK) return false;
    eos_mesh_info info;
    eos_mesh_get_info(m, &info);
    std::vector<float> v(3 * (size_t)info.n_verts), n(3 * (size_t)info.n_verts);
    std::vector<uint32_t> t(3 * (size_t)info.n_tris);
    eos_mesh_get_data(m, v.data(), n.data(), t.data());
    eos_mesh_destroy(m);
    auto V = [](const std::vector<float>& a, uint32_t i) { return vec3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); };
    m_Triangles.clear();
    for (uint32_t f = 0; f < info.n_tris; ++f) {
      const uint32_t* k = &t[3 * (size_t)f];
      m_Triangles.emplace_back(new Triangle(V(v, k[0]), V(v, k[1]), V(v, k[2]), V(n, k[0]), V(n, k[1]), V(n, k[2])));
      Triangle* tri = m_Triangles.back().get();
      tri->setTransformation(m_M);
      if (m_Material) tri->setMaterial(*m_Material);
      tri->setMaterialIndex(m_MaterialIndex);
      tri->setTransformationIndex(m_TransformationIndex);
    }
    m_Valid = true;
    return true;
  }
  const mat4& transformation() const { return m_M; }
  void setTransformation(const mat4& M) { m_M = M; }
  template <class M>
  void setTransformation(M& g) { m_M = mat4::from(g); }
  Material& getMaterial() { return m_OwnMaterial; }
  void setMaterial(const Material& m) {
    m_OwnMaterial = m;
    m_Material = &m_OwnMaterial;
  }
  unsigned int getNumTriangles() const { return (unsigned int)m_Triangles.size(); }
  Triangle* getTriangle(int i) { return m_Valid && i >= 0 && i < (int)m_Triangles.size() ? m_Triangles[i].get() : nullptr; }
  void setSceneStartIndex(int s) { m_SceneIndexStart = s; }
  void setSceneEndIndex(int e) { m_SceneIndexEnd = e; }
  void setMaterialIndex(int i) { m_MaterialIndex = i; }
  int getMaterialIndex(int) const { return m_MaterialIndex; }
  void setTransformationIndex(int i) { m_TransformationIndex = i; }
  int getTransformationIndex() const { return m_TransformationIndex; }

 private:
  std::vector<std::unique_ptr<Triangle>> m_Triangles;
  mat4 m_M;
  Material m_OwnMaterial;
  Material* m_Material = nullptr;
  int m_MaterialIndex = 0, m_TransformationIndex = 0;
  int m_SceneIndexStart = 0, m_SceneIndexEnd = 0;
  bool m_Valid = false;
};

// src/Camera.h:30-64
class Camera {
 public:
  template <class V> void setPosition(const V& p) { m_Position = vec3(p); }
  template <class V> void setViewingDirection(const V& d) { m_View = vec3(d); }
  template <class V> void setRightVector(const V& r) { m_Right = vec3(r); }
  template <class V> void setUpVector(const V& u) { m_Up = vec3(u); }
  void setWidth(int w) { m_Width = w; }
  void setHeight(int h) { m_Height = h; }
  const vec3& getPosition() const { return m_Position; }
  const vec3& getViewingDirection() const { return m_View; }
  const vec3& getRightVector() const { return m_Right; }
  const vec3& getUpVector() const { return m_Up; }
  int getWidth() const { return m_Width; }
  int getHeight() const { return m_Height; }

  eos_camera to_c() const {
    eos_camera c;
    const vec3* v[4] = {&m_Position, &m_View, &m_Right, &m_Up};
    float* o[4] = {c.position, c.view, c.right, c.up};
    for (int i = 0; i < 4; ++i) {
      o[i][0] = v[i]->x;
      o[i][1] = v[i]->y;
      o[i][2] = v[i]->z;
    }
    c.width = m_Width;
    c.height = m_Height;
    return c;
  }

 private:
  vec3 m_Position, m_View, m_Right, m_Up;
  int m_Width = 0, m_Height = 0;
};

// One library context per process and device (the reference keeps one CUDA context
// per GPU).  Created on first use on device 0.
inline eos_ctx* default_context(int device = 0) {
  struct Holder {
    eos_ctx* ctx = nullptr;
    ~Holder() {
      if (ctx) eos_ctx_destroy(ctx);
    }
  };
  static Holder h;
  if (!h.ctx) check(eos_ctx_create(device, &h.ctx), "eos_ctx_create");
  return h.ctx;
}

// src/Scene.h:42-118
class Scene {
 public:
  bool addSurface(Surface* s) {
    Triangle* t = dynamic_cast<Triangle*>(s);
    if (!t) return false;  // triangles only (src/cudaStructures.cu:342-348)
    m_Surfaces.push_back(t);
    return true;
  }
  // src/Scene.cpp:55-75: appends the mesh's triangles and records their index range.
  bool addTriangleMesh(TriangleMesh* mesh) {
    if (!mesh) return false;
    const int start = getNumSurfaces();
    for (unsigned int i = 0; i < mesh->getNumTriangles(); ++i) {
      Triangle* t = mesh->getTriangle((int)i);
      if (!t) return false;
      m_Surfaces.push_back(t);
    }
    mesh->setSceneStartIndex(start);
    mesh->setSceneEndIndex(getNumSurfaces() - start);
    return true;
  }
  bool addLightSource(LightSource* l) {
    if (!l) return false;
    m_Lights.push_back(l);
    return true;
  }
  int addMaterial(Material m) {
    m_Materials.push_back(m);
    return (int)m_Materials.size() - 1;
  }
  int addTransformation(const mat4& M) {
    m_Transforms.push_back(M);
    return (int)m_Transforms.size() - 1;
  }
  const Material& getMaterialAtIndex(int i) const { return m_Materials[i]; }
  int getNumMaterials() const { return (int)m_Materials.size(); }
  int getNumSurfaces() const { return (int)m_Surfaces.size(); }
  int getNumLightSources() const { return (int)m_Lights.size(); }
  const LightSource* getLightSource(int i) const { return i < (int)m_Lights.size() ? m_Lights[i] : nullptr; }
  Triangle* getSurface(int i) const { return i < (int)m_Surfaces.size() ? m_Surfaces[i] : nullptr; }
  void setAmbientRefractiveIndex(float n) { m_AmbientIndex = n; }
  float getAmbientRefractiveIndex() const { return m_AmbientIndex; }
  void setMaxTracedDepth(int d) { m_MaxTracedDepth = d; }
  int getMaxTracedDepth() const { return m_MaxTracedDepth; }
  void useBvh(bool u) { m_UseBvh = u; }
  bool isUsingBvh() const { return m_UseBvh; }
  void setAASamples(int s) { m_AASamples = s; }
  int getAASamples() const { return m_AASamples; }
  // The reference builds its CPU BVH here (src/Scene.cpp:204-209); the LBVH is built on the
  // GPU by createCudaScene, so flush only freezes the surface list.
  void flush() { m_Flushed = true; }

 private:
  std::vector<Triangle*> m_Surfaces;
  std::vector<LightSource*> m_Lights;
  std::vector<Material> m_Materials;
  std::vector<mat4> m_Transforms;
  float m_AmbientIndex = 1.0f;
  int m_MaxTracedDepth = 0;
  bool m_UseBvh = true;
  bool m_Flushed = false;
  int m_AASamples = 1;
};

// The device scene (src/cudaStructures.h:86-92): here the library's resident scene.
struct cudaScene_t {
  eos_scene* scene = nullptr;
  eos_ctx* ctx = nullptr;
  ~cudaScene_t() {
    if (scene) eos_scene_destroy(scene);
  }
};

// src/cudaStructures.cu:483-543: flattens the surfaces (one vertex triple per triangle,
// one material per triangle, as the reference's per-triangle material index) and builds
// the LBVH on the device.  The returned object owns the device scene.
inline cudaScene_t* createCudaScene(Scene* scene, eos_ctx* ctx = nullptr) {
  if (!scene) throw Error(EOS_ERR_INVALID_ARG, "createCudaScene");
  if (!ctx) ctx = default_context();
  const int n = scene->getNumSurfaces();
  std::vector<float> v(9 * (size_t)n), nrm(9 * (size_t)n);
  std::vector<uint32_t> tris(3 * (size_t)n), obj(n);
  std::vector<eos_material> mats;
  std::vector<const Material*> seen;
  for (int i = 0; i < n; ++i) {
    Triangle* t = scene->getSurface(i);
    const mat4& M = t->transformation();
    const bool ident = M.identity();
    const vec3 V[3] = {t->getV1(), t->getV2(), t->getV3()};
    const vec3 N[3] = {t->getN1(), t->getN2(), t->getN3()};
    for (int j = 0; j < 3; ++j) {
      vec3 p = ident ? V[j] : transform_point(M, V[j]);
      vec3 q = ident ? N[j] : transform_normal(M, N[j]);
      v[9 * i + 3 * j] = p.x; v[9 * i + 3 * j + 1] = p.y; v[9 * i + 3 * j + 2] = p.z;
      nrm[9 * i + 3 * j] = q.x; nrm[9 * i + 3 * j + 1] = q.y; nrm[9 * i + 3 * j + 2] = q.z;
      tris[3 * i + j] = (uint32_t)(3 * i + j);
    }
    // material per triangle: its scene material index, as the reference shades through
    // Scene::getMaterialAtIndex(intersection.getMaterialIndex()) (src/RayTracer.cpp:317,430)
    int mi = t->getMaterialIndex();
    if (mi < 0 || mi >= scene->getNumMaterials()) throw Error(EOS_ERR_INVALID_ARG, "createCudaScene: material index");
    obj[i] = (uint32_t)mi;
  }
  for (int k = 0; k < scene->getNumMaterials(); ++k) mats.push_back(scene->getMaterialAtIndex(k).to_c());
  if (mats.empty()) mats.push_back(Material().to_c());
  std::vector<eos_light> lights;
  for (int k = 0; k < scene->getNumLightSources(); ++k) {
    const LightSource* l = scene->getLightSource(k);
    eos_light c;
    c.position[0] = l->getPosition().x; c.position[1] = l->getPosition().y; c.position[2] = l->getPosition().z;
    c.color[0] = l->getLightColor().x; c.color[1] = l->getLightColor().y; c.color[2] = l->getLightColor().z;
    lights.push_back(c);
  }
  std::unique_ptr<cudaScene_t> cs(new cudaScene_t());
  cs->ctx = ctx;
  check(eos_scene_create(ctx, v.data(), nrm.data(), (uint32_t)(3 * n), tris.data(), obj.data(), (uint32_t)n,
                         mats.data(), (uint32_t)mats.size(), lights.data(), (uint32_t)lights.size(), nullptr,
                         &cs->scene),
        "createCudaScene");
  check(eos_scene_set_ambient_index(cs->scene, scene->getAmbientRefractiveIndex()), "createCudaScene");
  return cs.release();
}

// Scene file of a built device scene (eos_scene_save / eos_scene_load): a later run loads
// the tree instead of building it.  No reference counterpart.
inline void saveCudaScene(const cudaScene_t* cs, const std::string& path) {
  if (!cs) throw Error(EOS_ERR_INVALID_ARG, "saveCudaScene");
  check(eos_scene_save(cs->scene, path.c_str()), "saveCudaScene");
}

inline cudaScene_t* loadCudaScene(const std::string& path, eos_ctx* ctx = nullptr) {
  if (!ctx) ctx = default_context();
  std::unique_ptr<cudaScene_t> cs(new cudaScene_t());
  cs->ctx = ctx;
  check(eos_scene_load(ctx, path.c_str(), &cs->scene), "loadCudaScene");
  return cs.release();
}

// src/DeviceCameraHandler.h: the camera travels as kernel arguments, so the "device"
// camera is a host copy that the renderer reads at each frame.
class DeviceCameraHandler {
 public:
  Camera* setDeviceCamera(const Camera* host) {
    m_Camera = *host;
    return &m_Camera;
  }
  void updateDeviceCamera(const Camera* host) { m_Camera = *host; }
  Camera* getDeviceCamera() { return &m_Camera; }

 private:
  Camera m_Camera;
};

constexpr int kDefaultTraceDepth = 4;  // RAYTRACER_DEFAULT_TRACE_DEPTH, src/RayTracer.h:36

inline void render_rgba8(eos_ctx* ctx, const eos_scene* sc, const Camera& cam, int trace_depth, void* image,
                         int mode = EOS_MODE_PLAIN) {
  eos_camera c = cam.to_c();
  eos_render_params p{};
  p.trace_depth = trace_depth;
  p.pixel_offset = 0.0f;  // the reference's integer pixel positions
  p.spp = 1;
  p.mode = mode;
  check(eos_render(ctx, sc, &c, &p, nullptr, (uint8_t*)image, nullptr, nullptr, nullptr), "eos_render");
}

// src/DeviceRenderer.h:33-55
class DeviceRenderer {
 public:
  DeviceRenderer(Camera* camera, int width, int height) : m_Camera(camera), m_Width(width), m_Height(height) {}
  // Renders one frame into a caller-owned RGBA8 buffer of width*height*4 bytes.
  void renderCudaSceneToHostBufferMegaKernel(cudaScene_t* deviceScene, void* imageBuffer) {
    Camera c = *m_Camera;
    c.setWidth(m_Width);
    c.setHeight(m_Height);
    render_rgba8(deviceScene->ctx, deviceScene->scene, c, m_TraceDepth, imageBuffer, EOS_MODE_PLAIN);
  }
  void renderCudaSceneToHostBufferWarpShuffleMegaKernel(cudaScene_t* deviceScene, void* imageBuffer) {
    Camera c = *m_Camera;
    c.setWidth(m_Width);
    c.setHeight(m_Height);
    render_rgba8(deviceScene->ctx, deviceScene->scene, c, m_TraceDepth, imageBuffer, EOS_MODE_WAVEFRONT);
  }
  void setCamera(Camera* c) { m_Camera = c; }
  int getWidth() const { return m_Width; }
  int getHeight() const { return m_Height; }
  Camera* getDeviceCamera() const { return m_Camera; }
  void setTracedDepth(int d) {
    if (d > 0) m_TraceDepth = d;
  }

 private:
  Camera* m_Camera;
  int m_Width, m_Height;
  int m_TraceDepth = kDefaultTraceDepth;
};

// src/MultiDeviceRenderer.h:31-45 / src/MultiDeviceRenderer.cu:31-200: a copy of the
// scene on every GPU and the frame split into horizontal bands, one per GPU, rendered in
// parallel by one host thread each straight into the caller's buffer (eos_render with a
// row band).  The reference gives every GPU height / n rows and leaves the remainder
// unrendered; here the last band takes it.  `bands` > 0 sets the number of bands, which
// then cycle over the GPUs, each band with its own context.
class MultiDeviceRenderer {
 public:
  MultiDeviceRenderer(Scene* scene, Camera* camera, int width, int height, int bands = 0)
      : m_Width(width), m_Height(height) {
    (void)camera;
    int32_t n_dev = 0;
    check(eos_device_count(&n_dev), "eos_device_count");
    if (n_dev < 1) throw Error(EOS_ERR_NO_DEVICE, "MultiDeviceRenderer");
    const int n = bands > 0 ? bands : n_dev;
    for (int b = 0; b < n; ++b) {
      eos_ctx* ctx = nullptr;
      check(eos_ctx_create(b % n_dev, &ctx), "eos_ctx_create");
      m_Ctx.push_back(ctx);
      m_Scenes.emplace_back(createCudaScene(scene, ctx));
    }
  }
  ~MultiDeviceRenderer() {
    m_Scenes.clear();
    for (eos_ctx* c : m_Ctx) eos_ctx_destroy(c);
  }
  MultiDeviceRenderer(const MultiDeviceRenderer&) = delete;
  MultiDeviceRenderer& operator=(const MultiDeviceRenderer&) = delete;

  void renderSceneToHostBuffer(void* imageBuffer, Camera* hostCamera) {
    Camera c = *hostCamera;
    c.setWidth(m_Width);
    c.setHeight(m_Height);
    const eos_camera cc = c.to_c();
    const int n = (int)m_Ctx.size();
    std::vector<eos_status> status(n, EOS_OK);
    std::vector<std::thread> workers;
    for (int b = 0; b < n; ++b) {
      workers.emplace_back([&, b] {
        const int r0 = b * (m_Height / n), r1 = b + 1 == n ? m_Height : (b + 1) * (m_Height / n);
        if (r0 >= r1) return;
        eos_render_params p{};
        p.trace_depth = m_TraceDepth;
        p.pixel_offset = 0.0f;
        p.spp = 1;
        p.mode = EOS_MODE_PLAIN;
        p.row_begin = r0;
        p.row_end = r1;
        status[b] = eos_render(m_Ctx[b], m_Scenes[b]->scene, &cc, &p, nullptr,
                               (uint8_t*)imageBuffer + 4ull * r0 * m_Width, nullptr, nullptr, nullptr);
      });
    }
    for (std::thread& t : workers) t.join();
    for (eos_status s : status) check(s, "MultiDeviceRenderer::renderSceneToHostBuffer");
  }
  void setTracedDepth(int d) {
    if (d > 0) m_TraceDepth = d;
  }
  int getNumBands() const { return (int)m_Ctx.size(); }

 private:
  std::vector<eos_ctx*> m_Ctx;
  std::vector<std::unique_ptr<cudaScene_t>> m_Scenes;
  int m_Width, m_Height;
  int m_TraceDepth = kDefaultTraceDepth;
};

// src/RayTracer.h:38-68: the CPU renderer's call, run on the GPU.  A scene is uploaded
// on the first render and reused while the same Scene object is rendered.
class RayTracer {
 public:
  void render(const Scene& scene, const Camera& camera, unsigned char* outputImage) {
    if (m_Source != &scene) {
      m_Device.reset(createCudaScene(const_cast<Scene*>(&scene)));
      m_Source = &scene;
    }
    render_rgba8(m_Device->ctx, m_Device->scene, camera, m_TraceDepth, outputImage);
  }
  int getAASamples() const { return m_AASamples; }
  void setAASamples(int s) {
    if (s > 0) m_AASamples = s;
  }
  int getTracedDepth() const { return m_TraceDepth; }
  void setTracedDepth(int d) {
    if (d > 0) m_TraceDepth = d;
  }

 private:
  int m_AASamples = 0;
  int m_TraceDepth = kDefaultTraceDepth;
  const Scene* m_Source = nullptr;
  std::unique_ptr<cudaScene_t> m_Device;
};

}  // namespace eos

// The reference's C wrappers around its GPU kernel (src/kernelWrapper.h:30-34,
// src/kernelInvocations.cu:668-711), with the same names and arguments.  Each renders the
// frame that DeviceRenderer renders at its default trace depth (RayTracer semantics, see
// above) into `imageBuffer`, host or device memory of width * height RGBA8 pixels.
// `camera` is the facade's Camera (the copy DeviceCameraHandler hands out); the block /
// thread counts are accepted and ignored, as the library picks its own launch shape.
// rayTrace_MultiMegaKernel renders rows [(height / numGPUS) * gpuID, (height / numGPUS) *
// (gpuID + 1)) into a buffer of that band only, as the reference's per-GPU kernel does, on
// the device of the scene's context.  Errors throw eos::Error.
#if defined(__VECTOR_TYPES_H__) || __has_include(<vector_types.h>)
#include <vector_types.h>
using eos_uchar4_t = uchar4;
#else
using eos_uchar4_t = void;
#endif

extern "C" inline void rayTrace_MegaKernel(eos::cudaScene_t* deviceScene, eos::Camera* camera, int width, int height,
                                           eos_uchar4_t* imageBuffer, int blockdim[], int tpblock[]) {
  (void)blockdim;
  (void)tpblock;
  if (!deviceScene || !camera) throw eos::Error(EOS_ERR_INVALID_ARG, "rayTrace_MegaKernel");
  eos::Camera c = *camera;
  c.setWidth(width);
  c.setHeight(height);
  eos::render_rgba8(deviceScene->ctx, deviceScene->scene, c, eos::kDefaultTraceDepth, imageBuffer, EOS_MODE_PLAIN);
}

extern "C" inline void rayTrace_WarpShuffle_MegaKernel(eos::cudaScene_t* deviceScene, eos::Camera* camera, int width,
                                                       int height, eos_uchar4_t* imageBuffer, int blockdim[],
                                                       int tpblock) {
  (void)blockdim;
  (void)tpblock;
  if (!deviceScene || !camera) throw eos::Error(EOS_ERR_INVALID_ARG, "rayTrace_WarpShuffle_MegaKernel");
  eos::Camera c = *camera;
  c.setWidth(width);
  c.setHeight(height);
  eos::render_rgba8(deviceScene->ctx, deviceScene->scene, c, eos::kDefaultTraceDepth, imageBuffer,
                    EOS_MODE_WAVEFRONT);
}

extern "C" inline void rayTrace_MultiMegaKernel(eos::cudaScene_t* deviceScene, eos::Camera* camera, int width,
                                                int height, eos_uchar4_t* imageBuffer, int numGPUS, int gpuID,
                                                int blockdimp[], int tpblock[]) {
  (void)blockdimp;
  (void)tpblock;
  if (!deviceScene || !camera || numGPUS < 1 || gpuID < 0 || gpuID >= numGPUS || height / numGPUS < 1)
    throw eos::Error(EOS_ERR_INVALID_ARG, "rayTrace_MultiMegaKernel");
  eos::Camera cam = *camera;
  cam.setWidth(width);
  cam.setHeight(height);
  const eos_camera c = cam.to_c();
  const int rows = height / numGPUS;
  eos_render_params p{};
  p.trace_depth = eos::kDefaultTraceDepth;
  p.pixel_offset = 0.0f;
  p.spp = 1;
  p.mode = EOS_MODE_PLAIN;
  p.row_begin = rows * gpuID;
  p.row_end = rows * (gpuID + 1);
  eos::check(eos_render(deviceScene->ctx, deviceScene->scene, &c, &p, nullptr, (uint8_t*)imageBuffer, nullptr,
                        nullptr, nullptr),
             "rayTrace_MultiMegaKernel");
}

#endif  // EOS_EOS_HPP
