// Loads an OBJ file through the C++ facade's TriangleMesh and renders it with
// DeviceRenderer, the way the reference's main program loads objmodels/bunny.obj
// (src/main.cpp:374-406): material and indices set on the mesh before loadFromFile,
// Scene::addTriangleMesh, createCudaScene, renderCudaSceneToHostBufferMegaKernel.
//
//   facade_mesh <file.obj> <out.rgba> <width> <height> <trace_depth> <camera: 12 floats>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "eos/eos.hpp"

int main(int argc, char** argv) {
  if (argc != 6 + 12) {
    fprintf(stderr, "usage: %s file.obj out.rgba W H depth cam[12]\n", argv[0]);
    return 2;
  }
  const int W = atoi(argv[3]), H = atoi(argv[4]), td = atoi(argv[5]);
  float cam[12];
  for (int i = 0; i < 12; ++i) cam[i] = strtof(argv[6 + i], nullptr);
  try {
    eos::Scene scene;
    eos::Material mat(0.1f, eos::vec4(0.87f, 0.3f, 0.5f, 0.0f), eos::vec4(1.0f), 120);
    mat.setTransparent(false);
    mat.setReflective(true);
    mat.setReflectionIntensity(0.25f);
    const int mi = scene.addMaterial(mat);
    eos::TriangleMesh mesh;
    eos::mat4 M(1.0f);
    const int ti = scene.addTransformation(M);
    mesh.setTransformation(M);
    mesh.setTransformationIndex(ti);
    mesh.setMaterial(mat);
    mesh.setMaterialIndex(mi);
    if (!mesh.loadFromFile(argv[1])) {
      fprintf(stderr, "cannot load %s\n", argv[1]);
      return 3;
    }
    scene.addTriangleMesh(&mesh);
    eos::LightSource l1(eos::vec4(5.0f, 5.0f, 5.0f, 1.0f), eos::vec4(1.0f, 1.0f, 1.0f, 1.0f));
    eos::LightSource l2(eos::vec4(-4.0f, 3.0f, 2.0f, 1.0f), eos::vec4(0.6f, 0.7f, 0.9f, 1.0f));
    scene.addLightSource(&l1);
    scene.addLightSource(&l2);
    scene.flush();
    fprintf(stdout, "triangles %u\n", mesh.getNumTriangles());

    eos::Camera camera;
    camera.setPosition(eos::vec3(cam[0], cam[1], cam[2]));
    camera.setViewingDirection(eos::vec3(cam[3], cam[4], cam[5]));
    camera.setRightVector(eos::vec3(cam[6], cam[7], cam[8]));
    camera.setUpVector(eos::vec3(cam[9], cam[10], cam[11]));
    camera.setWidth(W);
    camera.setHeight(H);
    std::unique_ptr<eos::cudaScene_t> dscene(eos::createCudaScene(&scene));
    eos::DeviceRenderer renderer(&camera, W, H);
    renderer.setTracedDepth(td);
    std::vector<unsigned char> img(4 * (size_t)W * H, 0);
    renderer.renderCudaSceneToHostBufferMegaKernel(dscene.get(), img.data());
    FILE* o = fopen(argv[2], "wb");
    fwrite(img.data(), 1, img.size(), o);
    fclose(o);
  } catch (const eos::Error& e) {
    fprintf(stderr, "eos error: %s\n", e.what());
    return 1;
  }
  return 0;
}
