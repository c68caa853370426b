// Renders a scene through the C++ drop-in facade (include/eos/eos.hpp) the way a caller
// of the reference does (src/main.cpp:340-480): Material / Triangle / LightSource /
// Scene / Camera, createCudaScene, DeviceRenderer and RayTracer; the DeviceRenderer frame
// is rendered again from a saved and reloaded scene file and must not change, and the
// reference's C wrappers (rayTrace_MegaKernel and its two variants) must give the same
// frame as DeviceRenderer at its default depth.
//
//   facade_render <scene.bin> <out_device_renderer.rgba> <out_raytracer.rgba> [<out_multi.rgba>]
//
// The optional third image comes from MultiDeviceRenderer split into 3 row bands (they
// cycle over the visible GPUs).
//
// scene.bin: int32 n_verts, n_tris, n_mats, n_lights, width, height, trace_depth;
// float32 verts[3n], normals[3n]; uint32 tris[3m], tri_obj[m]; float32 mats[10k] (kd rgb,
// ks rgb, shininess, reflectivity, transparency, refractive index), lights[6l], camera[12].
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "eos/eos.hpp"

template <class T>
static bool read_n(FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return fread(v.data(), sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
  if (argc != 4 && argc != 5) {
    fprintf(stderr, "usage: %s scene.bin out_dr.rgba out_rt.rgba [out_multi.rgba]\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  int32_t hdr[7];
  if (fread(hdr, sizeof(int32_t), 7, f) != 7) return 2;
  const int nv = hdr[0], nt = hdr[1], nm = hdr[2], nl = hdr[3], W = hdr[4], H = hdr[5], td = hdr[6];
  std::vector<float> verts, normals, mats, lights, cam;
  std::vector<uint32_t> tris, obj;
  bool ok = read_n(f, verts, 3 * nv) && read_n(f, normals, 3 * nv) && read_n(f, tris, 3 * nt) && read_n(f, obj, nt) &&
            read_n(f, mats, 10 * nm) && read_n(f, lights, 6 * nl) && read_n(f, cam, 12);
  fclose(f);
  if (!ok) return 2;

  try {
    eos::Scene scene;
    scene.useBvh(true);
    scene.setAmbientRefractiveIndex(1.0f);
    for (int k = 0; k < nm; ++k) {
      const float* m = &mats[10 * k];
      eos::Material mat(0.0f, eos::vec4(m[0], m[1], m[2], 1.0f), eos::vec4(m[3], m[4], m[5], 1.0f), (int)m[6]);
      mat.setReflective(m[7] > 0.0f);
      mat.setReflectionIntensity(m[7]);
      mat.setTransparent(m[8] > 0.0f);
      mat.setRefractiveIndex(m[9]);
      scene.addMaterial(mat);
    }
    std::vector<std::unique_ptr<eos::Triangle>> owned;
    auto V = [&](const std::vector<float>& a, uint32_t i) { return eos::vec3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); };
    for (int i = 0; i < nt; ++i) {
      const uint32_t* t = &tris[3 * i];
      owned.emplace_back(new eos::Triangle(V(verts, t[0]), V(verts, t[1]), V(verts, t[2]), V(normals, t[0]),
                                           V(normals, t[1]), V(normals, t[2])));
      owned.back()->setMaterialIndex((int)obj[i]);
      scene.addSurface(owned.back().get());
    }
    std::vector<std::unique_ptr<eos::LightSource>> ls;
    for (int i = 0; i < nl; ++i) {
      const float* l = &lights[6 * i];
      ls.emplace_back(new eos::LightSource(eos::vec4(l[0], l[1], l[2], 1.0f), eos::vec4(l[3], l[4], l[5], 1.0f)));
      scene.addLightSource(ls.back().get());
    }
    scene.flush();

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

    // the same frame from a scene file of the built scene (saveCudaScene / loadCudaScene)
    const std::string scn = std::string(argv[2]) + ".scn";
    eos::saveCudaScene(dscene.get(), scn);
    std::unique_ptr<eos::cudaScene_t> loaded(eos::loadCudaScene(scn));
    std::vector<unsigned char> img_loaded(img.size(), 0);
    renderer.renderCudaSceneToHostBufferMegaKernel(loaded.get(), img_loaded.data());
    if (img_loaded != img) {
      fprintf(stderr, "the loaded scene renders a different frame\n");
      return 3;
    }

    // the reference's C wrappers give DeviceRenderer's frame at its default depth; two
    // bands of rayTrace_MultiMegaKernel stitch into the same frame
    {
      eos::DeviceRenderer dflt(&camera, W, H);
      std::vector<unsigned char> want(4 * (size_t)W * H, 0), got(want.size(), 1), got2(want.size(), 2);
      dflt.renderCudaSceneToHostBufferMegaKernel(dscene.get(), want.data());
      int blockdim[2] = {W / 16, H / 16}, tpb[2] = {16, 16};
      rayTrace_MegaKernel(dscene.get(), &camera, W, H, (eos_uchar4_t*)got.data(), blockdim, tpb);
      rayTrace_WarpShuffle_MegaKernel(dscene.get(), &camera, W, H, (eos_uchar4_t*)got2.data(), blockdim, 256);
      std::vector<unsigned char> bands(want.size(), 3);
      const size_t band_bytes = 4 * (size_t)W * (H / 2);
      for (int g = 0; g < 2; ++g)
        rayTrace_MultiMegaKernel(dscene.get(), &camera, W, H, (eos_uchar4_t*)(bands.data() + g * band_bytes), 2, g,
                                 blockdim, tpb);
      if (got != want || got2 != want || (H % 2 == 0 && bands != want)) {
        fprintf(stderr, "the C wrappers render a different frame\n");
        return 4;
      }
    }

    eos::RayTracer rt;
    rt.setTracedDepth(td);
    std::vector<unsigned char> img2(4 * (size_t)W * H, 0);
    rt.render(scene, camera, img2.data());

    FILE* o = fopen(argv[2], "wb");
    fwrite(img.data(), 1, img.size(), o);
    fclose(o);
    o = fopen(argv[3], "wb");
    fwrite(img2.data(), 1, img2.size(), o);
    fclose(o);
    if (argc == 5) {
      eos::MultiDeviceRenderer multi(&scene, &camera, W, H, 3);
      multi.setTracedDepth(td);
      std::vector<unsigned char> img3(4 * (size_t)W * H, 0);
      multi.renderSceneToHostBuffer(img3.data(), &camera);
      o = fopen(argv[4], "wb");
      fwrite(img3.data(), 1, img3.size(), o);
      fclose(o);
    }
  } catch (const eos::Error& e) {
    fprintf(stderr, "eos error: %s\n", e.what());
    return 1;
  }
  return 0;
}
