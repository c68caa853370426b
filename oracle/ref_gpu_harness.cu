// Test-only harness around the reference's own GPU render path -- a comparison point, not
// a checker.  Linked with the reference's GPU sources (src/kernelInvocations.cu,
// src/cudaStructures.cu) and its CPU scene code into oracle/_ref/libeosref_gpu.so by
// oracle/Makefile; only oracle/ref_gpu.py loads it, in a process of its own (the
// reference exits the process on any CUDA error, src/cudaQualifiers.h:35-45).
//
// It runs what the reference's DeviceRenderer::renderCudaSceneToHostBufferMegaKernel does
// (src/DeviceRenderer.cu:61-109): the scene made by createCudaScene
// (src/cudaStructures.cu:483-543) from the reference's own tree, the camera on the device,
// and the C wrapper rayTrace_MegaKernel (src/kernelWrapper.h:30) launching
// __rayTrace_MegaKernel (src/kernelInvocations.cu:172-310: primary rays and local Phong,
// no shadow or mirror rays) on (W/16) x (H/16) blocks of 16 x 16 threads.
#include <cstdio>
#include <cuda_runtime.h>

// Every device allocation of this library -- the reference's own in createCudaScene
// included -- gets kGuard zeroed bytes in front of it (GNU ld --wrap=cudaMalloc /
// --wrap=cudaFree, oracle/Makefile).  The reference's megakernel reads
// triangles->n1 / n2 / n3 [triIndex] with triIndex = -1 for a ray that hits nothing
// (src/kernelInvocations.cu:261) and multiplies the result by 0 afterwards; with the guard
// that read stays inside an allocation instead of possibly before the first one.
constexpr size_t kGuard = 256;
extern "C" cudaError_t __real_cudaMalloc(void** p, size_t bytes);
extern "C" cudaError_t __real_cudaFree(void* p);
extern "C" cudaError_t __wrap_cudaMalloc(void** p, size_t bytes) {
  void* raw = nullptr;
  cudaError_t e = __real_cudaMalloc(&raw, bytes + kGuard);
  if (e != cudaSuccess) return e;
  e = cudaMemset(raw, 0, kGuard);
  *p = (char*)raw + kGuard;
  return e;
}
extern "C" cudaError_t __wrap_cudaFree(void* p) { return __real_cudaFree(p ? (char*)p - kGuard : p); }

#include "Camera.h"
#include "Scene.h"
#include "cudaStructures.h"
#include "kernelWrapper.h"

extern "C" void* eosref_scene_ptr(void* h);  // ref_harness.cpp: the RefScene's Scene

extern "C" {

// The reference's device scene of a harness scene (createCudaScene; it is never freed, as
// in the reference).  The harness's triangles all name transformation 0 (identity,
// world-space vertices); the reference's main program registers each mesh's transformation
// with Scene::addTransformation (src/main.cpp:374-406), which only its GPU path reads
// (src/kernelInvocations.h:158-163), so the identity is registered here first.
void* eosrefgpu_upload(void* ref_scene) {
  Scene* scene = (Scene*)eosref_scene_ptr(ref_scene);
  if (scene->getNumTransformations() == 0) scene->addTransformation(glm::mat4(1.0f));
  return createCudaScene(scene);
}

// reps frames of the reference megakernel into a device image; ms = device time per frame
// (CUDA events around the launches, after one warm-up frame); rgba [h * w * 4] gets the
// last frame (rows the reference's grid does not cover stay 0).  Returns 0, or -1 when a
// CUDA call fails.
int eosrefgpu_render(void* d_scene, const float* c, int w, int h, int reps, unsigned char* rgba, float* ms) {
  Camera cam;
  cam.setPosition(glm::vec3(c[0], c[1], c[2]));
  cam.setViewingDirection(glm::vec3(c[3], c[4], c[5]));
  cam.setRightVector(glm::vec3(c[6], c[7], c[8]));
  cam.setUpVector(glm::vec3(c[9], c[10], c[11]));
  cam.setWidth(w);
  cam.setHeight(h);
  Camera* d_cam = nullptr;
  uchar4* d_img = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = -1;
  int grid[2] = {w / 16, h / 16}, block[2] = {16, 16};
  do {
    if (cudaMalloc((void**)&d_cam, sizeof(Camera)) != cudaSuccess) break;
    if (cudaMemcpy(d_cam, &cam, sizeof(Camera), cudaMemcpyHostToDevice) != cudaSuccess) break;
    if (cudaMalloc((void**)&d_img, sizeof(uchar4) * (size_t)w * h) != cudaSuccess) break;
    if (cudaMemset(d_img, 0, sizeof(uchar4) * (size_t)w * h) != cudaSuccess) break;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) break;
    rayTrace_MegaKernel((cudaScene_t*)d_scene, d_cam, w, h, d_img, grid, block);
    if (cudaDeviceSynchronize() != cudaSuccess) break;
    cudaEventRecord(e0);
    for (int r = 0; r < reps; ++r) rayTrace_MegaKernel((cudaScene_t*)d_scene, d_cam, w, h, d_img, grid, block);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / (float)(reps > 0 ? reps : 1);
    if (cudaMemcpy(rgba, d_img, sizeof(uchar4) * (size_t)w * h, cudaMemcpyDeviceToHost) != cudaSuccess) break;
    rc = 0;
  } while (0);
  if (rc != 0) std::fprintf(stderr, "eosrefgpu_render: %s\n", cudaGetErrorString(cudaGetLastError()));
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (d_img) cudaFree(d_img);
  if (d_cam) cudaFree(d_cam);
  return rc;
}

}  // extern "C"
