// Compatibility header for compiling the reference's PipeDemoStandalone/FSLBM.cu with CUDA 12,
// for TEST USE ONLY (it builds oracle/_ref/libfslbm_ref.so, the golden-fixture generator).
//
// CUDA 12 removed texture and surface *references* (`texture<>`, `surface<>`,
// cudaBindTextureToArray, cudaBindSurfaceToArray), which FSLBM.cu:39-40 and :542-543 use. This
// header emulates them over one plain float4 array in global memory:
//   tex3D(ref, x, y, z)        point sampling at floor(coord), clamp addressing (the defaults of
//                              an unnormalised texture reference), from ref_tex_src: the live
//                              field, or (race-free mode of the harness) a copy of it taken
//                              before the launches that read it
//   surf3Dwrite(v, ref, xb,y,z) store at x = xb / sizeof(float4); out-of-box writes are dropped
//                              and counted (the reference's launches never make one)
//   surf3Dread<T>(ref, xb,y,z) load at x = xb / sizeof(float4)
// The reference's kernels are compiled unchanged from where they lie; its main() is renamed by
// the harness and never called.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdio>
#include <cstdlib>
#include <string.h>
#include <ctime>
#include <fstream>
#include <iostream>
#include <vector>

template <class T, int D> struct RefSurface {};
template <class T, int D, cudaTextureReadMode M> struct RefTexture {};

__device__ float4* ref_field;        // lx*ly*lz cells, idx = x + lx*(y + ly*z)
__device__ const float4* ref_tex_src;  // what tex3D samples: ref_field or a snapshot of it
__device__ int ref_lx, ref_ly, ref_lz;
__device__ unsigned int ref_oob_writes;

__device__ __forceinline__ int ref_clamp(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

template <class A, class B, class C>
__device__ __forceinline__ float4 tex3D(RefTexture<float4, 3, cudaReadModeElementType>, A x, B y, C z) {
  const int ix = ref_clamp(int(floorf(float(x))), ref_lx);
  const int iy = ref_clamp(int(floorf(float(y))), ref_ly);
  const int iz = ref_clamp(int(floorf(float(z))), ref_lz);
  return ref_tex_src[ix + long(ref_lx) * (iy + long(ref_ly) * iz)];
}

__device__ __forceinline__ void surf3Dwrite(float4 v, RefSurface<void, 3>, int xb, int y, int z) {
  const int x = xb / int(sizeof(float4));
  if (x < 0 || y < 0 || z < 0 || x >= ref_lx || y >= ref_ly || z >= ref_lz) {
    atomicAdd(&ref_oob_writes, 1u);
    return;
  }
  ref_field[x + long(ref_lx) * (y + long(ref_ly) * z)] = v;
}

template <class T>
__device__ __forceinline__ T surf3Dread(RefSurface<void, 3>, int xb, int y, int z) {
  const int x = ref_clamp(xb / int(sizeof(float4)), ref_lx);
  return ref_field[x + long(ref_lx) * (ref_clamp(y, ref_ly) + long(ref_ly) * ref_clamp(z, ref_lz))];
}

static inline cudaError_t cudaBindSurfaceToArray(const RefSurface<void, 3>&, cudaArray_const_t) {
  return cudaErrorNotSupported;
}
static inline cudaError_t cudaBindTextureToArray(
    const RefTexture<float4, 3, cudaReadModeElementType>&, cudaArray_const_t) {
  return cudaErrorNotSupported;
}

// FSLBM.cu:39-40 declare `surface<void,3> surf;` and `texture<float4,...> vtexr;` at file scope.
// These macros turn them into device-resident emulation objects.
#define surface __device__ RefSurface
#define texture __device__ RefTexture
