/*
 * Compatibility header force-included (nvcc -include) when the reference's own
 * coneBeamGPU.cu is built into oracle/_ref/.  CUDA 12 removed texture
 * *references* (`texture<float,3,...>`, cudaBindTextureToArray, cudaUnbindTexture),
 * which the reference relies on (coneBeamGPU.cu:66, :839-866).  This header maps
 * them onto texture *objects* without touching the reference source:
 *
 *   - `texture<T,3,mode>` becomes a __device__ struct holding the texture-object
 *     handle plus the host-side sampler settings (addressMode/filterMode/normalized);
 *   - cudaBindTextureToArray builds a texture object for the cudaArray with exactly
 *     those settings and copies the handle into the device-side struct;
 *   - tex3D(texRef, x, y, z) samples through the object, so the hardware texture
 *     unit (linear filter, clamp addressing, 9-bit interpolation weights) does the
 *     interpolation, as it did for the reference.
 *
 * Test infrastructure only (oracle/_ref); nothing in the product includes it.
 */
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <texture_types.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct fcref_texture {
  cudaTextureObject_t obj;
  enum cudaTextureAddressMode addressMode[3];
  enum cudaTextureFilterMode filterMode;
  int normalized;
};

#define texture __device__ fcref_texture

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ inline T tex3D(const fcref_texture<T, Dim, Mode>& t, float x, float y, float z)
{
  return tex3D<T>(t.obj, x, y, z);
}

/* Host side: the reference writes sampler fields into its texture reference and then
 * binds a cudaArray.  The fields live on the host shadow of the __device__ struct. */
template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaBindTextureToArray(fcref_texture<T, Dim, Mode>& t, cudaArray* arr,
                                          const cudaChannelFormatDesc& /*desc*/)
{
  cudaResourceDesc res;
  memset(&res, 0, sizeof(res));
  res.resType = cudaResourceTypeArray;
  res.res.array.array = arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = t.addressMode[0];
  td.addressMode[1] = t.addressMode[1];
  td.addressMode[2] = t.addressMode[2];
  td.filterMode = t.filterMode;
  td.readMode = Mode;
  td.normalizedCoords = t.normalized;
  if (t.obj) {
    /* the reference rebinds while its previous kernel may still be sampling */
    cudaDeviceSynchronize();
    cudaDestroyTextureObject(t.obj);
  }
  cudaError_t e = cudaCreateTextureObject(&t.obj, &res, &td, nullptr);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(t, &t, sizeof(t));
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaUnbindTexture(fcref_texture<T, Dim, Mode>& t)
{
  cudaError_t e = cudaSuccess;
  if (t.obj) {
    cudaDeviceSynchronize();
    e = cudaDestroyTextureObject(t.obj);
  }
  t.obj = 0;
  return e;
}
