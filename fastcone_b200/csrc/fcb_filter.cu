// fcb_filter.cu -- FDK pre-processing and phantom voxelisation on the GPU.
//
// fcb_fdk_filter_device replaces the host-side numpy loops of fastcone.fbp / rampfilter
// (fastcone.py:260-292): cosine weight, zero-padding to 2W with the data at [0, W), real
// FFT, multiplication by pi*|fftfreq(2W)| (DC bin = 1/8 of the first bin), inverse FFT,
// crop to [0, W).  The FFTs are cuFFT batched R2C/C2R transforms over row batches; the
// weighting, padding, filter multiply, crop, 1/(2W) scaling and the cast to the storage
// type are this file's kernels.
#include <cufft.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

__global__ void pad_weight_kernel(const float* __restrict__ in, float* __restrict__ pad,
                                  long long row0, int nrows, int H, int W, float D,
                                  const float* __restrict__ zorig, int cosw)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)nrows * 2 * W;
  if (i >= total) return;
  const int c = (int)(i % (2 * W));
  const long long r = i / (2 * W);
  float v = 0.0f;
  if (c < W) {
    const long long gr = row0 + r;
    v = in[gr * W + c];
    if (cosw) {
      const int t = (int)(gr / H), h = (int)(gr % H);
      const float hh = (float)h - zorig[t];
      const float ww = (float)c - 0.5f * (float)W;
      v *= D / sqrtf(D * D + hh * hh + ww * ww);
    }
  }
  pad[i] = v;
}

__global__ void spectrum_mul_kernel(cufftComplex* __restrict__ spec, const float* __restrict__ filt,
                                    int nrows, int nbins)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nrows * nbins) return;
  const float f = filt[i % nbins];
  cufftComplex z = spec[i];
  z.x *= f;
  z.y *= f;
  spec[i] = z;
}

template <typename T>
__device__ __forceinline__ T to_store(float v);
template <>
__device__ __forceinline__ float to_store<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

template <typename T>
__global__ void crop_store_kernel(const float* __restrict__ pad, T* __restrict__ out, long long row0,
                                  int nrows, int W, float scale)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nrows * W) return;
  const int c = (int)(i % W);
  const long long r = i / W;
  out[(row0 + r) * W + c] = to_store<T>(pad[r * 2 * W + c] * scale);
}

// ------------------------------------------------------------------- phantom
constexpr int PH_MAX = 192;
struct PhParams {
  float* vol;
  int nx, ny, nz;
  int n;
  double e[PH_MAX * 16];
};

__global__ void phantom_kernel(const __grid_constant__ PhParams P, int e0)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nv = (long long)P.nx * P.ny * P.nz;
  if (i >= nv) return;
  const int x = (int)(i % P.nx);
  const long long r = i / P.nx;
  const int y = (int)(r % P.ny), z = (int)(r / P.ny);
  const double px = x - P.nx / 2, py = y - P.ny / 2, pz = z - P.nz / 2;
  double v = 0.0;
  for (int k = 0; k < P.n; k++) {
    const double* E = P.e + 16 * k;
    const double q0 = px - E[0], q1 = py - E[1], q2 = pz - E[2];
    const double b0 = E[6] * q0 + E[9] * q1 + E[12] * q2;
    const double b1 = E[7] * q0 + E[10] * q1 + E[13] * q2;
    const double b2 = E[8] * q0 + E[11] * q1 + E[14] * q2;
    const double rr = (b0 / E[3]) * (b0 / E[3]) + (b1 / E[4]) * (b1 / E[4]) + (b2 / E[5]) * (b2 / E[5]);
    if (rr <= 1.0) v += E[15];
  }
  if (e0 == 0) P.vol[i] = (float)v;
  else P.vol[i] = (float)((double)P.vol[i] + v);
}

}  // namespace fcb

using namespace fcb;

extern "C" int fcb_fdk_filter_device(const float* in, void* out, int outType, int nviews, int H,
                                     int W, float D, const float* zOrigin, int cosineWeight,
                                     int window, void* stream)
{
  if (!in || !out || nviews <= 0 || H <= 0 || W <= 0)
    return set_error(FCB_ERR_INVALID, "bad filter arguments");
  if (outType != FCB_F32 && outType != FCB_F16 && outType != FCB_BF16)
    return set_error(FCB_ERR_INVALID, "unknown output type");
  if (cosineWeight && (!zOrigin || !(D > 0.0f)))
    return set_error(FCB_ERR_INVALID, "cosine weighting needs D > 0 and zOrigin");
  if (window != FCB_FILTER_RAMLAK && window != FCB_FILTER_SHEPPLOGAN)
    return set_error(FCB_ERR_INVALID, "unknown filter window");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int n2 = 2 * W, nb = W + 1;
  // filter response, computed in double like numpy: |fftfreq(2W)|, DC = f1/8, * pi
  std::vector<float> filt(nb);
  for (int k = 0; k < nb; k++) {
    double f = (double)k / (double)n2;
    if (k == 0) f = 0.125 * (1.0 / (double)n2);
    if (window == FCB_FILTER_SHEPPLOGAN && k > 0) {
      const double x = M_PI * (double)k / (double)n2;
      f *= sin(x) / x;
    }
    filt[k] = (float)(M_PI * f);
  }
  const long long rows = (long long)nviews * H;
  const int batch = (int)std::min<long long>(rows, std::max<long long>(1, (256ll << 20) / (8ll * n2)));
  float *pad = nullptr, *dfilt = nullptr, *dz = nullptr;
  cufftComplex* spec = nullptr;
  cufftHandle pf = 0, pi = 0;
  int rc = FCB_OK;
  auto fail = [&](int code, const char* m) { rc = set_error(code, m); };
  do {
    if (cudaMalloc(&pad, (size_t)batch * n2 * sizeof(float)) != cudaSuccess) { fail(FCB_ERR_NOMEM, "filter scratch"); break; }
    if (cudaMalloc(&spec, (size_t)batch * nb * sizeof(cufftComplex)) != cudaSuccess) { fail(FCB_ERR_NOMEM, "filter scratch"); break; }
    if (cudaMalloc(&dfilt, nb * sizeof(float)) != cudaSuccess) { fail(FCB_ERR_NOMEM, "filter scratch"); break; }
    cudaMemcpyAsync(dfilt, filt.data(), nb * sizeof(float), cudaMemcpyHostToDevice, st);
    if (cosineWeight) {
      if (cudaMalloc(&dz, nviews * sizeof(float)) != cudaSuccess) { fail(FCB_ERR_NOMEM, "filter scratch"); break; }
      cudaMemcpyAsync(dz, zOrigin, nviews * sizeof(float), cudaMemcpyHostToDevice, st);
    }
    int n[1] = {n2};
    if (cufftPlanMany(&pf, 1, n, nullptr, 1, n2, nullptr, 1, nb, CUFFT_R2C, batch) != CUFFT_SUCCESS ||
        cufftPlanMany(&pi, 1, n, nullptr, 1, nb, nullptr, 1, n2, CUFFT_C2R, batch) != CUFFT_SUCCESS) {
      fail(FCB_ERR_CUDA, "cufftPlanMany failed");
      break;
    }
    cufftSetStream(pf, st);
    cufftSetStream(pi, st);
    const float scale = 1.0f / (float)n2;
    for (long long r0 = 0; r0 < rows; r0 += batch) {
      const int nr = (int)std::min<long long>(batch, rows - r0);
      long long tot = (long long)nr * n2;
      pad_weight_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(in, pad, r0, nr, H, W, D, dz, cosineWeight);
      // cuFFT plans are for `batch` rows; the tail batch is zero-padded in `pad`
      if (nr < batch) cudaMemsetAsync(pad + (size_t)nr * n2, 0, (size_t)(batch - nr) * n2 * sizeof(float), st);
      if (cufftExecR2C(pf, pad, spec) != CUFFT_SUCCESS) { fail(FCB_ERR_CUDA, "cufftExecR2C failed"); break; }
      tot = (long long)nr * nb;
      spectrum_mul_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(spec, dfilt, nr, nb);
      if (cufftExecC2R(pi, spec, pad) != CUFFT_SUCCESS) { fail(FCB_ERR_CUDA, "cufftExecC2R failed"); break; }
      tot = (long long)nr * W;
      const unsigned g = (unsigned)((tot + 255) / 256);
      if (outType == FCB_F32) crop_store_kernel<float><<<g, 256, 0, st>>>(pad, (float*)out, r0, nr, W, scale);
      else if (outType == FCB_F16) crop_store_kernel<__half><<<g, 256, 0, st>>>(pad, (__half*)out, r0, nr, W, scale);
      else crop_store_kernel<__nv_bfloat16><<<g, 256, 0, st>>>(pad, (__nv_bfloat16*)out, r0, nr, W, scale);
    }
    if (rc) break;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { fail(FCB_ERR_CUDA, cudaGetErrorString(e)); break; }
    // scratch is freed below; wait for the queued work that uses it
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { fail(FCB_ERR_CUDA, cudaGetErrorString(e)); break; }
  } while (0);
  if (pf) cufftDestroy(pf);
  if (pi) cufftDestroy(pi);
  cudaFree(pad);
  cudaFree(spec);
  cudaFree(dfilt);
  cudaFree(dz);
  return rc ? rc : ok();
}

extern "C" int fcb_phantom_device(float* vol, const int volDim[3], const double* params, int n,
                                  void* stream)
{
  if (!vol || !volDim || (n > 0 && !params) || n < 0) return set_error(FCB_ERR_INVALID, "bad phantom arguments");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const long long nv = (long long)volDim[0] * volDim[1] * volDim[2];
  if (nv <= 0) return set_error(FCB_ERR_INVALID, "bad volume size");
  for (int e0 = 0; e0 < std::max(n, 1); e0 += PH_MAX) {
    PhParams P;
    P.vol = vol;
    P.nx = volDim[0]; P.ny = volDim[1]; P.nz = volDim[2];
    P.n = std::max(0, std::min(PH_MAX, n - e0));
    for (int k = 0; k < P.n * 16; k++) P.e[k] = params[e0 * 16 + k];
    phantom_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(P, e0);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return ok();
}
