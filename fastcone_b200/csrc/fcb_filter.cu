// fcb_filter.cu -- FDK pre-processing and phantom voxelisation on the GPU.
//
// fcb_fdk_filter_device replaces the host-side numpy loops of fastcone.fbp / rampfilter
// (fastcone.py:260-292): cosine weight, zero-padding to 2W with the data at [0, W), real
// FFT, multiplication by pi*|fftfreq(2W)| (DC bin = 1/8 of the first bin), inverse FFT,
// crop to [0, W).  The apodised variants cosrampfilter / gaussrampfilter (fastcone.py:
// 294-319) transform rows of length W unpadded.  The FFTs are cuFFT batched R2C/C2R
// transforms over row batches; the weighting, padding, filter multiply, crop, 1/L scaling
// and the cast to the storage type are this file's kernels.
#include <cufft.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

// The three element-wise passes run on 2-D grids: x over a row's elements, y over the
// batch's rows (at most 65535), so no thread divides its index.  (Measured against the
// earlier one-dimensional form, which divided a 64-bit index per element: the same 2-4 TB/s;
// these passes are a third of the filter's time, cuFFT the rest.)

// Rows of W values at a pitch of `pitch` elements (pitch >= W) -> zero-padded rows of L.
__global__ void pad_weight_kernel(const float* __restrict__ in, float* __restrict__ pad,
                                  long long row0, int nrows, int H, int W, int pitch, int L, float D,
                                  const float* __restrict__ zorig, int cosw)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  const long long gr = row0 + r;
  __shared__ float s_hh;  // the row's detector height relative to its view's zOrigin
  if (cosw) {
    if (threadIdx.x == 0) {
      const long long t = gr / H;
      s_hh = (float)(gr - t * H) - zorig[t];
    }
    __syncthreads();
  }
  if (c >= L || r >= nrows) return;
  float v = 0.0f;
  if (c < W) {
    v = in[gr * pitch + c];
    if (cosw) {
      const float hh = s_hh;
      const float ww = (float)c - 0.5f * (float)W;
      v *= D / sqrtf(D * D + hh * hh + ww * ww);
    }
  }
  pad[(size_t)r * L + c] = v;
}

__global__ void spectrum_mul_kernel(cufftComplex* __restrict__ spec, const float* __restrict__ filt,
                                    int nrows, int nbins)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= nbins || r >= nrows) return;
  const float f = filt[c];
  cufftComplex z = spec[(size_t)r * nbins + c];
  z.x *= f;
  z.y *= f;
  spec[(size_t)r * nbins + c] = z;
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
                                  int nrows, int W, int pitch, int L, float scale)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= W || r >= nrows) return;
  out[(row0 + r) * pitch + c] = to_store<T>(pad[(size_t)r * L + c] * scale);
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

// Reusable filter: cuFFT plans, scratch (padded rows, spectra) and the filter response made
// once; execute() is stream-ordered, allocates nothing and does not synchronise.
struct fcb_filter_plan {
  int nviews = 0, H = 0, W = 0, outType = FCB_F32, window = FCB_FILTER_RAMLAK;
  int n2 = 0, nb = 0, batch = 0;
  float* pad = nullptr;
  cufftComplex* spec = nullptr;
  float* dfilt = nullptr;
  float* dz = nullptr;  // per-view zOrigin (nviews floats)
  cufftHandle pf = 0, pi = 0;
  ~fcb_filter_plan()
  {
    if (pf) cufftDestroy(pf);
    if (pi) cufftDestroy(pi);
    cudaFree(pad);
    cudaFree(spec);
    cudaFree(dfilt);
    cudaFree(dz);
  }
};

// Filter response on the plan's nb = L/2 + 1 frequency bins, in double like numpy.
//  RAMLAK / SHEPPLOGAN (fastcone.rampfilter, fastcone.py:272-292): L = 2W, pi * |fftfreq(2W)|
//    with the DC bin 1/8 of the first, times sinc for Shepp-Logan.
//  COSRAMP (fastcone.cosrampfilter, fastcone.py:294-304): L = W, a_k = |fftfreq(W)[k]| = k/W,
//    times cos(0.5 * a_k * pi / W) exactly as written there.
//  GAUSSRAMP (fastcone.gaussrampfilter, fastcone.py:306-319): L = W, a_k times a Gaussian of
//    standard deviation gaussScale * W centred at (W - 1) / 2 and shifted by -W/2 samples
//    (zero beyond the last sample), i.e. exp(-((k + 1/2) / sigma)^2 / 2) for k + W/2 <= W - 1.
static int filter_response(int W, int window, double gaussScale, int* L, std::vector<float>& filt)
{
  if (window == FCB_FILTER_RAMLAK || window == FCB_FILTER_SHEPPLOGAN) {
    *L = 2 * W;
  } else if (window == FCB_FILTER_COSRAMP || window == FCB_FILTER_GAUSSRAMP) {
    *L = W;
    if (window == FCB_FILTER_GAUSSRAMP && !(gaussScale > 0.0))
      return set_error(FCB_ERR_INVALID, "Gaussian window needs gaussScale > 0");
  } else {
    return set_error(FCB_ERR_INVALID, "unknown filter window");
  }
  const int nb = *L / 2 + 1;
  filt.assign(nb, 0.0f);
  for (int k = 0; k < nb; k++) {
    double f;
    if (*L == 2 * W) {
      f = (double)k / (double)*L;
      if (k == 0) f = 0.125 * (1.0 / (double)*L);
      if (window == FCB_FILTER_SHEPPLOGAN && k > 0) {
        const double x = M_PI * (double)k / (double)*L;
        f *= sin(x) / x;
      }
      f *= M_PI;
    } else {
      const double a = (double)k / (double)W;
      if (window == FCB_FILTER_COSRAMP) {
        f = a * cos(0.5 * a * M_PI / (double)W);
      } else {
        const double src = (double)k + 0.5 * (double)W;  // sample the shifted window reads
        const double sig = gaussScale * (double)W;
        const double d = ((double)k + 0.5) / sig;
        f = src <= (double)(W - 1) ? a * exp(-0.5 * d * d) : 0.0;
      }
    }
    filt[k] = (float)f;
  }
  return FCB_OK;
}

extern "C" int fcb_filter_plan_create_ex(int nviews, int H, int W, int outType, int window,
                                         double gaussScale, fcb_filter_plan** out)
try {
  if (!out) return set_error(FCB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (nviews <= 0 || H <= 0 || W <= 0) return set_error(FCB_ERR_INVALID, "bad filter sizes");
  if (outType != FCB_F32 && outType != FCB_F16 && outType != FCB_BF16)
    return set_error(FCB_ERR_INVALID, "unknown output type");
  std::vector<float> filt;
  int L = 0;
  FCB_TRY(filter_response(W, window, gaussScale, &L, filt));
  auto* pl = new fcb_filter_plan();
  pl->nviews = nviews; pl->H = H; pl->W = W; pl->outType = outType; pl->window = window;
  pl->n2 = L;
  pl->nb = L / 2 + 1;
  const long long rows = (long long)nviews * H;
  // rows per cuFFT batch: about 256 MB of padded rows, at most 65535 (the kernels' grid y)
  pl->batch = (int)std::min<long long>(std::min<long long>(rows, 65535),
                                       std::max<long long>(1, (256ll << 20) / (8ll * pl->n2)));
  int rc = FCB_OK;
  do {
    if (cudaMalloc(&pl->pad, (size_t)pl->batch * pl->n2 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&pl->spec, (size_t)pl->batch * pl->nb * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc(&pl->dfilt, pl->nb * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&pl->dz, nviews * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      rc = set_error(FCB_ERR_NOMEM, "filter scratch");
      break;
    }
    if (cudaMemcpy(pl->dfilt, filt.data(), pl->nb * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = set_error(FCB_ERR_CUDA, "filter response upload failed");
      break;
    }
    int n[1] = {pl->n2};
    if (cufftPlanMany(&pl->pf, 1, n, nullptr, 1, pl->n2, nullptr, 1, pl->nb, CUFFT_R2C, pl->batch) != CUFFT_SUCCESS ||
        cufftPlanMany(&pl->pi, 1, n, nullptr, 1, pl->nb, nullptr, 1, pl->n2, CUFFT_C2R, pl->batch) != CUFFT_SUCCESS) {
      rc = set_error(FCB_ERR_CUDA, "cufftPlanMany failed");
      break;
    }
  } while (0);
  if (rc) {
    delete pl;
    return rc;
  }
  *out = pl;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_filter_plan_create(int nviews, int H, int W, int outType, int window,
                                      fcb_filter_plan** out)
try {
  return fcb_filter_plan_create_ex(nviews, H, W, outType, window, 0.125, out);
}
FCB_CATCH_STATUS

namespace fcb {
// Filters the first `nviews` (<= the plan's) views of `in` into `out`, both with rows of the
// plan's W values at a pitch of `pitch` elements (in == out allowed for FP32 output).
// dzorig: device array of the views' zOrigin (cosine weight), or NULL without weighting.
// Stream-ordered, no allocation.
int filter_plan_run(fcb_filter_plan* pl, const float* in, void* out, int nviews, int pitch, float D,
                    const float* dzorig, int cosineWeight, cudaStream_t st)
{
  if (!pl || !in || !out) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  if (nviews <= 0 || nviews > pl->nviews || pitch < pl->W)
    return set_error(FCB_ERR_INVALID, "filter view count or row pitch out of range");
  if (cosineWeight && (!dzorig || !(D > 0.0f)))
    return set_error(FCB_ERR_INVALID, "cosine weighting needs D > 0 and zOrigin");
  const int n2 = pl->n2, nb = pl->nb, W = pl->W, H = pl->H, batch = pl->batch;
  if (cufftSetStream(pl->pf, st) != CUFFT_SUCCESS || cufftSetStream(pl->pi, st) != CUFFT_SUCCESS)
    return set_error(FCB_ERR_CUDA, "cufftSetStream failed");
  const float scale = 1.0f / (float)n2;
  const long long rows = (long long)nviews * H;
  for (long long r0 = 0; r0 < rows; r0 += batch) {
    const int nr = (int)std::min<long long>(batch, rows - r0);
    pad_weight_kernel<<<dim3((unsigned)((n2 + 255) / 256), (unsigned)nr), 256, 0, st>>>(
        in, pl->pad, r0, nr, H, W, pitch, n2, D, dzorig, cosineWeight);
    // cuFFT plans are for `batch` rows; the tail batch is zero-padded in `pad`
    if (nr < batch)
      FCB_CUDA_TRY(cudaMemsetAsync(pl->pad + (size_t)nr * n2, 0, (size_t)(batch - nr) * n2 * sizeof(float), st));
    if (cufftExecR2C(pl->pf, pl->pad, pl->spec) != CUFFT_SUCCESS) return set_error(FCB_ERR_CUDA, "cufftExecR2C failed");
    spectrum_mul_kernel<<<dim3((unsigned)((nb + 255) / 256), (unsigned)nr), 256, 0, st>>>(pl->spec, pl->dfilt,
                                                                                         nr, nb);
    if (cufftExecC2R(pl->pi, pl->spec, pl->pad) != CUFFT_SUCCESS) return set_error(FCB_ERR_CUDA, "cufftExecC2R failed");
    const dim3 g((unsigned)((W + 255) / 256), (unsigned)nr);
    if (pl->outType == FCB_F32)
      crop_store_kernel<float><<<g, 256, 0, st>>>(pl->pad, (float*)out, r0, nr, W, pitch, n2, scale);
    else if (pl->outType == FCB_F16)
      crop_store_kernel<__half><<<g, 256, 0, st>>>(pl->pad, (__half*)out, r0, nr, W, pitch, n2, scale);
    else
      crop_store_kernel<__nv_bfloat16><<<g, 256, 0, st>>>(pl->pad, (__nv_bfloat16*)out, r0, nr, W, pitch, n2, scale);
  }
  FCB_CUDA_TRY(cudaGetLastError());
  return FCB_OK;
}

int filter_plan_create(int nviews, int H, int W, int outType, int window, double gaussScale,
                       fcb_filter_plan** out)
{
  return fcb_filter_plan_create_ex(nviews, H, W, outType, window, gaussScale, out);
}

void filter_plan_destroy(fcb_filter_plan* pl) { delete pl; }
}  // namespace fcb

// out = filter(in) as outType; zOrigin (host, nviews floats) is read before the call returns.
extern "C" int fcb_filter_plan_execute(fcb_filter_plan* pl, const float* in, void* out, float D,
                                       const float* zOrigin, int cosineWeight, void* stream)
try {
  if (!pl || !in || !out) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  if (cosineWeight && (!zOrigin || !(D > 0.0f)))
    return set_error(FCB_ERR_INVALID, "cosine weighting needs D > 0 and zOrigin");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cosineWeight)
    FCB_CUDA_TRY(cudaMemcpyAsync(pl->dz, zOrigin, pl->nviews * sizeof(float), cudaMemcpyHostToDevice, st));
  FCB_TRY(filter_plan_run(pl, in, out, pl->nviews, pl->W, D, pl->dz, cosineWeight, st));
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_filter_plan_destroy(fcb_filter_plan* pl)
try {
  delete pl;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_fdk_filter_device(const float* in, void* out, int outType, int nviews, int H,
                                     int W, float D, const float* zOrigin, int cosineWeight,
                                     int window, void* stream)
try {
  if (!in || !out || nviews <= 0 || H <= 0 || W <= 0)
    return set_error(FCB_ERR_INVALID, "bad filter arguments");
  if (cosineWeight && (!zOrigin || !(D > 0.0f)))
    return set_error(FCB_ERR_INVALID, "cosine weighting needs D > 0 and zOrigin");
  fcb_filter_plan* pl = nullptr;
  FCB_TRY(fcb_filter_plan_create(nviews, H, W, outType, window, &pl));
  int rc = fcb_filter_plan_execute(pl, in, out, D, zOrigin, cosineWeight, stream);
  // the plan's scratch is freed below; wait for the queued work that uses it
  const cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
  fcb_filter_plan_destroy(pl);
  if (rc) return rc;
  if (e != cudaSuccess) return set_error(FCB_ERR_CUDA, cudaGetErrorString(e));
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_phantom_device(float* vol, const int volDim[3], const double* params, int n,
                                  void* stream)
try {
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
FCB_CATCH_STATUS
