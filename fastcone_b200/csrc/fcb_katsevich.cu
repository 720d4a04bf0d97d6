// fcb_katsevich.cu -- Katsevich filtering for helical cone-beam data (sm_100a).
//
// The reference has only the Katsevich backprojection weight (coneBeamGPU.cu:258-338) and
// expects pre-filtered, windowed data.  This file supplies the filtering of Katsevich's
// exact helical inversion in the flat-detector form of Noo, Pack & Heuscher (Phys. Med.
// Biol. 48 (2003) 3787-3818), on the virtual detector through the rotation axis
// (source-detector distance = source-axis distance D).  Detector pixel (i, j) sits at
// w = (i - W/2) pw, v = (j - H/2) pw; the published coordinate u runs along the source's
// direction of travel, u = s_u * w with s_u = -1 for a right-handed helix (angles and
// height increasing together).  Stages:
//   1. derivative at fixed ray direction  g1 = dg/dlam + (u^2+D^2)/D dg/du + u v/D dg/dv
//      and length correction g2 = D / sqrt(u^2+D^2+v^2) g1      (deriv_kernel)
//   2. forward height rebinning onto kappa-lines v_k(u, psi) = P/(2 pi)(psi + psi/tan(psi) u/D)
//      (rebin_fwd_kernel, per-(kappa, column) interpolation table built on the host in FP64)
//   3. Hilbert transform along u, band-limited kernel (1 - cos(pi n))/(pi n): a linear
//      convolution done with cuFFT (kernel spectrum in FP64 on the host); kats_hilbert_kernel
//      is the direct O(W^2) form, kept for comparison
//   4. backward rebinning through the kappa-line of smallest |psi| (rebin_bwd_kernel,
//      per-(row, column) table).
// Backprojection with weight U over each voxel's PI interval and norm dlam/(2 pi D) then
// reconstructs (fdk_tma_kernel with the Tam-Danielsson window).
#include <cufft.h>
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

__global__ void kats_deriv_kernel(const float* __restrict__ g, float* __restrict__ g2, int n, int H,
                                  int W, float dlam, float pw, float D, float su)
{
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)n * H * W;
  if (idx >= tot) return;
  const int i = (int)(idx % W);
  const long long r = idx / W;
  const int j = (int)(r % H), t = (int)(r / H);
  const size_t plane = (size_t)H * W;
  const float* gt = g + (size_t)t * plane;
  // dg/dlam: central inside, one-sided at the ends (numpy.gradient, edge order 1)
  float dl;
  if (n == 1) dl = 0.0f;
  else if (t == 0) dl = (g[plane + (size_t)j * W + i] - gt[(size_t)j * W + i]) / dlam;
  else if (t == n - 1) dl = (gt[(size_t)j * W + i] - g[(size_t)(t - 1) * plane + (size_t)j * W + i]) / dlam;
  else dl = (g[(size_t)(t + 1) * plane + (size_t)j * W + i] - g[(size_t)(t - 1) * plane + (size_t)j * W + i]) / (2.0f * dlam);
  // dg/du with u_i = su * (i - W/2) pw
  const float du = su * pw;
  float dgu;
  if (W == 1) dgu = 0.0f;
  else if (i == 0) dgu = (gt[(size_t)j * W + 1] - gt[(size_t)j * W]) / du;
  else if (i == W - 1) dgu = (gt[(size_t)j * W + i] - gt[(size_t)j * W + i - 1]) / du;
  else dgu = (gt[(size_t)j * W + i + 1] - gt[(size_t)j * W + i - 1]) / (2.0f * du);
  float dgv;
  if (H == 1) dgv = 0.0f;
  else if (j == 0) dgv = (gt[(size_t)W + i] - gt[i]) / pw;
  else if (j == H - 1) dgv = (gt[(size_t)j * W + i] - gt[(size_t)(j - 1) * W + i]) / pw;
  else dgv = (gt[(size_t)(j + 1) * W + i] - gt[(size_t)(j - 1) * W + i]) / (2.0f * pw);
  const float u = su * (float)(i - W / 2) * pw, v = (float)(j - H / 2) * pw;
  const float g1 = dl + ((u * u + D * D) / D) * dgu + (u * v / D) * dgv;
  g2[idx] = g1 * (D * rsqrtf(u * u + D * D + v * v));
}

// g3[t][k][i] = g2[t][j0][i] * (1-a) + g2[t][j0+1][i] * a from the (kappa, column) table
__global__ void kats_rebin_fwd_kernel(const float* __restrict__ g2, float* __restrict__ g3,
                                      const int* __restrict__ j0tab, const float* __restrict__ atab,
                                      int n, int H, int W, int K)
{
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)n * K * W;
  if (idx >= tot) return;
  const int i = (int)(idx % W);
  const long long r = idx / W;
  const int k = (int)(r % K), t = (int)(r / K);
  const int j0 = j0tab[(size_t)k * W + i];
  float val = 0.0f;
  if (j0 >= 0) {
    const float a = atab[(size_t)k * W + i];
    const float* col = g2 + (size_t)t * H * W + i;
    const float v0 = col[(size_t)j0 * W];
    const float v1 = (j0 + 1 < H) ? col[(size_t)(j0 + 1) * W] : v0;
    val = fmaf(a, v1 - v0, v0);
  }
  g3[idx] = val;
}

// Hilbert transform of each row along u: out[i] = sgn * sum_j h(i - j) in[j],
// h(m) = 2 / (pi m) for odd m, 0 otherwise; one block per row, the row staged in shared memory.
__global__ void kats_hilbert_kernel(const float* __restrict__ in, float* __restrict__ out, int W,
                                    float sgn)
{
  extern __shared__ float row[];
  const size_t r = blockIdx.x;
  for (int j = threadIdx.x; j < W; j += blockDim.x) row[j] = in[r * W + j];
  __syncthreads();
  const float c = sgn * 0.63661977236758134f;  // 2 / pi
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    float acc = 0.0f;
    // j = i - m with m odd: j runs over the columns of opposite parity to i
    for (int j = (i & 1) ^ 1; j < W; j += 2) acc = fmaf(row[j], __frcp_rn((float)(i - j)), acc);
    out[r * W + i] = c * acc;
  }
}

// FFT form of the same transform: rows zero-padded to L = 2W (linear, not circular,
// convolution for |i - j| < W), multiplied by the spectrum of the discrete kernel, inverted.
__global__ void kats_pad_kernel(const float* __restrict__ in, float* __restrict__ pad, long long row0,
                                int nrows, int W, int L)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nrows * L) return;
  const int c = (int)(i % L);
  const long long r = i / L;
  pad[i] = c < W ? in[(row0 + r) * W + c] : 0.0f;
}

// spec[r][k] *= i * himag[k] (the kernel is odd, so its spectrum is purely imaginary)
__global__ void kats_spec_kernel(cufftComplex* __restrict__ spec, const float* __restrict__ himag,
                                 int nrows, int nb)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nrows * nb) return;
  const float h = himag[i % nb];
  const cufftComplex z = spec[i];
  spec[i] = make_cuFloatComplex(-z.y * h, z.x * h);
}

__global__ void kats_crop_kernel(const float* __restrict__ pad, float* __restrict__ out, long long row0,
                                 int nrows, int W, int L, float scale)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nrows * W) return;
  const int c = (int)(i % W);
  const long long r = i / W;
  out[(row0 + r) * W + c] = scale * pad[r * L + c];
}

// gF[t][j][i] = g4[t][k0][i] * (1-a) + g4[t][k0+1][i] * a from the (row, column) table
__global__ void kats_rebin_bwd_kernel(const float* __restrict__ g4, float* __restrict__ gF,
                                      const int* __restrict__ k0tab, const float* __restrict__ atab,
                                      int n, int H, int W, int K)
{
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)n * H * W;
  if (idx >= tot) return;
  const int i = (int)(idx % W);
  const long long r = idx / W;
  const int j = (int)(r % H), t = (int)(r / H);
  const int k0 = k0tab[(size_t)j * W + i];
  const float a = atab[(size_t)j * W + i];
  const float* col = g4 + (size_t)t * K * W + i;
  const float v0 = col[(size_t)k0 * W], v1 = col[(size_t)(k0 + 1) * W];
  gF[idx] = fmaf(a, v1 - v0, v0);
}

}  // namespace fcb

using namespace fcb;

// np.interp-style lookup on an increasing abscissa: fractional index of x in xs.
static double frac_index(const std::vector<double>& xs, double x)
{
  const int n = (int)xs.size();
  if (x <= xs[0]) return 0.0;
  if (x >= xs[n - 1]) return (double)(n - 1);
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (xs[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo + (x - xs[lo]) / (xs[hi] - xs[lo]);
}

// Reusable Katsevich filter for one helix and detector: the kappa-line tables, the Hilbert
// kernel's spectrum, the cuFFT plans and the intermediate buffers are made once; execute()
// is stream-ordered, allocates nothing and does not synchronise.
struct fcb_katsevich_plan {
  int nviews = 0, H = 0, W = 0, K = 0, L = 0, nb = 0, batch = 0;
  float dlam = 0.0f, pw = 0.0f, D = 0.0f, su = 0.0f;
  float *g2 = nullptr, *g3 = nullptr, *g4 = nullptr, *dfa = nullptr, *dba = nullptr;
  int *dfj = nullptr, *dbk = nullptr;
  float *hpad = nullptr, *dhim = nullptr;
  cufftComplex* hspec = nullptr;
  cufftHandle pf = 0, pi = 0;
  ~fcb_katsevich_plan()
  {
    if (pf) cufftDestroy(pf);
    if (pi) cufftDestroy(pi);
    cudaFree(g2); cudaFree(g3); cudaFree(g4); cudaFree(dfa); cudaFree(dba); cudaFree(dfj);
    cudaFree(dbk); cudaFree(hpad); cudaFree(hspec); cudaFree(dhim);
  }
};

extern "C" int fcb_katsevich_plan_create(int nviews, int H, int W, const float* angles, float D,
                                         float pw, float pitch, int nkappa,
                                         fcb_katsevich_plan** out)
{
  if (!out) return set_error(FCB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (!angles || nviews < 2 || H < 2 || W < 2 || !(D > 0) || !(pw > 0) || pitch == 0.0f)
    return set_error(FCB_ERR_INVALID, "bad Katsevich filter arguments");
  // mean angular step; float32 angles of several turns carry ~1e-6 rad of rounding each
  const double dlam = ((double)angles[nviews - 1] - (double)angles[0]) / (nviews - 1);
  for (int t = 1; t < nviews; t++) {
    const double d = (double)angles[t] - (double)angles[t - 1];
    if (fabs(d - dlam) > 1e-3 * fabs(dlam) + 1e-5)
      return set_error(FCB_ERR_INVALID, "Katsevich filtering needs uniformly spaced views");
  }
  const double turn = (double)angles[nviews - 1] - (double)angles[0];
  const double su = ((turn >= 0.0) == (pitch >= 0.0)) ? -1.0 : 1.0;
  const int K = nkappa > 1 ? nkappa : 2 * H;
  // kappa-line tables (FP64): v_k(u_i, psi_k), forward (kappa, column) and backward (row, column)
  std::vector<double> u(W), v(H);
  for (int i = 0; i < W; i++) u[i] = su * (double)(i - W / 2) * pw;
  for (int j = 0; j < H; j++) v[j] = (double)(j - H / 2) * pw;
  double umax = 0.0;
  for (int i = 0; i < W; i++) umax = std::max(umax, fabs(u[i]));
  const double am = atan(umax / D);
  const double P = pitch;
  std::vector<int> fj0((size_t)K * W), bk0((size_t)H * W);
  std::vector<float> fa((size_t)K * W), ba((size_t)H * W);
  std::vector<double> vk(K);
  for (int i = 0; i < W; i++) {
    for (int k = 0; k < K; k++) {
      const double psi = -M_PI / 2 - am + (M_PI + 2 * am) * k / (double)(K - 1);
      const double cot = fabs(psi) < 1e-12 ? 1.0 : psi / tan(psi);
      vk[k] = (P / (2 * M_PI)) * (psi + cot * u[i] / D);
      // forward: linear interpolation in v, zero outside the detector rows
      const double x = vk[k];
      if (x < v[0] || x > v[H - 1]) {
        fj0[(size_t)k * W + i] = -1;
        fa[(size_t)k * W + i] = 0.0f;
      } else {
        const double f = frac_index(v, x);
        const int j0 = std::min((int)floor(f), H - 2);
        fj0[(size_t)k * W + i] = j0;
        fa[(size_t)k * W + i] = (float)(f - j0);
      }
    }
    for (int j = 0; j < H; j++) {
      const double f = frac_index(vk, v[j]);
      const int k0 = std::min((int)floor(f), K - 2);
      bk0[(size_t)j * W + i] = k0;
      ba[(size_t)j * W + i] = (float)(f - k0);
    }
  }
  // spectrum of the Hilbert kernel embedded in L = 2W: h(m) = 2/(pi m) for odd m,
  // h(L-m) = -h(m); H[k] = -2 i sum_{m odd < W} h(m) sin(2 pi k m / L)
  const int L = 2 * W, nb = W + 1;
  std::vector<float> himag(nb);
  for (int k = 0; k < nb; k++) {
    double acc = 0.0;
    for (int m = 1; m < W; m += 2) acc += (2.0 / (M_PI * m)) * sin(2.0 * M_PI * (double)k * m / L);
    himag[k] = (float)(-2.0 * acc);
  }
  auto* pl = new fcb_katsevich_plan();
  pl->nviews = nviews; pl->H = H; pl->W = W; pl->K = K; pl->L = L; pl->nb = nb;
  pl->dlam = (float)dlam; pl->pw = pw; pl->D = D; pl->su = (float)su;
  const long long rows = (long long)nviews * K;
  pl->batch = (int)std::min<long long>(rows, std::max<long long>(1, (256ll << 20) / (8ll * L)));
  const size_t nhw = (size_t)nviews * H * W, nkw = (size_t)nviews * K * W;
  int rc = FCB_OK;
  do {
    if (cudaMalloc(&pl->g2, nhw * 4) || cudaMalloc(&pl->g3, nkw * 4) || cudaMalloc(&pl->g4, nkw * 4) ||
        cudaMalloc(&pl->dfa, fa.size() * 4) || cudaMalloc(&pl->dba, ba.size() * 4) ||
        cudaMalloc(&pl->dfj, fj0.size() * 4) || cudaMalloc(&pl->dbk, bk0.size() * 4) ||
        cudaMalloc(&pl->hpad, (size_t)pl->batch * L * 4) ||
        cudaMalloc(&pl->hspec, (size_t)pl->batch * nb * sizeof(cufftComplex)) || cudaMalloc(&pl->dhim, nb * 4)) {
      cudaGetLastError();
      rc = set_error(FCB_ERR_NOMEM, "Katsevich filter scratch");
      break;
    }
    if (cudaMemcpy(pl->dfa, fa.data(), fa.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(pl->dba, ba.data(), ba.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(pl->dfj, fj0.data(), fj0.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(pl->dbk, bk0.data(), bk0.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(pl->dhim, himag.data(), nb * 4, cudaMemcpyHostToDevice)) {
      rc = set_error(FCB_ERR_CUDA, "Katsevich table upload failed");
      break;
    }
    int n1[1] = {L};
    if (cufftPlanMany(&pl->pf, 1, n1, nullptr, 1, L, nullptr, 1, nb, CUFFT_R2C, pl->batch) != CUFFT_SUCCESS ||
        cufftPlanMany(&pl->pi, 1, n1, nullptr, 1, nb, nullptr, 1, L, CUFFT_C2R, pl->batch) != CUFFT_SUCCESS) {
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

extern "C" int fcb_katsevich_plan_execute(fcb_katsevich_plan* pl, const float* in, float* out,
                                          void* stream)
{
  if (!pl || !in || !out) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int nviews = pl->nviews, H = pl->H, W = pl->W, K = pl->K, L = pl->L, nb = pl->nb;
  const size_t nhw = (size_t)nviews * H * W, nkw = (size_t)nviews * K * W;
  kats_deriv_kernel<<<(unsigned)((nhw + 255) / 256), 256, 0, st>>>(in, pl->g2, nviews, H, W, pl->dlam,
                                                                   pl->pw, pl->D, pl->su);
  kats_rebin_fwd_kernel<<<(unsigned)((nkw + 255) / 256), 256, 0, st>>>(pl->g2, pl->g3, pl->dfj, pl->dfa,
                                                                       nviews, H, W, K);
  // the published Hilbert transform runs along increasing u; along w it changes sign when u = -w
  const char* direct = getenv("FCB_KATS_DIRECT_HILBERT");
  if (direct && direct[0] == '1') {
    kats_hilbert_kernel<<<(unsigned)((size_t)nviews * K), 256, W * sizeof(float), st>>>(pl->g3, pl->g4, W,
                                                                                        pl->su);
  } else {
    if (cufftSetStream(pl->pf, st) != CUFFT_SUCCESS || cufftSetStream(pl->pi, st) != CUFFT_SUCCESS)
      return set_error(FCB_ERR_CUDA, "cufftSetStream failed");
    const float scale = pl->su / (float)L;
    const long long rows = (long long)nviews * K;
    const int batch = pl->batch;
    for (long long r0 = 0; r0 < rows; r0 += batch) {
      const int nr = (int)std::min<long long>(batch, rows - r0);
      kats_pad_kernel<<<(unsigned)(((long long)batch * L + 255) / 256), 256, 0, st>>>(pl->g3, pl->hpad, r0, nr, W, L);
      if (nr < batch)
        FCB_CUDA_TRY(cudaMemsetAsync(pl->hpad + (size_t)nr * L, 0, (size_t)(batch - nr) * L * 4, st));
      if (cufftExecR2C(pl->pf, pl->hpad, pl->hspec) != CUFFT_SUCCESS) return set_error(FCB_ERR_CUDA, "cufftExecR2C failed");
      kats_spec_kernel<<<(unsigned)(((long long)nr * nb + 255) / 256), 256, 0, st>>>(pl->hspec, pl->dhim, nr, nb);
      if (cufftExecC2R(pl->pi, pl->hspec, pl->hpad) != CUFFT_SUCCESS) return set_error(FCB_ERR_CUDA, "cufftExecC2R failed");
      kats_crop_kernel<<<(unsigned)(((long long)nr * W + 255) / 256), 256, 0, st>>>(pl->hpad, pl->g4, r0, nr, W, L, scale);
    }
  }
  kats_rebin_bwd_kernel<<<(unsigned)((nhw + 255) / 256), 256, 0, st>>>(pl->g4, out, pl->dbk, pl->dba, nviews, H,
                                                                      W, K);
  FCB_CUDA_TRY(cudaGetLastError());
  return ok();
}

extern "C" int fcb_katsevich_plan_destroy(fcb_katsevich_plan* pl)
{
  delete pl;
  return ok();
}

extern "C" int fcb_katsevich_filter_device(const float* in, float* out, int nviews, int H, int W,
                                           const float* angles, float D, float pw, float pitch,
                                           int nkappa, void* stream)
{
  if (!in || !out) return set_error(FCB_ERR_INVALID, "bad Katsevich filter arguments");
  fcb_katsevich_plan* pl = nullptr;
  FCB_TRY(fcb_katsevich_plan_create(nviews, H, W, angles, D, pw, pitch, nkappa, &pl));
  const int rc = fcb_katsevich_plan_execute(pl, in, out, stream);
  // the plan's buffers are freed below; wait for the queued work that uses them
  const cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
  fcb_katsevich_plan_destroy(pl);
  if (rc) return rc;
  if (e != cudaSuccess) return set_error(FCB_ERR_CUDA, cudaGetErrorString(e));
  return ok();
}
