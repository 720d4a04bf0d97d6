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
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

// Element-wise stages: each thread handles CPT consecutive columns (4 with 16-byte vector
// loads and stores when W is a multiple of 4, else 1); grid.x runs over the column groups of
// one view, grid.y over the views.
template <int CPT>
__device__ __forceinline__ void ldv(const float* __restrict__ p, float (&v)[CPT])
{
  if constexpr (CPT == 4) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    v[0] = *p;
  }
}
template <int CPT>
__device__ __forceinline__ void ldv(const int* __restrict__ p, int (&v)[CPT])
{
  if constexpr (CPT == 4) {
    const int4 x = *reinterpret_cast<const int4*>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    v[0] = *p;
  }
}
template <int CPT>
__device__ __forceinline__ void stv(float* __restrict__ p, const float (&v)[CPT])
{
  if constexpr (CPT == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else *p = v[0];
}

// Reciprocals of the step sizes, computed once on the host: the kernel multiplies instead
// of dividing (no per-element IEEE division).
struct KatsDerivConst {
  float idl, hidl;   // 1 / dlam, 1 / (2 dlam)
  float idu, hidu;   // 1 / du, 1 / (2 du), du = su pw
  float ipw, hipw;   // 1 / pw, 1 / (2 pw)
  float pw, D, iD, su;
};

template <int CPT>
__global__ void kats_deriv_kernel(const float* __restrict__ g, float* __restrict__ g2, int n, int H,
                                  int W, const KatsDerivConst K)
{
  const int Wq = W / CPT;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= H * Wq) return;
  const int t = blockIdx.y;
  const int j = q / Wq, i0 = (q - j * Wq) * CPT;
  const size_t plane = (size_t)H * W;
  const size_t o = (size_t)t * plane + (size_t)j * W + i0;
  float c[CPT], a[CPT], b[CPT], dl[CPT], dgu[CPT], dgv[CPT], r[CPT];
  ldv<CPT>(g + o, c);
  // dg/dlam: central inside, one-sided at the ends (numpy.gradient, edge order 1)
  if (n == 1) {
#pragma unroll
    for (int k = 0; k < CPT; k++) dl[k] = 0.0f;
  } else if (t == 0) {
    ldv<CPT>(g + o + plane, a);
#pragma unroll
    for (int k = 0; k < CPT; k++) dl[k] = (a[k] - c[k]) * K.idl;
  } else if (t == n - 1) {
    ldv<CPT>(g + o - plane, b);
#pragma unroll
    for (int k = 0; k < CPT; k++) dl[k] = (c[k] - b[k]) * K.idl;
  } else {
    ldv<CPT>(g + o + plane, a);
    ldv<CPT>(g + o - plane, b);
#pragma unroll
    for (int k = 0; k < CPT; k++) dl[k] = (a[k] - b[k]) * K.hidl;
  }
  // dg/du with u_i = su * (i - W/2) pw; e = the row from column i0 - 1 to i0 + CPT
  float e[CPT + 2];
  e[0] = i0 > 0 ? g[o - 1] : 0.0f;
#pragma unroll
  for (int k = 0; k < CPT; k++) e[k + 1] = c[k];
  e[CPT + 1] = i0 + CPT < W ? g[o + CPT] : 0.0f;
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    const int i = i0 + k;
    if (W == 1) dgu[k] = 0.0f;
    else if (i == 0) dgu[k] = (e[k + 2] - e[k + 1]) * K.idu;
    else if (i == W - 1) dgu[k] = (e[k + 1] - e[k]) * K.idu;
    else dgu[k] = (e[k + 2] - e[k]) * K.hidu;
  }
  if (H == 1) {
#pragma unroll
    for (int k = 0; k < CPT; k++) dgv[k] = 0.0f;
  } else if (j == 0) {
    ldv<CPT>(g + o + W, a);
#pragma unroll
    for (int k = 0; k < CPT; k++) dgv[k] = (a[k] - c[k]) * K.ipw;
  } else if (j == H - 1) {
    ldv<CPT>(g + o - W, b);
#pragma unroll
    for (int k = 0; k < CPT; k++) dgv[k] = (c[k] - b[k]) * K.ipw;
  } else {
    ldv<CPT>(g + o + W, a);
    ldv<CPT>(g + o - W, b);
#pragma unroll
    for (int k = 0; k < CPT; k++) dgv[k] = (a[k] - b[k]) * K.hipw;
  }
  const float v = (float)(j - H / 2) * K.pw;
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    const float u = K.su * (float)(i0 + k - W / 2) * K.pw;
    const float q2 = u * u + K.D * K.D;
    const float g1 = dl[k] + (q2 * K.iD) * dgu[k] + (u * v * K.iD) * dgv[k];
    r[k] = g1 * (K.D * rsqrtf(q2 + v * v));
  }
  stv<CPT>(g2 + o, r);
}

// g3[t][k][i] = g2[t][j0][i] * (1-a) + g2[t][j0+1][i] * a from the (kappa, column) table,
// into rows of length L whose columns [W, L) stay zero (the Hilbert transform's padding,
// written once when the plan is made).
template <int CPT>
__global__ void kats_rebin_fwd_kernel(const float* __restrict__ g2, float* __restrict__ g3,
                                      const int* __restrict__ j0tab, const float* __restrict__ atab,
                                      int H, int W, int K, int L)
{
  const int Wq = W / CPT;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= K * Wq) return;
  const int t = blockIdx.y;
  const int k = q / Wq, i0 = (q - k * Wq) * CPT;
  int j0[CPT];
  float a[CPT], val[CPT];
  ldv<CPT>(j0tab + (size_t)k * W + i0, j0);
  ldv<CPT>(atab + (size_t)k * W + i0, a);
  const float* base = g2 + (size_t)t * H * W + i0;
#pragma unroll
  for (int m = 0; m < CPT; m++) {
    val[m] = 0.0f;
    if (j0[m] >= 0) {
      const float* col = base + m;
      const float v0 = col[(size_t)j0[m] * W];
      const float v1 = (j0[m] + 1 < H) ? col[(size_t)(j0[m] + 1) * W] : v0;
      val[m] = fmaf(a[m], v1 - v0, v0);
    }
  }
  stv<CPT>(g3 + ((size_t)t * K + k) * L + i0, val);
}

// Hilbert transform of each row along u: out[i] = sgn * sum_j h(i - j) in[j],
// h(m) = 2 / (pi m) for odd m, 0 otherwise; one block per row (stride L), the row staged in
// shared memory (so the transform may run in place).
__global__ void kats_hilbert_kernel(float* __restrict__ rows, int W, int L, float sgn)
{
  extern __shared__ float row[];
  const size_t r = blockIdx.x;
  for (int j = threadIdx.x; j < W; j += blockDim.x) row[j] = rows[r * L + j];
  __syncthreads();
  const float c = sgn * 0.63661977236758134f;  // 2 / pi
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    float acc = 0.0f;
    // j = i - m with m odd: j runs over the columns of opposite parity to i
    for (int j = (i & 1) ^ 1; j < W; j += 2) acc = fmaf(row[j], __frcp_rn((float)(i - j)), acc);
    rows[r * L + i] = c * acc;
  }
}

// spec[r][k] *= i * himag[k] (the kernel is odd, so its spectrum is purely imaginary)
// One block per row.
__global__ void kats_spec_kernel(cufftComplex* __restrict__ spec, const float* __restrict__ himag,
                                 int nb)
{
  cufftComplex* row = spec + (size_t)blockIdx.x * nb;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const float h = himag[k];
    const cufftComplex z = row[k];
    row[k] = make_cuFloatComplex(-z.y * h, z.x * h);
  }
}

// gF[t0 + tl][j][i] = scale * (g4[tl][k0][i] * (1-a) + g4[tl][k0+1][i] * a) from the
// (row, column) table; g4 holds the transformed kappa rows (length L) of views t0, t0 + 1, ...
template <int CPT>
__global__ void kats_rebin_bwd_kernel(const float* __restrict__ g4, float* __restrict__ gF,
                                      const int* __restrict__ k0tab, const float* __restrict__ atab,
                                      int H, int W, int K, int L, float scale, int t0)
{
  const int Wq = W / CPT;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= H * Wq) return;
  const int tl = blockIdx.y;
  const int j = q / Wq, i0 = (q - j * Wq) * CPT;
  int k0[CPT];
  float a[CPT], r[CPT];
  ldv<CPT>(k0tab + (size_t)j * W + i0, k0);
  ldv<CPT>(atab + (size_t)j * W + i0, a);
  const float* base = g4 + (size_t)tl * K * L + i0;
#pragma unroll
  for (int m = 0; m < CPT; m++) {
    const float* col = base + m;
    const float v0 = col[(size_t)k0[m] * L], v1 = col[(size_t)(k0[m] + 1) * L];
    r[m] = scale * fmaf(a[m], v1 - v0, v0);
  }
  stv<CPT>(gF + ((size_t)(t0 + tl) * H + j) * W + i0, r);
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
  int nviews = 0, H = 0, W = 0, K = 0, L = 0, nb = 0;
  int vb = 0;  // views per transform batch (the batch is vb * K kappa rows)
  float dlam = 0.0f, pw = 0.0f, D = 0.0f, su = 0.0f;
  float *g2 = nullptr, *dfa = nullptr, *dba = nullptr;
  float* g3 = nullptr;  // kappa rows [views rounded up to whole batches][K][L]; [W, L) zero
  float* g4 = nullptr;  // one batch of transformed rows [vb][K][L]
  int *dfj = nullptr, *dbk = nullptr;
  float* dhim = nullptr;
  cufftComplex* hspec = nullptr;  // one batch of spectra
  cufftHandle pf = 0, pi = 0;
  ~fcb_katsevich_plan()
  {
    if (pf) cufftDestroy(pf);
    if (pi) cufftDestroy(pi);
    cudaFree(g2); cudaFree(g3); cudaFree(g4); cudaFree(dfa); cudaFree(dba); cudaFree(dfj);
    cudaFree(dbk); cudaFree(hspec); cudaFree(dhim);
  }
};

extern "C" int fcb_katsevich_plan_create(int nviews, int H, int W, const float* angles, float D,
                                         float pw, float pitch, int nkappa,
                                         fcb_katsevich_plan** out)
try {
  if (!out) return set_error(FCB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (!angles || nviews < 2 || H < 2 || W < 2 || !(D > 0) || !(pw > 0) || pitch == 0.0f)
    return set_error(FCB_ERR_INVALID, "bad Katsevich filter arguments");
  if (nviews > 65535 || H > 32768 || (nkappa > 1 && nkappa > 65535))
    return set_error(FCB_ERR_INVALID, "Katsevich filter sizes above the grid limits (65535 views)");
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
  // transform batches of whole views, up to 256 MiB of spectra each (larger batches gain
  // nothing per transform and make the cuFFT plans and buffers slower to create); the
  // kappa-row array is rounded up to whole batches and zeroed once (padding columns and rows
  // are never written)
  pl->vb = (int)std::min<long long>(nviews, std::max<long long>(1, (256ll << 20) / (8ll * nb * K)));
  const long long rows_alloc = (long long)((nviews + pl->vb - 1) / pl->vb) * pl->vb * K;
  const long long batch = (long long)pl->vb * K;
  const size_t nhw = (size_t)nviews * H * W;
  int rc = FCB_OK;
  do {
    if (cudaMalloc(&pl->g2, nhw * 4) || cudaMalloc(&pl->g3, (size_t)rows_alloc * L * 4) ||
        cudaMalloc(&pl->g4, (size_t)batch * L * 4) ||
        cudaMalloc(&pl->dfa, fa.size() * 4) || cudaMalloc(&pl->dba, ba.size() * 4) ||
        cudaMalloc(&pl->dfj, fj0.size() * 4) || cudaMalloc(&pl->dbk, bk0.size() * 4) ||
        cudaMalloc(&pl->hspec, (size_t)batch * nb * sizeof(cufftComplex)) || cudaMalloc(&pl->dhim, nb * 4)) {
      cudaGetLastError();
      rc = set_error(FCB_ERR_NOMEM, "Katsevich filter scratch");
      break;
    }
    if (cudaMemset(pl->g3, 0, (size_t)rows_alloc * L * 4) != cudaSuccess) {
      rc = set_error(FCB_ERR_CUDA, "Katsevich scratch initialisation failed");
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
    if (cufftPlanMany(&pl->pf, 1, n1, nullptr, 1, L, nullptr, 1, nb, CUFFT_R2C, (int)batch) != CUFFT_SUCCESS ||
        cufftPlanMany(&pl->pi, 1, n1, nullptr, 1, nb, nullptr, 1, L, CUFFT_C2R, (int)batch) != CUFFT_SUCCESS) {
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

extern "C" int fcb_katsevich_plan_execute(fcb_katsevich_plan* pl, const float* in, float* out,
                                          void* stream)
try {
  if (!pl || !in || !out) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int nviews = pl->nviews, H = pl->H, W = pl->W, K = pl->K, L = pl->L, nb = pl->nb;
  // 16-byte vector accesses need 4 | W and 16-byte aligned caller buffers (the plan's own are)
  const bool v4 = (W % 4) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0 &&
                  (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  const int cpt = v4 ? 4 : 1;
  const unsigned bx_hw = (unsigned)(((long long)H * (W / cpt) + 255) / 256);
  const unsigned bx_kw = (unsigned)(((long long)K * (W / cpt) + 255) / 256);
  KatsDerivConst KC;
  {
    const double dl = pl->dlam, du = (double)pl->su * pl->pw, pw = pl->pw, D = pl->D;
    KC.idl = (float)(1.0 / dl);
    KC.hidl = (float)(0.5 / dl);
    KC.idu = (float)(1.0 / du);
    KC.hidu = (float)(0.5 / du);
    KC.ipw = (float)(1.0 / pw);
    KC.hipw = (float)(0.5 / pw);
    KC.pw = pl->pw;
    KC.D = pl->D;
    KC.iD = (float)(1.0 / D);
    KC.su = pl->su;
  }
  if (v4) {
    kats_deriv_kernel<4><<<dim3(bx_hw, nviews), 256, 0, st>>>(in, pl->g2, nviews, H, W, KC);
    kats_rebin_fwd_kernel<4><<<dim3(bx_kw, nviews), 256, 0, st>>>(pl->g2, pl->g3, pl->dfj, pl->dfa, H, W, K, L);
  } else {
    kats_deriv_kernel<1><<<dim3(bx_hw, nviews), 256, 0, st>>>(in, pl->g2, nviews, H, W, KC);
    kats_rebin_fwd_kernel<1><<<dim3(bx_kw, nviews), 256, 0, st>>>(pl->g2, pl->g3, pl->dfj, pl->dfa, H, W, K, L);
  }
  auto rebin_bwd = [&](const float* rows, int t0, int nv, float scale) {
    if (v4) kats_rebin_bwd_kernel<4><<<dim3(bx_hw, nv), 256, 0, st>>>(rows, out, pl->dbk, pl->dba, H, W, K, L, scale, t0);
    else kats_rebin_bwd_kernel<1><<<dim3(bx_hw, nv), 256, 0, st>>>(rows, out, pl->dbk, pl->dba, H, W, K, L, scale, t0);
  };
  // the published Hilbert transform runs along increasing u; along w it changes sign when u = -w
  const char* direct = getenv("FCB_KATS_DIRECT_HILBERT");
  if (direct && direct[0] == '1') {
    kats_hilbert_kernel<<<(unsigned)((size_t)nviews * K), 256, W * sizeof(float), st>>>(pl->g3, W, L, pl->su);
    rebin_bwd(pl->g3, 0, nviews, 1.0f);
  } else {
    if (cufftSetStream(pl->pf, st) != CUFFT_SUCCESS || cufftSetStream(pl->pi, st) != CUFFT_SUCCESS)
      return set_error(FCB_ERR_CUDA, "cufftSetStream failed");
    const float scale = pl->su / (float)L;
    const int vb = pl->vb;
    // per batch of whole views: R2C of the zero-padded kappa rows, multiplication by the
    // kernel's spectrum, C2R into g4 (the padding in g3 stays zero), backward rebinning of
    // the batch's views with the 1/L normalisation and the direction sign
    for (int t0 = 0; t0 < nviews; t0 += vb) {
      const int nv = std::min(vb, nviews - t0);
      if (cufftExecR2C(pl->pf, pl->g3 + (size_t)t0 * K * L, pl->hspec) != CUFFT_SUCCESS)
        return set_error(FCB_ERR_CUDA, "cufftExecR2C failed");
      kats_spec_kernel<<<(unsigned)((long long)nv * K), 256, 0, st>>>(pl->hspec, pl->dhim, nb);
      if (cufftExecC2R(pl->pi, pl->hspec, pl->g4) != CUFFT_SUCCESS) return set_error(FCB_ERR_CUDA, "cufftExecC2R failed");
      rebin_bwd(pl->g4, t0, nv, scale);
    }
  }
  FCB_CUDA_TRY(cudaGetLastError());
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_katsevich_plan_destroy(fcb_katsevich_plan* pl)
try {
  delete pl;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_katsevich_filter_device(const float* in, float* out, int nviews, int H, int W,
                                           const float* angles, float D, float pw, float pitch,
                                           int nkappa, void* stream)
try {
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
FCB_CATCH_STATUS
