// fcb_backproject.cu -- voxel-driven cone-beam backprojection for sm_100a.
//
// Replaces GPU_Feldkamp_backproject_sinogram / GPU_Katsevich_backproject_sinogram
// (coneBeamGPU.cu:258-420), GPU_unweighted_backproject_sinogram (:178-255), their launchers
// (:565-704) and the problem-solver drivers (unit_coneBeamGPU.cu:173-305).
//
// Two kernels:
//  * fdk_tma_kernel -- aligned circular/helical geometry (FDK weight U^2, Katsevich U with
//    optional Tam-Danielsson window, or unweighted).  A CTA owns a 16 x 16 x NZ voxel
//    tile; per view a producer warp stages the tile's detector footprint (a fixed
//    BW x BH box, zero-filled outside the caller's window) into shared memory with a TMA
//    load, and 8 consumer warps interpolate bilinearly in FP32 from it.  Each thread owns
//    one (x, y) column and NZ z-voxels held in registers; along z only the detector row
//    changes, so the per-view work (U, w, weight) is amortised over NZ updates.  Per-view
//    parameters travel in the kernel's parameter space (a constant bank).
//  * bp_generic_kernel -- any detector orientation (misalignments) through a per-view 3x4
//    projective matrix, bilinear gathers from global memory; also the fallback for
//    projection buffers whose layout a TMA descriptor cannot describe.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <utility>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

// =====================================================================================
// TMA-staged FDK / Katsevich kernel
// =====================================================================================
struct FdkView {
  float c0, c1;  // den = 1 + c0 x + c1 y ; U = 1 / den
  float a0, a1;  // w = (a0 x + a1 y) U + wc
  float wc, hc;  // local window index of the detector centre (w) / source height (h)
  float e;       // h = U (hb z + e) + hc
  float wt;      // normalisation factor of the view
};

constexpr int FDK_MAXV = 900;      // views a launch's parameters can hold
constexpr int FDK_L2_VIEWS = 180;  // views per launch by default (see bp_plan_build)
constexpr int FDK_TX = 16, FDK_TY = 16;
constexpr int FDK_CWARPS = 8;                          // consumer warps
constexpr int FDK_THREADS = (FDK_CWARPS + 1) * 32;     // + producer warp

struct FdkParams {
  float* vol;
  int* status;
  int nx, ny, nz;               // local sub-volume extents (x fastest)
  int tiles_x, tiles_y, tiles_z;
  int tile0;                    // first tile of this launch (launches may cover z-ranges)
  float ox, oy, oz;             // coordinate of local voxel (0,0,0) relative to volDim/2
  int nviews, view0;
  int BW, BH, stages, wshift;
  float hb;                     // 1 / pixelWidth
  int wexp;                     // weight exponent: 2 FDK, 1 Katsevich, 0 unweighted
  int yfast;                    // tile raster: 0 x fastest, 1 y fastest (see fdk_tile)
  int piwin;                    // Tam-Danielsson window on/off
  float td_a;                   // window half-height scale P / (2 pi pw), pixels
  float td_r;                   // source-axis distance in pixels (D / pw)
  float td_sign;                // +1/-1: sense of the helix relative to the w axis
  float td_usc;                 // td_sign / td_r (a multiply per staged view instead of a division)
  // Bounded waits.  cwait_ns limits each consumer wait for a staged view (2 s by default).
  // stop_after >= 0 is a test hook: the producer stages only that many views, drains its
  // copies and leaves, so the consumers' next wait runs out and the kernel reports
  // DEV_TIMEOUT without any copy still in flight.
  unsigned long long cwait_ns;
  int stop_after;
  int pbufs;                    // 16-bit storage: tap-pair buffers (fdk_pair_kernel)
  FdkView v[FDK_MAXV];
};

static_assert(sizeof(FdkParams) + sizeof(CUtensorMap) < 32000, "kernel parameter space");

__device__ __forceinline__ void fdk_footprint(const FdkParams& P, const FdkView& V, float x0,
                                              float x1, float y0, float y1, float z0, float z1,
                                              float& wmin, float& wmax, float& hmin, float& hmax)
{
  wmin = 3.0e38f; wmax = -3.0e38f; hmin = 3.0e38f; hmax = -3.0e38f;
  const float hz0 = fmaf(P.hb, z0, V.e), hz1 = fmaf(P.hb, z1, V.e);
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float x = (c & 1) ? x1 : x0, y = (c & 2) ? y1 : y0;
    const float den = fmaf(V.c0, x, fmaf(V.c1, y, 1.0f));
    const float U = __frcp_rn(den);
    const float w = fmaf(fmaf(V.a0, x, V.a1 * y), U, V.wc);
    const float ha = fmaf(U, hz0, V.hc), hb = fmaf(U, hz1, V.hc);
    wmin = fminf(wmin, w); wmax = fmaxf(wmax, w);
    hmin = fminf(hmin, fminf(ha, hb)); hmax = fmaxf(hmax, fmaxf(ha, hb));
  }
}

// Tile of a linear tile index, z slowest.  The launch's views decide which of x and y runs
// fastest: the one that moves the detector column less, so that the CTAs resident at one
// time read a narrow band of detector columns and it stays in L2.
__device__ __forceinline__ void fdk_tile(const FdkParams& P, int tile, int& tx, int& ty, int& tz)
{
  const int layer = P.tiles_x * P.tiles_y;
  tz = tile / layer;
  const int r = tile - tz * layer;
  if (P.yfast) {
    ty = r % P.tiles_y;
    tx = r / P.tiles_y;
  } else {
    tx = r % P.tiles_x;
    ty = r / P.tiles_x;
  }
}

// Box origin of (tile, view): the footprint's lower corner minus one pixel, w aligned down
// to the TMA 16-byte rule.
__device__ __forceinline__ void fdk_box_origin(const FdkParams& P, const FdkView& V, int tx,
                                               int ty, int tz, int nzt, int& w0, int& h0,
                                               int& needw, int& needh, float* fp = nullptr)
{
  const float x0 = P.ox + tx * FDK_TX, y0 = P.oy + ty * FDK_TY, z0 = P.oz + tz * nzt;
  float wmin, wmax, hmin, hmax;
  fdk_footprint(P, V, x0, x0 + (FDK_TX - 1), y0, y0 + (FDK_TY - 1), z0, z0 + (nzt - 1), wmin,
                wmax, hmin, hmax);
  if (fp) { fp[0] = wmin; fp[1] = wmax; fp[2] = hmin; fp[3] = hmax; }
  // clamp far-away footprints so the integer math below stays defined
  wmin = fminf(fmaxf(wmin, -1.0e6f), 1.0e6f); wmax = fminf(fmaxf(wmax, -1.0e6f), 1.0e6f);
  hmin = fminf(fmaxf(hmin, -1.0e6f), 1.0e6f); hmax = fminf(fmaxf(hmax, -1.0e6f), 1.0e6f);
  const int wlo = __float2int_rd(wmin) - 1;
  w0 = (wlo >> P.wshift) << P.wshift;
  h0 = __float2int_rd(hmin) - 1;
  needw = __float2int_rd(wmax) + 3 - w0;
  needh = __float2int_rd(hmax) + 3 - h0;
}

// Katsevich PI window: true when no voxel of the tile can lie inside the Tam-Danielsson
// window of the view, so the view is skipped for the tile.  The window bounds are smooth in
// the detector column; over a tile's few columns their extremes are those at the ends and
// the middle to well under the 1-pixel margin kept here.
__device__ __forceinline__ bool fdk_tile_outside_window(const FdkParams& P, const FdkView& V,
                                                        float wmin, float wmax, float hmin,
                                                        float hmax)
{
  float lo = 3.0e38f, hi = -3.0e38f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float w = c == 0 ? wmin : (c == 1 ? 0.5f * (wmin + wmax) : wmax);
    const float u = (w - V.wc) * P.td_sign / P.td_r;
    const float q = P.td_a * (1.0f + u * u);
    const float at = atanf(u);
    hi = fmaxf(hi, V.hc + q * (1.5707963267948966f - at));
    lo = fminf(lo, V.hc - q * (1.5707963267948966f + at));
  }
  return hmin > hi + 1.0f || hmax < lo - 1.0f;
}

// Pre-pass: the largest footprint over all (tile, view) pairs sizes the staging box.
// Only the first and the last layer of z tiles are evaluated: for one view and one column of
// tiles the box width does not depend on z (w depends on x, y only) and the continuous
// extent of the rows, max over the corners of U (hb z1 + e) minus min of U (hb z0 + e), grows
// with the tile's distance from the source plane on either side, so it is largest in one of
// the two outer layers.  The plan adds one row for the floors of the box corners.
__global__ void fdk_footprint_kernel(const __grid_constant__ FdkParams P, int nzt, int ntiles,
                                     int* out_need)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int layer = P.tiles_x * P.tiles_y;
  const int nlayers = P.tiles_z > 1 ? 2 : 1;
  const long long total = (long long)layer * nlayers * P.nviews;
  (void)ntiles;
  int mw = 0, mh = 0;
  if (i < total) {
    const int t = (int)(i / P.nviews), v = (int)(i % P.nviews);
    const int tile = (t >= layer ? P.tiles_z - 1 : 0) * layer + t % layer;
    int tx, ty, tz;
    fdk_tile(P, tile, tx, ty, tz);
    int w0, h0, nw, nh;
    fdk_box_origin(P, P.v[v], tx, ty, tz, nzt, w0, h0, nw, nh);
    mw = nw;
    mh = nh;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mw = max(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    mh = max(mh, __shfl_xor_sync(0xffffffffu, mh, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out_need, mw);
    atomicMax(out_need + 1, mh);
  }
}

// ---- shared-memory taps: 32-bit addresses, immediate offsets, converted to float
typedef unsigned long long u64;

template <typename T, int OFF>
__device__ __forceinline__ float lds_tap(uint32_t a);
template <int OFF>
__device__ __forceinline__ float lds_f32(uint32_t a)
{
  float v;
  asm volatile("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(a), "n"(OFF));
  return v;
}
template <int OFF>
__device__ __forceinline__ uint32_t lds_u16(uint32_t a)
{
  unsigned short v;
  asm volatile("ld.shared.u16 %0, [%1+%2];" : "=h"(v) : "r"(a), "n"(OFF));
  return v;
}
template <typename T, int OFF>
struct Tap;
template <int OFF>
struct Tap<float, OFF> {
  static __device__ __forceinline__ float ld(uint32_t a) { return lds_f32<OFF * 4>(a); }
};
template <int OFF>
struct Tap<__half, OFF> {
  static __device__ __forceinline__ float ld(uint32_t a)
  {
    return __half2float(__ushort_as_half((unsigned short)lds_u16<OFF * 2>(a)));
  }
};
template <int OFF>
struct Tap<__nv_bfloat16, OFF> {
  static __device__ __forceinline__ float ld(uint32_t a) { return __uint_as_float(lds_u16<OFF * 2>(a) << 16); }
};

// Two FP32 taps (addresses a0 + OFF, a1 + OFF) loaded straight into the halves of one 64-bit
// f32x2 operand.
template <int OFF>
__device__ __forceinline__ unsigned long long lds_f32x2(uint32_t a0, uint32_t a1)
{
  unsigned long long r;
  asm volatile(
      "{\n\t.reg .f32 lo, hi;\n\t"
      "ld.shared.f32 lo, [%1+%3];\n\t"
      "ld.shared.f32 hi, [%2+%3];\n\t"
      "mov.b64 %0, {lo, hi};\n\t}"
      : "=l"(r)
      : "r"(a0), "r"(a1), "n"(OFF));
  return r;
}

// ---- 16-bit tap pairs: a staged 16-bit box rewritten as 32-bit words, word (r, c) holding
// tap (r, c) in its low half and tap (r, c + 1) in its high half, so that one 32-bit
// ld.shared gives both horizontal taps of a row
// A row's taps for two voxels from their tap-pair words at shared addresses a0, a1: LO =
// (tap c of voxel 0, tap c of voxel 1), HI = (tap c + 1 of voxel 0, of voxel 1), as f32x2
// operands written straight into their 64-bit registers.
template <typename T>
__device__ __forceinline__ void lds_pair_taps(uint32_t a0, uint32_t a1, unsigned long long& LO,
                                              unsigned long long& HI);
template <>
__device__ __forceinline__ void lds_pair_taps<__nv_bfloat16>(uint32_t a0, uint32_t a1, unsigned long long& LO,
                                                             unsigned long long& HI)
{
  asm volatile(
      "{\n\t.reg .b32 p, q, l0, l1, h0, h1;\n\t"
      "ld.shared.b32 p, [%2];\n\t"
      "ld.shared.b32 q, [%3];\n\t"
      "shl.b32 l0, p, 16;\n\t"
      "shl.b32 l1, q, 16;\n\t"
      "and.b32 h0, p, 0xffff0000;\n\t"
      "and.b32 h1, q, 0xffff0000;\n\t"
      "mov.b64 %0, {l0, l1};\n\t"
      "mov.b64 %1, {h0, h1};\n\t}"
      : "=l"(LO), "=l"(HI)
      : "r"(a0), "r"(a1));
}
template <>
__device__ __forceinline__ void lds_pair_taps<__half>(uint32_t a0, uint32_t a1, unsigned long long& LO,
                                                      unsigned long long& HI)
{
  asm volatile(
      "{\n\t.reg .b32 p, q;\n\t.reg .b16 p0, p1, q0, q1;\n\t.reg .f32 l0, l1, h0, h1;\n\t"
      "ld.shared.b32 p, [%2];\n\t"
      "ld.shared.b32 q, [%3];\n\t"
      "mov.b32 {p0, p1}, p;\n\t"
      "mov.b32 {q0, q1}, q;\n\t"
      "cvt.f32.f16 l0, p0;\n\t"
      "cvt.f32.f16 l1, q0;\n\t"
      "cvt.f32.f16 h0, p1;\n\t"
      "cvt.f32.f16 h1, q1;\n\t"
      "mov.b64 %0, {l0, l1};\n\t"
      "mov.b64 %1, {h0, h1};\n\t}"
      : "=l"(LO), "=l"(HI)
      : "r"(a0), "r"(a1));
}

// 8 staged 16-bit taps q (columns c .. c+7) and the first two of the next 16-byte chunk
// (nx) -> the pair words of columns c .. c+7
__device__ __forceinline__ void pair8(uint4 q, uint32_t nx, uint4& lo, uint4& hi)
{
  lo = make_uint4(q.x, __byte_perm(q.x, q.y, 0x5432), q.y, __byte_perm(q.y, q.z, 0x5432));
  hi = make_uint4(q.z, __byte_perm(q.z, q.w, 0x5432), q.w, __byte_perm(q.w, nx, 0x5432));
}

// ---- packed FP32 pairs (sm_100 f32x2 arithmetic): two z-voxels per instruction
__device__ __forceinline__ u64 pk2(float lo, float hi)
{
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void up2(u64 v, float& lo, float& hi)
{
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ u64 add2(u64 a, u64 b)
{
  u64 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 add2_rm(u64 a, u64 b)
{
  u64 r;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b)
{
  u64 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c)
{
  u64 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// f(integral_constant<int, K>) for K = lo, lo + 1, ..., hi, entered through a jump table on lo
// (nothing is tested for the K outside); lo <= hi < N, or lo >= N for none; N <= 32.
#define FCB_RUN_PAIR(K)                      \
  case K:                                    \
    if constexpr (K < N) {                   \
      f(std::integral_constant<int, K>{});   \
      if (hi == K) break;                    \
    }                                        \
    [[fallthrough]];
template <int N, typename F>
__device__ __forceinline__ void run_pairs(int lo, int hi, F&& f)
{
  static_assert(N <= 32, "pairs per thread");
  switch (lo) {
    FCB_RUN_PAIR(0) FCB_RUN_PAIR(1) FCB_RUN_PAIR(2) FCB_RUN_PAIR(3) FCB_RUN_PAIR(4)
    FCB_RUN_PAIR(5) FCB_RUN_PAIR(6) FCB_RUN_PAIR(7) FCB_RUN_PAIR(8) FCB_RUN_PAIR(9)
    FCB_RUN_PAIR(10) FCB_RUN_PAIR(11) FCB_RUN_PAIR(12) FCB_RUN_PAIR(13) FCB_RUN_PAIR(14)
    FCB_RUN_PAIR(15) FCB_RUN_PAIR(16) FCB_RUN_PAIR(17) FCB_RUN_PAIR(18) FCB_RUN_PAIR(19)
    FCB_RUN_PAIR(20) FCB_RUN_PAIR(21) FCB_RUN_PAIR(22) FCB_RUN_PAIR(23) FCB_RUN_PAIR(24)
    FCB_RUN_PAIR(25) FCB_RUN_PAIR(26) FCB_RUN_PAIR(27) FCB_RUN_PAIR(28) FCB_RUN_PAIR(29)
    FCB_RUN_PAIR(30) FCB_RUN_PAIR(31)
    default:
      break;
  }
}
#undef FCB_RUN_PAIR

// PI window: of the thread's NZ z-voxels (pairs k = (2k, 2k + 1)), the pairs that can lie
// inside the window of some lane of the warp, [plo, phi]; the warp runs only those
// (run_pairs: no taps loaded, no arithmetic for the others), the per-voxel test still decides
// inside.
// h(z_k) = h0 + k dh with dh > 0, so a lane's inside voxels are one run of k; one step of
// margin on each side covers the rounding of the incremental row positions.
template <int NACC>
__device__ __forceinline__ void piw_pairs(float lo, float hi, float h0, float dh, int& plo, int& phi)
{
  int a = 0, b = NACC - 1;
  if (dh > 0.0f) {
    const float lim = 2.0f * NACC + 4.0f;
    const float klo = fminf(fmaxf(__fdividef(lo - h0, dh), -4.0f), lim);
    const float khi = fminf(fmaxf(__fdividef(hi - h0, dh), -4.0f), lim);
    const int k0 = __float2int_ru(klo) - 1, k1 = __float2int_rd(khi) + 1;
    if (k1 < k0 || k1 < 0 || k0 > 2 * NACC - 1) {
      a = NACC;
      b = -1;
    } else {
      a = max(0, k0) >> 1;
      b = min(2 * NACC - 1, k1) >> 1;
    }
  }
  plo = __reduce_min_sync(0xffffffffu, a);
  phi = __reduce_max_sync(0xffffffffu, b);
}

// Resident CTAs per SM the register allocation must allow: 3 (the default 64 KB staging
// budget fits 3 CTAs) unless NZ = 64 needs the registers of 2.
template <int NZ>
constexpr int fdk_min_blocks() { return NZ >= 64 ? 2 : 3; }

template <typename T, int NZ, bool PIW, bool X2, int MINB = fdk_min_blocks<NZ>()>
__global__ void __launch_bounds__(FDK_THREADS, MINB) fdk_tma_kernel(const __grid_constant__ CUtensorMap tmap,
                                                              const __grid_constant__ FdkParams P)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int ES = (int)sizeof(T);
  // voxel pairs (X2) read FP32 taps; 16-bit storage runs fdk_pair_kernel, or this kernel's
  // one-tap-at-a-time path (X2 = false) for comparison
  static_assert(!X2 || ES == 4, "16-bit voxel pairs run in fdk_pair_kernel");
  constexpr int ESC = ES;  // bytes per position of the box the taps are read from
  const int stage_elems = P.BW * P.BH;
  const int stage_bytes = ((stage_elems * ES) + 127) & ~127;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + (size_t)P.stages * stage_bytes);
  uint64_t* empty = full + P.stages;
  // per stage: box origin w, h (as float bits: the consumers use them as floats); view (-1:
  // end of the list); rows the tile's footprint needs
  int4* origin = reinterpret_cast<int4*>(empty + P.stages);
  // per stage: the staged view's parameters, copied by the producer so that the consumers read
  // them from shared memory (the views of a launch overflow the constant cache while the
  // CTAs of an SM work on different views)
  FdkView* vstage = reinterpret_cast<FdkView*>(origin + P.stages);
  const uint32_t smem_base = dev::smem_u32(smem_raw);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int tx, ty, tz;
  fdk_tile(P, P.tile0 + blockIdx.x, tx, ty, tz);

  if (threadIdx.x == 0) {
    for (int s = 0; s < P.stages; s++) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], FDK_CWARPS);
    }
    dev::fence_mbar_init();
  }
  __syncthreads();

  if (warp == FDK_CWARPS) {
    // ------------------------------------------------------------- producer warp
    const uint32_t bytes = (uint32_t)(stage_elems * ES);
    int issued = 0;  // staged views so far
    int ps = 0;      // its ring slot (issued mod stages), kept by increments: no division
    uint32_t pround = 0;  // parity of issued / stages
    bool failed = false, stalled = false;
    if constexpr (PIW) {
      // the whole warp tests 32 views at a time against the PI window (most views miss a
      // tile of a helical scan); lane 0 stages the ones that reach it, in view order
      if (lane == 0) dev::tma_prefetch(&tmap);
      for (int vb = 0; vb < P.nviews && !failed && !stalled; vb += 32) {
        const int v = vb + lane;
        int w0 = 0, h0 = 0, nw = 0, nh = 0;
        bool need = false;
        if (v < P.nviews) {
          float fp[4];
          fdk_box_origin(P, P.v[v], tx, ty, tz, NZ, w0, h0, nw, nh, fp);
          need = !fdk_tile_outside_window(P, P.v[v], fp[0], fp[1], fp[2], fp[3]);
        }
        unsigned mask = __ballot_sync(0xffffffffu, need);
        while (mask) {
          if (issued == P.stop_after) {  // test hook (uniform over the warp)
            stalled = true;
            break;
          }
          const int l = __ffs(mask) - 1;
          mask &= mask - 1;
          const int sw0 = __shfl_sync(0xffffffffu, w0, l), sh0 = __shfl_sync(0xffffffffu, h0, l);
          const int snw = __shfl_sync(0xffffffffu, nw, l), snh = __shfl_sync(0xffffffffu, nh, l);
          int ok = 1;
          if (lane == 0) {
            const int s = ps;
            if (issued >= P.stages && !dev::mbar_wait(&empty[s], pround ^ 1u)) {
              ok = 0;
            } else {
              if (snw > P.BW || snh > P.BH) dev::record_status(P.status, DEV_RANGE);
              origin[s] = make_int4(__float_as_int((float)sw0), __float_as_int((float)sh0), vb + l, snh);
              vstage[s] = P.v[vb + l];
              dev::mbar_arrive_expect_tx(&full[s], bytes);
              dev::tma_load_3d(smem_raw + (size_t)s * stage_bytes, &tmap, &full[s], sw0, sh0,
                               P.view0 + vb + l);
            }
          }
          if (!__shfl_sync(0xffffffffu, ok, 0)) {
            failed = true;
            break;
          }
          issued++;
          if (++ps == P.stages) { ps = 0; pround ^= 1u; }
        }
      }
      if (lane != 0) return;
    } else {
      if (lane != 0) return;
      dev::tma_prefetch(&tmap);
      for (int v = 0; v < P.nviews; v++) {
        if (v == P.stop_after) {  // test hook
          stalled = true;
          break;
        }
        int w0, h0, nw, nh;
        fdk_box_origin(P, P.v[v], tx, ty, tz, NZ, w0, h0, nw, nh);
        const int s = ps;
        if (issued >= P.stages) {
          if (!dev::mbar_wait(&empty[s], pround ^ 1u)) {
            failed = true;
            break;
          }
        }
        if (nw > P.BW || nh > P.BH) dev::record_status(P.status, DEV_RANGE);
        origin[s] = make_int4(__float_as_int((float)w0), __float_as_int((float)h0), v, nh);
        vstage[s] = P.v[v];
        dev::mbar_arrive_expect_tx(&full[s], bytes);
        dev::tma_load_3d(smem_raw + (size_t)s * stage_bytes, &tmap, &full[s], w0, h0, P.view0 + v);
        issued++;
        if (++ps == P.stages) { ps = 0; pround ^= 1u; }
      }
    }
    if (PIW && !failed && !stalled) {
      // end of the view list: a slot whose phase completes without data, view -1
      const int s = ps;
      if (issued < P.stages || dev::mbar_wait(&empty[s], pround ^ 1u)) {
        origin[s] = make_int4(0, 0, -1, 0);
        dev::mbar_arrive(&full[s]);
      } else {
        failed = true;
      }
    }
    if (failed || stalled) {
      if (failed) dev::record_status(P.status, DEV_TIMEOUT);
      // drain: wait (bounded) for the copies still in flight before leaving
      for (int j = max(0, issued - P.stages); j < issued; j++)
        dev::mbar_wait(&full[j % P.stages], (j / P.stages) & 1, 100000000ull);
    }
    return;
  }

  // --------------------------------------------------------------- consumer warps
  const int xl = tx * FDK_TX + (warp & 1) * 8 + (lane & 7);
  const int yl = ty * FDK_TY + (warp >> 1) * 4 + (lane >> 3);
  const int zl = tz * NZ;
  const float x = P.ox + (float)xl, y = P.oy + (float)yl, zf = P.oz + (float)zl;
  const float MAGIC = 12582912.0f;  // 1.5 * 2^23: adding it in round-down mode floors
  const uint32_t MAGIC_BITS = 0x4B400000u;
  const uint32_t rowb = (uint32_t)(P.BW * ESC);  // bytes per row of the box read below

  constexpr int NACC = X2 ? NZ / 2 : NZ;
  static_assert(!X2 || (NZ % 2 == 0), "pairs");
  u64 acc2[X2 ? NACC : 1];
  float acc[X2 ? 1 : NACC];
#pragma unroll
  for (int k = 0; k < NACC; k++) {
    if constexpr (X2) acc2[k] = 0ull;
    else acc[k] = 0.0f;
  }

  // ring position j carries view j (all views staged) or the view the producer chose (PI
  // window: only views that reach the tile, then an end marker); its slot s = j mod stages
  // and the phase parity are kept by increments (no integer division per view)
  int s = 0;
  uint32_t ph = 0;
  for (int j = 0; PIW || j < P.nviews; j++) {
    if (!dev::mbar_wait(&full[s], ph, P.cwait_ns)) {
      dev::record_status(P.status, DEV_TIMEOUT);
      return;
    }
    const int4 org = origin[s];
    const int v = PIW ? org.z : j;
    if (PIW && v < 0) break;
    const FdkView V = vstage[s];

    const float den = fmaf(V.c0, x, fmaf(V.c1, y, 1.0f));
    // the approximate reciprocal (within 2 ulp): the staging box keeps a pixel of margin
    const float U = __fdividef(1.0f, den);
    const float wabs = fmaf(fmaf(V.a0, x, V.a1 * y), U, V.wc);
    float wl = wabs - __int_as_float(org.x);
    float h0 = fmaf(U, fmaf(P.hb, zf, V.e), V.hc) - __int_as_float(org.y);
    float dh = U * P.hb;
    float wt = V.wt;
    if (P.wexp >= 1) wt *= U;
    if (P.wexp >= 2) wt *= U;

    // memory safety: every tap must stay inside the staged box
    int iw = __float2int_rd(wl);
    const float hl = fmaf((float)(NZ - 1), dh, h0);
    // (0.01 px of slack covers the rounding of the incremental row stepping below)
    if (iw < 0 || iw > P.BW - 2 || !(h0 >= 0.0f) || !(hl + 0.01f < (float)(P.BH - 1))) {
      dev::record_status(P.status, DEV_RANGE);
      iw = 0; wl = 0.0f; h0 = 0.0f; dh = 0.0f; wt = 0.0f;
    }
    const float fw = wl - (float)iw;

    float lo = -3.0e38f, hi = 3.0e38f;  // Tam-Danielsson bounds (local h)
    if constexpr (PIW) {
      const float u = (wabs - V.wc) * P.td_usc;
      const float q = P.td_a * (1.0f + u * u);
      const float at = atanf(u);
      const float hsrc = V.hc - __int_as_float(org.y);
      hi = hsrc + q * (1.5707963267948966f - at);
      lo = hsrc - q * (1.5707963267948966f + at);
    }

    // byte address of tap (row r, column iw) = bits(MAGIC + r) * rowb + base
    const uint32_t base = smem_base + (uint32_t)s * (uint32_t)stage_bytes + (uint32_t)iw * ESC -
                          MAGIC_BITS * rowb;
    if constexpr (X2) {
      const u64 MAG2 = pk2(MAGIC, MAGIC);
      const u64 FW2 = pk2(fw, fw);
      const u64 WT2 = pk2(wt, wt);
      const u64 D2 = pk2(2.0f * dh, 2.0f * dh);
      // PI-window path, one voxel pair: taps from the staged box, the view's weight for the
      // voxels inside the window, accumulated into pair k; H holds the pair's two row
      // positions and steps to the next pair's.  (The path without the window keeps the
      // plain unrolled loop below: written through this lambda it ran 6 % slower.)
      auto pair = [&](auto kc, u64& H) {
        constexpr int k = decltype(kc)::value;
        const u64 T2 = add2_rm(H, MAG2);
        const u64 FH = sub2(H, sub2(T2, MAG2));
        float t0, t1;
        up2(T2, t0, t1);
        const uint32_t a0 = (uint32_t)__float_as_uint(t0) * rowb + base;
        const uint32_t a1 = (uint32_t)__float_as_uint(t1) * rowb + base;
        const uint32_t c0 = a0 + rowb, c1 = a1 + rowb;
        const u64 A = lds_f32x2<0>(a0, a1);
        const u64 B = lds_f32x2<4>(a0, a1);
        const u64 C = lds_f32x2<0>(c0, c1);
        const u64 Dd = lds_f32x2<4>(c0, c1);
        const u64 R0 = fma2(FW2, sub2(B, A), A);
        const u64 R1 = fma2(FW2, sub2(Dd, C), C);
        const u64 VAL = fma2(FH, sub2(R1, R0), R0);
        u64 W = WT2;
        if constexpr (PIW) {
          float h0k, h1k;
          up2(H, h0k, h1k);
          W = pk2((h0k >= lo && h0k <= hi) ? wt : 0.0f, (h1k >= lo && h1k <= hi) ? wt : 0.0f);
        }
        acc2[k] = fma2(W, VAL, acc2[k]);
        H = add2(H, D2);
      };
      if constexpr (PIW) {
        // only the pairs plo..phi that can lie inside some lane's window, entered through a
        // jump table: the pairs outside cost no test (57.4 against 60.6 ms per helical pass
        // with a warp-uniform test of every pair)
        int plo = 0, phi = NACC - 1;
        piw_pairs<NACC>(lo, hi, h0, dh, plo, phi);
        u64 H = fma2(pk2((float)plo, (float)plo), D2, pk2(h0, h0 + dh));
        run_pairs<NACC>(plo, phi, [&](auto kc) { pair(kc, H); });
      } else {
        u64 H = pk2(h0, h0 + dh);
#pragma unroll
        for (int k = 0; k < NACC; k++) {
          const u64 T2 = add2_rm(H, MAG2);
          const u64 FH = sub2(H, sub2(T2, MAG2));
          float t0, t1;
          up2(T2, t0, t1);
          const uint32_t a0 = (uint32_t)__float_as_uint(t0) * rowb + base;
          const uint32_t a1 = (uint32_t)__float_as_uint(t1) * rowb + base;
          const uint32_t c0 = a0 + rowb, c1 = a1 + rowb;
          const u64 A = lds_f32x2<0>(a0, a1);
          const u64 B = lds_f32x2<4>(a0, a1);
          const u64 C = lds_f32x2<0>(c0, c1);
          const u64 Dd = lds_f32x2<4>(c0, c1);
          const u64 R0 = fma2(FW2, sub2(B, A), A);
          const u64 R1 = fma2(FW2, sub2(Dd, C), C);
          const u64 VAL = fma2(FH, sub2(R1, R0), R0);
          acc2[k] = fma2(WT2, VAL, acc2[k]);
          H = add2(H, D2);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < NZ; k++) {
        const float hk = fmaf((float)k, dh, h0);
        const float t = __fadd_rd(hk, MAGIC);
        const uint32_t a = (uint32_t)__float_as_uint(t) * rowb + base;
        const uint32_t c = a + rowb;
        const float fh = hk - (t - MAGIC);
        const float ta = Tap<T, 0>::ld(a), tb = Tap<T, 1>::ld(a);
        const float tc = Tap<T, 0>::ld(c), td = Tap<T, 1>::ld(c);
        const float r0 = fmaf(fw, tb - ta, ta);
        const float r1 = fmaf(fw, td - tc, tc);
        const float val = fmaf(fh, r1 - r0, r0);
        float wk = wt;
        if constexpr (PIW) wk = (hk >= lo && hk <= hi) ? wt : 0.0f;
        acc[k] = fmaf(wk, val, acc[k]);
      }
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty[s]);
    if (++s == P.stages) { s = 0; ph ^= 1u; }
  }

  if (xl < P.nx && yl < P.ny) {
    float* out = P.vol + (size_t)yl * P.nx + xl;
    const size_t plane = (size_t)P.nx * P.ny;
#pragma unroll
    for (int k = 0; k < NACC; k++) {
      float v0, v1;
      int k0;
      if constexpr (X2) {
        up2(acc2[k], v0, v1);
        k0 = 2 * k;
        if (zl + k0 < P.nz) out[(size_t)(zl + k0) * plane] += v0;
        if (zl + k0 + 1 < P.nz) out[(size_t)(zl + k0 + 1) * plane] += v1;
      } else {
        (void)v1;
        v0 = acc[k];
        k0 = k;
        if (zl + k0 < P.nz) out[(size_t)(zl + k0) * plane] += v0;
      }
    }
  }
}

// =====================================================================================
// 16-bit storage: tap pairs prepared by the producer warp
// =====================================================================================
// The FP32 kernel reads four 32-bit taps per update from the staged box.  With 16-bit
// storage a row's two horizontal taps fit one 32-bit word, but the staged box holds them as
// (c, c+1) words only for even c.  Here the producer warp, besides issuing the TMA loads,
// rewrites every landed box into a tap-pair buffer (word (r, c) = taps (r, c) in its low and
// (r, c + 1) in its high half) and hands it to the consumers through an mbarrier ring, so a
// consumer reads two words per update and no block-wide barrier separates the views:
//   TMA stage ring (S boxes of 16-bit taps)  --full[s]-->  producer rewrite
//   pair ring (NP buffers)  --full2[p] (32 producer lanes)-->  consumers
//   consumers  --empty2[p] (one arrive per consumer warp)-->  producer
// The producer itself frees a TMA stage once it has rewritten it.  The views it selects
// (all, or with the PI window those that reach the tile) end with a marker buffer (view -1).
template <typename T, int NZ, bool PIW>
__global__ void __launch_bounds__(FDK_THREADS, 3) fdk_pair_kernel(const __grid_constant__ CUtensorMap tmap,
                                                                  const __grid_constant__ FdkParams P)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  static_assert(sizeof(T) == 2, "16-bit storage");
  const int S = P.stages, NP = P.pbufs;
  const int stage_elems = P.BW * P.BH;
  const int stage_bytes = ((stage_elems * 2) + 127) & ~127;
  const int pbuf_bytes = ((stage_elems * 4) + 127) & ~127;
  unsigned char* pairs = smem_raw + (size_t)S * stage_bytes;
  // box origins (w, h as float bits, view, rows needed): per pair buffer and per TMA stage
  int4* origin2 = reinterpret_cast<int4*>(pairs + (size_t)NP * pbuf_bytes);
  int4* sorg = origin2 + NP;
  FdkView* vpair = reinterpret_cast<FdkView*>(sorg + S);  // per pair buffer: its view's parameters
  uint64_t* full = reinterpret_cast<uint64_t*>(vpair + NP);
  uint64_t* full2 = full + S;
  uint64_t* empty2 = full2 + NP;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int tx, ty, tz;
  fdk_tile(P, P.tile0 + blockIdx.x, tx, ty, tz);

  if (threadIdx.x == 0) {
    for (int k = 0; k < S; k++) dev::mbar_init(&full[k], 1);
    for (int k = 0; k < NP; k++) {
      dev::mbar_init(&full2[k], 32);
      dev::mbar_init(&empty2[k], FDK_CWARPS);
    }
    dev::fence_mbar_init();
  }
  __syncthreads();

  if (warp == FDK_CWARPS) {
    // ------------------------------------------------------------- producer warp
    if (lane == 0) dev::tma_prefetch(&tmap);
    const uint32_t bytes = (uint32_t)(stage_elems * 2);
    // views in order, 32 tested at a time (PI window: those that reach the tile)
    int vb = -32;
    unsigned msk = 0;
    int lw0 = 0, lh0 = 0, lnw = 0, lnh = 0;
    bool exhausted = false, stalled = false, failed = false;
    int issued = 0, conv = 0;
    int is = 0;  // issued mod S, kept by increments (no division per view)
    auto issue_next = [&]() {
      if (exhausted) return;
      if (issued == P.stop_after) {  // test hook
        stalled = exhausted = true;
        return;
      }
      while (msk == 0) {
        vb += 32;
        if (vb >= P.nviews) {
          exhausted = true;
          return;
        }
        const int v = vb + lane;
        bool need = false;
        if (v < P.nviews) {
          float fp[4];
          fdk_box_origin(P, P.v[v], tx, ty, tz, NZ, lw0, lh0, lnw, lnh, fp);
          need = PIW ? !fdk_tile_outside_window(P, P.v[v], fp[0], fp[1], fp[2], fp[3]) : true;
        }
        msk = __ballot_sync(0xffffffffu, need);
      }
      const int l = __ffs(msk) - 1;
      msk &= msk - 1;
      const int w0 = __shfl_sync(0xffffffffu, lw0, l), h0 = __shfl_sync(0xffffffffu, lh0, l);
      const int nw = __shfl_sync(0xffffffffu, lnw, l), nh = __shfl_sync(0xffffffffu, lnh, l);
      const int s = is;  // free: its previous view has been rewritten
      if (lane == 0) {
        if (nw > P.BW || nh > P.BH) dev::record_status(P.status, DEV_RANGE);
        sorg[s] = make_int4(__float_as_int((float)w0), __float_as_int((float)h0), vb + l, nh);
        dev::mbar_arrive_expect_tx(&full[s], bytes);
        dev::tma_load_3d(smem_raw + (size_t)s * stage_bytes, &tmap, &full[s], w0, h0, P.view0 + vb + l);
      }
      __syncwarp();
      issued++;
      if (++is == S) is = 0;
    };
    for (int k = 0; k < S; k++) issue_next();
    const int cpr = P.BW / 8;  // 16-byte chunks per row (BW is a multiple of 8)
    const int nbox = P.BH * cpr;
    // conv mod S / mod NP and the parities of conv / S and conv / NP
    int cs = 0, cp = 0;
    uint32_t cph = 0, cpph = 0;
    while (conv < issued) {
      const int s = cs, p = cp;
      bool ok = dev::mbar_wait(&full[s], cph);
      if (ok && conv >= NP) ok = dev::mbar_wait(&empty2[p], cpph ^ 1u);
      if (!__all_sync(0xffffffffu, ok)) {
        failed = true;
        break;
      }
      const int4 o = sorg[s];
      // rewrite the rows the tile's footprint reaches (taps stay below row o.w - 1); the word
      // of a row's last column takes the next row's first tap, which no tap reads (columns
      // stay below BW - 1)
      const uint4* src = reinterpret_cast<const uint4*>(smem_raw + (size_t)s * stage_bytes);
      uint4* dst = reinterpret_cast<uint4*>(pairs + (size_t)p * pbuf_bytes);
      const int nconv = min(o.w, P.BH) * cpr;
      for (int e = lane; e < nconv; e += 32) {
        const uint32_t nx = e + 1 < nbox ? reinterpret_cast<const uint32_t*>(src + e + 1)[0] : 0u;
        uint4 lo, hi;
        pair8(src[e], nx, lo, hi);
        dst[2 * e] = lo;
        dst[2 * e + 1] = hi;
      }
      if (lane == 0) {
        origin2[p] = o;
        vpair[p] = P.v[o.z];
      }
      __syncwarp();
      dev::mbar_arrive(&full2[p]);  // all 32 lanes: their writes are released to the consumers
      conv++;
      if (++cs == S) { cs = 0; cph ^= 1u; }
      if (++cp == NP) { cp = 0; cpph ^= 1u; }
      issue_next();  // stage s is free again
    }
    if (failed) {
      if (lane == 0) {
        dev::record_status(P.status, DEV_TIMEOUT);
        // drain: wait (bounded) for the copies still in flight before leaving
        for (int j = conv; j < issued; j++) dev::mbar_wait(&full[j % S], (j / S) & 1, 100000000ull);
      }
      return;
    }
    if (stalled) return;  // every issued copy has landed and been handed over
    // end of the view list: a pair buffer whose phase completes without data, view -1
    const int p = cp;
    const bool ok = conv < NP || dev::mbar_wait(&empty2[p], cpph ^ 1u);
    if (__all_sync(0xffffffffu, ok)) {
      if (lane == 0) origin2[p] = make_int4(0, 0, -1, 0);
      __syncwarp();
      dev::mbar_arrive(&full2[p]);
    } else if (lane == 0) {
      dev::record_status(P.status, DEV_TIMEOUT);
    }
    return;
  }

  // --------------------------------------------------------------- consumer warps
  const int xl = tx * FDK_TX + (warp & 1) * 8 + (lane & 7);
  const int yl = ty * FDK_TY + (warp >> 1) * 4 + (lane >> 3);
  const int zl = tz * NZ;
  const float x = P.ox + (float)xl, y = P.oy + (float)yl, zf = P.oz + (float)zl;
  const float MAGIC = 12582912.0f;  // 1.5 * 2^23: adding it in round-down mode floors
  const uint32_t MAGIC_BITS = 0x4B400000u;
  const uint32_t rowb = (uint32_t)(P.BW * 4);  // bytes per row of a pair buffer
  const uint32_t pair0 = dev::smem_u32(pairs);
  constexpr int NACC = NZ / 2;
  u64 acc2[NACC];
#pragma unroll
  for (int k = 0; k < NACC; k++) acc2[k] = 0ull;

  // pair buffer of the next view (the views cycle through the NP buffers) and the parity of
  // its phase, kept by increments (no integer division per view)
  int p = 0;
  uint32_t ph = 0;
  for (;;) {
    if (!dev::mbar_wait(&full2[p], ph, P.cwait_ns)) {
      dev::record_status(P.status, DEV_TIMEOUT);
      return;
    }
    const int4 org = origin2[p];
    const int v = org.z;
    if (v < 0) break;
    const FdkView V = vpair[p];
    const float den = fmaf(V.c0, x, fmaf(V.c1, y, 1.0f));
    // the approximate reciprocal (within 2 ulp): the staging box keeps a pixel of margin
    const float U = __fdividef(1.0f, den);
    const float wabs = fmaf(fmaf(V.a0, x, V.a1 * y), U, V.wc);
    float wl = wabs - __int_as_float(org.x);
    float h0 = fmaf(U, fmaf(P.hb, zf, V.e), V.hc) - __int_as_float(org.y);
    float dh = U * P.hb;
    float wt = V.wt;
    if (P.wexp >= 1) wt *= U;
    if (P.wexp >= 2) wt *= U;
    // memory safety: every tap must stay inside the staged box
    int iw = __float2int_rd(wl);
    const float hl = fmaf((float)(NZ - 1), dh, h0);
    if (iw < 0 || iw > P.BW - 2 || !(h0 >= 0.0f) || !(hl + 0.01f < (float)(P.BH - 1))) {
      dev::record_status(P.status, DEV_RANGE);
      iw = 0; wl = 0.0f; h0 = 0.0f; dh = 0.0f; wt = 0.0f;
    }
    const float fw = wl - (float)iw;
    float lo = -3.0e38f, hi = 3.0e38f;  // Tam-Danielsson bounds (local h)
    if constexpr (PIW) {
      const float u = (wabs - V.wc) * P.td_usc;
      const float q = P.td_a * (1.0f + u * u);
      const float at = atanf(u);
      const float hsrc = V.hc - __int_as_float(org.y);
      hi = hsrc + q * (1.5707963267948966f - at);
      lo = hsrc - q * (1.5707963267948966f + at);
    }
    // byte address of tap pair (row r, column iw) = bits(MAGIC + r) * rowb + base
    const uint32_t base = pair0 + (uint32_t)p * (uint32_t)pbuf_bytes + (uint32_t)iw * 4u - MAGIC_BITS * rowb;
    const u64 MAG2 = pk2(MAGIC, MAGIC);
    const u64 FW2 = pk2(fw, fw);
    const u64 WT2 = pk2(wt, wt);
    const u64 D2 = pk2(2.0f * dh, 2.0f * dh);
    // PI-window path, one voxel pair, as in fdk_tma_kernel, from the tap-pair words
    auto pair = [&](auto kc, u64& H) {
      constexpr int k = decltype(kc)::value;
      const u64 T2 = add2_rm(H, MAG2);
      const u64 FH = sub2(H, sub2(T2, MAG2));
      float t0, t1;
      up2(T2, t0, t1);
      const uint32_t a0 = (uint32_t)__float_as_uint(t0) * rowb + base;
      const uint32_t a1 = (uint32_t)__float_as_uint(t1) * rowb + base;
      u64 A, B, C, Dd;
      lds_pair_taps<T>(a0, a1, A, B);
      lds_pair_taps<T>(a0 + rowb, a1 + rowb, C, Dd);
      const u64 R0 = fma2(FW2, sub2(B, A), A);
      const u64 R1 = fma2(FW2, sub2(Dd, C), C);
      const u64 VAL = fma2(FH, sub2(R1, R0), R0);
      u64 W = WT2;
      if constexpr (PIW) {
        float h0k, h1k;
        up2(H, h0k, h1k);
        W = pk2((h0k >= lo && h0k <= hi) ? wt : 0.0f, (h1k >= lo && h1k <= hi) ? wt : 0.0f);
      }
      acc2[k] = fma2(W, VAL, acc2[k]);
      H = add2(H, D2);
    };
    if constexpr (PIW) {
      // the pairs plo..phi only (see fdk_tma_kernel)
      int plo = 0, phi = NACC - 1;
      piw_pairs<NACC>(lo, hi, h0, dh, plo, phi);
      u64 H = fma2(pk2((float)plo, (float)plo), D2, pk2(h0, h0 + dh));
      run_pairs<NACC>(plo, phi, [&](auto kc) { pair(kc, H); });
    } else {
      u64 H = pk2(h0, h0 + dh);
#pragma unroll
      for (int k = 0; k < NACC; k++) {
        const u64 T2 = add2_rm(H, MAG2);
        const u64 FH = sub2(H, sub2(T2, MAG2));
        float t0, t1;
        up2(T2, t0, t1);
        const uint32_t a0 = (uint32_t)__float_as_uint(t0) * rowb + base;
        const uint32_t a1 = (uint32_t)__float_as_uint(t1) * rowb + base;
        u64 A, B, C, Dd;
        lds_pair_taps<T>(a0, a1, A, B);
        lds_pair_taps<T>(a0 + rowb, a1 + rowb, C, Dd);
        const u64 R0 = fma2(FW2, sub2(B, A), A);
        const u64 R1 = fma2(FW2, sub2(Dd, C), C);
        const u64 VAL = fma2(FH, sub2(R1, R0), R0);
        acc2[k] = fma2(WT2, VAL, acc2[k]);
        H = add2(H, D2);
      }
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty2[p]);
    if (++p == NP) { p = 0; ph ^= 1u; }
  }

  if (xl < P.nx && yl < P.ny) {
    float* out = P.vol + (size_t)yl * P.nx + xl;
    const size_t plane = (size_t)P.nx * P.ny;
#pragma unroll
    for (int k = 0; k < NACC; k++) {
      float v0, v1;
      up2(acc2[k], v0, v1);
      if (zl + 2 * k < P.nz) out[(size_t)(zl + 2 * k) * plane] += v0;
      if (zl + 2 * k + 1 < P.nz) out[(size_t)(zl + 2 * k + 1) * plane] += v1;
    }
  }
}

}  // namespace fcb

namespace fcb {
// =====================================================================================
// Generic projective-matrix kernel
// =====================================================================================
constexpr int GEN_MAXV = 480;
struct GenView {
  float m[12];
  float kappa;
  float wt;
  float wc, hc;  // local window column of the detector centre, row of the source (PI window)
};
struct GenParams {
  float* vol;
  const void* proj;
  int ptype;
  int nx, ny, nz;
  float ox, oy, oz;
  int WH0, WH1;
  int nviews, view0;
  int wexp;
  int piwin;    // Tam-Danielsson window (aligned helical geometry), as fdk_tma_kernel
  float td_a;   // window half-height scale P / (2 pi pw), pixels
  float td_r;   // source-axis distance in pixels (D / pw)
  float td_sign; // +1/-1: sense of the helix relative to the w axis
  // reference-compatible windows (NULL: ideal operator).  win[tile * wviews + view] holds
  // the first/last texel column and row of the sub-problem window, data-local; tiles are
  // sv0 x sv1 x sv2 voxels from volStart, ntx x nty of them per z layer.
  const int4* win;
  int sv0, sv1, sv2, ntx, nty, wviews;
  long long vox0, nvox;  // voxel range of this launch (launches may cover z-ranges)
  GenView v[GEN_MAXV];
};
static_assert(sizeof(GenParams) < 32000, "kernel parameter space");

__device__ __forceinline__ float gen_load(const void* base, int ptype, size_t i)
{
  if (ptype == FCB_F32) return __ldg(reinterpret_cast<const float*>(base) + i);
  const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(base) + i);
  if (ptype == FCB_F16) return __half2float(__ushort_as_half(u));
  return __uint_as_float(((uint32_t)u) << 16);
}

// One thread per (x, y) column and GEN_NZ consecutive z-voxels of the launch's z-range: the
// view's matrix rows are read once per column and the x, y parts of the three projective
// coordinates are shared, so a voxel-view costs one FMA per coordinate.
constexpr int GEN_NZ = 8;
__global__ void __launch_bounds__(256) bp_generic_kernel(const __grid_constant__ GenParams P)
{
  const long long plane = (long long)P.nx * P.ny;
  const int zfirst = (int)(P.vox0 / plane), zend = (int)((P.vox0 + P.nvox) / plane);
  const int ngz = (zend - zfirst + GEN_NZ - 1) / GEN_NZ;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= plane * ngz) return;
  const int xi = (int)(t % P.nx);
  const long long r = t / P.nx;
  const int yi = (int)(r % P.ny), zg = (int)(r / P.ny);
  const int zi0 = zfirst + zg * GEN_NZ;
  const int nzv = min(GEN_NZ, zend - zi0);
  const float x = P.ox + xi, y = P.oy + yi;
  float acc[GEN_NZ];
#pragma unroll
  for (int k = 0; k < GEN_NZ; k++) acc[k] = 0.0f;
  for (int v = 0; v < P.nviews; v++) {
    const GenView& V = P.v[v];
    const float bu = fmaf(V.m[0], x, fmaf(V.m[1], y, V.m[3]));
    const float bv = fmaf(V.m[4], x, fmaf(V.m[5], y, V.m[7]));
    const float bs = fmaf(V.m[8], x, fmaf(V.m[9], y, V.m[11]));
    const float mu = V.m[2], mv = V.m[6], ms = V.m[10];
    const size_t vb = (size_t)(P.view0 + v) * P.WH0 * P.WH1;
#pragma unroll
    for (int k = 0; k < GEN_NZ; k++) {
      if (k >= nzv) break;
      const int zi = zi0 + k;
      const float z = P.oz + zi;
      const float uu = fmaf(mu, z, bu), vv = fmaf(mv, z, bv), ss = fmaf(ms, z, bs);
      const float rs = 1.0f / ss;
      const float wl = uu * rs, hl = vv * rs;
      float wt = V.wt;
      if (P.wexp >= 1) wt *= V.kappa * rs;
      if (P.wexp >= 2) wt *= V.kappa * rs;
      if (P.win) {
        // the reference's texture window: texel indices clamp to the window edge, texels
        // outside the caller's data read zero (coneBeamGPU.cu:839-848, :1049-1088)
        const int tile = ((zi / P.sv2) * P.nty + yi / P.sv1) * P.ntx + xi / P.sv0;
        const int4 wb = P.win[(size_t)tile * P.wviews + P.view0 + v];
        const float wc = fminf(fmaxf(wl, (float)wb.x - 2.0f), (float)wb.y + 2.0f);
        const float hc = fminf(fmaxf(hl, (float)wb.z - 2.0f), (float)wb.w + 2.0f);
        const float fw = floorf(wc), fh = floorf(hc);
        const float a = wc - fw, b = hc - fh;
        const int i0 = min(max((int)fw, wb.x), wb.y), i1 = min(max((int)fw + 1, wb.x), wb.y);
        const int j0 = min(max((int)fh, wb.z), wb.w), j1 = min(max((int)fh + 1, wb.z), wb.w);
        const bool ci0 = i0 >= 0 && i0 < P.WH0, ci1 = i1 >= 0 && i1 < P.WH0;
        const bool cj0 = j0 >= 0 && j0 < P.WH1, cj1 = j1 >= 0 && j1 < P.WH1;
        const float t00 = ci0 && cj0 ? gen_load(P.proj, P.ptype, vb + (size_t)j0 * P.WH0 + i0) : 0.f;
        const float t10 = ci1 && cj0 ? gen_load(P.proj, P.ptype, vb + (size_t)j0 * P.WH0 + i1) : 0.f;
        const float t01 = ci0 && cj1 ? gen_load(P.proj, P.ptype, vb + (size_t)j1 * P.WH0 + i0) : 0.f;
        const float t11 = ci1 && cj1 ? gen_load(P.proj, P.ptype, vb + (size_t)j1 * P.WH0 + i1) : 0.f;
        const float r0 = fmaf(a, t10 - t00, t00), r1 = fmaf(a, t11 - t01, t01);
        acc[k] = fmaf(wt, fmaf(b, r1 - r0, r0), acc[k]);
        continue;
      }
      if (!(wl > -1.0f && wl < (float)P.WH0 && hl > -1.0f && hl < (float)P.WH1)) continue;
      if (P.piwin) {
        // the voxel sees the view only inside its PI interval (the staged kernel's test)
        const float u = (wl - V.wc) * P.td_sign / P.td_r;
        const float q = P.td_a * (1.0f + u * u);
        const float at = atanf(u);
        if (hl > V.hc + q * (1.5707963267948966f - at) || hl < V.hc - q * (1.5707963267948966f + at)) continue;
      }
      const float fw0 = floorf(wl), fh0 = floorf(hl);
      const int iw = (int)fw0, ih = (int)fh0;
      const float a = wl - fw0, b = hl - fh0;
      float t00 = 0.f, t10 = 0.f, t01 = 0.f, t11 = 0.f;
      if (ih >= 0) {
        if (iw >= 0) t00 = gen_load(P.proj, P.ptype, vb + (size_t)ih * P.WH0 + iw);
        if (iw + 1 < P.WH0) t10 = gen_load(P.proj, P.ptype, vb + (size_t)ih * P.WH0 + iw + 1);
      }
      if (ih + 1 < P.WH1) {
        if (iw >= 0) t01 = gen_load(P.proj, P.ptype, vb + (size_t)(ih + 1) * P.WH0 + iw);
        if (iw + 1 < P.WH0) t11 = gen_load(P.proj, P.ptype, vb + (size_t)(ih + 1) * P.WH0 + iw + 1);
      }
      const float r0 = fmaf(a, t10 - t00, t00), r1 = fmaf(a, t11 - t01, t01);
      acc[k] = fmaf(wt, fmaf(b, r1 - r0, r0), acc[k]);
    }
  }
  const size_t o = ((size_t)zi0 * P.ny + yi) * P.nx + xi;
#pragma unroll
  for (int k = 0; k < GEN_NZ; k++)
    if (k < nzv) P.vol[o + (size_t)k * plane] += acc[k];
}

}  // namespace fcb

namespace fcb {
// =====================================================================================
// PI-window pair count (FP64)
// =====================================================================================
// The voxel-view pairs of a helical Katsevich backprojection that lie inside each voxel's
// PI interval: the work the PI-window kernel does, counted exactly rather than sampled.
// The window is the Tam-Danielsson one (Noo, Pack & Heuscher 2003, flat detector through the
// axis): with U = D / (D + x cos a + y sin a), w = (y cos a - x sin a) U, u = sign * w / D and
// q = pitch / 2pi * (1 + u^2), voxel z is inside for view a when
//   -q (pi/2 + atan u) <= (z - hmp) U <= q (pi/2 - atan u).
// (z - hmp) U grows with z, so a column's inside voxels are one run of z, counted in closed
// form per (column, view).
struct PiView {
  double ca, sa, hmp;
};

__global__ void pi_pairs_kernel(const PiView* __restrict__ views, int nviews, int nx, int ny,
                                double x0, double y0, long long zlo, long long zhi, double D,
                                double pitch, double sgn, unsigned long long* count)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)nx * ny * nviews;
  unsigned long long c = 0;
  if (i < total) {
    const int t = (int)(i % nviews);
    const long long col = i / nviews;
    const double x = x0 + (double)(col % nx), y = y0 + (double)(col / nx);
    const PiView v = views[t];
    const double U = D / (D + x * v.ca + y * v.sa);
    const double w = (y * v.ca - x * v.sa) * U;
    const double u = sgn * w / D;
    const double q = pitch / (2.0 * M_PI) * (1.0 + u * u);
    const double at = atan(u);
    const double zmin = v.hmp + (-q * (0.5 * M_PI + at)) / U;
    const double zmax = v.hmp + (q * (0.5 * M_PI - at)) / U;
    // clamp before converting so that far-away runs stay defined
    const long long k0 = max(zlo, (long long)ceil(fmax(zmin, (double)zlo - 1.0)));
    const long long k1 = min(zhi - 1, (long long)floor(fmin(zmax, (double)zhi + 1.0)));
    if (k1 >= k0) c = (unsigned long long)(k1 - k0 + 1);
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}
}  // namespace fcb

// =====================================================================================
// Plans
// =====================================================================================
using namespace fcb;

struct fcb_bp_plan {
  Problem pb;
  int mode = 2;
  int ptype = FCB_F32;
  int path = 0;  // 0 generic, 1 tma
  int device = 0;
  int nz_tile = 32;
  int maxv = FDK_MAXV;
  int BW = 0, BH = 0, stages = 0, pbufs = 0, wshift = 2;
  long long updates = 0;
  std::vector<FdkParams> fdk;  // one per view chunk
  std::vector<GenParams> gen;
  std::vector<int> gen_parent;  // the view chunk (launch of `fdk`, or itself) each `gen` entry belongs to
  int4* d_win = nullptr;  // reference-compatible window table (device), when in use
  ~fcb_bp_plan()
  {
    if (d_win) cudaFree(d_win);
  }
};

namespace {

// Dynamic shared memory of one fdk_tma_kernel CTA: `stages` boxes of BW x BH elements of
// `es` bytes, a full and an empty barrier and a footprint record per stage.
size_t fdk_smem_bytes(int BW, int BH, int stages, size_t es)
{
  const size_t stage_bytes = ((size_t)BW * BH * es + 127) & ~(size_t)127;
  return stages * stage_bytes + stages * (2 * sizeof(uint64_t) + sizeof(int4) + sizeof(FdkView));
}

// Dynamic shared memory of one fdk_pair_kernel CTA: `stages` boxes of 16-bit taps, `pbufs`
// tap-pair buffers of BW x BH words, their footprint records and barriers.
size_t fdk_pair_smem_bytes(int BW, int BH, int stages, int pbufs)
{
  const size_t stage_bytes = ((size_t)BW * BH * 2 + 127) & ~(size_t)127;
  const size_t pbuf_bytes = ((size_t)BW * BH * 4 + 127) & ~(size_t)127;
  return stages * stage_bytes + pbufs * pbuf_bytes + (size_t)(stages + pbufs) * sizeof(int4) +
         (size_t)pbufs * sizeof(FdkView) + (size_t)(stages + 2 * pbufs) * sizeof(uint64_t);
}

// Launches chunk `chunk` (-1: all) over the z-tile layers [tz0, tz1) of the plan.
template <typename T, int NZ, bool PIW, bool X2, int MINB = fdk_min_blocks<NZ>()>
int launch_fdk(fcb_bp_plan* pl, const CUtensorMap& map, int chunk, int tz0, int tz1, cudaStream_t st)
{
  const size_t smem = fdk_smem_bytes(pl->BW, pl->BH, pl->stages, sizeof(T));
  auto kern = fdk_tma_kernel<T, NZ, PIW, X2, MINB>;
  FCB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int c = 0; c < (int)pl->fdk.size(); c++) {
    if (chunk >= 0 && c != chunk) continue;
    FdkParams& P = pl->fdk[c];
    const int layer = P.tiles_x * P.tiles_y;
    P.tile0 = tz0 * layer;
    const int ntiles = (tz1 - tz0) * layer;
    if (ntiles <= 0) continue;
    kern<<<ntiles, FDK_THREADS, smem, st>>>(map, P);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return FCB_OK;
}

// The same for 16-bit storage on fdk_pair_kernel.
template <typename T, bool PIW>
int launch_fdk_pair(fcb_bp_plan* pl, const CUtensorMap& map, int chunk, int tz0, int tz1, cudaStream_t st)
{
  const size_t smem = fdk_pair_smem_bytes(pl->BW, pl->BH, pl->stages, pl->pbufs);
  auto kern = fdk_pair_kernel<T, 32, PIW>;
  FCB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int c = 0; c < (int)pl->fdk.size(); c++) {
    if (chunk >= 0 && c != chunk) continue;
    FdkParams& P = pl->fdk[c];
    const int layer = P.tiles_x * P.tiles_y;
    P.tile0 = tz0 * layer;
    const int ntiles = (tz1 - tz0) * layer;
    if (ntiles <= 0) continue;
    kern<<<ntiles, FDK_THREADS, smem, st>>>(map, P);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return FCB_OK;
}

bool aligned_geometry(const Problem& pb) { return !pb.misaligned; }

// Fill FdkParams for views [v0, v0+n) (sizes/box filled by the caller).
void fill_fdk_views(const Problem& pb, int mode, int v0, int n, FdkParams* P)
{
  P->nviews = n;
  P->view0 = v0;
  for (int k = 0; k < n; k++) {
    const int t = v0 + k;
    const ViewGeom& g = pb.views[t];
    FdkView& V = P->v[k];
    V.c0 = (float)(g.ca / pb.D);
    V.c1 = (float)(g.sa / pb.D);
    V.a0 = (float)(-g.sa / pb.pw);
    V.a1 = (float)(g.ca / pb.pw);
    V.wc = (float)(pb.projDim[0] / 2 - pb.woff[t]);
    V.hc = (float)(pb.projDim[1] / 2 - pb.hoff[t]);
    V.e = (float)(-g.hmp / pb.pw);
    V.wt = (float)pb.norm[t];
  }
  (void)mode;
}

// Fill GenParams views [v0, v0+n): projective matrices, weights, window centre and source row.
void fill_gen_views(const Problem& pb, int v0, int n, GenParams* P)
{
  for (int k = 0; k < n; k++) {
    const int t = v0 + k;
    double M[12], kappa;
    view_matrix(pb, t, M, &kappa);
    for (int j = 0; j < 12; j++) P->v[k].m[j] = (float)M[j];
    P->v[k].kappa = (float)kappa;
    P->v[k].wt = (float)pb.norm[t];
    P->v[k].wc = (float)(pb.projDim[0] / 2 - pb.woff[t]);
    P->v[k].hc = (float)(pb.projDim[1] / 2 - pb.hoff[t]);
  }
}

}  // namespace

namespace fcb {
// Builds a plan.  `scratch` (>= 3 ints of device memory: status word, footprint maxima)
// receives the kernels' status and the footprint pre-pass result; the pre-pass runs on
// `st`.  scratch == NULL selects the library's per-device scratch word block.
static int bp_plan_build(const fcb_geometry* g, int kernelMode, int projType, int maxViewsPerLaunch,
                         int* scratch_in, cudaStream_t st, bool may_alloc, fcb_bp_plan** out)
{
  if (!out) return set_error(FCB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (projType != FCB_F32 && projType != FCB_F16 && projType != FCB_BF16)
    return set_error(FCB_ERR_INVALID, "unknown projection storage type");
  auto* pl = new fcb_bp_plan();
  pl->maxv = std::max(1, std::min(FDK_MAXV, maxViewsPerLaunch));
  // Views per launch.  A launch's CTAs drift apart in view index, so what stays in L2 is a
  // z-layer's detector rows of all the launch's views: at 1024^3 / 1536 x 1024, 900 views
  // (343 MB) overflow the 126 MB L2 and each launch reads ~0.55 TB from HBM, while 180
  // views keep it near the compulsory traffic (the volume's read-modify-write per launch)
  // at the same speed (measured 909 vs 906 ms per 1440-view step).  With the PI window most
  // views are skipped per tile, and the full launch size stays.
  if (maxViewsPerLaunch >= FDK_MAXV && !(kernelMode == 1 && g && g->piWindow)) pl->maxv = FDK_L2_VIEWS;
  // tuning knob: views per launch
  if (const char* e = getenv("FCB_FDK_VIEWS")) pl->maxv = std::max(1, std::min(FDK_MAXV, atoi(e)));
  // tuning knobs: z-voxels per thread (16/32/64) and the shared-memory budget per CTA
  if (const char* e = getenv("FCB_FDK_NZ")) {
    const int nz = atoi(e);
    if (nz == 16 || nz == 32 || nz == 64) pl->nz_tile = nz;
  }
  // only the FP32 pair path is instantiated for depths other than 32
  const char* sc = getenv("FCB_FDK_SCALAR");
  if (projType != FCB_F32 || (sc && sc[0] == '1')) pl->nz_tile = 32;
  int smem_budget = 64 * 1024, pair_budget = 0;
  if (const char* e = getenv("FCB_FDK_SMEM_KB")) {
    smem_budget = std::max(8, std::min(200, atoi(e))) * 1024;
    pair_budget = smem_budget;
  }
  int rc = make_problem(g, &pl->pb);
  if (rc) { delete pl; return rc; }
  Problem& pb = pl->pb;
  pl->mode = kernelMode == 0 ? 0 : (kernelMode == 1 ? 1 : 2);
  pl->ptype = projType;
  cudaGetDevice(&pl->device);
  const int nx = pb.volEnd[0] - pb.volStart[0], ny = pb.volEnd[1] - pb.volStart[1],
            nz = pb.volEnd[2] - pb.volStart[2];
  pl->updates = (long long)nx * ny * nz * pb.nviews;
  // every voxel must lie in front of the source
  const double rx = std::max(fabs((double)(pb.volStart[0] - pb.volDim[0] / 2)),
                             fabs((double)(pb.volEnd[0] - pb.volDim[0] / 2)));
  const double ry = std::max(fabs((double)(pb.volStart[1] - pb.volDim[1] / 2)),
                             fabs((double)(pb.volEnd[1] - pb.volDim[1] / 2)));
  if (sqrt(rx * rx + ry * ry) + 16.0 >= pb.D && !pb.misaligned) {
    delete pl;
    return set_error(FCB_ERR_INVALID, "volume reaches the source trajectory");
  }
  const float ox = (float)(pb.volStart[0] - pb.volDim[0] / 2);
  const float oy = (float)(pb.volStart[1] - pb.volDim[1] / 2);
  const float oz = (float)(pb.volStart[2] - pb.volDim[2] / 2);
  const int wexp = pl->mode == 0 ? 0 : (pl->mode == 1 ? 1 : 2);
  const bool piwin = pl->mode == 1 && pb.piWindow;
  const float td_a = (float)(pb.pitch / (2.0 * M_PI * pb.pw));
  const float td_r = (float)(pb.D / pb.pw);
  // The window's w axis runs against the source's direction of travel when the helix is
  // right-handed (angles and height increasing together); mirrored otherwise.
  const double turn = pb.nviews > 1 ? pb.angle[pb.nviews - 1] - pb.angle[0] : 1.0;
  const float td_sign = (turn >= 0.0) == (pb.pitch >= 0.0) ? -1.0f : 1.0f;

  // Reference-compatible windows: only when the reference's sub-problem windows cut off
  // part of a footprint does the result differ from the ideal operator; then the generic
  // kernel runs with the window table.
  RefWindows rw;
  bool compat = false;
  if (pb.referenceWindows && !piwin) {
    rc = ref_windows(pb, true, &rw);
    if (rc) { delete pl; return rc; }
    compat = rw.bp_matters;
  }
  if (compat) {
    if (!may_alloc) {
      delete pl;
      return set_error(FCB_ERR_INVALID,
                       "reference-compatible windows need a device table; this entry point allocates nothing");
    }
    const int ntile = rw.ntx * rw.nty * rw.ntz;
    std::vector<int4> tab((size_t)ntile * pb.nviews);
    for (int t = 0; t < ntile; t++)
      for (int v = 0; v < pb.nviews; v++) {
        const size_t o = (size_t)t * pb.nviews + v;
        tab[o] = make_int4(rw.ws[o] - pb.woff[v], rw.ws[o] + rw.subProjDim[0] - 1 - pb.woff[v],
                           rw.hs[o] - pb.hoff[v], rw.hs[o] + rw.subProjDim[1] - 1 - pb.hoff[v]);
      }
    if (cudaMalloc(&pl->d_win, tab.size() * sizeof(int4)) != cudaSuccess) {
      cudaGetLastError();
      pl->d_win = nullptr;
      delete pl;
      return set_error(FCB_ERR_NOMEM, "device allocation of the window table failed");
    }
    if (cudaMemcpy(pl->d_win, tab.data(), tab.size() * sizeof(int4), cudaMemcpyHostToDevice) !=
        cudaSuccess) {
      delete pl;
      return set_error(FCB_ERR_CUDA, "copy of the window table failed");
    }
  }

  if (aligned_geometry(pb) && !compat) {
    pl->path = 1;
    pl->wshift = projType == FCB_F32 ? 2 : 3;
    const int NZ = pl->nz_tile;
    const int tiles_x = (nx + FDK_TX - 1) / FDK_TX, tiles_y = (ny + FDK_TY - 1) / FDK_TY,
              tiles_z = (nz + NZ - 1) / NZ;
    for (int v0 = 0; v0 < pb.nviews; v0 += pl->maxv) {
      FdkParams P;
      memset(&P, 0, sizeof(P));
      P.nx = nx; P.ny = ny; P.nz = nz;
      P.tiles_x = tiles_x; P.tiles_y = tiles_y; P.tiles_z = tiles_z;
      P.ox = ox; P.oy = oy; P.oz = oz;
      P.hb = (float)(1.0 / pb.pw);
      P.wshift = pl->wshift;
      P.wexp = wexp;
      P.piwin = piwin ? 1 : 0;
      P.td_a = td_a; P.td_r = td_r; P.td_sign = td_sign;
      P.td_usc = (float)((double)td_sign / (double)td_r);
      P.cwait_ns = 2000000000ull;
      P.stop_after = -1;
      fill_fdk_views(pb, pl->mode, v0, std::min(pl->maxv, pb.nviews - v0), &P);
      // raster: y fastest when x moves the detector column more than y over these views
      // (w = (a0 x + a1 y) U + wc).  PI-window launches span most of a turn and stage few
      // views per tile; they keep x fastest (y fastest ran their pass 0.4 % slower).
      double sx = 0.0, sy = 0.0;
      for (int k = 0; k < P.nviews; k++) {
        sx += fabs((double)P.v[k].a0);
        sy += fabs((double)P.v[k].a1);
      }
      P.yfast = (!piwin && sx > sy) ? 1 : 0;
      pl->fdk.push_back(P);
    }
    // footprint pre-pass -> staging box
    int* scratch = scratch_in;
    if (!scratch) {
      rc = device_status_ptr(&scratch);
      if (rc) { delete pl; return rc; }
    }
    int* need = scratch + 1;
    const int ntiles = tiles_x * tiles_y * tiles_z;
    if (cudaMemsetAsync(need, 0, 2 * sizeof(int), st) != cudaSuccess) {
      delete pl;
      return set_error(FCB_ERR_CUDA, std::string("clearing the footprint maxima: ") +
                                         cudaGetErrorString(cudaGetLastError()));
    }
    for (const FdkParams& P : pl->fdk) {
      const long long total = (long long)tiles_x * tiles_y * (tiles_z > 1 ? 2 : 1) * P.nviews;
      const int blocks = (int)((total + 255) / 256);
      fdk_footprint_kernel<<<blocks, 256, 0, st>>>(P, NZ, ntiles, need);
    }
    int h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, need, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { delete pl; return set_error(FCB_ERR_CUDA, cudaGetErrorString(e)); }
    const int align = 1 << pl->wshift;
    pl->BW = ((h[0] + align - 1) / align) * align;
    // FP32 boxes: a row pitch of 4 mod 8 words puts the same column of consecutive rows in
    // different shared-memory banks (a multiple of 8 or 16 makes rows collide: at 48 the
    // slab case ran 13 % slower than at 44)
    if (projType == FCB_F32 && pl->BW % 8 == 0) pl->BW += 4;
    pl->BH = h[1] + 1;  // + 1: the inner z layers' corner floors (see fdk_footprint_kernel)
    if (pl->BW < align) pl->BW = align;
    if (pl->BH < 2) pl->BH = 2;
    // the largest dynamic shared memory a CTA of this device may opt into
    int smem_optin = 227 * 1024;  // sm_100
    if (cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, pl->device) !=
        cudaSuccess) {
      cudaGetLastError();
      smem_optin = 227 * 1024;
    }
    const size_t min_smem = projType == FCB_F32 ? fdk_smem_bytes(pl->BW, pl->BH, 2, 4)
                                                : fdk_pair_smem_bytes(pl->BW, pl->BH, 2, 2);
    if (pl->BW > 256 || pl->BH > 256 || min_smem > (size_t)smem_optin) {
      // footprint too large for one TMA box, or two staged boxes exceed a CTA's shared
      // memory (strong magnification: detector pixels much finer than voxels): generic kernel
      pl->path = 0;
      pl->fdk.clear();
    } else if (projType == FCB_F32) {
      const size_t stage_bytes = (((size_t)pl->BW * pl->BH * 4) + 127) & ~(size_t)127;
      const int st = (int)((size_t)smem_budget / stage_bytes);
      pl->stages = std::max(2, std::min(8, st));
    } else {
      // 16-bit storage (fdk_pair_kernel): two TMA stages of 16-bit taps and as many tap-pair
      // buffers (2..4) as the budget holds; the budget (74 KB unless set) keeps 3 CTAs per SM
      pl->stages = 2;
      const int budget = pair_budget > 0 ? pair_budget : 74 * 1024;
      int np = 2;
      while (np < 4 && fdk_pair_smem_bytes(pl->BW, pl->BH, 2, np + 1) <= (size_t)budget) np++;
      pl->pbufs = np;
    }
    if (pl->path == 1)
      for (FdkParams& P : pl->fdk) {
        P.BW = pl->BW; P.BH = pl->BH; P.stages = pl->stages; P.pbufs = pl->pbufs;
        P.status = scratch;
      }
  }
  if (pl->path == 0) {
    const int gmax = std::min(GEN_MAXV, pl->maxv);
    for (int v0 = 0; v0 < pb.nviews; v0 += gmax) {
      GenParams P;
      memset(&P, 0, sizeof(P));
      P.nx = nx; P.ny = ny; P.nz = nz;
      P.ox = ox; P.oy = oy; P.oz = oz;
      P.WH0 = pb.projWHSize[0]; P.WH1 = pb.projWHSize[1];
      P.ptype = projType;
      P.wexp = wexp;
      P.nviews = std::min(gmax, pb.nviews - v0);
      P.view0 = v0;
      P.piwin = piwin ? 1 : 0;
      P.td_a = td_a; P.td_r = td_r; P.td_sign = td_sign;
      fill_gen_views(pb, v0, P.nviews, &P);
      if (compat) {
        P.win = pl->d_win;
        P.sv0 = rw.subVolDim[0]; P.sv1 = rw.subVolDim[1]; P.sv2 = rw.subVolDim[2];
        P.ntx = rw.ntx; P.nty = rw.nty;
        P.wviews = pb.nviews;
      }
      pl->gen_parent.push_back((int)pl->gen.size());
      pl->gen.push_back(P);
    }
  }
  *out = pl;
  return ok();
}

int bp_plan_create_ex(const fcb_geometry* g, int kernelMode, int projType, int maxViewsPerLaunch,
                      fcb_bp_plan** out)
{
  return bp_plan_build(g, kernelMode, projType, maxViewsPerLaunch, nullptr, 0, true, out);
}

int bp_plan_chunks(const fcb_bp_plan* pl, std::vector<std::pair<int, int>>* ranges)
{
  ranges->clear();
  if (pl->path == 1) {
    for (const FdkParams& P : pl->fdk) ranges->push_back({P.view0, P.view0 + P.nviews});
  } else {
    for (const GenParams& P : pl->gen) ranges->push_back({P.view0, P.view0 + P.nviews});
  }
  return FCB_OK;
}

// Launch chunk `chunk` of the plan (-1: all chunks) over the volume planes [z0, z1) of the
// plan's sub-volume (z0, z1 multiples of the plan's z tile, or the volume's end; -1: all).
int bp_plan_execute_range(fcb_bp_plan* pl, int chunk, int z0, int z1, const void* proj,
                          float* volume, cudaStream_t st)
{
  if (!pl || !proj || !volume) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  const Problem& pb = pl->pb;
  const int nzv = pb.volEnd[2] - pb.volStart[2];
  if (z0 < 0) { z0 = 0; z1 = nzv; }
  if (z0 > z1 || z1 > nzv || (z0 % pl->nz_tile) || (z1 % pl->nz_tile && z1 != nzv))
    return set_error(FCB_ERR_INVALID, "plane range must follow the plan's z tiles");
  const int tz0 = z0 / pl->nz_tile, tz1 = (z1 + pl->nz_tile - 1) / pl->nz_tile;
  const size_t es = dtype_size(pl->ptype);
  bool tma_ok = pl->path == 1 && ((uintptr_t)proj % 16 == 0) &&
                ((size_t)pb.projWHSize[0] * es) % 16 == 0;
  if (pl->path == 1 && tma_ok) {
    CUtensorMap map;
    const CUtensorMapDataType dt = pl->ptype == FCB_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : pl->ptype == FCB_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                          : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    FCB_TRY(encode_tmap_3d(&map, dt, const_cast<void*>(proj), pb.projWHSize[0], pb.projWHSize[1],
                           pb.nviews, (uint64_t)pb.projWHSize[0] * es,
                           (uint64_t)pb.projWHSize[0] * pb.projWHSize[1] * es, pl->BW, pl->BH, 1));
    for (FdkParams& P : pl->fdk) P.vol = volume;
    const bool piw = pl->fdk[0].piwin != 0;
    // FCB_FDK_SCALAR=1 selects the one-voxel-per-instruction paths (for comparison)
    const char* scal = getenv("FCB_FDK_SCALAR");
    const bool scalar = scal && scal[0] == '1';
    if (pl->ptype == FCB_F32 && scalar) {
      if (piw) FCB_TRY((launch_fdk<float, 32, true, false>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<float, 32, false, false>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_F32 && pl->nz_tile == 16) {
      // FCB_FDK_MINB=4/5: register caps for 4 or 5 CTAs per SM (occupancy experiments)
      const char* mb = getenv("FCB_FDK_MINB");
      const int minb = mb ? atoi(mb) : 0;
      if (minb == 5) {
        if (piw) FCB_TRY((launch_fdk<float, 16, true, true, 5>(pl, map, chunk, tz0, tz1, st)));
        else FCB_TRY((launch_fdk<float, 16, false, true, 5>(pl, map, chunk, tz0, tz1, st)));
      } else if (minb == 4) {
        if (piw) FCB_TRY((launch_fdk<float, 16, true, true, 4>(pl, map, chunk, tz0, tz1, st)));
        else FCB_TRY((launch_fdk<float, 16, false, true, 4>(pl, map, chunk, tz0, tz1, st)));
      } else {
        if (piw) FCB_TRY((launch_fdk<float, 16, true, true>(pl, map, chunk, tz0, tz1, st)));
        else FCB_TRY((launch_fdk<float, 16, false, true>(pl, map, chunk, tz0, tz1, st)));
      }
    } else if (pl->ptype == FCB_F32 && pl->nz_tile == 64) {
      if (piw) FCB_TRY((launch_fdk<float, 64, true, true>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<float, 64, false, true>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_F32 && getenv("FCB_FDK_MINB4")) {
      // register cap for 4 CTAs per SM (occupancy experiment)
      if (piw) FCB_TRY((launch_fdk<float, 32, true, true, 4>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<float, 32, false, true, 4>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_F32) {
      if (piw) FCB_TRY((launch_fdk<float, 32, true, true>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<float, 32, false, true>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_F16 && scalar) {
      // 16-bit taps read one by one (the path before widening, for comparison)
      if (piw) FCB_TRY((launch_fdk<__half, 32, true, false>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<__half, 32, false, false>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_BF16 && scalar) {
      if (piw) FCB_TRY((launch_fdk<__nv_bfloat16, 32, true, false>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk<__nv_bfloat16, 32, false, false>(pl, map, chunk, tz0, tz1, st)));
    } else if (pl->ptype == FCB_F16) {
      if (piw) FCB_TRY((launch_fdk_pair<__half, true>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk_pair<__half, false>(pl, map, chunk, tz0, tz1, st)));
    } else {
      if (piw) FCB_TRY((launch_fdk_pair<__nv_bfloat16, true>(pl, map, chunk, tz0, tz1, st)));
      else FCB_TRY((launch_fdk_pair<__nv_bfloat16, false>(pl, map, chunk, tz0, tz1, st)));
    }
    return ok();
  }
  if (pl->gen.empty()) {
    // TMA path planned but this buffer cannot be described by a descriptor: build the
    // generic parameters on the fly, each staged launch's views in pieces of at most
    // GEN_MAXV (the generic kernel's parameter space holds fewer views)
    for (int fc = 0; fc < (int)pl->fdk.size(); fc++) {
      const FdkParams& F = pl->fdk[fc];
      for (int v0 = F.view0; v0 < F.view0 + F.nviews; v0 += GEN_MAXV) {
        GenParams P;
        memset(&P, 0, sizeof(P));
        P.nx = F.nx; P.ny = F.ny; P.nz = F.nz;
        P.ox = F.ox; P.oy = F.oy; P.oz = F.oz;
        P.WH0 = pb.projWHSize[0]; P.WH1 = pb.projWHSize[1];
        P.ptype = pl->ptype;
        P.wexp = F.wexp;
        P.nviews = std::min(GEN_MAXV, F.view0 + F.nviews - v0);
        P.view0 = v0;
        P.piwin = F.piwin;
        P.td_a = F.td_a;
        P.td_r = F.td_r;
        P.td_sign = F.td_sign;
        fill_gen_views(pb, v0, P.nviews, &P);
        pl->gen_parent.push_back(fc);
        pl->gen.push_back(P);
      }
    }
  }
  for (int c = 0; c < (int)pl->gen.size(); c++) {
    if (chunk >= 0 && pl->gen_parent[c] != chunk) continue;
    GenParams& P = pl->gen[c];
    P.vol = volume;
    P.proj = proj;
    const long long plane = (long long)P.nx * P.ny;
    P.vox0 = plane * z0;
    P.nvox = plane * (z1 - z0);
    if (P.nvox <= 0) continue;
    const long long threads = plane * ((z1 - z0 + GEN_NZ - 1) / GEN_NZ);
    bp_generic_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(P);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return ok();
}

int bp_plan_execute_chunk(fcb_bp_plan* pl, int chunk, const void* proj, float* volume,
                          cudaStream_t st)
{
  return bp_plan_execute_range(pl, chunk, -1, -1, proj, volume, st);
}

int bp_plan_z_tile(const fcb_bp_plan* pl) { return pl->nz_tile; }

}  // namespace fcb

extern "C" int fcb_bp_plan_create(const fcb_geometry* g, int kernelMode, int projType,
                                  fcb_bp_plan** out)
try {
  return bp_plan_create_ex(g, kernelMode, projType, FDK_MAXV, out);
}
FCB_CATCH_STATUS

extern "C" int fcb_bp_plan_execute(fcb_bp_plan* pl, const void* proj, float* volume, void* stream)
try {
  return bp_plan_execute_chunk(pl, -1, proj, volume, reinterpret_cast<cudaStream_t>(stream));
}
FCB_CATCH_STATUS

extern "C" int fcb_bp_plan_info(const fcb_bp_plan* pl, int* boxW, int* boxH, int* launches,
                                long long* updates)
try {
  if (!pl) return set_error(FCB_ERR_INVALID, "NULL plan");
  if (boxW) *boxW = pl->path == 1 ? pl->BW : 0;
  if (boxH) *boxH = pl->path == 1 ? pl->BH : 0;
  if (launches) *launches = pl->path == 1 ? (int)pl->fdk.size() : (int)pl->gen.size();
  if (updates) *updates = pl->updates;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_bp_plan_set_test_stall(fcb_bp_plan* pl, int stopAfterViews,
                                          unsigned long long consumerWaitNs)
try {
  if (!pl) return set_error(FCB_ERR_INVALID, "NULL plan");
  if (pl->path != 1) return set_error(FCB_ERR_INVALID, "the plan does not use the staged kernel");
  if (consumerWaitNs == 0 || consumerWaitNs > 2000000000ull)
    return set_error(FCB_ERR_INVALID, "consumer wait limit must lie in (0, 2 s]");
  for (FdkParams& P : pl->fdk) {
    P.stop_after = stopAfterViews < 0 ? -1 : stopAfterViews;
    P.cwait_ns = consumerWaitNs;
  }
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_bp_plan_destroy(fcb_bp_plan* pl)
try {
  delete pl;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_backproject_device(const fcb_geometry* g, int kernelMode, const void* proj,
                                      int projType, float* volume, void* stream)
try {
  fcb_bp_plan* pl = nullptr;
  FCB_TRY(fcb_bp_plan_create(g, kernelMode, projType, &pl));
  int rc = fcb_bp_plan_execute(pl, proj, volume, stream);
  fcb_bp_plan_destroy(pl);
  return rc;
}
FCB_CATCH_STATUS

// =====================================================================================
// Backprojection without device-memory allocation
// =====================================================================================
// Some callers cannot allocate device memory while they run: a process whose GPU memory
// is handed out by another allocator (a framework's caching pool, a fixed per-job
// budget on a shared GPU) or a timing-critical loop that must not stop for an
// allocation.  For them fcb_backproject_device_noalloc takes the few words of device
// scratch the backprojector needs (the kernels' status word and the footprint maxima of
// the staging-box pre-pass) from this file-scope array instead of cudaMalloc.  Every GPU
// that loads the library holds the array until the process exits.
constexpr int NOALLOC_SCRATCH_INTS = 64;  // 256 bytes; a call needs NOALLOC_NEEDED_INTS
constexpr int NOALLOC_NEEDED_INTS = 3;    // [0] status word, [1..2] footprint maxima
static __device__ __align__(256) int fcb_noalloc_scratch[NOALLOC_SCRATCH_INTS];

static_assert(NOALLOC_NEEDED_INTS <= NOALLOC_SCRATCH_INTS,
              "backprojection needs more scratch than the static array holds");

// Device address of fcb_noalloc_scratch on the current device.  The host-side name is only
// a stand-in for the symbol, so the address is looked up with the device current, on every
// call: the lookup allocates nothing, and an address cached across calls would go stale
// when the device's primary context is reset and created again.
static int noalloc_scratch_address(int** out)
{
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, fcb_noalloc_scratch);
  if (e != cudaSuccess)
    return set_error(FCB_ERR_CUDA, std::string("cudaGetSymbolAddress(fcb_noalloc_scratch): ") +
                                       cudaGetErrorString(e));
  *out = static_cast<int*>(p);
  return FCB_OK;
}

extern "C" int fcb_backproject_device_noalloc(const fcb_geometry* g, int kernelMode,
                                              const void* proj, int projType, float* volume,
                                              void* stream)
try {
  if (!proj || !volume) return set_error(FCB_ERR_INVALID, "NULL projection or volume pointer");
  int* scratch = nullptr;
  FCB_TRY(noalloc_scratch_address(&scratch));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: clear the status word and the maxima
  FCB_CUDA_TRY(cudaMemsetAsync(scratch, 0, NOALLOC_NEEDED_INTS * sizeof(int), st));
  fcb_bp_plan* pl = nullptr;
  FCB_TRY(bp_plan_build(g, kernelMode, projType, FDK_MAXV, scratch, st, false, &pl));
  int rc = bp_plan_execute_chunk(pl, -1, proj, volume, st);
  fcb_bp_plan_destroy(pl);
  if (rc) return rc;
  int status = 0;
  FCB_CUDA_TRY(cudaMemcpyAsync(&status, scratch, sizeof(int), cudaMemcpyDeviceToHost, st));
  FCB_CUDA_TRY(cudaStreamSynchronize(st));
  if (status & DEV_TIMEOUT) return set_error(FCB_ERR_TIMEOUT, "a bounded device-side wait timed out");
  if (status) return set_error(FCB_ERR_RANGE, "a kernel sample fell outside its staging window");
  return ok();
}
FCB_CATCH_STATUS

// Exact count of the voxel-view pairs inside the PI window over the geometry's sub-volume
// and views (helicalPitch != 0).  Synchronous; allocates a per-view table and a counter.
extern "C" int fcb_katsevich_pi_pairs(const fcb_geometry* g, long long* pairs, void* stream)
try {
  if (!g || !pairs) return set_error(FCB_ERR_INVALID, "NULL geometry or output");
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  if (pb.pitch == 0.0) return set_error(FCB_ERR_INVALID, "the PI window needs a helical pitch");
  const int n = pb.nviews;
  std::vector<PiView> hv(n);
  for (int t = 0; t < n; t++) hv[t] = PiView{pb.views[t].ca, pb.views[t].sa, pb.views[t].hmp};
  const double turn = n > 1 ? pb.angle[n - 1] - pb.angle[0] : 1.0;
  const double sgn = (turn >= 0.0) == (pb.pitch >= 0.0) ? -1.0 : 1.0;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  PiView* dv = nullptr;
  unsigned long long* dc = nullptr;
  struct Free {
    PiView*& v;
    unsigned long long*& c;
    ~Free()
    {
      cudaFree(v);
      cudaFree(c);
    }
  } fr{dv, dc};
  FCB_CUDA_TRY(cudaMalloc(&dv, (size_t)n * sizeof(PiView)));
  FCB_CUDA_TRY(cudaMalloc(&dc, sizeof(unsigned long long)));
  FCB_CUDA_TRY(cudaMemcpyAsync(dv, hv.data(), (size_t)n * sizeof(PiView), cudaMemcpyHostToDevice, st));
  FCB_CUDA_TRY(cudaMemsetAsync(dc, 0, sizeof(unsigned long long), st));
  const int nx = pb.volEnd[0] - pb.volStart[0], ny = pb.volEnd[1] - pb.volStart[1];
  const long long total = (long long)nx * ny * n;
  if (total > 0) {
    pi_pairs_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        dv, n, nx, ny, (double)(pb.volStart[0] - pb.volDim[0] / 2), (double)(pb.volStart[1] - pb.volDim[1] / 2),
        (long long)(pb.volStart[2] - pb.volDim[2] / 2), (long long)(pb.volEnd[2] - pb.volDim[2] / 2), pb.D,
        pb.pitch, sgn, dc);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  unsigned long long h = 0;
  FCB_CUDA_TRY(cudaMemcpyAsync(&h, dc, sizeof h, cudaMemcpyDeviceToHost, st));
  FCB_CUDA_TRY(cudaStreamSynchronize(st));
  *pairs = (long long)h;
  return ok();
}
FCB_CATCH_STATUS
