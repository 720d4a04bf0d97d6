// fcb_conv.cu -- 3x3x3 convolutions (16 -> 16 channels, stride 1, zero padding 1) for the
// learned reconstruction's CNN, on the 5th-generation tensor cores (sm_100a tcgen05).
//
// Activations are BF16 in a channel-half-major layout, [z][y][2][x][8]: for every (z, y) row
// the 8 channels of half 0 of all x, then those of half 1, so that a TMA box of one half of
// one row is contiguous (no 32-byte sector is fetched for 16 useful bytes).  Weights BF16
// [27 taps][16 out][16 in]; accumulation FP32 in tensor memory.  Implicit GEMM: a CTA owns
// 128 consecutive x-voxels of one (y, z) row -> D[128 x 16] = sum over 27 taps of
// A_tap[128 x 16 in] * B_tap[16 in x 16 out].  The A operands of the three x-shifts of a tap
// row are the same TMA-loaded row of 130 voxels addressed 16 bytes apart, so 9 row loads
// (x 2 channel halves) feed all 27 MMAs.  Out-of-volume rows/voxels arrive as zeros from the
// TMA unit, which is the zero padding.  One elected thread issues the 27
// tcgen05.mma.cta_group::1.kind::f16 (M=128, N=16, K=16) and commits to an mbarrier; four
// warps read their TMEM lane quadrant back (tcgen05.ld 32x32b.x16), add the bias, apply
// ReLU and store.
//
// The same kernels compute the input gradient (transposed, tap-flipped weights, prepared by
// the caller); conv3d16r_kernel (row reuse) is the default form.  The weight gradient, a
// 6912-entry reduction over all voxels, runs on the tensor cores too
// (conv3d16_wgrad_tc_kernel, BF16 dY) with a CUDA-core kernel for FP32 dY and comparison.
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "fcb_internal.h"

namespace fcb {
namespace tc {

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dev::smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D(tmem) (+)= A(smem desc) * B(smem desc), BF16 inputs, FP32 accumulator.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.u32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   dev::smem_u32(bar))
               : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns: thread i of the warp gets row (lane base + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle ("interleaved" core matrices of 8
// rows x 16 bytes): start address, leading byte offset (between the two 8-element K
// halves), stride byte offset (between 8-row groups), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major, N, M.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3, int c4)
{
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dev::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(dev::smem_u32(bar))
      : "memory");
}

// Offset (elements) of channel c of voxel (x, y, z) in the [z][y][2][x][8] layout.
__host__ __device__ __forceinline__ size_t act_index(int x, int y, int z, int c, int nx, int ny)
{
  return ((((size_t)z * ny + y) * 2 + (c >> 3)) * nx + x) * 8 + (c & 7);
}

}  // namespace tc

constexpr int CV_TILE = 128;                  // voxels per CTA tile (MMA M)
constexpr int CV_ROW = CV_TILE + 2;           // staged voxels per tap row (x halo)
constexpr int CV_BOX_BYTES = CV_ROW * 16;     // one channel half of one tap row
constexpr int CV_RB = 2176;                   // CV_BOX_BYTES rounded up to 128 B
static_assert((CV_ROW + 2) / 2 * 32 <= CV_RB && CV_BOX_BYTES <= CV_RB, "a staged box fits its slot");
constexpr int CV_A_BYTES = 9 * 2 * CV_RB;     // 39168
constexpr int CV_W_BYTES = 27 * 512;          // 13824
constexpr int CV_SMEM = CV_A_BYTES + CV_W_BYTES + 64 + 32 + 16;

struct ConvParams {
  int pairs;               // 1: boxes of voxel pairs (32-byte rows, even nx), 0: single voxels
  uint32_t box_bytes;      // bytes of one staged half-row box
  const __nv_bfloat16* w;  // [27][16 out][16 in]
  const float* bias;       // [16] or null
  void* out;               // [z][y][x][16], bf16 or f32
  int out_f32;
  int relu;
  int nx, ny, nz;
  int tiles_x;
  int* status;
};

__global__ void __launch_bounds__(128) conv3d16_kernel(const __grid_constant__ CUtensorMap xmap,
                                                       const __grid_constant__ ConvParams P)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  unsigned char* Wsm = smem + CV_A_BYTES;
  float* bias = reinterpret_cast<float*>(Wsm + CV_W_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(Wsm + CV_W_BYTES + 64);  // [0] tma, [1] mma
  uint32_t* tslot = reinterpret_cast<uint32_t*>(Wsm + CV_W_BYTES + 64 + 16);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const int x0 = (tile % P.tiles_x) * CV_TILE;
  const int yz = tile / P.tiles_x;
  const int y = yz % P.ny, z = yz / P.ny;

  if (threadIdx.x == 0) {
    dev::mbar_init(&bars[0], 1);
    dev::mbar_init(&bars[1], 1);
    dev::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tslot, 32);
    tc::tmem_relinquish();
  }
  tc::fence_before();
  __syncthreads();

  if (threadIdx.x == 0) {
    dev::tma_prefetch(&xmap);
    dev::mbar_arrive_expect_tx(&bars[0], 18u * P.box_bytes);
    for (int r = 0; r < 9; r++) {
      const int dz = r / 3, dy = r % 3;
      for (int kh = 0; kh < 2; kh++)
        tc::tma_load_5d(A + (r * 2 + kh) * CV_RB, &xmap, &bars[0], 0, P.pairs ? (x0 >> 1) - 1 : x0 - 1, kh,
                        y + dy - 1, z + dz - 1);
    }
  }
  // weights -> core-matrix layout: tap t, K half kh, row n (out channel): 16 bytes of 8 in-channels
  const uint4* wg = reinterpret_cast<const uint4*>(P.w);
  for (int i = threadIdx.x; i < 27 * 16 * 2; i += blockDim.x) {
    const int t = i / 32, n = (i / 2) % 16, kh = i % 2;
    reinterpret_cast<uint4*>(Wsm + t * 512 + kh * 256 + n * 16)[0] = wg[(t * 16 + n) * 2 + kh];
  }
  if (threadIdx.x < 16) bias[threadIdx.x] = P.bias ? P.bias[threadIdx.x] : 0.0f;
  // generic-proxy shared stores -> visible to the tensor core's async-proxy reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *tslot;

  bool ok = true;
  if (threadIdx.x == 0) {
    ok = dev::mbar_wait(&bars[0], 0);
    if (ok) {
      tc::fence_after();
      const uint32_t abase = dev::smem_u32(A), wbase = dev::smem_u32(Wsm);
      constexpr uint32_t IDESC = tc::idesc_bf16(CV_TILE, 16);
      for (int t = 0; t < 27; t++) {
        const int r = t / 3, dx = t % 3;
        const uint64_t ad = tc::smem_desc(abase + r * 2 * CV_RB + (dx + P.pairs) * 16, CV_RB, 128);
        const uint64_t bd = tc::smem_desc(wbase + t * 512, 256, 128);
        tc::mma_bf16(taddr, ad, bd, IDESC, t > 0 ? 1u : 0u);
      }
      tc::mma_commit(&bars[1]);
    } else {
      dev::record_status(P.status, DEV_TIMEOUT);
      dev::mbar_wait(&bars[0], 0, 100000000ull);  // let in-flight copies land before exit
    }
  }
  // every thread waits (bounded) for the MMA commit; the result must be warp-uniform
  // because tcgen05.ld is a warp-collective instruction
  const bool done = __all_sync(0xffffffffu, dev::mbar_wait(&bars[1], 0) ? 1 : 0) != 0;
  tc::fence_after();
  if (done) {
    uint32_t r[16];
    tc::tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16), r);
    const int row = warp * 32 + lane;
    const int xv = x0 + row;
    if (xv < P.nx) {
      float v[16];
#pragma unroll
      for (int c = 0; c < 16; c++) {
        v[c] = __uint_as_float(r[c]) + bias[c];
        if (P.relu) v[c] = fmaxf(v[c], 0.0f);
      }
      const size_t i0 = tc::act_index(xv, y, z, 0, P.nx, P.ny), i1 = tc::act_index(xv, y, z, 8, P.nx, P.ny);
      if (P.out_f32) {
        float4* o0 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i0);
        float4* o1 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i1);
        o0[0] = make_float4(v[0], v[1], v[2], v[3]);
        o0[1] = make_float4(v[4], v[5], v[6], v[7]);
        o1[0] = make_float4(v[8], v[9], v[10], v[11]);
        o1[1] = make_float4(v[12], v[13], v[14], v[15]);
      } else {
        uint32_t pk[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
          pk[q] = *reinterpret_cast<uint32_t*>(&b);
        }
        __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(P.out);
        *reinterpret_cast<uint4*>(ob + i0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4*>(ob + i1) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
      }
    }
  } else if (threadIdx.x == 32) {
    dev::record_status(P.status, DEV_TIMEOUT);
  }
  // MMAs must have finished before the accumulator columns are released
  if (!done && threadIdx.x == 0 && ok) dev::mbar_wait(&bars[1], 0, 100000000ull);
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 32);
}

// Persistent, pipelined form of the same convolution: one CTA per SM walks the row tiles
// (tile = blockIdx.x + i * gridDim.x) with warp-specialised roles --
//   warp 4 (one lane): TMA producer, 18 row boxes per tile into a ring of CVP_STAGES buffers;
//   warp 5 (one lane): MMA issuer, 27 tcgen05.mma per tile into one of two TMEM
//                       accumulators (16 columns each), commits to the ring's empty barrier
//                       and to the accumulator's full barrier;
//   warps 0-3:         epilogue, each reads its 32-lane TMEM quadrant of the finished
//                       accumulator, releases it, adds bias / ReLU and stores.
// The weights are staged once per CTA, TMEM is allocated once, and the loads of the next
// tiles, the MMAs of this one and the stores of the previous one overlap.  Every wait is
// bounded; a role that times out records the status and stops, and the others stop at their
// next (bounded) wait.
constexpr int CVP_STAGES = 4;
constexpr int CVP_THREADS = 192;
constexpr int CVP_SMEM = CVP_STAGES * CV_A_BYTES + CV_W_BYTES + 64 + 8 * (2 * CVP_STAGES + 4) + 16;

__global__ void __launch_bounds__(CVP_THREADS, 1) conv3d16p_kernel(const __grid_constant__ CUtensorMap xmap,
                                                                  const __grid_constant__ ConvParams P,
                                                                  int ntiles)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  unsigned char* Wsm = smem + CVP_STAGES * CV_A_BYTES;
  float* bias = reinterpret_cast<float*>(Wsm + CV_W_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(Wsm + CV_W_BYTES + 64);
  uint64_t* empty = full + CVP_STAGES;
  uint64_t* accf = empty + CVP_STAGES;  // [2] accumulator written (MMA commit)
  uint64_t* acce = accf + 2;            // [2] accumulator read (4 epilogue warps)
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nmine = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < CVP_STAGES; s++) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      dev::mbar_init(&accf[b], 1);
      dev::mbar_init(&acce[b], 4);
    }
    dev::fence_mbar_init();
  }
  if (warp == 5) {
    tc::tmem_alloc(tslot, 32);
    tc::tmem_relinquish();
  }
  const uint4* wg = reinterpret_cast<const uint4*>(P.w);
  for (int i = threadIdx.x; i < 27 * 16 * 2; i += blockDim.x) {
    const int t = i / 32, n = (i / 2) % 16, kh = i % 2;
    reinterpret_cast<uint4*>(Wsm + t * 512 + kh * 256 + n * 16)[0] = wg[(t * 16 + n) * 2 + kh];
  }
  if (threadIdx.x < 16) bias[threadIdx.x] = P.bias ? P.bias[threadIdx.x] : 0.0f;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *tslot;

  if (warp == 4) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      dev::tma_prefetch(&xmap);
      int issued = 0;
      for (int i = 0; i < nmine; i++) {
        const int s = i % CVP_STAGES;
        if (i >= CVP_STAGES && !dev::mbar_wait(&empty[s], ((i / CVP_STAGES) - 1) & 1)) {
          dev::record_status(P.status, DEV_TIMEOUT);
          break;
        }
        issued = i + 1;
        const int tile = blockIdx.x + i * gridDim.x;
        const int x0 = (tile % P.tiles_x) * CV_TILE;
        const int yz = tile / P.tiles_x;
        const int y = yz % P.ny, z = yz / P.ny;
        unsigned char* As = A + s * CV_A_BYTES;
        dev::mbar_arrive_expect_tx(&full[s], 18u * P.box_bytes);
        for (int r = 0; r < 9; r++) {
          const int dz = r / 3, dy = r % 3;
          for (int kh = 0; kh < 2; kh++)
            tc::tma_load_5d(As + (r * 2 + kh) * CV_RB, &xmap, &full[s], 0, P.pairs ? (x0 >> 1) - 1 : x0 - 1,
                            kh, y + dy - 1, z + dz - 1);
        }
      }
      // no copy may still be landing in shared memory when the CTA leaves (bounded waits;
      // immediate unless another role stopped early)
      for (int j = max(0, issued - CVP_STAGES); j < issued; j++)
        dev::mbar_wait(&full[j % CVP_STAGES], (j / CVP_STAGES) & 1, 100000000ull);
    }
  } else if (warp == 5) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t wbase = dev::smem_u32(Wsm);
      constexpr uint32_t IDESC = tc::idesc_bf16(CV_TILE, 16);
      for (int i = 0; i < nmine; i++) {
        const int s = i % CVP_STAGES, b = i & 1;
        if (!dev::mbar_wait(&full[s], (i / CVP_STAGES) & 1) ||
            (i >= 2 && !dev::mbar_wait(&acce[b], ((i >> 1) - 1) & 1))) {
          dev::record_status(P.status, DEV_TIMEOUT);
          break;
        }
        tc::fence_after();
        const uint32_t abase = dev::smem_u32(A + s * CV_A_BYTES);
        for (int t = 0; t < 27; t++) {
          const int r = t / 3, dx = t % 3;
          const uint64_t ad = tc::smem_desc(abase + r * 2 * CV_RB + (dx + P.pairs) * 16, CV_RB, 128);
          const uint64_t bd = tc::smem_desc(wbase + t * 512, 256, 128);
          tc::mma_bf16(taddr + (uint32_t)(b * 16), ad, bd, IDESC, t > 0 ? 1u : 0u);
        }
        tc::mma_commit(&empty[s]);
        tc::mma_commit(&accf[b]);
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    for (int i = 0; i < nmine; i++) {
      const int b = i & 1;
      // warp-uniform: tcgen05.ld below is a warp-collective instruction
      if (!__all_sync(0xffffffffu, dev::mbar_wait(&accf[b], (i >> 1) & 1))) {
        if (lane == 0) dev::record_status(P.status, DEV_TIMEOUT);
        break;
      }
      tc::fence_after();
      uint32_t r[16];
      tc::tmem_ld16(taddr + (uint32_t)(b * 16) + ((uint32_t)(warp * 32) << 16), r);
      tc::fence_before();
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&acce[b]);
      const int tile = blockIdx.x + i * gridDim.x;
      const int x0 = (tile % P.tiles_x) * CV_TILE;
      const int yz = tile / P.tiles_x;
      const int y = yz % P.ny, z = yz / P.ny;
      const int xv = x0 + warp * 32 + lane;
      if (xv < P.nx) {
        float v[16];
#pragma unroll
        for (int c = 0; c < 16; c++) {
          v[c] = __uint_as_float(r[c]) + bias[c];
          if (P.relu) v[c] = fmaxf(v[c], 0.0f);
        }
        const size_t i0 = tc::act_index(xv, y, z, 0, P.nx, P.ny), i1 = tc::act_index(xv, y, z, 8, P.nx, P.ny);
        if (P.out_f32) {
          float4* o0 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i0);
          float4* o1 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i1);
          o0[0] = make_float4(v[0], v[1], v[2], v[3]);
          o0[1] = make_float4(v[4], v[5], v[6], v[7]);
          o1[0] = make_float4(v[8], v[9], v[10], v[11]);
          o1[1] = make_float4(v[12], v[13], v[14], v[15]);
        } else {
          uint32_t pk[8];
#pragma unroll
          for (int q = 0; q < 8; q++) {
            __nv_bfloat162 bb = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
            pk[q] = *reinterpret_cast<uint32_t*>(&bb);
          }
          __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(P.out);
          *reinterpret_cast<uint4*>(ob + i0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          *reinterpret_cast<uint4*>(ob + i1) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
      }
    }
  }
  // all MMAs this CTA issued must be complete before the columns are released: the
  // epilogue waited for every accumulator commit, and the issuer waits (bounded) for its last
  // one in case the epilogue stopped early
  if (warp == 5 && lane == 0 && nmine > 0) {
    const int last = nmine - 1;
    dev::mbar_wait(&accf[last & 1], (last >> 1) & 1, 100000000ull);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 5) {
    tc::fence_after();
    tc::tmem_dealloc(taddr, 32);
  }
}

// Row-reusing form (default): a CTA walks chunks of CVR_YCH consecutive y rows of one
// (x tile, z) column.  Neighbouring tiles share two of their three dy rows, so the input rows
// live in a ring of 4 slots per dz (slot dz * 4 + (row & 3)) and each tile loads only its 3
// new rows (9 at the start of a chunk): a third of the row traffic of conv3d16p_kernel.
//   warp 4 (one lane): TMA producer; before refilling the slots of row y+1 it waits for
//                      the MMAs of tile y-2, the last reader of the row it replaces;
//   warp 5 (one lane): MMA issuer (27 MMAs per tile, taps addressed through the ring),
//                      commits to the tile's done barrier and to the accumulator barrier;
//   warps 0-3:         epilogue, as in conv3d16p_kernel.
constexpr int CVR_YCH = 32;                 // rows per chunk
constexpr int CVR_SLOTS = 12;               // 3 dz x 4 ring positions
constexpr int CVR_THREADS = 192;
constexpr int CVR_SMEM = CVR_SLOTS * 2 * CV_RB + CV_W_BYTES + 64 + 8 * (4 + 4 + 2 + 2) + 16;

__global__ void __launch_bounds__(CVR_THREADS, 2) conv3d16r_kernel(const __grid_constant__ CUtensorMap xmap,
                                                                  const __grid_constant__ ConvParams P,
                                                                  int nchunks)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* A = smem;
  unsigned char* Wsm = smem + CVR_SLOTS * 2 * CV_RB;
  float* bias = reinterpret_cast<float*>(Wsm + CV_W_BYTES);
  uint64_t* rows_full = reinterpret_cast<uint64_t*>(Wsm + CV_W_BYTES + 64);  // [4] per tile
  uint64_t* tile_done = rows_full + 4;                                         // [4] per tile
  uint64_t* accf = tile_done + 4;                                              // [2]
  uint64_t* acce = accf + 2;                                                   // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ych = (P.ny + CVR_YCH - 1) / CVR_YCH;

  if (threadIdx.x == 0) {
    for (int q = 0; q < 4; q++) {
      dev::mbar_init(&rows_full[q], 1);
      dev::mbar_init(&tile_done[q], 1);
    }
    for (int b = 0; b < 2; b++) {
      dev::mbar_init(&accf[b], 1);
      dev::mbar_init(&acce[b], 4);
    }
    dev::fence_mbar_init();
  }
  if (warp == 5) {
    tc::tmem_alloc(tslot, 32);
    tc::tmem_relinquish();
  }
  const uint4* wg = reinterpret_cast<const uint4*>(P.w);
  for (int i = threadIdx.x; i < 27 * 16 * 2; i += blockDim.x) {
    const int t = i / 32, n = (i / 2) % 16, kh = i % 2;
    reinterpret_cast<uint4*>(Wsm + t * 512 + kh * 256 + n * 16)[0] = wg[(t * 16 + n) * 2 + kh];
  }
  if (threadIdx.x < 16) bias[threadIdx.x] = P.bias ? P.bias[threadIdx.x] : 0.0f;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *tslot;

  // chunk c -> x tile, z, rows [y0, y1)
  auto chunk_of = [&](int c, int& x0, int& z, int& y0, int& y1) {
    const int yc = c % ych, col = c / ych;
    x0 = (col % P.tiles_x) * CV_TILE;
    z = col / P.tiles_x;
    y0 = yc * CVR_YCH;
    y1 = min(P.ny, y0 + CVR_YCH);
  };
  int last = -1;  // tiles this CTA handles, minus one (same count in every role)
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    int x0, z, y0, y1;
    chunk_of(c, x0, z, y0, y1);
    last += y1 - y0;
  }

  if (warp == 4) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      dev::tma_prefetch(&xmap);
      int i = 0, issued = 0;
      bool failed = false;
      for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
        int x0, z, y0, y1;
        chunk_of(c, x0, z, y0, y1);
        for (int y = y0; y < y1; y++, i++) {
          const bool start = y == y0;
          // slots about to be refilled must be done with: tile i-2 (in a chunk) or every
          // earlier tile (a new chunk replaces all rows)
          const int wt = start ? i - 1 : i - 2;
          if (wt >= 0 && !dev::mbar_wait(&tile_done[wt & 3], (wt >> 2) & 1)) {
            dev::record_status(P.status, DEV_TIMEOUT);
            failed = true;
            break;
          }
          const int r0 = start ? -1 : 1;  // new rows y + r0 .. y + 1
          const int nrows = 3 * (2 - r0);
          dev::mbar_arrive_expect_tx(&rows_full[i & 3], (uint32_t)nrows * 2u * P.box_bytes);
          for (int dz = 0; dz < 3; dz++)
            for (int dy = r0; dy <= 1; dy++) {
              const int yy = y + dy;
              unsigned char* slot = A + (dz * 4 + (yy & 3)) * 2 * CV_RB;
              for (int kh = 0; kh < 2; kh++)
                tc::tma_load_5d(slot + kh * CV_RB, &xmap, &rows_full[i & 3], 0,
                                P.pairs ? (x0 >> 1) - 1 : x0 - 1, kh, yy, z + dz - 1);
            }
          issued = i + 1;
        }
      }
      for (int j = max(0, issued - 4); j < issued; j++)
        dev::mbar_wait(&rows_full[j & 3], (j >> 2) & 1, 100000000ull);
    }
  } else if (warp == 5) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t wbase = dev::smem_u32(Wsm), abase = dev::smem_u32(A);
      constexpr uint32_t IDESC = tc::idesc_bf16(CV_TILE, 16);
      int i = 0;
      bool failed = false;
      for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
        int x0, z, y0, y1;
        chunk_of(c, x0, z, y0, y1);
        for (int y = y0; y < y1; y++, i++) {
          const int b = i & 1;
          if (!dev::mbar_wait(&rows_full[i & 3], (i >> 2) & 1) ||
              (i >= 2 && !dev::mbar_wait(&acce[b], ((i >> 1) - 1) & 1))) {
            dev::record_status(P.status, DEV_TIMEOUT);
            failed = true;
            break;
          }
          tc::fence_after();
          for (int t = 0; t < 27; t++) {
            const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
            const int slot = dz * 4 + ((y + dy - 1) & 3);
            const uint64_t ad = tc::smem_desc(abase + slot * 2 * CV_RB + (dx + P.pairs) * 16, CV_RB, 128);
            const uint64_t bd = tc::smem_desc(wbase + t * 512, 256, 128);
            tc::mma_bf16(taddr + (uint32_t)(b * 16), ad, bd, IDESC, t > 0 ? 1u : 0u);
          }
          tc::mma_commit(&tile_done[i & 3]);
          tc::mma_commit(&accf[b]);
        }
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 0-3)
    int i = 0;
    bool failed = false;
    for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
      int x0, z, y0, y1;
      chunk_of(c, x0, z, y0, y1);
      for (int y = y0; y < y1; y++, i++) {
        const int b = i & 1;
        if (!__all_sync(0xffffffffu, dev::mbar_wait(&accf[b], (i >> 1) & 1))) {
          if (lane == 0) dev::record_status(P.status, DEV_TIMEOUT);
          failed = true;
          break;
        }
        tc::fence_after();
        uint32_t r[16];
        tc::tmem_ld16(taddr + (uint32_t)(b * 16) + ((uint32_t)(warp * 32) << 16), r);
        tc::fence_before();
        __syncwarp();
        if (lane == 0) dev::mbar_arrive(&acce[b]);
        const int xv = x0 + warp * 32 + lane;
        if (xv < P.nx) {
          float v[16];
#pragma unroll
          for (int q = 0; q < 16; q++) {
            v[q] = __uint_as_float(r[q]) + bias[q];
            if (P.relu) v[q] = fmaxf(v[q], 0.0f);
          }
          const size_t i0 = tc::act_index(xv, y, z, 0, P.nx, P.ny), i1 = tc::act_index(xv, y, z, 8, P.nx, P.ny);
          if (P.out_f32) {
            float4* o0 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i0);
            float4* o1 = reinterpret_cast<float4*>(reinterpret_cast<float*>(P.out) + i1);
            o0[0] = make_float4(v[0], v[1], v[2], v[3]);
            o0[1] = make_float4(v[4], v[5], v[6], v[7]);
            o1[0] = make_float4(v[8], v[9], v[10], v[11]);
            o1[1] = make_float4(v[12], v[13], v[14], v[15]);
          } else {
            uint32_t pk[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
              __nv_bfloat162 bb = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
              pk[q] = *reinterpret_cast<uint32_t*>(&bb);
            }
            __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(P.out);
            *reinterpret_cast<uint4*>(ob + i0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(ob + i1) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
          }
        }
      }
    }
  }
  // every MMA issued must be complete before the columns are released
  if (warp == 5 && lane == 0 && last >= 0) dev::mbar_wait(&accf[last & 1], (last >> 1) & 1, 100000000ull);
  tc::fence_before();
  __syncthreads();
  if (warp == 5) {
    tc::fence_after();
    tc::tmem_dealloc(taddr, 32);
  }
}

// Weight gradient on the CUDA cores: dW[t][co][ci] += sum_v dY[v][co] * X[v + off(t)][ci].
// Thread (co, ci) slides along a row of 128 voxels keeping the three x-neighbours of each of
// the 9 tap rows in registers; CTAs loop over tiles and add their 27 partial sums once.
struct WgradParams {
  const __nv_bfloat16* x;
  const void* dy;
  int dy_f32;
  float* dw;
  int nx, ny, nz, tiles_x, ntiles;
};

__device__ __forceinline__ float ld_act(const __nv_bfloat16* p) { return __bfloat162float(*p); }

constexpr int WG_TILE = 64;
__global__ void __launch_bounds__(256) conv3d16_wgrad_kernel(const WgradParams P)
{
  __shared__ float xs[9][WG_TILE + 2][17];
  __shared__ float ds[WG_TILE][17];
  const int co = threadIdx.x >> 4, ci = threadIdx.x & 15;
  float acc[27];
#pragma unroll
  for (int t = 0; t < 27; t++) acc[t] = 0.0f;
  for (int tile = blockIdx.x; tile < P.ntiles; tile += gridDim.x) {
    const int x0 = (tile % P.tiles_x) * WG_TILE;
    const int yz = tile / P.tiles_x;
    const int y = yz % P.ny, z = yz / P.ny;
    __syncthreads();
    for (int i = threadIdx.x; i < 9 * (WG_TILE + 2) * 16; i += blockDim.x) {
      const int c = i & 15, xr = (i >> 4) % (WG_TILE + 2), r = i / (16 * (WG_TILE + 2));
      const int zz = z + r / 3 - 1, yy = y + r % 3 - 1, xx = x0 + xr - 1;
      float v = 0.0f;
      if (zz >= 0 && zz < P.nz && yy >= 0 && yy < P.ny && xx >= 0 && xx < P.nx)
        v = ld_act(P.x + tc::act_index(xx, yy, zz, c, P.nx, P.ny));
      xs[r][xr][c] = v;
    }
    for (int i = threadIdx.x; i < WG_TILE * 16; i += blockDim.x) {
      const int c = i & 15, xr = i >> 4, xx = x0 + xr;
      float v = 0.0f;
      if (xx < P.nx) {
        const size_t o = tc::act_index(xx, y, z, c, P.nx, P.ny);
        v = P.dy_f32 ? reinterpret_cast<const float*>(P.dy)[o]
                     : ld_act(reinterpret_cast<const __nv_bfloat16*>(P.dy) + o);
      }
      ds[xr][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 9; r++) {
      float a = xs[r][0][ci], b = xs[r][1][ci];
      for (int v = 0; v < WG_TILE; v++) {
        const float c = xs[r][v + 2][ci];
        const float g = ds[v][co];
        acc[r * 3 + 0] = fmaf(g, a, acc[r * 3 + 0]);
        acc[r * 3 + 1] = fmaf(g, b, acc[r * 3 + 1]);
        acc[r * 3 + 2] = fmaf(g, c, acc[r * 3 + 2]);
        a = b;
        b = c;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 27; t++) atomicAdd(P.dw + (t * 16 + co) * 16 + ci, acc[t]);
}

// Weight gradient on the tensor cores (BF16 dY).  dW[t][co][ci] = sum over voxels v of
// dY[v][co] X[v + off(t)][ci] is a GEMM whose reduction dimension K is the voxels, 16 per
// MMA.  For one input row r = (dz, dy) and u = the X voxels x0-1 .. x0+142 of a 128-voxel
// tile (9 K-steps of 16):
//   D_r[s*16 + co][ci] = sum_u A[s*16 + co][u] * X_r[u][ci],   A[s*16 + co][u] = dY[u + 1 - s][co]
// with dY taken as zero outside the tile: rows s = 0, 1, 2 of D_r are the taps dx = s of row
// r (v = u + 1 - s runs over the tile).  The three dy rows of one dz sit in consecutive
// shared-memory slots, so one MMA per (K-step, dz) covers them: M = 128 (rows 0-47 used),
// N = 48 (dy, ci), K = 16 -- 27 MMAs per tile give all 27 taps.  A lives in tensor memory:
// warps 0-1 write the three shifted copies of the tile's dY (lane = s*16 + co, 16-bit voxel
// pairs packed per 32-bit column) with tcgen05.st from the staged dY row; B is the staged X
// rows, MN-major straight from the activation layout (8 channels of one voxel = one 16-byte
// core-matrix row).  TMEM: 3 accumulators of 48 columns (144) + WGT_ABUF A buffers of 72.
// A CTA walks chunks of CVR_YCH consecutive y rows of one (x tile, z) column; each tile loads
// its 3 new X rows into a ring of WGT_RING positions per dz, rows at positions 0 and 1 also
// into positions WGT_RING and WGT_RING + 1, so that rows y-1, y, y+1 always occupy three
// consecutive slots (a uniform N stride for B); dY rows are staged WGT_LEAD deep;
//   warp 2 (one lane): TMA producer, up to WGT_LEAD tiles ahead of the MMAs;
//   warps 0-1:         A writers (per tile), then the epilogue: TMEM lanes 0-47 of the
//                      accumulators -> dW (FP32 atomics, once per CTA);
//   warp 3 (one lane): MMA issuer, commits to the tile's done barrier.
// Dynamic shared memory above half an SM's keeps one CTA per SM (512-column allocation).
constexpr int WGT_THREADS = 128;
constexpr int WGT_KSTEPS = 9;                        // 144 voxels u per tile
constexpr int WGT_XROW = 148;                        // staged X voxels per row (from x0 - 2)
constexpr int WGT_RB = 2432;                         // one channel half of a staged X row, 128-B multiple
static_assert(WGT_XROW * 16 <= WGT_RB && (WGT_KSTEPS * 16 + 1) * 16 <= WGT_XROW * 16, "X row slot");
constexpr int WGT_DY_BYTES = 2048;                   // one channel half of 128 dY voxels (TMA box)
constexpr int WGT_DYH = 2432;                        // its slot: 8 zero voxels, the box, 16 zero voxels
// Pipeline depth: X rows in a ring of WGT_RING positions per dz, so the producer runs up to
// WGT_LEAD = WGT_RING - 2 tiles ahead of the MMAs; as many dY stages; WGT_ABUF A buffers.
constexpr int WGT_RING = 8;
constexpr int WGT_LEAD = WGT_RING - 2;
constexpr int WGT_ABUF = 3;
constexpr int WGT_DY = WGT_LEAD * 2 * WGT_DYH;       // dY stages x 2 halves
constexpr int WGT_XPOS = WGT_RING + 2;               // ring positions + the two duplicates
constexpr int WGT_X = 3 * WGT_XPOS * 2 * WGT_RB;     // X row ring
constexpr int WGT_BAR = WGT_DY + WGT_X;
constexpr int WGT_NBAR = 2 * WGT_RING + WGT_ABUF + 1;
constexpr int WGT_SMEM_USED = WGT_BAR + 8 * WGT_NBAR + 16;
static_assert(WGT_DYH >= (8 + CV_TILE + 16) * 16 && WGT_DYH % 128 == 0 && WGT_DY % 128 == 0, "dY slots");
constexpr int WGT_SMEM = 200 * 1024;                 // > half an SM: one CTA per SM
static_assert(WGT_SMEM_USED <= WGT_SMEM, "wgrad shared memory");
constexpr uint32_t WGT_ACOL = 144;                   // first A column (after the 9 accumulators)
constexpr uint32_t WGT_ACOLS = WGT_KSTEPS * 8;       // 72 columns per A buffer
static_assert(WGT_ACOL + WGT_ABUF * WGT_ACOLS <= 512, "TMEM columns");

struct WgradTcParams {
  float* dw;
  int nx, ny, nz, tiles_x, pairs;
  uint32_t xbox_bytes;
  int* status;
};

namespace tc {
// D(tmem) (+)= A(tmem) * B(smem desc), BF16 inputs, FP32 accumulator.
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.u32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// 32 lanes x 8 consecutive 32-bit columns from registers: thread i writes lane (base + i).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8])
{
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
}  // namespace tc

__global__ void __launch_bounds__(WGT_THREADS, 1) conv3d16_wgrad_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                                         const __grid_constant__ CUtensorMap dymap,
                                                                         const __grid_constant__ WgradTcParams P,
                                                                         int nchunks)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* DY = smem;
  unsigned char* X = smem + WGT_DY;
  uint64_t* rows_full = reinterpret_cast<uint64_t*>(smem + WGT_BAR);  // [WGT_RING] per tile
  uint64_t* tile_done = rows_full + WGT_RING;                           // [WGT_RING] per tile
  uint64_t* a_full = tile_done + WGT_RING;                              // [WGT_ABUF] A buffer written
  uint64_t* fin = a_full + WGT_ABUF;                                    // every MMA of the CTA done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  volatile int* failed_flag = reinterpret_cast<volatile int*>(tslot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ych = (P.ny + CVR_YCH - 1) / CVR_YCH;

  if (threadIdx.x == 0) {
    for (int q = 0; q < WGT_RING; q++) {
      dev::mbar_init(&rows_full[q], 1);
      dev::mbar_init(&tile_done[q], 1);
    }
    for (int b = 0; b < WGT_ABUF; b++) dev::mbar_init(&a_full[b], 2);
    dev::mbar_init(fin, 1);
    *failed_flag = 0;
    dev::fence_mbar_init();
  }
  // the dY slots' margins (voxels x0-8 .. x0-1 and x0+128 .. x0+143) stay zero: dY outside
  // the tile, which the shifted copies must not see
  for (int q = threadIdx.x; q < 2 * WGT_LEAD * 24; q += blockDim.x) {
    const int slot = q / 24, v = q % 24;
    reinterpret_cast<uint4*>(DY + slot * WGT_DYH)[v < 8 ? v : 128 + v] = make_uint4(0, 0, 0, 0);
  }
  if (warp == 3) {
    tc::tmem_alloc(tslot, 512);
    tc::tmem_relinquish();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *tslot;

  auto chunk_of = [&](int c, int& x0, int& z, int& y0, int& y1) {
    const int yc = c % ych, col = c / ych;
    x0 = (col % P.tiles_x) * CV_TILE;
    z = col / P.tiles_x;
    y0 = yc * CVR_YCH;
    y1 = min(P.ny, y0 + CVR_YCH);
  };
  int last = -1;  // tiles this CTA handles, minus one
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    int x0, z, y0, y1;
    chunk_of(c, x0, z, y0, y1);
    last += y1 - y0;
  }

  if (warp == 2) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      dev::tma_prefetch(&xmap);
      dev::tma_prefetch(&dymap);
      int i = 0, issued = 0;
      bool failed = false;
      for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
        int x0, z, y0, y1;
        chunk_of(c, x0, z, y0, y1);
        for (int y = y0; y < y1; y++, i++) {
          const bool start = y == y0;
          // the X slot refilled now (row y + 1) was last read by tile i - WGT_LEAD, every slot
          // at a new chunk by tile i-1; the dY stage by the A writers of tile i - WGT_LEAD,
          // which finished before its MMAs
          const int wt = start ? i - 1 : i - WGT_LEAD;
          if (wt >= 0 && !dev::mbar_wait(&tile_done[wt % WGT_RING], (wt / WGT_RING) & 1)) {
            dev::record_status(P.status, DEV_TIMEOUT);
            *failed_flag = 1;
            failed = true;
            break;
          }
          const int r0 = start ? -1 : 1;  // new rows y + r0 .. y + 1
          int ncopies = 0;
          for (int dy = r0; dy <= 1; dy++) ncopies += ((y + dy) & (WGT_RING - 1)) < 2 ? 2 : 1;
          uint64_t* full = &rows_full[i % WGT_RING];
          dev::mbar_arrive_expect_tx(full, (uint32_t)(3 * ncopies) * 2u * P.xbox_bytes + 2u * WGT_DY_BYTES);
          for (int dz = 0; dz < 3; dz++)
            for (int dy = r0; dy <= 1; dy++) {
              const int yy = y + dy, pos = yy & (WGT_RING - 1);
              for (int dup = 0; dup < (pos < 2 ? 2 : 1); dup++) {
                unsigned char* slot = X + (dz * WGT_XPOS + pos + dup * WGT_RING) * 2 * WGT_RB;
                for (int kh = 0; kh < 2; kh++)
                  tc::tma_load_5d(slot + kh * WGT_RB, &xmap, full, 0, P.pairs ? (x0 >> 1) - 1 : x0 - 1, kh, yy,
                                  z + dz - 1);
              }
            }
          unsigned char* dst = DY + (i % WGT_LEAD) * 2 * WGT_DYH + 128;  // after the 8 zero voxels
          for (int kh = 0; kh < 2; kh++)
            tc::tma_load_5d(dst + kh * WGT_DYH, &dymap, full, 0, P.pairs ? (x0 >> 1) : x0, kh, y, z);
          issued = i + 1;
        }
      }
      for (int j = max(0, issued - WGT_RING); j < issued; j++)
        dev::mbar_wait(&rows_full[j % WGT_RING], (j / WGT_RING) & 1, 100000000ull);
    }
  } else if (warp == 3) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t xbase = dev::smem_u32(X);
      // M = 128 (rows 0-47 used), N = 48, A K-major in TMEM, B MN-major in shared memory
      constexpr uint32_t IDESC = tc::idesc_bf16(CV_TILE, 48) | (1u << 16);
      int i = 0;
      bool failed = false;
      for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
        int x0, z, y0, y1;
        chunk_of(c, x0, z, y0, y1);
        for (int y = y0; y < y1; y++, i++) {
          if (!dev::mbar_wait(&rows_full[i % WGT_RING], (i / WGT_RING) & 1) ||
              !dev::mbar_wait(&a_full[i % WGT_ABUF], (i / WGT_ABUF) & 1)) {
            dev::record_status(P.status, DEV_TIMEOUT);
            *failed_flag = 1;
            failed = true;
            break;
          }
          tc::fence_after();
          // MN-major B over the slots of rows y-1, y, y+1 of one dz: N core matrices (dy, ci
          // half) every WGT_RB bytes (SBO), K core matrices of 8 voxels every 128 bytes (LBO);
          // a K-step of 16 voxels moves the start address by 256 B (16 in the descriptor's
          // address field, which stays below 2^14 inside shared memory)
          uint64_t bd[3];
          const int p0 = (y - 1) & (WGT_RING - 1);
#pragma unroll
          for (int dz = 0; dz < 3; dz++)
            bd[dz] = tc::smem_desc(xbase + (dz * WGT_XPOS + p0) * 2 * WGT_RB + P.pairs * 16, 128, WGT_RB);
          const uint32_t aaddr = taddr + WGT_ACOL + (uint32_t)(i % WGT_ABUF) * WGT_ACOLS;
          for (int ks = 0; ks < WGT_KSTEPS; ks++) {
            const uint32_t acc = (i > 0 || ks > 0) ? 1u : 0u;
#pragma unroll
            for (int dz = 0; dz < 3; dz++)
              tc::mma_bf16_ts(taddr + (uint32_t)(dz * 48), aaddr + (uint32_t)(ks * 8), bd[dz] + (uint64_t)(ks * 16),
                              IDESC, acc);
          }
          tc::mma_commit(&tile_done[i % WGT_RING]);
        }
      }
      // one phase that completes when every MMA issued here has (or at once if none was)
      if (i > 0) tc::mma_commit(fin);
      else dev::mbar_arrive(fin);
    }
  } else {
    // ---------------------------------------------------------------- A writers (warps 0-1)
    const int m = warp * 32 + lane;  // TMEM lane = s * 16 + co
    const int s = m >> 4, co = m & 15;
    const int se = s < 3 ? s : 2;    // lanes 48-63 (unused rows of D) copy s = 2
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    int i = 0;
    bool failed = false;
    for (int c = blockIdx.x; c < nchunks && !failed; c += gridDim.x) {
      int x0, z, y0, y1;
      chunk_of(c, x0, z, y0, y1);
      for (int y = y0; y < y1; y++, i++) {
        // the dY row of tile i is staged, and the A buffer's previous readers (the MMAs of
        // tile i - WGT_ABUF) are done
        bool ok = dev::mbar_wait(&rows_full[i % WGT_RING], (i / WGT_RING) & 1);
        const int pt = i - WGT_ABUF;
        if (ok && pt >= 0) ok = dev::mbar_wait(&tile_done[pt % WGT_RING], (pt / WGT_RING) & 1);
        if (!__all_sync(0xffffffffu, ok)) {
          if (lane == 0) {
            dev::record_status(P.status, DEV_TIMEOUT);
            *failed_flag = 1;
          }
          failed = true;
          break;
        }
        tc::fence_after();
        // A[u] = dY[x0 + rel], rel = 16 ks + k - s: slot voxel rel + 8 (zero outside the tile)
        const unsigned short* dyb = reinterpret_cast<const unsigned short*>(
            DY + (i % WGT_LEAD) * 2 * WGT_DYH + (co >> 3) * WGT_DYH + (8 - se) * 16) + (co & 7);
        const uint32_t acol = WGT_ACOL + (uint32_t)(i % WGT_ABUF) * WGT_ACOLS;
#pragma unroll 1
        for (int ks = 0; ks < WGT_KSTEPS; ks++) {
          const unsigned short* p = dyb + ks * 16 * 8;
          uint32_t pk[8];
#pragma unroll
          for (int j = 0; j < 8; j++) pk[j] = (uint32_t)p[(2 * j) * 8] | ((uint32_t)p[(2 * j + 1) * 8] << 16);
          tc::tmem_st8(taddr + lane_base + acol + (uint32_t)(ks * 8), pk);
        }
        tc::tmem_wait_st();
        tc::fence_before();
        __syncwarp();
        if (lane == 0) dev::mbar_arrive(&a_full[i % WGT_ABUF]);
      }
    }
    // ---------------------------------------------------------------- epilogue
    if (last >= 0) {
      const bool done = __all_sync(0xffffffffu, dev::mbar_wait(fin, 0)) != 0;
      tc::fence_after();
      if (done && !*failed_flag) {
        for (int r = 0; r < 9; r++) {
          uint32_t v[16];
          tc::tmem_ld16(taddr + lane_base + (uint32_t)(r * 16), v);
          if (s < 3) {
            float* d = P.dw + ((r * 3 + s) * 16 + co) * 16;
#pragma unroll
            for (int q = 0; q < 16; q++) atomicAdd(d + q, __uint_as_float(v[q]));
          }
        }
      } else if (!done && lane == 0) {
        dev::record_status(P.status, DEV_TIMEOUT);
      }
    }
  }
  // every MMA issued must be complete before the columns are released
  if (warp == 3 && lane == 0 && last >= 0) dev::mbar_wait(fin, 0, 100000000ull);
  tc::fence_before();
  __syncthreads();
  if (warp == 3) {
    tc::fence_after();
    tc::tmem_dealloc(taddr, 512);
  }
}

}  // namespace fcb

using namespace fcb;

extern "C" int fcb_conv3d16_device(const void* x, const void* w, const float* bias, void* y, int yType,
                                   int nx, int ny, int nz, int relu, void* stream)
try {
  if (!x || !w || !y || nx <= 0 || ny <= 0 || nz <= 0 || (yType != FCB_F32 && yType != FCB_BF16))
    return set_error(FCB_ERR_INVALID, "bad conv3d arguments");
  if (((uintptr_t)x & 15) || ((uintptr_t)w & 15) || ((uintptr_t)y & 15))
    return set_error(FCB_ERR_INVALID, "conv3d buffers must be 16-byte aligned");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  CUtensorMap map;
  // [z][y][2][x][8]: dims (channels of a voxel pair or of one voxel, x, half, y, z).  With
  // even nx a box row is a voxel pair (32 bytes, one L2 sector): 66 pairs cover voxels
  // x0-2 .. x0+129, and the MMA operands start one voxel into the box.  Single-voxel rows
  // (16 bytes) would fetch every sector twice.
  const bool pairs = nx % 2 == 0;
  const uint64_t dims[5] = {pairs ? 16u : 8u, (uint64_t)(pairs ? nx / 2 : nx), 2, (uint64_t)ny, (uint64_t)nz};
  const uint64_t strides[4] = {pairs ? 32u : 16u, 16ull * nx, 32ull * nx, 32ull * nx * ny};
  const uint32_t box[5] = {pairs ? 16u : 8u, pairs ? (uint32_t)(CV_ROW + 2) / 2 : (uint32_t)CV_ROW, 1, 1, 1};
  FCB_TRY(encode_tmap(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, strides, box));
  int* status = nullptr;
  FCB_TRY(device_status_ptr(&status));
  ConvParams P;
  P.pairs = pairs ? 1 : 0;
  P.box_bytes = box[0] * box[1] * 2;
  P.w = reinterpret_cast<const __nv_bfloat16*>(w);
  P.bias = bias;
  P.out = y;
  P.out_f32 = yType == FCB_F32;
  P.relu = relu;
  P.nx = nx; P.ny = ny; P.nz = nz;
  P.tiles_x = (nx + CV_TILE - 1) / CV_TILE;
  P.status = status;
  const long long tiles = (long long)P.tiles_x * ny * nz;
  if (tiles > 0x7fffffffll) return set_error(FCB_ERR_RANGE, "conv3d volume too large");
  // FCB_CONV_SIMPLE=1: one CTA per tile; FCB_CONV_SIMPLE=2: persistent without row reuse
  // (for comparison); default: persistent with row reuse
  const char* env = getenv("FCB_CONV_SIMPLE");
  const int variant = env ? atoi(env) : 0;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (variant == 1) {
    FCB_CUDA_TRY(cudaFuncSetAttribute(conv3d16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM));
    conv3d16_kernel<<<(unsigned)tiles, 128, CV_SMEM, st>>>(map, P);
  } else if (variant == 2) {
    FCB_CUDA_TRY(cudaFuncSetAttribute(conv3d16p_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CVP_SMEM));
    const int grid = (int)std::min<long long>(tiles, sms);
    conv3d16p_kernel<<<grid, CVP_THREADS, CVP_SMEM, st>>>(map, P, (int)tiles);
  } else {
    const long long nchunks = (long long)P.tiles_x * nz * ((ny + CVR_YCH - 1) / CVR_YCH);
    FCB_CUDA_TRY(cudaFuncSetAttribute(conv3d16r_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CVR_SMEM));
    const int grid = (int)std::min<long long>(nchunks, 2ll * sms);
    conv3d16r_kernel<<<grid, CVR_THREADS, CVR_SMEM, st>>>(map, P, (int)nchunks);
  }
  FCB_CUDA_TRY(cudaGetLastError());
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_conv3d16_wgrad_device(const void* x, const void* dy, int dyType, float* dw, int nx, int ny,
                                         int nz, void* stream)
try {
  if (!x || !dy || !dw || nx <= 0 || ny <= 0 || nz <= 0 || (dyType != FCB_F32 && dyType != FCB_BF16))
    return set_error(FCB_ERR_INVALID, "bad conv3d wgrad arguments");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // BF16 dY: tensor cores (FCB_WGRAD_SIMT=1 selects the CUDA-core kernel for comparison)
  const char* simt = getenv("FCB_WGRAD_SIMT");
  if (dyType == FCB_BF16 && !(simt && simt[0] == '1')) {
    if (((uintptr_t)x & 15) || ((uintptr_t)dy & 15))
      return set_error(FCB_ERR_INVALID, "conv3d wgrad buffers must be 16-byte aligned");
    const bool pairs = nx % 2 == 0;
    const uint64_t dims[5] = {pairs ? 16u : 8u, (uint64_t)(pairs ? nx / 2 : nx), 2, (uint64_t)ny, (uint64_t)nz};
    const uint64_t strides[4] = {pairs ? 32u : 16u, 16ull * nx, 32ull * nx, 32ull * nx * ny};
    const uint32_t xbox[5] = {pairs ? 16u : 8u, pairs ? (uint32_t)WGT_XROW / 2 : (uint32_t)WGT_XROW - 2, 1, 1, 1};
    const uint32_t dybox[5] = {pairs ? 16u : 8u, pairs ? (uint32_t)CV_TILE / 2 : (uint32_t)CV_TILE, 1, 1, 1};
    CUtensorMap xmap, dymap;
    FCB_TRY(encode_tmap(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), dims, strides, xbox));
    FCB_TRY(encode_tmap(&dymap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(dy), dims, strides, dybox));
    int* status = nullptr;
    FCB_TRY(device_status_ptr(&status));
    WgradTcParams T;
    T.dw = dw;
    T.nx = nx; T.ny = ny; T.nz = nz;
    T.tiles_x = (nx + CV_TILE - 1) / CV_TILE;
    T.pairs = pairs ? 1 : 0;
    T.xbox_bytes = xbox[0] * xbox[1] * 2;
    T.status = status;
    const long long nchunks = (long long)T.tiles_x * nz * ((ny + CVR_YCH - 1) / CVR_YCH);
    if (nchunks > 0x7fffffffll) return set_error(FCB_ERR_RANGE, "conv3d volume too large");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    FCB_CUDA_TRY(cudaFuncSetAttribute(conv3d16_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, WGT_SMEM));
    const int grid = (int)std::min<long long>(nchunks, sms);
    conv3d16_wgrad_tc_kernel<<<grid, WGT_THREADS, WGT_SMEM, st>>>(xmap, dymap, T, (int)nchunks);
    FCB_CUDA_TRY(cudaGetLastError());
    return ok();
  }
  WgradParams P;
  P.x = reinterpret_cast<const __nv_bfloat16*>(x);
  P.dy = dy;
  P.dy_f32 = dyType == FCB_F32;
  P.dw = dw;
  P.nx = nx; P.ny = ny; P.nz = nz;
  P.tiles_x = (nx + WG_TILE - 1) / WG_TILE;
  P.ntiles = P.tiles_x * ny * nz;
  const int grid = std::min(P.ntiles, 148 * 4);
  conv3d16_wgrad_kernel<<<grid, 256, 0, st>>>(P);
  FCB_CUDA_TRY(cudaGetLastError());
  return ok();
}
FCB_CATCH_STATUS
