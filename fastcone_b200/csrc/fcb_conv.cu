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
// the caller).  conv3d16p_kernel is the persistent, pipelined form used by default.  The weight gradient, a 6912-entry reduction over all voxels, runs on the
// CUDA cores (fcb_conv3d16_wgrad_device).
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

}  // namespace fcb

using namespace fcb;

extern "C" int fcb_conv3d16_device(const void* x, const void* w, const float* bias, void* y, int yType,
                                   int nx, int ny, int nz, int relu, void* stream)
{
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

extern "C" int fcb_conv3d16_wgrad_device(const void* x, const void* dy, int dyType, float* dw, int nx, int ny,
                                         int nz, void* stream)
{
  if (!x || !dy || !dw || nx <= 0 || ny <= 0 || nz <= 0 || (dyType != FCB_F32 && dyType != FCB_BF16))
    return set_error(FCB_ERR_INVALID, "bad conv3d wgrad arguments");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
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
