// fcb_probe.cu -- measured ceilings for the rooflines of the staged kernels.
//
// The backprojector and the staged projector read their bilinear / trilinear taps from
// TMA-staged boxes in shared memory, so what bounds them is the rate at which an SM serves
// 32-bit ld.shared, not HBM.  fcb_smem_bandwidth measures that rate on the device at hand:
// every resident thread streams conflict-free ld.shared of 4, 8 or 16 bytes (each warp
// instruction covers all 32 banks, 128 bytes per wavefront), for a region long enough to
// time with CUDA events.  The result is a peak of the same kind as the HBM copy bandwidth
// used for memory-bound kernels: the plain access pattern, with nothing else to do.
#include "fcb_internal.h"

namespace fcb {

constexpr int PROBE_THREADS = 1024;
constexpr int PROBE_WORDS = 4096;  // 16 KB of shared memory per CTA

// One load of BYTES at shared address a + OFF (OFF an immediate), folded to 32 bits.
template <int BYTES, int OFF>
__device__ __forceinline__ uint32_t probe_ld(uint32_t a);
template <int OFF>
struct ProbeLd4 {
  static __device__ __forceinline__ uint32_t ld(uint32_t a)
  {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1+%2];" : "=r"(v) : "r"(a), "n"(OFF));
    return v;
  }
};
template <int OFF>
struct ProbeLd8 {
  static __device__ __forceinline__ uint32_t ld(uint32_t a)
  {
    uint32_t x, y;
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2+%3];" : "=r"(x), "=r"(y) : "r"(a), "n"(OFF));
    return x ^ y;
  }
};
template <int OFF>
struct ProbeLd16 {
  static __device__ __forceinline__ uint32_t ld(uint32_t a)
  {
    uint32_t x, y, z, w;
    asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4+%5];"
                 : "=r"(x), "=r"(y), "=r"(z), "=r"(w)
                 : "r"(a), "n"(OFF));
    return (x ^ y) ^ (z ^ w);
  }
};
template <int BYTES, int OFF>
__device__ __forceinline__ uint32_t probe_ld(uint32_t a)
{
  if constexpr (BYTES == 4) return ProbeLd4<OFF>::ld(a);
  else if constexpr (BYTES == 8) return ProbeLd8<OFF>::ld(a);
  else return ProbeLd16<OFF>::ld(a);
}

// K + 1 loads of consecutive warp rows (ROW = 32 * BYTES bytes apart) from address a.
template <int BYTES, int K>
struct ProbeRows {
  static __device__ __forceinline__ uint32_t run(uint32_t a)
  {
    return probe_ld<BYTES, K * 32 * BYTES>(a) ^ ProbeRows<BYTES, K - 1>::run(a);
  }
};
template <int BYTES>
struct ProbeRows<BYTES, -1> {
  static __device__ __forceinline__ uint32_t run(uint32_t) { return 0u; }
};

// Each thread reads BYTES at lane * BYTES of a warp row; a warp instruction reads one
// aligned row of 32 * BYTES bytes, so it touches each bank BYTES / 4 times (the minimum).
// Per iteration a warp reads 16 consecutive rows (immediate offsets, independent loads),
// then moves on by 16 rows within a 16 KB window.  `sink` receives the XOR of the values
// only when non-NULL (never in a measurement), which keeps the loads from being removed.
template <int BYTES>
__global__ void __launch_bounds__(PROBE_THREADS, 2) smem_probe_kernel(long long iters, uint32_t* sink)
{
  constexpr uint32_t ROW = 32 * BYTES;   // bytes one warp instruction reads
  constexpr uint32_t SPAN = PROBE_WORDS * 4;
  __shared__ __align__(16) uint32_t buf[(SPAN + 16 * ROW) / 4];
  for (int i = threadIdx.x; i < (int)((SPAN + 16 * ROW) / 4); i += blockDim.x) buf[i] = i * 2654435761u;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t base = dev::smem_u32(buf) + lane * BYTES;
  uint32_t off = (warp * ROW) % SPAN;  // a multiple of ROW below SPAN
  uint32_t acc = 0;
  for (long long it = 0; it < iters; it++) {
    acc ^= ProbeRows<BYTES, 15>::run(base + off);
    off = (off + 16 * ROW) % SPAN;
  }
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace fcb

using namespace fcb;

// Shared-memory load bandwidth of the current device with `bytesPerLoad` (4, 8 or 16) bytes
// per thread and instruction, conflict-free: two 1024-thread CTAs per SM, each thread
// issuing 16 * iters loads.  *ms = the kernel's CUDA-event time on `stream`, *bytes = the
// bytes loaded.  Synchronous.
extern "C" int fcb_smem_bandwidth(int bytesPerLoad, long long iters, float* ms, double* bytes,
                                  void* stream)
try {
  if (!ms || !bytes || iters <= 0) return set_error(FCB_ERR_INVALID, "bad probe arguments");
  if (bytesPerLoad != 4 && bytesPerLoad != 8 && bytesPerLoad != 16)
    return set_error(FCB_ERR_INVALID, "bytesPerLoad must be 4, 8 or 16");
  int dev = 0, sms = 0;
  FCB_CUDA_TRY(cudaGetDevice(&dev));
  FCB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int grid = 2 * sms;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  struct Ev {
    cudaEvent_t& a;
    cudaEvent_t& b;
    ~Ev()
    {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } evg{e0, e1};
  FCB_CUDA_TRY(cudaEventCreate(&e0));
  FCB_CUDA_TRY(cudaEventCreate(&e1));
  FCB_CUDA_TRY(cudaEventRecord(e0, st));
  if (bytesPerLoad == 4) smem_probe_kernel<4><<<grid, PROBE_THREADS, 0, st>>>(iters, nullptr);
  else if (bytesPerLoad == 8) smem_probe_kernel<8><<<grid, PROBE_THREADS, 0, st>>>(iters, nullptr);
  else smem_probe_kernel<16><<<grid, PROBE_THREADS, 0, st>>>(iters, nullptr);
  FCB_CUDA_TRY(cudaGetLastError());
  FCB_CUDA_TRY(cudaEventRecord(e1, st));
  FCB_CUDA_TRY(cudaEventSynchronize(e1));
  FCB_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
  *bytes = (double)grid * PROBE_THREADS * 16.0 * (double)iters * bytesPerLoad;
  return ok();
}
FCB_CATCH_STATUS
