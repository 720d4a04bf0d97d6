// fcb_internal.h -- declarations shared by the CUDA translation units of
// libfastcone_b200.so (not part of the public ABI; see include/fastcone_b200.h).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <exception>
#include <new>
#include <string>
#include <vector>

#include "fastcone_b200.h"

namespace fcb {

// ------------------------------------------------------------------ error plumbing
// Thread-local status of the last call (fcb_last_status / fcb_last_error).
int set_error(int code, const std::string& msg);
int ok();
#define FCB_CUDA_TRY(expr)                                                                 \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return ::fcb::set_error(e_ == cudaErrorMemoryAllocation ? FCB_ERR_NOMEM : FCB_ERR_CUDA, \
                              std::string(#expr) + ": " + cudaGetErrorString(e_));        \
  } while (0)
#define FCB_TRY(expr)            \
  do {                           \
    int s_ = (expr);             \
    if (s_ != FCB_OK) return s_; \
  } while (0)
// Every C entry point's body is a function-try-block ending in FCB_CATCH_STATUS: no C++
// exception (a failed host allocation, a copy thread that could not start) crosses the C
// boundary; it becomes a status like any other failure.
#define FCB_CATCH_STATUS                                                    \
  catch (const std::bad_alloc&)                                             \
  {                                                                         \
    return ::fcb::set_error(FCB_ERR_NOMEM, "host memory allocation failed"); \
  }                                                                         \
  catch (const std::exception& e)                                           \
  {                                                                         \
    return ::fcb::set_error(FCB_ERR_HOST, e.what());                        \
  }                                                                         \
  catch (...)                                                               \
  {                                                                         \
    return ::fcb::set_error(FCB_ERR_HOST, "unexpected host-side exception"); \
  }

// Device-side failure bits recorded in the per-device status word.
enum : int { DEV_TIMEOUT = 1, DEV_RANGE = 2 };

// Per-device status word (one int in global memory, allocated once per device).
int device_status_ptr(int** p);
// Unique id of the calling thread's current CUDA context (a reset device gets a new one);
// 0 when there is none or the driver cannot tell.
unsigned long long current_context_id();
// Reads and clears the status word after synchronising `stream`.
int collect_device_status(cudaStream_t stream);

// ------------------------------------------------------------------ geometry (FP64 host)
struct ViewGeom {
  // reference-units vectors (voxels), positions relative to the rotation axis / volume
  // centre (voxel g at g - volDim/2): source, detector centre, w and h pixel steps
  double s[3], d[3], w[3], h[3];
  double ca, sa, hmp;  // cos, sin of the angle, source height minus volDim[2]/2
};

struct Problem {
  int volDim[3], volStart[3], volEnd[3], projDim[3], projWHSize[2];
  int nviews;
  std::vector<int> woff, hoff;
  std::vector<double> angle, hmid, norm;
  double D, pw;
  bool misaligned;
  double mis[6];
  double pitch;  // helical pitch (voxels per turn), Katsevich window
  int piWindow;
  int referenceWindows;
  std::vector<ViewGeom> views;
};

int make_problem(const fcb_geometry* g, Problem* pb);

// Projective map of view t: [u, v, s] = M [x, y, z, 1] with x = voxel coordinate
// relative to the volume centre; (u/s, v/s) = continuous LOCAL window indices
// (pixel g of the window centred at g).  For the aligned geometry s is proportional
// to the source-voxel depth; kappa / s = U (= D / depth).
void view_matrix(const Problem& pb, int t, double M[12], double* kappa);

// The reference's sub-problem decomposition (fcb_refgeom.cpp): volume tiles (x fastest),
// per (tile, view) detector-window starts (global detector indices) and projector sweeps,
// the common window size, and whether they change the backprojection / the projection
// compared with the ideal operator.
struct RefWindows {
  int subVolDim[3] = {0, 0, 0};
  int subProjDim[2] = {0, 0};
  int ntx = 0, nty = 0, ntz = 0;
  std::vector<int> ws, hs, sweepStart, sweepSteps;  // [tile * nviews + view]
  bool bp_matters = false, proj_matters = false;
};
int ref_windows(const Problem& pb, bool with_misalign, RefWindows* rw);

// ------------------------------------------------------------------ TMA descriptors
int encode_tmap_3d(CUtensorMap* map, CUtensorMapDataType dtype, void* base, uint64_t d0,
                   uint64_t d1, uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes,
                   uint32_t b0, uint32_t b1, uint32_t b2);

// Tiled tensor map of any rank (1..5), no swizzle, zero fill out of bounds.
int encode_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int rank, void* base,
                const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box);

inline int dtype_size(int t) { return t == FCB_F32 ? 4 : 2; }

}  // namespace fcb

// ====================================================================== device helpers
#ifdef __CUDACC__
namespace fcb {
namespace dev {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase: false after `limit_ns` of global time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint64_t limit_ns = 2000000000ull)
{
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer() - t0 > limit_ns) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_prefetch(const CUtensorMap* map)
{
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// 3-D tiled TMA load into this CTA's own shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2)
{
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void record_status(int* status, int bits)
{
  if (status) atomicOr(status, bits);
}

}  // namespace dev
}  // namespace fcb
#endif
