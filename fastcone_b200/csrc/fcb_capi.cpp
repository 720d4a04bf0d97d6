// fcb_capi.cpp -- the reference-compatible C ABI and the host-buffer drivers.
//
// GPU_CB_* reproduce the entry points of wrapper.c (argument order of its definitions,
// which is the order fastcone.py calls), dispatching like GPU_CB_K_backproject
// (wrapper.c:134-143).  The host drivers replace the sub-problem loops of
// unit_coneBeamGPU.cu:88-305: instead of tiling through 1024x1024x512 textures with
// blocking pageable copies and host-side window caches, the whole sub-volume and the
// projection windows live in HBM; projections are streamed in view chunks on a copy
// stream while the backprojection of the previous chunk runs on the compute stream.
#include <stdio.h>
#include <string.h>

#include <stdlib.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#include "fcb_internal.h"

namespace fcb {
int project_launch(const Problem& pb, int method, const float* vol, float* proj, float* adj_vol,
                   unsigned long long* samples, cudaStream_t st);
int bp_plan_create_ex(const fcb_geometry* g, int kernelMode, int projType, int maxViewsPerLaunch,
                      fcb_bp_plan** out);
int bp_plan_chunks(const fcb_bp_plan* pl, std::vector<std::pair<int, int>>* ranges);
int bp_plan_execute_chunk(fcb_bp_plan* pl, int chunk, const void* proj, float* volume,
                          cudaStream_t st);
int bp_plan_execute_range(fcb_bp_plan* pl, int chunk, int z0, int z1, const void* proj,
                          float* volume, cudaStream_t st);
int bp_plan_z_tile(const fcb_bp_plan* pl);
int filter_plan_run(fcb_filter_plan* pl, const float* in, void* out, int nviews, int pitch, float D,
                    const float* dzorig, int cosineWeight, cudaStream_t st);
int filter_plan_create(int nviews, int H, int W, int outType, int window, double gaussScale,
                       fcb_filter_plan** out);
void filter_plan_destroy(fcb_filter_plan* pl);
}  // namespace fcb

using namespace fcb;

extern "C" int fcb_version(void) { return 10000; }

namespace {

struct DeviceGuard {
  int prev = -1;
  int rc = FCB_OK;
  explicit DeviceGuard(int dev)
  {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
      rc = set_error(FCB_ERR_NODEVICE, "no CUDA device");
      return;
    }
    if (dev < 0 || dev >= n) {
      rc = set_error(FCB_ERR_NODEVICE, "GPUID does not name a CUDA device");
      return;
    }
    cudaGetDevice(&prev);
    if (cudaSetDevice(dev) != cudaSuccess) rc = set_error(FCB_ERR_CUDA, "cudaSetDevice failed");
  }
  ~DeviceGuard()
  {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------------- device block cache
// The host entry points move whole problems through device memory on every call (13.4 GB
// for a 1024^3 / 1440-view backprojection); cudaMalloc and cudaFree of that much take from a
// few to over a hundred milliseconds per call.  A call's blocks are therefore kept per device
// when it ends and handed to later calls that fit in them (the smallest cached block of at
// least the request and at most twice it).  At most 8 blocks per device are kept (the oldest
// go back to the driver), fcb_release_device_cache returns them all, and FCB_HOST_CACHE=0
// frees every block when its call ends.
namespace {
struct CachedBlock {
  int dev;
  unsigned long long ctx;  // the context the block belongs to (a reset device has a new one)
  void* p;
  size_t bytes;
};
std::mutex g_cache_mu;
std::vector<CachedBlock> g_cache;  // oldest first
constexpr int CACHE_BLOCKS_PER_DEVICE = 8;

bool cache_enabled()
{
  const char* e = getenv("FCB_HOST_CACHE");
  return !(e && e[0] == '0');
}

// fcb_fbp_host's filter plans (cuFFT plans and about half a gigabyte of scratch each) are
// kept the same way, keyed by their parameters, at most 4 per device.
struct CachedFilter {
  int dev;
  unsigned long long ctx;
  int nviews, H, W, window;
  fcb_filter_plan* p;
};
std::vector<CachedFilter> g_fcache;  // oldest first
constexpr int CACHE_FILTERS_PER_DEVICE = 4;

// Forgets the cached entries of `dev` made in another context than `ctx` (the device was
// reset: their memory and plans went with the old context); the caller holds g_cache_mu.
void cache_forget_stale_locked(int dev, unsigned long long ctx)
{
  for (size_t i = 0; i < g_cache.size();) {
    if (g_cache[i].dev == dev && g_cache[i].ctx != ctx) g_cache.erase(g_cache.begin() + (long)i);
    else i++;
  }
  for (size_t i = 0; i < g_fcache.size();) {
    if (g_fcache[i].dev == dev && g_fcache[i].ctx != ctx) g_fcache.erase(g_fcache.begin() + (long)i);
    else i++;
  }
}

// Frees the cached blocks and filter plans of `dev` (-1: of every device); entries of a
// context that is gone are only forgotten.  The caller holds g_cache_mu.
void cache_drop_locked(int dev)
{
  if (g_cache.empty() && g_fcache.empty()) return;
  int cur = -1;
  cudaGetDevice(&cur);
  auto live = [](int d, unsigned long long c) {
    return cudaSetDevice(d) == cudaSuccess && current_context_id() == c;
  };
  for (size_t i = 0; i < g_fcache.size();) {
    if (dev < 0 || g_fcache[i].dev == dev) {
      if (live(g_fcache[i].dev, g_fcache[i].ctx)) filter_plan_destroy(g_fcache[i].p);
      g_fcache.erase(g_fcache.begin() + (long)i);
    } else {
      i++;
    }
  }
  for (size_t i = 0; i < g_cache.size();) {
    if (dev < 0 || g_cache[i].dev == dev) {
      if (live(g_cache[i].dev, g_cache[i].ctx)) cudaFree(g_cache[i].p);
      g_cache.erase(g_cache.begin() + (long)i);
    } else {
      i++;
    }
  }
  if (cur >= 0) cudaSetDevice(cur);
  cudaGetLastError();
}
}  // namespace

// RAII bundle of device buffers/streams/events of one host-driver call.
struct Scratch {
  struct Block {
    void* p;
    size_t bytes;
  };
  int dev = -1;
  unsigned long long ctx = 0;
  std::vector<Block> blocks;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  ~Scratch()
  {
    for (cudaStream_t s : streams) cudaStreamSynchronize(s);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
    if (blocks.empty()) return;
    if (!cache_enabled()) {
      for (const Block& b : blocks) cudaFree(b.p);
      return;
    }
    // every stream of the call has finished: the blocks are free for the next call
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (const Block& b : blocks) g_cache.push_back(CachedBlock{dev, ctx, b.p, b.bytes});
    int n = 0;
    for (const CachedBlock& c : g_cache) n += c.dev == dev;
    for (size_t i = 0; i < g_cache.size() && n > CACHE_BLOCKS_PER_DEVICE;) {
      if (g_cache[i].dev == dev) {
        cudaFree(g_cache[i].p);
        g_cache.erase(g_cache.begin() + (long)i);
        n--;
      } else {
        i++;
      }
    }
  }
  int alloc(void** p, size_t bytes)
  {
    if (dev < 0) {
      FCB_CUDA_TRY(cudaGetDevice(&dev));
      FCB_CUDA_TRY(cudaFree(nullptr));  // make sure the device's context exists
      ctx = current_context_id();
    }
    if (cache_enabled()) {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      cache_forget_stale_locked(dev, ctx);
      long best = -1;
      for (size_t i = 0; i < g_cache.size(); i++) {
        const CachedBlock& c = g_cache[i];
        if (c.dev == dev && c.bytes >= bytes && c.bytes <= 2 * bytes &&
            (best < 0 || c.bytes < g_cache[(size_t)best].bytes))
          best = (long)i;
      }
      if (best >= 0) {
        *p = g_cache[(size_t)best].p;
        blocks.push_back(Block{*p, g_cache[(size_t)best].bytes});
        g_cache.erase(g_cache.begin() + best);
        return FCB_OK;
      }
    }
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      cudaGetLastError();
      // memory held by the cache goes back to the driver, then one more try
      {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        cache_drop_locked(dev);
      }
      if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_error(FCB_ERR_NOMEM, "device allocation failed");
      }
    }
    blocks.push_back(Block{*p, bytes});
    return FCB_OK;
  }
  // high: the device's highest stream priority (its kernels' CTAs take SMs ahead of the
  // other streams' waiting CTAs)
  int stream(cudaStream_t* s, bool high = false)
  {
    int least = 0, greatest = 0;
    if (high) FCB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    FCB_CUDA_TRY(cudaStreamCreateWithPriority(s, cudaStreamNonBlocking, high ? greatest : 0));
    streams.push_back(*s);
    return FCB_OK;
  }
  int event(cudaEvent_t* e)
  {
    FCB_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    events.push_back(*e);
    return FCB_OK;
  }
};

// ---------------------------------------------------------------- pageable host buffers
// cudaMemcpyAsync from or to pageable memory goes through the driver's staging on the
// calling thread (about 9 GB/s on the B200 hosts measured).  Callers of the reference's API
// pass numpy arrays, which are pageable; for them the stager below fills a ring of pinned
// buffers with several host threads while DMA moves the previous ones, so that the PCIe
// link rather than one memcpy thread sets the pace.  Buffers that are already pinned or
// registered go straight to cudaMemcpyAsync.
bool is_pageable(const void* p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

void par_memcpy(void* dst, const void* src, size_t bytes, int nthreads)
{
  if (nthreads <= 1 || bytes < ((size_t)4 << 20)) {
    memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> th;
  const size_t part = ((bytes + nthreads - 1) / nthreads + 4095) & ~(size_t)4095;
  for (int t = 0; t < nthreads; t++) {
    const size_t o = (size_t)t * part;
    if (o >= bytes) break;
    const size_t nb = std::min(part, bytes - o);
    th.emplace_back([=] { memcpy((char*)dst + o, (const char*)src + o, nb); });
  }
  for (std::thread& x : th) x.join();
}

// The pinned buffers are made on the first staged call and kept until the process exits
// (3 x 64 MB of page-locked host memory: pinning them per call would cost more than small
// transfers save); calls that stage take turns on them.
std::mutex g_pin_mu;
void* g_pin[3] = {nullptr, nullptr, nullptr};

struct HostStager {
  static constexpr size_t PIECE = (size_t)64 << 20;  // bytes per pinned buffer
  static constexpr size_t MIN_BYTES = (size_t)64 << 20;  // smaller transfers copy directly
  static constexpr int NBUF = 3;
  void* buf[NBUF] = {nullptr, nullptr, nullptr};
  cudaEvent_t done[NBUF] = {nullptr, nullptr, nullptr};
  bool used[NBUF] = {false, false, false};
  int next = 0, nthreads = 1;
  bool ok = false;
  std::unique_lock<std::mutex> lock;

  // `bytes`: the pageable traffic of the call; below MIN_BYTES the stager stays off
  int init(size_t bytes)
  {
    if (bytes < MIN_BYTES || getenv("FCB_HOST_NOSTAGE")) return FCB_OK;
    lock = std::unique_lock<std::mutex>(g_pin_mu);
    for (int b = 0; b < NBUF; b++) {
      if (!g_pin[b] && cudaHostAlloc(&g_pin[b], PIECE, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        g_pin[b] = nullptr;
        return FCB_OK;  // not fatal: the caller falls back to plain copies
      }
      buf[b] = g_pin[b];
      if (cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return FCB_OK;
      }
    }
    unsigned hc = std::thread::hardware_concurrency();
    nthreads = (int)std::max(1u, std::min(16u, hc ? hc : 1u));
    if (const char* e = getenv("FCB_HOST_THREADS")) nthreads = std::max(1, std::min(64, atoi(e)));
    ok = true;
    return FCB_OK;
  }
  ~HostStager()
  {
    for (int b = 0; b < NBUF; b++) {
      if (done[b]) {
        cudaEventSynchronize(done[b]);
        cudaEventDestroy(done[b]);
      }
    }
  }
  int take(int* b)
  {
    *b = next;
    next = (next + 1) % NBUF;
    if (used[*b]) FCB_CUDA_TRY(cudaEventSynchronize(done[*b]));
    used[*b] = true;
    return FCB_OK;
  }
  // device rows [r0, r0 + nrows) of `width` bytes at pitch dpitch <- contiguous host rows;
  // returns once the host data sits in pinned memory (the DMA may still run on s)
  int h2d_rows(char* dst, size_t dpitch, const char* src, size_t width, size_t rows, cudaStream_t s)
  {
    const size_t per = std::max<size_t>(1, PIECE / width);
    for (size_t r0 = 0; r0 < rows; r0 += per) {
      const size_t nr = std::min(per, rows - r0);
      int b;
      FCB_TRY(take(&b));
      par_memcpy(buf[b], src + r0 * width, nr * width, nthreads);
      if (dpitch == width)
        FCB_CUDA_TRY(cudaMemcpyAsync(dst + r0 * width, buf[b], nr * width, cudaMemcpyHostToDevice, s));
      else
        FCB_CUDA_TRY(cudaMemcpy2DAsync(dst + r0 * dpitch, dpitch, buf[b], width, width, nr,
                                       cudaMemcpyHostToDevice, s));
      FCB_CUDA_TRY(cudaEventRecord(done[b], s));
    }
    return FCB_OK;
  }
  int h2d(void* dst, const void* src, size_t bytes, cudaStream_t s)
  {
    return h2d_rows((char*)dst, 1, (const char*)src, 1, bytes, s);
  }
  // host <- device after the work queued on s; synchronous.  The DMA of one piece overlaps
  // the host copy of the previous one.
  int d2h(void* dst, const void* src, size_t bytes, cudaStream_t s)
  {
    int pend = -1;
    size_t pend_o = 0, pend_n = 0;
    for (size_t o = 0; o < bytes; o += PIECE) {
      const size_t n = std::min(PIECE, bytes - o);
      int b;
      FCB_TRY(take(&b));
      FCB_CUDA_TRY(cudaMemcpyAsync(buf[b], (const char*)src + o, n, cudaMemcpyDeviceToHost, s));
      FCB_CUDA_TRY(cudaEventRecord(done[b], s));
      if (pend >= 0) {
        FCB_CUDA_TRY(cudaEventSynchronize(done[pend]));
        par_memcpy((char*)dst + pend_o, buf[pend], pend_n, nthreads);
      }
      pend = b;
      pend_o = o;
      pend_n = n;
    }
    if (pend >= 0) {
      FCB_CUDA_TRY(cudaEventSynchronize(done[pend]));
      par_memcpy((char*)dst + pend_o, buf[pend], pend_n, nthreads);
    }
    return FCB_OK;
  }
};

// Host window views [v0, v1) -> device buffer rows padded to `wpad` floats.
int copy_proj_h2d(float* d, const float* h, int v0, int v1, int W, int H, int wpad, cudaStream_t s,
                  HostStager* stager)
{
  const size_t rows = (size_t)(v1 - v0) * H;
  if (stager) {
    FCB_TRY(stager->h2d_rows(reinterpret_cast<char*>(d + (size_t)v0 * H * wpad), (size_t)wpad * sizeof(float),
                             reinterpret_cast<const char*>(h + (size_t)v0 * H * W), (size_t)W * sizeof(float),
                             rows, s));
  } else if (wpad == W) {
    FCB_CUDA_TRY(cudaMemcpyAsync(d + (size_t)v0 * H * W, h + (size_t)v0 * H * W,
                                 rows * W * sizeof(float), cudaMemcpyHostToDevice, s));
  } else {
    FCB_CUDA_TRY(cudaMemcpy2DAsync(d + (size_t)v0 * H * wpad, wpad * sizeof(float),
                                   h + (size_t)v0 * H * W, W * sizeof(float), W * sizeof(float), rows,
                                   cudaMemcpyHostToDevice, s));
  }
  return FCB_OK;
}

}  // namespace

// Phase times of one host-driver call, printed to stderr when FCB_HOST_TRACE is set.
struct HostTrace {
  bool on = getenv("FCB_HOST_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const
  {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

// FDK pre-processing done inside the host pipeline (fcb_fbp_host): each uploaded view chunk
// is cosine-weighted and ramp filtered in place on the device before its backprojection,
// and the filtered views go back to the caller's buffer `out`.
struct FbpFilter {
  int window;
  float D;
  const float* zOrigin;
  int cosine;
  float* out;
};

// Host-buffer backprojection, pipelined over view chunks and z-slabs of the volume:
//   copy-in stream : the first view chunk, the volume slab by slab, then the other chunks
//   compute stream : chunk by chunk as they arrive, each over all slabs (slab s of the first
//                    chunk as soon as slab s is in)
//   copy-out stream: slab s back to the host as soon as the last chunk has passed over it
//   (with `ff`: a filter stream filters each chunk as it lands, ahead of its backprojection,
//   and a fourth stream returns each filtered chunk to the caller)
// so the PCIe traffic (projections once, the volume in and out) hides behind the kernels
// except for the first chunk with the first slab, and the last slab.  One plan (one staging
// pre-pass) serves every slab: a slab is a range of the plan's z tiles.  Reference-compatible
// windows that change the result run as one slab (their tiling starts at volStart).
static int backproject_host_impl(int device, const fcb_geometry* g0, int kernelMode,
                                 const float* projections, float* volume, const FbpFilter* ff)
{
  if (!g0 || !projections || !volume) return set_error(FCB_ERR_INVALID, "NULL argument");
  HostTrace tr;
  DeviceGuard guard(device);
  if (guard.rc) return guard.rc;
  fcb_geometry g = *g0;
  if (kernelMode != 0) g.misAlignments = nullptr;
  const int W = g.projWHSize[0], H = g.projWHSize[1], n = g.projDim[2];
  if (W <= 0 || H <= 0 || n <= 0) return set_error(FCB_ERR_INVALID, "bad projection sizes");
  for (int a = 0; a < 3; a++)
    if (g.volEnd[a] <= g.volStart[a]) return set_error(FCB_ERR_INVALID, "empty volume range");
  if (g.referenceWindows) {
    // the reference's windows depend on the data width: decide on the caller's geometry,
    // and leave the rows unpadded when the windows change the result
    Problem p0;
    FCB_TRY(make_problem(&g, &p0));
    RefWindows rw;
    FCB_TRY(ref_windows(p0, true, &rw));
    if (!rw.bp_matters) g.referenceWindows = 0;
  }
  // TMA row pitch must be a multiple of 16 bytes
  const int wpad = g.referenceWindows ? W : (W + 3) & ~3;
  g.projWHSize[0] = wpad;  // zero columns beyond W change nothing (zero extension)

  const int chunk = 120;  // views per upload chunk
  fcb_bp_plan* plan = nullptr;
  FCB_TRY(bp_plan_create_ex(&g, kernelMode, FCB_F32, chunk, &plan));
  struct PlanGuard {
    fcb_bp_plan* p;
    ~PlanGuard() { fcb_bp_plan_destroy(p); }
  } pg{plan};
  std::vector<std::pair<int, int>> ranges;
  FCB_TRY(bp_plan_chunks(plan, &ranges));
  const double t_plan = tr.ms();

  // z-slabs: multiples of the plan's z tile, at least 64 planes, at most 8
  const int nx = g.volEnd[0] - g.volStart[0], ny = g.volEnd[1] - g.volStart[1],
            nz = g.volEnd[2] - g.volStart[2];
  const int zt = bp_plan_z_tile(plan);
  int nslab = g.referenceWindows ? 1 : std::max(1, std::min(8, nz / 64));
  const int slab = ((nz + nslab - 1) / nslab + zt - 1) / zt * zt;
  nslab = (nz + slab - 1) / slab;
  std::vector<int> z0, z1;
  // With four slabs or more the first and the last are small (64 planes rounded up to the z
  // tile): the first slab's upload delays the first kernel and the last slab's download
  // follows the last one, and neither overlaps anything.  Slab boundaries stay on z-tile
  // boundaries (a slab is a range of the plan's z tiles).
  const int ntz = (nz + zt - 1) / zt, et = (64 + zt - 1) / zt;  // tiles: all, per edge slab
  if (nslab >= 4 && ntz >= 4 * et) {
    const int nmid = nslab - 2, mt = (ntz - 2 * et + nmid - 1) / nmid;
    z0.push_back(0);
    z1.push_back(et * zt);
    for (int t = et; t < ntz - et; t += mt) {
      z0.push_back(t * zt);
      z1.push_back(std::min(ntz - et, t + mt) * zt);
    }
    z0.push_back((ntz - et) * zt);
    z1.push_back(nz);
  } else {
    for (int s = 0; s < nslab; s++) {
      z0.push_back(s * slab);
      z1.push_back(std::min(nz, s * slab + slab));
    }
  }
  nslab = (int)z0.size();

  const size_t plane = (size_t)nx * ny;
  const size_t nvox = plane * nz;
  Scratch sc;
  float *dvol = nullptr, *dproj = nullptr, *dz = nullptr;
  FCB_TRY(sc.alloc((void**)&dvol, nvox * sizeof(float)));
  FCB_TRY(sc.alloc((void**)&dproj, (size_t)n * H * wpad * sizeof(float)));
  cudaStream_t cs, xs, os, ps = nullptr, fs = nullptr;
  FCB_TRY(sc.stream(&cs));
  FCB_TRY(sc.stream(&xs));
  FCB_TRY(sc.stream(&os));
  fcb_filter_plan* fplan = nullptr;
  int fdev = -1, fkey[4] = {0, 0, 0, 0};  // the plan's device and (views, H, W, window)
  unsigned long long fctx = 0;             // and context
  struct FilterGuard {
    fcb_filter_plan*& p;
    cudaStream_t& s;
    int& dev;
    unsigned long long& ctx;
    int* key;
    ~FilterGuard()
    {
      if (!p) return;
      cudaStreamSynchronize(s);  // the plan's scratch is in use until the filter stream ends
      if (!cache_enabled()) {
        filter_plan_destroy(p);
        return;
      }
      std::lock_guard<std::mutex> lk(g_cache_mu);
      g_fcache.push_back(CachedFilter{dev, ctx, key[0], key[1], key[2], key[3], p});
      int n = 0;
      for (const CachedFilter& c : g_fcache) n += c.dev == dev;
      for (size_t i = 0; i < g_fcache.size() && n > CACHE_FILTERS_PER_DEVICE;) {
        if (g_fcache[i].dev == dev) {
          filter_plan_destroy(g_fcache[i].p);
          g_fcache.erase(g_fcache.begin() + (long)i);
          n--;
        } else {
          i++;
        }
      }
    }
  } fguard{fplan, fs, fdev, fctx, fkey};
  std::vector<cudaEvent_t> filt_done(ranges.size(), nullptr);
  if (ff) {
    int maxc = 1;
    for (const auto& r : ranges) maxc = std::max(maxc, r.second - r.first);
    // the filter of chunk c + 1 runs while chunk c is backprojected; at high priority its
    // CTAs are placed as the backprojection's retire instead of after all of them
    FCB_TRY(sc.stream(&fs, true));
    FCB_CUDA_TRY(cudaGetDevice(&fdev));
    fctx = current_context_id();
    fkey[0] = maxc; fkey[1] = H; fkey[2] = W; fkey[3] = ff->window;
    if (cache_enabled()) {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      cache_forget_stale_locked(fdev, fctx);
      for (size_t i = 0; i < g_fcache.size(); i++) {
        const CachedFilter& c = g_fcache[i];
        if (c.dev == fdev && c.nviews == maxc && c.H == H && c.W == W && c.window == ff->window) {
          fplan = c.p;
          g_fcache.erase(g_fcache.begin() + (long)i);
          break;
        }
      }
    }
    if (!fplan) FCB_TRY(filter_plan_create(maxc, H, W, FCB_F32, ff->window, 0.125, &fplan));
    FCB_TRY(sc.stream(&ps));
    if (ff->cosine) {
      FCB_TRY(sc.alloc((void**)&dz, (size_t)n * sizeof(float)));
      FCB_CUDA_TRY(cudaMemcpyAsync(dz, ff->zOrigin, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, fs));
    }
  }
  const double t_alloc = tr.ms();
  if (wpad != W) FCB_CUDA_TRY(cudaMemsetAsync(dproj, 0, (size_t)n * H * wpad * sizeof(float), xs));
  // pageable caller buffers (numpy arrays): pinned staging filled by host threads
  HostStager stager;
  const bool proj_pg = is_pageable(projections), vol_pg = is_pageable(volume);
  const bool out_pg = ff && is_pageable(ff->out);
  FCB_TRY(stager.init((proj_pg ? (size_t)n * H * W * sizeof(float) : 0) + (vol_pg ? 2 * nvox * sizeof(float) : 0) +
                      (out_pg ? (size_t)n * H * W * sizeof(float) : 0)));
  HostStager* pst = proj_pg && stager.ok ? &stager : nullptr;
  HostStager* vst = vol_pg && stager.ok ? &stager : nullptr;
  HostStager* fst = out_pg && stager.ok && wpad == W ? &stager : nullptr;
  // filter chunk c in place on the filter stream once `uploaded` has fired (so the next
  // chunk's filter overlaps this chunk's backprojection), then return it to the caller: on its
  // own stream at once, or (pageable output through the pinned ring) after every kernel is
  // queued.  The compute stream waits for filt_done[c] before backprojecting chunk c.
  auto filter_chunk = [&](int c, cudaEvent_t uploaded) -> int {
    const int v0 = ranges[c].first, nv = ranges[c].second - v0;
    float* p = dproj + (size_t)v0 * H * wpad;
    FCB_CUDA_TRY(cudaStreamWaitEvent(fs, uploaded, 0));
    FCB_TRY(filter_plan_run(fplan, p, p, nv, wpad, ff->D, ff->cosine ? dz + v0 : nullptr, ff->cosine, fs));
    FCB_TRY(sc.event(&filt_done[c]));
    FCB_CUDA_TRY(cudaEventRecord(filt_done[c], fs));
    if (!fst) {
      FCB_CUDA_TRY(cudaStreamWaitEvent(ps, filt_done[c], 0));
      float* h = ff->out + (size_t)v0 * H * W;
      if (wpad == W)
        FCB_CUDA_TRY(cudaMemcpyAsync(h, p, (size_t)nv * H * W * sizeof(float), cudaMemcpyDeviceToHost, ps));
      else
        FCB_CUDA_TRY(cudaMemcpy2DAsync(h, W * sizeof(float), p, wpad * sizeof(float), W * sizeof(float),
                                       (size_t)nv * H, cudaMemcpyDeviceToHost, ps));
    }
    return FCB_OK;
  };
  std::vector<cudaEvent_t> slab_done(nslab, nullptr);
  auto zoff = [&](int s) { return (size_t)z0[s] * plane; };
  auto slab_bytes = [&](int s) { return (size_t)(z1[s] - z0[s]) * plane * sizeof(float); };
  cudaEvent_t ev;
  cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (tr.on)
    for (cudaEvent_t& e : tev) FCB_CUDA_TRY(cudaEventCreate(&e));
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[0], xs));

  const int nch = (int)ranges.size();
  // Chunk-major over the first half of the view chunks (their kernels hide the upload of the
  // projections), then slab-major over the rest: each slab finishes in turn and its copy-out
  // overlaps the next slab's kernels, instead of every slab finishing with the last chunk.
  // Every voxel still sees the chunks in order 0, 1, ..., so the result is unchanged.
  int cm = nch >= 2 ? nch / 2 : 0;
  if (const char* e = getenv("FCB_HOST_CHUNK_MAJOR")) cm = std::max(0, std::min(nch, atoi(e)));
  auto copy_vol_slab = [&](int s) -> int {
    if (vst)
      FCB_TRY(vst->h2d(dvol + zoff(s), volume + zoff(s), slab_bytes(s), xs));
    else
      FCB_CUDA_TRY(cudaMemcpyAsync(dvol + zoff(s), volume + zoff(s), slab_bytes(s), cudaMemcpyHostToDevice, xs));
    FCB_TRY(sc.event(&ev));
    FCB_CUDA_TRY(cudaEventRecord(ev, xs));
    FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
    if (s == 0 && tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[1], cs));
    return FCB_OK;
  };
  auto finish_slab = [&](int s) -> int {
    FCB_TRY(sc.event(&ev));
    FCB_CUDA_TRY(cudaEventRecord(ev, cs));
    if (vst) {
      slab_done[s] = ev;  // staged copy-out below, once every kernel is queued
    } else {
      FCB_CUDA_TRY(cudaStreamWaitEvent(os, ev, 0));
      FCB_CUDA_TRY(cudaMemcpyAsync(volume + zoff(s), dvol + zoff(s), slab_bytes(s), cudaMemcpyDeviceToHost, os));
    }
    return FCB_OK;
  };
  for (int c = 0; c < cm; c++) {
    FCB_TRY(copy_proj_h2d(dproj, projections, ranges[c].first, ranges[c].second, W, H, wpad, xs, pst));
    FCB_TRY(sc.event(&ev));
    FCB_CUDA_TRY(cudaEventRecord(ev, xs));
    if (ff) {
      FCB_TRY(filter_chunk(c, ev));
      FCB_CUDA_TRY(cudaStreamWaitEvent(cs, filt_done[c], 0));
    } else {
      FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
    }
    for (int s = 0; s < nslab; s++) {
      if (c == 0) FCB_TRY(copy_vol_slab(s));
      FCB_TRY(bp_plan_execute_range(plan, c, z0[s], z1[s], dproj, dvol, cs));
    }
  }
  if (cm == 0)
    for (int s = 0; s < nslab; s++) FCB_TRY(copy_vol_slab(s));
  std::vector<cudaEvent_t> up(nch, nullptr);
  for (int c = cm; c < nch; c++) {
    FCB_TRY(copy_proj_h2d(dproj, projections, ranges[c].first, ranges[c].second, W, H, wpad, xs, pst));
    FCB_TRY(sc.event(&up[c]));
    FCB_CUDA_TRY(cudaEventRecord(up[c], xs));
    if (ff) FCB_TRY(filter_chunk(c, up[c]));
  }
  for (int s = 0; s < nslab; s++) {
    for (int c = cm; c < nch; c++) {
      if (s == 0) FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ff ? filt_done[c] : up[c], 0));
      FCB_TRY(bp_plan_execute_range(plan, c, z0[s], z1[s], dproj, dvol, cs));
    }
    FCB_TRY(finish_slab(s));
  }
  // pageable output of the filtered views: through the pinned ring, chunk by chunk
  if (fst)
    for (int c = 0; c < nch; c++) {
      const int v0 = ranges[c].first, nv = ranges[c].second - v0;
      FCB_CUDA_TRY(cudaStreamWaitEvent(os, filt_done[c], 0));
      FCB_TRY(fst->d2h(ff->out + (size_t)v0 * H * W, dproj + (size_t)v0 * H * wpad,
                       (size_t)nv * H * W * sizeof(float), os));
    }
  // staged copy-out of each slab as soon as its last kernel is done (os waits for it); the
  // later slabs' kernels run meanwhile
  if (vst)
    for (int s = 0; s < nslab; s++) {
      FCB_CUDA_TRY(cudaStreamWaitEvent(os, slab_done[s], 0));
      FCB_TRY(vst->d2h(volume + zoff(s), dvol + zoff(s), slab_bytes(s), os));
    }
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[2], cs));
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[3], os));
  FCB_CUDA_TRY(cudaStreamSynchronize(os));
  if (ps) FCB_CUDA_TRY(cudaStreamSynchronize(ps));
  if (fs) FCB_CUDA_TRY(cudaStreamSynchronize(fs));
  FCB_CUDA_TRY(cudaStreamSynchronize(cs));
  FCB_TRY(collect_device_status(cs));
  if (tr.on) {
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, tev[0], tev[1]);
    cudaEventElapsedTime(&b, tev[0], tev[2]);
    cudaEventElapsedTime(&c, tev[0], tev[3]);
    fprintf(stderr,
            "fcb_backproject_host: %d slab(s) of %d planes, %d view chunks; plan %.1f ms, "
            "alloc %.1f ms; first kernel at %.1f ms, kernels done %.1f ms, volume home %.1f ms "
            "(GPU clock from the first copy); call %.1f ms\n",
            nslab, slab, nch, t_plan, t_alloc - t_plan, a, b, c, tr.ms());
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
  }
  return ok();
}

extern "C" int fcb_backproject_host(int device, const fcb_geometry* g, int kernelMode,
                                    const float* projections, float* volume)
try {
  return backproject_host_impl(device, g, kernelMode, projections, volume, nullptr);
}
FCB_CATCH_STATUS

// fastcone.fbp on host buffers in one pipelined call: each view chunk is uploaded, cosine-
// weighted and ramp filtered on the device, written back over the caller's projections (the
// reference's fbp leaves the filtered projections in its input), and backprojected (FDK)
// into the volume while the next chunk moves.
extern "C" int fcb_fbp_host(int device, const fcb_geometry* g, int window, float cosineD,
                            const float* zOrigin, int cosineWeight, float* projections, float* volume)
try {
  if (!projections) return set_error(FCB_ERR_INVALID, "NULL argument");
  if (cosineWeight && (!zOrigin || !(cosineD > 0.0f)))
    return set_error(FCB_ERR_INVALID, "cosine weighting needs D > 0 and zOrigin");
  if (window != FCB_FILTER_RAMLAK && window != FCB_FILTER_SHEPPLOGAN && window != FCB_FILTER_COSRAMP &&
      window != FCB_FILTER_GAUSSRAMP)
    return set_error(FCB_ERR_INVALID, "unknown filter window");
  FbpFilter ff{window, cosineD, zOrigin, cosineWeight ? 1 : 0, projections};
  return backproject_host_impl(device, g, FCB_MODE_FDK, projections, volume, &ff);
}
FCB_CATCH_STATUS

extern "C" int fcb_project_host(int device, const fcb_geometry* g, int method, const float* volume,
                                float* projections)
try {
  if (!g || !projections || !volume) return set_error(FCB_ERR_INVALID, "NULL argument");
  DeviceGuard guard(device);
  if (guard.rc) return guard.rc;
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  const size_t nvox = (size_t)(g->volEnd[0] - g->volStart[0]) * (g->volEnd[1] - g->volStart[1]) *
                      (g->volEnd[2] - g->volStart[2]);
  const size_t np = (size_t)g->projDim[2] * g->projWHSize[0] * g->projWHSize[1];
  Scratch sc;
  float *dvol = nullptr, *dproj = nullptr;
  FCB_TRY(sc.alloc((void**)&dvol, nvox * sizeof(float)));
  FCB_TRY(sc.alloc((void**)&dproj, np * sizeof(float)));
  cudaStream_t cs, xs;
  FCB_TRY(sc.stream(&cs));
  FCB_TRY(sc.stream(&xs));
  cudaEvent_t ev;
  FCB_TRY(sc.event(&ev));
  // pageable caller buffers (numpy arrays): pinned staging filled by host threads
  HostStager stager;
  const bool proj_pg = is_pageable(projections), vol_pg = is_pageable(volume);
  FCB_TRY(stager.init((proj_pg ? 2 * np * sizeof(float) : 0) + (vol_pg ? nvox * sizeof(float) : 0)));
  if (proj_pg && stager.ok)
    FCB_TRY(stager.h2d(dproj, projections, np * sizeof(float), xs));
  else
    FCB_CUDA_TRY(cudaMemcpyAsync(dproj, projections, np * sizeof(float), cudaMemcpyHostToDevice, xs));
  FCB_CUDA_TRY(cudaEventRecord(ev, xs));
  if (vol_pg && stager.ok)
    FCB_TRY(stager.h2d(dvol, volume, nvox * sizeof(float), cs));
  else
    FCB_CUDA_TRY(cudaMemcpyAsync(dvol, volume, nvox * sizeof(float), cudaMemcpyHostToDevice, cs));
  FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
  FCB_TRY(project_launch(pb, method, dvol, dproj, nullptr, nullptr, cs));
  if (proj_pg && stager.ok)
    FCB_TRY(stager.d2h(projections, dproj, np * sizeof(float), cs));
  else
    FCB_CUDA_TRY(cudaMemcpyAsync(projections, dproj, np * sizeof(float), cudaMemcpyDeviceToHost, cs));
  FCB_CUDA_TRY(cudaStreamSynchronize(cs));
  FCB_TRY(collect_device_status(cs));
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_release_device_cache(void)
try {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  cache_drop_locked(-1);
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_sync_status(void* stream)
try {
  FCB_TRY(collect_device_status(reinterpret_cast<cudaStream_t>(stream)));
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_last_status(void);
extern "C" const char* fcb_last_error(void);

// ------------------------------------------------------------ reference-compatible symbols
namespace {
fcb_geometry make_geom(float* angles, float* hMidPlane, float D, float pw, int volDim[3],
                       int volStart[3], int volEnd[3], int projDim[3], int projWHSize[2],
                       int* projWOffset, int* projHOffset, float* norm, float* mis)
{
  fcb_geometry g;
  memset(&g, 0, sizeof(g));
  for (int i = 0; i < 3; i++) {
    g.volDim[i] = volDim ? volDim[i] : 0;
    g.volStart[i] = volStart ? volStart[i] : 0;
    g.volEnd[i] = volEnd ? volEnd[i] : 0;
    g.projDim[i] = projDim ? projDim[i] : 0;
  }
  g.projWHSize[0] = projWHSize ? projWHSize[0] : 0;
  g.projWHSize[1] = projWHSize ? projWHSize[1] : 0;
  g.projWOffset = projWOffset;
  g.projHOffset = projHOffset;
  g.angles = angles;
  g.hMidPlane = hMidPlane;
  g.sourceSampleDistance = D;
  g.pixelWidth = pw;
  g.normalizationFactor = norm;
  g.misAlignments = mis;
  g.referenceWindows = 1;  // drop-in: reproduce the reference's windows where they matter
  return g;
}
}  // namespace

extern "C" void GPU_CB_K_backproject(int GPUID, float* volume, float* projections, float* angles,
                                     float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                                     int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                                     int projWHSize[2], int* projWOffset, int* projHOffset,
                                     float* normalizationFactor, int kernelMode)
{
  fcb_geometry g = make_geom(angles, hMidPlane, sourceSampleDistance, pixelWidth, volDim, volStart,
                             volEnd, projDim, projWHSize, projWOffset, projHOffset,
                             normalizationFactor, nullptr);
  fcb_backproject_host(GPUID, &g, kernelMode == 0 ? 0 : (kernelMode == 1 ? 1 : 2), projections,
                       volume);
}

extern "C" void GPU_CB_backproject(int GPUID, float* volume, float* projections, float* angles,
                                   float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                                   int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                                   int projWHSize[2], int* projWOffset, int* projHOffset,
                                   float* normalizationFactor)
{
  GPU_CB_K_backproject(GPUID, volume, projections, angles, hMidPlane, sourceSampleDistance,
                       pixelWidth, volDim, volStart, volEnd, projDim, projWHSize, projWOffset,
                       projHOffset, normalizationFactor, 2);
}

extern "C" void GPU_CB_misalign_backproject(int GPUID, float* volume, float* projections,
                                            float* angles, float* hMidPlane,
                                            float sourceSampleDistance, float pixelWidth,
                                            int volDim[3], int volStart[3], int volEnd[3],
                                            int projDim[3], int projWHSize[2], int* projWOffset,
                                            int* projHOffset, float* normalizationFactor,
                                            float* misAlignments)
{
  fcb_geometry g = make_geom(angles, hMidPlane, sourceSampleDistance, pixelWidth, volDim, volStart,
                             volEnd, projDim, projWHSize, projWOffset, projHOffset,
                             normalizationFactor, misAlignments);
  fcb_backproject_host(GPUID, &g, 0, projections, volume);
}

extern "C" void GPU_CB_misalign_project(int GPUID, float* volume, float* projections, float* angles,
                                        float* hMidPlane, float sourceSampleDistance,
                                        float pixelWidth, int volDim[3], int volStart[3],
                                        int volEnd[3], int projDim[3], int projWHSize[2],
                                        int* projWOffset, int* projHOffset,
                                        float* normalizationFactor, float* misAlignments)
{
  fcb_geometry g = make_geom(angles, hMidPlane, sourceSampleDistance, pixelWidth, volDim, volStart,
                             volEnd, projDim, projWHSize, projWOffset, projHOffset,
                             normalizationFactor, misAlignments);
  fcb_project_host(GPUID, &g, FCB_PROJ_TEXTURE, volume, projections);
}

extern "C" void GPU_CB_project(int GPUID, float* volume, float* projections, float* angles,
                               float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                               int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                               int projWHSize[2], int* projWOffset, int* projHOffset,
                               float* normalizationFactor)
{
  GPU_CB_misalign_project(GPUID, volume, projections, angles, hMidPlane, sourceSampleDistance,
                          pixelWidth, volDim, volStart, volEnd, projDim, projWHSize, projWOffset,
                          projHOffset, normalizationFactor, nullptr);
}
