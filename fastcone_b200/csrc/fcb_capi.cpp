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

// RAII bundle of device buffers/streams/events of one host-driver call.
struct Scratch {
  std::vector<void*> dev;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  ~Scratch()
  {
    for (cudaStream_t s : streams) cudaStreamSynchronize(s);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
    for (void* p : dev) cudaFree(p);
  }
  int alloc(void** p, size_t bytes)
  {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return set_error(FCB_ERR_NOMEM, "device allocation failed");
    }
    dev.push_back(*p);
    return FCB_OK;
  }
  int stream(cudaStream_t* s)
  {
    FCB_CUDA_TRY(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
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

// Host window views [v0, v1) -> device buffer rows padded to `wpad` floats.
int copy_proj_h2d(float* d, const float* h, int v0, int v1, int W, int H, int wpad, cudaStream_t s)
{
  const size_t rows = (size_t)(v1 - v0) * H;
  if (wpad == W) {
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

// Host-buffer backprojection, pipelined over view chunks and z-slabs of the volume:
//   copy-in stream : the first view chunk, the volume slab by slab, then the other chunks
//   compute stream : chunk by chunk as they arrive, each over all slabs (slab s of the first
//                    chunk as soon as slab s is in)
//   copy-out stream: slab s back to the host as soon as the last chunk has passed over it
// so the PCIe traffic (projections once, the volume in and out) hides behind the kernels
// except for the first chunk with the first slab, and the last slab.  One plan (one staging
// pre-pass) serves every slab: a slab is a range of the plan's z tiles.  Reference-compatible
// windows that change the result run as one slab (their tiling starts at volStart).
extern "C" int fcb_backproject_host(int device, const fcb_geometry* g0, int kernelMode,
                                    const float* projections, float* volume)
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
  std::vector<int> z0(nslab), z1(nslab);
  for (int s = 0; s < nslab; s++) {
    z0[s] = s * slab;
    z1[s] = std::min(nz, z0[s] + slab);
  }

  const size_t plane = (size_t)nx * ny;
  const size_t nvox = plane * nz;
  Scratch sc;
  float *dvol = nullptr, *dproj = nullptr;
  FCB_TRY(sc.alloc((void**)&dvol, nvox * sizeof(float)));
  FCB_TRY(sc.alloc((void**)&dproj, (size_t)n * H * wpad * sizeof(float)));
  const double t_alloc = tr.ms();
  cudaStream_t cs, xs, os;
  FCB_TRY(sc.stream(&cs));
  FCB_TRY(sc.stream(&xs));
  FCB_TRY(sc.stream(&os));
  if (wpad != W) FCB_CUDA_TRY(cudaMemsetAsync(dproj, 0, (size_t)n * H * wpad * sizeof(float), xs));
  auto zoff = [&](int s) { return (size_t)z0[s] * plane; };
  auto slab_bytes = [&](int s) { return (size_t)(z1[s] - z0[s]) * plane * sizeof(float); };
  cudaEvent_t ev;
  cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (tr.on)
    for (cudaEvent_t& e : tev) FCB_CUDA_TRY(cudaEventCreate(&e));
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[0], xs));

  const int nch = (int)ranges.size();
  for (int c = 0; c < nch; c++) {
    FCB_TRY(copy_proj_h2d(dproj, projections, ranges[c].first, ranges[c].second, W, H, wpad, xs));
    FCB_TRY(sc.event(&ev));
    FCB_CUDA_TRY(cudaEventRecord(ev, xs));
    FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
    for (int s = 0; s < nslab; s++) {
      if (c == 0) {
        FCB_CUDA_TRY(cudaMemcpyAsync(dvol + zoff(s), volume + zoff(s), slab_bytes(s),
                                     cudaMemcpyHostToDevice, xs));
        FCB_TRY(sc.event(&ev));
        FCB_CUDA_TRY(cudaEventRecord(ev, xs));
        FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
        if (s == 0 && tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[1], cs));
      }
      FCB_TRY(bp_plan_execute_range(plan, c, z0[s], z1[s], dproj, dvol, cs));
      if (c == nch - 1) {
        FCB_TRY(sc.event(&ev));
        FCB_CUDA_TRY(cudaEventRecord(ev, cs));
        FCB_CUDA_TRY(cudaStreamWaitEvent(os, ev, 0));
        FCB_CUDA_TRY(cudaMemcpyAsync(volume + zoff(s), dvol + zoff(s), slab_bytes(s),
                                     cudaMemcpyDeviceToHost, os));
      }
    }
  }
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[2], cs));
  if (tr.on) FCB_CUDA_TRY(cudaEventRecord(tev[3], os));
  FCB_CUDA_TRY(cudaStreamSynchronize(os));
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

extern "C" int fcb_project_host(int device, const fcb_geometry* g, int method, const float* volume,
                                float* projections)
{
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
  FCB_CUDA_TRY(cudaMemcpyAsync(dproj, projections, np * sizeof(float), cudaMemcpyHostToDevice, xs));
  FCB_CUDA_TRY(cudaEventRecord(ev, xs));
  FCB_CUDA_TRY(cudaMemcpyAsync(dvol, volume, nvox * sizeof(float), cudaMemcpyHostToDevice, cs));
  FCB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
  FCB_TRY(project_launch(pb, method, dvol, dproj, nullptr, nullptr, cs));
  FCB_CUDA_TRY(cudaMemcpyAsync(projections, dproj, np * sizeof(float), cudaMemcpyDeviceToHost, cs));
  FCB_CUDA_TRY(cudaStreamSynchronize(cs));
  FCB_TRY(collect_device_status(cs));
  return ok();
}

extern "C" int fcb_sync_status(void* stream)
{
  FCB_TRY(collect_device_status(reinterpret_cast<cudaStream_t>(stream)));
  return ok();
}

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
