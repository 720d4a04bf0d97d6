/*
 * fastcone_b200.h -- C ABI of libfastcone_b200.so, a B200 (sm_100a) cone-beam CT
 * projector / backprojector that is a drop-in for Fastcone's libFastcone.so.
 *
 * Conventions (identical to the reference ABI, wrapper.c:112-249):
 *   - dimension arrays are [x, y, z] for volumes and [w, h, t] for projections;
 *   - `volume` is the volStart..volEnd sub-array of a volDim grid, x fastest;
 *   - `projections` holds projDim[2] views of projWHSize[0] x projWHSize[1] windows,
 *     view t's window placed at (projWOffset[t], projHOffset[t]) of a
 *     projDim[0] x projDim[1] detector; values outside a window are zero;
 *   - voxel g sits at g - volDim/2 (integer division), detector pixel g at
 *     (g - projDim/2) * pixelWidth; the source of view t is at distance
 *     sourceSampleDistance from the rotation axis at angle angles[t], height
 *     hMidPlane[t] (measured from volume element 0);
 *   - both directions ACCUMULATE: backprojection adds into `volume`, projection adds
 *     norm[t] * (A vol) into `projections`; backprojection multiplies view t by norm[t].
 *
 * Errors: the reference's void entry points record a status retrievable with
 * fcb_last_status()/fcb_last_error() (thread-local); every other entry point returns it.
 * No entry point exits the process or resets the device context.
 */
#ifndef FASTCONE_B200_H
#define FASTCONE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define FCB_OK 0
#define FCB_ERR_INVALID 1   /* bad argument (sizes, pointers, mode) */
#define FCB_ERR_CUDA 2      /* a CUDA runtime/driver call failed */
#define FCB_ERR_NOMEM 3     /* device or pinned host allocation failed */
#define FCB_ERR_TIMEOUT 4   /* a bounded device-side wait gave up (kernel status word) */
#define FCB_ERR_NODEVICE 5  /* GPUID does not name a CUDA device */
#define FCB_ERR_RANGE 6     /* geometry outside what a kernel's staging window supports */
#define FCB_ERR_HOST 7      /* a host-side failure other than memory (e.g. a copy thread) */

/* projection storage types for the device entry points */
#define FCB_F32 0
#define FCB_F16 1
#define FCB_BF16 2

/* backprojection kernel modes (wrapper.c:134-143: 0 unweighted, 1 Katsevich, else FDK) */
#define FCB_MODE_UNWEIGHTED 0
#define FCB_MODE_KATSEVICH 1
#define FCB_MODE_FDK 2

/* forward projector variants */
#define FCB_PROJ_TEXTURE 0   /* hardware texture trilinear (8-bit weights, like the reference) */
#define FCB_PROJ_EXPLICIT 1  /* explicit FP32 trilinear from TMA-staged volume bricks (global-memory
                                reads where a brick does not apply); exact transpose is
                                fcb_project_adjoint_device */
#define FCB_PROJ_EXPLICIT_GLOBAL 2 /* the same samples and arithmetic (bit-identical results), every
                                      tap read from global memory: the unstaged comparison */

/* ramp-filter windows for fcb_fdk_filter_device / fcb_filter_plan_create */
#define FCB_FILTER_RAMLAK 0      /* fastcone.rampfilter, fastcone.py:272-292 */
#define FCB_FILTER_SHEPPLOGAN 1  /* the same with the sinc (Shepp-Logan) apodisation */
#define FCB_FILTER_COSRAMP 2     /* fastcone.cosrampfilter, fastcone.py:294-304: rows of length W
                                    unpadded, |f| * cos(0.5 |f| pi / W), applied to every view */
#define FCB_FILTER_GAUSSRAMP 3   /* fastcone.gaussrampfilter, fastcone.py:306-319: rows of length W
                                    unpadded, |f| times the half-Gaussian of sigma = scale * W
                                    (scale 1/8 unless fcb_filter_plan_create_ex sets it) */

int fcb_version(void);
int fcb_last_status(void);
const char* fcb_last_error(void);

/* ====================================================================================
 * Reference-compatible entry points: same symbols, argument order and semantics as the
 * definitions in wrapper.c (the order fastcone.py calls them in).  Host buffers.
 * ==================================================================================== */

/* wrapper.c:112-146 (declared wrapper.h:48-62) */
void GPU_CB_K_backproject(int GPUID, float* volume, float* projections, float* angles,
                          float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                          int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                          int projWHSize[2], int* projWOffset, int* projHOffset,
                          float* normalizationFactor, int kernelMode);

/* wrapper.c:177-194 (declared wrapper.h:34-45): FDK */
void GPU_CB_backproject(int GPUID, float* volume, float* projections, float* angles,
                        float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                        int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                        int projWHSize[2], int* projWOffset, int* projHOffset,
                        float* normalizationFactor);

/* wrapper.c:149-174 (declared wrapper.h:64-80): unweighted, misaligned detector */
void GPU_CB_misalign_backproject(int GPUID, float* volume, float* projections, float* angles,
                                 float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                                 int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                                 int projWHSize[2], int* projWOffset, int* projHOffset,
                                 float* normalizationFactor, float* misAlignments);

/* wrapper.c:203-227 (declared wrapper.h:82-95) */
void GPU_CB_misalign_project(int GPUID, float* volume, float* projections, float* angles,
                             float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                             int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                             int projWHSize[2], int* projWOffset, int* projHOffset,
                             float* normalizationFactor, float* misAlignments);

/* wrapper.c:229-249 (declared wrapper.h:97-109) */
void GPU_CB_project(int GPUID, float* volume, float* projections, float* angles,
                    float* hMidPlane, float sourceSampleDistance, float pixelWidth,
                    int volDim[3], int volStart[3], int volEnd[3], int projDim[3],
                    int projWHSize[2], int* projWOffset, int* projHOffset,
                    float* normalizationFactor);

/* ====================================================================================
 * Status-returning entry points.
 * ==================================================================================== */

/* Problem description shared by the device entry points.  All pointers are HOST
 * pointers to small per-view arrays (nviews = projDim[2]); misAlignments may be NULL. */
typedef struct fcb_geometry {
  int volDim[3];
  int volStart[3];
  int volEnd[3];
  int projDim[3];
  int projWHSize[2];
  const int* projWOffset;
  const int* projHOffset;
  const float* angles;
  const float* hMidPlane;
  float sourceSampleDistance;
  float pixelWidth;
  const float* normalizationFactor;
  const float* misAlignments;
  float helicalPitch; /* source z advance per 2*pi rad (voxels); Katsevich PI window only */
  int piWindow;       /* Katsevich: 1 = apply the Tam-Danielsson window, 0 = dense */
  /* 1 = reproduce the reference's sub-problem detector windows and projector sweeps
   * (coneBeamGPU.cu:1509-1609, :1757-1786) where they change a result -- the GPU_CB_*
   * entry points always do; 0 = the ideal operator (zero-extended data, full support). */
  int referenceWindows;
} fcb_geometry;

/* Host-buffer versions of GPU_CB_K_backproject / GPU_CB_misalign_project that return
 * the status.  Replaces unit_coneBeamGPU.cu:173-305 and :88-171.  Pinned (page-locked)
 * caller buffers are copied by DMA directly; pageable ones of 64 MB or more go through
 * three 64 MB pinned buffers that the library makes on the first such call and keeps until
 * the process exits (calls from several threads take turns on them). */
int fcb_backproject_host(int device, const fcb_geometry* g, int kernelMode,
                         const float* projections, float* volume);
int fcb_project_host(int device, const fcb_geometry* g, int method, const float* volume,
                     float* projections);

/* fastcone.fbp (fastcone.py:260-270) on host buffers in one pipelined call: each view chunk
 * of `projections` is uploaded, optionally cosine-weighted by
 * cosineD / sqrt(cosineD^2 + (h - zOrigin[t])^2 + (w - W/2)^2) (detector pixels), filtered
 * with `window` (FCB_FILTER_*, as fcb_fdk_filter_device), written back over `projections`
 * (the reference's fbp leaves the filtered projections in its input) and backprojected with
 * the FDK weight into `volume` (+=, g's normalisation) while the next chunk is in flight.
 * Same buffer rules as fcb_backproject_host. */
int fcb_fbp_host(int device, const fcb_geometry* g, int window, float cosineD, const float* zOrigin,
                 int cosineWeight, float* projections, float* volume);

/* Device-pointer versions, stream-ordered on `stream` (a cudaStream_t, NULL = legacy
 * default).  `proj` holds FCB_F32/F16/BF16 values with the layout above; `volume` is
 * float.  They return once the work is queued; a device-side failure is reported by
 * the next call on the same thread that synchronises (fcb_sync_status). */
int fcb_backproject_device(const fcb_geometry* g, int kernelMode, const void* proj, int projType,
                           float* volume, void* stream);
int fcb_project_device(const fcb_geometry* g, int method, const float* volume, float* proj,
                       void* stream);
int fcb_project_adjoint_device(const fcb_geometry* g, const float* proj, float* volume,
                               void* stream);
/* fcb_project_device that also adds the number of trilinear samples taken to the 64-bit
 * device counter *samples (the Gsamples work count of benchmarks). */
int fcb_project_device_counted(const fcb_geometry* g, int method, const float* volume,
                               float* proj, unsigned long long* samples, void* stream);

/* Reusable backprojection plan (geometry digested once: per-view parameters, staging
 * window sizes).  execute() is asynchronous and allocates nothing. */
typedef struct fcb_bp_plan fcb_bp_plan;
int fcb_bp_plan_create(const fcb_geometry* g, int kernelMode, int projType, fcb_bp_plan** plan);
int fcb_bp_plan_execute(fcb_bp_plan* plan, const void* proj, float* volume, void* stream);
int fcb_bp_plan_info(const fcb_bp_plan* plan, int* boxW, int* boxH, int* launches,
                     long long* voxelViewUpdates);
int fcb_bp_plan_destroy(fcb_bp_plan* plan);
/* Test hook for the device-side timeout path, no counterpart in the reference.  On a plan
 * that uses the staged kernel (boxW > 0), later executes stage only the first
 * `stopAfterViews` views of each launch (< 0: all, the default), drain their copies and
 * leave, and each consumer wait for a staged view gives up after consumerWaitNs
 * nanoseconds (0 < consumerWaitNs <= 2e9; the default is 2e9).  With stopAfterViews >= 0
 * the kernels therefore end early with FCB_ERR_TIMEOUT recorded (reported by
 * fcb_sync_status) and the volume partly updated; no copy is left in flight and the
 * context stays usable. */
int fcb_bp_plan_set_test_stall(fcb_bp_plan* plan, int stopAfterViews,
                               unsigned long long consumerWaitNs);

/* Exact number of voxel-view pairs of the geometry's sub-volume and views that lie inside
 * the Katsevich PI window (the Tam-Danielsson bounds of the FP64 oracle; helicalPitch != 0):
 * the work of the PI-window backprojection, for throughput figures.  FP64, on the GPU;
 * synchronous (allocates a per-view table and a counter).  No counterpart in the reference,
 * whose Katsevich kernel (coneBeamGPU.cu:258-338) has no window. */
int fcb_katsevich_pi_pairs(const fcb_geometry* g, long long* pairs, void* stream);

/* Same backprojection as fcb_backproject_device, for callers that cannot allocate device
 * memory while they run (GPU memory owned by another allocator or a fixed budget, or a
 * timing-critical loop that must not stop for an allocation).  No counterpart in the
 * reference.  It calls no cudaMalloc/cudaFree and no allocating library routine: its
 * device scratch -- the kernels' status word and the staging-box footprint maxima, 3 ints
 * -- lives in a static 256-byte device array (64 ints) that every GPU loading the library
 * holds until exit; the scratch need is fixed and checked against the array's size when the
 * library is compiled.  Every call looks up the array's device address on the current
 * device (the lookup allocates nothing).  All calls share the array and clear it at their
 * start, so calls whose GPU work overlaps (concurrent streams or threads) race on it.
 * Geometries whose reference-compatible windows change the result need a device window
 * table and are refused with FCB_ERR_INVALID.  The call is synchronous: it waits for
 * `stream` and returns the kernels' device-side status. */
int fcb_backproject_device_noalloc(const fcb_geometry* g, int kernelMode, const void* proj,
                                   int projType, float* volume, void* stream);

/* Reusable projector (per-view parameters digested once; the texture method keeps its 3-D
 * CUDA array and texture object with the plan).  execute() is stream-ordered, allocates
 * nothing and does not synchronise: adjoint == 0 adds norm * A volume into proj, adjoint != 0
 * adds A^T (norm * proj) into volume (explicit method only).  A texture plan must not run
 * on two streams at once (its array holds the volume being projected). */
typedef struct fcb_proj_plan fcb_proj_plan;
int fcb_proj_plan_create(const fcb_geometry* g, int method, fcb_proj_plan** plan);
int fcb_proj_plan_execute(fcb_proj_plan* plan, const float* volume, float* proj, int adjoint,
                          void* stream);
int fcb_proj_plan_destroy(fcb_proj_plan* plan);
/* staged = 1 when the plan's explicit projector runs on TMA-staged bricks of brickC (cross,
 * contiguous) x 13 (along the ray) x brickZ voxels in `stages` shared-memory buffers. */
int fcb_proj_plan_info(const fcb_proj_plan* plan, int* staged, int* brickC, int* brickZ,
                       int* stages);

/* Waits for `stream` and returns FCB_ERR_TIMEOUT / FCB_ERR_RANGE if a kernel of this
 * library recorded a device-side failure since the previous check, else FCB_OK. */
int fcb_sync_status(void* stream);

/* The host-buffer entry points (GPU_CB_*, fcb_backproject_host, fcb_project_host,
 * fcb_fbp_host) keep the device blocks of a finished call and reuse them in later calls
 * that fit (at most 8 blocks per device; a failed allocation first returns them), and
 * fcb_fbp_host keeps its filter plans (cuFFT plans and scratch, at most 4 per device).  This
 * returns everything kept to the driver.  FCB_HOST_CACHE=0 in the environment frees each
 * call's blocks and plans when it ends instead. */
int fcb_release_device_cache(void);

/* FDK pre-processing on the GPU (fastcone.py:260-292): optional cosine weight
 * D / sqrt(D^2 + (h - zOrigin[t])^2 + (w - W/2)^2) in detector pixels, then the ramp
 * filter of fastcone.rampfilter (zero-pad rows to 2W, pi*|f| with DC = 1/8 of the first
 * bin; FCB_FILTER_SHEPPLOGAN multiplies by sinc(f); FCB_FILTER_COSRAMP / GAUSSRAMP are the
 * unpadded apodised variants of fastcone.py:294-319), output stored as outType.
 * in: float [nviews][H][W] device; out: [nviews][H][W] of outType (may alias in when
 * outType == FCB_F32). */
int fcb_fdk_filter_device(const float* in, void* out, int outType, int nviews, int H, int W,
                          float D, const float* zOrigin, int cosineWeight, int window,
                          void* stream);

/* The same filter as a reusable plan: cuFFT plans, scratch and the filter response are made
 * once; execute is stream-ordered, allocates nothing and does not synchronise (zOrigin, host,
 * is read before it returns).  One execute at a time per plan (the scratch is the plan's). */
typedef struct fcb_filter_plan fcb_filter_plan;
int fcb_filter_plan_create(int nviews, int H, int W, int outType, int window,
                           fcb_filter_plan** plan);
/* As fcb_filter_plan_create; gaussScale is the Gaussian's sigma as a fraction of W for
 * FCB_FILTER_GAUSSRAMP (gaussrampfilter's `scale`, fastcone.py:306) and ignored otherwise. */
int fcb_filter_plan_create_ex(int nviews, int H, int W, int outType, int window,
                              double gaussScale, fcb_filter_plan** plan);
int fcb_filter_plan_execute(fcb_filter_plan* plan, const float* in, void* out, float D,
                            const float* zOrigin, int cosineWeight, void* stream);
int fcb_filter_plan_destroy(fcb_filter_plan* plan);

/* Katsevich filtering of helical projections (no counterpart in the reference, whose
 * Katsevich backprojection, coneBeamGPU.cu:258-338, expects pre-filtered data): derivative
 * at fixed ray direction, length correction, rebinning onto nkappa kappa-lines (<= 1: 2H),
 * Hilbert transform along u, backward rebinning (Noo, Pack & Heuscher 2003, flat detector
 * through the axis).  in/out: float [nviews][H][W] device, uniformly spaced host angles,
 * pitch = source rise per turn (voxels).  Backprojecting the output with
 * FCB_MODE_KATSEVICH, piWindow = 1 and norm = (angle step) / (2 pi D) reconstructs.
 * Synchronous (its scratch is freed before it returns). */
int fcb_katsevich_filter_device(const float* in, float* out, int nviews, int H, int W,
                                const float* angles, float D, float pw, float pitch, int nkappa,
                                void* stream);

/* The same filter as a reusable plan for one helix and detector: kappa-line tables, the
 * Hilbert kernel's spectrum, cuFFT plans and intermediate buffers made once (nviews x H x W
 * floats plus nviews x nkappa x 2W floats of zero-padded kappa rows, plus 0.5 GiB of transform
 * batches); execute is stream-ordered, allocates nothing
 * and does not synchronise.  One execute at a time per plan. */
typedef struct fcb_katsevich_plan fcb_katsevich_plan;
int fcb_katsevich_plan_create(int nviews, int H, int W, const float* angles, float D, float pw,
                              float pitch, int nkappa, fcb_katsevich_plan** plan);
int fcb_katsevich_plan_execute(fcb_katsevich_plan* plan, const float* in, float* out, void* stream);
int fcb_katsevich_plan_destroy(fcb_katsevich_plan* plan);

/* 3x3x3 convolution, 16 -> 16 channels, stride 1, zero padding 1, on the tcgen05 tensor
 * cores (BF16 inputs, FP32 accumulation).  Activations in the channel-half-major layout
 * [nz][ny][2][nx][8] (channel c of voxel (x,y,z) at ((z*ny + y)*2 + c/8)*nx*8 + x*8 + c%8).
 * x: BF16, w: BF16 [27 taps (dz,dy,dx) z-major][16 out][16 in], bias: 16 floats or NULL,
 * y: the same layout, of yType (FCB_F32 / FCB_BF16), ReLU applied when relu != 0.  Buffers
 * 16-byte aligned.  The input gradient is the same call with dY as x and
 * w'[t][ci][co] = w[26 - t][co][ci].  No counterpart in the reference (the learned
 * reconstruction is new). */
int fcb_conv3d16_device(const void* x, const void* w, const float* bias, void* y, int yType, int nx,
                        int ny, int nz, int relu, void* stream);

/* Weight gradient of fcb_conv3d16_device: dw[t][co][ci] += sum_v dy[v][co] x[v + tap t][ci]
 * (FP32, accumulated); dy of dyType (FCB_F32 / FCB_BF16), x BF16, both [nz][ny][2][nx][8].
 * BF16 dy runs on the tcgen05 tensor cores (16-byte aligned buffers; FP32 accumulation in
 * tensor memory, one FP32 atomic add per output and CTA), FP32 dy on the CUDA cores. */
int fcb_conv3d16_wgrad_device(const void* x, const void* dy, int dyType, float* dw, int nx, int ny,
                              int nz, void* stream);

/* Ellipsoid phantom voxelisation: vol[z][y][x] = sum of densities of ellipsoids
 * containing the voxel centre (g - volDim/2).  params: n x 16 doubles (host):
 * centre(3), semi-axes(3), row-major rotation R (9, body = R^T (p - c)), density. */
int fcb_phantom_device(float* vol, const int volDim[3], const double* params, int n,
                       void* stream);

/* The reference's sub-problem decomposition of a geometry, as restated here for
 * referenceWindows = 1 (coneBeamGeometry::_setupSubProblem and ::_calculateSweep,
 * coneBeamGPU.cu:1509-1609, :1757-1786): tile size subVolDim[3], window size subProjDim[2],
 * tile counts tiles[3] (x, y, z), and per [tile][view] (tile = (z * ty + y) * tx + x) the
 * window's first detector column / row and the projector's sweep start / steps; matters[0]
 * / [1] = 1 when the windows change the backprojection / the projection.  Host only (no
 * device work); any output may be NULL -- call with NULL arrays first to learn the tile
 * counts.  No counterpart in the reference, whose windows are internal. */
int fcb_reference_windows(const fcb_geometry* g, int* subVolDim, int* subProjDim, int* tiles,
                          int* ws, int* hs, int* sweepStart, int* sweepSteps, int* matters);

/* Per view t, the global detector rows [rowLo[t], rowHi[t]) that the sub-volume
 * volStart..volEnd (widened by one voxel: the interpolation support) projects to, widened by
 * `margin` rows and clipped to the detector; rowLo = rowHi = 0 where the footprint misses the
 * detector.  FP64, host only.  Used to split one volume into z-slabs over several GPUs:
 * each slab needs only these rows of each view (mpi_fastcone.py:450-526 moves whole
 * per-chunk detector windows between MPI ranks for the same purpose). */
int fcb_detector_rows(const fcb_geometry* g, int margin, int* rowLo, int* rowHi);

/* Measured ceiling for the staged kernels' rooflines, no counterpart in the reference:
 * conflict-free shared-memory loads of bytesPerLoad (4, 8 or 16) bytes per thread by two
 * 1024-thread CTAs per SM of the current device, 16 * iters loads per thread.  *ms = the
 * kernel's CUDA-event time on `stream`, *bytes = the bytes loaded.  Synchronous. */
int fcb_smem_bandwidth(int bytesPerLoad, long long iters, float* ms, double* bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif
