// fcb_common.cpp -- error plumbing, per-device status word, FP64 geometry, TMA encoding.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "fcb_internal.h"

namespace fcb {

// ---------------------------------------------------------------------------- errors
static thread_local int t_status = FCB_OK;
static thread_local std::string t_msg;

int set_error(int code, const std::string& msg)
{
  t_status = code;
  t_msg = msg;
  return code;
}

int ok()
{
  t_status = FCB_OK;
  t_msg.clear();
  return FCB_OK;
}

// ------------------------------------------------------------------- device status
// The kernels' status words (and the small scratch of the plan pre-passes) live in a
// file-scope device array: every context that loads the library gets its own copy, zeroed
// when the module loads, so nothing is allocated and no address is cached across calls
// (a cached pointer would go stale when a device's primary context is reset and made
// again).  The address is looked up with the caller's device current, on every call.
static __device__ __align__(64) int g_status_words[16];

int device_status_ptr(int** p)
{
  void* a = nullptr;
  FCB_CUDA_TRY(cudaGetSymbolAddress(&a, g_status_words));
  *p = static_cast<int*>(a);
  return FCB_OK;
}

int collect_device_status(cudaStream_t stream)
{
  int* st = nullptr;
  FCB_TRY(device_status_ptr(&st));
  int h = 0;
  FCB_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, stream));
  FCB_CUDA_TRY(cudaStreamSynchronize(stream));
  if (h) {
    FCB_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(int), stream));
    FCB_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h & DEV_TIMEOUT)
      return set_error(FCB_ERR_TIMEOUT, "a bounded device-side wait timed out");
    return set_error(FCB_ERR_RANGE, "a kernel sample fell outside its staging window");
  }
  return FCB_OK;
}

// ---------------------------------------------------------------------- geometry
// FP64 version of the per-view construction of coneBeamGeometry::_calculateProblemGeometry
// (coneBeamGPU.cu:1672-1734): aligned source/detector, then misalignments Dw, Dh, Dl
// (pixels), Dphi, Dtheta, Dpsi (radians) applied in that order.
namespace {
struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double len(V3 a) { return sqrt(dot(a, a)); }
inline V3 nrm(V3 a) { return (1.0 / len(a)) * a; }
inline void put(double* o, V3 a)
{
  o[0] = a.x;
  o[1] = a.y;
  o[2] = a.z;
}
inline V3 get(const double* o) { return {o[0], o[1], o[2]}; }
}  // namespace

int make_problem(const fcb_geometry* g, Problem* pb)
{
  if (!g) return set_error(FCB_ERR_INVALID, "geometry is NULL");
  for (int i = 0; i < 3; i++) {
    pb->volDim[i] = g->volDim[i];
    pb->volStart[i] = g->volStart[i];
    pb->volEnd[i] = g->volEnd[i];
    pb->projDim[i] = g->projDim[i];
    if (g->volDim[i] <= 0 || g->volEnd[i] <= g->volStart[i] || g->projDim[i] <= 0)
      return set_error(FCB_ERR_INVALID, "non-positive volume/projection dimension");
  }
  pb->projWHSize[0] = g->projWHSize[0];
  pb->projWHSize[1] = g->projWHSize[1];
  if (g->projWHSize[0] <= 0 || g->projWHSize[1] <= 0)
    return set_error(FCB_ERR_INVALID, "non-positive projection window size");
  if (!g->angles || !g->hMidPlane || !g->normalizationFactor || !g->projWOffset || !g->projHOffset)
    return set_error(FCB_ERR_INVALID, "a per-view geometry array is NULL");
  if (!(g->sourceSampleDistance > 0.0f) || !(g->pixelWidth > 0.0f))
    return set_error(FCB_ERR_INVALID, "sourceSampleDistance and pixelWidth must be > 0");
  const int n = g->projDim[2];
  pb->nviews = n;
  pb->D = g->sourceSampleDistance;
  pb->pw = g->pixelWidth;
  pb->woff.assign(g->projWOffset, g->projWOffset + n);
  pb->hoff.assign(g->projHOffset, g->projHOffset + n);
  pb->angle.resize(n);
  pb->hmid.resize(n);
  pb->norm.resize(n);
  for (int t = 0; t < n; t++) {
    pb->angle[t] = g->angles[t];
    pb->hmid[t] = g->hMidPlane[t];
    pb->norm[t] = g->normalizationFactor[t];
  }
  pb->misaligned = false;
  for (int i = 0; i < 6; i++) {
    pb->mis[i] = g->misAlignments ? g->misAlignments[i] : 0.0;
    if (pb->mis[i] != 0.0) pb->misaligned = true;
  }
  pb->pitch = g->helicalPitch;
  pb->piWindow = g->piWindow;
  pb->referenceWindows = g->referenceWindows;
  pb->views.resize(n);
  const double D = pb->D, pw = pb->pw;
  const double* m = pb->mis;
  for (int t = 0; t < n; t++) {
    ViewGeom& v = pb->views[t];
    const double a = pb->angle[t];
    v.ca = cos(a);
    v.sa = sin(a);
    v.hmp = pb->hmid[t] - (double)(pb->volDim[2] / 2);
    V3 s = v3(-v.ca * D, -v.sa * D, v.hmp);
    V3 d = v3(0, 0, v.hmp);
    V3 h = v3(0, 0, pw);
    V3 w = v3(-pw * v.sa, pw * v.ca, 0);
    if (pb->misaligned) {
      d = d + m[0] * w;
      d = d + m[1] * h;
      d = d + m[2] * nrm(d - s);
      V3 whp = cross(w, h);
      h = len(h) * (cos(m[3]) * nrm(h) + sin(m[3]) * nrm(whp));
      whp = cross(w, h);
      w = len(w) * (cos(m[4]) * nrm(w) + sin(m[4]) * nrm(whp));
      whp = cross(w, h);
      V3 wnp = cross(w, whp), hnp = cross(h, whp);
      V3 w2 = len(w) * (cos(m[5]) * nrm(w) - sin(m[5]) * nrm(wnp));
      V3 h2 = len(h) * (cos(m[5]) * nrm(h) + sin(m[5]) * nrm(hnp));
      w = w2;
      h = h2;
    }
    put(v.s, s);
    put(v.d, d);
    put(v.w, w);
    put(v.h, h);
  }
  return FCB_OK;
}

void view_matrix(const Problem& pb, int t, double M[12], double* kappa)
{
  const ViewGeom& v = pb.views[t];
  V3 S = get(v.s), Dc = get(v.d), w = get(v.w), h = get(v.h);
  V3 n = cross(w, h);
  double c = dot(Dc - S, n);
  double g00 = dot(w, w), g01 = dot(w, h), g11 = dot(h, h);
  double det = g00 * g11 - g01 * g01;
  double i00 = g11 / det, i01 = -g01 / det, i11 = g00 / det;
  double kw = dot(w, S - Dc), kh = dot(h, S - Dc);
  V3 bw = c * w + kw * n, bh = c * h + kh * n;
  V3 Aw = i00 * bw + i01 * bh;
  V3 Ah = i01 * bw + i11 * bh;
  // local window index = detector index relative to the centre + projDim/2 - offset
  double cw = (double)(pb.projDim[0] / 2 - pb.woff[t]);
  double ch = (double)(pb.projDim[1] / 2 - pb.hoff[t]);
  V3 ru = Aw + cw * n, rv = Ah + ch * n;
  M[0] = ru.x; M[1] = ru.y; M[2] = ru.z; M[3] = -dot(ru, S);
  M[4] = rv.x; M[5] = rv.y; M[6] = rv.z; M[7] = -dot(rv, S);
  M[8] = n.x;  M[9] = n.y;  M[10] = n.z; M[11] = -dot(n, S);
  *kappa = pb.D * len(n);
}

// ---------------------------------------------------------------------- TMA
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

unsigned long long current_context_id()
{
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

static EncodeTiledFn get_encode()
{
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

int encode_tmap(CUtensorMap* map, CUtensorMapDataType dtype, int rank, void* base,
                const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box)
{
  EncodeTiledFn enc = get_encode();
  if (!enc) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  cuuint64_t d[5], st[4];
  cuuint32_t b[5], e[5];
  for (int i = 0; i < rank; i++) {
    d[i] = dims[i];
    b[i] = box[i];
    e[i] = 1;
    if (i + 1 < rank) st[i] = strides_bytes[i];
  }
  CUresult r = enc(map, dtype, rank, base, d, st, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[96];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d), rank %d", (int)r, rank);
    return set_error(FCB_ERR_CUDA, buf);
  }
  return FCB_OK;
}

int encode_tmap_3d(CUtensorMap* map, CUtensorMapDataType dtype, void* base, uint64_t d0,
                   uint64_t d1, uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes,
                   uint32_t b0, uint32_t b1, uint32_t b2)
{
  EncodeTiledFn enc = get_encode();
  if (!enc) return set_error(FCB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {stride1_bytes, stride2_bytes};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, dtype, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d): dims %llu %llu %llu box %u %u %u",
             (int)r, (unsigned long long)d0, (unsigned long long)d1, (unsigned long long)d2, b0,
             b1, b2);
    return set_error(FCB_ERR_CUDA, buf);
  }
  return FCB_OK;
}

}  // namespace fcb

extern "C" int fcb_last_status(void) { return fcb::t_status; }
extern "C" const char* fcb_last_error(void) { return fcb::t_msg.c_str(); }

// --------------------------------------------------------------- slab footprints
// Detector rows a sub-volume reaches in each view, for splitting one volume into z-slabs
// over several GPUs: the 8 corners of the interpolation support (voxel indices volStart - 1
// .. volEnd) through the view's projective map; a box in front of the source maps inside
// the hull of its corners' images.  Rows [lo, hi) are global detector rows; a view whose
// footprint misses the detector gets lo = hi = 0.
extern "C" int fcb_detector_rows(const fcb_geometry* g, int margin, int* rowLo, int* rowHi)
try {
  using namespace fcb;
  if (!rowLo || !rowHi || margin < 0) return set_error(FCB_ERR_INVALID, "bad detector-rows arguments");
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  const int W = pb.projDim[0], H = pb.projDim[1];
  double c[3][2];
  for (int a = 0; a < 3; a++) {
    c[a][0] = (double)(pb.volStart[a] - 1 - pb.volDim[a] / 2);
    c[a][1] = (double)(pb.volEnd[a] - pb.volDim[a] / 2);
  }
  for (int t = 0; t < pb.nviews; t++) {
    double M[12], kappa;
    view_matrix(pb, t, M, &kappa);
    double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
    bool behind = false;
    for (int k = 0; k < 8; k++) {
      const double x = c[0][k & 1], y = c[1][(k >> 1) & 1], z = c[2][(k >> 2) & 1];
      const double s = M[8] * x + M[9] * y + M[10] * z + M[11];
      if (!(s > 1e-9)) { behind = true; break; }
      const double u = (M[0] * x + M[1] * y + M[2] * z + M[3]) / s + pb.woff[t];
      const double v = (M[4] * x + M[5] * y + M[6] * z + M[7]) / s + pb.hoff[t];
      umin = std::min(umin, u); umax = std::max(umax, u);
      vmin = std::min(vmin, v); vmax = std::max(vmax, v);
    }
    if (behind) {
      rowLo[t] = 0;
      rowHi[t] = H;
      continue;
    }
    const double lo = std::floor(vmin) - margin, hi = std::floor(vmax) + 2 + margin;
    const double wl = std::floor(umin) - margin, wh = std::floor(umax) + 2 + margin;
    if (hi <= 0.0 || lo >= (double)H || wh <= 0.0 || wl >= (double)W) {
      rowLo[t] = rowHi[t] = 0;
      continue;
    }
    rowLo[t] = (int)std::max(0.0, lo);
    rowHi[t] = (int)std::min((double)H, hi);
  }
  return ok();
}
FCB_CATCH_STATUS
