// fcb_project.cu -- ray-driven cone-beam forward projector and its exact adjoint (sm_100a).
//
// Replaces GPU_new_project_volume (coneBeamGPU.cu:96-176), its launcher (:493-563) and the
// problem solver coneBeamProject (unit_coneBeamGPU.cu:88-171).  Sample lattice as in the
// reference: points S + m d at every integer distance m (voxels) from the source along the
// unit ray direction d (the reference marches from the integer sweep start in unit steps,
// coneBeamGPU.cu:160-172, :1781-1782).  Instead of sweeping a bounding sphere the kernels
// clip each ray to the support of the trilinear interpolant (the volume box widened by one
// voxel, which is where the reference's zero ring lets samples contribute), so every
// sample they take is one the reference takes and empty space is skipped.
//
//  * FCB_PROJ_TEXTURE: trilinear sampling by the texture unit from a 3-D CUDA array with
//    border (zero) addressing -- the reference's interpolation, 8-bit weights included;
//  * FCB_PROJ_EXPLICIT: FP32 trilinear with exact weights from volume bricks staged in
//    shared memory by TMA (project_brick_kernel); its transpose project_adjoint_brick_kernel
//    accumulates in shared-memory bricks; <A x, y> = <x, A^T y> to rounding;
//  * FCB_PROJ_EXPLICIT_GLOBAL: the same samples and arithmetic with every tap read from
//    global memory (project_explicit_kernel; transpose project_adjoint_kernel, a direct
//    scatter), the unstaged comparison and the fallback where bricks do not apply.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {

constexpr int PJ_MAXV = 560;
struct PjView {
  float s[3];    // source, local continuous voxel-index coordinates
  float p0[3];   // centre of local pixel (0,0), same coordinates
  float w[3];    // one pixel step along w
  float h[3];    // one pixel step along h
  float wt;      // normalisation factor
};
struct PjParams {
  const float* vol;
  float* proj;
  unsigned long long* samples;  // optional work counter
  cudaTextureObject_t tex;
  int nx, ny, nz;               // local volume extents
  int WH0, WH1;                 // window size
  int nviews, view0;
  // reference-compatible sub-problems (project_ref_kernel only): win[tile * wviews + view]
  // = {first window column, first window row (data-local), sweep start, sweep steps}
  const int4* win;
  int sv0, sv1, sv2, ntx, nty, ntz, spd0, spd1, wviews;
  // TMA-brick projector (project_brick_kernel only): brick cross / z extents, stages,
  // bytes per stage (128-byte multiple), status word
  int BC, BZ, stages, stage_bytes;
  int* status;
  PjView v[PJ_MAXV];
};
static_assert(sizeof(PjParams) + 2 * sizeof(CUtensorMap) < 32000, "kernel parameter space");

// Integer sample range [m0, m1] of S + m d inside the open box (-1, n) per axis.
__device__ __forceinline__ bool ray_clip(const float s[3], const float d[3], int nx, int ny,
                                         int nz, int& m0, int& m1)
{
  float lo = -3.0e38f, hi = 3.0e38f;
  const float n[3] = {(float)nx, (float)ny, (float)nz};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (fabsf(d[a]) < 1e-12f) {
      if (!(s[a] > -1.0f && s[a] < n[a])) return false;
      continue;
    }
    const float inv = 1.0f / d[a];
    float t0 = (-1.0f - s[a]) * inv, t1 = (n[a] - s[a]) * inv;
    if (t0 > t1) { const float tt = t0; t0 = t1; t1 = tt; }
    lo = fmaxf(lo, t0);
    hi = fminf(hi, t1);
  }
  if (!(hi > lo)) return false;
  m0 = (int)ceilf(lo);
  m1 = (int)floorf(hi);
  return m1 >= m0;
}

__device__ __forceinline__ void ray_of(const PjView& V, int wl, int hl, float s[3], float d[3])
{
  float p[3], len2 = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    p[a] = fmaf((float)hl, V.h[a], fmaf((float)wl, V.w[a], V.p0[a]));
    d[a] = p[a] - V.s[a];
    s[a] = V.s[a];
    len2 = fmaf(d[a], d[a], len2);
  }
  const float r = rsqrtf(len2);
#pragma unroll
  for (int a = 0; a < 3; a++) d[a] *= r;
}

__device__ __forceinline__ void count_samples(unsigned long long* ctr, long long n)
{
  if (!ctr) return;
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if ((threadIdx.x & 31) == 0 && n) atomicAdd(ctr, (unsigned long long)n);
}

__global__ void __launch_bounds__(256) project_tex_kernel(const __grid_constant__ PjParams P)
{
  const int wl = blockIdx.x * 16 + (threadIdx.x & 15);
  const int hl = blockIdx.y * 16 + (threadIdx.x >> 4);
  const int v = blockIdx.z;
  long long cnt = 0;
  if (wl < P.WH0 && hl < P.WH1) {
    const PjView& V = P.v[v];
    float s[3], d[3];
    ray_of(V, wl, hl, s, d);
    int m0, m1;
    float acc = 0.0f;
    if (ray_clip(s, d, P.nx, P.ny, P.nz, m0, m1)) {
      cnt = m1 - m0 + 1;
      // texel centres sit at index + 0.5
      const float bx = s[0] + 0.5f, by = s[1] + 0.5f, bz = s[2] + 0.5f;
      for (int m = m0; m <= m1; m++) {
        const float mf = (float)m;
        acc += tex3D<float>(P.tex, fmaf(mf, d[0], bx), fmaf(mf, d[1], by), fmaf(mf, d[2], bz));
      }
    }
    P.proj[((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl] += V.wt * acc;
  }
  count_samples(P.samples, cnt);
}

struct Tri {
  int i, j, k;
  float a, b, c;
};
// Cell and fractions of a sample position.  Floors by the round-down magic number: for
// |a| < 2^22, a + 1.5 * 2^23 rounded toward -inf is an integer whose bits hold
// 0x4B400000 + floor(a), and (a + M) - M == floorf(a) exactly, so the fractions a - floor(a)
// are the FP32 values floorf would give (sample positions lie within a voxel of the volume).
__device__ __forceinline__ Tri tri_of(float x, float y, float z)
{
  Tri t;
  const float M = 12582912.0f;
  const float tx = __fadd_rd(x, M), ty = __fadd_rd(y, M), tz = __fadd_rd(z, M);
  t.i = __float_as_int(tx) - 0x4B400000;
  t.j = __float_as_int(ty) - 0x4B400000;
  t.k = __float_as_int(tz) - 0x4B400000;
  t.a = x - (tx - M); t.b = y - (ty - M); t.c = z - (tz - M);
  return t;
}

// Trilinear interpolation with zero outside the volume, always in the same FP32 lerp order
// (x, then y, then z) so that every kernel that takes a sample computes it identically.
__device__ __forceinline__ float tri_lerp(const Tri& t, float v000, float v100, float v010,
                                          float v110, float v001, float v101, float v011,
                                          float v111)
{
  const float x00 = fmaf(t.a, v100 - v000, v000), x10 = fmaf(t.a, v110 - v010, v010);
  const float x01 = fmaf(t.a, v101 - v001, v001), x11 = fmaf(t.a, v111 - v011, v011);
  const float y0 = fmaf(t.b, x10 - x00, x00), y1 = fmaf(t.b, x11 - x01, x01);
  return fmaf(t.c, y1 - y0, y0);
}

__device__ __forceinline__ float tri_fetch(const float* __restrict__ vol, int nx, int ny, int nz,
                                           const Tri& t)
{
  const size_t sx = 1, sy = nx, sz = (size_t)nx * ny;
  if (t.i >= 0 && t.j >= 0 && t.k >= 0 && t.i + 1 < nx && t.j + 1 < ny && t.k + 1 < nz) {
    const float* p = vol + t.i * sx + t.j * sy + t.k * sz;
    return tri_lerp(t, __ldg(p), __ldg(p + sx), __ldg(p + sy), __ldg(p + sx + sy), __ldg(p + sz),
                    __ldg(p + sx + sz), __ldg(p + sy + sz), __ldg(p + sx + sy + sz));
  }
  float v[8];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int X = t.i + (q & 1), Y = t.j + ((q >> 1) & 1), Z = t.k + ((q >> 2) & 1);
    const bool in = X >= 0 && Y >= 0 && Z >= 0 && X < nx && Y < ny && Z < nz;
    v[q] = in ? __ldg(vol + X * sx + Y * sy + Z * sz) : 0.0f;
  }
  return tri_lerp(t, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]);
}

__global__ void __launch_bounds__(256) project_explicit_kernel(const __grid_constant__ PjParams P)
{
  const int wl = blockIdx.x * 16 + (threadIdx.x & 15);
  const int hl = blockIdx.y * 16 + (threadIdx.x >> 4);
  const int v = blockIdx.z;
  long long cnt = 0;
  if (wl < P.WH0 && hl < P.WH1) {
    const PjView& V = P.v[v];
    float s[3], d[3];
    ray_of(V, wl, hl, s, d);
    int m0, m1;
    float acc = 0.0f;
    if (ray_clip(s, d, P.nx, P.ny, P.nz, m0, m1)) {
      cnt = m1 - m0 + 1;
      for (int m = m0; m <= m1; m++) {
        const float mf = (float)m;
        const Tri t = tri_of(fmaf(mf, d[0], s[0]), fmaf(mf, d[1], s[1]), fmaf(mf, d[2], s[2]));
        acc += tri_fetch(P.vol, P.nx, P.ny, P.nz, t);
      }
    }
    P.proj[((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl] += V.wt * acc;
  }
  count_samples(P.samples, cnt);
}

// ------------------------------------------------------------------ TMA-brick projector
// Explicit FP32 trilinear sampling from volume bricks staged in shared memory by TMA.
// A CTA owns a bundle of 32 x 8 rays (detector pixels) of one view.  Its rays share the
// source, so the bundle is a thin frustum; the CTA walks it along the dominant axis of its
// central ray (x or y) in slabs of T planes (12, or 8 where the brick would otherwise keep
// occupancy low), and a producer warp stages, per slab, the
// brick of voxels the frustum can touch there -- T + 1 dominant planes x BC cross
// voxels x BZ z-planes -- with one 3-D TMA load (zero fill outside the volume) into a ring
// of `stages` buffers.  Eight consumer warps (one detector row each, lanes along the row)
// then take every sample of their ray inside the slab from shared memory.  For x-dominant
// bundles the bricks come from a y-fastest copy of the volume, so that in both cases the
// lanes of a warp walk along the brick's contiguous axis (no bank conflicts).
//
// Sample positions, weights and the order of the FP32 operations are those of
// project_explicit_kernel (tri_of / tri_lerp), so the two kernels agree bit for bit: taps
// outside the volume are the bricks' zero fill (tri_fetch reads zeros there too), and a
// sample whose taps are not inside the staged brick is taken from global memory by
// tri_fetch itself.
constexpr int PB_W = 32, PB_H = 8;              // rays per CTA: 32 pixels x 8 rows
constexpr int PB_CWARPS = PB_H;                 // one consumer warp per detector row
constexpr int PB_THREADS = (PB_CWARPS + 1) * 32;

struct Bundle {
  float s[3];     // source (local voxel-index coordinates)
  float d[4][3];  // unit directions of the bundle's four corner rays
  int xdom;       // 1: x is the dominant axis, bricks from the y-fastest copy
  int sgn;        // direction of travel along the dominant axis (+1 / -1)
};

__device__ __forceinline__ void bundle_of(const PjView& V, int bw0, int bh0, Bundle& B)
{
  float c[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    float s[3], d[3];
    ray_of(V, bw0 + (q & 1) * (PB_W - 1), bh0 + (q >> 1) * (PB_H - 1), s, d);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      B.d[q][a] = d[a];
      B.s[a] = s[a];
      c[a] += d[a];
    }
  }
  B.xdom = fabsf(c[0]) >= fabsf(c[1]) ? 1 : 0;
  B.sgn = (B.xdom ? c[0] : c[1]) > 0.0f ? 1 : -1;
}

// Brick of the slab whose samples have floor(dominant) in [a, a + T - 1]: the frustum's
// cross / z range between the dominant planes a and a + T (clipped to [lo, hi]), plus
// the +1 trilinear neighbour; the cross origin is aligned down to 4 voxels (16-byte TMA rule).
template <int T>
__device__ __forceinline__ void brick_extent(const Bundle& B, int a, float lo, float hi, int& c0,
                                             int& z0, int& needc, int& needz)
{
  // (selects instead of runtime array indices keep everything in registers)
  const bool xd = B.xdom != 0;
  const float sD = xd ? B.s[0] : B.s[1], sC = xd ? B.s[1] : B.s[0];
  float cmin = 3.0e38f, cmax = -3.0e38f, zmin = 3.0e38f, zmax = -3.0e38f;
  const float p0 = fmaxf((float)a, lo), p1 = fminf((float)(a + T), hi);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float dD = xd ? B.d[q][0] : B.d[q][1], dC = xd ? B.d[q][1] : B.d[q][0];
    const float inv = 1.0f / dD;
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const float t = ((e ? p1 : p0) - sD) * inv;
      const float c = fmaf(t, dC, sC), z = fmaf(t, B.d[q][2], B.s[2]);
      cmin = fminf(cmin, c); cmax = fmaxf(cmax, c);
      zmin = fminf(zmin, z); zmax = fmaxf(zmax, z);
    }
  }
  cmin = fminf(fmaxf(cmin, -1.0e6f), 1.0e6f); cmax = fminf(fmaxf(cmax, -1.0e6f), 1.0e6f);
  zmin = fminf(fmaxf(zmin, -1.0e6f), 1.0e6f); zmax = fminf(fmaxf(zmax, -1.0e6f), 1.0e6f);
  c0 = __float2int_rd(cmin) & ~3;
  z0 = __float2int_rd(zmin);
  needc = __float2int_rd(cmax) + 2 - c0;
  needz = __float2int_rd(zmax) + 2 - z0;
}

// Pre-pass: the largest brick over every (view, bundle, slab start) sizes the staged box.
template <int T>
__global__ void project_brick_extent_kernel(const __grid_constant__ PjParams P, int bx, int by,
                                            int* out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)P.nviews * bx * by;
  int mc = 0, mz = 0;
  if (i < total) {
    const int v = (int)(i / ((long long)bx * by));
    const int b = (int)(i % ((long long)bx * by));
    Bundle B;
    bundle_of(P.v[v], (b % bx) * PB_W, (b / bx) * PB_H, B);
    const int ndom = B.xdom ? P.nx : P.ny;
    for (int a = -T; a <= ndom; a++) {
      int c0, z0, nc, nz;
      brick_extent<T>(B, a, -1.0f, (float)ndom, c0, z0, nc, nz);
      mc = max(mc, nc);
      mz = max(mz, nz);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mc = max(mc, __shfl_xor_sync(0xffffffffu, mc, o));
    mz = max(mz, __shfl_xor_sync(0xffffffffu, mz, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, mc);
    atomicMax(out + 1, mz);
  }
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two samples of one ray per instruction, each
// lane doing exactly the scalar operation of tri_of / tri_lerp.
typedef unsigned long long pj_u64;
__device__ __forceinline__ pj_u64 pj_pk(float lo, float hi)
{
  pj_u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void pj_up(pj_u64 v, float& lo, float& hi)
{
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ pj_u64 pj_sub(pj_u64 a, pj_u64 b)
{
  pj_u64 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ pj_u64 pj_fma(pj_u64 a, pj_u64 b, pj_u64 c)
{
  pj_u64 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
// lerp of both lanes: a + t (b - a), as fmaf(t, b - a, a)
__device__ __forceinline__ pj_u64 pj_lerp(pj_u64 t, pj_u64 a, pj_u64 b) { return pj_fma(t, pj_sub(b, a), a); }
// a + b rounded toward -inf in both lanes: with b = 1.5 * 2^23 the result's bits hold
// floor(a) (|a| < 2^22), and (a + b) - b == floorf(a) exactly
__device__ __forceinline__ pj_u64 pj_add_rm(pj_u64 a, pj_u64 b)
{
  pj_u64 r;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

__device__ __forceinline__ float lds32(uint32_t a)
{
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// The consumer side of one bundle: every sample of this thread's ray, slab by slab, from the
// staged bricks.  XD: x is the dominant axis (bricks of the y-fastest copy: the brick's
// contiguous axis is y, its middle axis x).  Returns the ray sum; a timed-out wait records
// the status and returns what was summed (the caller's store then carries a partial sum
// that the status flags).
template <bool XD, int T>
__device__ __forceinline__ float brick_consume(const PjParams& P, unsigned char* smem_raw,
                                               uint64_t* full, uint64_t* empty, const int4* origin,
                                               int nsl, int sgn, const float s[3], const float d[3],
                                               int m0, int m1)
{
  const int lane = threadIdx.x & 31;
  const uint32_t sbase = dev::smem_u32(smem_raw);
  const uint32_t rowb = (uint32_t)P.BC * 4u, planeb = rowb * (uint32_t)(T + 1);
  const uint32_t ox = XD ? rowb : 4u, oy = XD ? 4u : rowb;
  const int BC1 = P.BC - 1, BZ1 = P.BZ - 1;
  // floors by the round-down magic number: bits(a + 1.5 * 2^23) = MAGIC_BITS + floor(a)
  const float MAGIC = 12582912.0f;
  const int MAGIC_BITS = 0x4B400000;
  const pj_u64 MAG2 = pj_pk(MAGIC, MAGIC);
  const pj_u64 D0 = pj_pk(d[0], d[0]), D1 = pj_pk(d[1], d[1]), D2 = pj_pk(d[2], d[2]);
  const pj_u64 S0 = pj_pk(s[0], s[0]), S1 = pj_pk(s[1], s[1]), S2 = pj_pk(s[2], s[2]);
  const float sD = XD ? s[0] : s[1], dD = XD ? d[0] : d[1];  // along the dominant axis
  float acc = 0.0f;
  int m = m0;
  for (int k = 0; k < nsl; k++) {
    const int st = k % P.stages;
    // warp-uniform outcome, so the warp-wide operations below stay converged
    if (!__all_sync(0xffffffffu, dev::mbar_wait(&full[st], (k / P.stages) & 1))) {
      dev::record_status(P.status, DEV_TIMEOUT);
      return acc;
    }
    const int4 o = origin[st];
    const int alo = o.y, ahi = o.y + T - 1;
    // brick-local indices straight from the magic-number bits
    const int offC = MAGIC_BITS + o.x, offD = MAGIC_BITS + alo, offZ = MAGIC_BITS + o.z;
    const uint32_t stb = sbase + (uint32_t)st * (uint32_t)P.stage_bytes;
    // one sample from the staged brick, or from global memory when its taps leave the brick
    auto single = [&](int q) -> float {
      const float mf = (float)q;
      const Tri t = tri_of(fmaf(mf, d[0], s[0]), fmaf(mf, d[1], s[1]), fmaf(mf, d[2], s[2]));
      const int ic = (XD ? t.j : t.i) - o.x, id = (XD ? t.i : t.j) - alo, iz = t.k - o.z;
      if ((unsigned)ic < (unsigned)BC1 && (unsigned)id < (unsigned)T && (unsigned)iz < (unsigned)BZ1) {
        // taps outside the volume are the brick's zero fill
        const uint32_t p = stb + (uint32_t)iz * planeb + (uint32_t)id * rowb + (uint32_t)ic * 4u;
        return tri_lerp(t, lds32(p), lds32(p + ox), lds32(p + oy), lds32(p + ox + oy), lds32(p + planeb),
                        lds32(p + planeb + ox), lds32(p + planeb + oy), lds32(p + planeb + ox + oy));
      }
      return tri_fetch(P.vol, P.nx, P.ny, P.nz, t);
    };
    // The ray's last sample in this slab.  Samples advance along the dominant axis in the
    // bundle's direction, so sample q is in the slab until its dominant floor (the same fmaf
    // and floor as the sample's own position) passes the slab's far plane: estimate the
    // crossing, then step to the exact sample.
    int mend = m - 1;
    if (m <= m1) {
      auto inside = [&](int q) {
        const int f = __float_as_int(__fadd_rd(fmaf((float)q, dD, sD), MAGIC)) - MAGIC_BITS;
        return sgn > 0 ? f <= ahi : f >= alo;
      };
      const float cross = __fdividef((float)(sgn > 0 ? ahi + 1 : alo) - sD, dD);
      int me = (int)fminf(fmaxf(floorf(cross), (float)(m - 1)), (float)m1);
      while (me + 1 <= m1 && inside(me + 1)) me++;
      while (me >= m && !inside(me)) me--;
      mend = me;
    }
    for (; m + 1 <= mend; m += 2) {
      // samples m and m+1 in f32x2 lanes, when both have their taps inside the brick
      const pj_u64 mm = pj_pk((float)m, (float)(m + 1));
      const pj_u64 X = pj_fma(mm, D0, S0), Y = pj_fma(mm, D1, S1), Z = pj_fma(mm, D2, S2);
      const pj_u64 TX = pj_add_rm(X, MAG2), TY = pj_add_rm(Y, MAG2), TZ = pj_add_rm(Z, MAG2);
      float tx0, tx1, ty0, ty1, tz0, tz1;
      pj_up(TX, tx0, tx1);
      pj_up(TY, ty0, ty1);
      pj_up(TZ, tz0, tz1);
      const int c0 = __float_as_int(XD ? ty0 : tx0) - offC, c1 = __float_as_int(XD ? ty1 : tx1) - offC;
      const int e0 = __float_as_int(XD ? tx0 : ty0) - offD, e1 = __float_as_int(XD ? tx1 : ty1) - offD;
      const int q0 = __float_as_int(tz0) - offZ, q1 = __float_as_int(tz1) - offZ;
      if ((unsigned)c0 < (unsigned)BC1 && (unsigned)e0 < (unsigned)T && (unsigned)q0 < (unsigned)BZ1 &&
          (unsigned)c1 < (unsigned)BC1 && (unsigned)e1 < (unsigned)T && (unsigned)q1 < (unsigned)BZ1) {
        // fractions a - floorf(a), the same FP32 operation as tri_of
        const pj_u64 ta = pj_sub(X, pj_sub(TX, MAG2));
        const pj_u64 tb = pj_sub(Y, pj_sub(TY, MAG2));
        const pj_u64 tc = pj_sub(Z, pj_sub(TZ, MAG2));
        const uint32_t p0 = stb + (uint32_t)q0 * planeb + (uint32_t)e0 * rowb + (uint32_t)c0 * 4u;
        const uint32_t p1 = stb + (uint32_t)q1 * planeb + (uint32_t)e1 * rowb + (uint32_t)c1 * 4u;
        const pj_u64 v000 = pj_pk(lds32(p0), lds32(p1));
        const pj_u64 v100 = pj_pk(lds32(p0 + ox), lds32(p1 + ox));
        const pj_u64 v010 = pj_pk(lds32(p0 + oy), lds32(p1 + oy));
        const pj_u64 v110 = pj_pk(lds32(p0 + ox + oy), lds32(p1 + ox + oy));
        const pj_u64 v001 = pj_pk(lds32(p0 + planeb), lds32(p1 + planeb));
        const pj_u64 v101 = pj_pk(lds32(p0 + planeb + ox), lds32(p1 + planeb + ox));
        const pj_u64 v011 = pj_pk(lds32(p0 + planeb + oy), lds32(p1 + planeb + oy));
        const pj_u64 v111 = pj_pk(lds32(p0 + planeb + ox + oy), lds32(p1 + planeb + ox + oy));
        const pj_u64 x00 = pj_lerp(ta, v000, v100), x10 = pj_lerp(ta, v010, v110);
        const pj_u64 x01 = pj_lerp(ta, v001, v101), x11 = pj_lerp(ta, v011, v111);
        const pj_u64 yy0 = pj_lerp(tb, x00, x10), yy1 = pj_lerp(tb, x01, x11);
        float r0, r1;
        pj_up(pj_lerp(tc, yy0, yy1), r0, r1);
        acc += r0;
        acc += r1;
      } else {
        acc += single(m);
        acc += single(m + 1);
      }
    }
    if (m <= mend) {
      acc += single(m);
      m++;
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty[st]);
  }
  return acc;
}

template <int MINB, int T>
__global__ void __launch_bounds__(PB_THREADS, MINB) project_brick_kernel(
    const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmT,
    const __grid_constant__ PjParams P)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + (size_t)P.stages * P.stage_bytes);
  uint64_t* empty = full + P.stages;
  int4* origin = reinterpret_cast<int4*>(empty + P.stages);
  int* range = reinterpret_cast<int*>(origin + P.stages);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int v = blockIdx.z;
  const PjView& V = P.v[v];
  const int bw0 = blockIdx.x * PB_W, bh0 = blockIdx.y * PB_H;
  Bundle B;
  bundle_of(V, bw0, bh0, B);
  const bool xd = B.xdom != 0;
  const int ndom = xd ? P.nx : P.ny;

  if (threadIdx.x == 0) {
    for (int st = 0; st < P.stages; st++) {
      dev::mbar_init(&full[st], 1);
      dev::mbar_init(&empty[st], PB_CWARPS);
    }
    range[0] = 0x7fffffff;
    range[1] = -0x7fffffff;
    dev::fence_mbar_init();
  }
  __syncthreads();

  // each consumer thread: its ray, clipped to the interpolant's support
  float s[3], d[3];
  int m0 = 1, m1 = 0;
  const int wl = bw0 + lane, hl = bh0 + warp;
  const bool pix = warp < PB_CWARPS && wl < P.WH0 && hl < P.WH1;
  if (pix) {
    ray_of(V, wl, hl, s, d);
    if (ray_clip(s, d, P.nx, P.ny, P.nz, m0, m1)) {
      const float sD = xd ? s[0] : s[1], dD = xd ? d[0] : d[1];
      const int f0 = (int)floorf(fmaf((float)m0, dD, sD));
      const int f1 = (int)floorf(fmaf((float)m1, dD, sD));
      atomicMin(&range[0], min(f0, f1));
      atomicMax(&range[1], max(f0, f1));
    } else {
      m0 = 1;
      m1 = 0;
    }
  }
  __syncthreads();
  const int fmin = range[0], fmax = range[1];
  const int nsl = fmax >= fmin ? (fmax - fmin) / T + 1 : 0;

  if (warp == PB_CWARPS) {
    // ------------------------------------------------------------- producer warp
    if (lane != 0) return;
    const CUtensorMap* tm = B.xdom ? &tmT : &tmV;
    dev::tma_prefetch(tm);
    const uint32_t bytes = (uint32_t)(P.BC * (T + 1) * P.BZ * 4);
    int issued = 0;
    bool failed = false;
    for (int k = 0; k < nsl; k++) {
      const int st = k % P.stages;
      if (k >= P.stages && !dev::mbar_wait(&empty[st], ((k / P.stages) - 1) & 1)) {
        failed = true;
        break;
      }
      const int a = B.sgn > 0 ? fmin + k * T : fmax - T + 1 - k * T;
      int c0, z0, nc, nz;
      brick_extent<T>(B, a, -1.0f, (float)ndom, c0, z0, nc, nz);
      origin[st] = make_int4(c0, a, z0, 0);
      dev::mbar_arrive_expect_tx(&full[st], bytes);
      dev::tma_load_3d(smem_raw + (size_t)st * P.stage_bytes, tm, &full[st], c0, a, z0);
      issued = k + 1;
    }
    if (failed) {
      dev::record_status(P.status, DEV_TIMEOUT);
      for (int k = max(0, issued - P.stages); k < issued; k++)
        dev::mbar_wait(&full[k % P.stages], (k / P.stages) & 1, 100000000ull);
    }
    return;
  }

  // --------------------------------------------------------------- consumer warps
  const float acc = xd ? brick_consume<true, T>(P, smem_raw, full, empty, origin, nsl, B.sgn, s, d, m0, m1)
                       : brick_consume<false, T>(P, smem_raw, full, empty, origin, nsl, B.sgn, s, d, m0, m1);
  if (pix) P.proj[((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl] += V.wt * acc;
  count_samples(P.samples, m1 - m0 + 1);
}

// Transpose of the brick projector, A^T: the same bundles, slabs and samples; each sample's
// eight weighted taps are added into a shared-memory brick (shared atomics, many rays meet
// in a voxel) and the brick is then added to global memory once per slab (only its nonzero
// voxels, contiguous along the brick's inner axis).  x-dominant bundles accumulate into a
// y-fastest buffer `volT` that transpose_add_kernel folds into the volume afterwards, so
// both orientations flush coalesced.  Samples whose taps leave the brick scatter straight
// to global memory.  Weights are those of project_adjoint_kernel; the pair with the brick
// projector passes the dot-product test to rounding.
template <int MINB, int T>
__global__ void __launch_bounds__(256, MINB) project_adjoint_brick_kernel(const __grid_constant__ PjParams P,
                                                                          float* vol, float* volT, int vec4)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* brick = reinterpret_cast<float*>(smem_raw);
  const int nb = P.BC * (T + 1) * P.BZ;
  int* range = reinterpret_cast<int*>(smem_raw + (size_t)nb * 4);
  int4* org = reinterpret_cast<int4*>(range + 4);
  int* box = reinterpret_cast<int*>(org + 1);  // cells touched in the slab: c, d, z min / max
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int v = blockIdx.z;
  const PjView& V = P.v[v];
  const int bw0 = blockIdx.x * PB_W, bh0 = blockIdx.y * PB_H;
  Bundle B;
  bundle_of(V, bw0, bh0, B);
  const bool xd = B.xdom != 0;
  const int ndom = xd ? P.nx : P.ny;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  for (int e = threadIdx.x; e < nb; e += blockDim.x) brick[e] = 0.0f;
  if (threadIdx.x == 0) {
    range[0] = 0x7fffffff;
    range[1] = -0x7fffffff;
  }
  __syncthreads();

  float s[3], d[3];
  int m0 = 1, m1 = 0;
  float y = 0.0f;
  // rays of a warp at least two pixels apart (one parity class of a 32 x 4 block): at the
  // same step their taps rarely share a voxel, so one shared atomic instruction rarely
  // serialises on an address
  const int pc = warp & 3, rg = warp >> 2;
  const int wl = bw0 + 2 * (lane & 15) + (pc & 1), hl = bh0 + 4 * rg + 2 * (lane >> 4) + (pc >> 1);
  if (wl < P.WH0 && hl < P.WH1) {
    y = V.wt * __ldg(P.proj + ((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl);
    ray_of(V, wl, hl, s, d);
    if (y != 0.0f && ray_clip(s, d, nx, ny, nz, m0, m1)) {
      const float sD = xd ? s[0] : s[1], dD = xd ? d[0] : d[1];
      const int f0 = (int)floorf(fmaf((float)m0, dD, sD));
      const int f1 = (int)floorf(fmaf((float)m1, dD, sD));
      atomicMin(&range[0], min(f0, f1));
      atomicMax(&range[1], max(f0, f1));
    } else {
      m0 = 1;
      m1 = 0;
    }
  }
  __syncthreads();
  const int fmin = range[0], fmax = range[1];
  const int nsl = fmax >= fmin ? (fmax - fmin) / T + 1 : 0;
  const size_t sy = nx, sz = (size_t)nx * ny;
  int m = m0;
  for (int k = 0; k < nsl; k++) {
    const int a = B.sgn > 0 ? fmin + k * T : fmax - T + 1 - k * T;
    if (threadIdx.x == 0) {
      int c0, z0, nc, nzz;
      brick_extent<T>(B, a, -1.0f, (float)ndom, c0, z0, nc, nzz);
      org[0] = make_int4(c0, a, z0, 0);
      box[0] = box[2] = box[4] = INT_MAX;
      box[1] = box[3] = box[5] = INT_MIN;
    }
    __syncthreads();
    const int4 o = org[0];
    const int alo = a, ahi = a + T - 1;
    // first and last brick cell of this ray in the slab: a straight line's cells lie in
    // the box they span
    int fc = INT_MAX, fd = 0, fz = 0, lc = 0, ld = 0, lz = 0;
    while (m <= m1) {
      const float mf = (float)m;
      const Tri t = tri_of(fmaf(mf, d[0], s[0]), fmaf(mf, d[1], s[1]), fmaf(mf, d[2], s[2]));
      const int idom = xd ? t.i : t.j;
      if (B.sgn > 0 ? idom > ahi : idom < alo) break;
      const int ic = (xd ? t.j : t.i) - o.x, id = idom - alo, iz = t.k - o.z;
      const float ab[2] = {1.0f - t.a, t.a}, bb[2] = {1.0f - t.b, t.b}, cb[2] = {1.0f - t.c, t.c};
      if ((unsigned)ic < (unsigned)(P.BC - 1) && (unsigned)id < (unsigned)T &&
          (unsigned)iz < (unsigned)(P.BZ - 1)) {
        float* b0 = brick + ((size_t)iz * (T + 1) + id) * P.BC + ic;
        if (fc == INT_MAX) {
          fc = ic;
          fd = id;
          fz = iz;
        }
        lc = ic;
        ld = id;
        lz = iz;
        const int ox = xd ? P.BC : 1, oy = xd ? 1 : P.BC, oz = P.BC * (T + 1);
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const float w = ab[q & 1] * bb[(q >> 1) & 1] * cb[(q >> 2) & 1];
          atomicAdd(b0 + (q & 1) * ox + ((q >> 1) & 1) * oy + ((q >> 2) & 1) * oz, w * y);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int X = t.i + (q & 1), Y = t.j + ((q >> 1) & 1), Z = t.k + ((q >> 2) & 1);
          if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
          const float w = ab[q & 1] * bb[(q >> 1) & 1] * cb[(q >> 2) & 1];
          atomicAdd(vol + X + Y * sy + Z * sz, w * y);
        }
      }
      m++;
    }
    if (vec4) {
      const bool hit = fc != INT_MAX;
      const int v[6] = {hit ? min(fc, lc) : INT_MAX, hit ? max(fc, lc) : INT_MIN,
                        hit ? min(fd, ld) : INT_MAX, hit ? max(fd, ld) : INT_MIN,
                        hit ? min(fz, lz) : INT_MAX, hit ? max(fz, lz) : INT_MIN};
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const int r = (q & 1) ? __reduce_max_sync(0xffffffffu, v[q]) : __reduce_min_sync(0xffffffffu, v[q]);
        if (lane == 0 && ((q & 1) ? r != INT_MIN : r != INT_MAX)) {
          if (q & 1) atomicMax(&box[q], r);
          else atomicMin(&box[q], r);
        }
      }
    }
    __syncthreads();
    // flush: brick element (c, dd, zz) -> voxel; y-fastest buffer for x-dominant bundles.
    // vec4: four cross-axis neighbours per step (16-byte shared loads and global float4
    // atomics): the brick's cross origin and extent are multiples of 4 and so are the
    // volume's x and y extents, so a group is wholly inside or outside the volume
    if (vec4) {
      // only the box of touched cells (their +1 corners included); the rest is zero
      float4* b4 = reinterpret_cast<float4*>(brick);
      const int cg0 = box[0] >> 2, ncg = ((box[1] + 1) >> 2) - cg0 + 1;
      const int d0 = box[2], ndd = box[3] + 2 - box[2], z0b = box[4], nzb = box[5] + 2 - box[4];
      const int ngr = box[0] == INT_MAX ? 0 : ncg * ndd * nzb;
      for (int gi = threadIdx.x; gi < ngr; gi += blockDim.x) {
        const int cg = cg0 + gi % ncg, rr = gi / ncg;
        const int dd = d0 + rr % ndd, zz = z0b + rr / ndd;
        const int e = (zz * (T + 1) + dd) * P.BC + cg * 4;
        const int e4 = e >> 2;
        const float4 val = b4[e4];
        if (val.x == 0.0f && val.y == 0.0f && val.z == 0.0f && val.w == 0.0f) continue;
        b4[e4] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const int c = cg * 4;
        const int gc = o.x + c, gd = a + dd, gz = o.z + zz;
        const int X = xd ? gd : gc, Y = xd ? gc : gd;
        if (X < 0 || Y < 0 || gz < 0 || X >= nx || Y >= ny || gz >= nz) continue;
        if (xd) atomicAdd(reinterpret_cast<float4*>(volT + (size_t)gz * sz + (size_t)X * ny + Y), val);
        else atomicAdd(reinterpret_cast<float4*>(vol + (size_t)gz * sz + (size_t)Y * nx + X), val);
      }
      __syncthreads();
      continue;
    }
    for (int e = threadIdx.x; e < nb; e += blockDim.x) {
      const float val = brick[e];
      if (val == 0.0f) continue;
      brick[e] = 0.0f;
      const int c = e % P.BC, r = e / P.BC;
      const int dd = r % (T + 1), zz = r / (T + 1);
      const int gc = o.x + c, gd = a + dd, gz = o.z + zz;
      const int X = xd ? gd : gc, Y = xd ? gc : gd;
      if (X < 0 || Y < 0 || gz < 0 || X >= nx || Y >= ny || gz >= nz) continue;
      if (xd) atomicAdd(volT + (size_t)gz * sz + (size_t)X * ny + Y, val);
      else atomicAdd(vol + (size_t)gz * sz + (size_t)Y * nx + X, val);
    }
    __syncthreads();
  }
}

// vol[z][y][x] += vt[z][x][y]
__global__ void transpose_add_kernel(const float* __restrict__ vt, float* __restrict__ vol, int nx,
                                     int ny)
{
  __shared__ float tile[32][33];
  const int z = blockIdx.z;
  const size_t plane = (size_t)nx * ny;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int y = y0 + threadIdx.x, x = x0 + r;
    if (x < nx && y < ny) tile[r][threadIdx.x] = vt[z * plane + (size_t)x * ny + y];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int x = x0 + threadIdx.x, y = y0 + r;
    if (x < nx && y < ny) vol[z * plane + (size_t)y * nx + x] += tile[threadIdx.x][r];
  }
}

// y-fastest copy of the volume: vt[z][x][y] = vol[z][y][x] (bricks of x-dominant bundles).
__global__ void transpose_xy_kernel(const float* __restrict__ vol, float* __restrict__ vt, int nx,
                                    int ny)
{
  __shared__ float tile[32][33];
  const int z = blockIdx.z;
  const size_t plane = (size_t)nx * ny;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int x = x0 + threadIdx.x, y = y0 + r;
    if (x < nx && y < ny) tile[r][threadIdx.x] = vol[z * plane + (size_t)y * nx + x];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int y = y0 + threadIdx.x, x = x0 + r;
    if (x < nx && y < ny) vt[z * plane + (size_t)x * ny + y] = tile[threadIdx.x][r];
  }
}

// Host side of the brick projector: box sizing (pre-pass), the y-fastest copy, tensor maps.
struct BrickSetup {
  bool ok = false;
  int BC = 0, BZ = 0, stages = 0, stage_bytes = 0;
  int minb = 1;  // resident CTAs per SM the kernel's registers are capped for (1 or 3)
  int T = 12;    // dominant planes per slab (8 or 12)
  size_t smem = 0;
};

// Sizes the bricks for the views of `chunks` (pre-pass on `st`, synchronises `st`).
// ok == false when the volume rows are not 16-byte multiples or the bricks do not fit.
int brick_setup(const std::vector<PjParams>& chunks, int nx, int ny, cudaStream_t st, BrickSetup* bs,
                bool for_adjoint = false)
{
  bs->ok = false;
  if (nx % 4 != 0 || ny % 4 != 0 || getenv("FCB_PROJ_NOBRICK")) return FCB_OK;
  int* scratch = nullptr;
  FCB_TRY(device_status_ptr(&scratch));
  int* need = scratch + 3;  // [3..4]: brick extents ([1..2] belong to the backprojector)
  // Slab depth, forward: the deepest of 12, 8 and 6 dominant planes with which three CTAs of
  // two brick buffers fit in an SM's shared memory, else 6 (on the 256^3 / 360-view
  // geometry 6 planes give three CTAs instead of one: 19.9 ms per pass instead of 29.7).
  // The transpose holds one brick and flushes it per slab; 8 planes suit it on both
  // measured geometries.  FCB_PROJ_SLAB=6|8|12 fixes the depth.
  const char* se = getenv("FCB_PROJ_SLAB");
  const int forced = se ? atoi(se) : 0;
  const int order_fwd[3] = {12, 8, 6}, order_adj[3] = {8, 6, 6};
  for (int oi = 0; oi < 3; oi++) {
    const int T = for_adjoint ? order_adj[oi] : order_fwd[oi];
    if (forced && forced != T) continue;
    FCB_CUDA_TRY(cudaMemsetAsync(need, 0, 2 * sizeof(int), st));
    for (const PjParams& P : chunks) {
      const int bx = (P.WH0 + PB_W - 1) / PB_W, by = (P.WH1 + PB_H - 1) / PB_H;
      const long long total = (long long)P.nviews * bx * by;
      const unsigned g = (unsigned)((total + 255) / 256);
      if (T == 12) project_brick_extent_kernel<12><<<g, 256, 0, st>>>(P, bx, by, need);
      else if (T == 8) project_brick_extent_kernel<8><<<g, 256, 0, st>>>(P, bx, by, need);
      else project_brick_extent_kernel<6><<<g, 256, 0, st>>>(P, bx, by, need);
      FCB_CUDA_TRY(cudaGetLastError());
    }
    int h[2] = {0, 0};
    FCB_CUDA_TRY(cudaMemcpyAsync(h, need, sizeof h, cudaMemcpyDeviceToHost, st));
    FCB_CUDA_TRY(cudaStreamSynchronize(st));
    const int BC = std::max(4, (h[0] + 3) & ~3), BZ = std::max(2, h[1]);
    if (BC > 128 || BZ > 64) continue;  // a wide cone: bricks would not pay
    const int box = BC * (T + 1) * BZ * 4;
    if (for_adjoint) {
      if ((size_t)box + 80 > 200 * 1024) continue;
      bs->ok = true;
      bs->T = T;
      bs->BC = BC;
      bs->BZ = BZ;
      return FCB_OK;
    }
    const int stage_bytes = (box + 127) & ~127;
    auto smem_of = [&](int n) {
      return (size_t)n * stage_bytes + n * (2 * sizeof(uint64_t) + sizeof(int4)) + 16;
    };
    // Two buffers and registers capped for three resident CTAs where three such CTAs fit
    // (512^3 / 90 views: 41.6 ms against 47.1 ms with three buffers and two CTAs);
    // otherwise up to four buffers in 96 KB.
    const bool three = 3 * (smem_of(2) + 1024) <= 228 * 1024;
    if (oi < 2 && !three && !forced) continue;  // try a shallower slab
    int stages = std::max(2, std::min(4, (96 * 1024) / stage_bytes)), minb = 1;
    if (three) {
      stages = 2;
      minb = 3;
    }
    // tuning knobs: FCB_PROJ_STAGES=2..6 buffers, FCB_PROJ_MINB=1|3 register cap
    if (const char* e = getenv("FCB_PROJ_STAGES")) stages = std::max(2, std::min(6, atoi(e)));
    if (const char* e = getenv("FCB_PROJ_MINB")) minb = e[0] == '3' ? 3 : 1;
    const size_t smem = smem_of(stages);
    if (smem > 200 * 1024) continue;
    bs->ok = true;
    bs->T = T;
    bs->BC = BC;
    bs->BZ = BZ;
    bs->stages = stages;
    bs->minb = minb;
    bs->stage_bytes = stage_bytes;
    bs->smem = smem;
    return FCB_OK;
  }
  return FCB_OK;
}

// Launches the brick projector over `chunks` (the volume and its y-fastest copy `vt`).
int brick_launch(std::vector<PjParams>& chunks, const BrickSetup& bs, const float* vol, float* vt,
                 int nx, int ny, int nz, cudaStream_t st)
{
  if ((uintptr_t)vol % 16 || (uintptr_t)vt % 16)
    return set_error(FCB_ERR_INVALID, "volume buffers must be 16-byte aligned");
  dim3 tg((nx + 31) / 32, (ny + 31) / 32, nz);
  transpose_xy_kernel<<<tg, dim3(32, 8), 0, st>>>(vol, vt, nx, ny);
  FCB_CUDA_TRY(cudaGetLastError());
  CUtensorMap mv, mt;
  FCB_TRY(encode_tmap_3d(&mv, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, const_cast<float*>(vol), nx, ny, nz,
                         (uint64_t)nx * 4, (uint64_t)nx * ny * 4, bs.BC, bs.T + 1, bs.BZ));
  FCB_TRY(encode_tmap_3d(&mt, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vt, ny, nx, nz, (uint64_t)ny * 4,
                         (uint64_t)nx * ny * 4, bs.BC, bs.T + 1, bs.BZ));
  int* status = nullptr;
  FCB_TRY(device_status_ptr(&status));
  auto pkern = bs.T == 12  ? (bs.minb == 3 ? project_brick_kernel<3, 12> : project_brick_kernel<1, 12>)
               : bs.T == 8 ? (bs.minb == 3 ? project_brick_kernel<3, 8> : project_brick_kernel<1, 8>)
                           : (bs.minb == 3 ? project_brick_kernel<3, 6> : project_brick_kernel<1, 6>);
  FCB_CUDA_TRY(cudaFuncSetAttribute(pkern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)bs.smem));
  for (PjParams& P : chunks) {
    P.BC = bs.BC;
    P.BZ = bs.BZ;
    P.stages = bs.stages;
    P.stage_bytes = bs.stage_bytes;
    P.status = status;
    dim3 grid((P.WH0 + PB_W - 1) / PB_W, (P.WH1 + PB_H - 1) / PB_H, P.nviews);
    pkern<<<grid, PB_THREADS, bs.smem, st>>>(mv, mt, P);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return FCB_OK;
}

// Launches the brick adjoint over `chunks`: vol += A^T (norm * proj), `vt` a scratch volume.
int brick_adjoint_launch(std::vector<PjParams>& chunks, const BrickSetup& bs, float* vol, float* vt,
                         int nx, int ny, int nz, cudaStream_t st)
{
  const size_t smem = (size_t)bs.BC * (bs.T + 1) * bs.BZ * 4 + 16 + 16 + 32;
  if (smem > 200 * 1024) return set_error(FCB_ERR_RANGE, "adjoint brick exceeds shared memory");
  FCB_CUDA_TRY(cudaMemsetAsync(vt, 0, (size_t)nx * ny * nz * sizeof(float), st));
  // 16-byte flush groups: 4 | nx, 4 | ny and both volumes 16-byte aligned (FCB_PROJ_FLUSH4=0
  // selects the element-wise flush, for comparison)
  const char* f4 = getenv("FCB_PROJ_FLUSH4");
  const int vec4 = (nx % 4 == 0 && ny % 4 == 0 && (uintptr_t)vol % 16 == 0 && (uintptr_t)vt % 16 == 0 &&
                    !(f4 && f4[0] == '0')) ? 1 : 0;
  // registers for 5 resident CTAs (the shared-memory limit of the usual brick) unless
  // FCB_PROJ_ADJ_MINB=4 lets the kernel keep its working set without spills
  const char* mb = getenv("FCB_PROJ_ADJ_MINB");
  const bool m4 = mb && mb[0] == '4';
  auto kern = bs.T == 12  ? (m4 ? project_adjoint_brick_kernel<4, 12> : project_adjoint_brick_kernel<5, 12>)
              : bs.T == 8 ? (m4 ? project_adjoint_brick_kernel<4, 8> : project_adjoint_brick_kernel<5, 8>)
                          : (m4 ? project_adjoint_brick_kernel<4, 6> : project_adjoint_brick_kernel<5, 6>);
  FCB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (PjParams& P : chunks) {
    P.BC = bs.BC;
    P.BZ = bs.BZ;
    dim3 grid((P.WH0 + PB_W - 1) / PB_W, (P.WH1 + PB_H - 1) / PB_H, P.nviews);
    kern<<<grid, 256, smem, st>>>(P, vol, vt, vec4);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  dim3 tg((nx + 31) / 32, (ny + 31) / 32, nz);
  transpose_add_kernel<<<tg, dim3(32, 8), 0, st>>>(vt, vol, nx, ny);
  FCB_CUDA_TRY(cudaGetLastError());
  return FCB_OK;
}

// The reference's sub-problem projection (unit_coneBeamGPU.cu:88-171): every volume tile
// of sv0 x sv1 x sv2 voxels is projected on its own, from a copy of the tile ringed by
// zeros, onto the pixels of its detector window only, marching its own integer sweep of
// sample distances.  Summed over tiles this is the ideal projection wherever the windows
// and sweeps cover the tile's shadow; elsewhere it reproduces what the reference loses.
// Used only when the restated windows show a difference (exact FP32 weights).
__global__ void __launch_bounds__(256) project_ref_kernel(const __grid_constant__ PjParams P)
{
  const int wl = blockIdx.x * 16 + (threadIdx.x & 15);
  const int hl = blockIdx.y * 16 + (threadIdx.x >> 4);
  const int v = blockIdx.z;
  if (wl >= P.WH0 || hl >= P.WH1) return;
  const PjView& V = P.v[v];
  float s[3], d[3];
  ray_of(V, wl, hl, s, d);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  float acc = 0.0f;
  for (int tk = 0; tk < P.ntz; tk++)
    for (int tj = 0; tj < P.nty; tj++)
      for (int ti = 0; ti < P.ntx; ti++) {
        const int tile = (tk * P.nty + tj) * P.ntx + ti;
        const int4 wb = P.win[(size_t)tile * P.wviews + P.view0 + v];
        if (wl < wb.x || wl >= wb.x + P.spd0 || hl < wb.y || hl >= wb.y + P.spd1) continue;
        const int ox = ti * P.sv0, oy = tj * P.sv1, oz = tk * P.sv2;
        const int ex = min(ox + P.sv0, nx), ey = min(oy + P.sv1, ny), ez = min(oz + P.sv2, nz);
        const float st[3] = {s[0] - ox, s[1] - oy, s[2] - oz};
        int m0, m1;
        if (!ray_clip(st, d, ex - ox, ey - oy, ez - oz, m0, m1)) continue;
        m0 = max(m0, wb.z);
        m1 = min(m1, wb.z + wb.w - 1);
        for (int m = m0; m <= m1; m++) {
          const float mf = (float)m;
          const Tri t = tri_of(fmaf(mf, d[0], s[0]), fmaf(mf, d[1], s[1]), fmaf(mf, d[2], s[2]));
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int X = t.i + (q & 1), Y = t.j + ((q >> 1) & 1), Z = t.k + ((q >> 2) & 1);
            if (X < ox || Y < oy || Z < oz || X >= ex || Y >= ey || Z >= ez) continue;
            const float w = ((q & 1) ? t.a : 1.0f - t.a) * (((q >> 1) & 1) ? t.b : 1.0f - t.b) *
                            (((q >> 2) & 1) ? t.c : 1.0f - t.c);
            acc = fmaf(w, __ldg(P.vol + X + Y * sy + Z * sz), acc);
          }
        }
      }
  P.proj[((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl] += V.wt * acc;
}

// Exact transpose of project_explicit_kernel: vol += A^T (norm * proj).
__global__ void __launch_bounds__(256) project_adjoint_kernel(const __grid_constant__ PjParams P,
                                                              float* vol)
{
  const int wl = blockIdx.x * 16 + (threadIdx.x & 15);
  const int hl = blockIdx.y * 16 + (threadIdx.x >> 4);
  const int v = blockIdx.z;
  if (wl >= P.WH0 || hl >= P.WH1) return;
  const PjView& V = P.v[v];
  const float y = V.wt * __ldg(P.proj + ((size_t)(P.view0 + v) * P.WH1 + hl) * P.WH0 + wl);
  if (y == 0.0f) return;
  float s[3], d[3];
  ray_of(V, wl, hl, s, d);
  int m0, m1;
  if (!ray_clip(s, d, P.nx, P.ny, P.nz, m0, m1)) return;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const size_t sy = nx, sz = (size_t)nx * ny;
  for (int m = m0; m <= m1; m++) {
    const float mf = (float)m;
    const Tri t = tri_of(fmaf(mf, d[0], s[0]), fmaf(mf, d[1], s[1]), fmaf(mf, d[2], s[2]));
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int X = t.i + (q & 1), Y = t.j + ((q >> 1) & 1), Z = t.k + ((q >> 2) & 1);
      if (X < 0 || Y < 0 || Z < 0 || X >= nx || Y >= ny || Z >= nz) continue;
      const float w = ((q & 1) ? t.a : 1.0f - t.a) * (((q >> 1) & 1) ? t.b : 1.0f - t.b) *
                      (((q >> 2) & 1) ? t.c : 1.0f - t.c);
      atomicAdd(vol + X + Y * sy + Z * sz, w * y);
    }
  }
}

// ------------------------------------------------------------------------------ host
static void fill_pj_views(const Problem& pb, int v0, int n, PjParams* P)
{
  P->nviews = n;
  P->view0 = v0;
  // local continuous voxel index = coordinate + volDim/2 - volStart
  const double off[3] = {(double)(pb.volDim[0] / 2 - pb.volStart[0]),
                         (double)(pb.volDim[1] / 2 - pb.volStart[1]),
                         (double)(pb.volDim[2] / 2 - pb.volStart[2])};
  for (int k = 0; k < n; k++) {
    const int t = v0 + k;
    const ViewGeom& g = pb.views[t];
    PjView& V = P->v[k];
    const double cw = (double)(pb.woff[t] - pb.projDim[0] / 2);
    const double ch = (double)(pb.hoff[t] - pb.projDim[1] / 2);
    for (int a = 0; a < 3; a++) {
      V.s[a] = (float)(g.s[a] + off[a]);
      V.p0[a] = (float)(g.d[a] + cw * g.w[a] + ch * g.h[a] + off[a]);
      V.w[a] = (float)g.w[a];
      V.h[a] = (float)g.h[a];
    }
    V.wt = (float)pb.norm[t];
  }
}

int project_launch(const Problem& pb, int method, const float* vol, float* proj, float* adj_vol,
                   unsigned long long* samples, cudaStream_t st)
{
  const int nx = pb.volEnd[0] - pb.volStart[0], ny = pb.volEnd[1] - pb.volStart[1],
            nz = pb.volEnd[2] - pb.volStart[2];
  // reference-compatible sub-problems, when they change the projection
  RefWindows rw;
  bool compat = false;
  if (pb.referenceWindows && !adj_vol) {
    FCB_TRY(ref_windows(pb, true, &rw));
    compat = rw.proj_matters;
  }
  int4* d_win = nullptr;
  if (compat) {
    const int ntile = rw.ntx * rw.nty * rw.ntz;
    std::vector<int4> tab((size_t)ntile * pb.nviews);
    for (int t = 0; t < ntile; t++)
      for (int v = 0; v < pb.nviews; v++) {
        const size_t o = (size_t)t * pb.nviews + v;
        tab[o] = make_int4(rw.ws[o] - pb.woff[v], rw.hs[o] - pb.hoff[v], rw.sweepStart[o],
                           rw.sweepSteps[o]);
      }
    FCB_CUDA_TRY(cudaMallocAsync((void**)&d_win, tab.size() * sizeof(int4), st));
    cudaError_t e = cudaMemcpyAsync(d_win, tab.data(), tab.size() * sizeof(int4),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the table is a local vector
    if (e != cudaSuccess) {
      cudaFreeAsync(d_win, st);
      return set_error(FCB_ERR_CUDA, cudaGetErrorString(e));
    }
  }
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  if (method == FCB_PROJ_TEXTURE && !adj_vol && !compat) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    FCB_CUDA_TRY(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(nx, ny, nz)));
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr(const_cast<float*>(vol), nx * sizeof(float), nx, ny);
    cp.dstArray = arr;
    cp.extent = make_cudaExtent(nx, ny, nz);
    cp.kind = cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaMemcpy3DAsync(&cp, st);
    if (e != cudaSuccess) {
      cudaFreeArray(arr);
      return set_error(FCB_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
    if (e != cudaSuccess) {
      cudaFreeArray(arr);
      return set_error(FCB_ERR_CUDA, cudaGetErrorString(e));
    }
  }
  std::vector<PjParams> chunks;
  for (int v0 = 0; v0 < pb.nviews; v0 += PJ_MAXV) {
    PjParams P;
    memset(&P, 0, sizeof(P));
    P.vol = vol;
    P.proj = proj;
    P.samples = samples;
    P.tex = tex;
    P.nx = nx; P.ny = ny; P.nz = nz;
    P.WH0 = pb.projWHSize[0]; P.WH1 = pb.projWHSize[1];
    fill_pj_views(pb, v0, std::min(PJ_MAXV, pb.nviews - v0), &P);
    if (compat) {
      P.win = d_win;
      P.sv0 = rw.subVolDim[0]; P.sv1 = rw.subVolDim[1]; P.sv2 = rw.subVolDim[2];
      P.ntx = rw.ntx; P.nty = rw.nty; P.ntz = rw.ntz;
      P.spd0 = rw.subProjDim[0]; P.spd1 = rw.subProjDim[1];
      P.wviews = pb.nviews;
    }
    chunks.push_back(P);
  }
  int rc = FCB_OK;
  if (method == FCB_PROJ_EXPLICIT && !compat) {
    BrickSetup bs;
    FCB_TRY(brick_setup(chunks, nx, ny, st, &bs, adj_vol != nullptr));
    if (bs.ok) {
      float* vt = nullptr;
      FCB_CUDA_TRY(cudaMallocAsync((void**)&vt, (size_t)nx * ny * nz * sizeof(float), st));
      rc = adj_vol ? brick_adjoint_launch(chunks, bs, adj_vol, vt, nx, ny, nz, st)
                   : brick_launch(chunks, bs, vol, vt, nx, ny, nz, st);
      cudaFreeAsync(vt, st);
      return rc;
    }
  }
  for (const PjParams& P : chunks) {
    dim3 grid((P.WH0 + 15) / 16, (P.WH1 + 15) / 16, P.nviews);
    if (compat) project_ref_kernel<<<grid, 256, 0, st>>>(P);
    else if (adj_vol) project_adjoint_kernel<<<grid, 256, 0, st>>>(P, adj_vol);
    else if (method == FCB_PROJ_TEXTURE) project_tex_kernel<<<grid, 256, 0, st>>>(P);
    else project_explicit_kernel<<<grid, 256, 0, st>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { rc = set_error(FCB_ERR_CUDA, cudaGetErrorString(e)); break; }
  }
  if (arr) {
    // the array must outlive the kernels that sample it
    cudaStreamSynchronize(st);
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
  }
  if (d_win) cudaFreeAsync(d_win, st);
  return rc;
}

}  // namespace fcb

using namespace fcb;

// Reusable projector: per-view parameters digested once; for the texture method a 3-D CUDA
// array and its texture object live with the plan, so execute() only copies the volume in
// (stream-ordered) and launches -- no allocation, no synchronisation.
struct fcb_proj_plan {
  Problem pb;
  int method = FCB_PROJ_EXPLICIT;
  int nx = 0, ny = 0, nz = 0;
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  std::vector<PjParams> chunks;
  BrickSetup bricks;     // explicit method: staged-brick projector, when it applies
  BrickSetup bricks_adj; // and its transpose's bricks (their own slab depth)
  float* vt = nullptr;   // its y-fastest volume copy
};

extern "C" int fcb_proj_plan_create(const fcb_geometry* g, int method, fcb_proj_plan** out)
try {
  if (!out) return set_error(FCB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (method != FCB_PROJ_TEXTURE && method != FCB_PROJ_EXPLICIT && method != FCB_PROJ_EXPLICIT_GLOBAL)
    return set_error(FCB_ERR_INVALID, "unknown projector method");
  auto* pl = new fcb_proj_plan();
  int rc = make_problem(g, &pl->pb);
  if (rc) { delete pl; return rc; }
  const Problem& pb = pl->pb;
  if (pb.referenceWindows) {
    RefWindows rw;
    rc = ref_windows(pb, true, &rw);
    if (rc) { delete pl; return rc; }
    if (rw.proj_matters) {
      delete pl;
      return set_error(FCB_ERR_INVALID,
                       "the reference's sub-problem windows change this projection; plans do not "
                       "reproduce them (use fcb_project_device)");
    }
  }
  pl->method = method;
  pl->nx = pb.volEnd[0] - pb.volStart[0];
  pl->ny = pb.volEnd[1] - pb.volStart[1];
  pl->nz = pb.volEnd[2] - pb.volStart[2];
  if (method == FCB_PROJ_TEXTURE) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaError_t e = cudaMalloc3DArray(&pl->arr, &cd, make_cudaExtent(pl->nx, pl->ny, pl->nz));
    if (e != cudaSuccess) { delete pl; return set_error(FCB_ERR_NOMEM, cudaGetErrorString(e)); }
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = pl->arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    e = cudaCreateTextureObject(&pl->tex, &rd, &td, nullptr);
    if (e != cudaSuccess) { cudaFreeArray(pl->arr); delete pl; return set_error(FCB_ERR_CUDA, cudaGetErrorString(e)); }
  }
  for (int v0 = 0; v0 < pb.nviews; v0 += PJ_MAXV) {
    PjParams P;
    memset(&P, 0, sizeof(P));
    P.tex = pl->tex;
    P.nx = pl->nx; P.ny = pl->ny; P.nz = pl->nz;
    P.WH0 = pb.projWHSize[0]; P.WH1 = pb.projWHSize[1];
    fill_pj_views(pb, v0, std::min(PJ_MAXV, pb.nviews - v0), &P);
    pl->chunks.push_back(P);
  }
  if (method == FCB_PROJ_EXPLICIT) {
    rc = brick_setup(pl->chunks, pl->nx, pl->ny, 0, &pl->bricks);
    if (rc == FCB_OK) rc = brick_setup(pl->chunks, pl->nx, pl->ny, 0, &pl->bricks_adj, true);
    if (rc == FCB_OK && (pl->bricks.ok || pl->bricks_adj.ok) &&
        cudaMalloc((void**)&pl->vt, (size_t)pl->nx * pl->ny * pl->nz * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      rc = set_error(FCB_ERR_NOMEM, "device allocation of the brick projector's volume copy failed");
    }
    if (rc) {
      fcb_proj_plan_destroy(pl);
      return rc;
    }
  }
  *out = pl;
  return ok();
}
FCB_CATCH_STATUS

// proj += norm * A vol (adjoint == 0), or vol += A^T (norm * proj) (adjoint != 0, explicit only).
extern "C" int fcb_proj_plan_execute(fcb_proj_plan* pl, const float* volume, float* proj, int adjoint,
                                     void* stream)
try {
  if (!pl || !volume || !proj) return set_error(FCB_ERR_INVALID, "NULL plan or buffer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (adjoint && pl->method == FCB_PROJ_TEXTURE)
    return set_error(FCB_ERR_INVALID, "the adjoint belongs to the explicit projector");
  if (adjoint ? pl->bricks_adj.ok : pl->bricks.ok) {
    for (PjParams& P : pl->chunks) {
      P.vol = volume;
      P.proj = proj;
    }
    if (adjoint)
      FCB_TRY(brick_adjoint_launch(pl->chunks, pl->bricks_adj, const_cast<float*>(volume), pl->vt, pl->nx,
                                   pl->ny, pl->nz, st));
    else
      FCB_TRY(brick_launch(pl->chunks, pl->bricks, volume, pl->vt, pl->nx, pl->ny, pl->nz, st));
    return ok();
  }
  if (pl->method == FCB_PROJ_TEXTURE) {
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr(const_cast<float*>(volume), pl->nx * sizeof(float), pl->nx, pl->ny);
    cp.dstArray = pl->arr;
    cp.extent = make_cudaExtent(pl->nx, pl->ny, pl->nz);
    cp.kind = cudaMemcpyDeviceToDevice;
    FCB_CUDA_TRY(cudaMemcpy3DAsync(&cp, st));
  }
  for (PjParams& P : pl->chunks) {
    P.vol = volume;
    P.proj = proj;
    dim3 grid((P.WH0 + 15) / 16, (P.WH1 + 15) / 16, P.nviews);
    if (adjoint) project_adjoint_kernel<<<grid, 256, 0, st>>>(P, const_cast<float*>(volume));
    else if (pl->method == FCB_PROJ_TEXTURE) project_tex_kernel<<<grid, 256, 0, st>>>(P);
    else project_explicit_kernel<<<grid, 256, 0, st>>>(P);
    FCB_CUDA_TRY(cudaGetLastError());
  }
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_proj_plan_info(const fcb_proj_plan* pl, int* staged, int* brickC, int* brickZ,
                                  int* stages)
try {
  if (!pl) return set_error(FCB_ERR_INVALID, "NULL plan");
  if (staged) *staged = pl->bricks.ok ? 1 : 0;
  if (brickC) *brickC = pl->bricks.BC;
  if (brickZ) *brickZ = pl->bricks.BZ;
  if (stages) *stages = pl->bricks.stages;
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_proj_plan_destroy(fcb_proj_plan* pl)
try {
  if (pl) {
    if (pl->tex) cudaDestroyTextureObject(pl->tex);
    if (pl->arr) cudaFreeArray(pl->arr);
    if (pl->vt) cudaFree(pl->vt);
    delete pl;
  }
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_project_device(const fcb_geometry* g, int method, const float* volume,
                                  float* proj, void* stream)
try {
  if (!volume || !proj) return set_error(FCB_ERR_INVALID, "NULL buffer");
  if (method != FCB_PROJ_TEXTURE && method != FCB_PROJ_EXPLICIT && method != FCB_PROJ_EXPLICIT_GLOBAL)
    return set_error(FCB_ERR_INVALID, "unknown projector method");
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  FCB_TRY(project_launch(pb, method, volume, proj, nullptr, nullptr,
                         reinterpret_cast<cudaStream_t>(stream)));
  return ok();
}
FCB_CATCH_STATUS

extern "C" int fcb_project_adjoint_device(const fcb_geometry* g, const float* proj, float* volume,
                                          void* stream)
try {
  if (!volume || !proj) return set_error(FCB_ERR_INVALID, "NULL buffer");
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  FCB_TRY(project_launch(pb, FCB_PROJ_EXPLICIT, nullptr, const_cast<float*>(proj), volume, nullptr,
                         reinterpret_cast<cudaStream_t>(stream)));
  return ok();
}
FCB_CATCH_STATUS

// Projector with a device-side sample counter (Gsamples accounting for benchmarks).
extern "C" int fcb_project_device_counted(const fcb_geometry* g, int method, const float* volume,
                                          float* proj, unsigned long long* samples_dev,
                                          void* stream)
try {
  if (!volume || !proj) return set_error(FCB_ERR_INVALID, "NULL buffer");
  Problem pb;
  FCB_TRY(make_problem(g, &pb));
  FCB_TRY(project_launch(pb, method, volume, proj, nullptr, samples_dev,
                         reinterpret_cast<cudaStream_t>(stream)));
  return ok();
}
FCB_CATCH_STATUS
