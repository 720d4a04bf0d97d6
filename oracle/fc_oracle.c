/*
 * fc_oracle.c -- CPU restatement of Fastcone's cone-beam operators (test infrastructure).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this file, as
 * the checker or as the timed CPU baseline; the product never links it.
 *
 * Every routine cites the reference lines it restates (paths are relative to the
 * Fastcone source tree).  Float expressions of the reference's host code are written in
 * the same order so that integer outputs of the geometry (windows, sweeps) come out
 * bit-identical when compiled with plain IEEE float (no -ffast-math, no FMA contraction:
 * the Makefile passes -ffp-contract=off).  Device-side float math of the reference is
 * restated in the same order but cannot be bit-identical (nvcc contracts to FMA and its
 * rsqrt is approximate); those paths are compared with a tolerance.
 */
#include "fc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* Block sizes of the reference kernels (coneBeamGPU.cu:52-56) -- they shape the tiling. */
#define ORC_PI 3.14159265358979323846
#define RB_X 8
#define RB_Y 8
#define RB_Z 8
#define RB_W 16
#define RB_H 16

/* ------------------------------------------------------------------------------------ */
/* float3 helpers (the operators of cutil_math.h as used by coneBeamGPU.cu)               */
/* ------------------------------------------------------------------------------------ */
typedef struct { float x, y, z; } f3;
static inline f3 mk(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add3(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 scl3(float s, f3 a) { return mk(a.x * s, a.y * s, a.z * s); }
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 cross3(f3 a, f3 b)
{
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len3(f3 a) { return sqrtf(dot3(a, a)); }
static inline f3 nrm3(f3 a) { return scl3(1.0f / sqrtf(dot3(a, a)), a); }

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* C's (int) conversion of a float, made defined for NaN/out-of-range inputs the way x86
 * cvttss2si behaves (0x80000000), which is what the reference's host code gets for the
 * zero-filled padded views. */
static inline int f2i_trunc(float v)
{
  if (!(v > -2147483648.0f && v < 2147483648.0f)) return (int)0x80000000u;
  return (int)v;
}

/* ------------------------------------------------------------------------------------ */
/* Geometry + sub-problem tiling: restates coneBeamGeometry (coneBeamGPU.cu:1360-1849)    */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  int volDim[3], volStart[3], volEnd[3], projDim[3], projWHSize[2];
  int npad;               /* views padded to nsp * subProjDim[2] (coneBeamGPU.cu:1547) */
  int* projWOffset;       /* padded copies (_padArrays, :1611-1624) */
  int* projHOffset;
  float *hMidPlane, *sina, *cosa, *src, *det, *hst, *wst;
  float D, pw;
  int subVolDim[3], subProjDim[3];
  int nsub, nsx, nsy, nsz, nsp;
  int *xxStart, *yyStart, *zzStart, *ttStart;
  int *wwStart, *hhStart; /* [nsub][subProjDim2] */
  int *sweepStart, *sweepNumSteps;
} rgeom;

static void rgeom_free(rgeom* g)
{
  free(g->projWOffset); free(g->projHOffset);
  free(g->hMidPlane); free(g->sina); free(g->cosa);
  free(g->src); free(g->det); free(g->hst); free(g->wst);
  free(g->xxStart); free(g->yyStart); free(g->zzStart); free(g->ttStart);
  free(g->wwStart); free(g->hhStart); free(g->sweepStart); free(g->sweepNumSteps);
  memset(g, 0, sizeof(*g));
}

/* _calculateProblemGeometry (coneBeamGPU.cu:1672-1734): float math, misalignments
 * Dw, Dh, Dl, Dphi, Dtheta, Dpsi applied in that order. */
static void rgeom_views(rgeom* g, const float* angles, const float* hMid, const float* mis)
{
  int n = g->projDim[2];
  for (int t = 0; t < n; t++) {
    g->hMidPlane[t] = hMid[t] - g->volDim[2] / 2;
    g->sina[t] = sinf(angles[t]);
    g->cosa[t] = cosf(angles[t]);
  }
  float m0 = mis ? mis[0] : 0.0f, m1 = mis ? mis[1] : 0.0f, m2 = mis ? mis[2] : 0.0f;
  float m3 = mis ? mis[3] : 0.0f, m4 = mis ? mis[4] : 0.0f, m5 = mis ? mis[5] : 0.0f;
  float pw = g->pw, D = g->D;
  for (int t = 0; t < n; t++) {
    float a = angles[t];
    f3 s = mk(-1.0f * cosf(a) * D, -1.0f * sinf(a) * D, hMid[t] - g->volDim[2] / 2);
    f3 d = mk(0.0f, 0.0f, hMid[t] - g->volDim[2] / 2);
    f3 h = mk(0.0f, 0.0f, pw);
    f3 w = mk(-1.0f * pw * sinf(a), pw * cosf(a), 0.0f);
    d = add3(d, scl3(m0, w));
    d = add3(d, scl3(m1, h));
    d = add3(d, scl3(m2, nrm3(sub3(d, s))));
    f3 whp = cross3(w, h);
    h = scl3(len3(h), add3(scl3(cosf(m3), nrm3(h)), scl3(sinf(m3), nrm3(whp))));
    whp = cross3(w, h);
    w = scl3(len3(w), add3(scl3(cosf(m4), nrm3(w)), scl3(sinf(m4), nrm3(whp))));
    whp = cross3(w, h);
    f3 wnp = cross3(w, whp);
    f3 hnp = cross3(h, whp);
    w = scl3(len3(w), sub3(scl3(cosf(m5), nrm3(w)), scl3(sinf(m5), nrm3(wnp))));
    h = scl3(len3(h), add3(scl3(cosf(m5), nrm3(h)), scl3(sinf(m5), nrm3(hnp))));
    g->src[3 * t] = s.x; g->src[3 * t + 1] = s.y; g->src[3 * t + 2] = s.z;
    g->det[3 * t] = d.x; g->det[3 * t + 1] = d.y; g->det[3 * t + 2] = d.z;
    g->hst[3 * t] = h.x; g->hst[3 * t + 1] = h.y; g->hst[3 * t + 2] = h.z;
    g->wst[3 * t] = w.x; g->wst[3 * t + 1] = w.y; g->wst[3 * t + 2] = w.z;
  }
}

/* _projectPoint (coneBeamGPU.cu:1816-1849). */
static void rgeom_project_point(const rgeom* g, float xc, float yc, float zc, int t,
                                float* wc, float* hc)
{
  f3 o = mk(xc - (g->volDim[0] / 2), yc - (g->volDim[1] / 2), zc - (g->volDim[2] / 2));
  f3 s = mk(g->src[3 * t], g->src[3 * t + 1], g->src[3 * t + 2]);
  f3 d = mk(g->det[3 * t], g->det[3 * t + 1], g->det[3 * t + 2]);
  f3 h = mk(g->hst[3 * t], g->hst[3 * t + 1], g->hst[3 * t + 2]);
  f3 w = mk(g->wst[3 * t], g->wst[3 * t + 1], g->wst[3 * t + 2]);
  f3 whp = nrm3(cross3(w, h));
  float dist = dot3(sub3(d, s), whp) / dot3(nrm3(sub3(o, s)), whp);
  f3 inter = sub3(add3(s, scl3(dist, nrm3(sub3(o, s)))), d);
  float wDotW = dot3(w, w), wDotH = dot3(w, h), hDotH = dot3(h, h);
  float iDotW = dot3(inter, w), iDotH = dot3(inter, h);
  *wc = (iDotW * hDotH - iDotH * wDotH) / (wDotW * hDotH - wDotH * wDotH);
  *hc = (iDotH * wDotW - iDotW * wDotH) / (wDotW * hDotH - wDotH * wDotH);
  *wc += (g->projDim[0] / 2);
  *hc += (g->projDim[1] / 2);
}

/* _projectCube (coneBeamGPU.cu:1788-1814). */
static void rgeom_project_cube(const rgeom* g, float x0, float x1, float y0, float y1,
                               float z0, float z1, int t, int* we, int* he)
{
  float wc[8], hc[8];
  rgeom_project_point(g, x0, y0, z0, t, wc + 0, hc + 0);
  rgeom_project_point(g, x1, y0, z0, t, wc + 1, hc + 1);
  rgeom_project_point(g, x0, y1, z0, t, wc + 2, hc + 2);
  rgeom_project_point(g, x1, y1, z0, t, wc + 3, hc + 3);
  rgeom_project_point(g, x0, y0, z1, t, wc + 4, hc + 4);
  rgeom_project_point(g, x1, y0, z1, t, wc + 5, hc + 5);
  rgeom_project_point(g, x0, y1, z1, t, wc + 6, hc + 6);
  rgeom_project_point(g, x1, y1, z1, t, wc + 7, hc + 7);
  we[0] = f2i_trunc(wc[0]);
  we[1] = f2i_trunc(wc[0]) + 1;
  he[0] = f2i_trunc(hc[0]);
  he[1] = f2i_trunc(hc[0]) + 1;
  for (int i = 1; i < 8; i++) {
    we[0] = imin(we[0], f2i_trunc(wc[i]));
    he[0] = imin(he[0], f2i_trunc(hc[i]));
    we[1] = imax(we[1], f2i_trunc(wc[i]) + 1);
    he[1] = imax(he[1], f2i_trunc(hc[i]) + 1);
  }
}

static int rgeom_build(rgeom* g, const int volDim[3], const int volStart[3],
                       const int volEnd[3], const int projDim[3], const int projWHSize[2],
                       const int* projWOffset, const int* projHOffset, const float* angles,
                       const float* hMid, float D, const float* mis, float pw)
{
  memset(g, 0, sizeof(*g));
  for (int i = 0; i < 3; i++) {
    g->volDim[i] = volDim[i]; g->volStart[i] = volStart[i]; g->volEnd[i] = volEnd[i];
    g->projDim[i] = projDim[i];
    if (volEnd[i] <= volStart[i] || projDim[i] <= 0) return -1;
  }
  g->projWHSize[0] = projWHSize[0]; g->projWHSize[1] = projWHSize[1];
  g->D = D; g->pw = pw;
  /* _setupSubProblem sizes (coneBeamGPU.cu:1517-1544), maxima from _init (:1413-1416) */
  const int maxSub[3] = {1024, 1024, 512};
  const int maxProj = 256;
  for (int t = 0; t < 3; t++) {
    g->subVolDim[t] = maxSub[t];
    if (g->subVolDim[t] > (volEnd[t] - volStart[t])) g->subVolDim[t] = volEnd[t] - volStart[t];
  }
  g->subVolDim[0] = ((g->subVolDim[0] + RB_X - 1) / RB_X) * RB_X;
  g->subVolDim[1] = ((g->subVolDim[1] + RB_Y - 1) / RB_Y) * RB_Y;
  g->subVolDim[2] = ((g->subVolDim[2] + 4 * RB_Z - 1) / (4 * RB_Z)) * 4 * RB_Z;
  g->subProjDim[0] = 1;
  g->subProjDim[1] = 1;
  int nsp = (projDim[2] + maxProj - 1) / maxProj;
  g->subProjDim[2] = (projDim[2] + nsp - 1) / nsp;
  g->nsx = (volEnd[0] - volStart[0] + g->subVolDim[0] - 1) / g->subVolDim[0];
  g->nsy = (volEnd[1] - volStart[1] + g->subVolDim[1] - 1) / g->subVolDim[1];
  g->nsz = (volEnd[2] - volStart[2] + g->subVolDim[2] - 1) / g->subVolDim[2];
  g->nsp = (projDim[2] + g->subProjDim[2] - 1) / g->subProjDim[2];
  g->nsub = g->nsx * g->nsy * g->nsz * g->nsp;
  g->npad = g->nsp * g->subProjDim[2];
  int np = g->npad > projDim[2] ? g->npad : projDim[2];
  /* per-view arrays, zero padded (_padArrays, :1611-1650) */
  g->projWOffset = (int*)calloc(np, sizeof(int));
  g->projHOffset = (int*)calloc(np, sizeof(int));
  g->hMidPlane = (float*)calloc(np, sizeof(float));
  g->sina = (float*)calloc(np, sizeof(float));
  g->cosa = (float*)calloc(np, sizeof(float));
  g->src = (float*)calloc(3 * np, sizeof(float));
  g->det = (float*)calloc(3 * np, sizeof(float));
  g->hst = (float*)calloc(3 * np, sizeof(float));
  g->wst = (float*)calloc(3 * np, sizeof(float));
  for (int t = 0; t < projDim[2]; t++) {
    g->projWOffset[t] = projWOffset[t];
    g->projHOffset[t] = projHOffset[t];
  }
  rgeom_views(g, angles, hMid, mis);
  int ns = g->nsub, spd2 = g->subProjDim[2];
  g->xxStart = (int*)malloc(ns * sizeof(int));
  g->yyStart = (int*)malloc(ns * sizeof(int));
  g->zzStart = (int*)malloc(ns * sizeof(int));
  g->ttStart = (int*)malloc(ns * sizeof(int));
  g->wwStart = (int*)malloc((size_t)ns * spd2 * sizeof(int));
  g->hhStart = (int*)malloc((size_t)ns * spd2 * sizeof(int));
  g->sweepStart = (int*)malloc((size_t)ns * spd2 * sizeof(int));
  g->sweepNumSteps = (int*)malloc((size_t)ns * spd2 * sizeof(int));
  int idx = 0;
  for (int kk = 0; kk < g->nsz; kk++)
    for (int jj = 0; jj < g->nsy; jj++)
      for (int ii = 0; ii < g->nsx; ii++)
        for (int pp = 0; pp < g->nsp; pp++) {
          g->xxStart[idx] = ii * g->subVolDim[0] + volStart[0];
          g->yyStart[idx] = jj * g->subVolDim[1] + volStart[1];
          g->zzStart[idx] = kk * g->subVolDim[2] + volStart[2];
          g->ttStart[idx] = pp * g->subProjDim[2];
          idx++;
        }
  /* detector windows (coneBeamGPU.cu:1567-1608) */
  for (int p = 0; p < ns; p++) {
    float xx = (float)g->xxStart[p], yy = (float)g->yyStart[p], zz = (float)g->zzStart[p];
    for (int t = 0; t < spd2; t++) {
      int we[2], he[2];
      int tg = t + g->ttStart[p];
      rgeom_project_cube(g, xx, xx + g->subVolDim[0], yy, yy + g->subVolDim[1], zz,
                         zz + g->subVolDim[2], tg, we, he);
      we[0] = imax(we[0], g->projWOffset[tg] - 4);
      we[1] = imax(we[1], g->projWOffset[tg] - 2);
      he[0] = imax(he[0], g->projHOffset[tg] - 4);
      he[1] = imax(he[1], g->projHOffset[tg] - 2);
      we[0] = imin(we[0], g->projWOffset[tg] + projWHSize[0] + 4);
      we[1] = imin(we[1], g->projWOffset[tg] + projWHSize[0] + 2);
      he[0] = imin(he[0], g->projHOffset[tg] + projWHSize[1] + 4);
      he[1] = imin(he[1], g->projHOffset[tg] + projWHSize[1] + 2);
      g->wwStart[(size_t)p * spd2 + t] = we[0];
      g->hhStart[(size_t)p * spd2 + t] = he[0];
      g->subProjDim[0] = imax(g->subProjDim[0], we[1] - we[0]);
      g->subProjDim[1] = imax(g->subProjDim[1], he[1] - he[0]);
    }
  }
  g->subProjDim[0] = RB_W * (1 + (g->subProjDim[0] / RB_W));
  g->subProjDim[1] = RB_H * (1 + (g->subProjDim[1] / RB_H));
  for (size_t i = 0; i < (size_t)ns * spd2; i++) {
    g->wwStart[i] -= (RB_W / 2);
    g->hhStart[i] -= (RB_H / 2);
  }
  /* _calculateSweep (coneBeamGPU.cu:1757-1786) */
  double r = 0.55 * sqrt((double)(g->subVolDim[0] * g->subVolDim[0] + g->subVolDim[1] * g->subVolDim[1] +
                                  g->subVolDim[2] * g->subVolDim[2]));
  for (int p = 0; p < ns; p++) {
    f3 c = mk((float)(g->xxStart[p] + 0.5 * g->subVolDim[0] - 0.5 * volDim[0]),
              (float)(g->yyStart[p] + 0.5 * g->subVolDim[1] - 0.5 * volDim[1]),
              (float)(g->zzStart[p] + 0.5 * g->subVolDim[2] - 0.5 * volDim[2]));
    for (int i = 0; i < spd2; i++) {
      int tg = i + g->ttStart[p];
      f3 s = mk(g->src[3 * tg], g->src[3 * tg + 1], g->src[3 * tg + 2]);
      g->sweepStart[(size_t)p * spd2 + i] = (int)(len3(sub3(c, s)) - r);
      g->sweepNumSteps[(size_t)p * spd2 + i] = (int)(2.0 * r);
    }
  }
  return 0;
}

int orc_ref_geometry(const int volDim[3], const int volStart[3], const int volEnd[3],
                     const int projDim[3], const int projWHSize[2],
                     const int* projWOffset, const int* projHOffset,
                     const float* angles, const float* hMid, float sourceSampleDistance,
                     const float* misAlignments, float pixelWidth,
                     orc_tiling_info* info,
                     int* xxStart, int* yyStart, int* zzStart, int* ttStart,
                     int* wwStart, int* hhStart, int* sweepStart, int* sweepNumSteps,
                     float* src, float* det, float* hstep, float* wstep,
                     float* hMidPlane, float* sina, float* cosa)
{
  rgeom g;
  if (rgeom_build(&g, volDim, volStart, volEnd, projDim, projWHSize, projWOffset, projHOffset,
                  angles, hMid, sourceSampleDistance, misAlignments, pixelWidth) != 0)
    return -1;
  info->subVolDim[0] = g.subVolDim[0]; info->subVolDim[1] = g.subVolDim[1];
  info->subVolDim[2] = g.subVolDim[2];
  info->subProjDim[0] = g.subProjDim[0]; info->subProjDim[1] = g.subProjDim[1];
  info->subProjDim[2] = g.subProjDim[2];
  info->numSubProblems = g.nsub;
  info->nsp = g.nsp;
  size_t ns = g.nsub, n2 = (size_t)g.nsub * g.subProjDim[2], np = g.npad;
#define CP(dst, srcp, n) if (dst) memcpy(dst, srcp, (n) * sizeof(*(dst)))
  CP(xxStart, g.xxStart, ns); CP(yyStart, g.yyStart, ns); CP(zzStart, g.zzStart, ns);
  CP(ttStart, g.ttStart, ns);
  CP(wwStart, g.wwStart, n2); CP(hhStart, g.hhStart, n2);
  CP(sweepStart, g.sweepStart, n2); CP(sweepNumSteps, g.sweepNumSteps, n2);
  CP(src, g.src, 3 * np); CP(det, g.det, 3 * np); CP(hstep, g.hst, 3 * np); CP(wstep, g.wst, 3 * np);
  CP(hMidPlane, g.hMidPlane, np); CP(sina, g.sina, np); CP(cosa, g.cosa, np);
#undef CP
  rgeom_free(&g);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Texture-unit emulation: linear filter, clamp addressing, unnormalised coordinates     */
/* (coneBeamGPU.cu:839-848).  Weights per the CUDA Programming Guide, "Texture Fetching": */
/* x_B = x - 0.5, i = floor(x_B), alpha = frac(x_B) held in 9-bit fixed point with 8     */
/* fractional bits (texq = 1: alpha rounded to a multiple of 1/256).                    */
/* ------------------------------------------------------------------------------------ */
static inline float texw(float a, int texq) { return texq ? nearbyintf(a * 256.0f) * (1.0f / 256.0f) : a; }

static inline void tex_axis(float x, int n, int texq, int* i0, int* i1, float* a)
{
  float xb = x - 0.5f;
  if (!(xb > -2.0f)) xb = -2.0f;            /* far outside: clamp gives the edge texel */
  if (!(xb < (float)n + 1.0f)) xb = (float)n + 1.0f;
  float f = floorf(xb);
  *a = texw(xb - f, texq);
  int i = (int)f;
  *i0 = imin(imax(i, 0), n - 1);
  *i1 = imin(imax(i + 1, 0), n - 1);
}

/* Projection window sampler for one sub-problem and one (local) view: the texel at
 * window index (ww, hh) is norm * P (fillCache, coneBeamGPU.cu:1049-1088) inside the
 * caller's data window and 0 elsewhere. */
typedef struct {
  const float* proj;
  int WH0, WH1, nviews;
  int wws, hhs;      /* window start (global detector index) */
  int woff, hoff;    /* caller data offsets for this view */
  int tg;            /* global view index */
  float nrm;
  int n0, n1;        /* window size (subProjDim[0], [1]) */
} pwin;

static inline float pwin_texel(const pwin* p, int ww, int hh)
{
  if (p->tg >= p->nviews) return 0.0f;
  int ws = ww + p->wws - p->woff, hs = hh + p->hhs - p->hoff;
  if (ws < 0 || ws >= p->WH0 || hs < 0 || hs >= p->WH1) return 0.0f;
  return p->nrm * p->proj[((size_t)p->tg * p->WH1 + hs) * p->WH0 + ws];
}

static inline float pwin_fetch(const pwin* p, float x, float y, int texq)
{
  int i0, i1, j0, j1;
  float a, b;
  tex_axis(x, p->n0, texq, &i0, &i1, &a);
  tex_axis(y, p->n1, texq, &j0, &j1, &b);
  float t00 = pwin_texel(p, i0, j0), t10 = pwin_texel(p, i1, j0);
  float t01 = pwin_texel(p, i0, j1), t11 = pwin_texel(p, i1, j1);
  return (1.0f - a) * (1.0f - b) * t00 + a * (1.0f - b) * t10 + (1.0f - a) * b * t01 + a * b * t11;
}

static inline void pwin_setup(pwin* p, const rgeom* g, int ss, int tl, const float* proj,
                              const float* norm)
{
  int tg = tl + g->ttStart[ss];
  p->proj = proj;
  p->WH0 = g->projWHSize[0]; p->WH1 = g->projWHSize[1];
  p->nviews = g->projDim[2];
  p->wws = g->wwStart[(size_t)ss * g->subProjDim[2] + tl];
  p->hhs = g->hhStart[(size_t)ss * g->subProjDim[2] + tl];
  p->tg = tg;
  p->woff = g->projWOffset[tg];
  p->hoff = g->projHOffset[tg];
  p->nrm = tg < g->projDim[2] ? norm[tg] : 0.0f;
  p->n0 = g->subProjDim[0]; p->n1 = g->subProjDim[1];
}

/* ------------------------------------------------------------------------------------ */
/* Reference-path backprojection kernels                                                 */
/* ------------------------------------------------------------------------------------ */

/* GPU_Feldkamp_backproject_sinogram / GPU_Katsevich_backproject_sinogram
 * (coneBeamGPU.cu:258-420) for one voxel of sub-problem ss with local indices (i, j, k).
 * The kernel gives each thread z-voxels k, k+8, k+16, k+24 of a 32-deep block and steps
 * hh by 8*U/pw between them (:402-408); that incremental stepping is reproduced. */
static float ref_fdk_voxel(const rgeom* g, int ss, int i, int j, int k, const float* proj,
                           const float* norm, int katsevich, int texq)
{
  int xxOffset = g->xxStart[ss] - g->volDim[0] / 2;
  int yyOffset = g->yyStart[ss] - g->volDim[1] / 2;
  int zzOffset = g->zzStart[ss] - g->volDim[2] / 2;
  int kb = k / 32, kq = (k % 32) / 8, kt = k % 8;
  int xx = i + xxOffset, yy = j + yyOffset, zz = kt + 32 * kb + zzOffset;
  float sample = g->D, pfv = 1.0f / g->pw;
  float acc = 0.0f;
  int spd2 = g->subProjDim[2];
  for (int tt = 0; tt < spd2; tt++) {
    int tg = tt + g->ttStart[ss];
    float sa = g->sina[tg], ca = g->cosa[tg];
    float nwo = (float)(g->wwStart[(size_t)ss * spd2 + tt] - g->projDim[0] / 2);
    float nho = (float)(g->hhStart[(size_t)ss * spd2 + tt] - g->projDim[1] / 2);
    float hmp = g->hMidPlane[tg];
    float temp = sample / (sample + (float)xx * ca + (float)yy * sa);
    float ww = ((float)yy * ca - (float)xx * sa) * temp * pfv - nwo + 0.5f;
    float hh = ((float)zz - hmp) * temp * pfv - nho + 0.5f;
    for (int q = 0; q < kq; q++) hh += (8 * temp * pfv);
    pwin p;
    pwin_setup(&p, g, ss, tt, proj, norm);
    float v = pwin_fetch(&p, ww, hh, texq);
    acc += (katsevich ? temp : temp * temp) * v;
  }
  return acc;
}

/* GPU_unweighted_backproject_sinogram (coneBeamGPU.cu:178-255), one voxel. */
static float ref_unweighted_voxel(const rgeom* g, int ss, int i, int j, int k,
                                  const float* proj, const float* norm, int texq)
{
  float ox = (float)i + (float)(g->xxStart[ss] - g->volDim[0] / 2);
  float oy = (float)j + (float)(g->yyStart[ss] - g->volDim[1] / 2);
  float oz = (float)k + (float)(g->zzStart[ss] - g->volDim[2] / 2);
  f3 o = mk(ox, oy, oz);
  float acc = 0.0f;
  int spd2 = g->subProjDim[2];
  for (int tt = 0; tt < spd2; tt++) {
    int tg = tt + g->ttStart[ss];
    f3 s = mk(g->src[3 * tg], g->src[3 * tg + 1], g->src[3 * tg + 2]);
    f3 d = mk(g->det[3 * tg], g->det[3 * tg + 1], g->det[3 * tg + 2]);
    f3 h = mk(g->hst[3 * tg], g->hst[3 * tg + 1], g->hst[3 * tg + 2]);
    f3 w = mk(g->wst[3 * tg], g->wst[3 * tg + 1], g->wst[3 * tg + 2]);
    f3 whp = cross3(w, h);
    float dist = dot3(sub3(d, s), whp) / dot3(sub3(o, s), whp);
    f3 inter = sub3(add3(scl3(dist, sub3(o, s)), s), d);
    float wDotW = dot3(w, w), wDotH = dot3(w, h), hDotH = dot3(h, h);
    float iDotW = dot3(inter, w), iDotH = dot3(inter, h);
    float ww = (iDotW * hDotH - iDotH * wDotH) / (wDotW * hDotH - wDotH * wDotH);
    float hh = (iDotH * wDotW - iDotW * wDotH) / (wDotW * hDotH - wDotH * wDotH);
    float nwo = (float)(g->wwStart[(size_t)ss * spd2 + tt] - g->projDim[0] / 2);
    float nho = (float)(g->hhStart[(size_t)ss * spd2 + tt] - g->projDim[1] / 2);
    pwin p;
    pwin_setup(&p, g, ss, tt, proj, norm);
    acc += pwin_fetch(&p, ww - nwo + 0.5f, hh - nho + 0.5f, texq);
  }
  return acc;
}

/* Driver: coneBeamBackproject / coneBeamRayTraceBackproject (unit_coneBeamGPU.cu:173-305):
 * for each sub-problem the kernel result is ADDED into the caller's volume over the part
 * of the tile inside volStart..volEnd (addCache, coneBeamGPU.cu:1090-1172). */
int orc_ref_backproject(float* volume, const float* projections,
                        const int volDim[3], const int volStart[3], const int volEnd[3],
                        const int projDim[3], const int projWHSize[2],
                        const int* projWOffset, const int* projHOffset,
                        const float* angles, const float* hMid, float sourceSampleDistance,
                        const float* norm, float pixelWidth, int kernelMode,
                        const float* misAlignments, int texq)
{
  rgeom g;
  if (rgeom_build(&g, volDim, volStart, volEnd, projDim, projWHSize, projWOffset, projHOffset,
                  angles, hMid, sourceSampleDistance, kernelMode == 0 ? misAlignments : NULL,
                  pixelWidth) != 0)
    return -1;
  int nx = volEnd[0] - volStart[0], ny = volEnd[1] - volStart[1];
  for (int ss = 0; ss < g.nsub; ss++) {
    int x0 = g.xxStart[ss], y0 = g.yyStart[ss], z0 = g.zzStart[ss];
    int kx = imin(g.subVolDim[0], volEnd[0] - x0);
    int ky = imin(g.subVolDim[1], volEnd[1] - y0);
    int kz = imin(g.subVolDim[2], volEnd[2] - z0);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int k = 0; k < kz; k++)
      for (int j = 0; j < ky; j++)
        for (int i = 0; i < kx; i++) {
          float v = kernelMode == 0
                        ? ref_unweighted_voxel(&g, ss, i, j, k, projections, norm, texq)
                        : ref_fdk_voxel(&g, ss, i, j, k, projections, norm, kernelMode == 1, texq);
          size_t di = (size_t)(x0 + i - volStart[0]) + (size_t)nx * ((y0 + j - volStart[1]) +
                      (size_t)ny * (z0 + k - volStart[2]));
          volume[di] += v;
        }
  }
  rgeom_free(&g);
  return 0;
}

int orc_ref_backproject_points(const int* xyz, int npts, float* out,
                               const float* projections,
                               const int volDim[3], const int volStart[3], const int volEnd[3],
                               const int projDim[3], const int projWHSize[2],
                               const int* projWOffset, const int* projHOffset,
                               const float* angles, const float* hMid,
                               float sourceSampleDistance, const float* norm,
                               float pixelWidth, int kernelMode, int texq)
{
  rgeom g;
  if (rgeom_build(&g, volDim, volStart, volEnd, projDim, projWHSize, projWOffset, projHOffset,
                  angles, hMid, sourceSampleDistance, NULL, pixelWidth) != 0)
    return -1;
#pragma omp parallel for schedule(dynamic, 16)
  for (int n = 0; n < npts; n++) {
    int gx = xyz[3 * n], gy = xyz[3 * n + 1], gz = xyz[3 * n + 2];
    float acc = 0.0f;
    for (int ss = 0; ss < g.nsub; ss++) {
      int i = gx - g.xxStart[ss], j = gy - g.yyStart[ss], k = gz - g.zzStart[ss];
      if (i < 0 || j < 0 || k < 0 || i >= g.subVolDim[0] || j >= g.subVolDim[1] || k >= g.subVolDim[2])
        continue;
      acc += kernelMode == 0 ? ref_unweighted_voxel(&g, ss, i, j, k, projections, norm, texq)
                             : ref_fdk_voxel(&g, ss, i, j, k, projections, norm, kernelMode == 1, texq);
    }
    out[n] = acc;
  }
  rgeom_free(&g);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Reference-path forward projection                                                     */
/* ------------------------------------------------------------------------------------ */

/* 3-D texel of the projector's padded volume tile: fillCache at (xxStart-1, ...) then
 * zeroCacheBoundary (unit_coneBeamGPU.cu:126-142, coneBeamGPU.cu:1179-1208). */
typedef struct {
  const float* vol;
  int vs[3], ve[3];  /* volStart, volEnd */
  int org[3];        /* global index of texel 0 = xxStart - 1 ... */
  int n[3];          /* padded tile dims */
} vtile;

static inline float vtile_texel(const vtile* v, int a, int b, int c)
{
  if (a == 0 || b == 0 || c == 0 || a == v->n[0] - 1 || b == v->n[1] - 1 || c == v->n[2] - 1)
    return 0.0f;
  int gx = a + v->org[0], gy = b + v->org[1], gz = c + v->org[2];
  if (gx < v->vs[0] || gy < v->vs[1] || gz < v->vs[2] || gx >= v->ve[0] || gy >= v->ve[1] ||
      gz >= v->ve[2])
    return 0.0f;
  size_t nx = v->ve[0] - v->vs[0], ny = v->ve[1] - v->vs[1];
  return v->vol[(size_t)(gx - v->vs[0]) + nx * ((size_t)(gy - v->vs[1]) + ny * (size_t)(gz - v->vs[2]))];
}

static inline float vtile_fetch(const vtile* v, float x, float y, float z, int texq)
{
  int i0, i1, j0, j1, k0, k1;
  float a, b, c;
  tex_axis(x, v->n[0], texq, &i0, &i1, &a);
  tex_axis(y, v->n[1], texq, &j0, &j1, &b);
  tex_axis(z, v->n[2], texq, &k0, &k1, &c);
  float r = 0.0f;
  r += (1.0f - a) * (1.0f - b) * (1.0f - c) * vtile_texel(v, i0, j0, k0);
  r += a * (1.0f - b) * (1.0f - c) * vtile_texel(v, i1, j0, k0);
  r += (1.0f - a) * b * (1.0f - c) * vtile_texel(v, i0, j1, k0);
  r += a * b * (1.0f - c) * vtile_texel(v, i1, j1, k0);
  r += (1.0f - a) * (1.0f - b) * c * vtile_texel(v, i0, j0, k1);
  r += a * (1.0f - b) * c * vtile_texel(v, i1, j0, k1);
  r += (1.0f - a) * b * c * vtile_texel(v, i0, j1, k1);
  r += a * b * c * vtile_texel(v, i1, j1, k1);
  return r;
}

/* coneBeamProject (unit_coneBeamGPU.cu:88-171) with GPU_new_project_volume
 * (coneBeamGPU.cu:96-176) and the launcher's offsets (:493-563). */
int orc_ref_project(const float* volume, float* projections,
                    const int volDim[3], const int volStart[3], const int volEnd[3],
                    const int projDim[3], const int projWHSize[2],
                    const int* projWOffset, const int* projHOffset,
                    const float* angles, const float* hMid, float sourceSampleDistance,
                    const float* norm, const float* misAlignments, float pixelWidth,
                    int texq)
{
  rgeom g;
  if (rgeom_build(&g, volDim, volStart, volEnd, projDim, projWHSize, projWOffset, projHOffset,
                  angles, hMid, sourceSampleDistance, misAlignments, pixelWidth) != 0)
    return -1;
  int spd0 = g.subProjDim[0], spd1 = g.subProjDim[1], spd2 = g.subProjDim[2];
  float* cache = (float*)malloc((size_t)spd0 * spd1 * spd2 * sizeof(float));
  for (int ss = 0; ss < g.nsub; ss++) {
    vtile v;
    for (int a = 0; a < 3; a++) {
      v.vs[a] = volStart[a]; v.ve[a] = volEnd[a]; v.n[a] = g.subVolDim[a] + 2;
    }
    v.vol = volume;
    v.org[0] = g.xxStart[ss] - 1; v.org[1] = g.yyStart[ss] - 1; v.org[2] = g.zzStart[ss] - 1;
    float offx = (float)(g.xxStart[ss] - volDim[0] / 2 - 1);
    float offy = (float)(g.yyStart[ss] - volDim[1] / 2 - 1);
    float offz = (float)(g.zzStart[ss] - volDim[2] / 2 - 1);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int tt = 0; tt < spd2; tt++)
      for (int hh = 0; hh < spd1; hh++) {
        int tg = tt + g.ttStart[ss];
        int nwo = g.wwStart[(size_t)ss * spd2 + tt] - projDim[0] / 2;
        int nho = g.hhStart[(size_t)ss * spd2 + tt] - projDim[1] / 2;
        f3 s = mk(g.src[3 * tg], g.src[3 * tg + 1], g.src[3 * tg + 2]);
        f3 d = mk(g.det[3 * tg], g.det[3 * tg + 1], g.det[3 * tg + 2]);
        f3 h = mk(g.hst[3 * tg], g.hst[3 * tg + 1], g.hst[3 * tg + 2]);
        f3 w = mk(g.wst[3 * tg], g.wst[3 * tg + 1], g.wst[3 * tg + 2]);
        int sst = g.sweepStart[(size_t)ss * spd2 + tt];
        int sns = g.sweepNumSteps[(size_t)ss * spd2 + tt];
        for (int ww = 0; ww < spd0; ww++) {
          f3 pos = add3(add3(d, scl3((float)(ww + nwo), w)), scl3((float)(hh + nho), h));
          f3 st = sub3(pos, s);
          st = scl3(1.0f / sqrtf(dot3(st, st)), st);
          pos = add3(s, scl3((float)sst, st));
          pos = sub3(pos, mk(offx - 0.5f, offy - 0.5f, offz - 0.5f));
          float acc = 0.0f;
          for (int q = 0; q < sns; q++) {
            acc += vtile_fetch(&v, pos.x, pos.y, pos.z, texq);
            pos = add3(pos, st);
          }
          cache[(size_t)ww + (size_t)spd0 * (hh + (size_t)spd1 * tt)] = acc;
        }
      }
    /* addCache into projections with norms (coneBeamGPU.cu:1134-1172) */
    for (int pp = 0; pp < spd2; pp++) {
      int pd = pp + g.ttStart[ss];
      if (pd >= projDim[2]) continue;
      int ws = g.wwStart[(size_t)ss * spd2 + pp], hs = g.hhStart[(size_t)ss * spd2 + pp];
      for (int hh = 0; hh < spd1; hh++) {
        int hd = hh + hs - g.projHOffset[pd];
        if (hd < 0 || hd >= projWHSize[1]) continue;
        for (int ww = 0; ww < spd0; ww++) {
          int wd = ww + ws - g.projWOffset[pd];
          if (wd < 0 || wd >= projWHSize[0]) continue;
          projections[((size_t)pd * projWHSize[1] + hd) * projWHSize[0] + wd] +=
              norm[pd] * cache[(size_t)ww + (size_t)spd0 * (hh + (size_t)spd1 * pp)];
        }
      }
    }
  }
  free(cache);
  rgeom_free(&g);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* FP64 oracle                                                                           */
/* ------------------------------------------------------------------------------------ */
typedef struct { double x, y, z; } d3;
static inline d3 dmk(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 dadd(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dsub(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dscl(double s, d3 a) { return dmk(a.x * s, a.y * s, a.z * s); }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b)
{
  return dmk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double dlen(d3 a) { return sqrt(ddot(a, a)); }
static inline d3 dnrm(d3 a) { return dscl(1.0 / sqrt(ddot(a, a)), a); }

/* FP64 per-view geometry: the same construction as _calculateProblemGeometry
 * (coneBeamGPU.cu:1672-1734) in double; positions relative to the volume centre. */
typedef struct { d3 s, d, h, w; double ca, sa, hmp; } dview;

static void dview_make(dview* v, double angle, double hMid, int volDim2, double D, double pw,
                       const float* mis)
{
  double m0 = mis ? mis[0] : 0, m1 = mis ? mis[1] : 0, m2 = mis ? mis[2] : 0;
  double m3 = mis ? mis[3] : 0, m4 = mis ? mis[4] : 0, m5 = mis ? mis[5] : 0;
  double hmp = hMid - (double)(volDim2 / 2);
  v->ca = cos(angle); v->sa = sin(angle); v->hmp = hmp;
  d3 s = dmk(-v->ca * D, -v->sa * D, hmp);
  d3 d = dmk(0, 0, hmp);
  d3 h = dmk(0, 0, pw);
  d3 w = dmk(-pw * v->sa, pw * v->ca, 0);
  d = dadd(d, dscl(m0, w));
  d = dadd(d, dscl(m1, h));
  d = dadd(d, dscl(m2, dnrm(dsub(d, s))));
  d3 whp = dcross(w, h);
  h = dscl(dlen(h), dadd(dscl(cos(m3), dnrm(h)), dscl(sin(m3), dnrm(whp))));
  whp = dcross(w, h);
  w = dscl(dlen(w), dadd(dscl(cos(m4), dnrm(w)), dscl(sin(m4), dnrm(whp))));
  whp = dcross(w, h);
  d3 wnp = dcross(w, whp), hnp = dcross(h, whp);
  d3 w2 = dscl(dlen(w), dsub(dscl(cos(m5), dnrm(w)), dscl(sin(m5), dnrm(wnp))));
  d3 h2 = dscl(dlen(h), dadd(dscl(cos(m5), dnrm(h)), dscl(sin(m5), dnrm(hnp))));
  v->s = s; v->d = d; v->h = h2; v->w = w2;
}

/* exact bilinear sample of view t's data window with zero extension; (wg, hg) are
 * continuous GLOBAL detector indices (pixel g centred at g). */
static inline double bil_window(const float* proj, int WH0, int WH1, int t, int woff,
                                int hoff, double wg, double hg)
{
  double wl = wg - woff, hl = hg - hoff;
  if (!(wl > -1.0 && wl < WH0 && hl > -1.0 && hl < WH1)) return 0.0;
  double fi = floor(wl), fj = floor(hl);
  double a = wl - fi, b = hl - fj;
  int i = (int)fi, j = (int)fj;
  const float* P = proj + (size_t)t * WH0 * WH1;
  double r = 0.0;
  if (j >= 0) {
    if (i >= 0) r += (1 - a) * (1 - b) * P[(size_t)j * WH0 + i];
    if (i + 1 < WH0) r += a * (1 - b) * P[(size_t)j * WH0 + i + 1];
  }
  if (j + 1 < WH1) {
    if (i >= 0) r += (1 - a) * b * P[(size_t)(j + 1) * WH0 + i];
    if (i + 1 < WH0) r += a * b * P[(size_t)(j + 1) * WH0 + i + 1];
  }
  return r;
}

static double bp_voxel_f64(int gx, int gy, int gz, const float* proj, const int volDim[3],
                           const int projDim[3], const int projWHSize[2], const int* woff,
                           const int* hoff, const dview* views, double D, const float* norm,
                           double pw, int mode)
{
  double x = gx - volDim[0] / 2, y = gy - volDim[1] / 2, z = gz - volDim[2] / 2;
  double W2 = projDim[0] / 2, H2 = projDim[1] / 2;
  double acc = 0.0;
  for (int t = 0; t < projDim[2]; t++) {
    const dview* v = &views[t];
    double wg, hg, wt;
    if (mode == 0) {
      d3 o = dmk(x, y, z);
      d3 whp = dcross(v->w, v->h);
      double dist = ddot(dsub(v->d, v->s), whp) / ddot(dsub(o, v->s), whp);
      d3 inter = dsub(dadd(dscl(dist, dsub(o, v->s)), v->s), v->d);
      double wDotW = ddot(v->w, v->w), wDotH = ddot(v->w, v->h), hDotH = ddot(v->h, v->h);
      double iDotW = ddot(inter, v->w), iDotH = ddot(inter, v->h);
      double den = wDotW * hDotH - wDotH * wDotH;
      wg = (iDotW * hDotH - iDotH * wDotH) / den + W2;
      hg = (iDotH * wDotW - iDotW * wDotH) / den + H2;
      wt = 1.0;
    } else {
      double U = D / (D + x * v->ca + y * v->sa);
      wg = (y * v->ca - x * v->sa) * U / pw + W2;
      hg = (z - v->hmp) * U / pw + H2;
      wt = mode == 1 ? U : U * U;
    }
    acc += norm[t] * wt * bil_window(proj, projWHSize[0], projWHSize[1], t, woff[t], hoff[t], wg, hg);
  }
  return acc;
}

static dview* make_views(int n, const float* angles, const float* hMid, int volDim2, double D,
                         double pw, const float* mis)
{
  dview* v = (dview*)malloc((size_t)n * sizeof(dview));
  for (int t = 0; t < n; t++) dview_make(&v[t], (double)angles[t], (double)hMid[t], volDim2, D, pw, mis);
  return v;
}

int orc_backproject_f64(double* vol, const float* projections,
                        const int volDim[3], const int volStart[3], const int volEnd[3],
                        const int projDim[3], const int projWHSize[2],
                        const int* projWOffset, const int* projHOffset,
                        const float* angles, const float* hMid, double D,
                        const float* norm, double pw, int kernelMode,
                        const float* misAlignments)
{
  int mode = kernelMode == 0 ? 0 : (kernelMode == 1 ? 1 : 2);
  dview* views = make_views(projDim[2], angles, hMid, volDim[2], D, pw,
                            mode == 0 ? misAlignments : NULL);
  int nx = volEnd[0] - volStart[0], ny = volEnd[1] - volStart[1], nz = volEnd[2] - volStart[2];
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        vol[(size_t)i + (size_t)nx * (j + (size_t)ny * k)] +=
            bp_voxel_f64(i + volStart[0], j + volStart[1], k + volStart[2], projections, volDim,
                         projDim, projWHSize, projWOffset, projHOffset, views, D, norm, pw, mode);
  free(views);
  return 0;
}

/* Katsevich backprojection with the PI-line window, FP64: vol += sum_t norm[t] U
 * bilinear(P_t) over views whose source angle lies in the voxel's PI interval, tested on
 * the virtual detector through the axis by the Tam-Danielsson bounds
 *   top(u) = (P/2pi)(1 + u^2/D^2)(pi/2 - atan(u/D)),  bottom(u) = -(P/2pi)(1 + u^2/D^2)(pi/2 + atan(u/D))
 * (Noo, Pack, Heuscher 2003, flat detector at distance D) with u the detector coordinate
 * along the source's direction of travel (u = -w for a right-handed helix here) and
 * heights relative to the source.  pitch = source rise per turn (voxels). */
/* One voxel's PI-window Katsevich sum (global voxel indices gx, gy, gz); *cnt += the
 * voxel-view pairs inside the window. */
static double kats_piwin_voxel_f64(int gx, int gy, int gz, const float* projections,
                                   const int volDim[3], const int projDim[3],
                                   const int projWHSize[2], const int* projWOffset,
                                   const int* projHOffset, const dview* views, double D,
                                   const float* norm, double pw, double pitch, double sgn,
                                   int64_t* cnt)
{
  const int n = projDim[2];
  const double W2 = projDim[0] / 2, H2 = projDim[1] / 2;
  const double x = gx - volDim[0] / 2, y = gy - volDim[1] / 2, z = gz - volDim[2] / 2;
  double acc = 0.0;
  int64_t c = 0;
  for (int t = 0; t < n; t++) {
    const dview* v = &views[t];
    const double U = D / (D + x * v->ca + y * v->sa);
    const double w = (y * v->ca - x * v->sa) * U; /* voxel units on the virtual detector */
    const double h = (z - v->hmp) * U;
    const double u = sgn * w / D;
    const double q = (pitch / (2.0 * ORC_PI)) * (1.0 + u * u);
    if (h > q * (ORC_PI / 2 - atan(u)) || h < -q * (ORC_PI / 2 + atan(u))) continue;
    c++;
    acc += norm[t] * U * bil_window(projections, projWHSize[0], projWHSize[1], t,
                                    projWOffset[t], projHOffset[t], w / pw + W2, h / pw + H2);
  }
  *cnt += c;
  return acc;
}

/* Sense of the helix relative to the detector's w axis: the window's u axis runs against
 * the source's direction of travel for a right-handed helix (angles and height rising
 * together). */
static double kats_sign(const float* angles, int n, double pitch)
{
  const double turn = n > 1 ? (double)angles[n - 1] - (double)angles[0] : 1.0;
  return ((turn >= 0.0) == (pitch >= 0.0)) ? -1.0 : 1.0;
}

/* Katsevich backprojection with the PI-line window, FP64: vol += sum_t norm[t] U
 * bilinear(P_t) over views whose source angle lies in the voxel's PI interval, tested on
 * the virtual detector through the axis by the Tam-Danielsson bounds
 *   top(u) = (P/2pi)(1 + u^2/D^2)(pi/2 - atan(u/D)),  bottom(u) = -(P/2pi)(1 + u^2/D^2)(pi/2 + atan(u/D))
 * (Noo, Pack, Heuscher 2003, flat detector at distance D) with u the detector coordinate
 * along the source's direction of travel (u = -w for a right-handed helix here) and
 * heights relative to the source.  pitch = source rise per turn (voxels). */
int orc_katsevich_piwin_f64(double* vol, const float* projections,
                            const int volDim[3], const int volStart[3], const int volEnd[3],
                            const int projDim[3], const int projWHSize[2],
                            const int* projWOffset, const int* projHOffset,
                            const float* angles, const float* hMid, double D,
                            const float* norm, double pw, double pitch, int64_t* pairs)
{
  const int n = projDim[2];
  dview* views = make_views(n, angles, hMid, volDim[2], D, pw, NULL);
  const double sgn = kats_sign(angles, n, pitch);
  const int nx = volEnd[0] - volStart[0], ny = volEnd[1] - volStart[1], nz = volEnd[2] - volStart[2];
  int64_t cnt = 0;
#pragma omp parallel for collapse(2) schedule(dynamic, 1) reduction(+ : cnt)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        vol[(size_t)i + (size_t)nx * (j + (size_t)ny * k)] +=
            kats_piwin_voxel_f64(i + volStart[0], j + volStart[1], k + volStart[2], projections,
                                 volDim, projDim, projWHSize, projWOffset, projHOffset, views, D,
                                 norm, pw, pitch, sgn, &cnt);
  free(views);
  if (pairs) *pairs = cnt;
  return 0;
}

/* The same at listed voxels (global indices xyz[3n..3n+2]); *pairs = their in-window
 * voxel-view pairs. */
int orc_katsevich_piwin_points_f64(const int* xyz, int npts, double* out,
                                   const float* projections,
                                   const int volDim[3], const int projDim[3],
                                   const int projWHSize[2], const int* projWOffset,
                                   const int* projHOffset, const float* angles,
                                   const float* hMid, double D, const float* norm, double pw,
                                   double pitch, int64_t* pairs)
{
  const int n = projDim[2];
  dview* views = make_views(n, angles, hMid, volDim[2], D, pw, NULL);
  const double sgn = kats_sign(angles, n, pitch);
  int64_t cnt = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : cnt)
  for (int p = 0; p < npts; p++)
    out[p] = kats_piwin_voxel_f64(xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2], projections, volDim,
                                  projDim, projWHSize, projWOffset, projHOffset, views, D, norm, pw,
                                  pitch, sgn, &cnt);
  free(views);
  if (pairs) *pairs = cnt;
  return 0;
}

int orc_backproject_points_f64(const int* xyz, int npts, double* out,
                               const float* projections,
                               const int volDim[3], const int volStart[3], const int volEnd[3],
                               const int projDim[3], const int projWHSize[2],
                               const int* projWOffset, const int* projHOffset,
                               const float* angles, const float* hMid, double D,
                               const float* norm, double pw, int kernelMode)
{
  (void)volStart; (void)volEnd;
  int mode = kernelMode == 0 ? 0 : (kernelMode == 1 ? 1 : 2);
  dview* views = make_views(projDim[2], angles, hMid, volDim[2], D, pw, NULL);
#pragma omp parallel for schedule(dynamic, 16)
  for (int n = 0; n < npts; n++)
    out[n] = bp_voxel_f64(xyz[3 * n], xyz[3 * n + 1], xyz[3 * n + 2], projections, volDim, projDim,
                          projWHSize, projWOffset, projHOffset, views, D, norm, pw, mode);
  free(views);
  return 0;
}

/* Ray through pixel (gw, gh) of view v: source S and unit direction dir, in coordinates
 * where voxel g sits at g - volDim/2. */
static inline void pixel_ray(const dview* v, int gw, int gh, const int projDim[3], d3* S, d3* dir)
{
  d3 P = dadd(dadd(v->d, dscl((double)(gw - projDim[0] / 2), v->w)),
              dscl((double)(gh - projDim[1] / 2), v->h));
  *S = v->s;
  *dir = dnrm(dsub(P, v->s));
}

/* Parameter range [m0, m1] of integer sample indices m along S + m dir whose trilinear
 * stencil touches the volume: continuous global index in (volStart-1, volEnd) per axis. */
static inline int ray_range(d3 S, d3 dir, const int volDim[3], const int volStart[3],
                            const int volEnd[3], long* m0, long* m1)
{
  double lo = -1e300, hi = 1e300;
  double so[3] = {S.x + volDim[0] / 2, S.y + volDim[1] / 2, S.z + volDim[2] / 2};
  double dd[3] = {dir.x, dir.y, dir.z};
  for (int a = 0; a < 3; a++) {
    double bl = volStart[a] - 1.0, bh = (double)volEnd[a];
    if (fabs(dd[a]) < 1e-300) {
      if (!(so[a] > bl && so[a] < bh)) return 0;
      continue;
    }
    double t0 = (bl - so[a]) / dd[a], t1 = (bh - so[a]) / dd[a];
    if (t0 > t1) { double tmp = t0; t0 = t1; t1 = tmp; }
    if (t0 > lo) lo = t0;
    if (t1 < hi) hi = t1;
  }
  if (!(hi > lo)) return 0;
  *m0 = (long)ceil(lo);
  *m1 = (long)floor(hi);
  if (*m1 < *m0) return 0;
  return 1;
}

/* trilinear weights of continuous global index p (zero outside volStart..volEnd-1):
 * calls cb(index, weight) for the up-to-8 voxels of the stencil. */
#define TRILIN_LOOP(p, volStart, volEnd, BODY)                                              \
  do {                                                                                    \
    double fx_ = floor((p)[0]), fy_ = floor((p)[1]), fz_ = floor((p)[2]);                 \
    double ax_ = (p)[0] - fx_, ay_ = (p)[1] - fy_, az_ = (p)[2] - fz_;                    \
    int ix_ = (int)fx_, iy_ = (int)fy_, iz_ = (int)fz_;                                   \
    for (int c_ = 0; c_ < 8; c_++) {                                                      \
      int X_ = ix_ + (c_ & 1), Y_ = iy_ + ((c_ >> 1) & 1), Z_ = iz_ + ((c_ >> 2) & 1);    \
      if (X_ < (volStart)[0] || Y_ < (volStart)[1] || Z_ < (volStart)[2] ||               \
          X_ >= (volEnd)[0] || Y_ >= (volEnd)[1] || Z_ >= (volEnd)[2])                    \
        continue;                                                                         \
      double W_ = ((c_ & 1) ? ax_ : 1 - ax_) * (((c_ >> 1) & 1) ? ay_ : 1 - ay_) *        \
                  (((c_ >> 2) & 1) ? az_ : 1 - az_);                                      \
      size_t I_ = (size_t)(X_ - (volStart)[0]) +                                          \
                  (size_t)((volEnd)[0] - (volStart)[0]) *                                 \
                      ((size_t)(Y_ - (volStart)[1]) +                                     \
                       (size_t)((volEnd)[1] - (volStart)[1]) * (size_t)(Z_ - (volStart)[2])); \
      BODY;                                                                               \
    }                                                                                     \
  } while (0)

int orc_project_f64(const float* volume, double* projections,
                    const int volDim[3], const int volStart[3], const int volEnd[3],
                    const int projDim[3], const int projWHSize[2],
                    const int* projWOffset, const int* projHOffset,
                    const float* angles, const float* hMid, double D,
                    const float* norm, const float* misAlignments, double pw)
{
  dview* views = make_views(projDim[2], angles, hMid, volDim[2], D, pw, misAlignments);
  int W0 = projWHSize[0], W1 = projWHSize[1];
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int t = 0; t < projDim[2]; t++)
    for (int hl = 0; hl < W1; hl++)
      for (int wl = 0; wl < W0; wl++) {
        d3 S, dir;
        pixel_ray(&views[t], wl + projWOffset[t], hl + projHOffset[t], projDim, &S, &dir);
        long m0, m1;
        double acc = 0.0;
        if (ray_range(S, dir, volDim, volStart, volEnd, &m0, &m1)) {
          for (long m = m0; m <= m1; m++) {
            double p[3] = {S.x + m * dir.x + volDim[0] / 2, S.y + m * dir.y + volDim[1] / 2,
                           S.z + m * dir.z + volDim[2] / 2};
            TRILIN_LOOP(p, volStart, volEnd, acc += W_ * volume[I_]);
          }
        }
        projections[((size_t)t * W1 + hl) * W0 + wl] += norm[t] * acc;
      }
  free(views);
  return 0;
}

int orc_project_adjoint_f64(double* volume, const float* projections,
                            const int volDim[3], const int volStart[3], const int volEnd[3],
                            const int projDim[3], const int projWHSize[2],
                            const int* projWOffset, const int* projHOffset,
                            const float* angles, const float* hMid, double D,
                            const float* norm, const float* misAlignments, double pw)
{
  dview* views = make_views(projDim[2], angles, hMid, volDim[2], D, pw, misAlignments);
  int W0 = projWHSize[0], W1 = projWHSize[1];
  /* sequential over rays: scatter (deterministic order) */
  for (int t = 0; t < projDim[2]; t++)
    for (int hl = 0; hl < W1; hl++)
      for (int wl = 0; wl < W0; wl++) {
        double y = norm[t] * projections[((size_t)t * W1 + hl) * W0 + wl];
        if (y == 0.0) continue;
        d3 S, dir;
        pixel_ray(&views[t], wl + projWOffset[t], hl + projHOffset[t], projDim, &S, &dir);
        long m0, m1;
        if (!ray_range(S, dir, volDim, volStart, volEnd, &m0, &m1)) continue;
        for (long m = m0; m <= m1; m++) {
          double p[3] = {S.x + m * dir.x + volDim[0] / 2, S.y + m * dir.y + volDim[1] / 2,
                         S.z + m * dir.z + volDim[2] / 2};
          TRILIN_LOOP(p, volStart, volEnd, volume[I_] += W_ * y);
        }
      }
  free(views);
  return 0;
}

int64_t orc_projector_sample_count(const int volDim[3], const int volStart[3],
                                   const int volEnd[3], const int projDim[3],
                                   const int projWHSize[2], const int* projWOffset,
                                   const int* projHOffset, const float* angles,
                                   const float* hMid, double D, double pw)
{
  dview* views = make_views(projDim[2], angles, hMid, volDim[2], D, pw, NULL);
  int64_t total = 0;
  int W0 = projWHSize[0], W1 = projWHSize[1];
#pragma omp parallel for collapse(2) reduction(+ : total) schedule(dynamic, 1)
  for (int t = 0; t < projDim[2]; t++)
    for (int hl = 0; hl < W1; hl++)
      for (int wl = 0; wl < W0; wl++) {
        d3 S, dir;
        pixel_ray(&views[t], wl + projWOffset[t], hl + projHOffset[t], projDim, &S, &dir);
        long m0, m1;
        if (ray_range(S, dir, volDim, volStart, volEnd, &m0, &m1)) total += (m1 - m0 + 1);
      }
  free(views);
  return total;
}

/* ------------------------------------------------------------------------------------ */
/* Ellipsoid phantom                                                                     */
/* ------------------------------------------------------------------------------------ */
int orc_phantom_voxelize(float* vol, const int volDim[3], const double* params, int n)
{
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < volDim[2]; k++)
    for (int j = 0; j < volDim[1]; j++)
      for (int i = 0; i < volDim[0]; i++) {
        double p[3] = {(double)(i - volDim[0] / 2), (double)(j - volDim[1] / 2),
                       (double)(k - volDim[2] / 2)};
        double v = 0.0;
        for (int e = 0; e < n; e++) {
          const double* E = params + 16 * e;
          double q[3] = {p[0] - E[0], p[1] - E[1], p[2] - E[2]};
          /* body coordinates = R^T q; R row-major in E[6..14] */
          double b0 = E[6] * q[0] + E[9] * q[1] + E[12] * q[2];
          double b1 = E[7] * q[0] + E[10] * q[1] + E[13] * q[2];
          double b2 = E[8] * q[0] + E[11] * q[1] + E[14] * q[2];
          double r = (b0 / E[3]) * (b0 / E[3]) + (b1 / E[4]) * (b1 / E[4]) + (b2 / E[5]) * (b2 / E[5]);
          if (r <= 1.0) v += E[15];
        }
        vol[(size_t)i + (size_t)volDim[0] * (j + (size_t)volDim[1] * k)] = (float)v;
      }
  return 0;
}

double orc_phantom_line_integral(const double* params, int n, const double p0[3], const double d[3])
{
  double total = 0.0;
  for (int e = 0; e < n; e++) {
    const double* E = params + 16 * e;
    double q[3] = {p0[0] - E[0], p0[1] - E[1], p0[2] - E[2]};
    double u[3], v[3];
    for (int a = 0; a < 3; a++) {
      double bq = E[6 + a] * q[0] + E[9 + a] * q[1] + E[12 + a] * q[2];
      double bd = E[6 + a] * d[0] + E[9 + a] * d[1] + E[12 + a] * d[2];
      u[a] = bq / E[3 + a];
      v[a] = bd / E[3 + a];
    }
    double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
    double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double disc = uv * uv - vv * (uu - 1.0);
    if (disc > 0.0) total += E[15] * 2.0 * sqrt(disc) / vv;
  }
  return total;
}
