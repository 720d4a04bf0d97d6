// fcb_refgeom.cpp -- the reference's sub-problem decomposition, for the reference-compatible
// window mode.
//
// Fastcone cuts every call into sub-problems (volume tiles of at most 1024 x 1024 x 512 x
// up to 256 views) and gives each (tile, view) a detector window computed from the tile's
// 8 projected corners, clipped to the data window +- 2..4 pixels, widened to a multiple of
// 16 and shifted left by 8 (coneBeamGeometry::_setupSubProblem, coneBeamGPU.cu:1509-1609);
// the projector additionally marches only over a per-(tile, view) sweep of
// (int)(2 * 0.55 |tile|) unit steps (_calculateSweep, :1757-1786).  The windows can cut off
// detector columns that the tile projects onto (then clamp addressing repeats the last
// in-window column), and the sweep can miss samples of small tiles.  This file computes
// the same integers as the reference does: float (FP32) vector arithmetic in the reference's
// expression order, C truncation for the int conversions.  The kernels use them only when
// they change a result (RefWindows::bp_matters / proj_matters).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fcb_internal.h"

namespace fcb {
namespace {

struct F3 {
  float x, y, z;
};
inline F3 f3(float x, float y, float z) { return {x, y, z}; }
inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 scl(float s, F3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len(F3 a) { return sqrtf(dot(a, a)); }
inline F3 nrm(F3 a) { return scl(1.0f / sqrtf(dot(a, a)), a); }

// C's float -> int conversion, defined for NaN / out-of-range inputs as x86 does it
// (the zero-padded views of the last view chunk produce NaNs in the reference too).
inline int trunc_i(float v)
{
  if (!(v > -2147483648.0f && v < 2147483648.0f)) return (int)0x80000000u;
  return (int)v;
}

struct View32 {
  F3 s, d, h, w;
};

// _calculateProblemGeometry in FP32 (coneBeamGPU.cu:1672-1734)
View32 view32(float angle, float hMid, int volDim2, float D, float pw, const float* m)
{
  View32 v;
  F3 s = f3(-1.0f * cosf(angle) * D, -1.0f * sinf(angle) * D, hMid - volDim2 / 2);
  F3 d = f3(0.0f, 0.0f, hMid - volDim2 / 2);
  F3 h = f3(0.0f, 0.0f, pw);
  F3 w = f3(-1.0f * pw * sinf(angle), pw * cosf(angle), 0.0f);
  d = add(d, scl(m[0], w));
  d = add(d, scl(m[1], h));
  d = add(d, scl(m[2], nrm(sub(d, s))));
  F3 whp = cross(w, h);
  h = scl(len(h), add(scl(cosf(m[3]), nrm(h)), scl(sinf(m[3]), nrm(whp))));
  whp = cross(w, h);
  w = scl(len(w), add(scl(cosf(m[4]), nrm(w)), scl(sinf(m[4]), nrm(whp))));
  whp = cross(w, h);
  F3 wnp = cross(w, whp), hnp = cross(h, whp);
  F3 w2 = scl(len(w), sub(scl(cosf(m[5]), nrm(w)), scl(sinf(m[5]), nrm(wnp))));
  F3 h2 = scl(len(h), add(scl(cosf(m[5]), nrm(h)), scl(sinf(m[5]), nrm(hnp))));
  v.s = s; v.d = d; v.h = h2; v.w = w2;
  return v;
}

// _projectPoint (coneBeamGPU.cu:1816-1849)
void project_point(const View32& v, const int volDim[3], const int projDim[3], float xc, float yc,
                   float zc, float* wc, float* hc)
{
  F3 o = f3(xc - (volDim[0] / 2), yc - (volDim[1] / 2), zc - (volDim[2] / 2));
  F3 whp = nrm(cross(v.w, v.h));
  float dist = dot(sub(v.d, v.s), whp) / dot(nrm(sub(o, v.s)), whp);
  F3 inter = sub(add(v.s, scl(dist, nrm(sub(o, v.s)))), v.d);
  float wDotW = dot(v.w, v.w), wDotH = dot(v.w, v.h), hDotH = dot(v.h, v.h);
  float iDotW = dot(inter, v.w), iDotH = dot(inter, v.h);
  *wc = (iDotW * hDotH - iDotH * wDotH) / (wDotW * hDotH - wDotH * wDotH);
  *hc = (iDotH * wDotW - iDotW * wDotH) / (wDotW * hDotH - wDotH * wDotH);
  *wc += (projDim[0] / 2);
  *hc += (projDim[1] / 2);
}

}  // namespace

int ref_windows(const Problem& pb, bool with_misalign, RefWindows* rw)
{
  const int* vd = pb.volDim;
  const int* vs = pb.volStart;
  const int* ve = pb.volEnd;
  const int n = pb.nviews;
  // sub-problem sizes (coneBeamGPU.cu:1413-1416, 1517-1544)
  const int maxSub[3] = {1024, 1024, 512};
  int sv[3];
  for (int a = 0; a < 3; a++) sv[a] = std::min(maxSub[a], ve[a] - vs[a]);
  sv[0] = ((sv[0] + 7) / 8) * 8;
  sv[1] = ((sv[1] + 7) / 8) * 8;
  sv[2] = ((sv[2] + 31) / 32) * 32;
  const int nsp = (n + 255) / 256;
  const int chunk = (n + nsp - 1) / nsp;
  rw->ntx = (ve[0] - vs[0] + sv[0] - 1) / sv[0];
  rw->nty = (ve[1] - vs[1] + sv[1] - 1) / sv[1];
  rw->ntz = (ve[2] - vs[2] + sv[2] - 1) / sv[2];
  for (int a = 0; a < 3; a++) rw->subVolDim[a] = sv[a];
  const int ntile = rw->ntx * rw->nty * rw->ntz;
  const int npad = ((n + chunk - 1) / chunk) * chunk;
  // per padded view: FP32 vectors; padded views (beyond n) are all-zero as in _padArrays
  std::vector<View32> V(npad);
  std::vector<int> woff(npad, 0), hoff(npad, 0);
  float mis[6];
  for (int i = 0; i < 6; i++) mis[i] = with_misalign ? (float)pb.mis[i] : 0.0f;
  for (int t = 0; t < npad; t++) {
    if (t < n) {
      V[t] = view32((float)pb.angle[t], (float)pb.hmid[t], vd[2], (float)pb.D, (float)pb.pw, mis);
      woff[t] = pb.woff[t];
      hoff[t] = pb.hoff[t];
    } else {
      memset(&V[t], 0, sizeof(View32));
    }
  }
  rw->ws.assign((size_t)ntile * n, 0);
  rw->hs.assign((size_t)ntile * n, 0);
  rw->sweepStart.assign((size_t)ntile * n, 0);
  rw->sweepSteps.assign((size_t)ntile * n, 0);
  std::vector<int> we0((size_t)ntile * npad), he0((size_t)ntile * npad);
  // continuous footprint of each (tile, view): the detector coordinates of the tile box
  std::vector<float> fw0((size_t)ntile * npad), fw1((size_t)ntile * npad);
  std::vector<float> fh0((size_t)ntile * npad), fh1((size_t)ntile * npad);
  int spd0 = 1, spd1 = 1;
  const int W0 = pb.projWHSize[0], W1 = pb.projWHSize[1];
  for (int k = 0; k < rw->ntz; k++)
    for (int j = 0; j < rw->nty; j++)
      for (int i = 0; i < rw->ntx; i++) {
        const int tile = (k * rw->nty + j) * rw->ntx + i;
        const float xx = (float)(i * sv[0] + vs[0]), yy = (float)(j * sv[1] + vs[1]), zz = (float)(k * sv[2] + vs[2]);
        for (int t = 0; t < npad; t++) {
          float wc[8], hc[8];
          const float xs[2] = {xx, xx + sv[0]}, ys[2] = {yy, yy + sv[1]}, zs[2] = {zz, zz + sv[2]};
          for (int c = 0; c < 8; c++)
            project_point(V[t], vd, pb.projDim, xs[c & 1], ys[(c >> 1) & 1], zs[(c >> 2) & 1], wc + c, hc + c);
          float a0 = wc[0], a1 = wc[0], b0 = hc[0], b1 = hc[0];
          for (int c = 1; c < 8; c++) {
            a0 = fminf(a0, wc[c]); a1 = fmaxf(a1, wc[c]);
            b0 = fminf(b0, hc[c]); b1 = fmaxf(b1, hc[c]);
          }
          fw0[(size_t)tile * npad + t] = a0; fw1[(size_t)tile * npad + t] = a1;
          fh0[(size_t)tile * npad + t] = b0; fh1[(size_t)tile * npad + t] = b1;
          int e[4] = {trunc_i(wc[0]), trunc_i(wc[0]) + 1, trunc_i(hc[0]), trunc_i(hc[0]) + 1};
          for (int c = 1; c < 8; c++) {
            e[0] = std::min(e[0], trunc_i(wc[c]));
            e[2] = std::min(e[2], trunc_i(hc[c]));
            e[1] = std::max(e[1], trunc_i(wc[c]) + 1);
            e[3] = std::max(e[3], trunc_i(hc[c]) + 1);
          }
          e[0] = std::max(e[0], woff[t] - 4);
          e[1] = std::max(e[1], woff[t] - 2);
          e[2] = std::max(e[2], hoff[t] - 4);
          e[3] = std::max(e[3], hoff[t] - 2);
          e[0] = std::min(e[0], woff[t] + W0 + 4);
          e[1] = std::min(e[1], woff[t] + W0 + 2);
          e[2] = std::min(e[2], hoff[t] + W1 + 4);
          e[3] = std::min(e[3], hoff[t] + W1 + 2);
          we0[(size_t)tile * npad + t] = e[0];
          he0[(size_t)tile * npad + t] = e[2];
          spd0 = std::max(spd0, e[1] - e[0]);
          spd1 = std::max(spd1, e[3] - e[2]);
        }
      }
  spd0 = 16 * (1 + spd0 / 16);
  spd1 = 16 * (1 + spd1 / 16);
  rw->subProjDim[0] = spd0;
  rw->subProjDim[1] = spd1;
  const double r = 0.55 * sqrt((double)(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]));
  rw->bp_matters = false;
  rw->proj_matters = false;
  for (int tile = 0; tile < ntile; tile++) {
    const int i = tile % rw->ntx, j = (tile / rw->ntx) % rw->nty, k = tile / (rw->ntx * rw->nty);
    const float xx = (float)(i * sv[0] + vs[0]), yy = (float)(j * sv[1] + vs[1]), zz = (float)(k * sv[2] + vs[2]);
    F3 c = f3((float)(xx + 0.5 * sv[0] - 0.5 * vd[0]), (float)(yy + 0.5 * sv[1] - 0.5 * vd[1]),
              (float)(zz + 0.5 * sv[2] - 0.5 * vd[2]));
    for (int t = 0; t < n; t++) {
      const size_t o = (size_t)tile * n + t;
      rw->ws[o] = we0[(size_t)tile * npad + t] - 8;
      rw->hs[o] = he0[(size_t)tile * npad + t] - 8;
      rw->sweepStart[o] = (int)(len(sub(c, V[t].s)) - r);
      rw->sweepSteps[o] = (int)(2.0 * r);
      const size_t q = (size_t)tile * npad + t;
      const int wlo = rw->ws[o], whi = rw->ws[o] + spd0 - 1;  // first / last window texel
      const int hlo = rw->hs[o], hhi = rw->hs[o] + spd1 - 1;
      // Backprojection: a coordinate beyond the window is clamped to the edge texel; that
      // equals the zero-extended value only when the edge texel lies outside the data.
      if ((fw0[q] < wlo && wlo > woff[t] - 1) || (fw1[q] > whi && whi < woff[t] + W0) ||
          (fh0[q] < hlo && hlo > hoff[t] - 1) || (fh1[q] > hhi && hhi < hoff[t] + W1))
        rw->bp_matters = true;
      // Projection: pixels outside the window receive nothing from this tile; its shadow
      // (footprint widened by two pixels for the zero ring) must stay inside the window
      // where it meets the data, and the sweep must cover the tile box widened by one voxel.
      if ((fw0[q] - 2 < wlo && wlo > woff[t]) || (fw1[q] + 2 > whi && whi < woff[t] + W0 - 1) ||
          (fh0[q] - 2 < hlo && hlo > hoff[t]) || (fh1[q] + 2 > hhi && hhi < hoff[t] + W1 - 1))
        rw->proj_matters = true;
      double dmin = 1e300, dmax = 0.0;
      for (int cc = 0; cc < 8; cc++) {
        const double px = xx - 1.0 + ((cc & 1) ? sv[0] + 1.0 : 0.0) - vd[0] / 2;
        const double py = yy - 1.0 + ((cc & 2) ? sv[1] + 1.0 : 0.0) - vd[1] / 2;
        const double pz = zz - 1.0 + ((cc & 4) ? sv[2] + 1.0 : 0.0) - vd[2] / 2;
        const double dx = px - V[t].s.x, dy = py - V[t].s.y, dz = pz - V[t].s.z;
        const double dd = sqrt(dx * dx + dy * dy + dz * dz);
        dmin = std::min(dmin, dd);
        dmax = std::max(dmax, dd);
      }
      (void)dmin;
      if (rw->sweepStart[o] > 0 && (double)(rw->sweepStart[o] + rw->sweepSteps[o] - 1) < dmax)
        rw->proj_matters = true;
    }
  }
  return FCB_OK;
}

}  // namespace fcb

// Inspection entry point: the restated windows of a geometry (see the header).
extern "C" int fcb_reference_windows(const fcb_geometry* g, int* subVolDim, int* subProjDim,
                                     int* tiles, int* ws, int* hs, int* sweepStart,
                                     int* sweepSteps, int* matters)
try {
  if (!g) return fcb::set_error(FCB_ERR_INVALID, "NULL geometry");
  fcb::Problem pb;
  FCB_TRY(fcb::make_problem(g, &pb));
  fcb::RefWindows rw;
  FCB_TRY(fcb::ref_windows(pb, true, &rw));
  for (int a = 0; a < 3; a++)
    if (subVolDim) subVolDim[a] = rw.subVolDim[a];
  if (subProjDim) { subProjDim[0] = rw.subProjDim[0]; subProjDim[1] = rw.subProjDim[1]; }
  if (tiles) { tiles[0] = rw.ntx; tiles[1] = rw.nty; tiles[2] = rw.ntz; }
  const size_t n = rw.ws.size();
  if (ws) memcpy(ws, rw.ws.data(), n * sizeof(int));
  if (hs) memcpy(hs, rw.hs.data(), n * sizeof(int));
  if (sweepStart) memcpy(sweepStart, rw.sweepStart.data(), n * sizeof(int));
  if (sweepSteps) memcpy(sweepSteps, rw.sweepSteps.data(), n * sizeof(int));
  if (matters) { matters[0] = rw.bp_matters ? 1 : 0; matters[1] = rw.proj_matters ? 1 : 0; }
  return fcb::ok();
}
FCB_CATCH_STATUS
