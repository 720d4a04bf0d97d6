/*
 * ref_driver.cu -- thin extern "C" entry points onto the reference's OWN code, built
 * from its unmodified sources (coneBeamGPU.cu, unit_coneBeamGPU.cu) into
 * oracle/_ref/libfastcone_ref.so by oracle/Makefile.  Test infrastructure only.
 *
 *  fcref_geometry      constructs the reference's coneBeamGeometry
 *                      (coneBeamGPU.cu:1360-1849) and copies out its tiling, windows,
 *                      sweeps and per-view vectors -- pure host code, runs without a GPU;
 *  fcref_backproject   dispatches exactly as GPU_CB_K_backproject (wrapper.c:112-146):
 *                      mode 0 -> coneBeamRayTraceBackproject with zero misalignments,
 *                      else coneBeamBackproject (1 = Katsevich, other = FDK); needs a GPU;
 *  fcref_project       coneBeamProject (unit_coneBeamGPU.cu:88-171); needs a GPU.
 *
 * wrapper.c itself is not built: its GPU_CB_misalign_project passes callbacks that exist
 * nowhere (wrapper.c:224).  cudaCleanup()/setDeviceNumber() are not called: the first
 * resets the context after every call (unit_coneBeamGPU.cu:63-67), the second exits the
 * process on a bad id; the current device is used instead.
 */
#include <string.h>
#include "coneBeamGPU.h"
#include "unit_coneBeamGPU.h"

/* unit_coneBeamGPU.h:70-85 declares coneBeamProject without pixelWidth, but the
 * definition (unit_coneBeamGPU.cu:88-103) has it, so it carries a C++-mangled symbol. */
int coneBeamProject(float* volume, float* projections, int volDim[3], int volStart[3],
                    int volEnd[3], int projDim[3], int projWHSize[2], int* projWOffset,
                    int* projHOffset, float* angles, float* hMidPlane,
                    float sourceSampleDistance, float* normalizationFactor,
                    float* misAlignments, float pixelWidth);

extern "C" {

int fcref_geometry(int* volDim, int* volStart, int* volEnd, int* projDim, int* projWHSize,
                   int* projWOffset, int* projHOffset, float* angles, float* hMid,
                   float sourceSampleDistance, float* misAlignments, float pixelWidth,
                   int* sizes /* subVolDim[3], subProjDim[3], numSubProblems */,
                   int* xxStart, int* yyStart, int* zzStart, int* ttStart, int* wwStart,
                   int* hhStart, int* sweepStart, int* sweepNumSteps, float* src, float* det,
                   float* hstep, float* wstep, float* hMidPlane, float* sina, float* cosa,
                   int capacity_sub, int capacity_views)
{
  float zeros[6] = {0, 0, 0, 0, 0, 0};
  coneBeamGeometry g(volDim, projDim, volStart, volEnd, projWHSize, projWOffset, projHOffset,
                     angles, hMid, sourceSampleDistance, misAlignments ? misAlignments : zeros,
                     pixelWidth);
  for (int i = 0; i < 3; i++) {
    sizes[i] = g.subVolDim[i];
    sizes[3 + i] = g.subProjDim[i];
  }
  sizes[6] = g.numSubProblems;
  int ns = g.numSubProblems, n2 = g.subProjDim[2];
  int np = ((projDim[2] + n2 - 1) / n2) * n2;
  if (ns > capacity_sub || np > capacity_views) return -1;
  for (int p = 0; p < ns; p++) {
    xxStart[p] = g.xxStart[p];
    yyStart[p] = g.yyStart[p];
    zzStart[p] = g.zzStart[p];
    ttStart[p] = g.ttStart[p];
    for (int t = 0; t < n2; t++) {
      wwStart[p * n2 + t] = g.wwStart[p][t];
      hhStart[p * n2 + t] = g.hhStart[p][t];
      sweepStart[p * n2 + t] = g.sweepStart[p][t];
      sweepNumSteps[p * n2 + t] = g.sweepNumSteps[p][t];
    }
  }
  memcpy(src, g.sourcePosition_xyz, 3 * np * sizeof(float));
  memcpy(det, g.detectorCentre_xyz, 3 * np * sizeof(float));
  memcpy(hstep, g.hStep_xyz, 3 * np * sizeof(float));
  memcpy(wstep, g.wStep_xyz, 3 * np * sizeof(float));
  memcpy(hMidPlane, g.hMidPlane, np * sizeof(float));
  memcpy(sina, g.sina, np * sizeof(float));
  memcpy(cosa, g.cosa, np * sizeof(float));
  return 0;
}

int fcref_backproject(float* volume, float* projections, float* angles, float* hMidPlane,
                      float sourceSampleDistance, float pixelWidth, int* volDim, int* volStart,
                      int* volEnd, int* projDim, int* projWHSize, int* projWOffset,
                      int* projHOffset, float* normalizationFactor, int kernelMode)
{
  int rc;
  if (kernelMode == 0) {
    float mis[6] = {0, 0, 0, 0, 0, 0};
    rc = coneBeamRayTraceBackproject(volume, projections, volDim, volStart, volEnd, projDim,
                                     projWHSize, projWOffset, projHOffset, angles, hMidPlane,
                                     sourceSampleDistance, normalizationFactor, mis, pixelWidth);
  } else {
    rc = coneBeamBackproject(volume, projections, volDim, volStart, volEnd, projDim, projWHSize,
                             projWOffset, projHOffset, angles, hMidPlane, sourceSampleDistance,
                             normalizationFactor, pixelWidth, kernelMode);
  }
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? rc : -(int)e;
}

int fcref_project(float* volume, float* projections, float* angles, float* hMidPlane,
                  float sourceSampleDistance, float pixelWidth, int* volDim, int* volStart,
                  int* volEnd, int* projDim, int* projWHSize, int* projWOffset, int* projHOffset,
                  float* normalizationFactor, float* misAlignments)
{
  float zeros[6] = {0, 0, 0, 0, 0, 0};
  int rc = coneBeamProject(volume, projections, volDim, volStart, volEnd, projDim, projWHSize,
                           projWOffset, projHOffset, angles, hMidPlane, sourceSampleDistance,
                           normalizationFactor, misAlignments ? misAlignments : zeros, pixelWidth);
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? rc : -(int)e;
}

}  // extern "C"
