/*
 * fc_oracle.h -- CPU restatement of the Fastcone cone-beam operators.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load this library, and only as the checker / the timed CPU
 * baseline.  The product (fastcone_b200/) never calls it.
 *
 * Two families of functions:
 *
 *  orc_ref_*   "reference path": a restatement of what Fastcone itself computes, in
 *              FP32, including its sub-problem tiling (coneBeamGPU.cu:1509-1609), its
 *              per-view detector windows, its host window caches
 *              (coneBeamGPU.cu:1049-1172) and its hardware-texture sampling (linear
 *              filter, clamp addressing, +0.5 texel offset, interpolation weights in
 *              9-bit fixed point with 8 fractional bits -- `texq` = 1; `texq` = 0 uses
 *              exact FP32 weights).  Arguments follow the reference's C ABI
 *              (wrapper.c:112-249, unit_coneBeamGPU.cu:88-305): dimension arrays in
 *              [x,y,z] / [w,h,t] order, volume = the volStart..volEnd sub-array of a
 *              volDim grid, projections = per-view windows of projWHSize at
 *              (projWOffset[t], projHOffset[t]); results are ADDED to the outputs.
 *
 *  orc_*_f64   FP64 oracle: the same operators with FP64 geometry and arithmetic and
 *              exact interpolation weights, on the ideal support (projections and
 *              volumes extended by zeros, projector samples at every integer distance
 *              from the source that touches the volume).  This is the error reference
 *              every GPU result reports rel-L2 / max-abs against.
 *
 * Parity pins: the geometry/tiling restatement is compared bit-for-bit with the
 * reference's own host code built from its sources (oracle/_ref, see Makefile), and
 * the orc_ref_* operators with outputs of the reference's own CUDA path recorded on a
 * B200 (tests/golden/).
 */
#ifndef FC_ORACLE_H
#define FC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sub-problem decomposition of the reference (coneBeamGeometry), flattened. */
typedef struct {
  int subVolDim[3];
  int subProjDim[3];
  int numSubProblems;
  int nsp; /* number of view chunks */
} orc_tiling_info;

/* Restated coneBeamGeometry: returns tiling sizes; if the array pointers are non-NULL
 * they receive, per sub-problem, xx/yy/zz/ttStart, ww/hhStart[nsub*subProjDim2],
 * sweepStart/NumSteps[nsub*subProjDim2], and per padded view the geometry vectors
 * src/det/hstep/wstep[3*nviews_padded], hMidPlane/sina/cosa[nviews_padded]. */
int orc_ref_geometry(const int volDim[3], const int volStart[3], const int volEnd[3],
                     const int projDim[3], const int projWHSize[2],
                     const int* projWOffset, const int* projHOffset,
                     const float* angles, const float* hMid, float sourceSampleDistance,
                     const float* misAlignments, float pixelWidth,
                     orc_tiling_info* info,
                     int* xxStart, int* yyStart, int* zzStart, int* ttStart,
                     int* wwStart, int* hhStart, int* sweepStart, int* sweepNumSteps,
                     float* src, float* det, float* hstep, float* wstep,
                     float* hMidPlane, float* sina, float* cosa);

/* Reference path backprojection.  kernelMode 0 = unweighted (ray-trace, uses
 * misAlignments, may be NULL), 1 = Katsevich weight U, anything else = FDK weight U^2
 * (wrapper.c:134-143). */
int orc_ref_backproject(float* volume, const float* projections,
                        const int volDim[3], const int volStart[3], const int volEnd[3],
                        const int projDim[3], const int projWHSize[2],
                        const int* projWOffset, const int* projHOffset,
                        const float* angles, const float* hMid, float sourceSampleDistance,
                        const float* norm, float pixelWidth, int kernelMode,
                        const float* misAlignments, int texq);

/* Reference path forward projection (coneBeamProject); projections += norm * A vol.
 * Does NOT apply fastcone.py's zeroing of detector column 0 (a Python-layer step). */
int orc_ref_project(const float* volume, float* projections,
                    const int volDim[3], const int volStart[3], const int volEnd[3],
                    const int projDim[3], const int projWHSize[2],
                    const int* projWOffset, const int* projHOffset,
                    const float* angles, const float* hMid, float sourceSampleDistance,
                    const float* norm, const float* misAlignments, float pixelWidth,
                    int texq);

/* Reference-path FDK/Katsevich value at a list of global voxel indices (x,y,z triples);
 * out[i] = the amount the reference would add to that voxel.  Lets full-size configs
 * be checked on sampled voxels, and times the reference path on a bounded sample. */
int orc_ref_backproject_points(const int* xyz, int npts, float* out,
                               const float* projections,
                               const int volDim[3], const int volStart[3], const int volEnd[3],
                               const int projDim[3], const int projWHSize[2],
                               const int* projWOffset, const int* projHOffset,
                               const float* angles, const float* hMid,
                               float sourceSampleDistance, const float* norm,
                               float pixelWidth, int kernelMode, int texq);

/* ---------------- FP64 oracle ---------------- */

/* Voxel-driven backprojection, FP64: weight U^p with p = 2 (FDK), 1 (Katsevich) or the
 * unweighted plane-intersection form (p = 0; uses misAlignments, may be NULL).
 * vol (double, volStart..volEnd sub-array) += sum_t norm[t] * U^p * bilinear(P_t). */
int orc_backproject_f64(double* vol, const float* projections,
                        const int volDim[3], const int volStart[3], const int volEnd[3],
                        const int projDim[3], const int projWHSize[2],
                        const int* projWOffset, const int* projHOffset,
                        const float* angles, const float* hMid, double D,
                        const float* norm, double pw, int kernelMode,
                        const float* misAlignments);

/* Katsevich backprojection (weight U) restricted to each voxel's PI interval (the
 * Tam-Danielsson window on the virtual detector), FP64; *pairs = voxel-view pairs inside.
 * pitch = source rise per turn, voxels. */
int orc_katsevich_piwin_f64(double* vol, const float* projections,
                            const int volDim[3], const int volStart[3], const int volEnd[3],
                            const int projDim[3], const int projWHSize[2],
                            const int* projWOffset, const int* projHOffset,
                            const float* angles, const float* hMid, double D,
                            const float* norm, double pw, double pitch, int64_t* pairs);

/* orc_katsevich_piwin_f64 at listed voxels: out[n] for the voxel at global indices
 * xyz[3n..3n+2]; *pairs = the in-window voxel-view pairs of those voxels. */
int orc_katsevich_piwin_points_f64(const int* xyz, int npts, double* out,
                                   const float* projections,
                                   const int volDim[3], const int projDim[3],
                                   const int projWHSize[2], const int* projWOffset,
                                   const int* projHOffset, const float* angles,
                                   const float* hMid, double D, const float* norm, double pw,
                                   double pitch, int64_t* pairs);

int orc_backproject_points_f64(const int* xyz, int npts, double* out,
                               const float* projections,
                               const int volDim[3], const int volStart[3], const int volEnd[3],
                               const int projDim[3], const int projWHSize[2],
                               const int* projWOffset, const int* projHOffset,
                               const float* angles, const float* hMid, double D,
                               const float* norm, double pw, int kernelMode);

/* Ray-driven forward projection, FP64: proj += norm[t] * sum over integer m of
 * trilinear(vol, S + m d), d = unit vector source->pixel, vol extended by zeros. */
int orc_project_f64(const float* volume, double* projections,
                    const int volDim[3], const int volStart[3], const int volEnd[3],
                    const int projDim[3], const int projWHSize[2],
                    const int* projWOffset, const int* projHOffset,
                    const float* angles, const float* hMid, double D,
                    const float* norm, const float* misAlignments, double pw);

/* Exact transpose of orc_project_f64: vol += A^T (norm * proj). */
int orc_project_adjoint_f64(double* volume, const float* projections,
                            const int volDim[3], const int volStart[3], const int volEnd[3],
                            const int projDim[3], const int projWHSize[2],
                            const int* projWOffset, const int* projHOffset,
                            const float* angles, const float* hMid, double D,
                            const float* norm, const float* misAlignments, double pw);

/* Number of projector samples (integer-distance lattice points whose trilinear stencil
 * touches the volume box) summed over all rays: the Gsamples work count. */
int64_t orc_projector_sample_count(const int volDim[3], const int volStart[3],
                                   const int volEnd[3], const int projDim[3],
                                   const int projWHSize[2], const int* projWOffset,
                                   const int* projHOffset, const float* angles,
                                   const float* hMid, double D, double pw);

/* ---------------- phantoms ---------------- */

/* Ellipsoid phantom: params per ellipsoid = cx,cy,cz (voxel units from the volume
 * centre volDim/2), a,b,c semi-axes (voxels), 9 rotation-matrix entries (row-major,
 * body = R^T (p - c)), density -> 16 doubles.  Voxel value = sum of densities of the
 * ellipsoids containing the voxel centre. */
int orc_phantom_voxelize(float* vol, const int volDim[3], const double* params, int n);

/* Analytic line integral (voxel-length units) of the ellipsoid phantom along the
 * segment from point p0 in direction d (unit), over the whole line. */
double orc_phantom_line_integral(const double* params, int n, const double p0[3],
                                 const double d[3]);

#ifdef __cplusplus
}
#endif
#endif
