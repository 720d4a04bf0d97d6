/*
 * Stand-in for the CUDA SDK <= 4.x header `cutil_math.h`, which the reference's
 * coneBeamGPU.cu includes (coneBeamGPU.cu:46) and which no current CUDA toolkit
 * ships.  It supplies only the float3 vector operators that translation unit uses:
 * + - * with scalars, the compound forms, dot, cross, length and normalize.
 *
 * Test infrastructure: used only to build the reference from its own sources into
 * oracle/_ref/ so that the CPU restatement can be checked against it.
 */
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define FCREF_HD __host__ __device__ inline

FCREF_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
FCREF_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
FCREF_HD float3 operator-(float3 a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
FCREF_HD float3 operator+(float3 a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
FCREF_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
FCREF_HD float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
FCREF_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
FCREF_HD void operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
FCREF_HD void operator-=(float3& a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
FCREF_HD void operator*=(float3& a, float s) { a.x *= s; a.y *= s; a.z *= s; }
FCREF_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FCREF_HD float3 cross(float3 a, float3 b)
{
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
FCREF_HD float length(float3 a) { return sqrtf(dot(a, a)); }
FCREF_HD float3 normalize(float3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
