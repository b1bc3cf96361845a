/*
 * Minimal float2/float3/float4 operator header used ONLY to compile the
 * reference sources under oracle/_ref (test infrastructure, never shipped).
 *
 * The reference includes <cutil_math.h> from the retired CUDA SDK, which is
 * not present in CUDA 12.9.  This header supplies just the operators and
 * helpers the reference uses (make_floatN(scalar), +, -, *, /, +=, dot,
 * normalize), written from their mathematical definitions.  normalize uses
 * rsqrtf on the device like the old SDK helper did; on the host it uses
 * 1/sqrtf.
 */
#ifndef ORACLE_REF_SHIM_CUTIL_MATH_H
#define ORACLE_REF_SHIM_CUTIL_MATH_H

#include <cuda_runtime.h>
#include <math.h>

/*
 * The reference uploads its parameter block with
 *     cudaMemcpyToSymbol((char *)&dev_param, host_param, sizeof(SysParam));
 * (SPH-3D-2/sph_system.cu:36).  Under the CUDA 3/4 runtime it was written
 * for, a char* argument was the symbol address itself.  Under CUDA 12 that
 * call binds to the template overload, which takes the address of the
 * temporary pointer instead, fails with an invalid-symbol error and leaves
 * dev_param zeroed (cell_size 0 -> every hash saturates -> out-of-bounds
 * cell writes).  This exact-match overload restores the old meaning so the
 * unmodified source uploads its constants.
 */
static inline cudaError_t cudaMemcpyToSymbol(char *symbol, const void *src, size_t count)
{
    return ::cudaMemcpyToSymbol((const void *)symbol, src, count, 0, cudaMemcpyHostToDevice);
}

#define SHIM_HD __host__ __device__ inline

SHIM_HD float2 make_float2(float s) { return make_float2(s, s); }
SHIM_HD float3 make_float3(float s) { return make_float3(s, s, s); }
SHIM_HD float4 make_float4(float s) { return make_float4(s, s, s, s); }

/* float2 */
SHIM_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
SHIM_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
SHIM_HD float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
SHIM_HD float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
SHIM_HD float2 operator*(float s, float2 a) { return make_float2(a.x * s, a.y * s); }
SHIM_HD float2 operator*(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
SHIM_HD float2 operator/(float2 a, float s) { return make_float2(a.x / s, a.y / s); }
SHIM_HD float2 operator/(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }
SHIM_HD void operator+=(float2 &a, float2 b) { a.x += b.x; a.y += b.y; }
SHIM_HD void operator-=(float2 &a, float2 b) { a.x -= b.x; a.y -= b.y; }
SHIM_HD float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }

/* float3 */
SHIM_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
SHIM_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
SHIM_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
SHIM_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
SHIM_HD float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
SHIM_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
SHIM_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
SHIM_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
SHIM_HD void operator+=(float3 &a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
SHIM_HD void operator-=(float3 &a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
SHIM_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

SHIM_HD float3 normalize(float3 v)
{
#ifdef __CUDA_ARCH__
    float inv = rsqrtf(dot(v, v));
#else
    float inv = 1.0f / sqrtf(dot(v, v));
#endif
    return v * inv;
}

/* float4 */
SHIM_HD float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
SHIM_HD float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
SHIM_HD void operator+=(float4 &a, float4 b) { a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w; }

#endif
