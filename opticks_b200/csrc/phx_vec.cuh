// phx_vec.cuh : float3 helpers for the device kernels.
//
// The photon physics is compared bit for bit with the reference build, so these helpers keep
// the operation order of the CUDA SDK "sutil" vector conventions that the reference compiles
// against (sysrap/scuda.h:437-627): dot is x*x' + y*y' + z*z' evaluated left to right, a
// vector divided by a scalar is a multiply by the reciprocal, normalize multiplies by
// 1/sqrtf(dot).  The library is always compiled with --use_fast_math, like the reference
// (cmake/Modules/OpticksCUDAFlags.cmake:95), so sqrtf/sinf/logf are the fast forms in both.
#pragma once
#include <cuda_runtime.h>

#define PHX_D __device__ __forceinline__

// Cold paths (generation, scattering, rare leaves) are called out of line so the hot bounce loop
// stays small enough for the instruction cache; PHX_OUTLINE=0 inlines everything (A/B builds).
#ifndef PHX_OUTLINE
#define PHX_OUTLINE 1
#endif
#if PHX_OUTLINE
#define PHX_COLD __device__ __noinline__
#else
#define PHX_COLD __device__ __forceinline__
#endif

#ifndef PHX_PI_F
#define PHX_PI_F 3.14159265358979323846f
#endif

PHX_D float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
PHX_D float3 f3s(float s) { return make_float3(s, s, s); }
PHX_D float3 operator+(const float3& a, const float3& b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
PHX_D float3 operator-(const float3& a, const float3& b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
PHX_D float3 operator-(const float3& a) { return make_float3(-a.x, -a.y, -a.z); }
PHX_D float3 operator*(const float3& a, const float3& b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
PHX_D float3 operator*(const float3& a, const float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
PHX_D float3 operator*(const float s, const float3& a) { return make_float3(a.x * s, a.y * s, a.z * s); }
PHX_D float3 operator/(const float3& a, const float s) { float inv = 1.0f / s; return a * inv; }
PHX_D float3 operator/(const float3& a, const float3& b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
PHX_D void operator+=(float3& a, const float3& b) { a.x += b.x; a.y += b.y; a.z += b.z; }
PHX_D float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PHX_D float3 cross(const float3& a, const float3& b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PHX_D float length(const float3& v) { return sqrtf(dot(v, v)); }
PHX_D float3 normalize(const float3& v) { float invLen = 1.0f / sqrtf(dot(v, v)); return v * invLen; }
PHX_D float3 fminf3(const float3& a, const float3& b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
PHX_D float3 fmaxf3(const float3& a, const float3& b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
PHX_D float hmin(const float3& a) { return fminf(fminf(a.x, a.y), a.z); }
PHX_D float hmax(const float3& a) { return fmaxf(fmaxf(a.x, a.y), a.z); }

PHX_D float2 operator-(const float2& a, const float2& b) { return make_float2(a.x - b.x, a.y - b.y); }
PHX_D float dot2(const float2& a, const float2& b) { return a.x * b.x + a.y * b.y; }
PHX_D float2 normalize2(const float2& v) { float invLen = 1.0f / sqrtf(dot2(v, v)); return make_float2(v.x * invLen, v.y * invLen); }

// row-vector transform by a 4x4 stored as four float4 rows (q0..q3): v' = v * M (w = 1 point, 0 dir)
PHX_D float3 xform_row(const float4* q, const float3& v, float w)
{
    float3 r;
    r.x = q[0].x * v.x + q[1].x * v.y + q[2].x * v.z + q[3].x * w;
    r.y = q[0].y * v.x + q[1].y * v.y + q[2].y * v.z + q[3].y * w;
    r.z = q[0].z * v.x + q[1].z * v.y + q[2].z * v.z + q[3].z * w;
    return r;
}
// column transform: v' = M * v using the upper 3x4 (used for normals with the inverse matrix)
PHX_D float3 xform_col(const float4* q, const float3& v, float w)
{
    float3 r;
    r.x = q[0].x * v.x + q[0].y * v.y + q[0].z * v.z + q[0].w * w;
    r.y = q[1].x * v.x + q[1].y * v.y + q[1].z * v.z + q[1].w * w;
    r.z = q[2].x * v.x + q[2].y * v.y + q[2].z * v.z + q[2].w * w;
    return r;
}

// CLHEP Hep3Vector::rotateUz: rotate frame so that z goes along unit vector u.
// Same float operation order as sysrap/smath.h:95-112 which restates CLHEP.
PHX_D void rotate_uz(float3& d, const float3& u)
{
    float up = u.x * u.x + u.y * u.y;
    if (up > 0.f) {
        up = sqrtf(up);
        float px = d.x, py = d.y, pz = d.z;
        d.x = (u.x * u.z * px - u.y * py) / up + u.x * pz;
        d.y = (u.y * u.z * px + u.x * py) / up + u.y * pz;
        d.z = -up * px + u.z * pz;
    } else if (u.z < 0.f) {
        d.x = -d.x;
        d.z = -d.z;
    }
}
