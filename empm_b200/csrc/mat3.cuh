// mat3.cuh — small 3-vector / 3x3 matrix helpers used by every kernel.
// Row-major 3x3 matrices held in registers; __host__ __device__ so the same
// code can be exercised on the CPU by the host-side debug hooks.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define EMPM_HD __host__ __device__ __forceinline__

struct V3 { float x, y, z; };
struct M3 { float m[9]; };   // m[3*r + c]

EMPM_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
EMPM_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
EMPM_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
EMPM_HD V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
EMPM_HD V3 operator*(V3 a, float s) { return v3(s * a.x, s * a.y, s * a.z); }
EMPM_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
EMPM_HD float length(V3 a) { return sqrtf(dot(a, a)); }
EMPM_HD V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
EMPM_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

EMPM_HD M3 m3_zero() { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = 0.f; return r; }
EMPM_HD M3 m3_identity() { M3 r = m3_zero(); r.m[0] = r.m[4] = r.m[8] = 1.f; return r; }
EMPM_HD M3 m3_diag(float a, float b, float c) { M3 r = m3_zero(); r.m[0] = a; r.m[4] = b; r.m[8] = c; return r; }
EMPM_HD M3 operator+(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] + b.m[i]; return r; }
EMPM_HD M3 operator-(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] - b.m[i]; return r; }
EMPM_HD M3 operator*(float s, const M3& a) { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = s * a.m[i]; return r; }
EMPM_HD M3 transpose(const M3& a) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[3 * j + i];
    return r;
}
EMPM_HD M3 operator*(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i + 0] * b.m[0 + j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
EMPM_HD V3 operator*(const M3& a, V3 v) {
    return v3(a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z,
              a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
              a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z);
}
EMPM_HD float det(const M3& a) {
    return a.m[0] * (a.m[4] * a.m[8] - a.m[5] * a.m[7])
         - a.m[1] * (a.m[3] * a.m[8] - a.m[5] * a.m[6])
         + a.m[2] * (a.m[3] * a.m[7] - a.m[4] * a.m[6]);
}
EMPM_HD M3 outer(V3 a, V3 b) {
    M3 r;
    r.m[0] = a.x * b.x; r.m[1] = a.x * b.y; r.m[2] = a.x * b.z;
    r.m[3] = a.y * b.x; r.m[4] = a.y * b.y; r.m[5] = a.y * b.z;
    r.m[6] = a.z * b.x; r.m[7] = a.z * b.y; r.m[8] = a.z * b.z;
    return r;
}
EMPM_HD float ddot(const M3& a, const M3& b) { float s = 0.f; for (int i = 0; i < 9; ++i) s += a.m[i] * b.m[i]; return s; }
EMPM_HD V3 col(const M3& a, int c) { return v3(a.m[c], a.m[3 + c], a.m[6 + c]); }

// ---- f9 plane access (three planes: float4 A, float4 B, float C) ----------
struct F9Planes {
    float4* a;
    float4* b;
    float*  c;
};
EMPM_HD F9Planes f9_planes(float* base, long long n) {
    F9Planes p;
    p.a = reinterpret_cast<float4*>(base);
    p.b = reinterpret_cast<float4*>(base) + n;
    p.c = reinterpret_cast<float*>(reinterpret_cast<float4*>(base) + 2 * n);
    return p;
}

#ifdef __CUDACC__
__device__ __forceinline__ M3 f9_load(const F9Planes& p, long long i) {
    float4 a = __ldg(p.a + i);
    float4 b = __ldg(p.b + i);
    float  c = __ldg(p.c + i);
    M3 r;
    r.m[0] = a.x; r.m[1] = a.y; r.m[2] = a.z; r.m[3] = a.w;
    r.m[4] = b.x; r.m[5] = b.y; r.m[6] = b.z; r.m[7] = b.w;
    r.m[8] = c;
    return r;
}
// Streaming stores: the particle planes are written once per substep and
// read once in the next; evict-first keeps the grid resident in L2.
__device__ __forceinline__ void f9_store(const F9Planes& p, long long i, const M3& r) {
    __stcs(p.a + i, make_float4(r.m[0], r.m[1], r.m[2], r.m[3]));
    __stcs(p.b + i, make_float4(r.m[4], r.m[5], r.m[6], r.m[7]));
    __stcs(p.c + i, r.m[8]);
}
#endif
