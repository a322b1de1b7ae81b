// dual.cuh — forward-mode dual numbers with N tangent directions.
//
// The adjoint of the constitutive update needs the Jacobian of a small
// spectral map (three singular values plus mu, lam and the yield stress in,
// three elastic singular values, three stress eigenvalues and the updated
// material scalars out). Evaluating the same templated code with Dual<6>
// gives all of it in one pass; evaluated with float it is the forward map.
// Branches compare values only, so a dual evaluation takes the same branch as
// the float evaluation of the same inputs.
#pragma once
#include "mat3.cuh"

namespace empm {

template <int N>
struct Dual {
    float v;
    float d[N];
};

template <int N>
EMPM_HD Dual<N> dconst(float v) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.f;
    return r;
}

template <int N>
EMPM_HD Dual<N> dseed(float v, int k) {
    Dual<N> r = dconst<N>(v);
    r.d[k] = 1.f;
    return r;
}

template <int N> EMPM_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> EMPM_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> EMPM_HD Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r; r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> EMPM_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> EMPM_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v / b.v;
    const float ib = 1.f / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> EMPM_HD Dual<N> operator+(const Dual<N>& a, float b) { Dual<N> r = a; r.v = a.v + b; return r; }
template <int N> EMPM_HD Dual<N> operator+(float b, const Dual<N>& a) { return a + b; }
template <int N> EMPM_HD Dual<N> operator-(const Dual<N>& a, float b) { Dual<N> r = a; r.v = a.v - b; return r; }
template <int N> EMPM_HD Dual<N> operator-(float b, const Dual<N>& a) { return -(a - b); }
template <int N> EMPM_HD Dual<N> operator*(const Dual<N>& a, float s) {
    Dual<N> r; r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N> EMPM_HD Dual<N> operator*(float s, const Dual<N>& a) { return a * s; }
template <int N> EMPM_HD Dual<N> operator/(const Dual<N>& a, float s) {
    Dual<N> r; r.v = a.v / s;
    const float is = 1.f / s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * is;
    return r;
}
template <int N> EMPM_HD Dual<N> operator/(float a, const Dual<N>& b) { return dconst<N>(a) / b; }

// scalar functions, overloaded for float and Dual so the constitutive code
// can be written once
EMPM_HD float sval(float a) { return a; }
template <int N> EMPM_HD float sval(const Dual<N>& a) { return a.v; }

EMPM_HD float slog(float a) { return logf(a); }
EMPM_HD float sexp(float a) { return expf(a); }
EMPM_HD float ssqrt(float a) { return sqrtf(a); }
EMPM_HD float spow(float a, float c) { return powf(a, c); }
EMPM_HD float smaxc(float a, float c) { return fmaxf(a, c); }   // max with a constant
EMPM_HD float sabs(float a) { return fabsf(a); }

template <int N> EMPM_HD Dual<N> slog(const Dual<N>& a) {
    Dual<N> r; r.v = logf(a.v);
    const float ia = 1.f / a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * ia;
    return r;
}
template <int N> EMPM_HD Dual<N> sexp(const Dual<N>& a) {
    Dual<N> r; r.v = expf(a.v);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * r.v;
    return r;
}
template <int N> EMPM_HD Dual<N> ssqrt(const Dual<N>& a) {
    Dual<N> r; r.v = sqrtf(a.v);
    const float h = r.v > 0.f ? 0.5f / r.v : 0.f;   // the derivative at 0 is taken as 0
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> EMPM_HD Dual<N> spow(const Dual<N>& a, float c) {
    Dual<N> r; r.v = powf(a.v, c);
    const float g = c * powf(a.v, c - 1.f);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * g;
    return r;
}
template <int N> EMPM_HD Dual<N> smaxc(const Dual<N>& a, float c) {
    return a.v >= c ? a : dconst<N>(c);   // NaN selects c, as fmaxf does
}
template <int N> EMPM_HD Dual<N> sabs(const Dual<N>& a) { return a.v < 0.f ? -a : a; }

}  // namespace empm
