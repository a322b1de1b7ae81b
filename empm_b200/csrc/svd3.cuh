// svd3.cuh — 3x3 singular value decomposition in FP32.
//
// Method: one-sided (Hestenes) Jacobi orthogonalisation of the columns of A
// (M. R. Hestenes, "Inversion of matrices by biorthogonalization and related
// results", J. SIAM 6, 1958; rotation angle from the symmetric 2x2 Schur
// decomposition, Golub & Van Loan, Matrix Computations, Alg. 8.5.2), followed
// by column sorting and a Givens QR factorisation of B = A V so that U is a
// product of proper rotations.
//
// Convention (the one the reference's stress formulas assume, wp.svd3 at
// phys_sim/diff_simulator/warp_mpm/mpm_utils.py:92,140,197,244,641):
//   A = U diag(s) V^T,  U, V in SO(3),  s.x >= s.y >= |s.z|,
//   s.z carries the sign of det(A).
#pragma once
#include "mat3.cuh"

#ifndef EMPM_SVD_MAX_SWEEPS
#define EMPM_SVD_MAX_SWEEPS 8
#endif

namespace empm {

// Rotate the column pair (p, q) of the 3x3 column arrays b and v so that
// b_p and b_q become orthogonal. Returns false when they already are.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ float fast_rcp(float x) { return __fdividef(1.f, x); }
#else
inline float fast_rcp(float x) { return 1.f / x; }
inline float rsqrtf(float x) { return 1.f / sqrtf(x); }
#endif

EMPM_HD bool jacobi_pair(float b[3][3], float v[3][3], int p, int q) {
    const float alpha = b[p][0] * b[p][0] + b[p][1] * b[p][1] + b[p][2] * b[p][2];
    const float beta  = b[q][0] * b[q][0] + b[q][1] * b[q][1] + b[q][2] * b[q][2];
    const float gamma = b[p][0] * b[q][0] + b[p][1] * b[q][1] + b[p][2] * b[q][2];
    // relative orthogonality |gamma| <= tol * sqrt(alpha * beta), squared; also true for a zero column
    if (gamma * gamma <= (1.6e-13f * alpha) * beta) return false;
    const float zeta = (beta - alpha) * fast_rcp(2.f * gamma);
    float t;
    const float az = fabsf(zeta);
    if (az > 1e15f) {
        t = fast_rcp(2.f * zeta);
    } else {
        const float h = 1.f + zeta * zeta;
        t = copysignf(fast_rcp(az + h * rsqrtf(h)), zeta);   // sign(zeta) / (|zeta| + sqrt(1 + zeta^2))
    }
    const float c = rsqrtf(1.f + t * t);
    const float s = c * t;
    for (int r = 0; r < 3; ++r) {
        const float bp = b[p][r], bq = b[q][r];
        b[p][r] = c * bp - s * bq;
        b[q][r] = s * bp + c * bq;
        const float vp = v[p][r], vq = v[q][r];
        v[p][r] = c * vp - s * vq;
        v[q][r] = s * vp + c * vq;
    }
    return true;
}

EMPM_HD void swap_cols(float a[3][3], int i, int j) {
    for (int r = 0; r < 3; ++r) { const float t = a[i][r]; a[i][r] = a[j][r]; a[j][r] = t; }
}

// Givens rotation on rows (p, q) of the row-major matrix m that zeroes
// m[q][c] using the pivot m[p][c]; the same rotation is folded into the
// columns of u (u accumulates G^T, so that m_original = u * m).
EMPM_HD void givens_rows(float m[3][3], float u[3][3], int p, int q, int c) {
    const float a = m[p][c], b = m[q][c];
    const float r2 = a * a + b * b;
    if (r2 == 0.f) return;
    const float inv = rsqrtf(r2);
    const float cs = a * inv, sn = b * inv;
    for (int k = 0; k < 3; ++k) {
        const float mp = m[p][k], mq = m[q][k];
        m[p][k] = cs * mp + sn * mq;
        m[q][k] = -sn * mp + cs * mq;
    }
    for (int k = 0; k < 3; ++k) {  // u is row-major: column ops on u[k][p], u[k][q]
        const float up = u[k][p], uq = u[k][q];
        u[k][p] = cs * up + sn * uq;
        u[k][q] = -sn * up + cs * uq;
    }
    m[q][c] = 0.f;
}

EMPM_HD void svd3(const M3& A, M3& U, V3& s, M3& V) {
    // b[c][r] = column c of B = A V, v[c][r] = column c of V
    float b[3][3], v[3][3];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) {
            b[c][r] = A.m[3 * r + c];
            v[c][r] = (r == c) ? 1.f : 0.f;
        }
    for (int sweep = 0; sweep < EMPM_SVD_MAX_SWEEPS; ++sweep) {
        bool rot = jacobi_pair(b, v, 0, 1);
        rot |= jacobi_pair(b, v, 0, 2);
        rot |= jacobi_pair(b, v, 1, 2);
        if (!rot) break;
    }
    // sort columns by decreasing norm
    float n0 = b[0][0] * b[0][0] + b[0][1] * b[0][1] + b[0][2] * b[0][2];
    float n1 = b[1][0] * b[1][0] + b[1][1] * b[1][1] + b[1][2] * b[1][2];
    float n2 = b[2][0] * b[2][0] + b[2][1] * b[2][1] + b[2][2] * b[2][2];
    if (n0 < n1) { swap_cols(b, 0, 1); swap_cols(v, 0, 1); const float t = n0; n0 = n1; n1 = t; }
    if (n0 < n2) { swap_cols(b, 0, 2); swap_cols(v, 0, 2); const float t = n0; n0 = n2; n2 = t; }
    if (n1 < n2) { swap_cols(b, 1, 2); swap_cols(v, 1, 2); const float t = n1; n1 = n2; n2 = t; }
    // make V a proper rotation (flip its last column together with B's)
    const float detv =
        v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) -
        v[1][0] * (v[0][1] * v[2][2] - v[0][2] * v[2][1]) +
        v[2][0] * (v[0][1] * v[1][2] - v[0][2] * v[1][1]);
    if (detv < 0.f) {
        for (int r = 0; r < 3; ++r) { v[2][r] = -v[2][r]; b[2][r] = -b[2][r]; }
    }
    // QR of B (row-major copy) by Givens: B = U R, R ~ diag(s)
    float m[3][3], u[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            m[r][c] = b[c][r];
            u[r][c] = (r == c) ? 1.f : 0.f;
        }
    givens_rows(m, u, 0, 1, 0);
    givens_rows(m, u, 0, 2, 0);
    givens_rows(m, u, 1, 2, 1);
    s = v3(m[0][0], m[1][1], m[2][2]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            U.m[3 * r + c] = u[r][c];
            V.m[3 * r + c] = v[c][r];
        }
}

}  // namespace empm
