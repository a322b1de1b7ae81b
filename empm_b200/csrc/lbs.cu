// lbs.cu — moving rendered Gaussians with the simulated particles: linear
// blend skinning over particle "bones", plus the neighbour searches feeding it.
//
// The reference moves every Gaussian of the scene once per rendered frame
// (phys_sim/engine/trainer_warp_mpm.py:1626-1659, scripts/interactive_viser.py:
// 258-275, scripts/gs/gs_render_dynamics.py:239-262) with the functions of
// third_party/gaussian_splatting/dynamic_utils.py:
//   * get_topk_indices (:248-265) and knn_weights_sparse (:295-302): exact
//     k nearest neighbours (bones among bones without themselves; bones of
//     each Gaussian), by dense distance matrices and torch.topk;
//   * calc_weights_vals_from_indices (:282-292): w = 1 / (|x - b| + 1e-6),
//     normalised over the k bones of the Gaussian;
//   * interpolate_motions_speedup (:305-491): per bone, the rotation that best
//     maps the offsets to its neighbours before the step onto the offsets
//     after it (SVD of F = sum_j new_j old_j^T, proper rotation U V^T), then
//     per Gaussian x' = sum_k w_k (R_k (x - b_k) + m_k + b_k) and a
//     quaternion q' = normalize(sum_k w_k q(R_k)) * q;
//   * interpolate_motions (:67-216): the same with dense [n, n_bones]
//     weights (inverse distance to every bone when none are given).
//
// Here the bone stage is two launches over bones (fit; resolve + quaternion)
// that leave a 16-float table per bone, and the Gaussian stage is one launch
// that gathers its k table rows. The bone table is small and stays in L2; the
// Gaussian stage streams its rows once, so it is bound by HBM bandwidth.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>
#include <string.h>
#include "../../include/empm_b200.h"
#include "ctx.hpp"
#include "mat3.cuh"
#include "svd3.cuh"

using namespace empm;

namespace {

inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

#define CKB(expr, what)                                                          \
    do {                                                                         \
        int _rc = empm_check_cuda(nullptr, (expr), what);                        \
        if (_rc != EMPM_OK) return _rc;                                          \
    } while (0)

// status bits
constexpr int kBadIndex = 1;

// counts[] written by the fit stage (device ints, zeroed by the caller entry)
enum { kRank0 = 0, kRank1 = 1, kRank23 = 2, kRank1NotClose = 3, kLastRank1 = 4, kLastRank23 = 5, kStatus = 6 };

__device__ __forceinline__ V3 load3(const float* a, long long i) {
    return v3(__ldg(a + 3 * i), __ldg(a + 3 * i + 1), __ldg(a + 3 * i + 2));
}

template <typename IdxT>
__device__ __forceinline__ long long load_idx(const IdxT* a, long long i) { return (long long)__ldg(a + i); }

// ---------------------------------------------------------------------------
// quaternions (w, x, y, z) of rotation matrices
// ---------------------------------------------------------------------------
// kornia 0.8.1 rotation_matrix_to_quaternion (eps = 1e-8), the conversion
// the sparse path calls (dynamic_utils.py:465-475): trace > 0 picks w as the
// pivot, otherwise the largest diagonal entry; divisions clamp the divisor at
// the smallest normal float.
__device__ __forceinline__ float sdiv(float num, float den) { return num / fmaxf(den, FLT_MIN); }

__device__ float4 quat_kornia(const M3& R) {
    const float m00 = R.m[0], m01 = R.m[1], m02 = R.m[2];
    const float m10 = R.m[3], m11 = R.m[4], m12 = R.m[5];
    const float m20 = R.m[6], m21 = R.m[7], m22 = R.m[8];
    const float eps = 1e-8f;
    const float trace = m00 + m11 + m22;
    if (trace > 0.f) {
        const float sq = sqrtf(trace + 1.f + eps) * 2.f;
        return make_float4(0.25f * sq, sdiv(m21 - m12, sq), sdiv(m02 - m20, sq), sdiv(m10 - m01, sq));
    }
    if (m00 > m11 && m00 > m22) {
        const float sq = sqrtf(1.f + m00 - m11 - m22 + eps) * 2.f;
        return make_float4(sdiv(m21 - m12, sq), 0.25f * sq, sdiv(m01 + m10, sq), sdiv(m02 + m20, sq));
    }
    if (m11 > m22) {
        const float sq = sqrtf(1.f + m11 - m00 - m22 + eps) * 2.f;
        return make_float4(sdiv(m02 - m20, sq), sdiv(m01 + m10, sq), 0.25f * sq, sdiv(m12 + m21, sq));
    }
    const float sq = sqrtf(1.f + m22 - m00 - m11 + eps) * 2.f;
    return make_float4(sdiv(m10 - m01, sq), sdiv(m02 + m20, sq), sdiv(m12 + m21, sq), 0.25f * sq);
}

// The reference's own mat2quat (dynamic_utils.py:25-64), used by the dense
// path (:209) and as the sparse path's fallback: the w pivot whenever the
// trace (clamped at -1) is above -1. Its other branches are kept as written,
// including the pivot component 0.5 * (0.5 / sqrt(.)) of :42,51,60.
__device__ float4 quat_mat2quat(const M3& R) {
    const float r00 = R.m[0], r01 = R.m[1], r02 = R.m[2];
    const float r10 = R.m[3], r11 = R.m[4], r12 = R.m[5];
    const float r20 = R.m[6], r21 = R.m[7], r22 = R.m[8];
    const float t = fmaxf(r00 + r11 + r22, -1.f);
    if (t > -1.f) {
        const float s = sqrtf(t + 1.f);
        const float f = 0.5f / s;
        return make_float4(0.5f * s, (r21 - r12) * f, (r02 - r20) * f, (r10 - r01) * f);
    }
    if (r00 >= r11 && r00 >= r22) {
        const float f = 0.5f / sqrtf(1.f + r00 - r11 - r22);
        return make_float4((r21 - r12) * f, 0.5f * f, (r10 + r01) * f, (r20 + r02) * f);
    }
    if (r11 >= r22 && r11 > r00) {
        const float f = 0.5f / sqrtf(1.f + r11 - r00 - r22);
        return make_float4((r02 - r20) * f, (r21 + r12) * f, 0.5f * f, (r01 + r10) * f);
    }
    const float f = 0.5f / sqrtf(1.f + r22 - r00 - r11);
    return make_float4((r10 - r01) * f, (r02 + r20) * f, (r12 + r21) * f, 0.5f * f);
}

// torch.nn.functional.normalize: q / max(|q|, 1e-12)
__device__ __forceinline__ float4 normalize4(float4 q) {
    const float n = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
    return make_float4(q.x / n, q.y / n, q.z / n, q.w / n);
}

__device__ __forceinline__ float4 quat_of(const M3& R, int convention) {
    return convention == EMPM_QUAT_MAT2QUAT ? quat_mat2quat(R) : quat_kornia(R);
}

// Hamilton product with (w, x, y, z) components (quaternion_multiply,
// dynamic_utils.py:449-457)
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    return make_float4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
                       a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                       a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y,
                       a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
}

// ---------------------------------------------------------------------------
// k nearest neighbours: one query per thread, candidates staged through
// shared memory, the KT best kept sorted in registers
// ---------------------------------------------------------------------------
constexpr int kKnnThreads = 128;
constexpr int kKnnTile = 1024;

template <int KT, typename IdxT>
__global__ void __launch_bounds__(kKnnThreads) k_knn(const float* __restrict__ q, int nq, const float* __restrict__ pts,
                                                     int np, int k, int exclude_self, IdxT* __restrict__ out_idx,
                                                     float* __restrict__ out_dist) {
    __shared__ float4 tile[kKnnTile];
    const int i = blockIdx.x * kKnnThreads + threadIdx.x;
    const bool live = i < nq;
    float qx = 0.f, qy = 0.f, qz = 0.f;
    if (live) { qx = __ldg(q + 3 * (long long)i); qy = __ldg(q + 3 * (long long)i + 1); qz = __ldg(q + 3 * (long long)i + 2); }
    float bd[KT];
    int bi[KT];
#pragma unroll
    for (int s = 0; s < KT; ++s) { bd[s] = INFINITY; bi[s] = -1; }
    const int self = (live && exclude_self) ? i : -1;
    for (int base = 0; base < np; base += kKnnTile) {
        const int m = min(kKnnTile, np - base);
        __syncthreads();
        for (int t = threadIdx.x; t < m; t += kKnnThreads) {
            const long long j = base + t;
            tile[t] = make_float4(__ldg(pts + 3 * j), __ldg(pts + 3 * j + 1), __ldg(pts + 3 * j + 2), 0.f);
        }
        __syncthreads();
        for (int t = 0; t < m; ++t) {
            const float4 p = tile[t];
            const float dx = qx - p.x, dy = qy - p.y, dz = qz - p.z;
            const float d = dx * dx + dy * dy + dz * dz;
            const int j = base + t;
            if (d < bd[KT - 1] && j != self) {
                // insertion keeps equal distances in index order (strict <)
#pragma unroll
                for (int s = KT - 1; s > 0; --s) {
                    if (d < bd[s - 1]) { bd[s] = bd[s - 1]; bi[s] = bi[s - 1]; }
                    else if (d < bd[s]) { bd[s] = d; bi[s] = j; }
                }
                if (d < bd[0]) { bd[0] = d; bi[0] = j; }
            }
        }
    }
    if (!live) return;
#pragma unroll
    for (int s = 0; s < KT; ++s) {
        if (s < k) {
            out_idx[(long long)i * k + s] = (IdxT)bi[s];
            if (out_dist) out_dist[(long long)i * k + s] = sqrtf(bd[s]);
        }
    }
}

template <typename IdxT>
int launch_knn(const float* q, int nq, const float* pts, int np, int k, int exclude_self, IdxT* idx, float* dist,
               cudaStream_t s) {
    const int g = blocks_for(nq, kKnnThreads);
    if (k <= 8) k_knn<8, IdxT><<<g, kKnnThreads, 0, s>>>(q, nq, pts, np, k, exclude_self, idx, dist);
    else if (k <= 16) k_knn<16, IdxT><<<g, kKnnThreads, 0, s>>>(q, nq, pts, np, k, exclude_self, idx, dist);
    else k_knn<32, IdxT><<<g, kKnnThreads, 0, s>>>(q, nq, pts, np, k, exclude_self, idx, dist);
    CKB(cudaGetLastError(), "k_knn");
    return EMPM_OK;
}

// ---------------------------------------------------------------------------
// inverse-distance weights of k given bones (calc_weights_vals_from_indices)
// ---------------------------------------------------------------------------
template <typename IdxT>
__global__ void k_idw(const float* __restrict__ bones, int n_bones, const float* __restrict__ pts, int n,
                      const IdxT* __restrict__ idx, int k, float* __restrict__ w, int* __restrict__ status) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const V3 x = load3(pts, p);
    const IdxT* row = idx + (long long)p * k;
    float sum = 0.f;
    bool bad = false;
    for (int s = 0; s < k; ++s) {
        const long long b = load_idx(row, s);
        if (b < 0 || b >= n_bones) { bad = true; continue; }
        sum += 1.f / (length(x - load3(bones, b)) + 1e-6f);
    }
    for (int s = 0; s < k; ++s) {
        const long long b = load_idx(row, s);
        float v = __int_as_float(0x7fc00000);
        if (!bad) v = (1.f / (length(x - load3(bones, b)) + 1e-6f)) / sum;
        w[(long long)p * k + s] = v;
    }
    if (bad) atomicOr(status, kBadIndex);
}

// ---------------------------------------------------------------------------
// bone stage
// ---------------------------------------------------------------------------
// rotation taking the x axis onto `axis` about axis x e_x (dynamic_utils.py:
// 369-393), for bones whose F has rank 1
__device__ M3 rank1_rotation(V3 axis) {
    const V3 ex = v3(1.f, 0.f, 0.f);
    V3 perp = cross(axis, ex);
    const float pn = length(perp);
    if (pn < 1e-6f) return m3_identity();
    perp = (1.f / pn) * perp;
    const V3 third = cross(ex, perp);
    const V3 third_after = cross(axis, perp);
    // R = Y X^T with X = [e_x perp third], Y = [axis perp third_after] (columns)
    M3 R;
    const V3 X[3] = {ex, perp, third};
    const V3 Y[3] = {axis, perp, third_after};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            R.m[3 * r + c] = comp(Y[0], r) * comp(X[0], c) + comp(Y[1], r) * comp(X[1], c) + comp(Y[2], r) * comp(X[2], c);
    return R;
}

// Per bone: F = sum_j ((b_j + m_j) - (b + m)) (b_j - b)^T over its neighbours
// (dynamic_utils.py:323-329, W = I), its numerical rank as
// torch.linalg.matrix_rank counts it (singular values above 3 eps_f32 s_max),
// and the candidate rotation of its class: U V^T (rank 2, 3; the SVD here has
// U, V in SO(3), so this is the proper rotation the reference assembles at
// :342-360), the rank-1 construction, or I (rank 0). work: 9 floats of R and
// the class, per bone.
template <typename IdxT>
__global__ void k_lbs_fit(const float* __restrict__ bones, const float* __restrict__ motions, int n_bones,
                          const IdxT* __restrict__ rel, int n_adj, float* __restrict__ work, int* __restrict__ counts) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    int cls = -1;
    bool bad = false;
    if (b < n_bones) {
        const V3 bp = load3(bones, b);
        const V3 bm = bp + load3(motions, b);
        M3 F = m3_zero();
        for (int j = 0; j < n_adj; ++j) {
            const long long r = load_idx(rel, (long long)b * n_adj + j);
            if (r < 0 || r >= n_bones) { bad = true; continue; }
            const V3 bj = load3(bones, r);
            const V3 old = bj - bp;
            const V3 nw = (bj + load3(motions, r)) - bm;
            F = F + outer(nw, old);
        }
        M3 U, V;
        V3 s;
        svd3(F, U, s, V);
        const float tol = 3.f * FLT_EPSILON * s.x;
        const int rank = (s.x > tol) + (s.y > tol) + (fabsf(s.z) > tol);
        M3 R;
        if (rank >= 2) {
            cls = kRank23;
            R = U * transpose(V);
        } else if (rank == 1) {
            cls = kRank1;
            // the reference then asserts torch.allclose(S[:, 1:], 0) (atol 1e-8)
            if (s.y > 1e-8f || fabsf(s.z) > 1e-8f) atomicAdd(counts + kRank1NotClose, 1);
            R = rank1_rotation(col(U, 0));
        } else {
            cls = kRank0;
            R = m3_identity();
        }
        float* o = work + 10 * (long long)b;
        for (int e = 0; e < 9; ++e) o[e] = R.m[e];
        o[9] = __int_as_float(cls);
        if (bad) atomicOr(counts + kStatus, kBadIndex);
    }
    // class counts, one atomic per warp and class (all bones would otherwise
    // queue on the same few words); every lane of the warp gets here. The
    // "last bone" of a class is read only when the class has exactly one
    // bone, so any writer will do.
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const unsigned m = __ballot_sync(0xffffffffu, cls == c);
        if (m && lane == __ffs(m) - 1) {
            atomicAdd(counts + c, __popc(m));
            if (c == kRank1) atomicExch(counts + kLastRank1, b);
            if (c == kRank23) atomicExch(counts + kLastRank23, b);
        }
    }
}

// Final rotation of every bone. The reference fits ranks 2-3 and rank 1 in
// two batches and assigns the batch it built last to all bones at once
// (dynamic_utils.py:337-407): that batch is the rank-1 one when any bone has
// rank 1, else the rank-2/3 one. The assignment succeeds only when the batch
// holds every bone, or one bone (broadcast to all); otherwise every bone gets
// the identity (:401-407). A rank-1 batch whose small singular values fail
// the allclose check becomes identities (:394-398).
// Unit quaternion (x, y, z, w) of a rotation matrix by Shepperd's method
// (S. W. Shepperd, "Quaternion from rotation matrix", J. Guidance and Control
// 1(3), 1978: the largest of 4w^2, 4x^2, 4y^2, 4z^2 picks the pivot), for
// rebuilding the bone rotation in the Gaussian stage.
__device__ float4 rotation_quat(const M3& R) {
    const float r00 = R.m[0], r11 = R.m[4], r22 = R.m[8];
    const float t = r00 + r11 + r22;
    float4 q;
    if (t >= r00 && t >= r11 && t >= r22) {
        const float h = 0.5f * sqrtf(fmaxf(1.f + t, 1e-30f)), f = 0.25f / h;
        q = make_float4((R.m[7] - R.m[5]) * f, (R.m[2] - R.m[6]) * f, (R.m[3] - R.m[1]) * f, h);
    } else if (r00 >= r11 && r00 >= r22) {
        const float h = 0.5f * sqrtf(fmaxf(1.f + r00 - r11 - r22, 1e-30f)), f = 0.25f / h;
        q = make_float4(h, (R.m[1] + R.m[3]) * f, (R.m[2] + R.m[6]) * f, (R.m[7] - R.m[5]) * f);
    } else if (r11 >= r22) {
        const float h = 0.5f * sqrtf(fmaxf(1.f - r00 + r11 - r22, 1e-30f)), f = 0.25f / h;
        q = make_float4((R.m[1] + R.m[3]) * f, h, (R.m[5] + R.m[7]) * f, (R.m[2] - R.m[6]) * f);
    } else {
        const float h = 0.5f * sqrtf(fmaxf(1.f - r00 - r11 + r22, 1e-30f)), f = 0.25f / h;
        q = make_float4((R.m[2] + R.m[6]) * f, (R.m[5] + R.m[7]) * f, h, (R.m[3] - R.m[1]) * f);
    }
    const float n = ::rsqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return make_float4(q.x * n, q.y * n, q.z * n, q.w * n);
}

// Bone table, 64 bytes (two 32-byte sectors) per bone:
//   (b.x, b.y, b.z, m.x) (m.y, m.z, qr.x, qr.y) (qr.z, qr.w, q.w, q.x) (q.y, q.z, 0, 0)
// b position, m motion, qr the rotation as a unit quaternion (x, y, z, w),
// q the blended quaternion of the caller's convention (w, x, y, z).
__global__ void k_lbs_resolve(const float* __restrict__ bones, const float* __restrict__ motions, int n_bones,
                              const float* __restrict__ work, const int* __restrict__ counts, int convention,
                              float4* __restrict__ table) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_bones) return;
    const int n1 = counts[kRank1], n23 = counts[kRank23];
    int src;
    if (n1 > 0) {
        src = n1 == n_bones ? b : (n1 == 1 ? counts[kLastRank1] : -1);
        if (counts[kRank1NotClose] > 0) src = -1;
    } else {
        src = n23 == n_bones ? b : (n23 == 1 ? counts[kLastRank23] : -1);
    }
    M3 R = m3_identity();
    if (src >= 0)
        for (int e = 0; e < 9; ++e) R.m[e] = work[10 * (long long)src + e];
    const V3 bp = load3(bones, b), m = load3(motions, b);
    const float4 qr = rotation_quat(R);
    const float4 q = normalize4(quat_of(R, convention));
    float4* row = table + 4 * (long long)b;
    row[0] = make_float4(bp.x, bp.y, bp.z, m.x);
    row[1] = make_float4(m.y, m.z, qr.x, qr.y);
    row[2] = make_float4(qr.z, qr.w, q.x, q.y);
    row[3] = make_float4(q.z, q.w, 0.f, 0.f);
}

// ---------------------------------------------------------------------------
// Gaussian stage
// ---------------------------------------------------------------------------
struct BoneRow {
    V3 b, m;
    float4 qr;   // (x, y, z, w)
    float4 q;    // (w, x, y, z) in .x .y .z .w
};

// A row is two 32-byte sectors; each is fetched with one 256-bit load (the
// table is 32-byte aligned, checked on the host).
__device__ __forceinline__ void ld_sector(const float4* p, float4& a, float4& b) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

__device__ __forceinline__ BoneRow bone_row(const float4* __restrict__ table, long long b) {
    const float4* t = table + 4 * b;
    float4 t0, t1, t2, t3;
    ld_sector(t, t0, t1);
    ld_sector(t + 2, t2, t3);
    BoneRow r;
    r.b = v3(t0.x, t0.y, t0.z);
    r.m = v3(t0.w, t1.x, t1.y);
    r.qr = make_float4(t1.z, t1.w, t2.x, t2.y);
    r.q = make_float4(t2.z, t2.w, t3.x, t3.y);
    return r;
}

__device__ __forceinline__ V3 bone_pos(const float4* __restrict__ table, long long b) {
    const float4 t0 = __ldg(table + 4 * b);
    return v3(t0.x, t0.y, t0.z);
}

// R (x - b) + m + b of one bone (dynamic_utils.py:433-440), R rebuilt from
// its unit quaternion
__device__ __forceinline__ V3 bone_apply(const BoneRow& r, V3 x) {
    const float qx = r.qr.x, qy = r.qr.y, qz = r.qr.z, qw = r.qr.w;
    const V3 l = x - r.b;
    const float xx = qx * qx, yy = qy * qy, zz = qz * qz;
    const float xy = qx * qy, xz = qx * qz, yz = qy * qz, wx = qw * qx, wy = qw * qy, wz = qw * qz;
    const V3 rl = v3((1.f - 2.f * (yy + zz)) * l.x + 2.f * (xy - wz) * l.y + 2.f * (xz + wy) * l.z,
                     2.f * (xy + wz) * l.x + (1.f - 2.f * (xx + zz)) * l.y + 2.f * (yz - wx) * l.z,
                     2.f * (xz - wy) * l.x + 2.f * (yz + wx) * l.y + (1.f - 2.f * (xx + yy)) * l.z);
    return (rl + r.m) + r.b;
}

// inverse distance 1 / (|x - b| + 1e-6) to a bone of the table
__device__ __forceinline__ float idw_term(const BoneRow& r, V3 x) {
    return 1.f / (length(x - r.b) + 1e-6f);
}

// w NULL: the weights are the normalised inverse distances to the k bones
// (calc_weights_vals_from_indices with the table's bones). They are computed
// in the same pass: the sums run over the unnormalised terms v_k and the
// position sum is divided by sum v_k at the end; the quaternion sum is
// normalised anyway. w_out (optional) then needs a second pass over the k
// bones' positions. The bone loop has no branches, so that the gathers of
// several bones are in flight together: an out-of-range index reads bone 0
// with weight 0 and marks the Gaussian bad. KT > 0: k == KT at compile time.
template <int KT, typename IdxT>
__global__ void __launch_bounds__(256) k_lbs_blend(const float4* __restrict__ table, int n_bones,
                                                   const float* xyz, const float* quat_in, int n,
                                                   const IdxT* __restrict__ idx, int k_rt, const float* __restrict__ w,
                                                   float* __restrict__ w_out, float* xyz_out, float* quat_out,
                                                   int* __restrict__ status) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int k = KT > 0 ? KT : k_rt;
    const V3 x = load3(xyz, p);
    const IdxT* row = idx + (long long)p * k;
    bool bad = false;
    V3 acc = v3(0.f, 0.f, 0.f);
    float4 qa = make_float4(0.f, 0.f, 0.f, 0.f);
    float sum = 0.f;
#pragma unroll 4
    for (int s = 0; s < k; ++s) {
        const long long bi = load_idx(row, s);
        const bool ok = bi >= 0 && bi < n_bones;
        bad |= !ok;
        const BoneRow r = bone_row(table, ok ? bi : 0);
        float ws = w ? __ldg(w + (long long)p * k + s) : idw_term(r, x);
        ws = ok ? ws : 0.f;
        sum += ws;
        acc = acc + bone_apply(r, x) * ws;
        qa = make_float4(qa.x + r.q.x * ws, qa.y + r.q.y * ws, qa.z + r.q.z * ws, qa.w + r.q.w * ws);
    }
    if (!w) {
        acc = acc * (1.f / sum);
        if (w_out && !bad)
            for (int s = 0; s < k; ++s) {
                const V3 bp = bone_pos(table, load_idx(row, s));
                w_out[(long long)p * k + s] = (1.f / (length(x - bp) + 1e-6f)) / sum;
            }
    }
    float4 qo = make_float4(0.f, 0.f, 0.f, 0.f);
    if (quat_in) qo = qmul(normalize4(qa), make_float4(quat_in[4 * (long long)p], quat_in[4 * (long long)p + 1],
                                                      quat_in[4 * (long long)p + 2], quat_in[4 * (long long)p + 3]));
    if (bad) {
        const float nan = __int_as_float(0x7fc00000);
        acc = v3(nan, nan, nan);
        qo = make_float4(nan, nan, nan, nan);
        atomicOr(status, kBadIndex);
    }
    xyz_out[3 * (long long)p] = acc.x;
    xyz_out[3 * (long long)p + 1] = acc.y;
    xyz_out[3 * (long long)p + 2] = acc.z;
    if (quat_in) {
        if ((reinterpret_cast<uintptr_t>(quat_out) & 15) == 0) {
            reinterpret_cast<float4*>(quat_out)[p] = qo;
        } else {
            quat_out[4 * (long long)p] = qo.x; quat_out[4 * (long long)p + 1] = qo.y;
            quat_out[4 * (long long)p + 2] = qo.z; quat_out[4 * (long long)p + 3] = qo.w;
        }
    }
}

// k = 16 with the weights computed here (the per-frame path): the block's
// index rows are contiguous in memory, so they are brought into shared memory
// with coalesced 16-byte loads first (a thread reading its own 64- or 128-byte
// row directly touches a separate sector per lane and index). Rows are padded
// to an odd number of 16-byte chunks, so that the per-thread 16-byte reads of
// shared memory are free of bank conflicts.
constexpr int kBlendThreads = 256;

template <typename IdxT>
__global__ void __launch_bounds__(kBlendThreads) k_lbs_blend16(const float4* __restrict__ table, int n_bones,
                                                               const float* xyz, const float* quat_in, int n,
                                                               const IdxT* __restrict__ idx, float* xyz_out,
                                                               float* quat_out, int* __restrict__ status) {
    constexpr int K = 16;
    constexpr int CH = K * (int)sizeof(IdxT) / 16;   // 16-byte chunks per row
    constexpr int STRIDE = CH + 1;
    __shared__ int4 rows[kBlendThreads * STRIDE];
    const long long first = (long long)blockIdx.x * kBlendThreads;
    const int nrows = (int)min((long long)kBlendThreads, (long long)n - first);
    const int4* src = reinterpret_cast<const int4*>(idx + first * K);
    for (int c = threadIdx.x; c < nrows * CH; c += kBlendThreads)
        rows[(c / CH) * STRIDE + (c % CH)] = __ldg(src + c);
    __syncthreads();
    const int t = threadIdx.x;
    if (t >= nrows) return;
    const long long p = first + t;
    const V3 x = load3(xyz, p);
    bool bad = false;
    V3 acc = v3(0.f, 0.f, 0.f);
    float4 qa = make_float4(0.f, 0.f, 0.f, 0.f);
    float sum = 0.f;
    constexpr int PER = 16 / (int)sizeof(IdxT);   // indices per chunk
#pragma unroll 1
    for (int c = 0; c < CH; ++c) {
        const int4 v = rows[t * STRIDE + c];
        IdxT e[PER];
        memcpy(e, &v, 16);
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const long long b = (long long)e[j];
            const bool ok = b >= 0 && b < n_bones;
            bad |= !ok;
            const BoneRow r = bone_row(table, ok ? b : 0);
            const float ws = ok ? idw_term(r, x) : 0.f;
            sum += ws;
            acc = acc + bone_apply(r, x) * ws;
            qa = make_float4(qa.x + r.q.x * ws, qa.y + r.q.y * ws, qa.z + r.q.z * ws, qa.w + r.q.w * ws);
        }
    }
    acc = acc * (1.f / sum);
    float4 qo = make_float4(0.f, 0.f, 0.f, 0.f);
    if (quat_in) qo = qmul(normalize4(qa), make_float4(quat_in[4 * p], quat_in[4 * p + 1], quat_in[4 * p + 2],
                                                      quat_in[4 * p + 3]));
    if (bad) {
        const float nan = __int_as_float(0x7fc00000);
        acc = v3(nan, nan, nan);
        qo = make_float4(nan, nan, nan, nan);
        atomicOr(status, kBadIndex);
    }
    xyz_out[3 * p] = acc.x;
    xyz_out[3 * p + 1] = acc.y;
    xyz_out[3 * p + 2] = acc.z;
    if (quat_in) {
        if ((reinterpret_cast<uintptr_t>(quat_out) & 15) == 0) {
            reinterpret_cast<float4*>(quat_out)[p] = qo;
        } else {
            quat_out[4 * p] = qo.x; quat_out[4 * p + 1] = qo.y; quat_out[4 * p + 2] = qo.z; quat_out[4 * p + 3] = qo.w;
        }
    }
}

template <typename IdxT>
void launch_blend(const float4* t, int n_bones, const float* xyz, const float* quat_in, int n, const IdxT* idx, int k,
                  const float* w, float* w_out, float* xyz_out, float* quat_out, int* status, cudaStream_t s) {
    const int g = blocks_for(n, kBlendThreads);
    if (k == 16 && !w && !w_out && (reinterpret_cast<uintptr_t>(idx) & 15) == 0)
        k_lbs_blend16<IdxT><<<g, kBlendThreads, 0, s>>>(t, n_bones, xyz, quat_in, n, idx, xyz_out, quat_out, status);
    else if (k == 16)
        k_lbs_blend<16, IdxT><<<g, kBlendThreads, 0, s>>>(t, n_bones, xyz, quat_in, n, idx, k, w, w_out, xyz_out,
                                                          quat_out, status);
    else
        k_lbs_blend<0, IdxT><<<g, kBlendThreads, 0, s>>>(t, n_bones, xyz, quat_in, n, idx, k, w, w_out, xyz_out,
                                                         quat_out, status);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

// Dense weights (interpolate_motions): one warp per Gaussian, lanes over all
// bones. weights NULL: 1 / max(|x - b|, 1e-4) over every bone, normalised
// (:168-178), and written to weights_out when it is given.
__global__ void __launch_bounds__(256) k_lbs_blend_dense(const float4* __restrict__ table, int n_bones,
                                                         const float* xyz, const float* quat_in, int n,
                                                         const float* __restrict__ w, float* __restrict__ w_out,
                                                         float* xyz_out, float* quat_out) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= n) return;   // whole warp
    const V3 x = load3(xyz, p);
    float sum = 1.f;
    if (!w) {
        float s = 0.f;
        for (int b = lane; b < n_bones; b += 32) s += 1.f / fmaxf(length(x - bone_pos(table, b)), 1e-4f);
        sum = warp_sum(s);
    }
    V3 acc = v3(0.f, 0.f, 0.f);
    float4 qa = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int b = lane; b < n_bones; b += 32) {
        const BoneRow r = bone_row(table, b);
        float ws;
        if (w) ws = __ldg(w + (long long)p * n_bones + b);
        else ws = (1.f / fmaxf(length(x - r.b), 1e-4f)) / sum;
        if (w_out) w_out[(long long)p * n_bones + b] = ws;
        acc = acc + bone_apply(r, x) * ws;
        qa = make_float4(qa.x + r.q.x * ws, qa.y + r.q.y * ws, qa.z + r.q.z * ws, qa.w + r.q.w * ws);
    }
    acc = v3(warp_sum(acc.x), warp_sum(acc.y), warp_sum(acc.z));
    qa = make_float4(warp_sum(qa.x), warp_sum(qa.y), warp_sum(qa.z), warp_sum(qa.w));
    if (lane == 0) {
        xyz_out[3 * (long long)p] = acc.x;
        xyz_out[3 * (long long)p + 1] = acc.y;
        xyz_out[3 * (long long)p + 2] = acc.z;
        if (quat_in) {
            const float4 qi = make_float4(quat_in[4 * (long long)p], quat_in[4 * (long long)p + 1],
                                          quat_in[4 * (long long)p + 2], quat_in[4 * (long long)p + 3]);
            const float4 qo = qmul(normalize4(qa), qi);
            quat_out[4 * (long long)p] = qo.x;
            quat_out[4 * (long long)p + 1] = qo.y;
            quat_out[4 * (long long)p + 2] = qo.z;
            quat_out[4 * (long long)p + 3] = qo.w;
        }
    }
}

__global__ void k_rotation_to_quat(const float* __restrict__ R9, int n, int convention, float* __restrict__ q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    M3 R;
    for (int e = 0; e < 9; ++e) R.m[e] = __ldg(R9 + 9 * (long long)i + e);
    const float4 v = quat_of(R, convention);
    q[4 * (long long)i] = v.x;
    q[4 * (long long)i + 1] = v.y;
    q[4 * (long long)i + 2] = v.z;
    q[4 * (long long)i + 3] = v.w;
}

bool idx_ok(int idx_bytes) { return idx_bytes == 4 || idx_bytes == 8; }

}  // namespace

extern "C" int empm_knn(const float* queries, int n_queries, const float* points, int n_points, int k,
                        int exclude_self, void* out_idx, int idx_bytes, float* out_dist, void* stream) {
    if (n_queries < 0 || n_points < 0 || k < 1 || k > EMPM_KNN_MAX_K || !idx_ok(idx_bytes))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "knn: bad sizes (k %d, idx_bytes %d)", k, idx_bytes);
    if (exclude_self && n_queries != n_points)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "knn: exclude_self needs queries == points");
    if (k > n_points - (exclude_self ? 1 : 0))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "knn: k %d exceeds the %d candidates", k,
                              n_points - (exclude_self ? 1 : 0));
    if (n_queries == 0) return EMPM_OK;
    if (!queries || !points || !out_idx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "knn: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (idx_bytes == 8)
        return launch_knn(queries, n_queries, points, n_points, k, exclude_self, (long long*)out_idx, out_dist, s);
    return launch_knn(queries, n_queries, points, n_points, k, exclude_self, (int*)out_idx, out_dist, s);
}

extern "C" int empm_idw_weights(const float* bones, int n_bones, const float* pts, int n, const void* idx,
                                int idx_bytes, int k, float* weights, int* status, void* stream) {
    if (n < 0 || n_bones < 0 || k < 1 || !idx_ok(idx_bytes))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "idw weights: bad sizes");
    if (n == 0) return EMPM_OK;
    if (!bones || !pts || !idx || !weights || !status)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "idw weights: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (idx_bytes == 8)
        k_idw<<<blocks_for(n, 256), 256, 0, s>>>(bones, n_bones, pts, n, (const long long*)idx, k, weights, status);
    else
        k_idw<<<blocks_for(n, 256), 256, 0, s>>>(bones, n_bones, pts, n, (const int*)idx, k, weights, status);
    CKB(cudaGetLastError(), "k_idw");
    return EMPM_OK;
}

extern "C" int empm_lbs_bones(const float* bones, const float* motions, int n_bones, const void* relations,
                              int idx_bytes, int n_adj, int convention, float* table, float* work, int* counts,
                              void* stream) {
    if (n_bones < 0 || n_adj < 0 || !idx_ok(idx_bytes) ||
        (convention != EMPM_QUAT_KORNIA && convention != EMPM_QUAT_MAT2QUAT))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs bones: bad arguments");
    if (!counts) return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs bones: NULL counts");
    cudaStream_t s = (cudaStream_t)stream;
    CKB(cudaMemsetAsync(counts, 0, sizeof(int) * EMPM_LBS_COUNTS, s), "lbs counts");
    if (n_bones == 0) return EMPM_OK;
    if (!bones || !motions || !table || !work || (n_adj > 0 && !relations))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs bones: NULL pointer");
    if (reinterpret_cast<uintptr_t>(table) & 31)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs bones: bone table must be 32-byte aligned");
    const int g = blocks_for(n_bones, 128);
    if (idx_bytes == 8)
        k_lbs_fit<<<g, 128, 0, s>>>(bones, motions, n_bones, (const long long*)relations, n_adj, work, counts);
    else
        k_lbs_fit<<<g, 128, 0, s>>>(bones, motions, n_bones, (const int*)relations, n_adj, work, counts);
    CKB(cudaGetLastError(), "k_lbs_fit");
    k_lbs_resolve<<<g, 128, 0, s>>>(bones, motions, n_bones, work, counts, convention,
                                    reinterpret_cast<float4*>(table));
    CKB(cudaGetLastError(), "k_lbs_resolve");
    return EMPM_OK;
}

extern "C" int empm_lbs_blend(const float* table, int n_bones, const float* xyz, const float* quat_in, int n,
                              const void* idx, int idx_bytes, int k, const float* weights, float* weights_out,
                              float* xyz_out, float* quat_out, int* status, void* stream) {
    if (n < 0 || n_bones < 0 || k < 1 || !idx_ok(idx_bytes))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs blend: bad sizes");
    if (n == 0) return EMPM_OK;
    if (!table || !xyz || !idx || !xyz_out || !status || (quat_in && !quat_out))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs blend: NULL pointer");
    if (n_bones == 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs blend: no bones");
    if (reinterpret_cast<uintptr_t>(table) & 31)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs blend: bone table must be 32-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    const float4* t = reinterpret_cast<const float4*>(table);
    if (idx_bytes == 8)
        launch_blend(t, n_bones, xyz, quat_in, n, (const long long*)idx, k, weights, weights_out, xyz_out, quat_out,
                     status, s);
    else
        launch_blend(t, n_bones, xyz, quat_in, n, (const int*)idx, k, weights, weights_out, xyz_out, quat_out, status,
                     s);
    CKB(cudaGetLastError(), "k_lbs_blend");
    return EMPM_OK;
}

extern "C" int empm_lbs_blend_dense(const float* table, int n_bones, const float* xyz, const float* quat_in, int n,
                                    const float* weights, float* weights_out, float* xyz_out, float* quat_out,
                                    void* stream) {
    if (n < 0 || n_bones < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs dense blend: bad sizes");
    if (n == 0) return EMPM_OK;
    if (!table || !xyz || !xyz_out || (quat_in && !quat_out) || n_bones == 0)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs dense blend: NULL pointer or no bones");
    if (reinterpret_cast<uintptr_t>(table) & 31)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "lbs dense blend: bone table must be 32-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    k_lbs_blend_dense<<<blocks_for((long long)n * 32, 256), 256, 0, s>>>(
        reinterpret_cast<const float4*>(table), n_bones, xyz, quat_in, n, weights, weights_out, xyz_out, quat_out);
    CKB(cudaGetLastError(), "k_lbs_blend_dense");
    return EMPM_OK;
}

extern "C" int empm_rotation_to_quat(const float* R9, int n, int convention, float* q, void* stream) {
    if (n < 0 || (convention != EMPM_QUAT_KORNIA && convention != EMPM_QUAT_MAT2QUAT))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "rotation_to_quat: bad arguments");
    if (n == 0) return EMPM_OK;
    if (!R9 || !q) return empm_set_error(nullptr, EMPM_ERR_INVALID, "rotation_to_quat: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    k_rotation_to_quat<<<blocks_for(n, 256), 256, 0, s>>>(R9, n, convention, q);
    CKB(cudaGetLastError(), "k_rotation_to_quat");
    return EMPM_OK;
}
