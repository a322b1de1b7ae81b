// losses.cu — training losses on the device: batched chamfer distance and
// its gradient.
//
// The reference trainer scores a rollout with pytorch3d's chamfer_distance
// (phys_sim/engine/trainer_warp_mpm.py:542-561, 617-642, 745-765): for point
// sets X and Y, mean over x of min_y |x - y|^2 plus mean over y of
// min_x |x - y|^2 (point_reduction "mean"). Here many (X, Y) pairs (one per
// population member and frame) are scored in one launch: pair p owns
// X rows [x_off[p], x_off[p+1]) and Y rows [y_off[p], y_off[p+1]). The nearest
// neighbours are found exactly, by brute force over shared-memory tiles of
// the other set, and kept for the gradient.
#include <cuda_runtime.h>
#include <float.h>
#include "../../include/empm_b200.h"
#include "ctx.hpp"

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

// For every query point q of pair blockIdx.y: nearest point of the pair's
// target set, its squared distance added to sum[pair].
__global__ void __launch_bounds__(kThreads) k_nn(const float* __restrict__ q, const int* __restrict__ q_off,
                                                 const float* __restrict__ t, const int* __restrict__ t_off,
                                                 int* __restrict__ nn, float* __restrict__ sum) {
    __shared__ float4 tile[kThreads];
    const int pair = blockIdx.y;
    const int q0 = __ldg(q_off + pair), q1 = __ldg(q_off + pair + 1);
    const int t0 = __ldg(t_off + pair), t1 = __ldg(t_off + pair + 1);
    const int i = q0 + blockIdx.x * kThreads + threadIdx.x;
    if (q0 + (int)(blockIdx.x * kThreads) >= q1) return;   // whole CTA beyond this pair's queries
    const bool live = i < q1;
    float qx = 0.f, qy = 0.f, qz = 0.f;
    if (live) { qx = __ldg(q + 3 * i); qy = __ldg(q + 3 * i + 1); qz = __ldg(q + 3 * i + 2); }
    float best = FLT_MAX;
    int arg = -1;
    for (int base = t0; base < t1; base += kThreads) {
        const int j = base + threadIdx.x;
        __syncthreads();
        tile[threadIdx.x] = j < t1 ? make_float4(__ldg(t + 3 * j), __ldg(t + 3 * j + 1), __ldg(t + 3 * j + 2), 0.f)
                                   : make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
        __syncthreads();
        const int m = min(kThreads, t1 - base);
        for (int k = 0; k < m; ++k) {
            const float4 p = tile[k];
            const float dx = qx - p.x, dy = qy - p.y, dz = qz - p.z;
            const float d = dx * dx + dy * dy + dz * dz;
            if (d < best) { best = d; arg = base + k; }
        }
    }
    if (live) nn[i] = arg;
    // warp-level partial sums (every lane of the CTA is still here; lanes
    // without a query add zero), one atomic per warp
    float v = (live && arg >= 0) ? best : 0.f;
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0 && v != 0.f) atomicAdd(sum + pair, v);
}

// Gradient in X of  g_xy[p] * sum_i |x_i - y_nn(i)|^2 + g_yx[p] * sum_j |y_j - x_nn(j)|^2
__global__ void k_chamfer_grad_x(const float* __restrict__ x, const int* __restrict__ pair_of_x,
                                 const float* __restrict__ y, const int* __restrict__ nn_x,
                                 const float* __restrict__ g_xy, float* __restrict__ gx, int nx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    const int j = nn_x[i];
    if (j < 0) return;
    const float g = 2.f * __ldg(g_xy + __ldg(pair_of_x + i));
    gx[3 * i] += g * (x[3 * i] - y[3 * j]);
    gx[3 * i + 1] += g * (x[3 * i + 1] - y[3 * j + 1]);
    gx[3 * i + 2] += g * (x[3 * i + 2] - y[3 * j + 2]);
}

__global__ void k_chamfer_grad_y_to_x(const float* __restrict__ x, const float* __restrict__ y,
                                      const int* __restrict__ pair_of_y, const int* __restrict__ nn_y,
                                      const float* __restrict__ g_yx, float* __restrict__ gx, int ny) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ny) return;
    const int i = nn_y[j];
    if (i < 0) return;
    const float g = 2.f * __ldg(g_yx + __ldg(pair_of_y + j));
    atomicAdd(gx + 3 * i, g * (x[3 * i] - y[3 * j]));
    atomicAdd(gx + 3 * i + 1, g * (x[3 * i + 1] - y[3 * j + 1]));
    atomicAdd(gx + 3 * i + 2, g * (x[3 * i + 2] - y[3 * j + 2]));
}

__global__ void k_pair_index(const int* off, int n_pairs, int* pair_of, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = n_pairs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= i) lo = mid; else hi = mid - 1;
    }
    pair_of[i] = lo;
}

}  // namespace

#define CKL(expr, what)                                                          \
    do {                                                                         \
        int _rc = empm_check_cuda(nullptr, (expr), what);                        \
        if (_rc != EMPM_OK) return _rc;                                          \
    } while (0)

extern "C" int empm_chamfer(const float* x, const int* x_off, int nx, int max_nx, const float* y, const int* y_off,
                            int ny, int max_ny, int n_pairs, float* sum_xy, float* sum_yx, int* nn_x, int* nn_y,
                            void* stream) {
    if (n_pairs < 1 || n_pairs > 65535 || nx < 0 || ny < 0 || max_nx < 0 || max_ny < 0)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad chamfer sizes (%d pairs)", n_pairs);
    if (!x_off || !y_off || !sum_xy || !sum_yx || (nx && (!x || !nn_x)) || (ny && (!y || !nn_y)))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "chamfer pointer is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    CKL(cudaMemsetAsync(sum_xy, 0, sizeof(float) * n_pairs, s), "chamfer");
    CKL(cudaMemsetAsync(sum_yx, 0, sizeof(float) * n_pairs, s), "chamfer");
    if (max_nx > 0) {
        k_nn<<<dim3(blocks_for(max_nx, kThreads), n_pairs), kThreads, 0, s>>>(x, x_off, y, y_off, nn_x, sum_xy);
        CKL(cudaGetLastError(), "k_nn (x -> y)");
    }
    if (max_ny > 0) {
        k_nn<<<dim3(blocks_for(max_ny, kThreads), n_pairs), kThreads, 0, s>>>(y, y_off, x, x_off, nn_y, sum_yx);
        CKL(cudaGetLastError(), "k_nn (y -> x)");
    }
    return EMPM_OK;
}

extern "C" int empm_chamfer_backward(const float* x, const int* x_off, int nx, const float* y, const int* y_off,
                                     int ny, int n_pairs, const int* nn_x, const int* nn_y, const float* g_xy,
                                     const float* g_yx, float* grad_x, int* scratch_pair, void* stream) {
    if (n_pairs < 1 || nx < 0 || ny < 0)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad chamfer sizes (%d pairs)", n_pairs);
    if (!x_off || !y_off || !g_xy || !g_yx || !grad_x || !scratch_pair || (nx && (!x || !nn_x)) ||
        (ny && (!y || !nn_y)))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "chamfer pointer is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    if (nx > 0) {
        k_pair_index<<<blocks_for(nx, 256), 256, 0, s>>>(x_off, n_pairs, scratch_pair, nx);
        CKL(cudaGetLastError(), "k_pair_index");
        k_chamfer_grad_x<<<blocks_for(nx, 256), 256, 0, s>>>(x, scratch_pair, y, nn_x, g_xy, grad_x, nx);
        CKL(cudaGetLastError(), "k_chamfer_grad_x");
    }
    if (ny > 0) {
        // the pair index of Y rows reuses the scratch after the X pass (stream order)
        k_pair_index<<<blocks_for(ny, 256), 256, 0, s>>>(y_off, n_pairs, scratch_pair, ny);
        CKL(cudaGetLastError(), "k_pair_index");
        k_chamfer_grad_y_to_x<<<blocks_for(ny, 256), 256, 0, s>>>(x, y, scratch_pair, nn_y, g_yx, grad_x, ny);
        CKL(cudaGetLastError(), "k_chamfer_grad_y_to_x");
    }
    return EMPM_OK;
}
