// restart.cuh — the static-pose restart, MPMWARPDiff.restart_and_compute_F_C
// (phys_sim/diff_simulator/warp_mpm/mpm_solver_diff.py:1214-1262).
//
// Particles sit at a static pose x and are given their deformation gradient
// towards target positions: the displacement target - x is scattered to the
// grid with weight * mass (set_F_C_p2g, mpm_utils.py:836-866), normalised by
// the grid mass without gravity or boundary conditions
// (grid_normalization_and_gravity with dt = 0, :426-438), and gathered back as
// F_trial = I + sum grid_v (x) dweight (set_F_C_g2p, :869-919). Every x then
// becomes its target; C is left as it is. Unsimulated particles keep their
// F_trial but are moved as well, as in the reference. With update_cov_with_F
// the packed covariances get the same displacement gradient (:918-919).
#pragma once
#include "kernels.cuh"

namespace empm {

__global__ void __launch_bounds__(128) k_restart_p2g(ParticleArrays P, const float* __restrict__ target,
                                                     const int* __restrict__ sel, Launch L, float4* grid,
                                                     unsigned char* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    if (sel && __ldg(sel + p) != 0) return;
    const StepConsts c = consts_of(L, find_instance_particle(L, p));
    const float4 xm = __ldg(P.x + p);
    const Stencil st = make_stencil(v3(xm.x, xm.y, xm.z), c.inv_dx);
    const V3 disp = v3(__ldg(target + 3 * p) - xm.x, __ldg(target + 3 * p + 1) - xm.y,
                       __ldg(target + 3 * p + 2) - xm.z);
    const bool in_grid = stencil_in_grid(st, c.G);
    if (!in_grid) atomicOr(c.status, EMPM_STATUS_OUT_OF_BAND);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int ix = st.b[0] + i, iy = st.b[1] + j, iz = st.b[2] + k;
                if (!in_grid && (ix < 0 || iy < 0 || iz < 0 || ix >= c.G || iy >= c.G || iz >= c.G)) continue;
                const float wm = st.w[0][i] * st.w[1][j] * st.w[2][k] * xm.w;
                red_add_v4(grid + gaddr(c, ix, iy, iz), make_float4(wm * disp.x, wm * disp.y, wm * disp.z, wm));
            }
    mark_stencil_blocks(flags, st, c);
}

// node displacement = accumulated (mass * displacement) / mass; zero the accumulator
__global__ void __launch_bounds__(256) k_restart_grid(float4* mom, float4* vel, const int* active) {
    const long long total = (long long)__ldg(active) * 64;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long node = ((long long)__ldg(active + 1 + (idx >> 6)) << 6) | (idx & 63);
        const float4 m = mom[node];
        mom[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 v = make_float4(0.f, 0.f, 0.f, m.w);
        if (m.w > 1e-15f) {
            const float inv = 1.f / m.w;
            v.x = m.x * inv;
            v.y = m.y * inv;
            v.z = m.z * inv;
        }
        vel[node] = v;
    }
}

// PhysGaussian covariance update (update_cov, mpm_utils.py:306-326):
// cov += dt (G cov + cov G^T) on the packed upper triangle
// (c00, c01, c02, c11, c12, c22) of particle p.
__device__ __forceinline__ void update_cov(float* cov, int p, const M3& G, float dt) {
    float* c = cov + 6 * (long long)p;
    M3 S;
    S.m[0] = c[0]; S.m[1] = c[1]; S.m[2] = c[2];
    S.m[3] = c[1]; S.m[4] = c[3]; S.m[5] = c[4];
    S.m[6] = c[2]; S.m[7] = c[4]; S.m[8] = c[5];
    const M3 N = S + dt * (G * S + S * transpose(G));
    c[0] = N.m[0]; c[1] = N.m[1]; c[2] = N.m[2];
    c[3] = N.m[4]; c[4] = N.m[5]; c[5] = N.m[8];
}

// cov (optional): covariance update with the displacement gradient and
// dt = 1, as set_F_C_g2p does when update_cov_with_F is set (:918-919)
__global__ void __launch_bounds__(128) k_restart_g2p(ParticleArrays P, const float* __restrict__ target,
                                                     const int* __restrict__ sel, Launch L, const float4* vel,
                                                     float* cov) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    const float4 xm = __ldg(P.x + p);
    if (!(sel && __ldg(sel + p) != 0)) {
        const StepConsts c = consts_of(L, find_instance_particle(L, p));
        const Stencil st = make_stencil(v3(xm.x, xm.y, xm.z), c.inv_dx);
        const bool in_grid = stencil_in_grid(st, c.G);
        const GlobalFetch fetch{vel, &c};
        const G2POut o = g2p_gather(st, c.inv_dx, fetch.bind(st, in_grid));
        f9_store(P.F, p, m3_identity() + o.gradv);
        if (cov) update_cov(cov, p, o.gradv, 1.f);
    }
    P.x[p] = make_float4(__ldg(target + 3 * p), __ldg(target + 3 * p + 1), __ldg(target + 3 * p + 2), xm.w);
}

// -------------------------------------------------------------------------
// in-place G2P of MPMWARPDiff.p2g2p (mpm_solver_diff.py:293-429)
// -------------------------------------------------------------------------
// g2p (mpm_utils.py:441-499) followed by clip_particle_x (:582-599), written
// back into the particle's own arrays: v, C, F_trial = (I + dt grad v) F_e,
// x += dt v (the atomic_add of :486) clamped to [2 dx, grid_lim - 2 dx], and,
// when cov is given (update_cov_with_F), cov += dt (G cov + cov G^T) with
// G = grad v. Unsimulated particles (selection != 0) are left as they are.
// Each thread reads and writes only its own particle, so in place is safe.
__global__ void __launch_bounds__(128) k_g2p_inplace(ParticleArrays P, F9Planes Fe, MaterialArrays M, Launch L,
                                                     const float4* vel, float* cov) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    if (M.sel && __ldg(M.sel + p) != 0) return;
    const StepConsts c = consts_of(L, find_instance_particle(L, p));
    if (c.step->hold) return;
    const float dt = c.step->dt;
    const float4 xm = P.x[p];
    const V3 x = v3(xm.x, xm.y, xm.z);
    const Stencil st = make_stencil(x, c.inv_dx);
    const bool in_grid = stencil_in_grid(st, c.G);
    const GlobalFetch fetch{vel, &c};
    const G2POut o = g2p_gather(st, c.inv_dx, fetch.bind(st, in_grid));
    const float dx = 1.f / c.inv_dx;
    const float lo = dx * 2.f, hi = c.grid_lim - dx * 2.f;
    V3 nx = x + dt * o.v;
    nx = v3(fminf(fmaxf(nx.x, lo), hi), fminf(fmaxf(nx.y, lo), hi), fminf(fmaxf(nx.z, lo), hi));
    const M3 Fn = (m3_identity() + dt * o.gradv) * f9_load(Fe, p);
    P.x[p] = make_float4(nx.x, nx.y, nx.z, xm.w);
    P.v[p] = make_float4(o.v.x, o.v.y, o.v.z, 0.f);
    f9_store(P.C, p, o.C);
    f9_store(P.F, p, Fn);
    if (cov) update_cov(cov, p, o.gradv, dt);
    unsigned flags = 0;
    if (!finite3(o.v) || !finite3(nx) || !isfinite(Fn.m[0] + Fn.m[4] + Fn.m[8])) flags |= EMPM_STATUS_NAN;
    if (fmaxf(fmaxf(fabsf(o.v.x), fabsf(o.v.y)), fabsf(o.v.z)) * dt > dx) flags |= EMPM_STATUS_CFL;
    if (!in_grid) flags |= EMPM_STATUS_OUT_OF_BAND;
    if (flags) atomicOr(c.status, flags);
}

}  // namespace empm
