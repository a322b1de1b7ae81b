// adjoint.cuh — reverse-mode kernels of one MLS-MPM substep (direct path:
// particles in the caller's order, one particle or node per thread).
//
// The reference obtains gradients by replaying Warp's generated adjoints of
// every launched kernel (tape.backward, interface.py:197,418,720,935). Here
// the adjoint of one substep is three hand-written kernels that run after the
// substep's forward grid has been recomputed (P2G, then the grid update in
// its variant that keeps the momentum and the block flags):
//
//   k_adj_g2p   per particle: adjoint of x', v', C', F' -> scatter of the node
//               velocity adjoint, and the particle's x and F_elastic adjoints
//               from the G2P gather;
//   k_adj_grid  per touched node: the boundary conditions replayed forwards
//               and transposed backwards, then normalisation -> adjoint of
//               the accumulated momentum and mass;
//   k_adj_p2g   per particle: gather of the momentum/mass adjoint -> adjoint
//               of v, C, mass, the stress, and x; then the constitutive
//               adjoint (spectral.cuh) -> F_trial, mu, lam and yield adjoints,
//               and the velocity modifiers' adjoint.
//
// The state of substep k is (x, v, C, F_trial, mu, lam, yield); mass is
// constant. Particles whose selection flag is set produce constant outputs,
// so their adjoints are zero. The quadratic B-spline weights are C1, so the
// x adjoint includes the weights' first and second derivatives.
#pragma once
#include "kernels.cuh"
#include "spectral.cuh"

// Minimum resident CTAs (of 128 threads) per SM asked of the compiler for the
// two particle kernels of the adjoint. The one-pass G2P adjoint keeps 18
// accumulators live across its stencil loop: at 4 CTAs (128 registers) it
// does not spill and took 43.5 us per 200k-particle substep, at 5 CTAs (96
// registers, 60 B spilled) 48.0 us, at 6 (80 registers, 132 B) 45.5 us.
#ifndef EMPM_ADJ_G2P_MIN_CTAS
#define EMPM_ADJ_G2P_MIN_CTAS 4
#endif
// 1: the G2P adjoint's scatter loops over the outer stencil axis at run time
#ifndef EMPM_ADJ_G2P_ROLL
#define EMPM_ADJ_G2P_ROLL 1
#endif
#ifndef EMPM_ADJ_P2G_MIN_CTAS
#define EMPM_ADJ_P2G_MIN_CTAS 4
#endif
// 1: the P2G adjoint's gather loops over the outer stencil axis at run time
// (a third of the unrolled code, for the instruction cache)
#ifndef EMPM_ADJ_P2G_ROLL
#define EMPM_ADJ_P2G_ROLL 1
#endif

namespace empm {

// second derivative of the quadratic B-spline weight at stencil offset o
EMPM_HD float bspline_d2(int o) { return o == 1 ? -2.f : 1.f; }

// ---------------------------------------------------------------------------
// G2P adjoint
// ---------------------------------------------------------------------------
struct AdjG2PArgs {
    ParticleArrays P;      // state of substep k (x)
    const float4*  x_next; // x after substep k (written by its G2P)
    F9Planes       Fe;     // elastic F of substep k
    MaterialArrays M;      // selection
    ParticleArrays Gn;     // adjoint of the state after substep k
    Launch         L;
    const float4*  vel;    // node velocities of substep k
    float4*        gacc;   // node velocity adjoint (accumulated here)
    float4*        gx;     // out: x adjoint through G2P
    F9Planes       gFe;    // out: F_elastic adjoint
    int            seg_cap;  // longest same-cell run summed with shuffles (a power of two)
};

// One pass over the stencil. Per node n (weight w, weight gradient dw, node
// velocity vg) with q_n = gv' + dt gx'_clamped + 4 inv_dx gC' (o_n - fx):
//   scatter   w q_n + gGv dw                       (gGv = dt gF' F_e^T)
//   x adjoint dot(vg, q_n) dw + inv_dx^2 H_n gGv^T vg
// and the forward's v' = sum w vg and grad v' = sum vg (x) dw, needed for the
// x and F_elastic adjoints, are summed in the same pass. Every sum factorises
// over the inner stencil axis (per row (i, j) the three nodes are combined
// with wz_k, dwz_k, (1, -2, 1) and k wz_k); the Hessian term is contracted
// with gGv row by row.
//
// Lanes whose particles share an instance and base cell (contiguous in cell
// order) sum their node-velocity adjoints with shuffles; the segment head
// issues one reduction per node, as k_p2g_warpagg does for the momentum.
// Every lane of the warp runs the node loop, invalid lanes with zeros.
// ROUNDS < 5: runs are capped at 2^ROUNDS lanes (a.seg_cap equals it), so the
// shuffle rounds the cap never needs are not compiled in; ROUNDS 5 takes any
// a.seg_cap.
template <int ROUNDS>
__global__ void __launch_bounds__(128, EMPM_ADJ_G2P_MIN_CTAS) k_adj_g2p(const AdjG2PArgs a) {
    const int seg_cap = ROUNDS < 5 ? (1 << ROUNDS) : a.seg_cap;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool live = p < a.L.n_total;
    const bool valid = live && !(a.M.sel && __ldg(a.M.sel + p) != 0);
    const int inst = live ? find_instance_particle(a.L, p) : 0;
    const StepConsts c = consts_of(a.L, inst);
    const float dt = c.step->dt;
    const float4 xm = valid ? __ldg(a.P.x + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    const V3 x = v3(xm.x, xm.y, xm.z);
    const Stencil st = make_stencil(x, valid ? c.inv_dx : 1.f);
    const bool in_grid = valid && stencil_in_grid(st, c.G);
    // segments of lanes with the same validity, instance and base cell
    const int b0 = valid ? st.b[0] : lane, b1 = valid ? st.b[1] : -1, b2 = valid ? st.b[2] : -1;
    const int u0 = __shfl_up_sync(0xffffffffu, b0, 1), u1 = __shfl_up_sync(0xffffffffu, b1, 1),
              u2 = __shfl_up_sync(0xffffffffu, b2, 1);
    const int uv = __shfl_up_sync(0xffffffffu, (int)valid, 1);
    const int ui = __shfl_up_sync(0xffffffffu, inst, 1);
    const bool run_head = lane == 0 || uv != (int)valid || ui != inst || u0 != b0 || u1 != b1 || u2 != b2;
    // runs longer than seg_cap (a power of two) get another head every seg_cap
    // lanes, as in k_p2g_warpagg
    const unsigned run_heads = __ballot_sync(0xffffffffu, run_head);
    const int run_start = 31 - __clz(run_heads & (0xffffffffu >> (31 - lane)));
    const bool head = run_head || ((lane - run_start) & (seg_cap - 1)) == 0;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const unsigned above = lane == 31 ? 0u : (heads & (0xffffffffu << (lane + 1)));
    const int end = above ? (__ffs(above) - 2) : 31;
    const int seglen = head ? end - lane + 1 : 1;
    const int maxlen = __reduce_max_sync(0xffffffffu, seglen);
    const unsigned take = (lane + 1 <= end ? 1u : 0u) | (lane + 2 <= end ? 2u : 0u) | (lane + 4 <= end ? 4u : 0u) |
                          (lane + 8 <= end ? 8u : 0u) | (lane + 16 <= end ? 16u : 0u);

    // x' = clamp(x + dt v'): the clamp passes the adjoint only strictly inside
    // the band. x + dt v' lies strictly inside it exactly when the clamped x'
    // that the forward G2P wrote does (a value clamped to a bound is not).
    const float dx = 1.f / c.inv_dx;
    const float lo = dx * 2.f, hi = c.grid_lim - dx * 2.f;
    const float4 xn = valid ? __ldg(a.x_next + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 gx4 = valid ? __ldg(a.Gn.x + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 gv4 = valid ? __ldg(a.Gn.v + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    const V3 gxu = v3(xn.x > lo && xn.x < hi ? gx4.x : 0.f, xn.y > lo && xn.y < hi ? gx4.y : 0.f,
                      xn.z > lo && xn.z < hi ? gx4.z : 0.f);
    // q_n = q0 + i Q0 + j Q1 + k Q2 with Q_c = 4 inv_dx gC'[:, c]; G_c = inv_dx gGv[:, c]
    V3 q0, Q0, Q1, Q2, G0, G1, G2;
    {
        const V3 gvt = v3(gv4.x, gv4.y, gv4.z) + dt * gxu;
        const M3 gC = valid ? f9_load(a.Gn.C, p) : m3_zero();
        const float c4 = 4.f * c.inv_dx;
        q0 = gvt - c4 * (gC * v3(st.fx[0], st.fx[1], st.fx[2]));
        Q0 = c4 * col(gC, 0);
        Q1 = c4 * col(gC, 1);
        Q2 = c4 * col(gC, 2);
        // F' = (I + dt grad v) F_e: gGv = dt gF' F_e^T
        const M3 gF = valid ? f9_load(a.Gn.F, p) : m3_zero();
        const M3 gGv = (dt * c.inv_dx) * (gF * transpose(valid ? f9_load(a.Fe, p) : m3_zero()));
        G0 = col(gGv, 0);
        G1 = col(gGv, 1);
        G2 = col(gGv, 2);
    }
    const float wz0 = st.w[2][0], wz1 = st.w[2][1], wz2 = st.w[2][2], kz2 = 2.f * wz2;
    const float uz0 = st.dw[2][0], uz1 = st.dw[2][1], uz2 = st.dw[2][2];
    const V3 zero = v3(0.f, 0.f, 0.f);
    V3 Vs = zero;                      // sum w vg (the forward's v')
    V3 D0 = zero, D1 = zero, D2 = zero;   // columns of sum vg (x) dweight / inv_dx
    // sum dot(vg, q) dweight + inv_dx sum H gGv^T vg, both over inv_dx (the
    // Hessian term contracted row by row: three accumulators instead of the
    // 18 of its moments, which let the kernel fit fewer registers)
    V3 X3 = zero;
    // node addresses: the block index sits above the 6 bits of the local
    // index, so the address of node (i, j, k) is a part of its row (i, j) plus
    // a part of k (formed once here)
    int zpart[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int iz = st.b[2] + k;
        zpart[k] = (iz >> 2) * 64 + (iz & 3);
    }
#if EMPM_ADJ_G2P_ROLL
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int i = 0; i < 3; ++i) {
        float wx, ux;
        bspline_at(st.fx[0], i, wx, ux);
        const float hx = bspline_d2(i);
        const V3 qi = q0 + (float)i * Q0;
        V3 Vi = zero;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wy = st.w[1][j], uy = st.dw[1][j];
            const float wxy = wx * wy, dxy = ux * wy, xdy = wx * uy;
            const V3 qij = j == 0 ? qi : qi + (float)j * Q1;
            // scatter value of node k: wz_k P + k wz_k Qr + dwz_k R
            const V3 P = wxy * qij + dxy * G0 + xdy * G1;
            const V3 Qr = wxy * Q2;
            const V3 R = wxy * G2;
            V3 vg[3];
            float sk[3];
            const int ix = st.b[0] + i, iy = st.b[1] + j;
            const long long row = (long long)(c.boff + ((ix >> 2) * c.NB + (iy >> 2)) * c.NB) * 64 +
                                  (ix & 3) * 16 + (iy & 3) * 4;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int iz = st.b[2] + k;
                const bool node_ok = valid && (in_grid || (ix >= 0 && iy >= 0 && iz >= 0 && ix < c.G && iy < c.G &&
                                                           iz < c.G));
                const long long addr = node_ok ? row + zpart[k] : 0;
                vg[k] = zero;
                if (node_ok) {
                    const float4 g4 = __ldg(a.vel + addr);
                    vg[k] = v3(g4.x, g4.y, g4.z);
                }
                const float wz = k == 0 ? wz0 : (k == 1 ? wz1 : wz2);
                const float uz = k == 0 ? uz0 : (k == 1 ? uz1 : uz2);
                V3 gvg = wz * P + uz * R;
                if (k == 1) gvg = gvg + wz1 * Qr;
                if (k == 2) gvg = gvg + kz2 * Qr;
                if (!node_ok) gvg = zero;
                sk[k] = dot(vg[k], qij);
                if (k) sk[k] += (float)k * dot(vg[k], Q2);
                // reduction rounds unrolled, each skipped by a warp-uniform branch
#pragma unroll
                for (int r = 0; r < ROUNDS; ++r) {
                    const int d = 1 << r;
                    if (d < maxlen) {
                        const float tx = __shfl_down_sync(0xffffffffu, gvg.x, d);
                        const float ty = __shfl_down_sync(0xffffffffu, gvg.y, d);
                        const float tz = __shfl_down_sync(0xffffffffu, gvg.z, d);
                        if (take & (1u << r)) { gvg.x += tx; gvg.y += ty; gvg.z += tz; }
                    }
                }
                if (head && node_ok) red_add_v4(a.gacc + addr, make_float4(gvg.x, gvg.y, gvg.z, 0.f));
            }
            const V3 T0 = wz0 * vg[0] + wz1 * vg[1] + wz2 * vg[2];
            const V3 T1 = uz0 * vg[0] + uz1 * vg[1] + uz2 * vg[2];
            const V3 T2 = vg[0] - 2.f * vg[1] + vg[2];
            const float sg0 = wz0 * sk[0] + wz1 * sk[1] + wz2 * sk[2];
            const float sg1 = uz0 * sk[0] + uz1 * sk[1] + uz2 * sk[2];
            Vi = Vi + wxy * T0;
            D0 = D0 + dxy * T0;
            D1 = D1 + xdy * T0;
            D2 = D2 + wxy * T1;
            // sum_n H_n gGv^T vg_n over the row, component a = sum_b dot(G_b, H[a][b] row sum), with
            // the pair row sums (hx wy) T0, (wx hy) T0, wxy T2, (ux uy) T0, dxy T1, xdy T1
            const float d00 = dot(G0, T0), d10 = dot(G1, T0), d01 = dot(G0, T1), d11 = dot(G1, T1);
            const float d21 = dot(G2, T1), d22 = dot(G2, T2);
            const float uxy = ux * uy;
            X3 = X3 + v3(dxy * (sg0 + d21) + (hx * wy) * d00 + uxy * d10,
                         xdy * (sg0 + d21) + uxy * d00 + (wx * bspline_d2(j)) * d10,
                         wxy * (sg1 + d22) + dxy * d01 + xdy * d11);
        }
        Vs = Vs + Vi;
    }
    if (!live) return;
    // F' = (I + dt grad v) F_e  ->  gF_e = (I + dt grad v)^T gF' (gF' read again rather than kept live)
    M3 A;   // I + dt grad v, grad v = inv_dx [D0 | D1 | D2] (columns)
    {
        const V3 dc[3] = {D0, D1, D2};
        const float s = dt * c.inv_dx;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cl = 0; cl < 3; ++cl) A.m[3 * r + cl] = (r == cl ? 1.f : 0.f) + s * comp(dc[cl], r);
    }
    f9_store(a.gFe, p, transpose(A) * (valid ? f9_load(a.Gn.F, p) : m3_zero()));
    // With G = inv_dx gGv the Hessian term inv_dx^2 sum H gGv^T vg is inv_dx sum H G^T vg (in X3).
    // The forward's C' = 4 inv_dx (...) enters the x adjoint as -4 inv_dx^2 gC'^T v' = -inv_dx (dot(Q_c, v'))_c.
    const V3 QV = v3(dot(Q0, Vs), dot(Q1, Vs), dot(Q2, Vs));
    const V3 gxa = gxu + c.inv_dx * (X3 - QV);
    a.gx[p] = make_float4(gxa.x, gxa.y, gxa.z, 0.f);
}

// ---------------------------------------------------------------------------
// grid adjoint over the touched blocks
// ---------------------------------------------------------------------------
struct AdjGridArgs {
    float4*        mom;     // accumulation of substep k; zeroed here
    float4*        gacc;    // node velocity adjoint; zeroed here
    float4*        gmom;    // out: adjoint of the accumulation (momentum xyz, mass w)
    unsigned char* flags;   // touched blocks of substep k; cleared here
    Launch         L;
};

// The grid adjoint of one node of block b (instance inst) whose accumulated
// momentum and mass are m: the forward update is replayed to learn which
// collider projections applied, then their transposes, the damping and the
// normalisation are applied to the node velocity adjoint (gacc, zeroed here).
__device__ __forceinline__ void adj_grid_node(const AdjGridArgs& a, int b, int inst, int lane, float4 m) {
    const InstanceConsts* I = a.L.inst + inst;
    const int G = __ldg(&I->G), NB = __ldg(&I->NB), boff = __ldg(&I->boff);
    const float damping = __ldg(&I->damping);
    const EmpmStep& st = a.L.steps[(size_t)a.L.table * a.L.n_inst + inst];
    const long long node = ((long long)b << 6) | lane;
    const float4 g4 = a.gacc[node];
    a.gacc[node] = make_float4(0.f, 0.f, 0.f, 0.f);
    V3 v = grid_velocity(m, st.dt, v3(__ldg(&I->g[0]), __ldg(&I->g[1]), __ldg(&I->g[2])), damping);
    unsigned long long codes = 0;
    if (st.n_colliders > 0) {
        int i, j, k;
        node_coords(((long long)(b - boff) << 6) | lane, NB, i, j, k);
        if (i < G && j < G && k < G) {
            const long long dense = ((long long)i * G + j) * G + k;
            apply_colliders_rec(st, i, j, k, G, __ldg(&I->dx), dense, v,
                                [&](int cidx, unsigned code) { codes |= (unsigned long long)code << (4 * cidx); });
        }
    }
    V3 g = v3(g4.x, g4.y, g4.z);
    for (int cidx = st.n_colliders - 1; codes != 0 && cidx >= 0; --cidx) {
        const unsigned code = (unsigned)(codes >> (4 * cidx)) & 15u;
        if (code & 1u) g.x = 0.f;
        if (code & 2u) g.y = 0.f;
        if (code & 4u) g.z = 0.f;
        if (code & 8u) g = g * 0.3f;
    }
    if (damping < 1.f) g = g - (1.f - damping) * g;
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m.w > 1e-15f) {
        const float inv = 1.f / m.w;
        out = make_float4(g.x * inv, g.y * inv, g.z * inv, -(g.x * m.x + g.y * m.y + g.z * m.z) * inv * inv);
    }
    a.gmom[node] = out;
}

// Over the blocks flagged in the grid (the recomputed substep): the kept
// momentum is read from the grid and zeroed there, and the flags cleared.
__global__ void __launch_bounds__(256) k_adj_grid(const AdjGridArgs a) {
    const int nblocks = a.L.nblocks;
    const int group = threadIdx.x >> 6;
    const int lane = threadIdx.x & 63;
    for (int base = blockIdx.x * 4; base < nblocks; base += gridDim.x * 4) {
        const int b = base + group;
        const bool active = b < nblocks && a.flags[b] != 0;
        __syncthreads();   // every group has read its flag before any is cleared
        if (!active) continue;
        const long long node = ((long long)b << 6) | lane;
        const float4 m = a.mom[node];
        a.mom[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        adj_grid_node(a, b, find_instance_block(a.L, b), lane, m);
        if (lane == 0) a.flags[b] = 0;
    }
}

// Over the blocks of a store slot (a stored substep): the momentum is read
// from the slot, so the grid's accumulator and flags are not used. One thread
// per node, grid-stride. With rslot, the same launch then writes the node
// velocities of the previous substep's slot back into the grid (vel) for the
// next G2P adjoint: this pass reads no velocities from the grid, and the G2P
// adjoint of this substep has already read them.
__global__ void __launch_bounds__(256) k_adj_grid_stored(const AdjGridArgs a, const float4* __restrict__ slot,
                                                         const int* __restrict__ slot_list, float4* __restrict__ vel,
                                                         const float4* __restrict__ rslot,
                                                         const int* __restrict__ rlist) {
    const long long total = (long long)__ldg(slot_list) * 64;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const long long k = idx >> 6;
        const int lane = (int)(idx & 63);
        const int b = __ldg(slot_list + 1 + k);
        adj_grid_node(a, b, find_instance_block(a.L, b), lane, __ldg(slot + k * 128 + lane));
    }
    if (!rslot) return;
    const long long rtotal = (long long)__ldg(rlist) * 64;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < rtotal; idx += stride) {
        const long long k = idx >> 6;
        const int in_block = (int)(idx & 63);
        const int b = __ldg(rlist + 1 + k);
        vel[((long long)b << 6) | in_block] = __ldg(rslot + k * 128 + 64 + in_block);
    }
}

// ---------------------------------------------------------------------------
// P2G + constitutive adjoint
// ---------------------------------------------------------------------------
struct AdjP2GArgs {
    ParticleArrays P;      // state of substep k (v after the velocity modifiers)
    MaterialArrays M;      // mu, lam, yield at the start of substep k; vol; selection; caller index
    Launch         L;      // step table with the modifiers
    const float4*  gmom;   // adjoint of the accumulation
    const float4*  gx;     // x adjoint through G2P
    F9Planes       gFe;    // F_elastic adjoint
    ParticleArrays G;      // out: adjoint of the state of substep k
    float*         g_mu;   // in: adjoint after substep k; out: before it
    float*         g_lam;
    float*         g_ys;
    float*         g_mass; // accumulated over substeps
};

// MAT: the material every instance of the launch uses (plasticine 5 and jelly
// 0 have kernels of their own), or -1 (switch per instance).
template <int MAT = -1>
__global__ void __launch_bounds__(128, EMPM_ADJ_P2G_MIN_CTAS) k_adj_p2g(const AdjP2GArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.L.n_total) return;
    if (a.M.sel && __ldg(a.M.sel + p) != 0) {
        a.G.x[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        a.G.v[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        f9_store(a.G.C, p, m3_zero());
        f9_store(a.G.F, p, m3_zero());
        return;   // material scalars are untouched by the substep: their adjoints carry over
    }
    const StepConsts c = consts_of(a.L, find_instance_particle(a.L, p));
    const EmpmStep& step = *c.step;
    const float dt = step.dt;
    const float4 xm = __ldg(a.P.x + p);
    const V3 x = v3(xm.x, xm.y, xm.z);
    const float mass = xm.w;
    const float4 vv = __ldg(a.P.v + p);
    const V3 v = v3(vv.x, vv.y, vv.z);
    const float vol = __ldg(a.M.vol + p);
    const M3 Cd = damp_affine(f9_load(a.P.C, p), c.rpic);

    // The gather runs before the constitutive evaluation, so that the SVD and
    // its dual-number Jacobians are not held in registers across it. The
    // stress enters the gather only through the force term's x derivative,
    // sum_n H_n Sv^T gmv_n (H_n the weight Hessian); the gather keeps its
    // moments sum_n H_n[pair] gmv_n and contracts them with Sv afterwards.
    const Stencil st = make_stencil(x, c.inv_dx);
    const bool in_grid = stencil_in_grid(st, c.G);
    const float dx = c.dx;
    const float idx2 = c.inv_dx * c.inv_dx;
    // Every sum of the gather factorises over the inner stencil axis: per row
    // (i, j) the three nodes are combined with the weights wz_k, dwz_k, the
    // second derivatives (1, -2, 1) and k wz_k, then the rows are summed with
    // weights in x and y. v + Cd dpos at node (i, j, k) is e_ij + k c2 with
    // c2 = dx Cd[:, 2], so s_k = gm_k + dot(gmv_k, e_ij) + k dot(gmv_k, c2).
    const V3 zero = v3(0.f, 0.f, 0.f);
    V3 Wg = zero, Im = zero, Jm = zero, Km = zero;   // sum w gmv, and its moments in i, j, k
    V3 S0 = zero, S1 = zero, S2 = zero;              // columns of sum gmv (x) dweight / inv_dx
    V3 X3 = zero;                                    // sum s dweight / inv_dx
    float gmass = 0.f;
    V3 Hg[6];                       // sum H[pair] gmv, pairs xx, yy, zz, xy, xz, yz (grid units)
#pragma unroll
    for (int r = 0; r < 6; ++r) Hg[r] = zero;
    const StencilAddr sa = stencil_addr(c.boff, c.NB, st.b);
    const V3 Cd0 = col(Cd, 0), Cd1 = col(Cd, 1), c2 = dx * col(Cd, 2);
    const V3 e0 = v - st.fx[2] * c2;
    const float wz0 = st.w[2][0], wz1 = st.w[2][1], wz2 = st.w[2][2], kz2 = 2.f * wz2;
    const float uz0 = st.dw[2][0], uz1 = st.dw[2][1], uz2 = st.dw[2][2];
#if EMPM_ADJ_P2G_ROLL
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int i = 0; i < 3; ++i) {
        float wx, ux;
        bspline_at(st.fx[0], i, wx, ux);
        const float hx = bspline_d2(i);
        const V3 ei = e0 + (((float)i - st.fx[0]) * dx) * Cd0;
        V3 Wi = zero;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float4 g[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                g[k] = (in_grid || node_in_grid(st.b, i, j, k, c.G)) ? __ldg(a.gmom + sa.at(i, j, k))
                                                                     : make_float4(0.f, 0.f, 0.f, 0.f);
            const V3 g0 = v3(g[0].x, g[0].y, g[0].z), g1 = v3(g[1].x, g[1].y, g[1].z),
                     g2 = v3(g[2].x, g[2].y, g[2].z);
            const V3 eij = ei + (((float)j - st.fx[1]) * dx) * Cd1;
            const float s0 = g[0].w + dot(g0, eij);
            const float s1 = g[1].w + dot(g1, eij) + dot(g1, c2);
            const float s2 = g[2].w + dot(g2, eij) + 2.f * dot(g2, c2);
            const V3 T0 = wz0 * g0 + wz1 * g1 + wz2 * g2;
            const V3 T1 = uz0 * g0 + uz1 * g1 + uz2 * g2;
            const V3 T2 = g0 - 2.f * g1 + g2;
            const V3 Tk = wz1 * g1 + kz2 * g2;
            const float sg0 = wz0 * s0 + wz1 * s1 + wz2 * s2;
            const float sg1 = uz0 * s0 + uz1 * s1 + uz2 * s2;
            const float wy = st.w[1][j], uy = st.dw[1][j];
            const float wxy = wx * wy, dxy = ux * wy, xdy = wx * uy;
            gmass += wxy * sg0;
            const V3 Wr = wxy * T0;
            Wi = Wi + Wr;
            if (j) Jm = Jm + (float)j * Wr;
            Km = Km + wxy * Tk;
            S0 = S0 + dxy * T0;
            S1 = S1 + xdy * T0;
            S2 = S2 + wxy * T1;
            X3 = X3 + v3(dxy * sg0, xdy * sg0, wxy * sg1);
            Hg[0] = Hg[0] + (hx * wy) * T0;
            Hg[1] = Hg[1] + (wx * bspline_d2(j)) * T0;
            Hg[2] = Hg[2] + wxy * T2;
            Hg[3] = Hg[3] + (ux * uy) * T0;
            Hg[4] = Hg[4] + dxy * T1;
            Hg[5] = Hg[5] + xdy * T1;
        }
        Wg = Wg + Wi;
        Im = Im + (float)i * Wi;
    }
    // sum (w gmv) (x) dpos, columns dx (moment - fx Wg); sum gmv (x) dweight, columns inv_dx S
    M3 gCd, gSv;
    {
        const V3 cc[3] = {dx * (Im - st.fx[0] * Wg), dx * (Jm - st.fx[1] * Wg), dx * (Km - st.fx[2] * Wg)};
        const V3 sc[3] = {c.inv_dx * S0, c.inv_dx * S1, c.inv_dx * S2};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cl = 0; cl < 3; ++cl) {
                gCd.m[3 * r + cl] = comp(cc[cl], r);
                gSv.m[3 * r + cl] = comp(sc[cl], r);
            }
    }
    V3 gxa = (mass * c.inv_dx) * X3 - mass * (transpose(Cd) * Wg);

    V3 gv = mass * Wg;
    {
        gCd = mass * gCd;
        M3 gC = m3_zero();
        if (!(c.rpic < -0.001f)) gC = (1.f - c.rpic) * gCd + (c.rpic / 2.f) * (gCd - transpose(gCd));
        f9_store(a.G.C, p, gC);
    }

    // velocity modifiers, in reverse order (mpm_solver_diff.py:977-991, 1022-1036,
    // 1098-1142, 1198-1212, 1332-1348, 1391-1410). A modifier that overwrites v
    // cuts the adjoint; the rotation modifier's dependence on x is not
    // differentiated.
    if (step.n_modifiers > 0) {
        const int mi = a.M.pid ? __ldg(a.M.pid + p) : p;
        for (int m = step.n_modifiers - 1; m >= 0; --m) {
            const EmpmModifier& md = step.modifiers[m];
            if (md.gate != EMPM_GATE_APPLY) continue;
            const int mk = md.mask ? __ldg(md.mask + mi) : 0;
            switch (md.kind) {
                case EMPM_MOD_IMPULSE:
                    if (mk == 1) gmass -= dot(gv, v3(md.vec[0], md.vec[1], md.vec[2])) * dt / (mass * mass);
                    break;
                case EMPM_MOD_SET_VELOCITY:
                case EMPM_MOD_ROTATION:
                    if (mk == 1) gv = v3(0.f, 0.f, 0.f);
                    break;
                case EMPM_MOD_SET_VELOCITY_LAYERED:
                    if (mk >= (int)md.scale[0]) gv = v3(0.f, 0.f, 0.f);
                    break;
                case EMPM_MOD_MOVER:
                    if (mk == 1) gxa = gxa + md.scale[0] * cross(gv, v3(md.normal[0], md.normal[1], md.normal[2]));
                    break;
                default: break;
            }
        }
    }
    a.G.v[p] = make_float4(gv.x, gv.y, gv.z, 0.f);
    a.g_mass[p] += gmass;
    const M3 g_tau = (-vol * dt) * gSv;

    SpectralEval e;
    spectral_eval<MAT>(f9_load(a.P.F, p), __ldg(a.M.mu + p), __ldg(a.M.lam + p), __ldg(a.M.ys + p), dt, *c.ms, e);
    {
        // sum_n H_n Sv^T gmv_n, component a = sum_b dot(column b of Sv, sum_n H_n[a][b] gmv_n)
        const M3 Sv = (-vol) * spectral_tau(e);
        const V3 c0 = v3(Sv.m[0], Sv.m[3], Sv.m[6]);
        const V3 c1 = v3(Sv.m[1], Sv.m[4], Sv.m[7]);
        const V3 c2 = v3(Sv.m[2], Sv.m[5], Sv.m[8]);
        const V3 hS = v3(dot(c0, Hg[0]) + dot(c1, Hg[3]) + dot(c2, Hg[4]),
                         dot(c0, Hg[3]) + dot(c1, Hg[1]) + dot(c2, Hg[5]),
                         dot(c0, Hg[4]) + dot(c1, Hg[5]) + dot(c2, Hg[2]));
        gxa = gxa + (dt * idx2) * hS;
        const float4 gxg = __ldg(a.gx + p);
        a.G.x[p] = make_float4(gxa.x + gxg.x, gxa.y + gxg.y, gxa.z + gxg.z, 0.f);
    }

    const SpectralGrad sg = spectral_adjoint(e, f9_load(a.gFe, p), g_tau, a.g_mu[p], a.g_lam[p], a.g_ys[p]);
    f9_store(a.G.F, p, sg.gFt);
    a.g_mu[p] = sg.g_mu;
    a.g_lam[p] = sg.g_lam;
    a.g_ys[p] = sg.g_ys;
}

// dL/dE, dL/dnu from dL/dmu, dL/dlam (compute_mu_lam_from_E_nu, mpm_utils.py:277-283),
// and dL/ddensity from dL/dmass with mass = density * vol (mpm_data_structure.py:719-726)
__global__ void k_prepare_adjoint(const float* E, const float* nu, const float* g_mu, const float* g_lam, float* g_E,
                                  float* g_nu, const float* vol, const float* g_mass, float* g_density, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (g_E && g_nu) {
        const float e = E[p], q = nu[p];
        const float a = 1.f + q, b = 1.f - 2.f * q;
        const float dmu_dE = 1.f / (2.f * a), dlam_dE = q / (a * b);
        const float dmu_dnu = -e / (2.f * a * a), dlam_dnu = e * (1.f + 2.f * q * q) / (a * a * b * b);
        g_E[p] = g_mu[p] * dmu_dE + g_lam[p] * dlam_dE;
        g_nu[p] = g_mu[p] * dmu_dnu + g_lam[p] * dlam_dnu;
    }
    if (g_density) g_density[p] = g_mass[p] * vol[p];
}

// ---------------------------------------------------------------------------
// stored substeps of a segment (EMPM_OPT_ADJ_STORE)
// ---------------------------------------------------------------------------
// The node velocities of a store slot back into the grid, where the G2P
// adjoint gathers them (the grid adjoint reads the momenta from the slot).
__global__ void __launch_bounds__(256) k_restore_grid(float4* __restrict__ vel, const float4* __restrict__ src,
                                                      const int* __restrict__ src_list) {
    const long long total = (long long)__ldg(src_list) * 64;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long slot = idx >> 6;
        const int in_block = (int)(idx & 63);
        const int b = __ldg(src_list + 1 + slot);
        vel[((long long)b << 6) | in_block] = __ldg(src + slot * 128 + 64 + in_block);
    }
}

}  // namespace empm
