// kernels.cuh — __global__ kernels of one MLS-MPM substep over a batch of
// independent simulation instances (a single simulation is a batch of one).
//
// Batch layout: the particles of instance i occupy [poff_i, poff_i + n_i) of
// every particle array, both in the caller's order and in the library's
// cell-sorted order (the sort key starts with the instance's grid blocks, so
// a sort never moves a particle across instances); the grids are the
// instances' blocked grids one after the other, instance i starting at the
// global 4^3 block boff_i. Every kernel looks its instance up in a small
// device table by particle index or block index.
//
// Launch paths:
//   * direct: one particle per thread, 16-byte vector reductions into the grid;
//   * sorted (rollouts): particles in cell order, re-sorted every few substeps;
//     P2G sums the contributions of same-cell particles of a warp with
//     shuffles and issues one reduction per cell and node (default), or
//     accumulates per chunk in a shared-memory node tile (option);
//     G2P gathers directly or from a staged shared-memory tile (option);
//   * the grid update visits only the 4^3 node blocks that P2G touched.
#pragma once
#include <limits.h>
#include "../../include/empm_b200.h"
#include "grid.cuh"
#include "substep.cuh"

// Minimum resident CTAs per SM asked of the compiler for the two particle
// kernels of the sorted path (register caps: 65536 / (threads x CTAs)).
#ifndef EMPM_P2G_MIN_CTAS
#define EMPM_P2G_MIN_CTAS 4
#endif
#ifndef EMPM_G2P_MIN_CTAS
#define EMPM_G2P_MIN_CTAS 8
#endif
// ... and for the fused G2P + stress + P2G kernel
#ifndef EMPM_FUSED_MIN_CTAS
#define EMPM_FUSED_MIN_CTAS 4
#endif
// 1: each warp of the fused kernel first copies the grid nodes its lanes'
// stencils cover (their bounding box, at most EMPM_WARP_TILE_NODES nodes) into
// shared memory and gathers from there; warps whose box is larger, leaves the
// grid or spans two instances gather from global memory. Measured on the
// population workload it is slower than gathering through L1 (648 us per
// launch with 128-node boxes, 613 us with 192, against 595 us), so it is off.
#ifndef EMPM_FUSED_WARP_TILE
#define EMPM_FUSED_WARP_TILE 0
#endif
#ifndef EMPM_WARP_TILE_NODES
#define EMPM_WARP_TILE_NODES 128
#endif
// 1: the fused kernel's G2P gathers with a run-time outer stencil loop
// (population workload: 598 us per launch against 604 us fully unrolled; at 3
// or 2 CTAs per SM 603-608 and 722 us)
#ifndef EMPM_FUSED_G2P_LOOP
#define EMPM_FUSED_G2P_LOOP 1
#endif

namespace empm {

// -------------------------------------------------------------------------
// instance table and per-launch context
// -------------------------------------------------------------------------
struct InstanceConsts {
    int   n, poff;            // particles
    int   G, NB, boff;        // grid: resolution, blocks per axis, first global block
    float dx, inv_dx, grid_lim, rpic, damping;
    float g[3];
    MaterialScalars ms;
};

struct Launch {
    const InstanceConsts* inst;
    int             n_inst;
    int             n_total;       // particles over all instances
    int             nblocks;       // grid blocks over all instances
    const EmpmStep* steps;         // device step tables: steps[table * n_inst + instance]
    int             table;         // step table of this substep
    unsigned*       status;
};

// per-instance view used by the particle/node device functions
struct StepConsts {
    int   G, NB, boff;
    float dx, inv_dx, grid_lim, rpic;
    // the material constants stay in the instance table: the return maps read
    // them only when a particle yields, so they are not held in registers
    // across a particle's substep (fused population kernel 560 -> 558 us)
    const MaterialScalars* ms;
    const EmpmStep* step;
    unsigned* status;
};

__device__ __forceinline__ int find_instance_particle(const Launch& L, int p) {
    int lo = 0, hi = L.n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&L.inst[mid].poff) <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_instance_block(const Launch& L, int b) {
    int lo = 0, hi = L.n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&L.inst[mid].boff) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ StepConsts consts_of(const Launch& L, int i) {
    const InstanceConsts* I = L.inst + i;
    StepConsts c;
    c.G = __ldg(&I->G);
    c.NB = __ldg(&I->NB);
    c.boff = __ldg(&I->boff);
    c.dx = __ldg(&I->dx);
    c.inv_dx = __ldg(&I->inv_dx);
    c.grid_lim = __ldg(&I->grid_lim);
    c.rpic = __ldg(&I->rpic);
    c.ms = &I->ms;
    c.step = L.steps + (size_t)L.table * L.n_inst + i;
    c.status = L.status;
    return c;
}

__device__ __forceinline__ long long gaddr(const StepConsts& c, int i, int j, int k) {
    return ((long long)(c.boff + block_of(i, j, k, c.NB)) << 6) | ((i & 3) << 4) | ((j & 3) << 2) | (k & 3);
}

// Addresses of the 27 nodes of a stencil with base node b: gaddr of node
// b + (i, j, k) is x(i) + y[j] + z[k]. The block index sits above the 6 bits of
// the local index, so gaddr's OR is a sum of one term per axis; x(i) carries
// the instance's block offset. Valid only for nodes inside the grid.
struct StencilAddr {
    int bx, boff, nb2;   // x[i] is rebuilt from these where it is used (fewer live registers)
    int y[3], z[3];
    EMPM_HD long long x(int i) const {
        const int ix = bx + i;
        return ((long long)(boff + (ix >> 2) * nb2) << 6) | ((ix & 3) << 4);
    }
    EMPM_HD long long at(int i, int j, int k) const { return x(i) + (long long)(y[j] + z[k]); }
};

EMPM_HD StencilAddr stencil_addr(int boff, int NB, const int b[3]) {
    StencilAddr a;
    a.bx = b[0];
    a.boff = boff;
    a.nb2 = NB * NB;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        const int iy = b[1] + o, iz = b[2] + o;
        a.y[o] = (((iy >> 2) * NB) << 6) | ((iy & 3) << 2);
        a.z[o] = ((iz >> 2) << 6) | (iz & 3);
    }
    return a;
}

// stencil node (i, j, k) inside the instance's grid (for stencils that are not entirely inside)
EMPM_HD bool node_in_grid(const int b[3], int i, int j, int k, int G) {
    const int ix = b[0] + i, iy = b[1] + j, iz = b[2] + k;
    return ix >= 0 && iy >= 0 && iz >= 0 && ix < G && iy < G && iz < G;
}

// -------------------------------------------------------------------------
// particle arrays
// -------------------------------------------------------------------------
struct ParticleArrays {
    float4*  x;      // (x, y, z, mass)
    float4*  v;      // (vx, vy, vz, 0)
    F9Planes C;
    F9Planes F;      // F_trial
};

struct MaterialArrays {
    const float* vol;
    float*       mu;
    float*       lam;
    float*       ys;
    const int*   sel;   // NULL = all simulated
    const int*   pid;   // caller index of each particle (NULL = identity)
};

// Stress + everything P2G needs for particle p (modifiers applied, material
// write-back, elastic F handed to G2P). Returns false for unsimulated particles.
template <int MAT = -1>
__device__ __forceinline__ bool prepare_particle(const ParticleArrays& P, const MaterialArrays& M, F9Planes Fe,
                                                 const StepConsts& c, int p, P2GParticle& q) {
    if (M.sel && __ldg(M.sel + p) != 0) return false;
    const EmpmStep& st = *c.step;
    if (st.hold) return false;   // held instance: no contribution this substep
    const float4 xm = __ldg(P.x + p);
    const float4 vv = __ldg(P.v + p);
    const V3 x = v3(xm.x, xm.y, xm.z);
    V3 v = v3(vv.x, vv.y, vv.z);
    if (st.n_modifiers > 0) {
        const int mi = M.pid ? __ldg(M.pid + p) : p;
        if (apply_modifiers(st, mi, x, xm.w, v)) P.v[p] = make_float4(v.x, v.y, v.z, vv.w);
    }
    float mu = __ldg(M.mu + p), lam = __ldg(M.lam + p), ys = __ldg(M.ys + p);
    const ConstitutiveOut co = constitutive<MAT>(f9_load(P.F, p), mu, lam, ys, st.dt, *c.ms);
    f9_store(Fe, p, co.F);
    if (co.mat_changed) { M.mu[p] = mu; M.lam[p] = lam; M.ys[p] = ys; }
    q.st = make_stencil(x, c.inv_dx);
    q.wm_scale = xm.w;
    q.v = v;
    q.Cd = damp_affine(f9_load(P.C, p), c.rpic);
    q.Sv = (-__ldg(M.vol + p)) * co.tau;
    return true;
}

__device__ __forceinline__ void mark_stencil_blocks(unsigned char* flags, const Stencil& st, const StepConsts& c) {
    const int G = c.G;
    const int lo[3] = {max(st.b[0], 0), max(st.b[1], 0), max(st.b[2], 0)};
    const int hi[3] = {min(st.b[0] + 2, G - 1), min(st.b[1] + 2, G - 1), min(st.b[2] + 2, G - 1)};
    for (int bi = lo[0] >> 2; bi <= hi[0] >> 2; ++bi)
        for (int bj = lo[1] >> 2; bj <= hi[1] >> 2; ++bj)
            for (int bk = lo[2] >> 2; bk <= hi[2] >> 2; ++bk) flags[c.boff + (bi * c.NB + bj) * c.NB + bk] = 1;
}

// direct scatter of one prepared particle into the blocked grid
__device__ __forceinline__ void scatter_global(const P2GParticle& q, const StepConsts& c, float4* grid,
                                               unsigned char* flags) {
    const int G = c.G;
    const bool in_grid = stencil_in_grid(q.st, G);
    if (!in_grid) atomicOr(c.status, EMPM_STATUS_OUT_OF_BAND);
    const P2GPre pre = p2g_pre(q, c.dx, c.inv_dx, c.step->dt);
    p2g_emit(pre, [&](int i, int j, int k, float4 v) {
        if (in_grid || node_in_grid(q.st.b, i, j, k, G))
            red_add_v4(grid + gaddr(c, q.st.b[0] + i, q.st.b[1] + j, q.st.b[2] + k), v);
    });
    mark_stencil_blocks(flags, q.st, c);
}

// -------------------------------------------------------------------------
// direct path
// -------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_p2g_direct(ParticleArrays P, MaterialArrays M, F9Planes Fe, Launch L,
                                                    float4* grid, unsigned char* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    const StepConsts c = consts_of(L, find_instance_particle(L, p));
    P2GParticle q;
    if (!prepare_particle(P, M, Fe, c, p, q)) return;
    scatter_global(q, c, grid, flags);
}

// -------------------------------------------------------------------------
// grid update over touched 4^3 blocks (both paths)
// -------------------------------------------------------------------------
struct GridUpdateArgs {
    float4*        mom;      // accumulation; zeroed here for the next substep
    float4*        vel;      // node velocity after the boundary conditions (w = node mass)
    unsigned char* flags;    // touched blocks; cleared here
    Launch         L;
    // optional store slot of the listed blocks (stored segments): per listed
    // block its 64 node momenta, then its 64 node velocities; the list count
    // and ids; a running maximum of the counts. A substep with more than
    // store_cap listed blocks stores only its count.
    float4*        store = nullptr;
    int*           store_list = nullptr;
    int            store_cap = 0;
    int*           max_count = nullptr;
};

// One touched 4^3 block (64 nodes, two per lane of the calling warp):
// normalisation, gravity, damping and boundary conditions.
template <bool kKeep>
__device__ __forceinline__ void grid_update_block(const GridUpdateArgs& a, int b, int lane) {
    const int inst = find_instance_block(a.L, b);
    const InstanceConsts* I = a.L.inst + inst;
    const int G = __ldg(&I->G), NB = __ldg(&I->NB), boff = __ldg(&I->boff);
    const float dx = __ldg(&I->dx), damping = __ldg(&I->damping);
    const V3 g = v3(__ldg(&I->g[0]), __ldg(&I->g[1]), __ldg(&I->g[2]));
    const EmpmStep& st = a.L.steps[(size_t)a.L.table * a.L.n_inst + inst];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int in_block = lane + 32 * h;
        const long long node = ((long long)b << 6) | in_block;
        const float4 m = a.mom[node];
        if (!kKeep) a.mom[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        V3 v = grid_velocity(m, st.dt, g, damping);
        if (st.n_colliders > 0) {
            int i, j, k;
            node_coords(((long long)(b - boff) << 6) | in_block, NB, i, j, k);
            if (i < G && j < G && k < G) {
                const long long dense = ((long long)i * G + j) * G + k;
                apply_colliders(st, i, j, k, G, dx, dense, v);
            }
        }
        a.vel[node] = make_float4(v.x, v.y, v.z, m.w);
    }
}

// Grid update over the touched blocks. Each warp reads 32 block flags at a
// time (coalesced), takes the set ones from a ballot and updates those
// blocks; each lane clears its own flag afterwards, so no block-wide barrier
// is needed. kKeep leaves the accumulation and the flags in place (the
// adjoint replays the boundary conditions from the accumulated momentum).
template <bool kKeep>
__device__ __forceinline__ void grid_update_blocks(const GridUpdateArgs& a) {
    const int nblocks = a.L.nblocks;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < nblocks; base += nwarps * 32) {
        const long long b = base + lane;
        const bool active = b < nblocks && a.flags[b] != 0;
        unsigned mask = __ballot_sync(0xffffffffu, active);
        while (mask) {
            const int j = __ffs(mask) - 1;
            mask &= mask - 1;
            grid_update_block<kKeep>(a, (int)(base + j), lane);
        }
        if (!kKeep && active) a.flags[b] = 0;
    }
}

__global__ void __launch_bounds__(256) k_grid_update_sparse(const GridUpdateArgs a) { grid_update_blocks<false>(a); }

// Touched blocks -> list: active[0] counts them, active[1 + i] are their ids
// (in no particular order) and active[1 + nblocks + i] their instances (the
// lookup done once per block here rather than once per node by the update).
// Clears the flags unless kKeep. active holds 1 + 2 * nblocks ints.
template <bool kKeep>
__global__ void __launch_bounds__(256) k_collect_blocks(unsigned char* flags, int nblocks, int* active, const Launch L) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool on = b < nblocks && flags[b] != 0;
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (m == 0u) return;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(active, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (on) {
        const int slot = base + __popc(m & ((1u << lane) - 1u));
        active[1 + slot] = b;
        active[1 + nblocks + slot] = find_instance_block(L, b);
        if (!kKeep) flags[b] = 0;
    }
}

// Grid update over the listed blocks, one thread per node (grid-stride).
template <bool kKeep>
__global__ void __launch_bounds__(256) k_grid_update_list(const GridUpdateArgs a, const int* active) {
    const int count = __ldg(active);
    const long long total = (long long)count * 64;
    if (a.store && blockIdx.x == 0 && threadIdx.x == 0) {
        a.store_list[0] = count;
        if (a.max_count) atomicMax(a.max_count, count);
    }
    const bool save = a.store && count <= a.store_cap;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int b = __ldg(active + 1 + (idx >> 6));
        const int in_block = (int)(idx & 63);
        const int inst = __ldg(active + 1 + a.L.nblocks + (idx >> 6));
        const InstanceConsts* I = a.L.inst + inst;
        const EmpmStep& st = a.L.steps[(size_t)a.L.table * a.L.n_inst + inst];
        const long long node = ((long long)b << 6) | in_block;
        const float4 m = a.mom[node];
        if (!kKeep) a.mom[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        V3 v = grid_velocity(m, st.dt, v3(__ldg(&I->g[0]), __ldg(&I->g[1]), __ldg(&I->g[2])), __ldg(&I->damping));
        if (st.n_colliders > 0) {
            const int G = __ldg(&I->G), NB = __ldg(&I->NB), boff = __ldg(&I->boff);
            int i, j, k;
            node_coords(((long long)(b - boff) << 6) | in_block, NB, i, j, k);
            if (i < G && j < G && k < G) {
                const long long dense = ((long long)i * G + j) * G + k;
                apply_colliders(st, i, j, k, G, __ldg(&I->dx), dense, v);
            }
        }
        const float4 v4 = make_float4(v.x, v.y, v.z, m.w);
        a.vel[node] = v4;
        if (save) {
            const long long slot = idx >> 6;
            a.store[slot * 128 + in_block] = m;
            a.store[slot * 128 + 64 + in_block] = v4;
            if (in_block == 0) a.store_list[1 + slot] = b;
        }
    }
}

// Grid update over the listed blocks, one warp per block and two nodes per
// lane (grid-stride over the list): the block id, its instance, the instance
// constants and the step table are read once per warp, where
// k_grid_update_list reads them once per node.
template <bool kKeep>
__global__ void __launch_bounds__(256) k_grid_update_warps(const GridUpdateArgs a, const int* active) {
    const int count = __ldg(active);
    if (a.store && blockIdx.x == 0 && threadIdx.x == 0) {
        a.store_list[0] = count;
        if (a.max_count) atomicMax(a.max_count, count);
    }
    const bool save = a.store && count <= a.store_cap;
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long slot = warp; slot < count; slot += nwarps) {
        const int b = __ldg(active + 1 + slot);
        const int inst = __ldg(active + 1 + a.L.nblocks + slot);
        const InstanceConsts* I = a.L.inst + inst;
        const EmpmStep& st = a.L.steps[(size_t)a.L.table * a.L.n_inst + inst];
        const V3 g = v3(__ldg(&I->g[0]), __ldg(&I->g[1]), __ldg(&I->g[2]));
        const float damping = __ldg(&I->damping);
        const float dt = st.dt;
        const int n_coll = st.n_colliders;
        const int G = __ldg(&I->G), NB = __ldg(&I->NB), boff = __ldg(&I->boff);
        const float dx = __ldg(&I->dx);
        const long long base = (long long)b << 6;
        const float4 m0 = a.mom[base + lane];
        const float4 m1 = a.mom[base + lane + 32];
        if (!kKeep) {
            a.mom[base + lane] = make_float4(0.f, 0.f, 0.f, 0.f);
            a.mom[base + lane + 32] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int in_block = lane + 32 * h;
            const float4 m = h ? m1 : m0;
            V3 v = grid_velocity(m, dt, g, damping);
            if (n_coll > 0) {
                int i, j, k;
                node_coords(((long long)(b - boff) << 6) | in_block, NB, i, j, k);
                if (i < G && j < G && k < G) {
                    const long long dense = ((long long)i * G + j) * G + k;
                    apply_colliders(st, i, j, k, G, dx, dense, v);
                }
            }
            const float4 v4 = make_float4(v.x, v.y, v.z, m.w);
            a.vel[base + in_block] = v4;
            if (save) {
                a.store[slot * 128 + in_block] = m;
                a.store[slot * 128 + 64 + in_block] = v4;
            }
        }
        if (save && lane == 0) a.store_list[1 + slot] = b;
    }
}

// -------------------------------------------------------------------------
// G2P (shared by both paths through the fetch functor)
// -------------------------------------------------------------------------
template <typename Fetch>
__device__ __forceinline__ void g2p_particle(const ParticleArrays& P, F9Planes Fe, const MaterialArrays& M,
                                             const ParticleArrays& out, const StepConsts& c, int p, Fetch fetch) {
    if (M.sel && __ldg(M.sel + p) != 0) {
        __stcs(out.x + p, make_float4(0.f, 0.f, 0.f, __ldg(P.x + p).w));
        __stcs(out.v + p, make_float4(0.f, 0.f, 0.f, 0.f));
        f9_store(out.C, p, m3_zero());
        f9_store(out.F, p, m3_identity());
        return;
    }
    if (c.step->hold) {   // held instance: the state passes through unchanged
        __stcs(out.x + p, __ldg(P.x + p));
        __stcs(out.v + p, __ldg(P.v + p));
        f9_store(out.C, p, f9_load(P.C, p));
        f9_store(out.F, p, f9_load(P.F, p));
        return;
    }
    const float dt = c.step->dt;
    const float4 xm = __ldg(P.x + p);
    const V3 x = v3(xm.x, xm.y, xm.z);
    const Stencil st = make_stencil(x, c.inv_dx);
    const bool in_grid = stencil_in_grid(st, c.G);
    const G2POut o = g2p_gather(st, c.inv_dx, fetch.bind(st, in_grid));
    const float dx = 1.f / c.inv_dx;
    const float lo = dx * 2.f, hi = c.grid_lim - dx * 2.f;
    V3 nx = x + dt * o.v;
    nx = v3(fminf(fmaxf(nx.x, lo), hi), fminf(fmaxf(nx.y, lo), hi), fminf(fmaxf(nx.z, lo), hi));
    const M3 Fn = (m3_identity() + dt * o.gradv) * f9_load(Fe, p);
    __stcs(out.x + p, make_float4(nx.x, nx.y, nx.z, xm.w));
    __stcs(out.v + p, make_float4(o.v.x, o.v.y, o.v.z, 0.f));
    f9_store(out.C, p, o.C);
    f9_store(out.F, p, Fn);
    unsigned flags = 0;
    if (!finite3(o.v) || !finite3(nx) || !isfinite(Fn.m[0] + Fn.m[4] + Fn.m[8])) flags |= EMPM_STATUS_NAN;
    if (fmaxf(fmaxf(fabsf(o.v.x), fabsf(o.v.y)), fabsf(o.v.z)) * dt > dx) flags |= EMPM_STATUS_CFL;
    if (!in_grid) flags |= EMPM_STATUS_OUT_OF_BAND;
    if (flags) atomicOr(c.status, flags);
}

// Node velocities from the blocked grid. bind() precomputes the stencil's
// node addresses; nodes outside the grid read as zero.
struct GlobalFetch {
    const float4* vel;
    const StepConsts* c;
    struct Bound {
        const float4* vel;
        StencilAddr sa;
        const int* b;
        int G;
        bool in_grid;
        __device__ __forceinline__ V3 operator()(int i, int j, int k) const {
            if (!in_grid && !node_in_grid(b, i, j, k, G)) return v3(0.f, 0.f, 0.f);
            const float4 g = __ldg(vel + sa.at(i, j, k));
            return v3(g.x, g.y, g.z);
        }
    };
    __device__ __forceinline__ Bound bind(const Stencil& st, bool in_grid) const {
        return Bound{vel, stencil_addr(c->boff, c->NB, st.b), st.b, c->G, in_grid};
    }
};

// Node velocities from a warp's shared-memory copy of the nodes its lanes'
// stencils cover: a box with origin o and extents e (tile index
// ((i - o0) * e1 + (j - o1)) * e2 + (k - o2)). The outer axis may be a run-time
// index (g2p_gather_rt), so its term is formed per call.
struct WarpTileFetch {
    const float4* tile;
    int o0, o1, o2, e1, e2;
    struct Bound {
        const float4* tile;
        int x0, e12;
        int y[3], z[3];
        __device__ __forceinline__ V3 operator()(int i, int j, int k) const {
            const float4 g = tile[x0 + i * e12 + y[j] + z[k]];
            return v3(g.x, g.y, g.z);
        }
    };
    __device__ __forceinline__ Bound bind(const Stencil& st, bool) const {
        Bound b;
        b.tile = tile;
        b.e12 = e1 * e2;
        b.x0 = (st.b[0] - o0) * b.e12;
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            b.y[o] = (st.b[1] + o - o1) * e2;
            b.z[o] = st.b[2] + o - o2;
        }
        return b;
    }
};

__global__ void __launch_bounds__(128, EMPM_G2P_MIN_CTAS) k_g2p_direct(ParticleArrays P, F9Planes Fe, MaterialArrays M,
                                                    ParticleArrays out, Launch L, const float4* vel) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    const StepConsts c = consts_of(L, find_instance_particle(L, p));
    GlobalFetch f{vel, &c};
    g2p_particle(P, Fe, M, out, c, p, f);
}

// -------------------------------------------------------------------------
// sorted path: cell keys, counting sort, permutation
// -------------------------------------------------------------------------
// Sort key of a particle: its base cell in block-major order over the whole
// batch, ((boff + block) << 6) | in-block cell, so one counting sort orders
// particles by instance, 4^3 block and cell. Out-of-band cells are clamped.
__global__ void k_sort_keys(const float4* x, Launch L, int* keys, int* ranks, int* cell_counts, int* block_counts) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.n_total) return;
    const int inst = find_instance_particle(L, p);
    const InstanceConsts* I = L.inst + inst;
    const int G = __ldg(&I->G), NB = __ldg(&I->NB);
    const float inv_dx = __ldg(&I->inv_dx);
    const float4 xm = __ldg(x + p);
    const float xs[3] = {xm.x, xm.y, xm.z};
    int b[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int t = base_node(xs[a], inv_dx);
        b[a] = t < 0 ? 0 : (t >= G ? G - 1 : t);
    }
    const int blk = __ldg(&I->boff) + block_of(b[0], b[1], b[2], NB);
    const int key = (blk << 6) | ((b[0] & 3) << 4) | ((b[1] & 3) << 2) | (b[2] & 3);
    keys[p] = key;
    ranks[p] = atomicAdd(cell_counts + key, 1);
    atomicAdd(block_counts + blk, 1);
}

// number of chunks (<= `chunk` particles, never spanning two blocks) per block
__global__ void k_chunk_counts(const int* block_counts, int* chunk_counts, int nblocks, int chunk) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    chunk_counts[b] = (block_counts[b] + chunk - 1) / chunk;
}

// Cell offsets: one warp per block, exclusive scan of its 64 cell counts on
// top of the block's start offset; writes the block's chunks; zeroes the
// counts for the next sort. Empty blocks only report the chunk total.
__global__ void k_cell_scan(int* cell_counts, int* block_counts, const int* block_offsets, const int* chunk_offsets,
                            const int* chunk_counts, int* cell_offsets, int2* chunks, int* nchunks, int nblocks,
                            int chunk) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nblocks) return;
    const int cnt = block_counts[warp];
    if (warp == nblocks - 1 && lane == 0) *nchunks = chunk_offsets[warp] + chunk_counts[warp];
    if (cnt == 0) return;
    const long long c0 = (long long)warp * 64 + 2 * lane;
    const int a = cell_counts[c0], b = cell_counts[c0 + 1];
    int incl = a + b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    const int off = block_offsets[warp];
    const int excl = incl - (a + b) + off;
    cell_offsets[c0] = excl;
    cell_offsets[c0 + 1] = excl + a;
    cell_counts[c0] = 0;
    cell_counts[c0 + 1] = 0;
    const int co = chunk_offsets[warp];
    for (int k = lane; k * chunk < cnt; k += 32) chunks[co + k] = make_int2(off + k * chunk, min(chunk, cnt - k * chunk));
    __syncwarp();
    if (lane == 0) block_counts[warp] = 0;
}

struct PermuteArgs {
    ParticleArrays src, dst;
    const float* vol_s; float* vol_d;
    const float* mu_s;  float* mu_d;
    const float* lam_s; float* lam_d;
    const float* ys_s;  float* ys_d;
    const int*   sel_s; int*   sel_d;
    const int*   pid_s; int*   pid_d;   // pid_s NULL: source is in caller order
    F9Planes     fe_s, fe_d;             // elastic F (fe_s.a NULL: not moved)
    const int*   keys;
    const int*   ranks;
    const int*   offsets;    // cell offsets
    int n;
};

// src order -> sorted order: dst = cell_offsets[keys[p]] + ranks[p]
__global__ void k_sort_scatter(const PermuteArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int d = __ldg(a.offsets + __ldg(a.keys + p)) + __ldg(a.ranks + p);
    a.dst.x[d] = __ldg(a.src.x + p);
    a.dst.v[d] = __ldg(a.src.v + p);
    f9_store(a.dst.C, d, f9_load(a.src.C, p));
    f9_store(a.dst.F, d, f9_load(a.src.F, p));
    a.vol_d[d] = __ldg(a.vol_s + p);
    a.mu_d[d] = __ldg(a.mu_s + p);
    a.lam_d[d] = __ldg(a.lam_s + p);
    a.ys_d[d] = __ldg(a.ys_s + p);
    a.sel_d[d] = a.sel_s ? __ldg(a.sel_s + p) : 0;
    a.pid_d[d] = a.pid_s ? __ldg(a.pid_s + p) : p;
    if (a.fe_s.a) f9_store(a.fe_d, d, f9_load(a.fe_s, p));
}

struct UnsortArgs {
    ParticleArrays src, dst;      // sorted -> caller order
    F9Planes Fe_s, Fe_d;          // elastic F of the last substep
    const float* mu_s;  float* mu_d;
    const float* lam_s; float* lam_d;
    const float* ys_s;  float* ys_d;
    const int*   pid;
    int n;
};

__global__ void k_unsort(const UnsortArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int d = __ldg(a.pid + p);
    a.dst.x[d] = __ldg(a.src.x + p);
    a.dst.v[d] = __ldg(a.src.v + p);
    f9_store(a.dst.C, d, f9_load(a.src.C, p));
    f9_store(a.dst.F, d, f9_load(a.src.F, p));
    f9_store(a.Fe_d, d, f9_load(a.Fe_s, p));
    a.mu_d[d] = __ldg(a.mu_s + p);
    a.lam_d[d] = __ldg(a.lam_s + p);
    a.ys_d[d] = __ldg(a.ys_s + p);
}

// -------------------------------------------------------------------------
// sorted path, default P2G: warp-aggregated reductions
// -------------------------------------------------------------------------
// Lanes whose particles share an instance and base cell form a contiguous
// segment of the warp (cell-sorted order); for each of the 27 stencil nodes
// the segment's contributions are summed with shuffles and only the segment
// head issues the 16-byte reduction to the grid.
//
// Same-cell runs are split every seg_cap = 2^ROUNDS lanes, so a segment sums
// in at most ROUNDS shuffle rounds; the rounds a run cap never needs are not
// compiled in (smaller code for the instruction cache).
// The warp-aggregated scatter of one prepared particle per lane (all 32
// lanes of the warp take part; lanes with valid == false contribute zeros and
// never write). c: the lane's instance constants for this substep.
template <int ROUNDS>
__device__ __forceinline__ void warpagg_scatter(bool valid, int inst, const P2GParticle& q, const StepConsts& c,
                                                float4* grid, unsigned char* flags) {
    constexpr int seg_cap = 1 << ROUNDS;
    const int lane = threadIdx.x & 31;
    // a segment is a run of lanes with the same validity, instance and base
    // cell; lanes without a particle contribute zeros and never write
    const int b0 = valid ? q.st.b[0] : lane, b1 = valid ? q.st.b[1] : 0, b2 = valid ? q.st.b[2] : 0;
    const int u0 = __shfl_up_sync(0xffffffffu, b0, 1), u1 = __shfl_up_sync(0xffffffffu, b1, 1),
              u2 = __shfl_up_sync(0xffffffffu, b2, 1);
    const int uv = __shfl_up_sync(0xffffffffu, (int)valid, 1);
    const int ui = __shfl_up_sync(0xffffffffu, inst, 1);
    const bool run_head = lane == 0 || uv != (int)valid || ui != inst || u0 != b0 || u1 != b1 || u2 != b2;
    // runs longer than seg_cap (a power of two) get another head every
    // seg_cap lanes: fewer shuffle rounds below, more reductions into the grid
    const unsigned run_heads = __ballot_sync(0xffffffffu, run_head);
    const int run_start = 31 - __clz(run_heads & (0xffffffffu >> (31 - lane)));
    const bool head = run_head || ((lane - run_start) & (seg_cap - 1)) == 0;
    const unsigned heads = __ballot_sync(0xffffffffu, head);
    const unsigned above = lane == 31 ? 0u : (heads & (0xffffffffu << (lane + 1)));
    const int end = above ? (__ffs(above) - 2) : 31;
    const int seglen = head ? end - lane + 1 : 1;
    const int maxlen = __reduce_max_sync(0xffffffffu, seglen);
    const int G = c.G;
    const bool in_grid = valid && stencil_in_grid(q.st, G);
    if (valid && !in_grid) atomicOr(c.status, EMPM_STATUS_OUT_OF_BAND);
    P2GPre pre;
    if (valid) {
        pre = p2g_pre(q, c.dx, c.inv_dx, c.step->dt);
    } else {
        pre.st = make_stencil(v3(0.f, 0.f, 0.f), 1.f);
        pre.m = 0.f;
        pre.a = v3(0.f, 0.f, 0.f);
        pre.B = m3_zero();
        pre.S = m3_zero();
    }
    // The reduction rounds are unrolled: each is skipped by a warp-uniform
    // branch once 2^r >= maxlen, and the per-lane "partner inside my segment"
    // tests are formed once instead of per node. The node address is formed
    // only in the head lanes (keeping precomputed per-axis address terms live
    // across the 27 nodes measured slower here).
    unsigned take = 0;
#pragma unroll
    for (int r = 0; r < ROUNDS; ++r) take |= lane + (1 << r) <= end ? 1u << r : 0u;
    p2g_emit(pre, [&](int i, int j, int k, float4 v) {
#pragma unroll
        for (int r = 0; r < ROUNDS; ++r) {
            const int d = 1 << r;
            if (d < maxlen) {
                const float tx = __shfl_down_sync(0xffffffffu, v.x, d);
                const float ty = __shfl_down_sync(0xffffffffu, v.y, d);
                const float tz = __shfl_down_sync(0xffffffffu, v.z, d);
                const float tw = __shfl_down_sync(0xffffffffu, v.w, d);
                if (take & (1u << r)) { v.x += tx; v.y += ty; v.z += tz; v.w += tw; }
            }
        }
        if (head && valid && (in_grid || node_in_grid(q.st.b, i, j, k, G)))
            red_add_v4(grid + gaddr(c, q.st.b[0] + i, q.st.b[1] + j, q.st.b[2] + k), v);
    });
    if (head && valid) mark_stencil_blocks(flags, q.st, c);
}

// Same-cell runs are split every seg_cap = 2^ROUNDS lanes, so a segment sums
// in at most ROUNDS shuffle rounds; the rounds a run cap never needs are not
// compiled in (smaller code for the instruction cache).
template <int ROUNDS, int MAT = -1>
__global__ void __launch_bounds__(256, EMPM_P2G_MIN_CTAS) k_p2g_warpagg(ParticleArrays P, MaterialArrays M, F9Planes Fe, Launch L,
                                                     float4* grid, unsigned char* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int inst = p < L.n_total ? find_instance_particle(L, p) : 0;
    const StepConsts c = consts_of(L, inst);
    P2GParticle q;
    bool valid = false;
    if (p < L.n_total) valid = prepare_particle<MAT>(P, M, Fe, c, p, q);
    warpagg_scatter<ROUNDS>(valid, inst, q, c, grid, flags);
}

// -------------------------------------------------------------------------
// sorted path, fused: the G2P of substep s-1 and the stress + P2G of substep s
// in one pass over the particles
// -------------------------------------------------------------------------
// Between two such kernels a particle's persistent state is its position and
// its elastic F (plus the material scalars); its velocity, affine matrix and
// trial F are consumed by the P2G in the same thread, so they are not written
// back. Position and elastic F are updated in place: a thread reads and writes
// only its own particle. The grid velocities of substep s-1 (vel) are read,
// the accumulator of substep s (mom, cleared by the grid update of s-1) is
// written: the two are separate buffers. A run of fused substeps starts with
// the separate stress + P2G and ends with the separate G2P, which writes the
// full state. Held instances (step-table hold) must stay held once held within
// the run: when a particle's instance becomes held at substep s, its state
// after the G2P of s-1 is written in full, then left alone.
// MINB: resident CTAs per SM asked of the compiler. Launches over few
// particles (CTAs of 64 threads, a few warps per SM) use MINB = 1: registers
// are then not what limits them, so the kernel keeps all its state in
// registers and gathers with the unrolled loop (C1, 20k particles: 25.3 ->
// 23.7 us per substep).
template <int ROUNDS, int MAT = -1, int MINB = EMPM_FUSED_MIN_CTAS>
__global__ void __launch_bounds__(256, MINB) k_g2p2g(ParticleArrays P, MaterialArrays M, F9Planes Fe,
                                                                  Launch L, int g2p_table, const float4* vel,
                                                                  float4* mom, unsigned char* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int inst = p < L.n_total ? find_instance_particle(L, p) : 0;
    const StepConsts c = consts_of(L, inst);   // substep s: stress + P2G
    P2GParticle q;
    bool valid = false;
    // which lanes run the G2P of substep s-1 (simulated, not held)
    bool g_on = false;
    float4 xm = make_float4(0.f, 0.f, 0.f, 0.f);
    if (p < L.n_total && !(M.sel && __ldg(M.sel + p) != 0)) {
        g_on = !L.steps[(size_t)g2p_table * L.n_inst + inst].hold;
        if (g_on) xm = __ldg(P.x + p);
    }
#if EMPM_FUSED_WARP_TILE
    // the warp's stencil nodes into shared memory (all lanes take part)
    __shared__ float4 s_tile[256 / 32][EMPM_WARP_TILE_NODES];
    const int wlane = threadIdx.x & 31;
    float4* wtile = s_tile[threadIdx.x >> 5];
    int gb[3] = {0, 0, 0};
    if (g_on) {
        gb[0] = base_node(xm.x, c.inv_dx);
        gb[1] = base_node(xm.y, c.inv_dx);
        gb[2] = base_node(xm.z, c.inv_dx);
    }
    const unsigned g_lanes = __ballot_sync(0xffffffffu, g_on);
    int box_o[3], box_e[3];
    bool tiled = false;
    if (g_lanes) {
        int hi[3];
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3) {
            box_o[a3] = __reduce_min_sync(0xffffffffu, g_on ? gb[a3] : INT_MAX);
            hi[a3] = __reduce_max_sync(0xffffffffu, g_on ? gb[a3] : INT_MIN);
            box_e[a3] = hi[a3] - box_o[a3] + 3;
        }
        const int imin = __reduce_min_sync(0xffffffffu, g_on ? inst : INT_MAX);
        const int imax = __reduce_max_sync(0xffffffffu, g_on ? inst : INT_MIN);
        const int leader = __ffs(g_lanes) - 1;
        const int Gw = __shfl_sync(0xffffffffu, c.G, leader);
        const int NBw = __shfl_sync(0xffffffffu, c.NB, leader);
        const int boffw = __shfl_sync(0xffffffffu, c.boff, leader);
        const int count = box_e[0] * box_e[1] * box_e[2];
        tiled = imin == imax && count <= EMPM_WARP_TILE_NODES && box_o[0] >= 0 && box_o[1] >= 0 &&
                box_o[2] >= 0 && hi[0] + 2 < Gw && hi[1] + 2 < Gw && hi[2] + 2 < Gw;
        if (tiled) {
            const int e12 = box_e[1] * box_e[2];
            for (int t = wlane; t < count; t += 32) {
                const int ti = t / e12, tr = t - ti * e12;
                const int tj = tr / box_e[2], tk = tr - tj * box_e[2];
                const int gi = box_o[0] + ti, gj = box_o[1] + tj, gk = box_o[2] + tk;
                const long long addr = ((long long)(boffw + block_of(gi, gj, gk, NBw)) << 6) | ((gi & 3) << 4) |
                                       ((gj & 3) << 2) | (gk & 3);
                wtile[t] = __ldg(vel + addr);
            }
        }
        __syncwarp();
    }
#endif
    if (g_on) {
        {
            const EmpmStep& sg = L.steps[(size_t)g2p_table * L.n_inst + inst];   // substep s-1: G2P
            const float dt = sg.dt;
            const V3 x = v3(xm.x, xm.y, xm.z);
            const Stencil st = make_stencil(x, c.inv_dx);
            const bool in_grid = stencil_in_grid(st, c.G);
#if EMPM_FUSED_WARP_TILE
            G2POut o;
            if (tiled) {
                const WarpTileFetch fetch{wtile, box_o[0], box_o[1], box_o[2], box_e[1], box_e[2]};
                o = g2p_gather_rt(st, c.inv_dx, fetch.bind(st, in_grid));
            } else {
                const GlobalFetch fetch{vel, &c};
                o = g2p_gather_rt(st, c.inv_dx, fetch.bind(st, in_grid));
            }
#else
            GlobalFetch fetch{vel, &c};
            G2POut o;
            if (EMPM_FUSED_G2P_LOOP && MINB > 1) o = g2p_gather_rt(st, c.inv_dx, fetch.bind(st, in_grid));
            else o = g2p_gather(st, c.inv_dx, fetch.bind(st, in_grid));
#endif
            const float dx = 1.f / c.inv_dx;   // as g2p_particle computes it
            const float lo = dx * 2.f, hi = c.grid_lim - dx * 2.f;
            V3 nx = x + dt * o.v;
            nx = v3(fminf(fmaxf(nx.x, lo), hi), fminf(fmaxf(nx.y, lo), hi), fminf(fmaxf(nx.z, lo), hi));
            const M3 Fn = (m3_identity() + dt * o.gradv) * f9_load(Fe, p);
            P.x[p] = make_float4(nx.x, nx.y, nx.z, xm.w);
            unsigned bad = 0;
            if (!finite3(o.v) || !finite3(nx) || !isfinite(Fn.m[0] + Fn.m[4] + Fn.m[8])) bad |= EMPM_STATUS_NAN;
            if (fmaxf(fmaxf(fabsf(o.v.x), fabsf(o.v.y)), fabsf(o.v.z)) * dt > dx) bad |= EMPM_STATUS_CFL;
            if (!in_grid) bad |= EMPM_STATUS_OUT_OF_BAND;
            if (bad) atomicOr(c.status, bad);
            const EmpmStep& sp = *c.step;
            if (sp.hold) {
                // held from substep s on: keep the state after this G2P
                P.v[p] = make_float4(o.v.x, o.v.y, o.v.z, 0.f);
                f9_store(P.C, p, o.C);
                f9_store(P.F, p, Fn);
            } else {
                V3 v = o.v;
                if (sp.n_modifiers > 0) {
                    const int mi = M.pid ? __ldg(M.pid + p) : p;
                    apply_modifiers(sp, mi, nx, xm.w, v);
                }
                float mu = __ldg(M.mu + p), lam = __ldg(M.lam + p), ys = __ldg(M.ys + p);
                const ConstitutiveOut co = constitutive<MAT>(Fn, mu, lam, ys, sp.dt, *c.ms);
                f9_store(Fe, p, co.F);
                if (co.mat_changed) { M.mu[p] = mu; M.lam[p] = lam; M.ys[p] = ys; }
                q.st = make_stencil(nx, c.inv_dx);
                q.wm_scale = xm.w;
                q.v = v;
                q.Cd = damp_affine(o.C, c.rpic);
                q.Sv = (-__ldg(M.vol + p)) * co.tau;
                valid = true;
            }
        }
    }
    warpagg_scatter<ROUNDS>(valid, inst, q, c, mom, flags);
}

// Stored segments of a differentiable rollout (cell-sorted): the G2P of
// substep k-1 and the stress + P2G of substep k in one pass, writing what the
// reverse pass reads instead of handing state from kernel to kernel: the full
// state before substep k (its velocity after the modifiers, as the P2G of the
// separate kernels leaves it), the mu / lam / yield snapshot before substep k
// and the elastic F of substep k. Segments hold no instances (step-table hold)
// and their particles stay in one order, so every thread writes only its own
// particle of the substep-k arrays.
struct SegmentStoreArgs {
    ParticleArrays prev;     // state before substep k-1 (x read)
    F9Planes       fe_prev;  // elastic F of substep k-1
    ParticleArrays cur;      // out: state before substep k
    F9Planes       fe_cur;   // out: elastic F of substep k
    float*         snap;     // out: mu | lam | yield before substep k, stride np
    long long      np;
};

template <int ROUNDS, int MAT = -1, int MINB = EMPM_FUSED_MIN_CTAS>
__global__ void __launch_bounds__(256, MINB) k_g2p2g_store(MaterialArrays M, Launch L, int g2p_table,
                                                                        const float4* vel, float4* mom,
                                                                        unsigned char* flags, SegmentStoreArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int inst = p < L.n_total ? find_instance_particle(L, p) : 0;
    const StepConsts c = consts_of(L, inst);   // substep k: stress + P2G
    P2GParticle q;
    bool valid = false;
    if (p < L.n_total) {
        const float mu0 = __ldg(M.mu + p), lam0 = __ldg(M.lam + p), ys0 = __ldg(M.ys + p);
        a.snap[p] = mu0;
        a.snap[a.np + p] = lam0;
        a.snap[2 * a.np + p] = ys0;
        const float4 xm = __ldg(a.prev.x + p);
        if (M.sel && __ldg(M.sel + p) != 0) {
            // unsimulated: the G2P writes the reference's constant state, no P2G
            a.cur.x[p] = make_float4(0.f, 0.f, 0.f, xm.w);
            a.cur.v[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            f9_store(a.cur.C, p, m3_zero());
            f9_store(a.cur.F, p, m3_identity());
        } else {
            const float dt = L.steps[(size_t)g2p_table * L.n_inst + inst].dt;   // substep k-1
            const V3 x = v3(xm.x, xm.y, xm.z);
            const Stencil st = make_stencil(x, c.inv_dx);
            const bool in_grid = stencil_in_grid(st, c.G);
            const GlobalFetch fetch{vel, &c};
            G2POut o;
            if (MINB > 1) o = g2p_gather_rt(st, c.inv_dx, fetch.bind(st, in_grid));
            else o = g2p_gather(st, c.inv_dx, fetch.bind(st, in_grid));
            const float dx = 1.f / c.inv_dx;   // as g2p_particle computes it
            const float lo = dx * 2.f, hi = c.grid_lim - dx * 2.f;
            V3 nx = x + dt * o.v;
            nx = v3(fminf(fmaxf(nx.x, lo), hi), fminf(fmaxf(nx.y, lo), hi), fminf(fmaxf(nx.z, lo), hi));
            const M3 Fn = (m3_identity() + dt * o.gradv) * f9_load(a.fe_prev, p);
            unsigned bad = 0;
            if (!finite3(o.v) || !finite3(nx) || !isfinite(Fn.m[0] + Fn.m[4] + Fn.m[8])) bad |= EMPM_STATUS_NAN;
            if (fmaxf(fmaxf(fabsf(o.v.x), fabsf(o.v.y)), fabsf(o.v.z)) * dt > dx) bad |= EMPM_STATUS_CFL;
            if (!in_grid) bad |= EMPM_STATUS_OUT_OF_BAND;
            if (bad) atomicOr(c.status, bad);
            const EmpmStep& sp = *c.step;
            V3 v = o.v;
            if (sp.n_modifiers > 0) {
                const int mi = M.pid ? __ldg(M.pid + p) : p;
                apply_modifiers(sp, mi, nx, xm.w, v);
            }
            a.cur.x[p] = make_float4(nx.x, nx.y, nx.z, xm.w);
            a.cur.v[p] = make_float4(v.x, v.y, v.z, 0.f);
            f9_store(a.cur.C, p, o.C);
            f9_store(a.cur.F, p, Fn);
            float mu = mu0, lam = lam0, ys = ys0;
            const ConstitutiveOut co = constitutive<MAT>(Fn, mu, lam, ys, sp.dt, *c.ms);
            f9_store(a.fe_cur, p, co.F);
            if (co.mat_changed) { M.mu[p] = mu; M.lam[p] = lam; M.ys[p] = ys; }
            q.st = make_stencil(nx, c.inv_dx);
            q.wm_scale = xm.w;
            q.v = v;
            q.Cd = damp_affine(o.C, c.rpic);
            q.Sv = (-__ldg(M.vol + p)) * co.tau;
            valid = true;
        }
    }
    warpagg_scatter<ROUNDS>(valid, inst, q, c, mom, flags);
}

// k_g2p2g_store at the default run cap (4) for a launch whose instances all
// use material (plasticine 5 and jelly 0 have kernels of their own, -1 any);
// few: a launch over few particles (the MINB = 1 variant, as for k_g2p2g).
// Returns false for other run caps (the caller runs the separate kernels).
static inline bool launch_g2p2g_store(int grid_ctas, int threads, cudaStream_t s, const MaterialArrays& M,
                                      const Launch& L, int g2p_table, const float4* vel, float4* mom,
                                      unsigned char* flags, const SegmentStoreArgs& a, int seg_cap, int material,
                                      bool few = false) {
    if (seg_cap != 4) return false;
    if (few && material == 5) k_g2p2g_store<2, 5, 1><<<grid_ctas, threads, 0, s>>>(M, L, g2p_table, vel, mom, flags, a);
    else if (few && material == 0) k_g2p2g_store<2, 0, 1><<<grid_ctas, threads, 0, s>>>(M, L, g2p_table, vel, mom, flags, a);
    else if (material == 5) k_g2p2g_store<2, 5><<<grid_ctas, threads, 0, s>>>(M, L, g2p_table, vel, mom, flags, a);
    else if (material == 0) k_g2p2g_store<2, 0><<<grid_ctas, threads, 0, s>>>(M, L, g2p_table, vel, mom, flags, a);
    else k_g2p2g_store<2, -1><<<grid_ctas, threads, 0, s>>>(M, L, g2p_table, vel, mom, flags, a);
    return true;
}

static inline void launch_g2p2g(int grid_ctas, int threads, cudaStream_t s, const ParticleArrays& P,
                                const MaterialArrays& M, const F9Planes& Fe, const Launch& L, int g2p_table,
                                const float4* vel, float4* mom, unsigned char* flags, int seg_cap,
                                int material = -1, bool few = false) {
    // few: a launch over few particles (CTAs of 64 threads) takes the MINB = 1
    // variant where one is compiled (plasticine and jelly at run cap 4)
#define EMPM_G2P2G(R, MAT) k_g2p2g<R, MAT><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, g2p_table, vel, mom, flags)
    if (few && material == 5 && seg_cap == 4) {
        k_g2p2g<2, 5, 1><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, g2p_table, vel, mom, flags);
        return;
    }
    if (few && material == 0 && seg_cap == 4) {
        k_g2p2g<2, 0, 1><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, g2p_table, vel, mom, flags);
        return;
    }
    if (material == 5 && seg_cap == 4) { EMPM_G2P2G(2, 5); return; }
    if (material == 5 && seg_cap == 8) { EMPM_G2P2G(3, 5); return; }
    if (material == 0 && seg_cap == 4) { EMPM_G2P2G(2, 0); return; }
    if (material == 0 && seg_cap == 8) { EMPM_G2P2G(3, 0); return; }
    switch (seg_cap) {
        case 1: EMPM_G2P2G(0, -1); break;
        case 2: EMPM_G2P2G(1, -1); break;
        case 4: EMPM_G2P2G(2, -1); break;
        case 8: EMPM_G2P2G(3, -1); break;
        case 16: EMPM_G2P2G(4, -1); break;
        default: EMPM_G2P2G(5, -1); break;
    }
#undef EMPM_G2P2G
}

// k_p2g_warpagg for a run cap seg_cap (a power of two in 1..32). material:
// the material id every instance of the launch uses, or -1 when they differ;
// plasticine (5) and jelly (0) at run caps 4 and 8 have kernels compiled for
// that material alone.
static inline void launch_p2g_warpagg(int grid_ctas, int threads, cudaStream_t s, const ParticleArrays& P,
                                      const MaterialArrays& M, const F9Planes& Fe, const Launch& L, float4* mom,
                                      unsigned char* flags, int seg_cap, int material = -1) {
    if (material == 5 && seg_cap == 4) { k_p2g_warpagg<2, 5><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); return; }
    if (material == 5 && seg_cap == 8) { k_p2g_warpagg<3, 5><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); return; }
    if (material == 0 && seg_cap == 4) { k_p2g_warpagg<2, 0><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); return; }
    if (material == 0 && seg_cap == 8) { k_p2g_warpagg<3, 0><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); return; }
    switch (seg_cap) {
        case 1: k_p2g_warpagg<0><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
        case 2: k_p2g_warpagg<1><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
        case 4: k_p2g_warpagg<2><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
        case 8: k_p2g_warpagg<3><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
        case 16: k_p2g_warpagg<4><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
        default: k_p2g_warpagg<5><<<grid_ctas, threads, 0, s>>>(P, M, Fe, L, mom, flags); break;
    }
}

// -------------------------------------------------------------------------
// sorted path, optional: shared-memory node tiles over chunks of particles
// -------------------------------------------------------------------------
constexpr int TILE_THREADS = 256;     // = chunk size

struct ChunkList {
    const int2* chunks;    // (first sorted index, count); never spans two 4^3 blocks
    const int*  nchunks;   // device count
};

__device__ __forceinline__ float sel3(const float (&a)[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }

// one node contribution with runtime stencil offsets (no local-memory indexing)
__device__ __forceinline__ float4 p2g_node_dyn(const P2GPre& p, int i, int j, int k) {
    const Stencil& st = p.st;
    const float wx = sel3(st.w[0], i), wy = sel3(st.w[1], j), wz = sel3(st.w[2], k);
    const float dwx = sel3(st.dw[0], i), dwy = sel3(st.dw[1], j), dwz = sel3(st.dw[2], k);
    const V3 a = p.a + (float)i * col(p.B, 0) + (float)j * col(p.B, 1) + (float)k * col(p.B, 2);
    const float wm = (wx * wy * wz) * p.m;
    const V3 c = wm * a + (dwx * wy * wz) * col(p.S, 0) + (wx * dwy * wz) * col(p.S, 1) + (wx * wy * dwz) * col(p.S, 2);
    return make_float4(c.x, c.y, c.z, wm);
}

struct TileBox {
    int o[3];   // origin node
    int e[3];   // extent in nodes
    int count;  // e0 * e1 * e2
};

// bounding box of the chunk's stencils (base .. base + 2) in shared memory
__device__ __forceinline__ TileBox chunk_box(bool active, const int (&b)[3], int* s_min, int* s_max) {
    if (threadIdx.x < 3) { s_min[threadIdx.x] = INT_MAX; s_max[threadIdx.x] = INT_MIN; }
    __syncthreads();
    int mn[3], mx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) { mn[a] = active ? b[a] : INT_MAX; mx[a] = active ? b[a] : INT_MIN; }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], d));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], d));
        }
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int a = 0; a < 3; ++a) { atomicMin(s_min + a, mn[a]); atomicMax(s_max + a, mx[a]); }
    __syncthreads();
    TileBox tb;
    tb.count = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        tb.o[a] = s_min[a];
        tb.e[a] = s_max[a] - s_min[a] + 3;
        tb.count *= tb.e[a];
    }
    if (s_min[0] == INT_MAX) tb.count = 0;
    return tb;
}

struct TiledArgs {
    ParticleArrays P;
    MaterialArrays M;
    F9Planes Fe;
    Launch L;
    ChunkList cl;
    float4* grid;             // P2G: accumulation; G2P: node velocities
    unsigned char* flags;     // P2G marks touched blocks
    ParticleArrays out;       // G2P output
    int tile_cap;             // nodes in the shared tile
};

__global__ void __launch_bounds__(TILE_THREADS, 2) k_p2g_tiled(const TiledArgs a) {
    extern __shared__ float4 tile[];
    __shared__ int s_min[3], s_max[3];
    const int nch = *a.cl.nchunks;
    for (int ci = blockIdx.x; ci < nch; ci += gridDim.x) {
        const int2 ch = a.cl.chunks[ci];
        const StepConsts c = consts_of(a.L, find_instance_particle(a.L, ch.x));
        const float dt = c.step->dt;
        const int p = ch.x + (int)threadIdx.x;
        bool active = threadIdx.x < (unsigned)ch.y;
        int base[3] = {0, 0, 0};
        if (active) {
            const float4 xm = __ldg(a.P.x + p);
            base[0] = base_node(xm.x, c.inv_dx);
            base[1] = base_node(xm.y, c.inv_dx);
            base[2] = base_node(xm.z, c.inv_dx);
            if (a.M.sel && __ldg(a.M.sel + p) != 0) active = false;
        }
        const TileBox tb = chunk_box(active, base, s_min, s_max);
        const bool use_tile = tb.count > 0 && tb.count <= a.tile_cap;
        if (use_tile)
            for (int t = threadIdx.x; t < tb.count; t += TILE_THREADS) tile[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        if (active) {
            P2GParticle q;
            if (prepare_particle(a.P, a.M, a.Fe, c, p, q)) {
                if (use_tile) {
                    const P2GPre pre = p2g_pre(q, c.dx, c.inv_dx, dt);
                    // stagger the 27 stencil offsets across lanes so particles of the
                    // same cell do not hit the same shared-memory node together
                    int s = (int)(threadIdx.x % 27u);
                    int i = s / 9, j = (s / 3) % 3, k = s % 3;
                    const int li0 = q.st.b[0] - tb.o[0], lj0 = q.st.b[1] - tb.o[1], lk0 = q.st.b[2] - tb.o[2];
                    for (int it = 0; it < 27; ++it) {
                        const float4 v = p2g_node_dyn(pre, i, j, k);
                        float* dst = reinterpret_cast<float*>(tile + ((li0 + i) * tb.e[1] + (lj0 + j)) * tb.e[2] + (lk0 + k));
                        atomicAdd(dst + 0, v.x);
                        atomicAdd(dst + 1, v.y);
                        atomicAdd(dst + 2, v.z);
                        atomicAdd(dst + 3, v.w);
                        if (++k == 3) { k = 0; if (++j == 3) { j = 0; if (++i == 3) i = 0; } }
                    }
                } else {
                    scatter_global(q, c, a.grid, a.flags);
                }
            }
        }
        __syncthreads();
        if (use_tile) {
            const int e12 = tb.e[1] * tb.e[2];
            for (int t = threadIdx.x; t < tb.count; t += TILE_THREADS) {
                const float4 v = tile[t];
                if (v.w == 0.f && v.x == 0.f && v.y == 0.f && v.z == 0.f) continue;
                const int gi = tb.o[0] + t / e12, gj = tb.o[1] + (t / tb.e[2]) % tb.e[1], gk = tb.o[2] + t % tb.e[2];
                if (gi < 0 || gj < 0 || gk < 0 || gi >= c.G || gj >= c.G || gk >= c.G) {
                    atomicOr(c.status, EMPM_STATUS_OUT_OF_BAND);
                    continue;
                }
                red_add_v4(a.grid + gaddr(c, gi, gj, gk), v);
            }
            // mark the 4^3 blocks the tile overlaps
            const int lo[3] = {max(tb.o[0], 0) >> 2, max(tb.o[1], 0) >> 2, max(tb.o[2], 0) >> 2};
            const int hi[3] = {min(tb.o[0] + tb.e[0] - 1, c.G - 1) >> 2, min(tb.o[1] + tb.e[1] - 1, c.G - 1) >> 2,
                               min(tb.o[2] + tb.e[2] - 1, c.G - 1) >> 2};
            const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
            const int nmark = (n0 > 0 && n1 > 0 && n2 > 0) ? n0 * n1 * n2 : 0;
            for (int t = threadIdx.x; t < nmark; t += TILE_THREADS) {
                const int bi = lo[0] + t / (n1 * n2), bj = lo[1] + (t / n2) % n1, bk = lo[2] + t % n2;
                a.flags[c.boff + (bi * c.NB + bj) * c.NB + bk] = 1;
            }
        }
        __syncthreads();
    }
}

// Node velocities from the chunk's shared-memory tile (the stencil lies in it).
struct TileFetch {
    const float4* tile;
    int o0, o1, o2, e1, e2;
    struct Bound {
        const float4* tile;
        int x[3], y[3], z[3];   // tile index of node (i, j, k) = x[i] + y[j] + z[k]
        __device__ __forceinline__ V3 operator()(int i, int j, int k) const {
            const float4 g = tile[x[i] + y[j] + z[k]];
            return v3(g.x, g.y, g.z);
        }
    };
    __device__ __forceinline__ Bound bind(const Stencil& st, bool) const {
        Bound b;
        b.tile = tile;
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            b.x[o] = (st.b[0] + o - o0) * e1 * e2;
            b.y[o] = (st.b[1] + o - o1) * e2;
            b.z[o] = st.b[2] + o - o2;
        }
        return b;
    }
};

__global__ void __launch_bounds__(TILE_THREADS, 2) k_g2p_tiled(const TiledArgs a) {
    extern __shared__ float4 tile[];
    __shared__ int s_min[3], s_max[3];
    const int nch = *a.cl.nchunks;
    for (int ci = blockIdx.x; ci < nch; ci += gridDim.x) {
        const int2 ch = a.cl.chunks[ci];
        const StepConsts c = consts_of(a.L, find_instance_particle(a.L, ch.x));
        const int p = ch.x + (int)threadIdx.x;
        const bool active = threadIdx.x < (unsigned)ch.y;
        bool stenciled = active;
        int base[3] = {0, 0, 0};
        if (active) {
            if (a.M.sel && __ldg(a.M.sel + p) != 0) stenciled = false;
            const float4 xm = __ldg(a.P.x + p);
            base[0] = base_node(xm.x, c.inv_dx);
            base[1] = base_node(xm.y, c.inv_dx);
            base[2] = base_node(xm.z, c.inv_dx);
        }
        const TileBox tb = chunk_box(stenciled, base, s_min, s_max);
        const bool use_tile = tb.count > 0 && tb.count <= a.tile_cap && tb.o[0] >= 0 && tb.o[1] >= 0 && tb.o[2] >= 0 &&
                              tb.o[0] + tb.e[0] <= c.G && tb.o[1] + tb.e[1] <= c.G && tb.o[2] + tb.e[2] <= c.G;
        if (use_tile) {
            const int e12 = tb.e[1] * tb.e[2];
            for (int t = threadIdx.x; t < tb.count; t += TILE_THREADS) {
                const int gi = tb.o[0] + t / e12, gj = tb.o[1] + (t / tb.e[2]) % tb.e[1], gk = tb.o[2] + t % tb.e[2];
                tile[t] = __ldg(a.grid + gaddr(c, gi, gj, gk));
            }
        }
        __syncthreads();
        if (active) {
            if (use_tile) {
                TileFetch f{tile, tb.o[0], tb.o[1], tb.o[2], tb.e[1], tb.e[2]};
                g2p_particle(a.P, a.Fe, a.M, a.out, c, p, f);
            } else {
                GlobalFetch f{a.grid, &c};
                g2p_particle(a.P, a.Fe, a.M, a.out, c, p, f);
            }
        }
        __syncthreads();
    }
}

}  // namespace empm
