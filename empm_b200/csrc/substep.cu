// substep.cu — single-instance kernels and the C ABI of libempm_b200.so.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdarg.h>
#include "../../include/empm_b200.h"
#include "substep.cuh"
#include "ctx.hpp"

using namespace empm;

namespace {

struct P2GArgs {
    const float4* x;
    float4*       v;        // old state's v (modifiers write back in place)
    F9Planes      C;
    F9Planes      F;        // F_trial
    F9Planes      Fe;       // receives the elastic F
    const float*  vol;
    float*        mu;
    float*        lam;
    float*        ys;
    const int*    sel;
    float4*       grid;     // momentum + mass accumulation
    unsigned*     status;
    int           n;
    int           G;
    float         dx, inv_dx;
    float         rpic;
    MaterialScalars ms;
    const EmpmStep* step;
};

// Fused return map + stress + APIC P2G scatter, one particle per thread,
// 16-byte vector reductions into the node float4 (px, py, pz, m).
__global__ void __launch_bounds__(128) k_stress_p2g(const P2GArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    if (a.sel && __ldg(a.sel + p) != 0) return;
    const EmpmStep& st = *a.step;
    const float4 xm = __ldg(a.x + p);
    const float4 vv = __ldg(a.v + p);
    const V3 x = v3(xm.x, xm.y, xm.z);
    V3 v = v3(vv.x, vv.y, vv.z);
    const float mass = xm.w;
    if (st.n_modifiers > 0 && apply_modifiers(st, p, x, mass, v))
        a.v[p] = make_float4(v.x, v.y, v.z, vv.w);

    float mu = __ldg(a.mu + p), lam = __ldg(a.lam + p), ys = __ldg(a.ys + p);
    const ConstitutiveOut co = constitutive(f9_load(a.F, p), mu, lam, ys, st.dt, a.ms);
    f9_store(a.Fe, p, co.F);
    if (co.mat_changed) { a.mu[p] = mu; a.lam[p] = lam; a.ys[p] = ys; }

    P2GParticle q;
    q.st = make_stencil(x, a.inv_dx);
    q.wm_scale = mass;
    q.v = v;
    q.Cd = damp_affine(f9_load(a.C, p), a.rpic);
    q.Sv = (-__ldg(a.vol + p)) * co.tau;
    const bool in_grid = stencil_in_grid(q.st, a.G);
    if (!in_grid) atomicOr(a.status, EMPM_STATUS_OUT_OF_BAND);
    const int G = a.G;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int ix = q.st.b[0] + i, iy = q.st.b[1] + j, iz = q.st.b[2] + k;
                if (!in_grid && (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G)) continue;
                const float4 c = p2g_node(q, i, j, k, a.dx, a.inv_dx, st.dt);
                red_add_v4(a.grid + ((long long)ix * G + iy) * G + iz, c);
            }
}

struct GridArgs {
    float4*  mom;    // read, then zeroed for the next substep
    float4*  vel;    // node velocity after BCs (w = node mass)
    int      G;
    float    dx;
    V3       g;
    float    damping;
    const EmpmStep* step;
};

__global__ void __launch_bounds__(256) k_grid_update(const GridArgs a) {
    const long long total = (long long)a.G * a.G * a.G;
    const EmpmStep& st = *a.step;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const float4 m = a.mom[idx];
        a.mom[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
        V3 v = grid_velocity(m, st.dt, a.g, a.damping);
        if (st.n_colliders > 0) {
            const int k = (int)(idx % a.G);
            const int j = (int)((idx / a.G) % a.G);
            const int i = (int)(idx / ((long long)a.G * a.G));
            apply_colliders(st, i, j, k, a.G, a.dx, idx, v);
        }
        a.vel[idx] = make_float4(v.x, v.y, v.z, m.w);
    }
}

struct G2PArgs {
    const float4* x;
    F9Planes      Fe;
    const int*    sel;
    const float4* vel;
    float4*       x_out;
    float4*       v_out;
    F9Planes      C_out;
    F9Planes      F_out;
    unsigned*     status;
    int           n;
    int           G;
    float         inv_dx;
    float         grid_lim;
    const EmpmStep* step;
};

__global__ void __launch_bounds__(128) k_g2p(const G2PArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    if (a.sel && __ldg(a.sel + p) != 0) {
        // the reference leaves unsimulated particles at partial_clone's values
        __stcs(a.x_out + p, make_float4(0.f, 0.f, 0.f, __ldg(a.x + p).w));
        __stcs(a.v_out + p, make_float4(0.f, 0.f, 0.f, 0.f));
        f9_store(a.C_out, p, m3_zero());
        f9_store(a.F_out, p, m3_identity());
        return;
    }
    const float dt = a.step->dt;
    const float4 xm = __ldg(a.x + p);
    const V3 x = v3(xm.x, xm.y, xm.z);
    const Stencil st = make_stencil(x, a.inv_dx);
    const int G = a.G;
    const bool in_grid = stencil_in_grid(st, G);
    const G2POut o = g2p_gather(st, a.inv_dx, [&](int i, int j, int k) {
        const int ix = st.b[0] + i, iy = st.b[1] + j, iz = st.b[2] + k;
        if (!in_grid && (ix < 0 || iy < 0 || iz < 0 || ix >= G || iy >= G || iz >= G)) return v3(0.f, 0.f, 0.f);
        const float4 g = __ldg(a.vel + ((long long)ix * G + iy) * G + iz);
        return v3(g.x, g.y, g.z);
    });
    const float dx = 1.f / a.inv_dx;
    const float lo = dx * 2.f, hi = a.grid_lim - dx * 2.f;
    V3 nx = x + dt * o.v;
    nx = v3(fminf(fmaxf(nx.x, lo), hi), fminf(fmaxf(nx.y, lo), hi), fminf(fmaxf(nx.z, lo), hi));
    const M3 Fn = (m3_identity() + dt * o.gradv) * f9_load(a.Fe, p);
    __stcs(a.x_out + p, make_float4(nx.x, nx.y, nx.z, xm.w));
    __stcs(a.v_out + p, make_float4(o.v.x, o.v.y, o.v.z, 0.f));
    f9_store(a.C_out, p, o.C);
    f9_store(a.F_out, p, Fn);
    unsigned flags = 0;
    if (!finite3(o.v) || !finite3(nx) || !isfinite(Fn.m[0] + Fn.m[4] + Fn.m[8])) flags |= EMPM_STATUS_NAN;
    if (fmaxf(fmaxf(fabsf(o.v.x), fabsf(o.v.y)), fabsf(o.v.z)) * dt > dx) flags |= EMPM_STATUS_CFL;
    if (!in_grid) flags |= EMPM_STATUS_OUT_OF_BAND;
    if (flags) atomicOr(a.status, flags);
}

// ---- layout conversion and preparation kernels ---------------------------

__global__ void k_pack(const float* x3, const float* v3p, const float* C9, const float* F9, const float* mass,
                       int keep_mass, float4* x, float4* v, F9Planes C, F9Planes F, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (x3) {
        const float w = keep_mass ? x[p].w : (mass ? mass[p] : 0.f);
        x[p] = make_float4(x3[3 * p], x3[3 * p + 1], x3[3 * p + 2], w);
    }
    if (v3p) v[p] = make_float4(v3p[3 * p], v3p[3 * p + 1], v3p[3 * p + 2], 0.f);
    if (C9) { M3 m; for (int i = 0; i < 9; ++i) m.m[i] = C9[9 * p + i]; f9_store(C, p, m); }
    if (F9) { M3 m; for (int i = 0; i < 9; ++i) m.m[i] = F9[9 * p + i]; f9_store(F, p, m); }
}

__global__ void k_unpack(const float4* x, const float4* v, F9Planes C, F9Planes F,
                         float* x3, float* v3p, float* C9, float* F9, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (x3) { const float4 a = x[p]; x3[3 * p] = a.x; x3[3 * p + 1] = a.y; x3[3 * p + 2] = a.z; }
    if (v3p) { const float4 a = v[p]; v3p[3 * p] = a.x; v3p[3 * p + 1] = a.y; v3p[3 * p + 2] = a.z; }
    if (C9) { const M3 m = f9_load(C, p); for (int i = 0; i < 9; ++i) C9[9 * p + i] = m.m[i]; }
    if (F9) { const M3 m = f9_load(F, p); for (int i = 0; i < 9; ++i) F9[9 * p + i] = m.m[i]; }
}

// compute_mu_lam_from_E_nu (mpm_utils.py:277-283) and get_float_array_product
// (mpm_data_structure.py:719-726).
__global__ void k_prepare(const float* E, const float* nu, float* mu, float* lam,
                          const float* density, const float* vol, float4* x, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (E && nu) {
        const float e = E[p], q = nu[p];
        mu[p] = e / (2.f * (1.f + q));
        lam[p] = e * q / ((1.f + q) * (1.f - 2.f * q));
    }
    if (density && vol && x) x[p].w = density[p] * vol[p];
}

__global__ void k_debug_stress(const float* Ft9, float* mu, float* lam, float* ys, float dt, MaterialScalars ms,
                               float* F9, float* S9, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    M3 Ft;
    for (int i = 0; i < 9; ++i) Ft.m[i] = Ft9[9 * p + i];
    float m = mu[p], l = lam[p], y = ys[p];
    const ConstitutiveOut co = constitutive(Ft, m, l, y, dt, ms);
    mu[p] = m; lam[p] = l; ys[p] = y;
    for (int i = 0; i < 9; ++i) { F9[9 * p + i] = co.F.m[i]; S9[9 * p + i] = co.tau.m[i]; }
}

inline int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

static_assert(sizeof(EmpmCollider) == 104, "EmpmCollider layout changed: update empm_b200/_native.py");
static_assert(sizeof(EmpmModifier) == 88, "EmpmModifier layout changed: update empm_b200/_native.py");
static_assert(sizeof(EmpmStep) == 2384, "EmpmStep layout changed: update empm_b200/_native.py");

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

static thread_local char g_err[512] = "";

int empm_set_error(EmpmCtx* ctx, int code, const char* fmt, ...) {
    char* dst = ctx ? ctx->err : g_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    if (ctx) snprintf(g_err, sizeof(g_err), "%s", ctx->err);
    return code;
}

int empm_check_cuda(EmpmCtx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EMPM_OK;
    return empm_set_error(ctx, e == cudaErrorMemoryAllocation ? EMPM_ERR_OOM : EMPM_ERR_CUDA,
                          "%s: %s", what, cudaGetErrorString(e));
}

#define CK(expr, what)                                            \
    do {                                                          \
        int _rc = empm_check_cuda(ctx, (expr), what);             \
        if (_rc != EMPM_OK) return _rc;                           \
    } while (0)

extern "C" int empm_version(void) { return 100; }

static int validate_params(EmpmCtx* ctx, const EmpmModelParams* p) {
    if (!p) return empm_set_error(ctx, EMPM_ERR_INVALID, "params is NULL");
    if (p->n_grid < 4 || p->n_grid > 1024) return empm_set_error(ctx, EMPM_ERR_INVALID, "n_grid %d out of [4, 1024]", p->n_grid);
    if (!(p->grid_lim > 0.f)) return empm_set_error(ctx, EMPM_ERR_INVALID, "grid_lim must be > 0");
    if (p->material < 0 || p->material > 6) return empm_set_error(ctx, EMPM_ERR_UNSUPPORTED, "material id %d not in 0..6", p->material);
    return EMPM_OK;
}

extern "C" int empm_ctx_create(const EmpmModelParams* params, int n_particles, int max_steps, EmpmCtx** out) {
    EmpmCtx* ctx = nullptr;
    if (!out) return empm_set_error(nullptr, EMPM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = validate_params(nullptr, params);
    if (rc) return rc;
    if (n_particles < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "n_particles < 0");
    if (max_steps < 1 || max_steps > 100000) return empm_set_error(nullptr, EMPM_ERR_INVALID, "max_steps %d out of [1, 100000]", max_steps);
    ctx = new EmpmCtx();
    ctx->params = *params;
    ctx->n_particles = n_particles;
    ctx->max_steps = max_steps;
    const long long G = params->n_grid;
    const size_t grid_bytes = (size_t)(G * G * G) * sizeof(float4);
    cudaError_t e = cudaGetDevice(&ctx->device);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->grid_mom, grid_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->grid_vel, grid_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_steps, sizeof(EmpmStep) * (size_t)max_steps);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(ctx->grid_mom, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(ctx->grid_vel, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_a, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_b, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        rc = empm_check_cuda(nullptr, e, "empm_ctx_create");
        empm_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return EMPM_OK;
}

extern "C" int empm_ctx_destroy(EmpmCtx* ctx) {
    if (!ctx) return EMPM_OK;
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    for (cudaEvent_t ev : ctx->timing_events) cudaEventDestroy(ev);
    if (ctx->grid_mom) cudaFree(ctx->grid_mom);
    if (ctx->grid_vel) cudaFree(ctx->grid_vel);
    if (ctx->d_steps) cudaFree(ctx->d_steps);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
    if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
    delete ctx;
    return EMPM_OK;
}

extern "C" int empm_ctx_set_params(EmpmCtx* ctx, const EmpmModelParams* params) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = validate_params(ctx, params);
    if (rc) return rc;
    if (params->n_grid != ctx->params.n_grid)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_grid cannot change (%d -> %d)", ctx->params.n_grid, params->n_grid);
    if (memcmp(&ctx->params, params, sizeof(EmpmModelParams)) != 0) ctx->graph_valid = false;
    ctx->params = *params;
    return EMPM_OK;
}

extern "C" int empm_prepare(EmpmCtx* ctx, const float* E, const float* nu, float* mu, float* lam,
                            const float* density, const float* vol, float* x, int n, void* stream) {
    if (n < 0) return empm_set_error(ctx, EMPM_ERR_INVALID, "n < 0");
    if ((E || nu) && !(E && nu && mu && lam)) return empm_set_error(ctx, EMPM_ERR_INVALID, "E, nu, mu, lam must all be given");
    if (n == 0) return EMPM_OK;
    k_prepare<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(E, nu, mu, lam, density, vol,
                                                                    reinterpret_cast<float4*>(x), n);
    CK(cudaGetLastError(), "k_prepare");
    return EMPM_OK;
}

extern "C" int empm_pack_particles(const float* x3, const float* v3p, const float* C9, const float* F9,
                                   const float* mass, int keep_mass, EmpmParticles* dst, int n, void* stream) {
    EmpmCtx* ctx = nullptr;
    if (!dst || n < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad pack arguments");
    if (n == 0) return EMPM_OK;
    k_pack<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        x3, v3p, C9, F9, mass, keep_mass, reinterpret_cast<float4*>(dst->x), reinterpret_cast<float4*>(dst->v),
        f9_planes(dst->C, n), f9_planes(dst->F, n), n);
    CK(cudaGetLastError(), "k_pack");
    return EMPM_OK;
}

extern "C" int empm_unpack_particles(const EmpmParticles* src, float* x3, float* v3p, float* C9, float* F9,
                                     int n, void* stream) {
    EmpmCtx* ctx = nullptr;
    if (!src || n < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad unpack arguments");
    if (n == 0) return EMPM_OK;
    k_unpack<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4*>(src->x), reinterpret_cast<const float4*>(src->v),
        f9_planes(src->C, n), f9_planes(src->F, n), x3, v3p, C9, F9, n);
    CK(cudaGetLastError(), "k_unpack");
    return EMPM_OK;
}

static int check_particles(EmpmCtx* ctx, const EmpmParticles* p, const char* name) {
    if (!p || !p->x || !p->v || !p->C || !p->F)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "%s: particle plane pointer is NULL", name);
    if (((uintptr_t)p->x | (uintptr_t)p->v | (uintptr_t)p->C | (uintptr_t)p->F) & 15u)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "%s: particle planes must be 16-byte aligned", name);
    return EMPM_OK;
}

static int check_material(EmpmCtx* ctx, const EmpmMaterial* m) {
    if (!m || !m->vol || !m->mu || !m->lam || !m->yield_stress || !m->F_elastic)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "material pointer is NULL");
    if ((uintptr_t)m->F_elastic & 15u) return empm_set_error(ctx, EMPM_ERR_INVALID, "F_elastic must be 16-byte aligned");
    return EMPM_OK;
}

static void timing_mark(EmpmCtx* ctx, int kernel, int which, cudaStream_t stream) {
    if (!ctx->timing) return;
    int idx = ctx->timing_count[kernel];
    if (idx >= ctx->timing_capacity) return;
    cudaEventRecord(ctx->timing_events[((size_t)kernel * ctx->timing_capacity + idx) * 2 + which], stream);
    if (which == 1) ctx->timing_count[kernel] = idx + 1;
}

// Enqueue the three kernels of substep `s` (schedule at d_steps + s).
static int launch_substep(EmpmCtx* ctx, const EmpmParticles* in, EmpmParticles* out, const EmpmMaterial* mat,
                          const EmpmStep* d_step, cudaStream_t stream) {
    const EmpmModelParams& P = ctx->params;
    const int n = ctx->n_particles;
    const int G = P.n_grid;
    const float dx = P.grid_lim / (float)G;
    const float inv_dx = (float)G / P.grid_lim;
    MaterialScalars ms;
    ms.material = P.material;
    ms.softening = P.softening;
    ms.hardening = P.hardening;
    ms.xi = P.xi;
    ms.plastic_viscosity = P.plastic_viscosity;
    ms.alpha = P.alpha;
    if (n > 0) {
        P2GArgs a;
        a.x = reinterpret_cast<const float4*>(in->x);
        a.v = reinterpret_cast<float4*>(in->v);
        a.C = f9_planes(in->C, n);
        a.F = f9_planes(in->F, n);
        a.Fe = f9_planes(mat->F_elastic, n);
        a.vol = mat->vol;
        a.mu = mat->mu;
        a.lam = mat->lam;
        a.ys = mat->yield_stress;
        a.sel = mat->selection;
        a.grid = ctx->grid_mom;
        a.status = ctx->d_status;
        a.n = n;
        a.G = G;
        a.dx = dx;
        a.inv_dx = inv_dx;
        a.rpic = P.rpic_damping;
        a.ms = ms;
        a.step = d_step;
        timing_mark(ctx, 0, 0, stream);
        k_stress_p2g<<<blocks_for(n, 128), 128, 0, stream>>>(a);
        timing_mark(ctx, 0, 1, stream);
        CK(cudaGetLastError(), "k_stress_p2g");
    }
    {
        GridArgs g;
        g.mom = ctx->grid_mom;
        g.vel = ctx->grid_vel;
        g.G = G;
        g.dx = dx;
        g.g = v3(P.gravity[0], P.gravity[1], P.gravity[2]);
        g.damping = P.grid_v_damping_scale;
        g.step = d_step;
        const long long total = (long long)G * G * G;
        int nb = blocks_for(total, 256);
        if (nb > 148 * 16) nb = 148 * 16;
        timing_mark(ctx, 1, 0, stream);
        k_grid_update<<<nb, 256, 0, stream>>>(g);
        timing_mark(ctx, 1, 1, stream);
        CK(cudaGetLastError(), "k_grid_update");
    }
    if (n > 0) {
        G2PArgs a;
        a.x = reinterpret_cast<const float4*>(in->x);
        a.Fe = f9_planes(mat->F_elastic, n);
        a.sel = mat->selection;
        a.vel = ctx->grid_vel;
        a.x_out = reinterpret_cast<float4*>(out->x);
        a.v_out = reinterpret_cast<float4*>(out->v);
        a.C_out = f9_planes(out->C, n);
        a.F_out = f9_planes(out->F, n);
        a.status = ctx->d_status;
        a.n = n;
        a.G = G;
        a.inv_dx = inv_dx;
        a.grid_lim = P.grid_lim;
        a.step = d_step;
        timing_mark(ctx, 2, 0, stream);
        k_g2p<<<blocks_for(n, 128), 128, 0, stream>>>(a);
        timing_mark(ctx, 2, 1, stream);
        CK(cudaGetLastError(), "k_g2p");
    }
    return EMPM_OK;
}

static int upload_steps(EmpmCtx* ctx, const EmpmStep* steps, int n_steps, cudaStream_t stream) {
    if (!steps) return empm_set_error(ctx, EMPM_ERR_INVALID, "steps is NULL");
    if (n_steps < 1 || n_steps > ctx->max_steps)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d out of [1, %d]", n_steps, ctx->max_steps);
    for (int s = 0; s < n_steps; ++s) {
        if (steps[s].n_colliders < 0 || steps[s].n_colliders > EMPM_MAX_COLLIDERS ||
            steps[s].n_modifiers < 0 || steps[s].n_modifiers > EMPM_MAX_MODIFIERS)
            return empm_set_error(ctx, EMPM_ERR_INVALID, "step %d: collider/modifier count out of range", s);
    }
    // pageable source: the runtime stages it before returning, so the caller may reuse it
    CK(cudaMemcpyAsync(ctx->d_steps, steps, sizeof(EmpmStep) * (size_t)n_steps, cudaMemcpyHostToDevice, stream),
       "upload step table");
    return EMPM_OK;
}

extern "C" int empm_substep(EmpmCtx* ctx, const EmpmParticles* in, EmpmParticles* out, const EmpmMaterial* mat,
                            const EmpmStep* step, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, in, "in");
    if (!rc) rc = check_particles(ctx, out, "out");
    if (!rc) rc = check_material(ctx, mat);
    if (rc) return rc;
    if (in->x == out->x) return empm_set_error(ctx, EMPM_ERR_INVALID, "in and out must be distinct buffers");
    cudaStream_t s = (cudaStream_t)stream;
    rc = upload_steps(ctx, step, 1, s);
    if (rc) return rc;
    return launch_substep(ctx, in, out, mat, ctx->d_steps, s);
}

extern "C" int empm_rollout(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat,
                            const EmpmStep* steps, int n_steps, int use_graph, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, a, "a");
    if (!rc) rc = check_particles(ctx, b, "b");
    if (!rc) rc = check_material(ctx, mat);
    if (rc) return rc;
    if (a->x == b->x) return empm_set_error(ctx, EMPM_ERR_INVALID, "a and b must be distinct buffers");
    cudaStream_t s = (cudaStream_t)stream;
    rc = upload_steps(ctx, steps, n_steps, s);
    if (rc) return rc;
    if (!use_graph) {
        for (int i = 0; i < n_steps; ++i) {
            const EmpmParticles* in = (i & 1) ? b : a;
            EmpmParticles* out = (i & 1) ? a : b;
            rc = launch_substep(ctx, in, out, mat, ctx->d_steps + i, s);
            if (rc) return rc;
        }
        return EMPM_OK;
    }
    // CUDA graph path: capture on the context's own stream (legacy stream 0
    // cannot be captured), joined to the caller's stream by events.
    GraphKey key;
    memset(&key, 0, sizeof(key));
    key.a = *a;
    key.b = *b;
    key.mat = *mat;
    key.n_steps = n_steps;
    if (!ctx->graph_valid || memcmp(&key, &ctx->graph_key, sizeof(key)) != 0) {
        if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
        ctx->graph_valid = false;
        const bool timing_was = ctx->timing;
        ctx->timing = false;
        cudaError_t cap = cudaStreamBeginCapture(ctx->own_stream, cudaStreamCaptureModeThreadLocal);
        if (cap != cudaSuccess) { ctx->timing = timing_was; CK(cap, "begin capture"); }
        for (int i = 0; i < n_steps && rc == EMPM_OK; ++i) {
            const EmpmParticles* in = (i & 1) ? b : a;
            EmpmParticles* out = (i & 1) ? a : b;
            rc = launch_substep(ctx, in, out, mat, ctx->d_steps + i, ctx->own_stream);
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->own_stream, &graph);
        ctx->timing = timing_was;
        if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
        CK(e, "end capture");
        e = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        CK(e, "graph instantiate");
        ctx->graph_key = key;
        ctx->graph_valid = true;
    }
    CK(cudaEventRecord(ctx->ev_a, s), "record");
    CK(cudaStreamWaitEvent(ctx->own_stream, ctx->ev_a, 0), "wait");
    CK(cudaGraphLaunch(ctx->graph_exec, ctx->own_stream), "graph launch");
    CK(cudaEventRecord(ctx->ev_b, ctx->own_stream), "record");
    CK(cudaStreamWaitEvent(s, ctx->ev_b, 0), "wait");
    return EMPM_OK;
}

extern "C" int empm_read_status(EmpmCtx* ctx, uint32_t* status, void* stream) {
    if (!ctx || !status) return empm_set_error(ctx, EMPM_ERR_INVALID, "bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned h = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "read status");
    CK(cudaStreamSynchronize(s), "sync");
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), s), "clear status");
    *status = h;
    return EMPM_OK;
}

extern "C" int empm_last_error(EmpmCtx* ctx, char* buf, int len) {
    if (!buf || len <= 0) return EMPM_ERR_INVALID;
    snprintf(buf, (size_t)len, "%s", ctx ? ctx->err : g_err);
    return EMPM_OK;
}

extern "C" int empm_debug_stress(const EmpmModelParams* params, const float* F_trial9, float* mu, float* lam,
                                 float* yield_stress, float dt, float* F_out9, float* stress_out9, int n, void* stream) {
    EmpmCtx* ctx = nullptr;
    int rc = validate_params(nullptr, params);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!F_trial9 || !mu || !lam || !yield_stress || !F_out9 || !stress_out9)))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad empm_debug_stress arguments");
    if (n == 0) return EMPM_OK;
    MaterialScalars ms;
    ms.material = params->material;
    ms.softening = params->softening;
    ms.hardening = params->hardening;
    ms.xi = params->xi;
    ms.plastic_viscosity = params->plastic_viscosity;
    ms.alpha = params->alpha;
    k_debug_stress<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(F_trial9, mu, lam, yield_stress, dt, ms,
                                                                         F_out9, stress_out9, n);
    CK(cudaGetLastError(), "k_debug_stress");
    return EMPM_OK;
}

extern "C" int empm_ctx_grid(EmpmCtx* ctx, float** momentum, float** velocity) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (momentum) *momentum = reinterpret_cast<float*>(ctx->grid_mom);
    if (velocity) *velocity = reinterpret_cast<float*>(ctx->grid_vel);
    return EMPM_OK;
}

extern "C" int empm_ctx_timing(EmpmCtx* ctx, int enable, int max_launches) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    ctx->timing_count[0] = ctx->timing_count[1] = ctx->timing_count[2] = 0;
    if (!enable) { ctx->timing = false; return EMPM_OK; }
    if (max_launches < 1 || max_launches > 1000000)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "max_launches %d out of [1, 1000000]", max_launches);
    const size_t need = (size_t)3 * max_launches * 2;
    while (ctx->timing_events.size() < need) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev), "cudaEventCreate");
        ctx->timing_events.push_back(ev);
    }
    ctx->timing_capacity = max_launches;
    ctx->timing = true;
    return EMPM_OK;
}

extern "C" int empm_ctx_kernel_times(EmpmCtx* ctx, float* total_ms3, int* launches3) {
    if (!ctx || !total_ms3 || !launches3) return empm_set_error(ctx, EMPM_ERR_INVALID, "bad arguments");
    for (int k = 0; k < 3; ++k) {
        float total = 0.f;
        for (int i = 0; i < ctx->timing_count[k]; ++i) {
            const size_t base = ((size_t)k * ctx->timing_capacity + i) * 2;
            CK(cudaEventSynchronize(ctx->timing_events[base + 1]), "cudaEventSynchronize");
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->timing_events[base], ctx->timing_events[base + 1]), "cudaEventElapsedTime");
            total += ms;
        }
        total_ms3[k] = total;
        launches3[k] = ctx->timing_count[k];
    }
    return EMPM_OK;
}
