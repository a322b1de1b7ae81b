// substep.cu — launch orchestration and the C ABI of libempm_b200.so.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdarg.h>
#include <mutex>
#include <algorithm>
#include "../../include/empm_b200.h"
#include <cub/device/device_scan.cuh>
#include "kernels.cuh"
#include "adjoint.cuh"
#include "restart.cuh"
#include "ctx.hpp"

using namespace empm;

namespace {

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
static_assert(sizeof(EmpmStep) == 2392, "EmpmStep layout changed: update empm_b200/_native.py");

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

extern "C" int empm_version(void) { return 110; }

static int validate_params(EmpmCtx* ctx, const EmpmModelParams* p) {
    if (!p) return empm_set_error(ctx, EMPM_ERR_INVALID, "params is NULL");
    if (p->n_grid < 4 || p->n_grid > 1024) return empm_set_error(ctx, EMPM_ERR_INVALID, "n_grid %d out of [4, 1024]", p->n_grid);
    if (!(p->grid_lim > 0.f)) return empm_set_error(ctx, EMPM_ERR_INVALID, "grid_lim must be > 0");
    if (p->material < 0 || p->material > 6) return empm_set_error(ctx, EMPM_ERR_UNSUPPORTED, "material id %d not in 0..6", p->material);
    return EMPM_OK;
}

static void free_sorted(SortedBuffers& sb) {
    for (int i = 0; i < 2; ++i) {
        if (sb.part[i]) cudaFree(sb.part[i]);
        if (sb.matf[i]) cudaFree(sb.matf[i]);
        if (sb.mati[i]) cudaFree(sb.mati[i]);
        if (sb.fe[i]) cudaFree(sb.fe[i]);
    }
    void* ptrs[] = {sb.keys, sb.ranks, sb.block_counts, sb.block_offsets, sb.chunk_counts, sb.chunk_offsets,
                    sb.cell_counts, sb.cell_offsets, sb.chunks, sb.nchunks, sb.scan_tmp};
    for (void* q : ptrs) if (q) cudaFree(q);
    sb = SortedBuffers();
}

static void free_store(AdjointBuffers& ab) {
    void* ptrs[] = {ab.gsave, ab.gsave_list, ab.fe_store};
    for (void* q : ptrs) if (q) cudaFree(q);
    ab.gsave = nullptr;
    ab.gsave_list = nullptr;
    ab.fe_store = nullptr;
    ab.store_cap = 0;
}

static void free_adjoint(AdjointBuffers& ab) {
    free_store(ab);
    void* ptrs[] = {ab.states, ab.mats, ab.work, ab.fe, ab.gfe, ab.gx, ab.gacc, ab.gmom, ab.gstate, ab.gmats};
    for (void* q : ptrs) if (q) cudaFree(q);
    ab = AdjointBuffers();
}

static InstanceConsts instance_consts(const EmpmModelParams& P, int n, int poff, int boff) {
    InstanceConsts I;
    I.n = n;
    I.poff = poff;
    I.G = P.n_grid;
    I.NB = grid_nb(P.n_grid);
    I.boff = boff;
    I.dx = P.grid_lim / (float)P.n_grid;
    I.inv_dx = (float)P.n_grid / P.grid_lim;
    I.grid_lim = P.grid_lim;
    I.rpic = P.rpic_damping;
    I.damping = P.grid_v_damping_scale;
    I.g[0] = P.gravity[0];
    I.g[1] = P.gravity[1];
    I.g[2] = P.gravity[2];
    I.ms.material = P.material;
    I.ms.softening = P.softening;
    I.ms.hardening = P.hardening;
    I.ms.xi = P.xi;
    I.ms.plastic_viscosity = P.plastic_viscosity;
    I.ms.alpha = P.alpha;
    return I;
}

// Captured rollout graphs no longer match the context (options, instance
// tables, step-table storage): recapture on next use.
static void invalidate_graphs(EmpmCtx* ctx) {
    for (GraphEntry& g : ctx->graphs) g.valid = false;
    ctx->epoch++;
}

static void destroy_graphs(EmpmCtx* ctx) {
    for (GraphEntry& g : ctx->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.valid = false;
    }
    ctx->epoch++;
}

static int upload_instances(EmpmCtx* ctx) {
    std::vector<InstanceConsts> h(ctx->n_inst);
    for (int i = 0; i < ctx->n_inst; ++i) h[i] = instance_consts(ctx->params[i], ctx->counts[i], ctx->poff[i], ctx->boff[i]);
    CK(cudaMemcpy(ctx->d_inst, h.data(), sizeof(InstanceConsts) * h.size(), cudaMemcpyHostToDevice), "upload instances");
    ctx->params_version++;
    invalidate_graphs(ctx);
    return EMPM_OK;
}

static int ensure_step_capacity(EmpmCtx* ctx, int n_tables) {
    const size_t need = (size_t)n_tables * ctx->n_inst;
    if (need <= ctx->step_entries) return EMPM_OK;
    if (ctx->d_steps) {
        CK(cudaDeviceSynchronize(), "sync before step-table growth");
        cudaFree(ctx->d_steps);
        ctx->d_steps = nullptr;
        ctx->step_entries = 0;
    }
    CK(cudaMalloc(&ctx->d_steps, sizeof(EmpmStep) * need), "step table");
    ctx->step_entries = need;
    invalidate_graphs(ctx);
    return EMPM_OK;
}

extern "C" int empm_batch_create(const EmpmModelParams* params, const int* n_particles, int n_instances, int max_steps,
                                 EmpmCtx** out) {
    if (!out) return empm_set_error(nullptr, EMPM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!params || !n_particles || n_instances < 1 || n_instances > 4096)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad batch arguments (n_instances %d)", n_instances);
    if (max_steps < 1 || max_steps > 100000)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "max_steps %d out of [1, 100000]", max_steps);
    long long total = 0, blocks = 0;
    for (int i = 0; i < n_instances; ++i) {
        int rc = validate_params(nullptr, params + i);
        if (rc) return rc;
        if (n_particles[i] < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "instance %d: n_particles < 0", i);
        total += n_particles[i];
        const long long nb = grid_nb(params[i].n_grid);
        blocks += nb * nb * nb;
    }
    if (total > 0x3fffffffLL) return empm_set_error(nullptr, EMPM_ERR_INVALID, "too many particles (%lld)", total);
    if (blocks > (1LL << 25)) return empm_set_error(nullptr, EMPM_ERR_INVALID, "grids too large (%lld blocks)", blocks);
    EmpmCtx* ctx = new EmpmCtx();
    ctx->n_inst = n_instances;
    ctx->params.assign(params, params + n_instances);
    ctx->counts.assign(n_particles, n_particles + n_instances);
    int po = 0, bo = 0;
    for (int i = 0; i < n_instances; ++i) {
        ctx->poff.push_back(po);
        ctx->boff.push_back(bo);
        po += n_particles[i];
        const int nb = grid_nb(params[i].n_grid);
        bo += nb * nb * nb;
    }
    ctx->n_particles = (int)total;
    ctx->nblocks = blocks;
    ctx->cap_particles = (int)total;
    ctx->cap_blocks = blocks;
    ctx->cap_inst = n_instances;
    const size_t grid_bytes = (size_t)blocks * 64 * sizeof(float4);
    cudaError_t e = cudaGetDevice(&ctx->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_inst, sizeof(InstanceConsts) * n_instances);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->grid_mom, grid_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->grid_vel, grid_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->flags, (size_t)blocks);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->active, sizeof(int) * (2 * (size_t)blocks + 1));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(ctx->grid_mom, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(ctx->grid_vel, 0, grid_bytes);
    if (e == cudaSuccess) e = cudaMemset(ctx->flags, 0, (size_t)blocks);
    if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_a, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_b, cudaEventDisableTiming);
    int rc = EMPM_OK;
    if (e != cudaSuccess) rc = empm_check_cuda(nullptr, e, "empm_batch_create");
    if (rc == EMPM_OK) rc = upload_instances(ctx);
    if (rc == EMPM_OK) rc = ensure_step_capacity(ctx, max_steps);
    if (rc == EMPM_OK) rc = empm_check_cuda(nullptr, cudaDeviceSynchronize(), "empm_batch_create");
    if (rc != EMPM_OK) {
        empm_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return EMPM_OK;
}

extern "C" int empm_ctx_create(const EmpmModelParams* params, int n_particles, int max_steps, EmpmCtx** out) {
    return empm_batch_create(params, &n_particles, 1, max_steps, out);
}

extern "C" int empm_ctx_destroy(EmpmCtx* ctx) {
    if (!ctx) return EMPM_OK;
    destroy_graphs(ctx);
    for (AdjSegGraph& g : ctx->adj_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t ev : ctx->timing_events) cudaEventDestroy(ev);
    free_sorted(ctx->sb);
    free_adjoint(ctx->adj);
    void* ptrs[] = {ctx->d_inst, ctx->grid_mom, ctx->grid_vel, ctx->flags, ctx->active, ctx->d_steps, ctx->d_status};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
    if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
    delete ctx;
    return EMPM_OK;
}

extern "C" int empm_ctx_set_option(EmpmCtx* ctx, int option, int value) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    switch (option) {
        case EMPM_OPT_SORT_EVERY:
            if (value < 0) return empm_set_error(ctx, EMPM_ERR_INVALID, "sort_every must be >= 0");
            ctx->sort_every = value;
            break;
        case EMPM_OPT_P2G_MODE:
            if (value < 0 || value > 2) return empm_set_error(ctx, EMPM_ERR_INVALID, "p2g mode %d not in 0..2", value);
            ctx->p2g_mode = value;
            break;
        case EMPM_OPT_G2P_TILE: ctx->g2p_tile = value != 0; break;
        case EMPM_OPT_TILE_CAP:
            if (value < 27 || value > 3072) return empm_set_error(ctx, EMPM_ERR_INVALID, "tile_cap %d out of [27, 3072]", value);
            ctx->tile_cap = value;
            break;
        case EMPM_OPT_ADJ_STORE: ctx->adj_store = value != 0; break;
        case EMPM_OPT_FUSE: ctx->fuse = value != 0; break;
        case EMPM_OPT_SEGMENT_GRAPH: ctx->segment_graph = value != 0; break;
        case EMPM_OPT_SEG_CAP:
            if (value < 1 || value > 32 || (value & (value - 1)) != 0)
                return empm_set_error(ctx, EMPM_ERR_INVALID, "seg_cap %d not a power of two in 1..32", value);
            ctx->seg_cap = value;
            break;
        default: return empm_set_error(ctx, EMPM_ERR_INVALID, "unknown option %d", option);
    }
    invalidate_graphs(ctx);
    ctx->resident = false;
    return EMPM_OK;
}

extern "C" int empm_batch_set_params(EmpmCtx* ctx, int instance, const EmpmModelParams* params) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (instance < 0 || instance >= ctx->n_inst)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "instance %d out of [0, %d)", instance, ctx->n_inst);
    int rc = validate_params(ctx, params);
    if (rc) return rc;
    if (params->n_grid != ctx->params[instance].n_grid)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_grid cannot change (%d -> %d)", ctx->params[instance].n_grid,
                              params->n_grid);
    if (memcmp(&ctx->params[instance], params, sizeof(EmpmModelParams)) == 0) return EMPM_OK;
    ctx->params[instance] = *params;
    return upload_instances(ctx);
}

extern "C" int empm_batch_reserve(EmpmCtx* ctx, int max_particles, long long max_blocks, int max_instances) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (max_particles < 0 || max_particles > 0x3fffffff || max_blocks < 0 || max_blocks > (1LL << 25) ||
        max_instances < 0 || max_instances > 4096)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "reserve sizes out of range (%d particles, %lld blocks, %d instances)",
                              max_particles, max_blocks, max_instances);
    const bool grow_p = max_particles > ctx->cap_particles;
    const bool grow_b = max_blocks > ctx->cap_blocks;
    const bool grow_i = max_instances > ctx->cap_inst;
    if (!grow_p && !grow_b && !grow_i) return EMPM_OK;
    CK(cudaDeviceSynchronize(), "sync before reserve");
    destroy_graphs(ctx);
    ctx->resident = false;
    if (grow_b) {
        const size_t grid_bytes = (size_t)max_blocks * 64 * sizeof(float4);
        cudaFree(ctx->grid_mom);
        cudaFree(ctx->grid_vel);
        cudaFree(ctx->flags);
        cudaFree(ctx->active);
        ctx->grid_mom = ctx->grid_vel = nullptr;
        ctx->flags = nullptr;
        ctx->active = nullptr;
        CK(cudaMalloc(&ctx->grid_mom, grid_bytes), "reserve grid");
        CK(cudaMalloc(&ctx->grid_vel, grid_bytes), "reserve grid");
        CK(cudaMalloc(&ctx->flags, (size_t)max_blocks), "reserve grid");
        CK(cudaMalloc(&ctx->active, sizeof(int) * (2 * (size_t)max_blocks + 1)), "reserve grid");
        CK(cudaMemset(ctx->grid_mom, 0, grid_bytes), "reserve grid");
        CK(cudaMemset(ctx->grid_vel, 0, grid_bytes), "reserve grid");
        CK(cudaMemset(ctx->flags, 0, (size_t)max_blocks), "reserve grid");
        ctx->cap_blocks = max_blocks;
    }
    if (grow_i) {
        cudaFree(ctx->d_inst);
        ctx->d_inst = nullptr;
        CK(cudaMalloc(&ctx->d_inst, sizeof(InstanceConsts) * (size_t)max_instances), "reserve instance table");
        ctx->cap_inst = max_instances;
        int rc = upload_instances(ctx);
        if (rc) return rc;
    }
    if (grow_p) ctx->cap_particles = max_particles;
    free_sorted(ctx->sb);       // re-allocated at the new capacity on next use
    free_adjoint(ctx->adj);
    // step tables for blocks of up to 128 substeps of max_instances instances
    const size_t entries = (size_t)128 * ctx->cap_inst;
    if (entries > ctx->step_entries) {
        cudaFree(ctx->d_steps);
        ctx->d_steps = nullptr;
        ctx->step_entries = 0;
        CK(cudaMalloc(&ctx->d_steps, sizeof(EmpmStep) * entries), "reserve step tables");
        ctx->step_entries = entries;
    }
    CK(cudaDeviceSynchronize(), "reserve");
    return EMPM_OK;
}

extern "C" int empm_batch_reconfigure(EmpmCtx* ctx, const EmpmModelParams* params, const int* n_particles,
                                      int n_instances, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (!params || !n_particles || n_instances < 1)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "bad reconfigure arguments (n_instances %d)", n_instances);
    if (n_instances > ctx->cap_inst)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "%d instances exceed the context's capacity of %d", n_instances,
                              ctx->cap_inst);
    long long total = 0, blocks = 0;
    for (int i = 0; i < n_instances; ++i) {
        int rc = validate_params(ctx, params + i);
        if (rc) return rc;
        if (n_particles[i] < 0) return empm_set_error(ctx, EMPM_ERR_INVALID, "instance %d: n_particles < 0", i);
        total += n_particles[i];
        const long long nb = grid_nb(params[i].n_grid);
        blocks += nb * nb * nb;
    }
    if (total > ctx->cap_particles || blocks > ctx->cap_blocks)
        return empm_set_error(ctx, EMPM_ERR_INVALID,
                              "batch of %lld particles / %lld blocks exceeds the context's capacity (%d / %lld)", total,
                              blocks, ctx->cap_particles, ctx->cap_blocks);
    ctx->n_inst = n_instances;
    ctx->params.assign(params, params + n_instances);
    ctx->counts.assign(n_particles, n_particles + n_instances);
    ctx->poff.clear();
    ctx->boff.clear();
    int po = 0, bo = 0;
    for (int i = 0; i < n_instances; ++i) {
        ctx->poff.push_back(po);
        ctx->boff.push_back(bo);
        po += n_particles[i];
        const int nb = grid_nb(params[i].n_grid);
        bo += nb * nb * nb;
    }
    ctx->n_particles = (int)total;
    ctx->nblocks = blocks;
    // stream-ordered upload: kernels of the previous layout still queued on
    // this stream read the old table
    std::vector<InstanceConsts> h(n_instances);
    for (int i = 0; i < n_instances; ++i) h[i] = instance_consts(ctx->params[i], ctx->counts[i], ctx->poff[i], ctx->boff[i]);
    CK(cudaMemcpyAsync(ctx->d_inst, h.data(), sizeof(InstanceConsts) * h.size(), cudaMemcpyHostToDevice,
                       (cudaStream_t)stream), "upload instances");
    ctx->params_version++;
    invalidate_graphs(ctx);
    ctx->resident = false;
    return EMPM_OK;
}

extern "C" int empm_ctx_set_params(EmpmCtx* ctx, const EmpmModelParams* params) {
    return empm_batch_set_params(ctx, 0, params);
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

// True when a and b share any particle buffer (x, v, C or F_trial in either
// role): the G2P of one substep would overwrite state that other threads of
// the same launch still read.
static bool particles_alias(const EmpmParticles* a, const EmpmParticles* b) {
    const void* pa[4] = {a->x, a->v, a->C, a->F};
    const void* pb[4] = {b->x, b->v, b->C, b->F};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            if (pa[i] == pb[j]) return true;
    return false;
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

static Launch make_launch(EmpmCtx* ctx, int table) {
    Launch L;
    L.inst = ctx->d_inst;
    L.n_inst = ctx->n_inst;
    L.n_total = ctx->n_particles;
    L.nblocks = (int)ctx->nblocks;
    L.steps = ctx->d_steps;
    L.table = table;
    L.status = ctx->d_status;
    return L;
}

// the same on another step-table array (a stored segment's own)
static Launch make_launch_on(EmpmCtx* ctx, const EmpmStep* steps, int table) {
    Launch L = make_launch(ctx, table);
    L.steps = steps;
    return L;
}

static ParticleArrays particle_arrays(const EmpmParticles* p, int n) {
    ParticleArrays a;
    a.x = reinterpret_cast<float4*>(p->x);
    a.v = reinterpret_cast<float4*>(p->v);
    a.C = f9_planes(p->C, n);
    a.F = f9_planes(p->F, n);
    return a;
}

// x4 | v4 | C | F packed in one allocation; plane offsets use n rounded up
// to a multiple of 4 so that every float4 plane starts on a 16-byte boundary
static size_t padded4(int n) { return ((size_t)n + 3) & ~(size_t)3; }

static ParticleArrays particle_arrays(float* base, int n) {
    const size_t np = padded4(n);
    ParticleArrays a;
    a.x = reinterpret_cast<float4*>(base);
    a.v = reinterpret_cast<float4*>(base + 4 * np);
    a.C = f9_planes(base + 8 * np, n);
    a.F = f9_planes(base + 17 * np, n);
    return a;
}

// Grid update of one substep: the touched blocks are collected into a list
// (the count is reset first), then every node of the listed blocks is
// updated by its own thread. kKeep leaves the momentum and the flags in place.
// Threads per block of the P2G kernels: the kernel's usual size, or 64 when
// that would leave fewer than two blocks per SM (small instances would
// otherwise run on a fraction of the SMs; measured 16.7 -> 15.0 us for 20k
// particles; G2P measured no better). The kernels use no block-wide
// synchronisation, so any multiple of the warp size works.
// 1: the grid update runs one warp per touched block (k_grid_update_warps),
// 0: one thread per node (k_grid_update_list)
#ifndef EMPM_GRID_UPDATE_WARPS
#define EMPM_GRID_UPDATE_WARPS 1
#endif

static int particle_threads(const EmpmCtx* ctx, long long n, int usual) {
    return blocks_for(n, usual) >= 2LL * ctx->sm_count ? usual : 64;
}

// The material id all instances share, or -1 when they differ.
static int uniform_material(const EmpmCtx* ctx) {
    if (ctx->n_inst < 1) return -1;
    const int m = ctx->params[0].material;
    for (int i = 1; i < ctx->n_inst; ++i)
        if (ctx->params[i].material != m) return -1;
    return m;
}

// Optional store slot for launch_grid_update_list (stored segments).
struct GridStoreSlot {
    float4* blocks;
    int*    list;
    int     cap;
    int*    max_count;
};

template <bool kKeep>
static int launch_grid_update_list(EmpmCtx* ctx, const Launch& L, cudaStream_t stream,
                                   const GridStoreSlot* store = nullptr) {
    GridUpdateArgs g;
    g.mom = ctx->grid_mom;
    g.vel = ctx->grid_vel;
    g.flags = ctx->flags;
    g.L = L;
    if (store) {
        g.store = store->blocks;
        g.store_list = store->list;
        g.store_cap = store->cap;
        g.max_count = store->max_count;
    }
    CK(cudaMemsetAsync(ctx->active, 0, sizeof(int), stream), "reset touched-block count");
    k_collect_blocks<kKeep><<<blocks_for(ctx->nblocks, 256), 256, 0, stream>>>(ctx->flags, (int)ctx->nblocks,
                                                                               ctx->active, L);
    CK(cudaGetLastError(), "k_collect_blocks");
#if EMPM_GRID_UPDATE_WARPS
    k_grid_update_warps<kKeep><<<ctx->sm_count * 8, 256, 0, stream>>>(g, ctx->active);
#else
    k_grid_update_list<kKeep><<<ctx->sm_count * 8, 256, 0, stream>>>(g, ctx->active);
#endif
    CK(cudaGetLastError(), "k_grid_update_list");
    return EMPM_OK;
}

static int launch_grid_update(EmpmCtx* ctx, int table, cudaStream_t stream) {
    timing_mark(ctx, 1, 0, stream);
    const int rc = launch_grid_update_list<false>(ctx, make_launch(ctx, table), stream);
    timing_mark(ctx, 1, 1, stream);
    return rc;
}

// Direct path: particles in the caller's order, one particle per thread.
static int launch_substep_direct(EmpmCtx* ctx, const EmpmParticles* in, EmpmParticles* out, const EmpmMaterial* mat,
                                 int table, cudaStream_t stream) {
    const int n = ctx->n_particles;
    const Launch L = make_launch(ctx, table);
    const ParticleArrays Pin = particle_arrays(in, n);
    const ParticleArrays Pout = particle_arrays(out, n);
    MaterialArrays M;
    M.vol = mat->vol;
    M.mu = mat->mu;
    M.lam = mat->lam;
    M.ys = mat->yield_stress;
    M.sel = mat->selection;
    M.pid = nullptr;
    const F9Planes Fe = f9_planes(mat->F_elastic, n);
    if (n > 0) {
        timing_mark(ctx, 0, 0, stream);
        const int tp = particle_threads(ctx, n, 128);
        k_p2g_direct<<<blocks_for(n, tp), tp, 0, stream>>>(Pin, M, Fe, L, ctx->grid_mom, ctx->flags);
        timing_mark(ctx, 0, 1, stream);
        CK(cudaGetLastError(), "k_p2g_direct");
    }
    int rc = launch_grid_update(ctx, table, stream);
    if (rc) return rc;
    if (n > 0) {
        timing_mark(ctx, 2, 0, stream);
        k_g2p_direct<<<blocks_for(n, 128), 128, 0, stream>>>(Pin, Fe, M, Pout, L, ctx->grid_vel);
        timing_mark(ctx, 2, 1, stream);
        CK(cudaGetLastError(), "k_g2p_direct");
    }
    return EMPM_OK;
}

static int ensure_sorted_buffers(EmpmCtx* ctx) {
    SortedBuffers& sb = ctx->sb;
    if (sb.allocated && sb.n >= ctx->n_particles && sb.nb >= ctx->nblocks) return EMPM_OK;
    free_sorted(sb);
    ctx->resident = false;
    ctx->epoch++;
    // sized for the context's capacity, so that re-laid batches reuse them
    const int n = ctx->cap_particles;
    const size_t nblocks = (size_t)ctx->cap_blocks;
    sb.max_chunks = (int)((size_t)n / TILE_THREADS + nblocks + 1);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaMalloc(&sb.part[i], sizeof(float) * 26 * padded4(n) + 64);
        if (e == cudaSuccess) e = cudaMalloc(&sb.matf[i], sizeof(float) * 4 * (size_t)n + 64);
        if (e == cudaSuccess) e = cudaMalloc(&sb.mati[i], sizeof(int) * 2 * (size_t)n + 64);
        if (e == cudaSuccess) e = cudaMalloc(&sb.fe[i], sizeof(float) * 9 * (size_t)n + 64);
    }
    if (e == cudaSuccess) e = cudaMalloc(&sb.keys, sizeof(int) * (size_t)n + 64);
    if (e == cudaSuccess) e = cudaMalloc(&sb.ranks, sizeof(int) * (size_t)n + 64);
    if (e == cudaSuccess) e = cudaMalloc(&sb.block_counts, sizeof(int) * nblocks);
    if (e == cudaSuccess) e = cudaMalloc(&sb.block_offsets, sizeof(int) * nblocks);
    if (e == cudaSuccess) e = cudaMalloc(&sb.chunk_counts, sizeof(int) * nblocks);
    if (e == cudaSuccess) e = cudaMalloc(&sb.chunk_offsets, sizeof(int) * nblocks);
    if (e == cudaSuccess) e = cudaMalloc(&sb.cell_counts, sizeof(int) * nblocks * 64);
    if (e == cudaSuccess) e = cudaMalloc(&sb.cell_offsets, sizeof(int) * nblocks * 64);
    if (e == cudaSuccess) e = cudaMalloc(&sb.chunks, sizeof(int2) * (size_t)sb.max_chunks);
    if (e == cudaSuccess) e = cudaMalloc(&sb.nchunks, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(sb.block_counts, 0, sizeof(int) * nblocks);
    if (e == cudaSuccess) e = cudaMemset(sb.cell_counts, 0, sizeof(int) * nblocks * 64);
    if (e == cudaSuccess) e = cudaMemset(sb.nchunks, 0, sizeof(int));
    if (e == cudaSuccess) {
        size_t bytes = 0;
        e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, sb.block_counts, sb.block_offsets, (int)nblocks);
        if (e == cudaSuccess) {
            sb.scan_tmp_bytes = bytes;
            e = cudaMalloc(&sb.scan_tmp, bytes + 16);
        }
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        free_sorted(sb);
        return empm_check_cuda(ctx, e, "sorted-path buffers");
    }
    sb.allocated = true;
    sb.n = n;
    sb.nb = (long long)nblocks;
    return EMPM_OK;
}

struct SortedState {
    int pc = 0;   // particle buffer holding the current state
    int mc = 0;   // material buffer of the current sort epoch
};

static MaterialArrays sorted_material(EmpmCtx* ctx, int mc) {
    const int n = ctx->n_particles;
    MaterialArrays M;
    float* f = ctx->sb.matf[mc];
    int* i = ctx->sb.mati[mc];
    M.vol = f;
    M.mu = f + n;
    M.lam = f + 2 * (size_t)n;
    M.ys = f + 3 * (size_t)n;
    M.sel = i;
    M.pid = i + n;
    return M;
}

// Sort `src` (the caller's arrays when user_src is given, else the current
// sorted state) into the other sorted buffers: cell keys and ranks, block
// scan (CUB), per-block cell scan and chunk list, scatter.
static int launch_sort(EmpmCtx* ctx, SortedState& ss, const ParticleArrays* user_src, const EmpmMaterial* user_mat,
                       cudaStream_t stream) {
    SortedBuffers& sb = ctx->sb;
    const int n = ctx->n_particles;
    const int nblocks = (int)ctx->nblocks;
    PermuteArgs a;
    if (user_src) {
        a.src = *user_src;
        a.vol_s = user_mat->vol;
        a.mu_s = user_mat->mu;
        a.lam_s = user_mat->lam;
        a.ys_s = user_mat->yield_stress;
        a.sel_s = user_mat->selection;
        a.pid_s = nullptr;
    } else {
        a.src = particle_arrays(sb.part[ss.pc], n);
        const MaterialArrays M = sorted_material(ctx, ss.mc);
        a.vol_s = M.vol; a.mu_s = M.mu; a.lam_s = M.lam; a.ys_s = M.ys; a.sel_s = M.sel; a.pid_s = M.pid;
    }
    const int dp = user_src ? ss.pc : 1 - ss.pc;
    const int dm = user_src ? ss.mc : 1 - ss.mc;
    // elastic F travels with the sort: particles of a held instance keep
    // theirs (the others' is rewritten by their next stress + P2G)
    a.fe_s = F9Planes{};
    if (user_src) {
        if (user_mat->F_elastic) a.fe_s = f9_planes(user_mat->F_elastic, n);
    } else {
        a.fe_s = f9_planes(sb.fe[ss.mc], n);
    }
    a.fe_d = f9_planes(sb.fe[dm], n);
    a.dst = particle_arrays(sb.part[dp], n);
    const MaterialArrays D = sorted_material(ctx, dm);
    a.vol_d = const_cast<float*>(D.vol); a.mu_d = D.mu; a.lam_d = D.lam; a.ys_d = D.ys;
    a.sel_d = const_cast<int*>(D.sel); a.pid_d = const_cast<int*>(D.pid);
    a.keys = sb.keys;
    a.ranks = sb.ranks;
    a.offsets = sb.cell_offsets;
    a.n = n;
    const Launch L = make_launch(ctx, 0);
    k_sort_keys<<<blocks_for(n, 256), 256, 0, stream>>>(reinterpret_cast<const float4*>(a.src.x), L, sb.keys, sb.ranks,
                                                        sb.cell_counts, sb.block_counts);
    CK(cudaGetLastError(), "k_sort_keys");
    k_chunk_counts<<<blocks_for(nblocks, 256), 256, 0, stream>>>(sb.block_counts, sb.chunk_counts, nblocks, TILE_THREADS);
    CK(cudaGetLastError(), "k_chunk_counts");
    size_t bytes = sb.scan_tmp_bytes;
    CK(cub::DeviceScan::ExclusiveSum(sb.scan_tmp, bytes, sb.block_counts, sb.block_offsets, nblocks, stream), "block scan");
    bytes = sb.scan_tmp_bytes;
    CK(cub::DeviceScan::ExclusiveSum(sb.scan_tmp, bytes, sb.chunk_counts, sb.chunk_offsets, nblocks, stream), "chunk scan");
    k_cell_scan<<<blocks_for((long long)nblocks * 32, 256), 256, 0, stream>>>(
        sb.cell_counts, sb.block_counts, sb.block_offsets, sb.chunk_offsets, sb.chunk_counts, sb.cell_offsets,
        sb.chunks, sb.nchunks, nblocks, TILE_THREADS);
    CK(cudaGetLastError(), "k_cell_scan");
    k_sort_scatter<<<blocks_for(n, 256), 256, 0, stream>>>(a);
    CK(cudaGetLastError(), "k_sort_scatter");
    ss.pc = dp;
    ss.mc = dm;
    return EMPM_OK;
}

static TiledArgs sorted_args(EmpmCtx* ctx, const SortedState& ss, int table) {
    SortedBuffers& sb = ctx->sb;
    const int n = ctx->n_particles;
    TiledArgs t;
    t.P = particle_arrays(sb.part[ss.pc], n);
    t.M = sorted_material(ctx, ss.mc);
    t.Fe = f9_planes(sb.fe[ss.mc], n);
    t.L = make_launch(ctx, table);
    t.cl.chunks = sb.chunks;
    t.cl.nchunks = sb.nchunks;
    t.grid = ctx->grid_mom;
    t.flags = ctx->flags;
    t.out = particle_arrays(sb.part[1 - ss.pc], n);
    t.tile_cap = 0;
    return t;
}

// stress + P2G of one substep on the sorted state
static int launch_p2g_sorted(EmpmCtx* ctx, const SortedState& ss, int table, cudaStream_t stream) {
    const int n = ctx->n_particles;
    TiledArgs t = sorted_args(ctx, ss, table);
    t.tile_cap = ctx->p2g_mode == 1 ? ctx->tile_cap : 0;
    const size_t smem = sizeof(float4) * (size_t)ctx->tile_cap;
    timing_mark(ctx, 0, 0, stream);
    if (ctx->p2g_mode == 2) {
        const int tp = particle_threads(ctx, n, 256);
        launch_p2g_warpagg(blocks_for(n, tp), tp, stream, t.P, t.M, t.Fe, t.L, ctx->grid_mom, ctx->flags,
                           ctx->seg_cap, uniform_material(ctx));
    } else {
        k_p2g_tiled<<<ctx->sm_count * 2, TILE_THREADS, smem, stream>>>(t);
    }
    timing_mark(ctx, 0, 1, stream);
    CK(cudaGetLastError(), "k_p2g_sorted");
    return EMPM_OK;
}

// G2P of one substep: the sorted state -> the other particle buffer
static int launch_g2p_sorted(EmpmCtx* ctx, SortedState& ss, int table, cudaStream_t stream) {
    const int n = ctx->n_particles;
    TiledArgs t = sorted_args(ctx, ss, table);
    t.grid = ctx->grid_vel;
    t.tile_cap = ctx->g2p_tile ? ctx->tile_cap : 0;
    const size_t smem = sizeof(float4) * (size_t)ctx->tile_cap;
    timing_mark(ctx, 2, 0, stream);
    if (ctx->g2p_tile) {
        k_g2p_tiled<<<ctx->sm_count * 2, TILE_THREADS, smem, stream>>>(t);
    } else {
        k_g2p_direct<<<blocks_for(n, 128), 128, 0, stream>>>(t.P, t.Fe, t.M, t.out, t.L, ctx->grid_vel);
    }
    timing_mark(ctx, 2, 1, stream);
    CK(cudaGetLastError(), "k_g2p_sorted");
    ss.pc = 1 - ss.pc;
    return EMPM_OK;
}

static int launch_substep_sorted(EmpmCtx* ctx, SortedState& ss, int table, cudaStream_t stream) {
    int rc = launch_p2g_sorted(ctx, ss, table, stream);
    if (!rc) rc = launch_grid_update(ctx, table, stream);
    if (!rc) rc = launch_g2p_sorted(ctx, ss, table, stream);
    return rc;
}

// Fused G2P of substep g2p_table and stress + P2G of substep `table`, in
// place on the sorted state's positions and the elastic F buffer.
static int launch_g2p2g_sorted(EmpmCtx* ctx, const SortedState& ss, int g2p_table, int table, cudaStream_t stream) {
    const int n = ctx->n_particles;
    const TiledArgs t = sorted_args(ctx, ss, table);
    const int tp = particle_threads(ctx, n, 256);
    timing_mark(ctx, 6, 0, stream);
    launch_g2p2g(blocks_for(n, tp), tp, stream, t.P, t.M, t.Fe, t.L, g2p_table, ctx->grid_vel, ctx->grid_mom,
                 ctx->flags, ctx->seg_cap, uniform_material(ctx), tp < 256);
    timing_mark(ctx, 6, 1, stream);
    CK(cudaGetLastError(), "k_g2p2g");
    return EMPM_OK;
}

static bool use_fused(const EmpmCtx* ctx) {
    return ctx->fuse && ctx->fuse_ok && ctx->p2g_mode == 2 && !ctx->g2p_tile;
}

// Substeps [first, first + count) of a rollout on the sorted state, with no
// cell sort among them: separately, or as one run of fused kernels (the
// run's first stress + P2G and last G2P separate).
static int launch_sorted_run(EmpmCtx* ctx, SortedState& ss, int first, int count, int n_tables,
                             cudaStream_t stream) {
    auto table = [&](int i) { return n_tables == 1 ? 0 : i; };
    int rc = EMPM_OK;
    if (count < 2 || !use_fused(ctx)) {
        for (int i = first; i < first + count && rc == EMPM_OK; ++i) rc = launch_substep_sorted(ctx, ss, table(i), stream);
        return rc;
    }
    rc = launch_p2g_sorted(ctx, ss, table(first), stream);
    if (!rc) rc = launch_grid_update(ctx, table(first), stream);
    for (int i = first + 1; i < first + count && rc == EMPM_OK; ++i) {
        rc = launch_g2p2g_sorted(ctx, ss, table(i - 1), table(i), stream);
        if (!rc) rc = launch_grid_update(ctx, table(i), stream);
    }
    if (!rc) rc = launch_g2p_sorted(ctx, ss, table(first + count - 1), stream);
    return rc;
}

static bool use_sorted(EmpmCtx* ctx) {
    return ctx->sort_every > 0 && ctx->n_particles > 0;
}

// The whole launch sequence of a rollout (also what a graph captures). On the
// sorted path, ss / since carry the sorted state: with EMPM_ROLLOUT_RESUME the
// sequence starts from them instead of sorting the caller's buffers, and on
// return they hold the state it ends in. The cell sort repeats once since
// reaches sort_every substeps, so the cadence continues across resumed calls.
// With EMPM_ROLLOUT_KEEP the result stays in the sorted buffers only.
static int launch_rollout(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat, int n_tables,
                          int n_steps, int flags, SortedState& ss, int& since, cudaStream_t stream) {
    int rc = EMPM_OK;
    if (!use_sorted(ctx)) {
        for (int i = 0; i < n_steps && rc == EMPM_OK; ++i) {
            const EmpmParticles* in = (i & 1) ? b : a;
            EmpmParticles* out = (i & 1) ? a : b;
            rc = launch_substep_direct(ctx, in, out, mat, n_tables == 1 ? 0 : i, stream);
        }
        return rc;
    }
    const int n = ctx->n_particles;
    if (!(flags & EMPM_ROLLOUT_RESUME)) {
        ss = SortedState();
        const ParticleArrays ua = particle_arrays(a, n);
        rc = launch_sort(ctx, ss, &ua, mat, stream);
        since = 0;
    }
    for (int i = 0; i < n_steps && rc == EMPM_OK;) {
        if (since >= ctx->sort_every) {
            rc = launch_sort(ctx, ss, nullptr, nullptr, stream);
            since = 0;
        }
        // the substeps up to the next cell sort
        const int count = std::min(n_steps - i, ctx->sort_every - since);
        if (rc == EMPM_OK) rc = launch_sorted_run(ctx, ss, i, count, n_tables, stream);
        since += count;
        i += count;
    }
    if (rc || (flags & EMPM_ROLLOUT_KEEP)) return rc;
    UnsortArgs u;
    u.src = particle_arrays(ctx->sb.part[ss.pc], n);
    u.dst = particle_arrays((n_steps & 1) ? b : a, n);
    u.Fe_s = f9_planes(ctx->sb.fe[ss.mc], n);
    u.Fe_d = f9_planes(mat->F_elastic, n);
    const MaterialArrays M = sorted_material(ctx, ss.mc);
    u.mu_s = M.mu; u.mu_d = mat->mu;
    u.lam_s = M.lam; u.lam_d = mat->lam;
    u.ys_s = M.ys; u.ys_d = mat->yield_stress;
    u.pid = M.pid;
    u.n = n;
    k_unsort<<<blocks_for(n, 256), 256, 0, stream>>>(u);
    CK(cudaGetLastError(), "k_unsort");
    return EMPM_OK;
}

static int check_steps(EmpmCtx* ctx, const EmpmStep* steps, int n_tables) {
    if (!steps) return empm_set_error(ctx, EMPM_ERR_INVALID, "steps is NULL");
    if (n_tables < 1 || n_tables > 100000) return empm_set_error(ctx, EMPM_ERR_INVALID, "n_tables %d out of [1, 100000]", n_tables);
    const size_t total = (size_t)n_tables * ctx->n_inst;
    for (size_t s = 0; s < total; ++s) {
        if (steps[s].n_colliders < 0 || steps[s].n_colliders > EMPM_MAX_COLLIDERS ||
            steps[s].n_modifiers < 0 || steps[s].n_modifiers > EMPM_MAX_MODIFIERS)
            return empm_set_error(ctx, EMPM_ERR_INVALID, "step entry %zu: collider/modifier count out of range", s);
    }
    return EMPM_OK;
}

static int upload_steps(EmpmCtx* ctx, const EmpmStep* steps, int n_tables, cudaStream_t stream) {
    int rc = check_steps(ctx, steps, n_tables);
    if (rc) return rc;
    const size_t total = (size_t)n_tables * ctx->n_inst;
    rc = ensure_step_capacity(ctx, n_tables);
    if (rc) return rc;
    // pageable source: the runtime stages it before returning, so the caller may reuse it
    CK(cudaMemcpyAsync(ctx->d_steps, steps, sizeof(EmpmStep) * total, cudaMemcpyHostToDevice, stream),
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
    if (particles_alias(in, out)) return empm_set_error(ctx, EMPM_ERR_INVALID, "in and out must be distinct buffers");
    cudaStream_t s = (cudaStream_t)stream;
    rc = upload_steps(ctx, step, 1, s);
    if (rc) return rc;
    return launch_substep_direct(ctx, in, out, mat, 0, s);
}

extern "C" int empm_substep_inplace(EmpmCtx* ctx, EmpmParticles* state, const EmpmMaterial* mat,
                                    const EmpmStep* step, float* cov, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, state, "state");
    if (!rc) rc = check_material(ctx, mat);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = upload_steps(ctx, step, 1, s);
    if (rc) return rc;
    const int n = ctx->n_particles;
    const Launch L = make_launch(ctx, 0);
    const ParticleArrays P = particle_arrays(state, n);
    MaterialArrays M;
    M.vol = mat->vol;
    M.mu = mat->mu;
    M.lam = mat->lam;
    M.ys = mat->yield_stress;
    M.sel = mat->selection;
    M.pid = nullptr;
    const F9Planes Fe = f9_planes(mat->F_elastic, n);
    if (n > 0) {
        const int tp = particle_threads(ctx, n, 128);
        k_p2g_direct<<<blocks_for(n, tp), tp, 0, s>>>(P, M, Fe, L, ctx->grid_mom, ctx->flags);
        CK(cudaGetLastError(), "k_p2g_direct (in place)");
    }
    rc = launch_grid_update(ctx, 0, s);
    if (rc) return rc;
    if (n > 0) {
        k_g2p_inplace<<<blocks_for(n, 128), 128, 0, s>>>(P, Fe, M, L, ctx->grid_vel, cov);
        CK(cudaGetLastError(), "k_g2p_inplace");
    }
    return EMPM_OK;
}

extern "C" int empm_rollout_ex(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat,
                               const EmpmStep* steps, int n_tables, int n_steps, int flags, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, a, "a");
    if (!rc) rc = check_particles(ctx, b, "b");
    if (!rc) rc = check_material(ctx, mat);
    if (rc) return rc;
    if (particles_alias(a, b)) return empm_set_error(ctx, EMPM_ERR_INVALID, "a and b must be distinct buffers");
    if (n_steps < 1 || n_steps > 100000) return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d out of [1, 100000]", n_steps);
    if (n_tables != 1 && n_tables != n_steps)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_tables must be 1 or n_steps (%d, %d)", n_tables, n_steps);
    if (flags & ~(EMPM_ROLLOUT_GRAPH | EMPM_ROLLOUT_RESUME | EMPM_ROLLOUT_KEEP))
        return empm_set_error(ctx, EMPM_ERR_INVALID, "unknown rollout flags %#x", flags);
    cudaStream_t s = (cudaStream_t)stream;
    const bool sorted = use_sorted(ctx);
    if (!sorted) flags &= EMPM_ROLLOUT_GRAPH;   // the direct path always writes the caller's buffers
    rc = upload_steps(ctx, steps, n_tables, s);
    if (rc) return rc;
    // fused runs keep no velocity between substeps: an instance released from
    // a hold (hold 1 in one table, 0 in a later one) needs the separate kernels
    ctx->fuse_ok = true;
    for (int inst = 0; inst < ctx->n_inst && ctx->fuse_ok; ++inst)
        for (int t = 1; t < n_tables; ++t)
            if (steps[(size_t)(t - 1) * ctx->n_inst + inst].hold && !steps[(size_t)t * ctx->n_inst + inst].hold) {
                ctx->fuse_ok = false;
                break;
            }
    if (sorted) {
        rc = ensure_sorted_buffers(ctx);
        if (rc) return rc;
    }
    if ((flags & EMPM_ROLLOUT_RESUME) && !ctx->resident)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "EMPM_ROLLOUT_RESUME: no sorted state to continue from");
    SortedState ss;
    int since = 0;
    if (flags & EMPM_ROLLOUT_RESUME) {
        ss.pc = ctx->resident_pc;
        ss.mc = ctx->resident_mc;
        since = ctx->resident_since;
    }
    ctx->resident = false;
    if (!(flags & EMPM_ROLLOUT_GRAPH)) {
        rc = launch_rollout(ctx, a, b, mat, n_tables, n_steps, flags, ss, since, s);
        if (rc) return rc;
    } else {
        // CUDA graph path: capture on the context's own stream (legacy stream 0
        // cannot be captured), joined to the caller's stream by events. The
        // graphs are cached by launch key, which includes the sorted state a
        // resumed sequence starts in.
        GraphKey key;
        memset(&key, 0, sizeof(key));
        key.a = *a;
        key.b = *b;
        key.mat = *mat;
        key.n_steps = n_steps;
        key.n_tables = n_tables;
        key.sort_every = ctx->sort_every;
        key.p2g_mode = ctx->p2g_mode;
        key.g2p_tile = ctx->g2p_tile;
        key.tile_cap = ctx->tile_cap;
        key.seg_cap = ctx->seg_cap;
        key.fuse = use_fused(ctx) ? 1 : 0;
        key.params_version = ctx->params_version;
        key.flags = flags & (EMPM_ROLLOUT_RESUME | EMPM_ROLLOUT_KEEP);
        if (flags & EMPM_ROLLOUT_RESUME) {
            key.start_pc = ss.pc;
            key.start_mc = ss.mc;
            key.start_since = since;
        }
        GraphEntry* g = nullptr;
        for (GraphEntry& e : ctx->graphs)
            if (e.valid && memcmp(&key, &e.key, sizeof(key)) == 0) { g = &e; break; }
        if (!g) {
            g = &ctx->graphs[0];
            for (GraphEntry& e : ctx->graphs) {
                if (!e.valid) { g = &e; break; }
                if (e.used < g->used) g = &e;
            }
            if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
            g->valid = false;
            const bool timing_was = ctx->timing;
            ctx->timing = false;
            cudaError_t cap = cudaStreamBeginCapture(ctx->own_stream, cudaStreamCaptureModeThreadLocal);
            if (cap != cudaSuccess) { ctx->timing = timing_was; CK(cap, "begin capture"); }
            rc = launch_rollout(ctx, a, b, mat, n_tables, n_steps, flags, ss, since, ctx->own_stream);
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamEndCapture(ctx->own_stream, &graph);
            ctx->timing = timing_was;
            if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
            CK(e, "end capture");
            e = cudaGraphInstantiate(&g->exec, graph, 0);
            cudaGraphDestroy(graph);
            CK(e, "graph instantiate");
            g->key = key;
            g->valid = true;
            g->end_pc = ss.pc;
            g->end_mc = ss.mc;
            g->end_since = since;
        }
        g->used = ++ctx->graph_clock;
        ss.pc = g->end_pc;
        ss.mc = g->end_mc;
        since = g->end_since;
        CK(cudaEventRecord(ctx->ev_a, s), "record");
        CK(cudaStreamWaitEvent(ctx->own_stream, ctx->ev_a, 0), "wait");
        CK(cudaGraphLaunch(g->exec, ctx->own_stream), "graph launch");
        CK(cudaEventRecord(ctx->ev_b, ctx->own_stream), "record");
        CK(cudaStreamWaitEvent(s, ctx->ev_b, 0), "wait");
    }
    if (sorted) {
        ctx->resident = true;
        ctx->resident_pc = ss.pc;
        ctx->resident_mc = ss.mc;
        ctx->resident_since = since;
    }
    return EMPM_OK;
}

extern "C" int empm_rollout(EmpmCtx* ctx, EmpmParticles* a, EmpmParticles* b, const EmpmMaterial* mat,
                            const EmpmStep* steps, int n_tables, int n_steps, int use_graph, void* stream) {
    return empm_rollout_ex(ctx, a, b, mat, steps, n_tables, n_steps, use_graph ? EMPM_ROLLOUT_GRAPH : 0, stream);
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

extern "C" int empm_batch_info(EmpmCtx* ctx, int* n_instances, int* particle_offsets, int* block_offsets) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (n_instances) *n_instances = ctx->n_inst;
    for (int i = 0; i < ctx->n_inst; ++i) {
        if (particle_offsets) particle_offsets[i] = ctx->poff[i];
        if (block_offsets) block_offsets[i] = ctx->boff[i];
    }
    return EMPM_OK;
}

extern "C" int empm_ctx_timing(EmpmCtx* ctx, int enable, int max_launches) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    for (int k = 0; k < EmpmCtx::kTimedKernels; ++k) ctx->timing_count[k] = 0;
    if (!enable) { ctx->timing = false; return EMPM_OK; }
    if (max_launches < 1 || max_launches > 1000000)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "max_launches %d out of [1, 1000000]", max_launches);
    const size_t need = (size_t)EmpmCtx::kTimedKernels * max_launches * 2;
    while (ctx->timing_events.size() < need) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev), "cudaEventCreate");
        ctx->timing_events.push_back(ev);
    }
    ctx->timing_capacity = max_launches;
    ctx->timing = true;
    return EMPM_OK;
}

static int kernel_times(EmpmCtx* ctx, int first, float* total_ms3, int* launches3) {
    if (!ctx || !total_ms3 || !launches3) return empm_set_error(ctx, EMPM_ERR_INVALID, "bad arguments");
    for (int j = 0; j < 3; ++j) {
        const int k = first + j;
        float total = 0.f;
        for (int i = 0; i < ctx->timing_count[k]; ++i) {
            const size_t base = ((size_t)k * ctx->timing_capacity + i) * 2;
            CK(cudaEventSynchronize(ctx->timing_events[base + 1]), "cudaEventSynchronize");
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->timing_events[base], ctx->timing_events[base + 1]), "cudaEventElapsedTime");
            total += ms;
        }
        total_ms3[j] = total;
        launches3[j] = ctx->timing_count[k];
    }
    return EMPM_OK;
}

extern "C" int empm_ctx_kernel_times(EmpmCtx* ctx, float* total_ms3, int* launches3) {
    return kernel_times(ctx, 0, total_ms3, launches3);
}

extern "C" int empm_ctx_adjoint_kernel_times(EmpmCtx* ctx, float* total_ms3, int* launches3) {
    return kernel_times(ctx, 3, total_ms3, launches3);
}

extern "C" int empm_ctx_fused_kernel_times(EmpmCtx* ctx, float* total_ms, int* launches) {
    if (!ctx || !total_ms || !launches) return empm_set_error(ctx, EMPM_ERR_INVALID, "bad arguments");
    const int k = 6;
    float total = 0.f;
    for (int i = 0; i < ctx->timing_count[k]; ++i) {
        const size_t base = ((size_t)k * ctx->timing_capacity + i) * 2;
        CK(cudaEventSynchronize(ctx->timing_events[base + 1]), "cudaEventSynchronize");
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->timing_events[base], ctx->timing_events[base + 1]), "cudaEventElapsedTime");
        total += ms;
    }
    *total_ms = total;
    *launches = ctx->timing_count[k];
    return EMPM_OK;
}

// ===========================================================================
// Reverse mode
// ===========================================================================
namespace {

__global__ void k_debug_stress_adjoint(const float* Ft9, const float* mu, const float* lam, const float* ys,
                                       float dt, MaterialScalars ms, const float* gF9, const float* gS9,
                                       float* g_mu, float* g_lam, float* g_ys, float* gFt9, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    M3 Ft, gF, gS;
    for (int i = 0; i < 9; ++i) { Ft.m[i] = Ft9[9 * p + i]; gF.m[i] = gF9[9 * p + i]; gS.m[i] = gS9[9 * p + i]; }
    SpectralEval e;
    spectral_eval(Ft, mu[p], lam[p], ys[p], dt, ms, e);
    const SpectralGrad g = spectral_adjoint(e, gF, gS, g_mu[p], g_lam[p], g_ys[p]);
    for (int i = 0; i < 9; ++i) gFt9[9 * p + i] = g.gFt.m[i];
    g_mu[p] = g.g_mu;
    g_lam[p] = g.g_lam;
    g_ys[p] = g.g_ys;
}

// Adjoint state between the caller's order and cell order: to_sorted gathers
// dst[i] = src[pid[i]]; otherwise scatters dst[pid[i]] = src[i].
struct GradPermuteArgs {
    ParticleArrays src, dst;
    const float* s_mu; const float* s_lam; const float* s_ys; const float* s_mass;
    float* d_mu; float* d_lam; float* d_ys; float* d_mass;
    const int* pid;
    int n;
    int to_sorted;
};

__global__ void k_permute_grad(const GradPermuteArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int u = __ldg(a.pid + i);
    const int s = a.to_sorted ? u : i;
    const int d = a.to_sorted ? i : u;
    a.dst.x[d] = __ldg(a.src.x + s);
    a.dst.v[d] = __ldg(a.src.v + s);
    f9_store(a.dst.C, d, f9_load(a.src.C, s));
    f9_store(a.dst.F, d, f9_load(a.src.F, s));
    a.d_mu[d] = __ldg(a.s_mu + s);
    a.d_lam[d] = __ldg(a.s_lam + s);
    a.d_ys[d] = __ldg(a.s_ys + s);
    a.d_mass[d] = __ldg(a.s_mass + s);
}

}  // namespace

// packed x4 | v4 | C | F state at base (the layout of particle_arrays(float*, n))
static EmpmParticles packed_particles(float* base, int n) {
    const size_t np = padded4(n);
    EmpmParticles p;
    p.x = base;
    p.v = base + 4 * np;
    p.C = base + 8 * np;
    p.F = base + 17 * np;
    return p;
}

static int ensure_adjoint_buffers(EmpmCtx* ctx, int n_steps) {
    AdjointBuffers& ab = ctx->adj;
    if (ab.gacc && (ab.cap_n < ctx->n_particles || ab.cap_blocks < ctx->nblocks)) {
        CK(cudaDeviceSynchronize(), "sync before adjoint buffer growth");
        free_adjoint(ab);
    }
    const size_t np = padded4(ctx->cap_particles);
    if (!ab.gacc) {
        ctx->epoch++;
        const size_t grid_bytes = (size_t)ctx->cap_blocks * 64 * sizeof(float4);
        ab.cap_n = ctx->cap_particles;
        ab.cap_blocks = ctx->cap_blocks;
        CK(cudaMalloc(&ab.gacc, grid_bytes), "adjoint grid");
        CK(cudaMalloc(&ab.gmom, grid_bytes), "adjoint grid");
        CK(cudaMemset(ab.gacc, 0, grid_bytes), "adjoint grid");
        CK(cudaMalloc(&ab.work, 3 * np * sizeof(float)), "adjoint material");
        CK(cudaMalloc(&ab.fe, 9 * np * sizeof(float)), "adjoint elastic F");
        CK(cudaMalloc(&ab.gfe, 9 * np * sizeof(float)), "adjoint elastic F");
        CK(cudaMalloc(&ab.gx, np * sizeof(float4)), "adjoint x");
        CK(cudaMalloc(&ab.gstate, 26 * np * sizeof(float)), "adjoint state");
        CK(cudaMalloc(&ab.gmats, 4 * np * sizeof(float)), "adjoint material");
    }
    if (n_steps > ab.capacity) {
        ctx->epoch++;
        if (ab.states) CK(cudaDeviceSynchronize(), "sync before adjoint buffer growth");
        if (ab.states) cudaFree(ab.states);
        if (ab.mats) cudaFree(ab.mats);
        ab.states = nullptr;
        ab.mats = nullptr;
        ab.capacity = 0;
        CK(cudaMalloc(&ab.states, (size_t)(n_steps + 1) * 26 * np * sizeof(float)), "adjoint segment states");
        CK(cudaMalloc(&ab.mats, (size_t)n_steps * 3 * np * sizeof(float)), "adjoint segment material");
        ab.capacity = n_steps;
    }
    if (ctx->adj_store && n_steps > ab.store_cap) {
        // the store is an optimisation: when it does not fit, the reverse
        // pass recomputes instead (free_store leaves store_cap at 0)
        if (ab.store_cap) CK(cudaDeviceSynchronize(), "sync before adjoint store growth");
        free_store(ab);
        ctx->epoch++;
        const size_t nb = (size_t)ab.cap_blocks;
        cudaError_t e = cudaMalloc(&ab.gsave, (size_t)n_steps * nb * 128 * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc(&ab.gsave_list, (size_t)n_steps * (nb + 1) * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&ab.fe_store, (size_t)n_steps * 9 * np * sizeof(float));
        if (e == cudaSuccess) {
            ab.store_cap = n_steps;
        } else {
            free_store(ab);
            if (e != cudaErrorMemoryAllocation) return empm_check_cuda(ctx, e, "adjoint store");
            cudaGetLastError();   // an allocation failure is not sticky; clear it
        }
    }
    return EMPM_OK;
}

// One forward substep on explicit particle arrays (the states of a segment).
static int launch_substep_arrays(EmpmCtx* ctx, const ParticleArrays& Pin, const ParticleArrays& Pout,
                                 const MaterialArrays& M, F9Planes Fe, int table, bool warpagg, cudaStream_t s) {
    const int n = ctx->n_particles;
    const Launch L = make_launch(ctx, table);
    timing_mark(ctx, 0, 0, s);
    if (warpagg) launch_p2g_warpagg(blocks_for(n, 256), 256, s, Pin, M, Fe, L, ctx->grid_mom, ctx->flags, ctx->seg_cap,
                                    uniform_material(ctx));
    else k_p2g_direct<<<blocks_for(n, 128), 128, 0, s>>>(Pin, M, Fe, L, ctx->grid_mom, ctx->flags);
    timing_mark(ctx, 0, 1, s);
    CK(cudaGetLastError(), "adjoint segment P2G");
    int rc = launch_grid_update(ctx, table, s);
    if (rc) return rc;
    timing_mark(ctx, 2, 0, s);
    k_g2p_direct<<<blocks_for(n, 128), 128, 0, s>>>(Pin, Fe, M, Pout, L, ctx->grid_vel);
    timing_mark(ctx, 2, 1, s);
    CK(cudaGetLastError(), "adjoint segment G2P");
    return EMPM_OK;
}

// Where a segment's forward data lives, for its reverse pass: the state
// before every substep, mu / lam / yield snapshots, and with the store each
// substep's touched grid blocks and elastic F; vol, selection and caller
// index in the order the segment runs in.
struct SegmentData {
    int n = 0, n_steps = 0;
    size_t np = 0;
    bool sorted = false;
    bool store = false;
    float* states = nullptr;   // (n_steps + 1) packed states
    float* mats = nullptr;     // n_steps x (mu | lam | yield)
    float4* gsave = nullptr;   // n_steps x cap_blocks x 128 float4
    int* glist = nullptr;      // n_steps x (1 + cap_blocks)
    float* fe = nullptr;       // n_steps x f9 planes
    size_t cap_blocks = 0;     // grid blocks per substep slot
    int* max_count = nullptr;  // running maximum of the touched-block counts, or NULL
    const EmpmStep* steps = nullptr;   // device step tables: [n_steps) as run, [n_steps, 2 n_steps) for recomputing
    MaterialArrays base;
};

// Forward over the segment from d.states[0] with mu / lam / yield in the
// adjoint work arrays (updated in place), keeping the state before every
// substep and the material snapshots. The last substep runs too, although
// the state after it is only needed by the caller: its P2G writes the
// velocity modifiers into that substep's stored velocities, which the reverse
// pass reads. With the store, P2G writes each substep's elastic F straight
// into its store slot and the grid update saves the touched grid blocks; on
// the sorted path (run cap 4, EMPM_OPT_FUSE) every substep after the first
// runs its stress + P2G in one kernel with the previous substep's G2P
// (k_g2p2g_store), which writes the stored state and snapshot itself.
static int segment_forward(EmpmCtx* ctx, const SegmentData& d, cudaStream_t s) {
    AdjointBuffers& ab = ctx->adj;
    const int n = d.n;
    const size_t np = d.np;
    const size_t state_floats = 26 * np;
    MaterialArrays Mw = d.base;
    Mw.mu = ab.work;
    Mw.lam = ab.work + np;
    Mw.ys = ab.work + 2 * np;
    const F9Planes Fe = f9_planes(ab.fe, n);
    // sorted stored segments: from the second substep on, the G2P of the
    // previous substep and the stress + P2G of this one run as one kernel
    // that writes the stored state, snapshot and elastic F itself
    const bool fused = d.store && d.sorted && ctx->fuse && ctx->seg_cap == 4 && d.n_steps > 1;
    for (int k = 0; k < d.n_steps; ++k) {
        const ParticleArrays Pin = particle_arrays(d.states + (size_t)k * state_floats, n);
        const ParticleArrays Pout = particle_arrays(d.states + (size_t)(k + 1) * state_floats, n);
        if (!d.store) {
            CK(cudaMemcpyAsync(d.mats + (size_t)k * 3 * np, ab.work, 3 * np * sizeof(float), cudaMemcpyDeviceToDevice,
                               s), "snapshot");
            const int rc = launch_substep_arrays(ctx, Pin, Pout, Mw, Fe, k, d.sorted, s);
            if (rc) return rc;
            continue;
        }
        const F9Planes Fk = f9_planes(d.fe + (size_t)k * 9 * np, n);
        const Launch Lk = make_launch_on(ctx, d.steps, k);
        if (fused && k > 0) {
            SegmentStoreArgs sa;
            sa.prev = particle_arrays(d.states + (size_t)(k - 1) * state_floats, n);
            sa.fe_prev = f9_planes(d.fe + (size_t)(k - 1) * 9 * np, n);
            sa.cur = Pin;
            sa.fe_cur = Fk;
            sa.snap = d.mats + (size_t)k * 3 * np;
            sa.np = (long long)np;
            timing_mark(ctx, 6, 0, s);
            const int tp = particle_threads(ctx, n, 256);
            launch_g2p2g_store(blocks_for(n, tp), tp, s, Mw, Lk, k - 1, ctx->grid_vel, ctx->grid_mom, ctx->flags, sa,
                               ctx->seg_cap, uniform_material(ctx), tp < 256);
            timing_mark(ctx, 6, 1, s);
            CK(cudaGetLastError(), "k_g2p2g_store");
        } else {
            CK(cudaMemcpyAsync(d.mats + (size_t)k * 3 * np, ab.work, 3 * np * sizeof(float), cudaMemcpyDeviceToDevice,
                               s), "snapshot");
            timing_mark(ctx, 0, 0, s);
            if (d.sorted) launch_p2g_warpagg(blocks_for(n, 256), 256, s, Pin, Mw, Fk, Lk, ctx->grid_mom, ctx->flags,
                                             ctx->seg_cap, uniform_material(ctx));
            else k_p2g_direct<<<blocks_for(n, 128), 128, 0, s>>>(Pin, Mw, Fk, Lk, ctx->grid_mom, ctx->flags);
            timing_mark(ctx, 0, 1, s);
            CK(cudaGetLastError(), "adjoint segment P2G");
        }
        // the grid update stores the touched blocks as it goes, and clears the
        // accumulator and the touched flags as for a plain substep
        timing_mark(ctx, 1, 0, s);
        GridStoreSlot slot;
        slot.blocks = d.gsave + (size_t)k * d.cap_blocks * 128;
        slot.list = d.glist + (size_t)k * (d.cap_blocks + 1);
        slot.cap = (int)d.cap_blocks;
        slot.max_count = d.max_count;
        const int rc = launch_grid_update_list<false>(ctx, Lk, s, &slot);
        if (rc) return rc;
        timing_mark(ctx, 1, 1, s);
        if (fused && k + 1 < d.n_steps) continue;   // the next fused kernel runs this G2P
        timing_mark(ctx, 2, 0, s);
        k_g2p_direct<<<blocks_for(n, 128), 128, 0, s>>>(Pin, Fk, Mw, Pout, Lk, ctx->grid_vel);
        timing_mark(ctx, 2, 1, s);
        CK(cudaGetLastError(), "adjoint segment G2P");
    }
    return EMPM_OK;
}

// The reverse pass: for each substep from the last, its grid (restored from
// the store, or recomputed from the stored state with the step tables
// [n_steps, 2 n_steps) that omit the velocity modifiers), then the three
// adjoint kernels (segment_reverse_unpermute then takes the adjoint back into
// the caller's order). Gp / gm_*: the incoming adjoint in the segment's order
// (updated in place).
static int segment_reverse(EmpmCtx* ctx, const SegmentData& d, ParticleArrays Gp, float* gm_mu, float* gm_lam,
                           float* gm_ys, float* gm_mass, cudaStream_t s) {
    AdjointBuffers& ab = ctx->adj;
    const int n = d.n, n_steps = d.n_steps;
    const size_t np = d.np;
    const size_t state_floats = 26 * np;
    MaterialArrays Mw = d.base;
    Mw.mu = ab.work;
    Mw.lam = ab.work + np;
    Mw.ys = ab.work + 2 * np;
    const F9Planes Fe = f9_planes(ab.fe, n);
    const F9Planes gFe = f9_planes(ab.gfe, n);
    const int grid_ctas = ctx->sm_count * 8;
    long long nb = (ctx->nblocks + 3) / 4;
    if (nb > grid_ctas) nb = grid_ctas;
    for (int k = n_steps - 1; k >= 0; --k) {
        float* snap = d.mats + (size_t)k * 3 * np;
        const ParticleArrays Pk = particle_arrays(d.states + (size_t)k * state_floats, n);
        const Launch Lk = make_launch_on(ctx, d.steps, k);
        F9Planes Fk = Fe;
        const float4* slot = d.store ? d.gsave + (size_t)k * d.cap_blocks * 128 : nullptr;
        const int* slot_list = d.store ? d.glist + (size_t)k * (d.cap_blocks + 1) : nullptr;
        if (d.store) {
            Fk = f9_planes(d.fe + (size_t)k * 9 * np, n);
            // the grid adjoint of substep k + 1 restored this substep's velocities
            if (k == n_steps - 1) {
                k_restore_grid<<<grid_ctas, 256, 0, s>>>(ctx->grid_vel, slot, slot_list);
                CK(cudaGetLastError(), "k_restore_grid");
            }
        } else {
            CK(cudaMemcpyAsync(ab.work, snap, 3 * np * sizeof(float), cudaMemcpyDeviceToDevice, s),
               "restore snapshot");
            const Launch Lrec = make_launch_on(ctx, d.steps, n_steps + k);
            timing_mark(ctx, 0, 0, s);
            if (d.sorted) launch_p2g_warpagg(blocks_for(n, 256), 256, s, Pk, Mw, Fe, Lrec, ctx->grid_mom,
                                             ctx->flags, ctx->seg_cap, uniform_material(ctx));
            else k_p2g_direct<<<blocks_for(n, 128), 128, 0, s>>>(Pk, Mw, Fe, Lrec, ctx->grid_mom, ctx->flags);
            timing_mark(ctx, 0, 1, s);
            CK(cudaGetLastError(), "P2G (adjoint recompute)");
            timing_mark(ctx, 1, 0, s);
            const int rc = launch_grid_update_list<true>(ctx, Lrec, s);
            timing_mark(ctx, 1, 1, s);
            if (rc) return rc;
        }
        AdjG2PArgs ag;
        ag.P = Pk;
        ag.x_next = particle_arrays(d.states + (size_t)(k + 1) * state_floats, n).x;
        ag.Fe = Fk;
        ag.M = Mw;
        ag.Gn = Gp;
        ag.L = Lk;
        ag.vel = ctx->grid_vel;
        ag.gacc = ab.gacc;
        ag.gx = ab.gx;
        ag.gFe = gFe;
        ag.seg_cap = ctx->seg_cap;
        timing_mark(ctx, 3, 0, s);
        if (ag.seg_cap == 4)
            k_adj_g2p<2><<<blocks_for(n, 128), 128, 0, s>>>(ag);
        else
            k_adj_g2p<5><<<blocks_for(n, 128), 128, 0, s>>>(ag);
        timing_mark(ctx, 3, 1, s);
        CK(cudaGetLastError(), "k_adj_g2p");
        AdjGridArgs gg;
        gg.mom = ctx->grid_mom;
        gg.gacc = ab.gacc;
        gg.gmom = ab.gmom;
        gg.flags = ctx->flags;
        gg.L = Lk;
        timing_mark(ctx, 4, 0, s);
        if (d.store) {
            const float4* rslot = k > 0 ? d.gsave + (size_t)(k - 1) * d.cap_blocks * 128 : nullptr;
            const int* rlist = k > 0 ? d.glist + (size_t)(k - 1) * (d.cap_blocks + 1) : nullptr;
            k_adj_grid_stored<<<grid_ctas, 256, 0, s>>>(gg, slot, slot_list, ctx->grid_vel, rslot, rlist);
        }
        else k_adj_grid<<<(int)nb, 256, 0, s>>>(gg);
        timing_mark(ctx, 4, 1, s);
        CK(cudaGetLastError(), "k_adj_grid");
        AdjP2GArgs ap;
        ap.P = Pk;
        ap.M = Mw;
        ap.M.mu = snap;
        ap.M.lam = snap + np;
        ap.M.ys = snap + 2 * np;
        ap.L = Lk;
        ap.gmom = ab.gmom;
        ap.gx = ab.gx;
        ap.gFe = gFe;
        ap.G = Gp;
        ap.g_mu = gm_mu;
        ap.g_lam = gm_lam;
        ap.g_ys = gm_ys;
        ap.g_mass = gm_mass;
        timing_mark(ctx, 5, 0, s);
        switch (uniform_material(ctx)) {
            case 5: k_adj_p2g<5><<<blocks_for(n, 128), 128, 0, s>>>(ap); break;
            case 0: k_adj_p2g<0><<<blocks_for(n, 128), 128, 0, s>>>(ap); break;
            default: k_adj_p2g<-1><<<blocks_for(n, 128), 128, 0, s>>>(ap); break;
        }
        timing_mark(ctx, 5, 1, s);
        CK(cudaGetLastError(), "k_adj_p2g");
    }
    return EMPM_OK;
}

// The adjoint of a sorted segment back into the caller's order.
static int segment_reverse_unpermute(EmpmCtx* ctx, const SegmentData& d, ParticleArrays Gp, float* gm_mu,
                                     float* gm_lam, float* gm_ys, float* gm_mass, EmpmParticles* grad,
                                     EmpmMaterialGrad* gmat, cudaStream_t s) {
    const int n = d.n;
    if (d.sorted) {
        GradPermuteArgs back;
        back.src = Gp;
        back.dst = particle_arrays(grad, n);
        back.s_mu = gm_mu; back.s_lam = gm_lam; back.s_ys = gm_ys; back.s_mass = gm_mass;
        back.d_mu = gmat->mu; back.d_lam = gmat->lam; back.d_ys = gmat->yield_stress; back.d_mass = gmat->mass;
        back.pid = d.base.pid;
        back.n = n;
        back.to_sorted = 0;
        k_permute_grad<<<blocks_for(n, 256), 256, 0, s>>>(back);
        CK(cudaGetLastError(), "k_permute_grad");
    }
    return EMPM_OK;
}

// Runs body(stream) for stream s: replayed from a cached graph (a stored
// segment's, or one of the context's for checkpointed segments) when its key
// still matches, captured first otherwise (on the context's own
// stream, joined to s by events, as the rollout graphs are). Kernel timing
// and EMPM_OPT_SEGMENT_GRAPH 0 run the body directly. A substep loop of a
// stored segment touches only the segment's and the context's buffers
// (unsorted reverse passes also the caller's, which are in the key), so one
// capture serves every later pass of a pooled segment.
template <typename Body>
static int run_segment_body(EmpmCtx* ctx, cudaGraphExec_t& exec, SegGraphKey& have, const SegGraphKey& want,
                            cudaStream_t s, Body body) {
    if (ctx->timing || !ctx->segment_graph) return body(s);
    if (!exec || memcmp(&have, &want, sizeof(want)) != 0) {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        CK(cudaStreamBeginCapture(ctx->own_stream, cudaStreamCaptureModeThreadLocal), "begin segment capture");
        const int rc = body(ctx->own_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->own_stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        CK(e, "end segment capture");
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            exec = nullptr;
            return empm_check_cuda(ctx, e, "segment graph instantiate");
        }
        have = want;
    }
    CK(cudaEventRecord(ctx->ev_a, s), "record");
    CK(cudaStreamWaitEvent(ctx->own_stream, ctx->ev_a, 0), "wait");
    CK(cudaGraphLaunch(exec, ctx->own_stream), "segment graph launch");
    CK(cudaEventRecord(ctx->ev_b, ctx->own_stream), "record");
    CK(cudaStreamWaitEvent(s, ctx->ev_b, 0), "wait");
    return EMPM_OK;
}

static SegGraphKey segment_key(const EmpmCtx* ctx) {
    SegGraphKey k;
    memset(&k, 0, sizeof(k));
    k.epoch = ctx->epoch;
    k.params_version = ctx->params_version;
    k.seg_cap = ctx->seg_cap;
    k.p2g_mode = ctx->p2g_mode;
    k.sort_every = ctx->sort_every;
    k.n = ctx->n_particles;
    return k;
}

extern "C" int empm_adjoint_segment(EmpmCtx* ctx, const EmpmParticles* ckpt, const float* ckpt_mu,
                                    const float* ckpt_lam, const float* ckpt_yield, const EmpmMaterial* mat,
                                    const EmpmStep* steps, int n_steps, EmpmParticles* grad,
                                    EmpmMaterialGrad* gmat, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, ckpt, "ckpt");
    if (!rc) rc = check_particles(ctx, grad, "grad");
    if (rc) return rc;
    if (!ckpt_mu || !ckpt_lam || !ckpt_yield)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "checkpoint mu / lam / yield pointer is NULL");
    if (!mat || !mat->vol) return empm_set_error(ctx, EMPM_ERR_INVALID, "mat or mat->vol is NULL");
    if (!gmat || !gmat->mu || !gmat->lam || !gmat->yield_stress || !gmat->mass)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "material gradient pointer is NULL");
    if (n_steps < 1 || n_steps > 100000)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d out of [1, 100000]", n_steps);
    if (!steps) return empm_set_error(ctx, EMPM_ERR_INVALID, "steps is NULL");
    for (size_t e = 0; e < (size_t)n_steps * ctx->n_inst; ++e)
        if (steps[e].hold) return empm_set_error(ctx, EMPM_ERR_UNSUPPORTED, "held substeps cannot be differentiated");
    const int n = ctx->n_particles;
    cudaStream_t s = (cudaStream_t)stream;
    // tables [0, n_steps): as given. [n_steps, 2 n_steps): the same without the
    // velocity modifiers, for recomputing a substep from a stored state whose
    // velocities already include them.
    AdjointBuffers& ab = ctx->adj;
    const size_t per = (size_t)n_steps * ctx->n_inst;
    ab.tables.assign(steps, steps + per);
    ab.tables.insert(ab.tables.end(), steps, steps + per);
    for (size_t t = per; t < 2 * per; ++t) ab.tables[t].n_modifiers = 0;
    rc = upload_steps(ctx, ab.tables.data(), 2 * n_steps, s);
    if (rc) return rc;
    if (n == 0) return EMPM_OK;
    rc = ensure_adjoint_buffers(ctx, n_steps);
    if (rc) return rc;

    ctx->resident = false;   // the sort below reuses the rollout's sorted buffers
    const size_t np = padded4(n);
    const size_t state_floats = 26 * np;
    float* mu_w = ab.work;
    float* lam_w = ab.work + np;
    float* ys_w = ab.work + 2 * np;
    const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;

    // 1. the checkpoint as segment state 0: in cell order when the context
    //    sorts (the whole segment then runs in that order), else as given
    const bool sorted = ctx->sort_every > 0;
    MaterialArrays base;
    base.vol = mat->vol;
    base.mu = base.lam = base.ys = nullptr;
    base.sel = mat->selection;
    base.pid = nullptr;
    ParticleArrays Gp = particle_arrays(grad, n);
    float* gm_mu = gmat->mu;
    float* gm_lam = gmat->lam;
    float* gm_ys = gmat->yield_stress;
    float* gm_mass = gmat->mass;
    GradPermuteArgs perm;
    if (sorted) {
        rc = ensure_sorted_buffers(ctx);
        if (rc) return rc;
        SortedState ss;
        const ParticleArrays ua = particle_arrays(ckpt, n);
        EmpmMaterial um = *mat;
        um.mu = const_cast<float*>(ckpt_mu);
        um.lam = const_cast<float*>(ckpt_lam);
        um.yield_stress = const_cast<float*>(ckpt_yield);
        um.F_elastic = nullptr;   // not an input of a segment (its P2G recomputes it)
        rc = launch_sort(ctx, ss, &ua, &um, s);
        if (rc) return rc;
        CK(cudaMemcpyAsync(ab.states, ctx->sb.part[ss.pc], state_floats * sizeof(float), d2d, s), "sorted checkpoint");
        const MaterialArrays SM = sorted_material(ctx, ss.mc);
        CK(cudaMemcpyAsync(mu_w, SM.mu, sizeof(float) * n, d2d, s), "sorted checkpoint");
        CK(cudaMemcpyAsync(lam_w, SM.lam, sizeof(float) * n, d2d, s), "sorted checkpoint");
        CK(cudaMemcpyAsync(ys_w, SM.ys, sizeof(float) * n, d2d, s), "sorted checkpoint");
        base.vol = SM.vol;
        base.sel = SM.sel;
        base.pid = SM.pid;
        // incoming adjoint into cell order
        const EmpmParticles gs = packed_particles(ab.gstate, n);
        perm.src = Gp;
        perm.dst = particle_arrays(&gs, n);
        perm.s_mu = gmat->mu; perm.s_lam = gmat->lam; perm.s_ys = gmat->yield_stress; perm.s_mass = gmat->mass;
        gm_mu = ab.gmats;
        gm_lam = ab.gmats + np;
        gm_ys = ab.gmats + 2 * np;
        gm_mass = ab.gmats + 3 * np;
        perm.d_mu = gm_mu; perm.d_lam = gm_lam; perm.d_ys = gm_ys; perm.d_mass = gm_mass;
        perm.pid = SM.pid;
        perm.n = n;
        perm.to_sorted = 1;
        k_permute_grad<<<blocks_for(n, 256), 256, 0, s>>>(perm);
        CK(cudaGetLastError(), "k_permute_grad");
        Gp = perm.dst;
    } else {
        const EmpmParticles s0 = packed_particles(ab.states, n);
        CK(cudaMemcpyAsync(s0.x, ckpt->x, sizeof(float4) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.v, ckpt->v, sizeof(float4) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.C, ckpt->C, 9 * sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.F, ckpt->F, 9 * sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(mu_w, ckpt_mu, sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(lam_w, ckpt_lam, sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(ys_w, ckpt_yield, sizeof(float) * n, d2d, s), "copy checkpoint");
    }
    SegmentData d;
    d.n = n;
    d.n_steps = n_steps;
    d.np = np;
    d.sorted = sorted;
    d.store = ab.store_cap >= n_steps;
    d.states = ab.states;
    d.mats = ab.mats;
    d.gsave = ab.gsave;
    d.glist = ab.gsave_list;
    d.fe = ab.fe_store;
    d.cap_blocks = (size_t)ab.cap_blocks;
    d.steps = ctx->d_steps;
    d.base = base;
    // the re-run and the reverse pass replay a graph captured by an earlier
    // call with the same key: on the sorted path they touch only the
    // context's buffers; on the caller-order path the caller's material and
    // adjoint arrays are part of the key
    SegGraphKey key = segment_key(ctx);
    key.n_steps = n_steps;
    key.store = d.store ? 1 : 0;
    if (!sorted) {
        const void* b[10] = {mat->vol, mat->selection, grad->x, grad->v, grad->C, grad->F,
                             gmat->mu, gmat->lam, gmat->yield_stress, gmat->mass};
        memcpy(key.buf, b, sizeof(b));
    }
    AdjSegGraph* g = &ctx->adj_graphs[0];
    for (AdjSegGraph& e : ctx->adj_graphs) {
        if (e.exec && memcmp(&e.key, &key, sizeof(key)) == 0) { g = &e; break; }
        if (e.used < g->used) g = &e;
    }
    g->used = ++ctx->graph_clock;
    rc = run_segment_body(ctx, g->exec, g->key, key, s, [&](cudaStream_t bs) {
        int r = segment_forward(ctx, d, bs);
        if (!r) r = segment_reverse(ctx, d, Gp, gm_mu, gm_lam, gm_ys, gm_mass, bs);
        return r;
    });
    if (rc) return rc;
    return segment_reverse_unpermute(ctx, d, Gp, gm_mu, gm_lam, gm_ys, gm_mass, grad, gmat, s);
}

// ---------------------------------------------------------------------------
// stored segments: the forward keeps what the reverse pass needs
// ---------------------------------------------------------------------------
static size_t segment_bytes(size_t np, size_t cap_blocks, int n_steps) {
    const size_t k = (size_t)n_steps;
    return ((k + 1) * 26 * np + k * 3 * np + k * 9 * np + np) * sizeof(float) + 2 * np * sizeof(int) +
           k * cap_blocks * 128 * sizeof(float4) + k * (cap_blocks + 1) * sizeof(int);
}

static size_t segment_bytes(const EmpmCtx* ctx, size_t np, size_t cap_blocks, int n_steps) {
    return segment_bytes(np, cap_blocks, n_steps) + (size_t)n_steps * ctx->n_inst * sizeof(EmpmStep) + sizeof(int);
}

static void segment_free(EmpmSegment* seg) {
    void* ptrs[] = {seg->states, seg->mats, seg->gsave, seg->glist, seg->fe, seg->vol, seg->sel, seg->pid,
                    seg->max_count, seg->d_tables};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (seg->fwd_exec) cudaGraphExecDestroy(seg->fwd_exec);
    if (seg->rev_exec) cudaGraphExecDestroy(seg->rev_exec);
    seg->fwd_exec = seg->rev_exec = nullptr;
    seg->d_tables = nullptr;
    seg->tables_on_device = false;
    seg->states = seg->mats = seg->fe = seg->vol = nullptr;
    seg->gsave = nullptr;
    seg->glist = seg->sel = seg->pid = seg->max_count = nullptr;
}

// block slots per substep: 0 (or more than the context has) means all of them
static size_t segment_block_cap(const EmpmCtx* ctx, int block_cap) {
    return (block_cap <= 0 || block_cap > ctx->cap_blocks) ? (size_t)ctx->cap_blocks : (size_t)block_cap;
}

extern "C" int empm_segment_bytes(EmpmCtx* ctx, int n_steps, int block_cap, size_t* out) {
    if (!ctx || !out) return empm_set_error(ctx, EMPM_ERR_INVALID, "ctx or out is NULL");
    if (n_steps < 1 || n_steps > 100000)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d out of [1, 100000]", n_steps);
    *out = segment_bytes(ctx, padded4(ctx->n_particles), segment_block_cap(ctx, block_cap), n_steps);
    return EMPM_OK;
}

extern "C" int empm_segment_create(EmpmCtx* ctx, int n_steps, int block_cap, EmpmSegment** out) {
    if (!ctx || !out) return empm_set_error(ctx, EMPM_ERR_INVALID, "ctx or out is NULL");
    *out = nullptr;
    if (n_steps < 1 || n_steps > 100000)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d out of [1, 100000]", n_steps);
    EmpmSegment* seg = new EmpmSegment();
    seg->ctx = ctx;
    seg->n = ctx->n_particles;
    seg->n_steps = n_steps;
    seg->n_inst = ctx->n_inst;
    seg->np = padded4(ctx->n_particles);
    seg->cap_blocks = (size_t)ctx->cap_blocks;
    seg->block_cap = segment_block_cap(ctx, block_cap);
    const size_t np = seg->np, k = (size_t)n_steps, nb = seg->block_cap;
    cudaError_t e = cudaMalloc(&seg->states, (k + 1) * 26 * np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&seg->mats, k * 3 * np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&seg->fe, k * 9 * np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&seg->gsave, k * nb * 128 * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&seg->glist, k * (nb + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&seg->vol, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&seg->sel, np * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&seg->pid, np * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&seg->max_count, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&seg->d_tables, k * (size_t)ctx->n_inst * sizeof(EmpmStep));
    if (e != cudaSuccess) {
        segment_free(seg);
        delete seg;
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();   // an allocation failure is not sticky; clear it
            return empm_set_error(ctx, EMPM_ERR_OOM, "segment store of %d substeps (%zu bytes) does not fit", n_steps,
                                  segment_bytes(ctx, np, nb, n_steps));
        }
        return empm_check_cuda(ctx, e, "segment store");
    }
    *out = seg;
    return EMPM_OK;
}

extern "C" int empm_segment_destroy(EmpmSegment* seg) {
    if (!seg) return EMPM_OK;
    segment_free(seg);
    delete seg;
    return EMPM_OK;
}

static int check_segment(EmpmCtx* ctx, const EmpmSegment* seg) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    if (!seg) return empm_set_error(ctx, EMPM_ERR_INVALID, "segment is NULL");
    if (seg->ctx != ctx) return empm_set_error(ctx, EMPM_ERR_INVALID, "segment belongs to another context");
    if (seg->n != ctx->n_particles || seg->n_inst != ctx->n_inst || seg->cap_blocks != (size_t)ctx->cap_blocks)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "segment was made for %d particles, %d instances, %zu blocks; "
                              "the context now has %d, %d, %lld", seg->n, seg->n_inst, seg->cap_blocks,
                              ctx->n_particles, ctx->n_inst, (long long)ctx->cap_blocks);
    return EMPM_OK;
}

static SegmentData segment_data(const EmpmSegment* seg) {
    SegmentData d;
    d.n = seg->n;
    d.n_steps = seg->n_steps;
    d.np = seg->np;
    d.sorted = seg->sorted;
    d.store = true;
    d.states = seg->states;
    d.mats = seg->mats;
    d.gsave = seg->gsave;
    d.glist = seg->glist;
    d.fe = seg->fe;
    d.cap_blocks = seg->block_cap;
    d.max_count = seg->max_count;
    d.steps = seg->d_tables;
    d.base.vol = seg->vol;
    d.base.mu = d.base.lam = d.base.ys = nullptr;
    d.base.sel = seg->has_sel ? seg->sel : nullptr;
    d.base.pid = seg->sorted ? seg->pid : nullptr;
    return d;
}

extern "C" int empm_segment_forward(EmpmCtx* ctx, EmpmSegment* seg, const EmpmParticles* ckpt, const float* ckpt_mu,
                                    const float* ckpt_lam, const float* ckpt_yield, const EmpmMaterial* mat,
                                    const EmpmStep* steps, int n_steps, EmpmParticles* out, void* stream) {
    int rc = check_segment(ctx, seg);
    if (!rc) rc = check_particles(ctx, ckpt, "ckpt");
    if (!rc) rc = check_particles(ctx, out, "out");
    if (!rc) rc = check_material(ctx, mat);
    if (rc) return rc;
    if (!ckpt_mu || !ckpt_lam || !ckpt_yield)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "checkpoint mu / lam / yield pointer is NULL");
    if (n_steps != seg->n_steps)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "n_steps %d, the segment holds %d", n_steps, seg->n_steps);
    if (!steps) return empm_set_error(ctx, EMPM_ERR_INVALID, "steps is NULL");
    const size_t per = (size_t)n_steps * ctx->n_inst;
    rc = check_steps(ctx, steps, n_steps);
    if (rc) return rc;
    for (size_t e = 0; e < per; ++e)
        if (steps[e].hold) return empm_set_error(ctx, EMPM_ERR_UNSUPPORTED, "held substeps cannot be differentiated");
    cudaStream_t s = (cudaStream_t)stream;
    seg->ready = false;
    seg->checked = false;
    seg->max_touched = 0;
    // the segment keeps its own device copy of its step tables (uploaded only
    // when they change), so its captured substep loop can be replayed as is
    if (!seg->tables_on_device || seg->tables.size() != per ||
        memcmp(seg->tables.data(), steps, per * sizeof(EmpmStep)) != 0) {
        seg->tables.assign(steps, steps + per);
        seg->tables_on_device = false;
        CK(cudaMemcpyAsync(seg->d_tables, seg->tables.data(), per * sizeof(EmpmStep), cudaMemcpyHostToDevice, s),
           "segment step tables");
        seg->tables_on_device = true;
    }
    const int n = seg->n;
    if (n == 0) {
        seg->ready = true;
        return EMPM_OK;
    }
    rc = ensure_adjoint_buffers(ctx, 0);
    if (rc) return rc;
    AdjointBuffers& ab = ctx->adj;
    const size_t np = seg->np;
    const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;
    CK(cudaMemsetAsync(seg->max_count, 0, sizeof(int), s), "reset touched-block maximum");
    ctx->resident = false;   // a sort here reuses the rollout's sorted buffers
    seg->sorted = ctx->sort_every > 0;
    seg->has_sel = seg->sorted || mat->selection != nullptr;
    if (seg->sorted) {
        rc = ensure_sorted_buffers(ctx);
        if (rc) return rc;
        SortedState ss;
        const ParticleArrays ua = particle_arrays(ckpt, n);
        EmpmMaterial um = *mat;
        um.mu = const_cast<float*>(ckpt_mu);
        um.lam = const_cast<float*>(ckpt_lam);
        um.yield_stress = const_cast<float*>(ckpt_yield);
        um.F_elastic = nullptr;   // not an input of a segment (its P2G recomputes it)
        rc = launch_sort(ctx, ss, &ua, &um, s);
        if (rc) return rc;
        CK(cudaMemcpyAsync(seg->states, ctx->sb.part[ss.pc], 26 * np * sizeof(float), d2d, s), "sorted checkpoint");
        const MaterialArrays SM = sorted_material(ctx, ss.mc);
        CK(cudaMemcpyAsync(ab.work, SM.mu, sizeof(float) * n, d2d, s), "sorted checkpoint");
        CK(cudaMemcpyAsync(ab.work + np, SM.lam, sizeof(float) * n, d2d, s), "sorted checkpoint");
        CK(cudaMemcpyAsync(ab.work + 2 * np, SM.ys, sizeof(float) * n, d2d, s), "sorted checkpoint");
        CK(cudaMemcpyAsync(seg->vol, SM.vol, sizeof(float) * n, d2d, s), "sorted material");
        CK(cudaMemcpyAsync(seg->sel, SM.sel, sizeof(int) * n, d2d, s), "sorted material");
        CK(cudaMemcpyAsync(seg->pid, SM.pid, sizeof(int) * n, d2d, s), "sorted material");
    } else {
        const EmpmParticles s0 = packed_particles(seg->states, n);
        CK(cudaMemcpyAsync(s0.x, ckpt->x, sizeof(float4) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.v, ckpt->v, sizeof(float4) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.C, ckpt->C, 9 * sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(s0.F, ckpt->F, 9 * sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(ab.work, ckpt_mu, sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(ab.work + np, ckpt_lam, sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(ab.work + 2 * np, ckpt_yield, sizeof(float) * n, d2d, s), "copy checkpoint");
        CK(cudaMemcpyAsync(seg->vol, mat->vol, sizeof(float) * n, d2d, s), "copy material");
        if (seg->has_sel) CK(cudaMemcpyAsync(seg->sel, mat->selection, sizeof(int) * n, d2d, s), "copy material");
    }
    const SegmentData d = segment_data(seg);
    rc = run_segment_body(ctx, seg->fwd_exec, seg->fwd_key, segment_key(ctx), s,
                          [&](cudaStream_t bs) { return segment_forward(ctx, d, bs); });
    if (rc) return rc;
    // the state after the last substep, its elastic F and the updated
    // material scalars, in the caller's order
    float* last = seg->states + (size_t)n_steps * 26 * np;
    float* fe_last = seg->fe + (size_t)(n_steps - 1) * 9 * np;
    if (seg->sorted) {
        UnsortArgs u;
        u.src = particle_arrays(last, n);
        u.dst = particle_arrays(out, n);
        u.Fe_s = f9_planes(fe_last, n);
        u.Fe_d = f9_planes(mat->F_elastic, n);
        u.mu_s = ab.work; u.mu_d = mat->mu;
        u.lam_s = ab.work + np; u.lam_d = mat->lam;
        u.ys_s = ab.work + 2 * np; u.ys_d = mat->yield_stress;
        u.pid = seg->pid;
        u.n = n;
        k_unsort<<<blocks_for(n, 256), 256, 0, s>>>(u);
        CK(cudaGetLastError(), "k_unsort");
    } else {
        const EmpmParticles f = packed_particles(last, n);
        CK(cudaMemcpyAsync(out->x, f.x, sizeof(float4) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(out->v, f.v, sizeof(float4) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(out->C, f.C, 9 * sizeof(float) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(out->F, f.F, 9 * sizeof(float) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(mat->F_elastic, fe_last, 9 * sizeof(float) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(mat->mu, ab.work, sizeof(float) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(mat->lam, ab.work + np, sizeof(float) * n, d2d, s), "segment result");
        CK(cudaMemcpyAsync(mat->yield_stress, ab.work + 2 * np, sizeof(float) * n, d2d, s), "segment result");
    }
    seg->ready = true;
    return EMPM_OK;
}

extern "C" int empm_segment_blocks(EmpmSegment* seg, int* max_touched, int* block_cap, void* stream) {
    if (!seg) return empm_set_error(nullptr, EMPM_ERR_INVALID, "segment is NULL");
    EmpmCtx* ctx = seg->ctx;
    if (!seg->ready) return empm_set_error(ctx, EMPM_ERR_INVALID, "segment has no completed forward pass");
    if (!seg->checked) {
        int m = 0;
        if (seg->n > 0) {
            CK(cudaMemcpyAsync(&m, seg->max_count, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream),
               "read touched-block maximum");
            CK(cudaStreamSynchronize((cudaStream_t)stream), "read touched-block maximum");
        }
        seg->max_touched = m;
        seg->checked = true;
    }
    if (max_touched) *max_touched = seg->max_touched;
    if (block_cap) *block_cap = (int)seg->block_cap;
    return EMPM_OK;
}

extern "C" int empm_segment_reverse(EmpmCtx* ctx, EmpmSegment* seg, EmpmParticles* grad, EmpmMaterialGrad* gmat,
                                    void* stream) {
    int rc = check_segment(ctx, seg);
    if (!rc) rc = check_particles(ctx, grad, "grad");
    if (rc) return rc;
    if (!gmat || !gmat->mu || !gmat->lam || !gmat->yield_stress || !gmat->mass)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "material gradient pointer is NULL");
    if (!seg->ready) return empm_set_error(ctx, EMPM_ERR_INVALID, "segment has no completed forward pass");
    rc = empm_segment_blocks(seg, nullptr, nullptr, stream);
    if (rc) return rc;
    if ((size_t)seg->max_touched > seg->block_cap)
        return empm_set_error(ctx, EMPM_ERR_INVALID, "segment touched %d grid blocks in a substep, over its capacity "
                              "of %zu: make it with block_cap >= %d and run the forward pass again",
                              seg->max_touched, seg->block_cap, seg->max_touched);
    cudaStream_t s = (cudaStream_t)stream;
    const int n = seg->n;
    if (n == 0) return EMPM_OK;
    rc = ensure_adjoint_buffers(ctx, 0);
    if (rc) return rc;
    AdjointBuffers& ab = ctx->adj;
    const size_t np = seg->np;
    ParticleArrays Gp = particle_arrays(grad, n);
    float* gm_mu = gmat->mu;
    float* gm_lam = gmat->lam;
    float* gm_ys = gmat->yield_stress;
    float* gm_mass = gmat->mass;
    if (seg->sorted) {
        // incoming adjoint into the segment's cell order
        const EmpmParticles gs = packed_particles(ab.gstate, n);
        GradPermuteArgs perm;
        perm.src = Gp;
        perm.dst = particle_arrays(&gs, n);
        perm.s_mu = gmat->mu; perm.s_lam = gmat->lam; perm.s_ys = gmat->yield_stress; perm.s_mass = gmat->mass;
        gm_mu = ab.gmats;
        gm_lam = ab.gmats + np;
        gm_ys = ab.gmats + 2 * np;
        gm_mass = ab.gmats + 3 * np;
        perm.d_mu = gm_mu; perm.d_lam = gm_lam; perm.d_ys = gm_ys; perm.d_mass = gm_mass;
        perm.pid = seg->pid;
        perm.n = n;
        perm.to_sorted = 1;
        k_permute_grad<<<blocks_for(n, 256), 256, 0, s>>>(perm);
        CK(cudaGetLastError(), "k_permute_grad");
        Gp = perm.dst;
    }
    const SegmentData d = segment_data(seg);
    SegGraphKey key = segment_key(ctx);
    if (!seg->sorted) {   // the loop then works on the caller's adjoint arrays
        const void* b[8] = {grad->x, grad->v, grad->C, grad->F, gmat->mu, gmat->lam, gmat->yield_stress, gmat->mass};
        memcpy(key.buf, b, sizeof(b));
    }
    rc = run_segment_body(ctx, seg->rev_exec, seg->rev_key, key, s, [&](cudaStream_t bs) {
        return segment_reverse(ctx, d, Gp, gm_mu, gm_lam, gm_ys, gm_mass, bs);
    });
    if (rc) return rc;
    return segment_reverse_unpermute(ctx, d, Gp, gm_mu, gm_lam, gm_ys, gm_mass, grad, gmat, s);
}

extern "C" int empm_restart_F(EmpmCtx* ctx, EmpmParticles* p, const float* target, const int* selection,
                              float* cov, void* stream) {
    if (!ctx) return empm_set_error(nullptr, EMPM_ERR_INVALID, "ctx is NULL");
    int rc = check_particles(ctx, p, "particles");
    if (rc) return rc;
    if (!target) return empm_set_error(ctx, EMPM_ERR_INVALID, "target is NULL");
    const int n = ctx->n_particles;
    if (n == 0) return EMPM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const Launch L = make_launch(ctx, 0);
    const ParticleArrays P = particle_arrays(p, n);
    k_restart_p2g<<<blocks_for(n, 128), 128, 0, s>>>(P, target, selection, L, ctx->grid_mom, ctx->flags);
    CK(cudaGetLastError(), "k_restart_p2g");
    CK(cudaMemsetAsync(ctx->active, 0, sizeof(int), s), "reset touched-block count");
    k_collect_blocks<false><<<blocks_for(ctx->nblocks, 256), 256, 0, s>>>(ctx->flags, (int)ctx->nblocks, ctx->active,
                                                                          L);
    CK(cudaGetLastError(), "k_collect_blocks");
    k_restart_grid<<<ctx->sm_count * 8, 256, 0, s>>>(ctx->grid_mom, ctx->grid_vel, ctx->active);
    CK(cudaGetLastError(), "k_restart_grid");
    k_restart_g2p<<<blocks_for(n, 128), 128, 0, s>>>(P, target, selection, L, ctx->grid_vel, cov);
    CK(cudaGetLastError(), "k_restart_g2p");
    return EMPM_OK;
}

extern "C" int empm_prepare_adjoint(const float* E, const float* nu, const float* g_mu, const float* g_lam,
                                    float* g_E, float* g_nu, const float* vol, const float* g_mass,
                                    float* g_density, int n, void* stream) {
    EmpmCtx* ctx = nullptr;
    if (n < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "n < 0");
    const bool en = g_E || g_nu;
    if (en && !(E && nu && g_mu && g_lam && g_E && g_nu))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "E, nu, g_mu, g_lam, g_E, g_nu must all be given");
    if (g_density && !(vol && g_mass))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "vol and g_mass are needed for g_density");
    if (n == 0) return EMPM_OK;
    k_prepare_adjoint<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        E, nu, g_mu, g_lam, en ? g_E : nullptr, en ? g_nu : nullptr, vol, g_mass, g_density, n);
    CK(cudaGetLastError(), "k_prepare_adjoint");
    return EMPM_OK;
}

extern "C" int empm_debug_stress_adjoint(const EmpmModelParams* params, const float* F_trial9, const float* mu,
                                         const float* lam, const float* yield_stress, float dt, const float* g_F9,
                                         const float* g_stress9, float* g_mu, float* g_lam, float* g_yield,
                                         float* g_F_trial9, int n, void* stream) {
    EmpmCtx* ctx = nullptr;
    int rc = validate_params(nullptr, params);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!F_trial9 || !mu || !lam || !yield_stress || !g_F9 || !g_stress9 || !g_mu || !g_lam ||
                            !g_yield || !g_F_trial9)))
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad empm_debug_stress_adjoint arguments");
    if (n == 0) return EMPM_OK;
    MaterialScalars ms;
    ms.material = params->material;
    ms.softening = params->softening;
    ms.hardening = params->hardening;
    ms.xi = params->xi;
    ms.plastic_viscosity = params->plastic_viscosity;
    ms.alpha = params->alpha;
    k_debug_stress_adjoint<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
        F_trial9, mu, lam, yield_stress, dt, ms, g_F9, g_stress9, g_mu, g_lam, g_yield, g_F_trial9, n);
    CK(cudaGetLastError(), "k_debug_stress_adjoint");
    return EMPM_OK;
}

// ===========================================================================
// Allocation-free substep
// ===========================================================================
// For callers that cannot allocate device memory when they step the
// simulation. One example is a host application that reserves all of its
// device memory at start-up and then runs the simulator inside a
// fixed-budget control or rendering loop, where a cudaMalloc could stall the
// loop or fail. Another is code that runs while a memory pool owned by
// another framework must not grow. These callers still pass every input and
// output buffer. The grid scratch that a context would allocate comes from
// file-scope device arrays sized for grids up to
// EMPM_NOALLOC_MAX_GRID^3 nodes. Every GPU that loads the library holds
// them (8 MiB of grid plus a few KiB) until the process exits.

namespace {
constexpr int kNoallocNB = (EMPM_NOALLOC_MAX_GRID + 3) / 4;
constexpr long long kNoallocBlocks = (long long)kNoallocNB * kNoallocNB * kNoallocNB;
constexpr int kNoallocMaxDevices = 64;

__device__ __align__(256) float4 g_noalloc_grid[2 * kNoallocBlocks * 64];   // accumulator | velocities
__device__ __align__(256) unsigned char g_noalloc_flags[kNoallocBlocks];
__device__ __align__(256) InstanceConsts g_noalloc_inst[1];
__device__ __align__(256) EmpmStep g_noalloc_step[1];
__device__ __align__(256) unsigned g_noalloc_status[1];

// Writes the call's instance constants and schedule into the file-scope
// arrays (device code names them directly) and clears the status word it
// was given. Kernel arguments are copied when the launch is issued, so the
// host's structs may go out of scope at once and no pageable host-to-device
// copy (which would wait for the stream) is needed.
__global__ void k_noalloc_setup(const InstanceConsts ic, const EmpmStep st, unsigned* status, int clear_status) {
    g_noalloc_inst[0] = ic;
    g_noalloc_step[0] = st;
    if (clear_status) *status = 0u;
}

// Device addresses of the arrays above. In host code their names are host-side
// stand-ins, not device addresses, so the addresses are looked up once per
// device with cudaGetSymbolAddress while that device is current.
struct NoallocPtrs {
    bool           ready = false;
    float4*        grid = nullptr;
    unsigned char* flags = nullptr;
    InstanceConsts* inst = nullptr;
    EmpmStep*      step = nullptr;
    unsigned*      status = nullptr;
};
NoallocPtrs g_noalloc_ptrs[kNoallocMaxDevices];
std::mutex g_noalloc_mutex;

int noalloc_setup(int device, NoallocPtrs** out) {
    EmpmCtx* ctx = nullptr;
    if (device < 0 || device >= kNoallocMaxDevices)
        return empm_set_error(nullptr, EMPM_ERR_UNSUPPORTED, "device %d beyond the %d supported", device,
                              kNoallocMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocPtrs& p = g_noalloc_ptrs[device];
    if (!p.ready) {
        CK(cudaGetSymbolAddress((void**)&p.grid, g_noalloc_grid), "cudaGetSymbolAddress(grid)");
        CK(cudaGetSymbolAddress((void**)&p.flags, g_noalloc_flags), "cudaGetSymbolAddress(flags)");
        CK(cudaGetSymbolAddress((void**)&p.inst, g_noalloc_inst), "cudaGetSymbolAddress(instance)");
        CK(cudaGetSymbolAddress((void**)&p.step, g_noalloc_step), "cudaGetSymbolAddress(step)");
        CK(cudaGetSymbolAddress((void**)&p.status, g_noalloc_status), "cudaGetSymbolAddress(status)");
        p.ready = true;
    }
    *out = &p;
    return EMPM_OK;
}
}  // namespace

extern "C" int empm_substep_noalloc(const EmpmModelParams* params, const EmpmParticles* in, EmpmParticles* out,
                                    const EmpmMaterial* mat, const EmpmStep* step, int n_particles,
                                    uint32_t* status, void* stream) {
    EmpmCtx* ctx = nullptr;
    int rc = validate_params(nullptr, params);
    if (rc) return rc;
    if (params->n_grid > EMPM_NOALLOC_MAX_GRID)
        return empm_set_error(nullptr, EMPM_ERR_INVALID,
                              "n_grid %d exceeds the allocation-free maximum of %d (use a context for larger grids)",
                              params->n_grid, EMPM_NOALLOC_MAX_GRID);
    if (n_particles < 0) return empm_set_error(nullptr, EMPM_ERR_INVALID, "n_particles < 0");
    if (!step || step->n_colliders < 0 || step->n_colliders > EMPM_MAX_COLLIDERS || step->n_modifiers < 0 ||
        step->n_modifiers > EMPM_MAX_MODIFIERS)
        return empm_set_error(nullptr, EMPM_ERR_INVALID, "bad step schedule");
    rc = check_particles(nullptr, in, "in");
    if (!rc) rc = check_particles(nullptr, out, "out");
    if (!rc) rc = check_material(nullptr, mat);
    if (rc) return rc;
    if (particles_alias(in, out)) return empm_set_error(nullptr, EMPM_ERR_INVALID, "in and out must be distinct buffers");
    int device = 0;
    CK(cudaGetDevice(&device), "cudaGetDevice");
    NoallocPtrs* P = nullptr;
    rc = noalloc_setup(device, &P);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int NB = grid_nb(params->n_grid);
    const long long nblocks = (long long)NB * NB * NB;
    const InstanceConsts ic = instance_consts(*params, n_particles, 0, 0);
    // the arrays keep the previous call's contents: reset what must start at zero
    CK(cudaMemsetAsync(P->grid, 0, sizeof(float4) * (size_t)nblocks * 64, s), "clear grid scratch");
    CK(cudaMemsetAsync(P->flags, 0, (size_t)nblocks, s), "clear block flags");
    // the caller's status word accumulates across calls (the caller clears it);
    // the internal one is cleared every call
    unsigned* status_word = status ? reinterpret_cast<unsigned*>(status) : P->status;
    k_noalloc_setup<<<1, 1, 0, s>>>(ic, *step, status_word, status ? 0 : 1);
    CK(cudaGetLastError(), "k_noalloc_setup");
    Launch L;
    L.inst = P->inst;
    L.n_inst = 1;
    L.n_total = n_particles;
    L.nblocks = (int)nblocks;
    L.steps = P->step;
    L.table = 0;
    L.status = status_word;
    const ParticleArrays Pin = particle_arrays(in, n_particles);
    const ParticleArrays Pout = particle_arrays(out, n_particles);
    MaterialArrays M;
    M.vol = mat->vol;
    M.mu = mat->mu;
    M.lam = mat->lam;
    M.ys = mat->yield_stress;
    M.sel = mat->selection;
    M.pid = nullptr;
    const F9Planes Fe = f9_planes(mat->F_elastic, n_particles);
    float4* mom = P->grid;
    float4* vel = P->grid + nblocks * 64;
    if (n_particles > 0) {
        k_p2g_direct<<<blocks_for(n_particles, 128), 128, 0, s>>>(Pin, M, Fe, L, mom, P->flags);
        CK(cudaGetLastError(), "k_p2g_direct (allocation-free)");
    }
    GridUpdateArgs g;
    g.mom = mom;
    g.vel = vel;
    g.flags = P->flags;
    g.L = L;
    long long nb = (nblocks + 3) / 4;
    if (nb > 148 * 8) nb = 148 * 8;
    k_grid_update_sparse<<<(int)nb, 256, 0, s>>>(g);
    CK(cudaGetLastError(), "k_grid_update_sparse (allocation-free)");
    if (n_particles > 0) {
        k_g2p_direct<<<blocks_for(n_particles, 128), 128, 0, s>>>(Pin, Fe, M, Pout, L, vel);
        CK(cudaGetLastError(), "k_g2p_direct (allocation-free)");
    }
    return EMPM_OK;
}
