// ctx.hpp — the opaque EmpmCtx behind the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "../../include/empm_b200.h"

struct GraphKey {
    EmpmParticles a;
    EmpmParticles b;
    EmpmMaterial  mat;
    int           n_steps;
    int           sort_every;
    int           p2g_mode;
    int           g2p_tile;
    int           tile_cap;
};

// Particle and material buffers of the sorted path (cell-block order).
struct SortedBuffers {
    bool   allocated = false;
    int    n = 0;
    float* part[2] = {nullptr, nullptr};   // x4 | v4 | C f9 | F f9 per buffer (ping-pong per substep)
    float* fe = nullptr;                   // elastic F handed from P2G to G2P (f9)
    float* matf[2] = {nullptr, nullptr};   // vol | mu | lam | ys (ping-pong per sort)
    int*   mati[2] = {nullptr, nullptr};   // sel | pid
    int*   keys = nullptr;
    int*   ranks = nullptr;
    int*   counts = nullptr;               // [NB^3] particles per block, zero between sorts
    int*   offsets = nullptr;              // [NB^3] block start offsets
    int*   cell_counts = nullptr;          // [NB^3 * 64], zero between sorts
    int*   cell_offsets = nullptr;         // [NB^3 * 64]
    int2*  chunks = nullptr;               // [max_chunks]
    int*   nchunks = nullptr;
    int    max_chunks = 0;
};

struct EmpmCtx {
    EmpmModelParams params{};
    int          device = 0;
    int          sm_count = 148;
    int          n_particles = 0;
    int          max_steps = 0;
    int          NB = 0;                   // 4^3 node blocks per axis
    float4*      grid_mom = nullptr;       // P2G accumulation (px, py, pz, m), blocked layout; zero between substeps
    float4*      grid_vel = nullptr;       // node velocity after the grid update, blocked layout
    unsigned char* flags = nullptr;        // touched node blocks of the current substep
    EmpmStep*    d_steps = nullptr;        // device copy of the step schedule
    unsigned*    d_status = nullptr;       // EMPM_STATUS_* bits
    cudaStream_t own_stream = nullptr;     // capture stream for the graph path
    cudaEvent_t  ev_a = nullptr;
    cudaEvent_t  ev_b = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    GraphKey     graph_key{};
    bool         graph_valid = false;
    // launch options (empm_ctx_set_option)
    int          sort_every = 16;          // 0 = direct path for rollouts too
    int          p2g_mode = 2;             // 0 direct reductions, 1 shared-memory tile, 2 warp-aggregated
    int          g2p_tile = 1;
    int          tile_cap = 1024;          // nodes per shared-memory tile (16 B each)
    SortedBuffers sb;
    // per-kernel event timing (stream path only)
    bool         timing = false;
    int          timing_capacity = 0;
    int          timing_count[3] = {0, 0, 0};
    std::vector<cudaEvent_t> timing_events;   // [3][capacity][2]
    char         err[512] = {0};
};

int empm_set_error(EmpmCtx* ctx, int code, const char* fmt, ...);
int empm_check_cuda(EmpmCtx* ctx, cudaError_t e, const char* what);
