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
};

struct EmpmCtx {
    EmpmModelParams params{};
    int          device = 0;
    int          n_particles = 0;
    int          max_steps = 0;
    float4*      grid_mom = nullptr;   // P2G accumulation (px, py, pz, m); zero between substeps
    float4*      grid_vel = nullptr;   // node velocity after the grid update
    EmpmStep*    d_steps = nullptr;    // device copy of the step schedule
    unsigned*    d_status = nullptr;   // EMPM_STATUS_* bits
    cudaStream_t own_stream = nullptr; // capture stream for the graph path
    cudaEvent_t  ev_a = nullptr;
    cudaEvent_t  ev_b = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    GraphKey     graph_key{};
    bool         graph_valid = false;
    // per-kernel event timing (stream path only)
    bool         timing = false;
    int          timing_capacity = 0;
    int          timing_count[3] = {0, 0, 0};
    std::vector<cudaEvent_t> timing_events;   // [3][capacity][2]
    char         err[512] = {0};
};

int empm_set_error(EmpmCtx* ctx, int code, const char* fmt, ...);
int empm_check_cuda(EmpmCtx* ctx, cudaError_t e, const char* what);
