// ctx.hpp — the opaque EmpmCtx behind the C ABI: one batch of independent
// simulation instances (a single simulation is a batch of one).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "../../include/empm_b200.h"

namespace empm { struct InstanceConsts; }

struct GraphKey {
    EmpmParticles a;
    EmpmParticles b;
    EmpmMaterial  mat;
    int           n_steps;
    int           n_tables;
    int           sort_every;
    int           p2g_mode;
    int           g2p_tile;
    int           tile_cap;
    int           seg_cap;
    int           fuse;                       // fused G2P + P2G runs in use (option and hold pattern)
    unsigned long long params_version;
    int           flags;                      // EMPM_ROLLOUT_RESUME / EMPM_ROLLOUT_KEEP
    int           start_pc, start_mc, start_since;   // sorted state a resumed sequence starts in
};

// What a segment's captured substep loop depends on besides the segment's
// own buffers: the context epoch and options, and the caller's buffers where
// the loop works on them directly (unsorted segments).
struct SegGraphKey {
    unsigned long long epoch;
    unsigned long long params_version;
    int                seg_cap, p2g_mode, sort_every, n;
    int                n_steps, store;
    const void*        buf[10];
};

// A captured re-run + reverse pass of a checkpointed segment
// (empm_adjoint_segment), cached per context by its key.
struct AdjSegGraph {
    SegGraphKey        key{};
    cudaGraphExec_t    exec = nullptr;
    unsigned long long used = 0;
};

// One captured rollout launch sequence and the sorted state it ends in.
struct GraphEntry {
    GraphKey        key{};
    cudaGraphExec_t exec = nullptr;
    bool            valid = false;
    int             end_pc = 0, end_mc = 0, end_since = 0;
    unsigned long long used = 0;
};

// Particle and material buffers of the sorted path (cell order).
struct SortedBuffers {
    bool   allocated = false;
    int    n = 0;                          // particle capacity
    long long nb = 0;                      // block capacity
    float* part[2] = {nullptr, nullptr};   // x4 | v4 | C f9 | F f9 per buffer (ping-pong per substep)
    float* fe[2] = {nullptr, nullptr};     // elastic F handed from P2G to G2P (f9), per sort epoch like matf:
                                           // a cell sort permutes it, so held particles keep their own
    float* matf[2] = {nullptr, nullptr};   // vol | mu | lam | ys (ping-pong per sort)
    int*   mati[2] = {nullptr, nullptr};   // sel | pid
    int*   keys = nullptr;
    int*   ranks = nullptr;
    int*   block_counts = nullptr;         // [nblocks], zero between sorts
    int*   block_offsets = nullptr;        // [nblocks]
    int*   chunk_counts = nullptr;         // [nblocks]
    int*   chunk_offsets = nullptr;        // [nblocks]
    int*   cell_counts = nullptr;          // [nblocks * 64], zero between sorts
    int*   cell_offsets = nullptr;         // [nblocks * 64]
    int2*  chunks = nullptr;               // [max_chunks]
    int*   nchunks = nullptr;
    int    max_chunks = 0;
    void*  scan_tmp = nullptr;             // CUB scan scratch
    size_t scan_tmp_bytes = 0;
};

// Buffers of the reverse-mode path (empm_adjoint_segment), allocated on first use.
struct AdjointBuffers {
    int     capacity = 0;      // substeps per segment the buffers hold
    int     cap_n = 0;         // particle capacity of the per-particle buffers
    long long cap_blocks = 0;  // block capacity of the grid buffers
    float*  states = nullptr;  // capacity + 1 packed particle states (x4 | v4 | C f9 | F f9)
    float*  mats = nullptr;    // capacity snapshots of mu | lam | yield
    float*  work = nullptr;    // mu | lam | yield updated by the recomputed substeps
    float*  fe = nullptr;      // elastic F of the substep being differentiated (f9)
    float*  gfe = nullptr;     // its adjoint (f9)
    float4* gx = nullptr;      // x adjoint through G2P
    float4* gacc = nullptr;    // node velocity adjoint (blocked grid), zero between substeps
    float4* gmom = nullptr;    // adjoint of the P2G accumulation (blocked grid)
    float*  gstate = nullptr;  // state adjoint in cell order (packed like states)
    float*  gmats = nullptr;   // mu | lam | yield | mass adjoints in cell order
    // stored substeps (EMPM_OPT_ADJ_STORE): per substep of the segment, the
    // touched blocks' node momentum and velocity (128 float4 per block), their
    // list (count, ids) and the elastic F, so the reverse pass need not
    // recompute P2G and the grid update
    int     store_cap = 0;     // substeps the store holds (0 = not allocated)
    float4* gsave = nullptr;   // store_cap x cap_blocks x 128 float4
    int*    gsave_list = nullptr;  // store_cap x (1 + cap_blocks)
    float*  fe_store = nullptr;    // store_cap x f9 planes of cap_n particles
    std::vector<EmpmStep> tables;   // host staging of the step tables
};

struct EmpmCtx {
    // instances
    int          n_inst = 0;
    std::vector<EmpmModelParams> params;   // per instance
    std::vector<int> counts;               // particles per instance
    std::vector<int> poff;                 // first particle of each instance
    std::vector<int> boff;                 // first global 4^3 block of each instance
    int          n_particles = 0;          // total
    long long    nblocks = 0;              // total 4^3 grid blocks
    // capacities the device buffers are sized for (empm_batch_reserve);
    // empm_batch_reconfigure re-lays instances within them without allocating
    int          cap_particles = 0;
    long long    cap_blocks = 0;
    int          cap_inst = 0;
    empm::InstanceConsts* d_inst = nullptr;
    unsigned long long params_version = 0;
    // device
    int          device = 0;
    int          sm_count = 148;
    size_t       step_entries = 0;         // capacity of the step-table array, in EmpmStep entries
    float4*      grid_mom = nullptr;       // P2G accumulation (px, py, pz, m), blocked layout; zero between substeps
    float4*      grid_vel = nullptr;       // node velocity after the grid update, blocked layout
    unsigned char* flags = nullptr;        // touched node blocks of the current substep
    int*         active = nullptr;         // [1 + blocks]: number of touched blocks, then their ids
    EmpmStep*    d_steps = nullptr;        // device copy of the step schedules
    unsigned*    d_status = nullptr;       // EMPM_STATUS_* bits
    cudaStream_t own_stream = nullptr;     // capture stream for the graph path
    cudaEvent_t  ev_a = nullptr;
    cudaEvent_t  ev_b = nullptr;
    static constexpr int kGraphs = 16;     // cached rollout graphs (LRU)
    GraphEntry   graphs[kGraphs];
    unsigned long long graph_clock = 0;
    // bumped whenever captured launch sequences stop matching the context
    // (options, instance tables, reallocated buffers): segment graphs compare it
    unsigned long long epoch = 1;
    int          segment_graph = 1;        // stored segments replay their substeps from a CUDA graph
    static constexpr int kAdjGraphs = 4;   // cached checkpointed-segment graphs (LRU)
    AdjSegGraph  adj_graphs[kAdjGraphs];
    // the sorted state the last rollout ended in, which EMPM_ROLLOUT_RESUME
    // continues from: particle / material buffer and substeps since its sort
    bool         resident = false;
    int          resident_pc = 0, resident_mc = 0, resident_since = 0;
    // launch options (empm_ctx_set_option)
    int          sort_every = 32;          // 0 = direct path for rollouts too
    int          p2g_mode = 2;             // 0 direct reductions, 1 shared-memory tile, 2 warp-aggregated
    int          g2p_tile = 0;
    int          tile_cap = 1024;          // nodes per shared-memory tile (16 B each)
    int          seg_cap = 4;              // warp-aggregated P2G: longest same-cell run per head
    int          adj_store = 1;            // adjoint segments store substep grids instead of recomputing
    int          fuse = 1;                 // sorted rollouts fuse the G2P of one substep with the P2G of the next
    bool         fuse_ok = true;           // the uploaded step tables allow it (holds never released)
    SortedBuffers sb;
    AdjointBuffers adj;
    // per-kernel event timing (stream path only)
    bool         timing = false;
    int          timing_capacity = 0;
    // timed kernels: 0 stress+P2G, 1 grid update, 2 G2P, 3 adjoint G2P, 4 adjoint grid, 5 adjoint P2G,
    // 6 fused G2P + stress + P2G
    static constexpr int kTimedKernels = 7;
    int          timing_count[kTimedKernels] = {0, 0, 0, 0, 0, 0, 0};
    std::vector<cudaEvent_t> timing_events;   // [kTimedKernels][capacity][2]
    char         err[512] = {0};
};

// A segment of a differentiable rollout kept on the device from its forward
// pass (empm_segment_forward) to its reverse pass (empm_segment_reverse): the
// state before every substep, the mu / lam / yield snapshots, each substep's
// touched grid blocks and elastic F, vol / selection / caller index in the
// order it ran in, and its step tables.
struct EmpmSegment {
    EmpmCtx* ctx = nullptr;
    int      n = 0, n_steps = 0, n_inst = 0;
    size_t   np = 0, cap_blocks = 0;
    size_t   block_cap = 0;       // grid blocks each substep's store slot holds
    bool     sorted = false, has_sel = false, ready = false;
    bool     checked = false;     // max_touched read back since the last forward pass
    int      max_touched = 0;
    float*   states = nullptr;    // (n_steps + 1) packed states
    float*   mats = nullptr;      // n_steps x (mu | lam | yield)
    float4*  gsave = nullptr;     // n_steps x block_cap x 128 float4
    int*     glist = nullptr;     // n_steps x (1 + block_cap)
    float*   fe = nullptr;        // n_steps x f9 planes
    float*   vol = nullptr;       // [np]
    int*     sel = nullptr;       // [np]
    int*     pid = nullptr;       // [np] caller index of each position (cell order)
    int*     max_count = nullptr; // device: largest touched-block count of the forward pass
    std::vector<EmpmStep> tables;
    EmpmStep* d_tables = nullptr; // device copy of tables, read by the segment's kernels
    bool     tables_on_device = false;
    // the substep loops of the forward and reverse passes, captured once and
    // replayed while the key (context epoch, options, buffers) still matches
    SegGraphKey     fwd_key{}, rev_key{};
    cudaGraphExec_t fwd_exec = nullptr, rev_exec = nullptr;
};

int empm_set_error(EmpmCtx* ctx, int code, const char* fmt, ...);
int empm_check_cuda(EmpmCtx* ctx, cudaError_t e, const char* what);
