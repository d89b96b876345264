// ccs_host.h -- host-side structures shared by the CUDA translation units.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "ccs_cuda.h"

namespace ccs {

struct CageCountsH {
    int32_t V, F, E, H;
};

// Device copy of a cage (cc_Mesh arrays, same layouts).
struct DevCage {
    int32_t* he = nullptr;      // H x 7 words
    cc_Crease* cr = nullptr;    // E
    float* pts = nullptr;       // V x 3
    float* uvs = nullptr;       // U x 2
    int32_t* v2h = nullptr;
    int32_t* e2h = nullptr;
    int32_t* f2h = nullptr;
    int32_t* fsz = nullptr;     // F x face size (halfedges per cage face)
    int32_t V = 0, U = 0, H = 0, E = 0, F = 0;
};

// Counts of one depth and the offsets of its arrays in the packed hierarchy.
struct Level {
    int32_t d;
    int32_t V, F, E, H, C;        // counts at depth d
    int64_t heOff, crOff, ptOff;  // offset of depth-d records (d >= 1)
};

// One timed launch (profiling mode).
struct TimedLaunch {
    int kernel, level;
    int64_t units;
    cudaEvent_t a, b;
};

struct Profiler {
    bool on = false;
    std::vector<TimedLaunch> pending;
    void begin(cudaStream_t s, int kernel, int level, int64_t units);
    void end(cudaStream_t s);
};

// Launch context: everything a refine pass needs.
struct Ctx {
    const DevCage* cage;
    int32_t rw;                  // 4 or 3 words per refined halfedge record
    int32_t D;
    const Level* lv;             // D + 1 entries
    int32_t* he;                 // refined halfedges (cumH records)
    cc_Crease* cr;               // refined creases
    cudaStream_t stream;
    Profiler* prof;
    int* err;                    // device error word
    // optional second stream for independent launches of one step (forked
    // from and joined back into `stream` by the two events); null = serial
    cudaStream_t side = nullptr;
    cudaEvent_t forkEv = nullptr, joinEv = nullptr;
};

// Forward passes (ccs_forward.cu).  All return cudaError_t of the launches.
cudaError_t run_topology(const Ctx& c, bool topo, bool uv);
cudaError_t run_creases(const Ctx& c);
// mode: CCS_POINTS_*; deterministic selects the fixed-order scatter sum.
cudaError_t run_points(const Ctx& c, const float* cagePts, float* pts, int mode, bool deterministic);
// Fused scatter pipeline (ccs_level.cu): cage step, then two kernels per quad
// level.  topo = also refine halfedges, UVs and creases.  mode must be
// CCS_POINTS_SCATTER or CCS_POINTS_NOCREASES_SCATTER.
cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool deterministic);

// Adjoint (ccs_adjoint.cu).  `work` holds cumV x 3 floats; `stats` (may be
// null: the rings are then walked per halfedge) holds adjoint_stats_count(c)
// float4 entries, 16-byte aligned.
cudaError_t run_adjoint(const Ctx& c, const float* gradPts, float* work, float* gradCage, int64_t cumV,
                        float4* stats);
// Older vertices of the largest quad level the adjoint visits: max V(d-1), 1 <= d < D.
inline int64_t adjoint_stats_count(const Ctx& c) {
    int64_t m = 0;
    for (int d = 1; d < c.D; ++d) m = c.lv[d - 1].V > m ? c.lv[d - 1].V : m;
    return m;
}

}  // namespace ccs
