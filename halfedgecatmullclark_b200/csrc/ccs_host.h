// ccs_host.h -- host-side structures shared by the CUDA translation units.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

#include "ccs_cuda.h"

namespace ccs {

// RAII: make a subd's device current, restore the caller's afterwards.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// A launch whose grid may be scheduled while the previous kernel in the
// stream drains (programmatic stream serialization); the kernel must begin
// with chain_wait_then_release().
template <class... KArgs, class... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t s,
                                  Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

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
    // V x the ring shape of each cage vertex, which no refinement changes:
    // valence in bits 0-29, boundary in bit 30 (null: walked when needed)
    int32_t* vshape = nullptr;
    int32_t V = 0, U = 0, H = 0, E = 0, F = 0;
};

// The cage step of a point rule as a sparse linear map (ccs_cagemap.cu):
// CSR rows over the cage points, rows in depth 1's layout (or, for the
// transpose, one row per cage vertex over depth 1's points).
struct CageMap {
    int32_t* rowptr = nullptr;
    int32_t* col = nullptr;
    float* w = nullptr;
    int32_t rows = 0;
    int64_t nnz = 0;
};
struct CageMaps {
    CageMap creased;    // the scatter rule (:1437-1463, :1602-1648, :1872-1991)
    CageMap creasedT;   // its transpose: the adjoint's cage level
    CageMap smooth;     // the NoCreases scatter rule (:1517-1548, :1713-1756)
};
int build_cage_maps(const cc_Mesh* cage, CageMaps* out);
void free_cage_map(CageMap* m);
cudaError_t launch_cage_map(const CageMap& m, const float* in, float* out, cudaStream_t s);

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
    float ms = -1.0f;            // a profiled graph's replay: time already read, no events
};

struct Profiler {
    bool on = false;
    // while a profiled CUDA graph is being recorded, begin/end put event
    // record nodes into it (cudaEventRecordExternal) instead of recording
    // on the stream; the graph's replays then time its launches as they run
    bool capture = false;
    std::vector<TimedLaunch> pending;
    // begin returns the record's index; end closes that record (or the last)
    int begin(cudaStream_t s, int kernel, int level, int64_t units);
    void end(cudaStream_t s, int index = -1);
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
    // ring statistics of the older vertices, level d (1 <= d < D) at
    // stats + statsOff[d], V(d-1) entries; null = not kept
    float4* stats = nullptr;
    const int64_t* statsOff = nullptr;
    bool fusable = true;         // the twin relation vertex(twin h) = vertex(next h) holds
    // the cage step's linear maps (default atomic pass; null = not built)
    const CageMaps* maps = nullptr;
    // TMA tensor maps of the child records each level d writes (level d+1's
    // records as rows of 128 bytes), indexed by d; null / 0 = not available
    const CUtensorMap* childMaps = nullptr;
    const uint8_t* childMapOk = nullptr;
};

// Rows per box of the child-record tensor maps: 32 rows of 128 bytes (the
// children of 64 parent halfedges).  A block stores its tile as consecutive
// boxes, 4 KB apart in shared memory.
static constexpr int kChildBoxRows = 32;

// Encodes the tensor map of the child records written by the step d -> d+1
// (rows of 128 bytes over level d+1's 16-byte records, kChildBoxRows-row
// boxes, 128-byte swizzle); false when the driver entry point is missing or the
// encoding is refused.
bool encode_child_map(CUtensorMap* map, int32_t* levelRecords, int64_t parentHalfedges);

// A cage and all its arrays in one page-locked (else malloc'd) host block
// (ccs_ccm.cu); NULL when out of memory.  free_cage_block takes such a cage.
cc_Mesh* alloc_cage_block(int32_t V, int32_t U, int32_t H, int32_t E, int32_t F);
void free_cage_block(cc_Mesh* m);

// Read-only view of a subd for the exporters (ccs_export.cu).
struct SubdView {
    const DevCage* cage;
    int32_t D, rw;
    const Level* lv;             // D + 1 entries
    const int32_t* he;           // refined halfedges (all levels)
    const float* pts;            // refined points (all levels)
    cudaStream_t stream;
    int device;
    bool topo;                   // topology refined
};
bool subd_view(const cc_Subd* subd, SubdView* out);

// Records `s` as the calling thread's ccs_LastError_cuda() status; returns s.
int set_last_error(int s);

inline float4* stats_at(const Ctx& c, int d) {
    return (c.stats && c.statsOff && d >= 1 && d < c.D) ? c.stats + c.statsOff[d] : nullptr;
}

// Forward passes (ccs_forward.cu).  All return cudaError_t of the launches.
cudaError_t run_topology(const Ctx& c, bool topo, bool uv);
cudaError_t run_creases(const Ctx& c);
// mode: CCS_POINTS_*; deterministic selects the fixed-order scatter sum.
cudaError_t run_points(const Ctx& c, const float* cagePts, float* pts, int mode, bool deterministic);
// Fused scatter pipeline (ccs_level.cu): cage step, then two kernels per quad
// level.  topo = also refine halfedges, UVs and creases.  mode must be
// CCS_POINTS_SCATTER or CCS_POINTS_NOCREASES_SCATTER.
cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool deterministic);

// Per-halfedge normals of the finest level (ccs_normals.cu): `pts` all
// levels' points (cumV x 3), `out` H(D) x 3.
cudaError_t run_normals(const Ctx& c, const float* pts, float* out, bool smooth);

// Ring statistics of the older vertices of every quad level (ccs_level.cu),
// from the refined halfedges and creases.
cudaError_t run_ring_stats(const Ctx& c);

// Adjoint (ccs_adjoint.cu).  `work` holds cumV x 3 floats.  Reads the ring
// statistics of c.stats when kept (else walks the rings per halfedge).
cudaError_t run_adjoint(const Ctx& c, const float* gradPts, float* work, float* gradCage, int64_t cumV);

}  // namespace ccs
