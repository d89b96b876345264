// ccs_batch.cu -- many cages of uneven size and depth refined together.
//
// Every cage keeps the single-mesh layout (its own packed halfedges, creases
// and points), placed one after the other in batch-wide buffers.  Work is
// cut into tiles of 256 items that never span two cages (so the lane
// structure the level kernels rely on -- quads in 4 adjacent lanes, a parent
// face's 16 children in 16 lanes -- holds in every tile).  For each depth d
// one persistent kernel covers every cage still active at d: its blocks
// stride over the tiles of one phase, meet at a grid barrier, and go on
// with the next phase:
//
//   forward, d = 0:  cage topology + creases + face points (+ clearing)
//                    | edge points | vertex points (+ shape statistics of level 1)
//   forward, d >= 1: kernel A tiles + crease tiles (+ creased-edge statistics
//                    of level d) | vertex pass tiles (+ shape statistics of
//                    level d + 1)
//   adjoint, d = 0:  edge gathers | face gathers | vertex gathers
//   adjoint, d >= 1: edge pass | face + vertex pass
//
// The default vertex pass sums with float atomics (the single-mesh default);
// CCS_FLAG_DETERMINISTIC selects the exact pass (older vertices one thread
// each, face centres and edge midpoints in the warp; one thread per vertex
// with a sorted ring at d <= 1), bit-identical to the reference.  The older
// vertices' ring statistics are built while the topology is refined and kept
// per level for the points-only forward and the adjoint.
//
// The tile bodies are the single-mesh ones (ccs_tiles.cuh).  The kernels run
// as cooperative launches (all blocks resident), and every barrier wait is
// bounded: a wait that gives up sets an error word, the kernel returns, and
// the host reports CCS_ERR_TIMEOUT.  A tile -> cage lookup is a binary
// search over the per-phase tile prefix sums.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBatchBlock = 256;
static constexpr int kMaxBatchDepth = 10;

enum Phase {
    PH_CAGE_TOPO = 0,   // 4 H0 child halfedges
    PH_CAGE_CREASE,     // E0 creases
    PH_CAGE_FACE,       // F0 faces
    PH_CAGE_ZERO,       // V0 vertex slots of depth 1 (atomic pass)
    PH_CAGE_EDGE,       // H0 halfedges
    PH_CAGE_VERT,       // V0 vertices (sorted ring) or H0 halfedges (atomics): max of both
    PH_A,               // H_d parent halfedges
    PH_A_CREASE,        // C_d creases
    PH_CREASE_STATS,    // C_d creases of depth d (statistics of the older vertices)
    PH_SHAPE_NEXT,      // V_d vertices: shape statistics of depth d + 1
    PH_V,               // d >= 2: V_(d-1) older vertices (exact pass)
    PH_B,               // H_d halfedges; exact pass at d = 1: V_1 vertices
    PH_ADJ_EDGE,        // H_d
    PH_ADJ_FACE,        // F_d (cage)
    PH_ADJ_VERT,        // V_0 (cage) or H_d
    PH_ZERO3,           // d = 1: V_2 vertex slots of depth 3 (the one-pass step of depth 2)
    PH_CREASE_STATS_NEXT,  // C_(d+1) creases of depth d + 1 (their statistics, before depth d + 1)
    PH_DIST,            // d = 0: the points whose fitting gradient P - T the distance adjoint
                        // writes before its steps (every level but a depth >= 3 cage's finest)
    PH_AF,              // d >= 2: F_d faces (the points-only step and the exact vertex pass)
    PH_ADJ_FSTEP,       // d >= 2: F_d faces (the adjoint step, one thread per face)
    PH_COUNT
};

struct BatchCage {
    DevCage cage;        // pointers into the batch's cage arrays
    int32_t depth;
    int32_t uv;          // UV codes are refined
    int64_t cagePt;      // first cage point of this cage in the batch's cage-point buffer
    int64_t he, cr, pt;  // first record / crease / point of this cage's hierarchy
    int64_t stats[kMaxBatchDepth + 1];  // level d's ring statistics (V(d-1) entries), 1 <= d < depth
    Level lv[kMaxBatchDepth + 1];
};

// Points of a cage whose fitting gradient the distance adjoint writes to the
// working buffer first: all of them, but for a cage of depth >= 3 not its
// finest level, which the first adjoint step reads as P - T directly.
__host__ __device__ inline int64_t dist_points(const BatchCage& bc) {
    const Level& f = bc.lv[bc.depth];
    return bc.depth >= 3 ? f.ptOff : f.ptOff + f.V;
}

struct GridSync {
    unsigned int count;
    unsigned int gen;
    int err;
};

struct BatchArgs {
    const BatchCage* __restrict__ cages;
    const int64_t* __restrict__ tiles;   // [(d * PH_COUNT + phase) * (count + 1) + c]
    int32_t count;
    int32_t* he;
    cc_Crease* cr;
    const float* cagePts;
    float* pts;
    float* work;                         // adjoint: running gradient per refined point
    const float* target = nullptr;       // distance adjoint: the points' target (null: plain adjoint)
    float* gradCage;                     // adjoint output
    float4* stats;                       // ring statistics of the older vertices, every level
    GridSync* sync;
    unsigned int spinCap;                // polls before a barrier wait gives up
};

// ---------------------------------------------------------------------------
// device side
// ---------------------------------------------------------------------------
static constexpr unsigned kSpinCap = 1u << 22;

// Grid-wide barrier for a cooperative launch.  `expected` blocks must arrive;
// a waiting block gives up after `cap` polls (about a second with the
// default cap), records CCS_ERR_TIMEOUT and leaves.
__device__ bool grid_sync(GridSync* gs, unsigned int cap, unsigned int expected) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned int* vgen = &gs->gen;
        const unsigned int g = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&gs->count, 1u) + 1u;
        if (arrived == expected) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        } else {
            unsigned int spins = 0;
            while (*vgen == g) {
                if (++spins > cap || *(volatile int*)&gs->err) {
                    atomicExch(&gs->err, CCS_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(256);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ int find_cage(const int64_t* ts, int32_t count, int64_t t) {
    int lo = 0, hi = count;            // ts[lo] <= t < ts[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ts[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ CageView batch_cage_view(const BatchCage& bc) {
    CageView L;
    L.t = make_cage_tables(bc.cage);
    L.cr = bc.cage.cr;
    L.V = bc.cage.V; L.F = bc.cage.F; L.E = bc.cage.E; L.H = bc.cage.H; L.C = bc.cage.E;
    L.d = 0;
    return L;
}

__device__ __forceinline__ QuadView<4> batch_quad_view(const BatchArgs& a, const BatchCage& bc, int d) {
    QuadView<4> L;
    L.t = make_cage_tables(bc.cage);
    L.he = a.he + 4 * (bc.he + bc.lv[d].heOff);
    L.cr = a.cr + bc.cr + bc.lv[d].crOff;
    const Level& lv = bc.lv[d];
    L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C;
    L.d = d;
    return L;
}

// Runs `body(cage, tile index within the cage)` over one phase's tiles.
template <class Body>
__device__ __forceinline__ void for_tiles(const BatchArgs& a, int d, int phase, Body body) {
    const int64_t* ts = a.tiles + ((int64_t)d * PH_COUNT + phase) * (a.count + 1);
    const int64_t total = ts[a.count];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const int c = find_cage(ts, a.count, t);
        body(a.cages[c], t - ts[c]);
    }
}

__device__ __forceinline__ QuadView<4> batch_quad_view_stats(const BatchArgs& a, const BatchCage& bc, int d) {
    QuadView<4> L = batch_quad_view(a, bc, d);
    L.ostats = a.stats + bc.stats[d];
    return L;
}

// ---------------------------------------------------------------------------
// Forward and adjoint bodies, one function per section (a section is the
// work between two grid barriers).  The fused schedule runs all sections of a
// depth in one cooperative launch with grid barriers between them; the split
// schedule launches each section on its own (ordinary launches, each kernel
// with its own register budget).
// ---------------------------------------------------------------------------
// shape statistics of depth d + 1 (valence, boundary; cage tables only)
template <bool TOPO>
__device__ __forceinline__ void fwd_shape_next(const BatchArgs& a, int d) {
    if (!TOPO) return;
    const int tid = threadIdx.x;
    for_tiles(a, d, PH_SHAPE_NEXT, [&](const BatchCage& bc, int64_t lt) {
        const int64_t v = lt * kBatchBlock + tid;
        if (d + 1 < bc.depth && v < bc.lv[d].V)
            shape_stats_item(make_cage_tables(bc.cage), d + 1, a.stats + bc.stats[d + 1], (int32_t)v);
    });
}

// d = 0, section 1: cage topology, creases, face points, clearing
template <bool TOPO, bool CREASED, bool DET>
__device__ __forceinline__ void fwd_cage_s1(const BatchArgs& a) {
    const int tid = threadIdx.x;
    if (TOPO) {
        for_tiles(a, 0, PH_CAGE_TOPO, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i >= 4 * (int64_t)bc.cage.H) return;
            int32_t* out = a.he + 4 * (bc.he + bc.lv[1].heOff);
            if (bc.uv) cage_topology_item<4, true, true>(make_cage_tables(bc.cage), out, i);
            else cage_topology_item<4, true, false>(make_cage_tables(bc.cage), out, i);
        });
        for_tiles(a, 0, PH_CAGE_CREASE, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i < bc.cage.E) crease_item(bc.cage.cr, a.cr + bc.cr + bc.lv[1].crOff, (int32_t)i);
        });
    }
    for_tiles(a, 0, PH_CAGE_FACE, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        if (i >= bc.cage.F) return;
        face_point_item<CageView, false>(batch_cage_view(bc), a.cagePts + 3 * bc.cagePt,
                                         a.pts + 3 * (bc.pt + bc.lv[1].ptOff), (int32_t)i);
    });
    if (!DET) {
        for_tiles(a, 0, PH_CAGE_ZERO, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i < bc.cage.V) st3(a.pts + 3 * (bc.pt + bc.lv[1].ptOff + i), zero3());
        });
    }
}

// d = 0, section 2: edge points
template <bool CREASED>
__device__ __forceinline__ void fwd_cage_s2(const BatchArgs& a) {
    const int tid = threadIdx.x;
    for_tiles(a, 0, PH_CAGE_EDGE, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        if (i >= bc.cage.H) return;
        edge_owner_item<CageView, CREASED>(batch_cage_view(bc), a.cagePts + 3 * bc.cagePt,
                                           a.pts + 3 * (bc.pt + bc.lv[1].ptOff), (int32_t)i);
    });
}

// d = 0, section 3: vertex points (+ shape statistics of depth 1)
template <bool TOPO, bool CREASED, bool DET>
__device__ __forceinline__ void fwd_cage_s3(const BatchArgs& a) {
    const int tid = threadIdx.x;
    for_tiles(a, 0, PH_CAGE_VERT, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        const float* cp = a.cagePts + 3 * bc.cagePt;
        float* pout = a.pts + 3 * (bc.pt + bc.lv[1].ptOff);
        if (DET) {
            if (i < bc.cage.V) vertex_det_item<CageView, CREASED>(batch_cage_view(bc), cp, pout, (int32_t)i);
        } else {
            // warp-collective: every lane of the tile takes part
            vertex_atomic_item<CageView, CREASED>(batch_cage_view(bc), cp, pout, (int32_t)i, i < bc.cage.H);
        }
    });
    fwd_shape_next<TOPO>(a, 0);
}

// Quad levels.  Deterministic pass, every depth d >= 1: section 1 = kernel A
// tiles, crease tiles, creased-edge statistics of depth d; section 2 = the
// exact vertex pass + shape statistics of depth d + 1.  Default (atomic)
// pass: depth 1 as the deterministic schedule plus the clearing of depth 3's
// slots, and a section 3 with the creased-edge statistics of depth 2; depth
// d >= 2: section 1 = one-pass step tiles (tile_level_ab, which clear depth
// d + 2's slots), crease tiles, shape statistics of depth d + 1; section 2 =
// the creased-edge statistics of depth d + 1 (after its shape entries).
__device__ __forceinline__ LevelArgs batch_level_args(const BatchArgs& a, const BatchCage& bc, int d) {
    const Level& lv = bc.lv[d];
    LevelArgs la;
    la.in = a.he + 4 * (bc.he + lv.heOff);
    la.out = a.he + 4 * (bc.he + bc.lv[d + 1].heOff);
    la.crIn = a.cr + bc.cr + lv.crOff;
    la.crOut = a.cr + bc.cr + bc.lv[d + 1].crOff;
    la.pin = a.pts + 3 * (bc.pt + lv.ptOff);
    la.pout = a.pts + 3 * (bc.pt + bc.lv[d + 1].ptOff);
    la.H = lv.H; la.V = lv.V; la.F = lv.F; la.E = lv.E; la.C = lv.C;
    return la;
}

template <bool TOPO>
__device__ __forceinline__ void fwd_crease_tiles(const BatchArgs& a, int d) {
    if (!TOPO) return;
    const int tid = threadIdx.x;
    for_tiles(a, d, PH_A_CREASE, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        if (i < bc.lv[d].C)
            crease_item(a.cr + bc.cr + bc.lv[d].crOff, a.cr + bc.cr + bc.lv[d + 1].crOff, (int32_t)i);
    });
}

// creased edges of depth dd into the older vertices' statistics (their shape
// entries must be written)
__device__ __forceinline__ void fwd_crease_stats(const BatchArgs& a, int d, int phase, int dd) {
    const int tid = threadIdx.x;
    for_tiles(a, d, phase, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        if (dd < bc.depth && i < bc.lv[dd].C)
            crease_stats_item(batch_quad_view(a, bc, dd), bc.lv[dd - 1].V, a.stats + bc.stats[dd], (int32_t)i);
    });
}

// default pass, depth d >= 2, section 1 (the points-only step: one thread
// per face, fq_points; with the topology: one thread per parent halfedge,
// tile_level_ab)
template <bool TOPO, bool CREASED>
__device__ __forceinline__ void fwd_level_ab(const BatchArgs& a, int d, int32_t* tile) {
        if (!TOPO) {
            for_tiles(a, d, PH_AF, [&](const BatchCage& bc, int64_t lt) {
                LevelArgs la = batch_level_args(a, bc, d);
                la.ostats = a.stats + bc.stats[d];
                la.d = d;
                const int64_t f = lt * kBatchBlock + threadIdx.x;
                const bool valid = f < bc.lv[d].F;
                int4 r[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) r[k] = make_int4(-1, 0, 0, 0);
                if (valid) load_face_records<4>(la.in, f, r);
                fq_points<4, CREASED>(la, f, valid, r);
                if (d + 2 <= bc.depth) {
                    float* z = a.pts + 3 * (bc.pt + bc.lv[d + 2].ptOff);
                    const int64_t n = 3 * (int64_t)bc.lv[d + 1].V;
                    const int64_t stride = (((int64_t)bc.lv[d].F + kBatchBlock - 1) / kBatchBlock) * kBatchBlock;
                    for (int64_t i = f; i < n; i += stride) z[i] = 0.0f;
                }
            });
            return;
        }
        for_tiles(a, d, PH_A, [&](const BatchCage& bc, int64_t lt) {
            LevelArgs la = batch_level_args(a, bc, d);
            la.ostats = a.stats + bc.stats[d];
            if (d + 2 <= bc.depth) {
                la.zeroNext = a.pts + 3 * (bc.pt + bc.lv[d + 2].ptOff);
                la.zeroNextN = 3 * (int64_t)bc.lv[d + 1].V;
            }
            const int64_t stride = (((int64_t)bc.lv[d].H + kBatchBlock - 1) / kBatchBlock) * kBatchBlock;
            if (bc.uv) tile_level_ab<kBatchBlock, 4, TOPO, true, CREASED>(la, lt * kBatchBlock, tile, stride);
            else tile_level_ab<kBatchBlock, 4, TOPO, false, CREASED>(la, lt * kBatchBlock, tile, stride);
            __syncthreads();   // the tile's shared memory is reused by the next tile
        });
        fwd_crease_tiles<TOPO>(a, d);
        fwd_shape_next<TOPO>(a, d);
}

// section 1 of depth 1, and of every depth in the deterministic pass
template <bool TOPO, bool CREASED, bool DET>
__device__ __forceinline__ void fwd_level_s1(const BatchArgs& a, int d, int32_t* tile) {
    const int tid = threadIdx.x;
    for_tiles(a, d, PH_A, [&](const BatchCage& bc, int64_t lt) {
        LevelArgs la = batch_level_args(a, bc, d);
        la.zeroV = DET ? 0 : 1;          // the atomic pass accumulates into cleared slots
        if (bc.uv) tile_level_a<kBatchBlock, 4, TOPO, true, true, CREASED>(la, lt * kBatchBlock, tile);
        else tile_level_a<kBatchBlock, 4, TOPO, false, true, CREASED>(la, lt * kBatchBlock, tile);
        __syncthreads();   // the tile's shared memory is reused by the next tile
    });
    fwd_crease_tiles<TOPO>(a, d);
    if (TOPO) fwd_crease_stats(a, d, PH_CREASE_STATS, d);
    if (!DET) {
        for_tiles(a, d, PH_ZERO3, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (bc.depth >= 3 && i < bc.lv[2].V) st3(a.pts + 3 * (bc.pt + bc.lv[3].ptOff + i), zero3());
        });
    }
}

// section 2: the vertex pass + shape statistics of depth d + 1 (depth 1 or the
// deterministic pass); the creased-edge statistics of depth d + 1 (d >= 2,
// default pass)
template <bool TOPO, bool CREASED, bool DET>
__device__ __forceinline__ void fwd_level_s2(const BatchArgs& a, int d) {
    const int tid = threadIdx.x;
    if (!DET && d >= 2) {
        if (TOPO) fwd_crease_stats(a, d, PH_CREASE_STATS_NEXT, d + 1);
        return;
    }
    if (DET && d >= 2) {
        for_tiles(a, d, PH_V, [&](const BatchCage& bc, int64_t lt) {
            const int64_t v = lt * kBatchBlock + tid;
            if (v < bc.lv[d - 1].V)
                old_vertex_item<4, CREASED>(batch_quad_view(a, bc, d), a.pts + 3 * (bc.pt + bc.lv[d].ptOff),
                                            a.pts + 3 * (bc.pt + bc.lv[d + 1].ptOff), (int32_t)v);
        });
        for_tiles(a, d, PH_AF, [&](const BatchCage& bc, int64_t lt) {
            tile_face_exact<4, CREASED, false>(batch_quad_view(a, bc, d), a.pts + 3 * (bc.pt + bc.lv[d].ptOff),
                                        a.pts + 3 * (bc.pt + bc.lv[d + 1].ptOff), lt * kBatchBlock);
        });
        fwd_shape_next<TOPO>(a, d);
        return;
    }
    for_tiles(a, d, PH_B, [&](const BatchCage& bc, int64_t lt) {
        const float* pin = a.pts + 3 * (bc.pt + bc.lv[d].ptOff);
        float* pout = a.pts + 3 * (bc.pt + bc.lv[d + 1].ptOff);
        if (!DET) {
            const QuadView<4> L = batch_quad_view_stats(a, bc, d);
            if (d >= 2) tile_level_b<4, CREASED, true>(L, pin, pout, lt * kBatchBlock);
            else tile_level_b<4, CREASED, false>(L, pin, pout, lt * kBatchBlock);
        } else {
            const QuadView<4> L = batch_quad_view(a, bc, d);
            const int64_t v = lt * kBatchBlock + tid;
            if (v < L.V) vertex_det_item<QuadView<4>, CREASED>(L, pin, pout, (int32_t)v);
        }
    });
    fwd_shape_next<TOPO>(a, d);
}

// section 3 (default pass, depth 1): the creased-edge statistics of depth 2
template <bool TOPO>
__device__ __forceinline__ void fwd_level_s3(const BatchArgs& a, int d) {
    if (TOPO) fwd_crease_stats(a, d, PH_CREASE_STATS_NEXT, d + 1);
}

__device__ __forceinline__ float* adj_gnew(const BatchArgs& a, const BatchCage& bc, int d) {
    return a.work + 3 * (bc.pt + bc.lv[d + 1].ptOff);
}

// adjoint, d = 0: three gathers (sections 1-3)
template <int S>
__device__ __forceinline__ void adj_cage_section(const BatchArgs& a) {
    const int tid = threadIdx.x;
    if (S == 1) {
        for_tiles(a, 0, PH_ADJ_EDGE, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i < bc.cage.H) adj_edge_item(batch_cage_view(bc), adj_gnew(a, bc, 0), (int32_t)i);
        });
    } else if (S == 2) {
        for_tiles(a, 0, PH_ADJ_FACE, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i < bc.cage.F) adj_face_item(batch_cage_view(bc), adj_gnew(a, bc, 0), (int32_t)i);
        });
    } else {
        for_tiles(a, 0, PH_ADJ_VERT, [&](const BatchCage& bc, int64_t lt) {
            const int64_t i = lt * kBatchBlock + tid;
            if (i < bc.cage.V)
                adj_vertex_item(batch_cage_view(bc), adj_gnew(a, bc, 0), a.gradCage + 3 * bc.cagePt, (int32_t)i);
        });
    }
}

// adjoint, d >= 2: one pass, one thread per face (adj_face_step_tile)
__device__ __forceinline__ void adj_level_step(const BatchArgs& a, int d) {
    for_tiles(a, d, PH_ADJ_FSTEP, [&](const BatchCage& bc, int64_t lt) {
        float* gOld = a.work + 3 * (bc.pt + bc.lv[d].ptOff);
        const QuadView<4> L = batch_quad_view_stats(a, bc, d);
        const int64_t f = lt * kBatchBlock + threadIdx.x;
        if (a.target && d + 1 == bc.depth) {
            // distance adjoint, the cage's finest level: its gradient P - T as it is read
            const int64_t o = 3 * (bc.pt + bc.lv[d + 1].ptOff);
            adj_face_step_tile<4, GradDistance>(L, GradDistance{a.pts + o, a.target + o}, gOld, f);
        } else {
            adj_face_step_tile<4, GradArray>(L, GradArray{adj_gnew(a, bc, d)}, gOld, f);
        }
    });
}

// distance adjoint, before its steps: work = P - T over the PH_DIST points
__global__ void __launch_bounds__(kBatchBlock)
k_batch_dist_init(BatchArgs a, int) {
    const int tid = threadIdx.x;
    for_tiles(a, 0, PH_DIST, [&](const BatchCage& bc, int64_t lt) {
        const int64_t i = lt * kBatchBlock + tid;
        if (i >= dist_points(bc)) return;
        const int64_t o = 3 * (bc.pt + i);
        a.work[o + 0] = fsub(a.pts[o + 0], a.target[o + 0]);
        a.work[o + 1] = fsub(a.pts[o + 1], a.target[o + 1]);
        a.work[o + 2] = fsub(a.pts[o + 2], a.target[o + 2]);
    });
}

// adjoint, d = 1: edge pass (section 1), point pass (section 2)
template <int S>
__device__ __forceinline__ void adj_level_section(const BatchArgs& a, int d) {
    if (S == 1) {
        for_tiles(a, d, PH_ADJ_EDGE, [&](const BatchCage& bc, int64_t lt) {
            adj_quad_edge_tile<4>(batch_quad_view_stats(a, bc, d), adj_gnew(a, bc, d), lt * kBatchBlock);
        });
    } else {
        for_tiles(a, d, PH_ADJ_VERT, [&](const BatchCage& bc, int64_t lt) {
            float* gOld = a.work + 3 * (bc.pt + bc.lv[d].ptOff);
            if (d >= 2) adj_quad_point_tile<4, true>(batch_quad_view_stats(a, bc, d), adj_gnew(a, bc, d), gOld, lt * kBatchBlock);
            else adj_quad_point_tile<4, false>(batch_quad_view_stats(a, bc, d), adj_gnew(a, bc, d), gOld, lt * kBatchBlock);
        });
    }
}

// fused schedule: one cooperative launch per depth, grid barriers between sections
template <bool TOPO, bool CREASED, bool DET>
__global__ void __launch_bounds__(kBatchBlock)
k_batch_forward(BatchArgs a, int d) {
    __shared__ __align__(128) int32_t tile[kBatchBlock * 4 * 4];
    if (d == 0) {
        fwd_cage_s1<TOPO, CREASED, DET>(a);
        if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
        fwd_cage_s2<CREASED>(a);
        if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
        fwd_cage_s3<TOPO, CREASED, DET>(a);
        return;
    }
    if (!DET && d >= 2) fwd_level_ab<TOPO, CREASED>(a, d, tile);
    else fwd_level_s1<TOPO, CREASED, DET>(a, d, tile);
    if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
    fwd_level_s2<TOPO, CREASED, DET>(a, d);
    if (TOPO && !DET && d == 1) {
        if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
        fwd_level_s3<TOPO>(a, d);
    }
}

__global__ void __launch_bounds__(kBatchBlock)
k_batch_adjoint(BatchArgs a, int d) {
    if (d == 0) {
        adj_cage_section<1>(a);
        if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
        adj_cage_section<2>(a);
        if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
        adj_cage_section<3>(a);
        return;
    }
    if (d >= 2) {
        adj_level_step(a, d);
        return;
    }
    adj_level_section<1>(a, d);
    if (!grid_sync(a.sync, a.spinCap, gridDim.x)) return;
    adj_level_section<2>(a, d);
}

// split schedule, adjoint, depth d >= 2: the one-pass step on its own register budget
#ifndef CCS_BATCH_ADJ_STEP_MIN_BLOCKS
#define CCS_BATCH_ADJ_STEP_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(kBatchBlock, CCS_BATCH_ADJ_STEP_MIN_BLOCKS)
k_batch_adj_step(BatchArgs a, int d) {
    adj_level_step(a, d);
}

// split schedule: one ordinary launch per section (kernel boundaries order them)
enum Section { SEC_CAGE_1 = 0, SEC_CAGE_2, SEC_CAGE_3, SEC_LEVEL_1, SEC_LEVEL_2, SEC_LEVEL_3 };

template <bool TOPO, bool CREASED, bool DET, int S>
__global__ void __launch_bounds__(kBatchBlock)
k_batch_forward_section(BatchArgs a, int d) {
    if constexpr (S == SEC_CAGE_1) fwd_cage_s1<TOPO, CREASED, DET>(a);
    else if constexpr (S == SEC_CAGE_2) fwd_cage_s2<CREASED>(a);
    else if constexpr (S == SEC_CAGE_3) fwd_cage_s3<TOPO, CREASED, DET>(a);
    else if constexpr (S == SEC_LEVEL_1) {
        __shared__ __align__(128) int32_t tile[kBatchBlock * 4 * 4];
        fwd_level_s1<TOPO, CREASED, DET>(a, d, tile);
    } else if constexpr (S == SEC_LEVEL_2) {
        fwd_level_s2<TOPO, CREASED, DET>(a, d);
    } else {
        fwd_level_s3<TOPO>(a, d);
    }
}

// split schedule, default pass, depth d >= 2: section 1 on its own register
// budget (the single-mesh steps': 6 blocks of 256 for the per-halfedge tile,
// 3 for the per-face one)
template <bool TOPO, bool CREASED>
__global__ void __launch_bounds__(kBatchBlock, TOPO ? 6 : 3)
k_batch_level_ab(BatchArgs a, int d) {
    __shared__ __align__(128) int32_t tile[kBatchBlock * 4 * 4];
    fwd_level_ab<TOPO, CREASED>(a, d, tile);
}

template <int S>
__global__ void __launch_bounds__(kBatchBlock)
k_batch_adjoint_section(BatchArgs a, int d) {
    if constexpr (S == SEC_CAGE_1) adj_cage_section<1>(a);
    else if constexpr (S == SEC_CAGE_2) adj_cage_section<2>(a);
    else if constexpr (S == SEC_CAGE_3) adj_cage_section<3>(a);
    else if constexpr (S == SEC_LEVEL_1) adj_level_section<1>(a, d);
    else adj_level_section<2>(a, d);
}

// A one-block barrier that waits for a second arrival that never comes: the
// bounded wait must give up and report, leaving the context usable.
__global__ void k_barrier_timeout_probe(GridSync* gs, unsigned int cap) {
    grid_sync(gs, cap, 2u);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int level_counts_ex(const cc_Mesh* cage, int32_t D, std::vector<Level>* out);   // ccs_capi.cu
int validate_cage_ex(const cc_Mesh* m);                                           // ccs_capi.cu
bool twins_consistent_ex(const cc_Mesh* m);                                       // ccs_capi.cu
int set_last_error(int status);                                                  // ccs_capi.cu

}  // namespace ccs

struct ccs_Batch {
    int device = 0;
    int32_t count = 0, maxDepth = 0;
    uint32_t flags = 0;
    std::vector<ccs::BatchCage> host;        // descriptors (device pointers inside)
    std::vector<int64_t> tiles;              // host copy of the tile prefix sums
    ccs::BatchCage* dCages = nullptr;
    int64_t* dTiles = nullptr;
    // cage arrays (concatenated)
    int32_t *cHe = nullptr, *cV2h = nullptr, *cE2h = nullptr, *cF2h = nullptr, *cFsz = nullptr;
    cc_Crease* cCr = nullptr;
    float *cUv = nullptr, *cagePts = nullptr;
    // hierarchy and buffers
    int32_t* he = nullptr;
    cc_Crease* cr = nullptr;
    float *pts = nullptr, *work = nullptr, *gradCage = nullptr;
    ccs::GridSync* sync = nullptr;
    int64_t totH = 0, totC = 0, totV = 0, totCagePts = 0, totStats = 0;
    float4* stats = nullptr;                 // adjoint ring statistics (totStats entries)
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    int blocksPerSM = 0;                     // 0 = as many as fit
    bool split = false;                      // one launch per section instead of per depth
    int numSMs = 148;
    bool graphOk = true;
    bool topoReady = false;                  // ccs_BatchRefine_cuda has run
    const float* target = nullptr;           // the distance adjoint's target (its graph holds it)
    std::map<int, cudaGraphExec_t> graphs;
    std::mutex mu;
};

namespace ccs {

static const int kPhasesPerDepth = PH_COUNT;

static int64_t phase_units(const BatchCage& bc, int d, int ph) {
    if (d >= bc.depth) return 0;
    const Level& lv = bc.lv[d];
    switch (ph) {
        case PH_CAGE_TOPO: return d == 0 ? 4 * (int64_t)lv.H : 0;
        case PH_CAGE_CREASE: return d == 0 ? lv.E : 0;
        case PH_CAGE_FACE: return d == 0 ? lv.F : 0;
        case PH_CAGE_ZERO: return d == 0 ? lv.V : 0;
        case PH_CAGE_EDGE: return d == 0 ? lv.H : 0;
        case PH_CAGE_VERT: return d == 0 ? (lv.H > lv.V ? lv.H : lv.V) : 0;
        case PH_A: return d >= 1 ? lv.H : 0;
        case PH_A_CREASE: return d >= 1 ? lv.C : 0;
        case PH_CREASE_STATS: return d >= 1 ? lv.C : 0;
        case PH_SHAPE_NEXT: return d + 1 < bc.depth ? lv.V : 0;
        case PH_V: return d >= 2 ? bc.lv[d - 1].V : 0;
        case PH_B: return d == 1 ? (lv.H > lv.V ? lv.H : lv.V) : (d >= 2 ? lv.H : 0);
        case PH_ADJ_EDGE: return lv.H;
        case PH_ADJ_FACE: return d == 0 ? lv.F : 0;
        case PH_ADJ_VERT: return d == 0 ? lv.V : lv.H;
        case PH_ZERO3: return d == 1 && bc.depth >= 3 ? bc.lv[2].V : 0;
        case PH_CREASE_STATS_NEXT: return d >= 1 && d + 1 < bc.depth ? bc.lv[d + 1].C : 0;
        case PH_DIST: return d == 0 ? dist_points(bc) : 0;
        case PH_AF: return d >= 2 ? lv.F : 0;
        case PH_ADJ_FSTEP: return d >= 2 ? lv.F : 0;
        default: return 0;
    }
}

static void free_batch(ccs_Batch* b) {
    if (!b) return;
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(b->dCages); cudaFree(b->dTiles);
    cudaFree(b->cHe); cudaFree(b->cV2h); cudaFree(b->cE2h); cudaFree(b->cF2h); cudaFree(b->cFsz);
    cudaFree(b->cCr); cudaFree(b->cUv); cudaFree(b->cagePts);
    cudaFree(b->he); cudaFree(b->cr); cudaFree(b->pts); cudaFree(b->work); cudaFree(b->gradCage);
    cudaFree(b->stats);
    cudaFree(b->sync);
    if (b->ownStream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

template <class T>
static bool bmalloc(T** p, int64_t n) {
    return cudaMalloc((void**)p, sizeof(T) * (size_t)(n > 0 ? n : 1)) == cudaSuccess;
}

static int batch_create(const cc_Mesh* const* cages, const int32_t* depths, int32_t count, uint32_t flags,
                        ccs_Batch** out) {
    if (!out || !cages || !depths || count <= 0) return CCS_ERR_ARG;
    *out = nullptr;
    if (flags & CCS_FLAG_NO_UV) return CCS_ERR_UNSUPPORTED;
    ccs_Batch* b = new (std::nothrow) ccs_Batch();
    if (!b) return CCS_ERR_ALLOC;
    b->count = count;
    b->flags = flags;
    b->host.resize(count);
    int64_t oHe = 0, oCr = 0, oUv = 0, oV = 0, oE = 0, oF = 0;
    for (int32_t c = 0; c < count; ++c) {
        const cc_Mesh* m = cages[c];
        const int32_t D = depths[c];
        if (D < 1 || D > kMaxBatchDepth) { delete b; return CCS_ERR_ARG; }
        int st = validate_cage_ex(m);
        if (st != CCS_OK) { delete b; return st; }
        if (!twins_consistent_ex(m)) { delete b; return CCS_ERR_UNSUPPORTED; }
        std::vector<Level> lv;
        st = level_counts_ex(m, D, &lv);
        if (st != CCS_OK) { delete b; return st; }
        BatchCage& bc = b->host[c];
        memset(&bc, 0, sizeof bc);
        bc.depth = D;
        bc.uv = m->uvCount > 0;
        for (int d = 0; d <= D; ++d) bc.lv[d] = lv[d];
        bc.cage.V = m->vertexCount; bc.cage.U = m->uvCount; bc.cage.H = m->halfedgeCount;
        bc.cage.E = m->edgeCount; bc.cage.F = m->faceCount;
        // offsets for now; turned into device pointers below
        bc.cage.he = (int32_t*)(intptr_t)oHe; bc.cage.cr = (cc_Crease*)(intptr_t)oE;
        bc.cage.uvs = (float*)(intptr_t)oUv; bc.cage.v2h = (int32_t*)(intptr_t)oV;
        bc.cage.e2h = (int32_t*)(intptr_t)oE; bc.cage.f2h = (int32_t*)(intptr_t)oF;
        bc.cage.fsz = (int32_t*)(intptr_t)oF;
        bc.cagePt = oV;
        bc.he = b->totH; bc.cr = b->totC; bc.pt = b->totV;
        for (int d = 1; d < D; ++d) {            // level d: V(d-1) older vertices
            bc.stats[d] = b->totStats;
            b->totStats += lv[d - 1].V;
        }
        const Level& last = lv[D];
        b->totH += last.heOff + last.H;
        b->totC += last.crOff + last.C;
        b->totV += last.ptOff + last.V;
        oHe += m->halfedgeCount; oCr += m->edgeCount; oUv += m->uvCount;
        oV += m->vertexCount; oE += m->edgeCount; oF += m->faceCount;
        b->maxDepth = std::max(b->maxDepth, D);
    }
    b->totCagePts = oV;
    if (cudaGetDevice(&b->device) != cudaSuccess) { delete b; return CCS_ERR_CUDA; }
    cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, b->device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { delete b; return CCS_ERR_CUDA; }
    b->ownStream = true;
    if (!bmalloc(&b->cHe, 7 * oHe) || !bmalloc(&b->cCr, oE) || !bmalloc(&b->cUv, 2 * oUv) ||
        !bmalloc(&b->cV2h, oV) || !bmalloc(&b->cE2h, oE) || !bmalloc(&b->cF2h, oF) || !bmalloc(&b->cFsz, oF) ||
        !bmalloc(&b->cagePts, 3 * oV) || !bmalloc(&b->he, 4 * b->totH) || !bmalloc(&b->cr, b->totC) ||
        !bmalloc(&b->pts, 3 * b->totV) || !bmalloc(&b->sync, 1) || !bmalloc(&b->stats, b->totStats)) {
        free_batch(b);
        return CCS_ERR_ALLOC;
    }
    // upload the cages
    for (int32_t c = 0; c < count; ++c) {
        const cc_Mesh* m = cages[c];
        BatchCage& bc = b->host[c];
        const int64_t iHe = (int64_t)(intptr_t)bc.cage.he, iE = (int64_t)(intptr_t)bc.cage.e2h;
        const int64_t iUv = (int64_t)(intptr_t)bc.cage.uvs, iV = (int64_t)(intptr_t)bc.cage.v2h;
        const int64_t iF = (int64_t)(intptr_t)bc.cage.f2h;
        bc.cage.he = b->cHe + 7 * iHe; bc.cage.cr = b->cCr + iE; bc.cage.uvs = b->cUv + 2 * iUv;
        bc.cage.v2h = b->cV2h + iV; bc.cage.e2h = b->cE2h + iE; bc.cage.f2h = b->cF2h + iF;
        bc.cage.fsz = b->cFsz + iF; bc.cage.pts = b->cagePts + 3 * iV;
        std::vector<int32_t> fsz((size_t)m->faceCount, 0);
        for (int32_t h = 0; h < m->halfedgeCount; ++h) ++fsz[(size_t)m->halfedges[h].faceID];
        cudaStream_t st = b->stream;
        if (cudaMemcpyAsync(bc.cage.he, m->halfedges, sizeof(cc_Halfedge) * (size_t)m->halfedgeCount, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(bc.cage.cr, m->creases, sizeof(cc_Crease) * (size_t)m->edgeCount, cudaMemcpyHostToDevice, st) ||
            (m->uvCount > 0 && cudaMemcpyAsync(bc.cage.uvs, m->uvs, sizeof(float) * 2 * (size_t)m->uvCount, cudaMemcpyHostToDevice, st)) ||
            cudaMemcpyAsync(bc.cage.v2h, m->vertexToHalfedgeIDs, sizeof(int32_t) * (size_t)m->vertexCount, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(bc.cage.e2h, m->edgeToHalfedgeIDs, sizeof(int32_t) * (size_t)m->edgeCount, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(bc.cage.f2h, m->faceToHalfedgeIDs, sizeof(int32_t) * (size_t)m->faceCount, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(bc.cage.fsz, fsz.data(), sizeof(int32_t) * fsz.size(), cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(bc.cage.pts, m->vertexPoints, sizeof(float) * 3 * (size_t)m->vertexCount, cudaMemcpyHostToDevice, st) ||
            cudaStreamSynchronize(st)) {
            free_batch(b);
            return CCS_ERR_CUDA;
        }
    }
    // tile prefix sums per (depth, phase)
    const int64_t stride = (int64_t)count + 1;
    b->tiles.assign((size_t)(b->maxDepth * kPhasesPerDepth * stride), 0);
    for (int d = 0; d < b->maxDepth; ++d)
        for (int ph = 0; ph < PH_COUNT; ++ph) {
            int64_t* ts = &b->tiles[(size_t)((d * PH_COUNT + ph) * stride)];
            for (int32_t c = 0; c < count; ++c)
                ts[c + 1] = ts[c] + (phase_units(b->host[c], d, ph) + kBatchBlock - 1) / kBatchBlock;
        }
    if (!bmalloc(&b->dCages, count) || !bmalloc(&b->dTiles, (int64_t)b->tiles.size()) ||
        cudaMemcpy(b->dCages, b->host.data(), sizeof(BatchCage) * (size_t)count, cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->dTiles, b->tiles.data(), sizeof(int64_t) * b->tiles.size(), cudaMemcpyHostToDevice)) {
        free_batch(b);
        return CCS_ERR_ALLOC;
    }
    *out = b;
    return CCS_OK;
}

// gradient of every refined point and of the cage points
static bool adjoint_buffers(ccs_Batch* b) {
    if (b->work) return true;
    if (bmalloc(&b->work, 3 * b->totV) && bmalloc(&b->gradCage, 3 * b->totCagePts)) return true;
    cudaFree(b->work); cudaFree(b->gradCage);
    b->work = nullptr; b->gradCage = nullptr;
    return false;
}

static BatchArgs batch_args(ccs_Batch* b) {
    BatchArgs a;
    a.cages = b->dCages; a.tiles = b->dTiles; a.count = b->count;
    a.he = b->he; a.cr = b->cr; a.cagePts = b->cagePts; a.pts = b->pts;
    a.work = b->work; a.gradCage = b->gradCage; a.stats = b->stats; a.sync = b->sync;
    a.spinCap = kSpinCap;
    return a;
}

// A persistent launch: as many blocks as are resident at once (capped by the
// schedule's blocks per SM), never more than the phase's tiles.  Cooperative
// for the fused schedule, whose kernels meet at grid barriers.  The split
// schedule with no blocks-per-SM cap launches one block per tile instead.
template <class Kernel>
static cudaError_t launch_persistent(ccs_Batch* b, Kernel kernel, int64_t maxTiles, BatchArgs a, int d, bool coop) {
    if (maxTiles <= 0) return cudaSuccess;
    int64_t grid;
    if (!coop && b->blocksPerSM == 0) {
        // split schedule, default: one block per tile, so the hardware
        // scheduler overlaps the tiles' descriptor look-ups and gathers
        grid = std::min<int64_t>(maxTiles, 0x7fffffff);
    } else {
        int perSM = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, kBatchBlock, 0);
        if (e != cudaSuccess || perSM <= 0) return e != cudaSuccess ? e : cudaErrorLaunchOutOfResources;
        if (b->blocksPerSM > 0) perSM = std::min(perSM, b->blocksPerSM);
        grid = (int64_t)perSM * b->numSMs;
        grid = std::max<int64_t>(1, std::min<int64_t>(grid, maxTiles));
    }
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBatchBlock);
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = coop ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, a, d);
}

template <class Kernel>
static cudaError_t launch_coop(ccs_Batch* b, Kernel kernel, int64_t maxTiles, BatchArgs a, int d) {
    return launch_persistent(b, kernel, std::max<int64_t>(maxTiles, 1), a, d, true);
}

static int64_t max_tiles(const ccs_Batch* b, int d, std::initializer_list<int> phases) {
    int64_t m = 0;
    const int64_t stride = (int64_t)b->count + 1;
    for (int ph : phases) m = std::max(m, b->tiles[(size_t)((d * PH_COUNT + ph) * stride + b->count)]);
    return m;
}

enum BatchOp { BOP_REFINE = 0, BOP_POINTS = 1, BOP_ADJOINT = 2, BOP_ADJOINT_DIST = 3 };

// split schedule, forward: the sections of depth d as ordinary launches
template <bool TOPO, bool CREASED, bool DET>
static cudaError_t forward_sections(ccs_Batch* b, const BatchArgs& a, int d) {
    cudaError_t e;
    if (d == 0) {
        e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_CAGE_1>,
                              max_tiles(b, 0, {PH_CAGE_TOPO, PH_CAGE_CREASE, PH_CAGE_FACE, PH_CAGE_ZERO}), a, 0, false);
        if (e == cudaSuccess)
            e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_CAGE_2>,
                                  max_tiles(b, 0, {PH_CAGE_EDGE}), a, 0, false);
        if (e == cudaSuccess)
            e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_CAGE_3>,
                                  max_tiles(b, 0, {PH_CAGE_VERT, PH_SHAPE_NEXT}), a, 0, false);
        return e;
    }
    if (!DET && d >= 2) {
        e = launch_persistent(b, k_batch_level_ab<TOPO, CREASED>,
                              TOPO ? max_tiles(b, d, {PH_A, PH_A_CREASE, PH_SHAPE_NEXT}) : max_tiles(b, d, {PH_AF}),
                              a, d, false);
        if (e == cudaSuccess && TOPO)
            e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_LEVEL_2>,
                                  max_tiles(b, d, {PH_CREASE_STATS_NEXT}), a, d, false);
        return e;
    }
    e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_LEVEL_1>,
                          max_tiles(b, d, {PH_A, PH_A_CREASE, PH_CREASE_STATS, PH_ZERO3}), a, d, false);
    if (e == cudaSuccess)
        e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_LEVEL_2>,
                              max_tiles(b, d, {PH_V, PH_B, PH_SHAPE_NEXT}), a, d, false);
    if (e == cudaSuccess && TOPO && !DET && d == 1)
        e = launch_persistent(b, k_batch_forward_section<TOPO, CREASED, DET, SEC_LEVEL_3>,
                              max_tiles(b, d, {PH_CREASE_STATS_NEXT}), a, d, false);
    return e;
}

static cudaError_t enqueue_batch(ccs_Batch* b, int op, bool creased) {
    BatchArgs a = batch_args(b);
    cudaError_t e = cudaMemsetAsync(b->sync, 0, sizeof(GridSync), b->stream);
    if (e != cudaSuccess) return e;
    if (op == BOP_ADJOINT || op == BOP_ADJOINT_DIST) {
        e = cudaMemsetAsync(b->gradCage, 0, sizeof(float) * 3 * (size_t)b->totCagePts, b->stream);
        if (op == BOP_ADJOINT_DIST) {
            // P - T into the working buffer, but for the finest levels the
            // first adjoint step reads as P - T itself
            a.target = b->target;
            if (e == cudaSuccess)
                e = launch_persistent(b, k_batch_dist_init, max_tiles(b, 0, {PH_DIST}), a, 0, false);
        }
        for (int d = b->maxDepth - 1; d >= 0 && e == cudaSuccess; --d) {
            if (!b->split) {
                const int64_t mt = max_tiles(b, d, {PH_ADJ_EDGE, PH_ADJ_FACE, PH_ADJ_VERT});
                e = launch_coop(b, k_batch_adjoint, mt, a, d);
            } else if (d == 0) {
                e = launch_persistent(b, k_batch_adjoint_section<SEC_CAGE_1>, max_tiles(b, 0, {PH_ADJ_EDGE}), a, 0, false);
                if (e == cudaSuccess)
                    e = launch_persistent(b, k_batch_adjoint_section<SEC_CAGE_2>, max_tiles(b, 0, {PH_ADJ_FACE}), a, 0, false);
                if (e == cudaSuccess)
                    e = launch_persistent(b, k_batch_adjoint_section<SEC_CAGE_3>, max_tiles(b, 0, {PH_ADJ_VERT}), a, 0, false);
            } else if (d >= 2) {
                e = launch_persistent(b, k_batch_adj_step, max_tiles(b, d, {PH_ADJ_FSTEP}), a, d, false);
            } else {
                e = launch_persistent(b, k_batch_adjoint_section<SEC_LEVEL_1>, max_tiles(b, d, {PH_ADJ_EDGE}), a, d, false);
                if (e == cudaSuccess)
                    e = launch_persistent(b, k_batch_adjoint_section<SEC_LEVEL_2>, max_tiles(b, d, {PH_ADJ_VERT}), a, d, false);
            }
        }
        return e;
    }
    const bool topo = op == BOP_REFINE;
    const bool det = (b->flags & CCS_FLAG_DETERMINISTIC) != 0;
    if (b->split) {
        const int v = (topo ? 4 : 0) + (creased ? 2 : 0) + (det ? 1 : 0);
        for (int d = 0; d < b->maxDepth && e == cudaSuccess; ++d) {
            switch (v) {
                case 0: e = forward_sections<false, false, false>(b, a, d); break;
                case 1: e = forward_sections<false, false, true>(b, a, d); break;
                case 2: e = forward_sections<false, true, false>(b, a, d); break;
                case 3: e = forward_sections<false, true, true>(b, a, d); break;
                case 4: e = forward_sections<true, false, false>(b, a, d); break;
                case 5: e = forward_sections<true, false, true>(b, a, d); break;
                case 6: e = forward_sections<true, true, false>(b, a, d); break;
                default: e = forward_sections<true, true, true>(b, a, d); break;
            }
        }
        return e;
    }
    for (int d = 0; d < b->maxDepth && e == cudaSuccess; ++d) {
        const int64_t mt = d == 0 ? max_tiles(b, 0, {PH_CAGE_TOPO, PH_CAGE_CREASE, PH_CAGE_FACE, PH_CAGE_ZERO,
                                                      PH_CAGE_EDGE, PH_CAGE_VERT, PH_SHAPE_NEXT})
                                  : max_tiles(b, d, {PH_A, PH_A_CREASE, PH_CREASE_STATS, PH_V, PH_B, PH_SHAPE_NEXT,
                                                     PH_ZERO3, PH_CREASE_STATS_NEXT});
        const int v = (topo ? 4 : 0) + (creased ? 2 : 0) + (det ? 1 : 0);
        switch (v) {
            case 0: e = launch_coop(b, k_batch_forward<false, false, false>, mt, a, d); break;
            case 1: e = launch_coop(b, k_batch_forward<false, false, true>, mt, a, d); break;
            case 2: e = launch_coop(b, k_batch_forward<false, true, false>, mt, a, d); break;
            case 3: e = launch_coop(b, k_batch_forward<false, true, true>, mt, a, d); break;
            case 4: e = launch_coop(b, k_batch_forward<true, false, false>, mt, a, d); break;
            case 5: e = launch_coop(b, k_batch_forward<true, false, true>, mt, a, d); break;
            case 6: e = launch_coop(b, k_batch_forward<true, true, false>, mt, a, d); break;
            default: e = launch_coop(b, k_batch_forward<true, true, true>, mt, a, d); break;
        }
    }
    return e;
}

// Graph replay when possible; a cooperative launch that cannot be captured
// falls back to direct launches for the life of the batch.
static int run_batch(ccs_Batch* b, int op, bool creased) {
    const int key = op * 2 + (creased ? 1 : 0);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (b->stream) cudaStreamIsCapturing(b->stream, &cap);
    if (b->graphOk && b->stream && !(b->flags & CCS_FLAG_NO_GRAPH) && cap == cudaStreamCaptureStatusNone) {
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            bool ok = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            cudaError_t e = ok ? enqueue_batch(b, op, creased) : cudaErrorUnknown;
            if (ok) ok = cudaStreamEndCapture(b->stream, &graph) == cudaSuccess && e == cudaSuccess && graph;
            if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (!ok) {
                b->graphOk = false;
            } else {
                it = b->graphs.emplace(key, exec).first;
            }
        }
        if (b->graphOk) return cudaGraphLaunch(it->second, b->stream) == cudaSuccess ? CCS_OK : CCS_ERR_CUDA;
    }
    return enqueue_batch(b, op, creased) == cudaSuccess ? CCS_OK : CCS_ERR_CUDA;
}

struct BatchDevice {
    int prev = -1, dev;
    explicit BatchDevice(int d) : dev(d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~BatchDevice() {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
};

}  // namespace ccs

using namespace ccs;

extern "C" {

int ccs_BatchCreate_cuda(const cc_Mesh* const* cages, const int32_t* depths, int32_t count, uint32_t flags,
                         ccs_Batch** out) {
    return set_last_error(batch_create(cages, depths, count, flags, out));
}

void ccs_BatchRelease_cuda(ccs_Batch* batch) {
    if (!batch) return;
    BatchDevice g(batch->device);
    if (batch->stream) cudaStreamSynchronize(batch->stream);
    free_batch(batch);
}

int ccs_BatchRefine_cuda(ccs_Batch* batch, int mode) {
    if (!batch || (mode != CCS_POINTS_SCATTER && mode != CCS_POINTS_NOCREASES_SCATTER)) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    BatchDevice g(batch->device);
    const int st = run_batch(batch, BOP_REFINE, mode == CCS_POINTS_SCATTER);
    if (st == CCS_OK) batch->topoReady = true;
    return set_last_error(st);
}

int ccs_BatchRefinePoints_cuda(ccs_Batch* batch, int mode) {
    if (!batch || (mode != CCS_POINTS_SCATTER && mode != CCS_POINTS_NOCREASES_SCATTER)) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    if (!batch->topoReady) return set_last_error(CCS_ERR_STATE);
    BatchDevice g(batch->device);
    return set_last_error(run_batch(batch, BOP_POINTS, mode == CCS_POINTS_SCATTER));
}

int ccs_BatchAdjointPoints_cuda(ccs_Batch* batch) {
    if (!batch) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    if (!batch->topoReady) return set_last_error(CCS_ERR_STATE);
    BatchDevice g(batch->device);
    if (!adjoint_buffers(batch)) return set_last_error(CCS_ERR_ALLOC);
    return set_last_error(run_batch(batch, BOP_ADJOINT, true));
}

int ccs_BatchAdjointDistance_cuda(ccs_Batch* batch, const float* target) {
    if (!batch || !target) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    if (!batch->topoReady) return set_last_error(CCS_ERR_STATE);
    BatchDevice g(batch->device);
    if (!adjoint_buffers(batch)) return set_last_error(CCS_ERR_ALLOC);
    if (batch->target != target) {
        // this operation's graph holds the target's address: capture anew
        auto it = batch->graphs.find(BOP_ADJOINT_DIST * 2 + 1);
        if (it != batch->graphs.end()) {
            cudaGraphExecDestroy(it->second);
            batch->graphs.erase(it);
        }
        batch->target = target;
    }
    return set_last_error(run_batch(batch, BOP_ADJOINT_DIST, true));
}

int ccs_BatchGetArrays_cuda(ccs_Batch* batch, ccs_BatchArrays* out) {
    if (!batch || !out) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    BatchDevice g(batch->device);
    if (!adjoint_buffers(batch)) return set_last_error(CCS_ERR_ALLOC);
    out->halfedges = batch->he;
    out->creases = batch->cr;
    out->points = batch->pts;
    out->cagePoints = batch->cagePts;
    out->gradPoints = batch->work;
    out->gradCagePoints = batch->gradCage;
    out->halfedgeCount = batch->totH;
    out->creaseCount = batch->totC;
    out->pointCount = batch->totV;
    out->cagePointCount = batch->totCagePts;
    return set_last_error(CCS_OK);
}

int ccs_BatchCageInfo_cuda(const ccs_Batch* batch, int32_t cage, ccs_BatchCageInfo* out) {
    if (!batch || !out || cage < 0 || cage >= batch->count) return set_last_error(CCS_ERR_ARG);
    const BatchCage& bc = batch->host[(size_t)cage];
    const Level& last = bc.lv[bc.depth];
    out->depth = bc.depth;
    out->cagePointOffset = bc.cagePt;
    out->cagePointCount = bc.cage.V;
    out->halfedgeOffset = bc.he;
    out->halfedgeCount = last.heOff + last.H;
    out->creaseOffset = bc.cr;
    out->creaseCount = last.crOff + last.C;
    out->pointOffset = bc.pt;
    out->pointCount = last.ptOff + last.V;
    out->finestPointOffset = bc.pt + last.ptOff;
    out->finestPointCount = last.V;
    return set_last_error(CCS_OK);
}

int ccs_BatchSetStream_cuda(ccs_Batch* batch, void* stream) {
    if (!batch) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    BatchDevice g(batch->device);
    if (batch->stream) cudaStreamSynchronize(batch->stream);
    if (batch->ownStream && batch->stream) cudaStreamDestroy(batch->stream);
    batch->stream = (cudaStream_t)stream;
    batch->ownStream = false;
    return set_last_error(CCS_OK);
}

int ccs_BatchSetSchedule_cuda(ccs_Batch* batch, int32_t blocksPerSM) {
    if (!batch || blocksPerSM < 0) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    if (batch->blocksPerSM != blocksPerSM) {
        for (auto& kv : batch->graphs) cudaGraphExecDestroy(kv.second);
        batch->graphs.clear();
        batch->blocksPerSM = blocksPerSM;
    }
    return set_last_error(CCS_OK);
}

int ccs_BatchSetLaunchMode_cuda(ccs_Batch* batch, int32_t split) {
    if (!batch || split < 0 || split > 1) return set_last_error(CCS_ERR_ARG);
    std::lock_guard<std::mutex> lock(batch->mu);
    if (batch->split != (split != 0)) {
        for (auto& kv : batch->graphs) cudaGraphExecDestroy(kv.second);
        batch->graphs.clear();
        batch->split = split != 0;
    }
    return set_last_error(CCS_OK);
}

int ccs_BatchSynchronize_cuda(ccs_Batch* batch) {
    if (!batch) return set_last_error(CCS_ERR_ARG);
    BatchDevice g(batch->device);
    if (cudaStreamSynchronize(batch->stream) != cudaSuccess) return set_last_error(CCS_ERR_CUDA);
    GridSync gs;
    if (cudaMemcpy(&gs, batch->sync, sizeof gs, cudaMemcpyDeviceToHost) != cudaSuccess) return set_last_error(CCS_ERR_CUDA);
    return set_last_error(gs.err ? CCS_ERR_TIMEOUT : CCS_OK);
}

int ccs_BarrierTimeoutSelfTest_cuda(void) {
    GridSync* gs = nullptr;
    if (cudaMalloc((void**)&gs, sizeof(GridSync)) != cudaSuccess) return set_last_error(CCS_ERR_ALLOC);
    int st = CCS_ERR_CUDA;
    GridSync h{0u, 0u, 0};
    if (cudaMemcpy(gs, &h, sizeof h, cudaMemcpyHostToDevice) == cudaSuccess) {
        k_barrier_timeout_probe<<<1, 32>>>(gs, 1u << 14);
        if (cudaDeviceSynchronize() == cudaSuccess && cudaMemcpy(&h, gs, sizeof h, cudaMemcpyDeviceToHost) == cudaSuccess)
            st = h.err == CCS_ERR_TIMEOUT ? CCS_ERR_TIMEOUT : CCS_OK;
    }
    cudaFree(gs);
    return set_last_error(st);
}

int ccs_BatchDownload_cuda(ccs_Batch* batch, int32_t cage, cc_Subd* subd) {
    if (!batch || !subd || cage < 0 || cage >= batch->count) return set_last_error(CCS_ERR_ARG);
    const BatchCage& bc = batch->host[(size_t)cage];
    if (subd->maxDepth != bc.depth || !subd->halfedges || !subd->creases || !subd->vertexPoints)
        return set_last_error(CCS_ERR_ARG);
    BatchDevice g(batch->device);
    const Level& last = bc.lv[bc.depth];
    const int64_t nH = last.heOff + last.H, nC = last.crOff + last.C, nV = last.ptOff + last.V;
    cudaStream_t st = batch->stream;
    if (cudaMemcpyAsync(subd->halfedges, batch->he + 4 * bc.he, 16 * (size_t)nH, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(subd->creases, batch->cr + bc.cr, sizeof(cc_Crease) * (size_t)nC, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(subd->vertexPoints, batch->pts + 3 * bc.pt, 12 * (size_t)nV, cudaMemcpyDeviceToHost, st) ||
        cudaStreamSynchronize(st))
        return set_last_error(CCS_ERR_CUDA);
    return set_last_error(CCS_OK);
}

}  // extern "C"
