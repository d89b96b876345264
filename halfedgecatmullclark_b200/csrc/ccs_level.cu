// ccs_level.cu -- refinement steps for quad levels (depth d >= 1).
//
// Default pass, depth d >= 2: one launch per step, k_level_fq (one thread
// per depth-d face, the four faces of a parent quad in a quad of lanes):
//   - the face's four records (one 64-byte read), then every load they
//     allow: the four vertex points, crease sharpness, the corner's ring
//     statistics, across the two parent edges the twin quads' other
//     vertices;
//   - the face's 16 child records (+ UV codes) through a swizzled shared
//     tile (24 KB for a block of 96 faces) and TMA tensor stores of 32-row
//     boxes, issued first and left to drain while the points are computed (no
//     multicast);
//   - its face point, the inner edge it shares with the next lane (that
//     lane's face point by shuffle), its two outer edge points (the twin
//     face rebuilt), all in the reference's operation order and stored once;
//   - its four vertex shares: a face centre's four summed by the quad's lane
//     0 and stored, an edge midpoint's pair and the corner's share by float
//     atomics into slots the previous step cleared; it clears the slots of
//     the next step;
//   - extra blocks refine the creases and add the next level's crease
//     statistics.
// The points-only call runs the same kernel without the records.  k_level_ab
// (tile_level_ab: one thread per parent halfedge, a parent quad's 16
// children in a 16-lane group) is the same step for 12-byte records and for
// levels without a tensor map.
// Depth 1 (children of n-gons, no 16-lane structure), cages without kept
// statistics, and the deterministic pass run the step as kernel A
// (k_level_a: records, face and edge points, clearing; for the exact pass at
// depth >= 2 k_level_fq without its vertex shares) then a vertex pass:
//   default (k_level_b): the vertex shares as above, read back from memory;
//   deterministic (CCS_FLAG_DETERMINISTIC): every vertex summed by one thread
//      in increasing halfedge order, the reference's one-thread order --
//      bit-identical points.  Depth >= 2: k_level_fq_exact (one thread per
//      face: face centres summed in the quad of lanes, edge midpoints by the
//      parent pair's owner with the twin side's shares rebuilt; from depth 3
//      also the grandparent's centre and edge midpoints) beside k_level_v
//      (one ring walk per remaining older vertex -- of depth d-1, or of
//      depth d-2 from depth 3 -- on a second stream).  Depth 1:
//      k_vertex_det.
//
// Face and edge points are evaluated in the reference's operation order in
// every kernel; topology, creases, UVs, face and edge points are
// bit-identical to the reference in both modes.
//
// Twin relation used here: for a twin pair (h, t), vertex(t) = vertex(next h)
// and vertex(next t) = vertex(h).  The C ABI checks this on the cage (it is
// then preserved by every refinement step) and uses the unfused kernels for
// cages that break it.
#include <cstdint>
#include <cstring>

#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBlockL = 256;

static inline unsigned nblocksL(int64_t n) { return (unsigned)((n + kBlockL - 1) / kBlockL); }

// kernel A: blocks [0, nbH) take one tile of parent halfedges each, the
// blocks after them refine the level's creases.  (A persistent form that
// prefetched the next tile's records and left each bulk store in flight ran
// 1.5x slower at depth 5: 5 resident blocks per SM instead of 8 hid less of
// the gather latency than the extra overlap won.)
// Thread 0 of a block asks L2 for the records of tile `tile + ahead` (a bulk
// prefetch: no shared memory, no wait; nothing when that tile is past the
// level's end).
template <int RW>
__device__ __forceinline__ void prefetch_records_ahead(const int32_t* in, int64_t H, int64_t tile, int ahead) {
    if (ahead <= 0 || threadIdx.x != 0) return;
    const int64_t p0 = (tile + ahead) * kBlockL;
    if (p0 >= H) return;
    const int64_t n = (H - p0) < kBlockL ? (H - p0) : kBlockL;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                 :: "l"(in + (int64_t)RW * p0), "r"((uint32_t)(n * 4 * RW)) : "memory");
}

// blocks ahead whose records kernel A and the vertex passes prefetch (0:
// none): one wave at 8 resident blocks.  The exact pass at depth 5 of the
// headline workload: kernel A 0.377 -> 0.348 ms, its face-centre and
// edge-midpoint pass 0.508 -> 0.500 ms, the refine 1.225 -> 1.177 ms
#ifndef CCS_A_PREFETCH_AHEAD
#define CCS_A_PREFETCH_AHEAD 1184
#endif
#ifndef CCS_B_PREFETCH_AHEAD
#define CCS_B_PREFETCH_AHEAD 1184
#endif

#ifndef CCS_A_MIN_BLOCKS
#define CCS_A_MIN_BLOCKS 8
#endif
template <int RW, bool TOPO, bool UV, bool CREASED>
__global__ void __launch_bounds__(kBlockL, CCS_A_MIN_BLOCKS)
k_level_a(LevelArgs a) {
    const int nbH = (a.H + kBlockL - 1) / kBlockL;
    if ((int)blockIdx.x >= nbH) {
        if (!TOPO) return;
        const int64_t i = (int64_t)(blockIdx.x - nbH) * kBlockL + threadIdx.x;
        if (i < a.C) {
            const float2 sh = crease_item(a.crIn, a.crOut, (int32_t)i);
            if (a.statsNext) crease_stats_next<RW>(a, (int32_t)i, sh);
        }
        return;
    }
    prefetch_records_ahead<RW>(a.in, a.H, blockIdx.x, CCS_A_PREFETCH_AHEAD);
    __shared__ __align__(128) int32_t tile[kBlockL * 4 * RW];
    tile_level_a<kBlockL, RW, TOPO, UV, true, CREASED>(a, (int64_t)blockIdx.x * kBlockL, tile);
    // the slots the step after next accumulates into (zeroNextN = 0: none)
    for (int64_t i = (int64_t)blockIdx.x * kBlockL + threadIdx.x; i < a.zeroNextN; i += (int64_t)nbH * kBlockL)
        a.zeroNext[i] = 0.0f;
}

// depth d >= 2, default pass: kernel A and the vertex pass in one launch
// (tile_level_ab); blocks after the halfedge tiles refine the creases
#ifndef CCS_AB_MIN_BLOCKS
#define CCS_AB_MIN_BLOCKS 6
#endif
// where k_level_ab writes its child records (tile_level_ab's EARLY): 2 =
// first, the tensor store left to drain while the points are computed
// (measured at depth 5 of the headline workload: 0.480 ms, against 0.485
// ms after the record's gathers are issued (1) and 0.489 ms after the
// points (0); letting only warp 0 wait for the tile at a split named
// barrier added spills and measured 0.486 ms)
#ifndef CCS_AB_EARLY_STORE
#define CCS_AB_EARLY_STORE 2
#endif
// blocks ahead whose records k_level_ab asks L2 to fetch (0: none): one
// wave of the grid, 148 SMs x 6 resident blocks.  Measured at depth 5 of the
// headline workload: 0.478 -> 0.455 ms for the full step and 0.346 ->
// 0.317 ms for the points-only step, the same for 444 to 1776 blocks ahead
#ifndef CCS_AB_PREFETCH_AHEAD
#define CCS_AB_PREFETCH_AHEAD 888
#endif
template <int RW, bool TOPO, bool UV, bool CREASED, bool TMAP>
__global__ void __launch_bounds__(kBlockL, CCS_AB_MIN_BLOCKS)
k_level_ab(LevelArgs a, const __grid_constant__ CUtensorMap childMap) {
    chain_wait_then_release();
    const int nbH = (a.H + kBlockL - 1) / kBlockL;
    if ((int)blockIdx.x >= nbH) {
        if (!TOPO) return;
        const int64_t i = (int64_t)(blockIdx.x - nbH) * kBlockL + threadIdx.x;
        if (i < a.C) {
            const float2 sh = crease_item(a.crIn, a.crOut, (int32_t)i);
            if (a.statsNext) crease_stats_next<RW>(a, (int32_t)i, sh);
        }
        return;
    }
    // the records of the tile about one wave ahead, fetched into L2 while
    // this one runs
    prefetch_records_ahead<RW>(a.in, a.H, blockIdx.x, CCS_AB_PREFETCH_AHEAD);
    __shared__ __align__(1024) int32_t tile[TOPO ? kBlockL * 4 * RW : 4];
    // one tile per block: the child records' store is issued first and left
    // to drain while the points are computed
    tile_level_ab<kBlockL, RW, TOPO, UV, CREASED, TMAP, CCS_AB_EARLY_STORE>(
        a, (int64_t)blockIdx.x * kBlockL, tile, (int64_t)nbH * kBlockL, &childMap);
}

// ---------------------------------------------------------------------------
// quad level d >= 2, one thread per depth-d face: the whole step d -> d+1
// (TOPO) or its points only
// ---------------------------------------------------------------------------
// At depth d >= 2 the halfedges 16 G + 4 j + k are child k of the children
// j = 0..3 of the depth-(d-1) face G (CatmullClark.h:2760-2795), on 9
// points: the corner C_j = vertex(16 G + 4 j) (an older vertex: its ring
// statistics are in `ostats`), the midpoint M_j = vertex(16 G + 4 j + 1) =
// vertex(16 G + 4 (j+1) + 3) of parent edge j and the centre Z = vertex(16 G
// + 4 j + 2); face j runs C_j, M_j, Z, M_{j-1}.  The refinement also fixes
// the inner twins (twin(4 j + 1) = 4 (j+1) + 2: one edge, inner edge j), the
// two halves of parent edge j (edges e(4 j) and e(4 (j+1) + 3) = e(4 j) ^ 1)
// and the twin side of parent edge j: child 3 of one face and child 0 of the
// next face of one parent quad, whose centre the two rebuilt twin faces
// share (CatmullClark.h:2778-2781).
// Lane j of a quad of lanes takes face j: its face point, inner edge j with
// the next lane's face point, its two outer edges (the twin face rebuilt from
// the twin quad's other two vertices, as tile_level_ab does) and its four
// vertex shares.  The values of other lanes it needs -- the next lane's face
// point and midpoint share, the previous lane's inner edge point and twin
// centre, the centre's four shares -- come by shuffles.  Every value is
// evaluated with the same operations in the same order as tile_level_ab.
// Stores: the face point, inner edge j, the outer edge points it owns and,
// by lane 0, the centre (shares summed in face order); float atomics: the
// corner's share and midpoint M_j's pair (j, 1) + (j+1, 3), except where
// they meet inside a grandparent's 16 lanes (fq_points).  Against the
// lane-per-halfedge tile this evaluates every face and inner edge point once,
// needs 24 shuffles per face instead of about 36 per halfedge and takes no
// per-lane branches on the child position.
// TOPO (16-byte records): the face's 16 child records (tile_level_ab's rules)
// go through a 128-byte swizzled shared tile to TMA tensor stores of
// kChildBoxRows-row boxes issued before the points are evaluated; the extra
// blocks refine the creases.  The vertex slots [0, V) of depth d+1 must be
// zero on entry; every thread clears its share of `zeroNext`.
static constexpr int kBlockF = 128;                      // faces per block of the points-only step

// Resident blocks and the L2 prefetch of the records one wave ahead (blocks
// of 128 faces; the full step's own block size below).
// Depth 5 of the headline workload: 7 blocks (70 registers) against 6 and 8
// the same for the full step and 0.221 against 0.232 ms (8, 64 registers)
// for the points-only step; the prefetch 0.236 -> 0.221 ms for the
// points-only step, the full step the same at 1036 blocks ahead and 3 %
// slower at 2072.
#ifndef CCS_FQ_MIN_BLOCKS
#define CCS_FQ_MIN_BLOCKS 7
#endif
#ifndef CCS_FQ_PREFETCH_AHEAD
#define CCS_FQ_PREFETCH_AHEAD 1036
#endif

// The full step's blocks (BF faces: a multiple of 32 for whole warps and of
// 16 for whole grandparent groups): the 16 BF child records' tile in shared
// memory bounds the resident blocks (128 faces: 32 KB, 6 blocks per SM).
// Depth 5 of the headline workload, with the tile stored as 32-row boxes:
// 64 faces 0.375 ms, 96 (24 KB, 9 blocks) 0.373, 128 0.375, 160 0.379 ms;
// with 128-row boxes 128 faces took 0.382 ms.
#ifndef CCS_FQT_FACES
#define CCS_FQT_FACES 96
#endif
#ifndef CCS_FQT_MIN_BLOCKS
#define CCS_FQT_MIN_BLOCKS 9
#endif
// VERTS = false: kernel A of the exact pass (child records, face and edge
// points; the vertex points are summed afterwards in the reference's order).
template <int RW, bool TOPO, bool UV, bool CREASED, int BF, bool VERTS = true>
__global__ void __launch_bounds__(BF, TOPO ? CCS_FQT_MIN_BLOCKS : CCS_FQ_MIN_BLOCKS)
k_level_fq(LevelArgs a, const __grid_constant__ CUtensorMap childMap) {
    static_assert(!TOPO || RW == 4, "the child records go out through the 16-byte record tensor map");
    static_assert(BF % 32 == 0, "whole warps: every lane of a warp takes part in the shuffles");
    chain_wait_then_release();
    const int64_t nF = (int64_t)a.H >> 2;                  // depth-d faces (H = 16 n at d >= 2)
    const int nbF = (int)((nF + BF - 1) / BF);
    if (TOPO && (int)blockIdx.x >= nbF) {
        const int64_t i = (int64_t)(blockIdx.x - nbF) * BF + threadIdx.x;
        if (i < a.C) {
            const float2 sh = crease_item(a.crIn, a.crOut, (int32_t)i);
            if (a.statsNext) crease_stats_next<RW>(a, (int32_t)i, sh);
        }
        return;
    }
    const int64_t f = (int64_t)blockIdx.x * BF + threadIdx.x;
    if (threadIdx.x == 0 && CCS_FQ_PREFETCH_AHEAD > 0) {
        const int64_t p0 = ((int64_t)blockIdx.x + CCS_FQ_PREFETCH_AHEAD * kBlockF / BF) * BF;
        if (p0 < nF) {
            const int64_t n = (nF - p0) < BF ? (nF - p0) : BF;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(a.in + (int64_t)RW * 4 * p0), "r"((uint32_t)(n * 16 * RW)) : "memory");
        }
    }
    const bool valid = f < nF;                             // the four lanes of a quad agree
    const int32_t h0 = (int32_t)(4 * f);
    int4 r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = make_int4(-1, 0, 0, 0);
    if (valid) load_face_records<RW>(a.in, f, r);

    if constexpr (TOPO) {
        // child m of halfedge h0 + k is child record 16 f + 4 k + m: row 2 f + k / 2
        // of the level's 128-byte rows, chunk 4 (k & 1) + m
        __shared__ __align__(1024) int4 tile[BF * 16];
        float u[4], v[4];
        if (UV) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                u[k] = uv_dec_fast((uint32_t)r[k].w);
                v[k] = uv_dec_fast((uint32_t)r[k].w >> 16);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int kn = (k + 1) & 3, ko = (k + 2) & 3, kp = (k + 3) & 3;
            const int32_t h = h0 + k, next = h0 + kn, prev = h0 + kp;
            const int32_t tw = r[k].x, ed = r[k].y, ptw = r[kp].x, ped = r[kp].y;
            int4 c[4];
            c[0] = make_int4(child(qnext(tw), 3), 2 * ed + (h > tw ? 0 : 1), r[k].z, r[k].w);
            c[1] = make_int4(child(next, 2), 2 * a.E + h, a.V + a.F + ed, 0);
            c[2] = make_int4(child(prev, 1), 2 * a.E + prev, a.V + (int32_t)f, 0);
            c[3] = make_int4(child(ptw, 0), 2 * ped + (prev > ptw ? 1 : 0), a.V + a.F + ped, 0);
            if (UV) {
                c[1].w = (int32_t)uv_enc_fast(flerp(u[k], u[kn], 0.5f), flerp(v[k], v[kn], 0.5f));
                c[2].w = (int32_t)uv_enc_fast(fquarter(fadd(fadd(fadd(u[k], u[kn]), u[ko]), u[kp])),
                                              fquarter(fadd(fadd(fadd(v[k], v[kn]), v[ko]), v[kp])));
                c[3].w = (int32_t)uv_enc_fast(flerp(u[k], u[kp], 0.5f), flerp(v[k], v[kp], 0.5f));
            }
            // rows 2 t and 2 t + 8 have the same swizzle, so lanes 4..7 of each
            // quarter-warp write the children in the order 1 0 3 2: the eight
            // 16-byte stores of a quarter-warp then land on distinct banks
            // (depth 5 of the headline workload: 0.421 -> 0.417 ms)
            const int row = 2 * threadIdx.x + (k >> 1);
            const int flip = (threadIdx.x >> 2) & 1;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int4 cm = flip ? c[m ^ 1] : c[m];
                tile[row * 8 + ((4 * (k & 1) + (m ^ flip)) ^ (row & 7))] = cm;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0)
            tensor_store_rows_async(&childMap, tile, (int32_t)(2 * (int64_t)blockIdx.x * BF), 2 * BF,
                                    (int32_t)(a.H >> 1));
    }

    fq_points<RW, CREASED, VERTS>(a, f, valid, r);

    // the slots the step after next accumulates into
    const int64_t nT = (int64_t)nbF * BF;
    if (VERTS)
        for (int64_t i = f; i < a.zeroNextN; i += nT) a.zeroNext[i] = 0.0f;
    if (TOPO && threadIdx.x == 0) bulk_wait_read();
}

// default vertex pass: one tile of halfedges per block
template <int RW, bool CREASED, bool STRUCT>
__global__ void __launch_bounds__(kBlockL, 8)
k_level_b(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout) {
    prefetch_records_ahead<RW>(L.he, L.H, blockIdx.x, CCS_B_PREFETCH_AHEAD);
    tile_level_b<RW, CREASED, STRUCT>(L, pin, pout, (int64_t)blockIdx.x * kBlockL);
}

// exact vertex pass (d >= 2): face centres and edge midpoints, one thread
// per depth-d face, its records prefetched into L2 one wave ahead
#ifndef CCS_FQ_EXACT_PREFETCH_AHEAD
#define CCS_FQ_EXACT_PREFETCH_AHEAD 1036
#endif
#ifndef CCS_FQ_EXACT_MIN_BLOCKS
#define CCS_FQ_EXACT_MIN_BLOCKS 7
#endif
template <int RW, bool CREASED, bool GRAND>
__global__ void __launch_bounds__(kBlockF, CCS_FQ_EXACT_MIN_BLOCKS)
k_level_fq_exact(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout) {
    if (threadIdx.x == 0 && CCS_FQ_EXACT_PREFETCH_AHEAD > 0) {
        const int64_t nF = (int64_t)L.H >> 2;
        const int64_t p0 = ((int64_t)blockIdx.x + CCS_FQ_EXACT_PREFETCH_AHEAD) * kBlockF;
        if (p0 < nF) {
            const int64_t n = (nF - p0) < kBlockF ? (nF - p0) : kBlockF;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(L.he + 4 * RW * p0), "r"((uint32_t)(n * 16 * RW)) : "memory");
        }
    }
    tile_face_exact<RW, CREASED, GRAND>(L, pin, pout, (int64_t)blockIdx.x * kBlockF);
}

// exact vertex pass (d >= 2): one thread per older vertex v < Vold (its own
// launch, on a second stream beside k_level_fq_exact, which sums the rest)
template <int RW, bool CREASED>
__global__ void __launch_bounds__(kBlockL)
k_level_v(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout, int32_t Vold) {
    const int64_t v = (int64_t)blockIdx.x * kBlockL + threadIdx.x;
    if (v < Vold) old_vertex_item<RW, CREASED>(L, pin, pout, (int32_t)v);
}

// ring statistics of the older vertices of level d: shape (valence and
// boundary, one thread per vertex, no level data read), then the creased
// edges' sharpness (one thread per crease of the level, float atomics)
__global__ void __launch_bounds__(kBlockL)
k_shape_stats(CageTables t, int32_t d, float4* __restrict__ out, int32_t Vold) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Vold) shape_stats_item(t, d, out, (int32_t)i);
}

template <int RW>
__global__ void __launch_bounds__(kBlockL)
k_crease_stats(QuadView<RW> L, float4* __restrict__ out, int32_t Vold) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.C) crease_stats_item(L, Vold, out, (int32_t)i);
}

// Shape statistics of every level 1..D-1 in one launch: item i of the packed
// table (level j + 1 in [off[j], off[j + 1]), V(j) entries) is vertex
// i - off[j] of level j + 1.
static constexpr int kMaxShapeLevels = 32;
struct ShapeLevels {
    int64_t off[kMaxShapeLevels + 1];
    int32_t n = 0;
};

__device__ __forceinline__ void shape_levels_item(const CageTables& t, float4* __restrict__ stats,
                                                  const ShapeLevels& sl, int64_t i) {
    int j = 0;
    while (j + 1 < sl.n && i >= sl.off[j + 1]) ++j;
    shape_stats_item(t, j + 1, stats + sl.off[j], (int32_t)(i - sl.off[j]));
}

// The second stream's share of the cage step in one launch: blocks
// [0, nbT) refine the cage's halfedges (4 children each, + UV codes),
// [nbT, nbT + nbC) its creases, the rest build the shape half of every
// level's ring statistics (nbT = nbC = 0: the statistics alone).
template <int RW, bool UV>
__global__ void __launch_bounds__(kBlockL)
k_cage_side(CageTables t, int32_t* __restrict__ recOut, const cc_Crease* __restrict__ crIn,
            cc_Crease* __restrict__ crOut, int32_t C, float4* __restrict__ stats, ShapeLevels sl, int nbT,
            int nbC) {
    const int b = blockIdx.x;
    if (b < nbT) {
        const int64_t c = (int64_t)b * kBlockL + threadIdx.x;
        if (c < 4 * (int64_t)t.n.H) cage_topology_item<RW, true, UV>(t, recOut, c);
        return;
    }
    if (b < nbT + nbC) {
        const int64_t e = (int64_t)(b - nbT) * kBlockL + threadIdx.x;
        if (e < C) crease_item(crIn, crOut, (int32_t)e);
        return;
    }
    const int64_t i = (int64_t)(b - nbT - nbC) * kBlockL + threadIdx.x;
    if (i < sl.off[sl.n]) shape_levels_item(t, stats, sl, i);
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
// The packed layout of the statistics of levels 1..D-1 (false: none kept).
static bool shape_levels(const Ctx& c, ShapeLevels* sl) {
    const int n = c.D - 1;
    if (!c.stats || !c.statsOff || n < 1 || n > kMaxShapeLevels) return false;
    sl->n = n;
    for (int j = 0; j < n; ++j) sl->off[j] = c.statsOff[j + 1];
    sl->off[n] = c.statsOff[n] + c.lv[n - 1].V;
    return true;
}

// One k_cage_side launch on `s`: with `topo` the cage's topology and creases
// beside the statistics (profiled as "cage_side"), else the statistics alone
// ("ring_stats" at level 0, every level).
template <int RW, bool UV>
static void cage_side_launch(const Ctx& c, const ShapeLevels& sl, bool topo, cudaStream_t s) {
    const int32_t C = c.lv[0].C;
    const int nbT = topo ? (int)nblocksL(4 * (int64_t)c.lv[0].H) : 0;
    const int nbC = topo ? (int)nblocksL(C) : 0;
    const unsigned nb = (unsigned)(nbT + nbC) + nblocksL(sl.off[sl.n]);
    c.prof->begin(s, topo ? CCS_K_CAGE_SIDE : CCS_K_RING_STATS, 0, sl.off[sl.n]);
    k_cage_side<RW, UV><<<nb, kBlockL, 0, s>>>(make_cage_tables(*c.cage), c.he + (int64_t)RW * c.lv[1].heOff,
                                              c.cage->cr, c.cr + c.lv[1].crOff, C, c.stats, sl, nbT, nbC);
    c.prof->end(s);
}

static void cage_side(const Ctx& c, const ShapeLevels& sl, bool topo, bool uv, cudaStream_t s) {
    if (c.rw == 4 && uv) cage_side_launch<4, true>(c, sl, topo, s);
    else if (c.rw == 4) cage_side_launch<4, false>(c, sl, topo, s);
    else cage_side_launch<3, false>(c, sl, topo, s);
}

template <int RW>
static QuadView<RW> quad_view_l(const Ctx& c, int d) {
    QuadView<RW> L;
    const Level& lv = c.lv[d];
    L.t = make_cage_tables(*c.cage);
    L.he = c.he + (int64_t)RW * lv.heOff;
    L.cr = c.cr + lv.crOff;
    L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C;
    L.d = d;
    return L;
}

// The shape half needs no level data; the crease half reads the level's
// creases and halfedges and must follow the shape half.
static void shape_stats_level(const Ctx& c, int d, cudaStream_t s) {
    float4* out = stats_at(c, d);
    if (!out || d < 1) return;
    const int32_t Vold = c.lv[d - 1].V;
    c.prof->begin(s, CCS_K_RING_STATS, d, Vold);
    k_shape_stats<<<nblocksL(Vold), kBlockL, 0, s>>>(make_cage_tables(*c.cage), d, out, Vold);
    c.prof->end(s);
}

template <int RW>
static void crease_stats_level(const Ctx& c, int d, cudaStream_t s) {
    float4* out = stats_at(c, d);
    if (!out || d < 1 || c.lv[d].C <= 0) return;
    const QuadView<RW> L = quad_view_l<RW>(c, d);
    c.prof->begin(s, CCS_K_CREASE_STATS, d, L.C);
    k_crease_stats<RW><<<nblocksL(L.C), kBlockL, 0, s>>>(L, out, c.lv[d - 1].V);
    c.prof->end(s);
}

template <int RW>
static void ring_stats_level(const Ctx& c, int d, cudaStream_t s) {
    shape_stats_level(c, d, s);
    crease_stats_level<RW>(c, d, s);
}

cudaError_t run_ring_stats(const Ctx& c) {
    ShapeLevels sl;
    if (shape_levels(c, &sl)) {
        cage_side(c, sl, false, false, c.stream);       // the shape half of every level
        for (int d = 1; d < c.D; ++d) {
            if (c.rw == 4) crease_stats_level<4>(c, d, c.stream);
            else crease_stats_level<3>(c, d, c.stream);
        }
        return cudaGetLastError();
    }
    for (int d = 1; d < c.D; ++d) {
        if (c.rw == 4) ring_stats_level<4>(c, d, c.stream);
        else ring_stats_level<3>(c, d, c.stream);
    }
    return cudaGetLastError();
}

// Work on the second stream between a fork from and a join into the main
// stream; on the main stream itself when there is no second stream.
struct Fork {
    const Ctx& c;
    bool on;
    explicit Fork(const Ctx& cx, bool want = true) : c(cx), on(want && cx.side && cx.forkEv && cx.joinEv) {
        if (on) {
            cudaEventRecord(c.forkEv, c.stream);
            cudaStreamWaitEvent(c.side, c.forkEv, 0);
        }
    }
    cudaStream_t stream() const { return on ? c.side : c.stream; }
    void join() {
        if (on) {
            cudaEventRecord(c.joinEv, c.side);
            cudaStreamWaitEvent(c.stream, c.joinEv, 0);
            on = false;
        }
    }
};

// The crease half of depth d+1's ring statistics from the crease items of
// the step d -> d+1 (needs the shape half written first).
static void fold_crease_stats(const Ctx& c, int d, LevelArgs& a) {
    a.statsNext = stats_at(c, d + 1);
    a.t = make_cage_tables(*c.cage);
    a.d = d;
}

// Slots [0, V(d+1)) of depth d+2: where the step d+1 -> d+2 accumulates.
static void next_slots(const Ctx& c, int d, float* pts, LevelArgs& a) {
    if (d + 2 <= c.D) {
        a.zeroNext = pts + 3 * c.lv[d + 2].ptOff;
        a.zeroNextN = 3 * (int64_t)c.lv[d + 1].V;
    }
}

template <int RW, bool CREASED>
static void level_ab(const Ctx& c, int d, bool topo, bool uv, float* pts) {
    const Level& lv = c.lv[d];
    LevelArgs a;
    a.in = c.he + (int64_t)RW * lv.heOff;
    a.out = c.he + (int64_t)RW * c.lv[d + 1].heOff;
    a.crIn = c.cr + lv.crOff;
    a.crOut = c.cr + c.lv[d + 1].crOff;
    a.pin = pts + 3 * lv.ptOff;
    a.pout = pts + 3 * c.lv[d + 1].ptOff;
    a.H = lv.H; a.V = lv.V; a.F = lv.F; a.E = lv.E; a.C = lv.C;
    a.d = d;
    a.ostats = stats_at(c, d);
    if (topo) fold_crease_stats(c, d, a);
    next_slots(c, d, pts, a);
    const unsigned nb = nblocksL(lv.H) + (topo ? nblocksL(lv.C) : 0u);
    c.prof->begin(c.stream, topo ? CCS_K_LEVEL_STEP : CCS_K_LEVEL_STEP_POINTS, d, lv.H);
    const bool tmap = RW == 4 && topo && c.childMaps && c.childMapOk && c.childMapOk[d];
    CUtensorMap none;
    memset(&none, 0, sizeof none);
    const CUtensorMap& map = tmap ? c.childMaps[d] : none;
    const unsigned nbf = (unsigned)((((int64_t)lv.H >> 2) + kBlockF - 1) / kBlockF);
    if (RW == 4 && topo && tmap) {
        constexpr int BF = CCS_FQT_FACES;
        const unsigned nbc = (unsigned)((((int64_t)lv.H >> 2) + BF - 1) / BF + ((int64_t)lv.C + BF - 1) / BF);
        if (uv) launch_chained(k_level_fq<4, true, true, CREASED, BF>, nbc, BF, c.stream, a, map);
        else launch_chained(k_level_fq<4, true, false, CREASED, BF>, nbc, BF, c.stream, a, map);
    } else if (topo) {
        // 12-byte records, or a level whose tensor map could not be encoded
        if (RW == 4 && uv) launch_chained(k_level_ab<RW, true, true, CREASED, false>, nb, kBlockL, c.stream, a, map);
        else launch_chained(k_level_ab<RW, true, false, CREASED, false>, nb, kBlockL, c.stream, a, map);
    } else {
        launch_chained(k_level_fq<RW, false, false, CREASED, kBlockF>, nbf, kBlockF, c.stream, a, map);
    }
    c.prof->end(c.stream);
}

template <int RW, bool CREASED>
static void level_a(const Ctx& c, int d, bool topo, bool uv, const float* pin, float* pout, bool zeroV,
                    float* clearNext = nullptr) {
    const Level& lv = c.lv[d];
    LevelArgs a;
    a.in = c.he + (int64_t)RW * lv.heOff;
    a.out = c.he + (int64_t)RW * c.lv[d + 1].heOff;
    a.crIn = c.cr + lv.crOff;
    a.crOut = c.cr + c.lv[d + 1].crOff;
    a.pin = pin;
    a.pout = pout;
    a.H = lv.H; a.V = lv.V; a.F = lv.F; a.E = lv.E; a.C = lv.C;
    a.zeroV = zeroV ? 1 : 0;
    if (topo) fold_crease_stats(c, d, a);
    if (clearNext) next_slots(c, d, clearNext, a);   // clearNext = the points of every depth
    const unsigned nb = nblocksL(lv.H) + (topo ? nblocksL(lv.C) : 0u);
    c.prof->begin(c.stream, topo ? CCS_K_LEVEL_FUSED : CCS_K_FACE_POINTS, d, lv.H);
    const bool tmap = RW == 4 && topo && c.childMaps && c.childMapOk && c.childMapOk[d];
    if (RW == 4 && d >= 2 && !zeroV && !clearNext && c.fusable && (tmap || !topo)) {
        // depth >= 2 of the exact pass: the per-face kernel without the
        // vertex shares (the same records, face and edge points).  Depth 5 of
        // the headline workload: 0.347 -> 0.317 ms with the records, 0.324 ->
        // 0.134 ms for the points-only call's face and edge points
        if (topo) {
            constexpr int BF = CCS_FQT_FACES;
            const unsigned nbc = (unsigned)((((int64_t)lv.H >> 2) + BF - 1) / BF + ((int64_t)lv.C + BF - 1) / BF);
            if (uv) launch_chained(k_level_fq<4, true, true, CREASED, BF, false>, nbc, BF, c.stream, a, c.childMaps[d]);
            else launch_chained(k_level_fq<4, true, false, CREASED, BF, false>, nbc, BF, c.stream, a, c.childMaps[d]);
        } else {
            CUtensorMap none;
            memset(&none, 0, sizeof none);
            const unsigned nbf = (unsigned)((((int64_t)lv.H >> 2) + kBlockF - 1) / kBlockF);
            launch_chained(k_level_fq<4, false, false, CREASED, kBlockF, false>, nbf, kBlockF, c.stream, a, none);
        }
    } else if (topo) {
        if (RW == 4 && uv) k_level_a<RW, true, true, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
        else k_level_a<RW, true, false, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
    } else {
        k_level_a<RW, false, false, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
    }
    c.prof->end(c.stream);
}

template <int RW, bool CREASED>
static void level_b(const Ctx& c, int d, const float* pin, float* pout) {
    QuadView<RW> L = quad_view_l<RW>(c, d);
    L.ostats = stats_at(c, d);
    c.prof->begin(c.stream, CCS_K_LEVEL_POINTS, d, L.H);
    const unsigned nb = nblocksL(L.H);
    if (d >= 2) k_level_b<RW, CREASED, true><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    else k_level_b<RW, CREASED, false><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    c.prof->end(c.stream);
}

// exact pass, d >= 2: older vertices on the second stream beside the rest
// (both read only kernel A's output and write disjoint vertex slots)
template <int RW, bool CREASED>
static void level_b_exact(const Ctx& c, int d, const float* pin, float* pout) {
    const QuadView<RW> L = quad_view_l<RW>(c, d);
    // from depth 3 the per-face pass also sums the corners that are centres
    // and edge midpoints of depth d-2 faces (vertex ids V(d-2) .. V(d-1))
    const bool grand = d >= 3 && c.fusable;
    const int32_t Vold = grand ? c.lv[d - 2].V : c.lv[d - 1].V;
    Fork f(c);
    c.prof->begin(f.stream(), CCS_K_OLD_VERTICES, d, Vold);
    k_level_v<RW, CREASED><<<nblocksL(Vold), kBlockL, 0, f.stream()>>>(L, pin, pout, Vold);
    c.prof->end(f.stream());
    c.prof->begin(c.stream, CCS_K_EXACT_POINTS, d, L.H);
    const unsigned nb = (unsigned)((((int64_t)L.H >> 2) + kBlockF - 1) / kBlockF);
    if (grand) k_level_fq_exact<RW, CREASED, true><<<nb, kBlockF, 0, c.stream>>>(L, pin, pout);
    else k_level_fq_exact<RW, CREASED, false><<<nb, kBlockF, 0, c.stream>>>(L, pin, pout);
    c.prof->end(c.stream);
    f.join();
}

// Declared in ccs_forward.cu: the one-thread-per-vertex sorted pass of one
// quad level, and the cage step.
cudaError_t run_vertex_det_level(const Ctx& c, int d, const float* pin, float* pout, bool creased);
cudaError_t run_cage_step(const Ctx& c, bool topo, bool uv, const float* cagePts, float* pout, int mode, bool det,
                          cudaStream_t topoStream);

// With the topology, the older vertices' ring statistics of every level are
// built on the way (read by the default pass and by the adjoint): the shape
// half of all levels on the second stream from the start (`shapes`, joined
// before the first crease half), the crease half of level 1 beside kernel A
// of depth 1, that of level d+1 by the crease items of the step d -> d+1.  The default pass runs depth 1 as
// kernel A + vertex pass and every deeper level as one k_level_ab launch,
// which reads the statistics of its level and clears the slots the next
// level accumulates into (depth 3's are cleared by a memset at depth 1).
template <int RW, bool CREASED>
static cudaError_t fused_levels(const Ctx& c, bool topo, bool uv, float* pts, bool det, Fork& shapes) {
#ifdef CCS_NO_LEVEL_AB
    bool ab = false;
#else
    bool ab = !det;
#endif
    for (int d = 2; d < c.D; ++d) ab = ab && stats_at(c, d) != nullptr;
    for (int d = 1; d < c.D; ++d) {
        const float* pin = pts + 3 * c.lv[d].ptOff;
        float* pout = pts + 3 * c.lv[d + 1].ptOff;
        const int step = c.prof->begin(c.stream, CCS_K_STEP, d, c.lv[d].H);
        // at depth 1 kernel A also clears the slots depth 3 accumulates into
        // (the first k_level_ab step's; each k_level_ab clears the next's)
        float* clear3 = (ab && d == 1 && c.D >= 3) ? pts : nullptr;
        if (topo && d == 1) {
            // level 1's creases come from the cage step: the crease half of
            // its statistics beside kernel A (whose crease items add level 2's)
            shapes.join();
            Fork f(c);
            crease_stats_level<RW>(c, 1, f.stream());
            level_a<RW, CREASED>(c, d, topo, uv, pin, pout, !det, clear3);
            f.join();
        } else if (ab && d >= 2) {
            level_ab<RW, CREASED>(c, d, topo, uv, pts);
            c.prof->end(c.stream, step);
            continue;
        } else {
            level_a<RW, CREASED>(c, d, topo, uv, pin, pout, !det, clear3);
        }
        if (!det) {
            level_b<RW, CREASED>(c, d, pin, pout);
        } else if (d >= 2) {
            level_b_exact<RW, CREASED>(c, d, pin, pout);
        } else {
            const cudaError_t e = run_vertex_det_level(c, d, pin, pout, CREASED);
            if (e != cudaSuccess) return e;
        }
        c.prof->end(c.stream, step);
    }
    return cudaGetLastError();
}

// `det` selects the exact pass (the reference's one-thread summation order).
cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool det) {
    const bool creased = mode == CCS_POINTS_SCATTER;
    const bool uv = c.cage->U > 0 && c.rw == 4;
    // beside the cage step's points, on the second stream: its topology and
    // creases and the shape half of every level's ring statistics, in one
    // launch when the statistics are kept
    Fork shapes(c, topo && c.stats);
    ShapeLevels sl;
    const bool side = topo && shape_levels(c, &sl);
    if (side) cage_side(c, sl, true, uv, shapes.stream());
    else if (topo)
        for (int d = 1; d < c.D; ++d) shape_stats_level(c, d, shapes.stream());
    const int step = c.prof->begin(c.stream, CCS_K_STEP, 0, c.lv[0].H);
    cudaError_t e = run_cage_step(c, topo && !side, uv, cagePts, pts + 3 * c.lv[1].ptOff, mode, det,
                                  shapes.stream());
    c.prof->end(c.stream, step);
    if (e == cudaSuccess) {
        if (c.rw == 4)
            e = creased ? fused_levels<4, true>(c, topo, uv, pts, det, shapes)
                        : fused_levels<4, false>(c, topo, uv, pts, det, shapes);
        else
            e = creased ? fused_levels<3, true>(c, topo, false, pts, det, shapes)
                        : fused_levels<3, false>(c, topo, false, pts, det, shapes);
    }
    shapes.join();
    return e;
}

}  // namespace ccs
