// ccs_level.cu -- fused refinement step for quad levels (depth d >= 1).
//
// One step d -> d+1 runs as two kernels:
//
//   A  (one thread per parent halfedge; the 4 lanes of a face are adjacent)
//      - reads the parent record with one 16-byte load (a warp reads 512
//        contiguous bytes); the face's other records come from the 3 sibling
//        lanes through shuffles;
//      - builds the 4 child records (topology + UV code) in shared memory;
//        one thread then writes the block's 16 KB tile with a single
//        cp.async.bulk store (TMA engine, no multicast);
//      - face point of its face (lanes' vertex points combined by shuffles,
//        in halfedge order), stored by the face's first lane;
//      - edge point of its edge, computed and stored by the pair's larger
//        halfedge: both halves of the edge rule, the twin face's point
//        rebuilt from the twin quad's four records (the same value, bit for
//        bit, as the twin quad's lanes store);
//      - extra blocks refine the creases of the level.
//   B  (depth d >= 2; vertex points, no atomics; two launches)
//      - k_level_v: the older vertices (v < V(d-1)), one thread per
//        vertex: one walk of the ring, every share, summed in increasing
//        halfedge order;
//      - k_level_b: one tile of halfedges per block, one thread per
//        halfedge: a face centre's 4 shares meet in 4 lanes of a 16-lane
//        group and an edge midpoint's 4 shares in the lane of the parent
//        pair's owner (the twin side's 2 shares rebuilt from face and edge
//        points), ring statistics from the known structure of refined
//        levels, sums in increasing halfedge order.
//   At depth 1 (children of n-gons) the vertex pass is one thread per vertex
//   with the ring sorted (k_vertex_det).
//
// Every float expression is evaluated in the reference's order and every sum
// in its one-thread order, so topology, creases, UVs and all points are
// bit-identical to the reference's single-threaded refinement.
//
// Twin relation used by A: for a twin pair (h, t), vertex(t) = vertex(next h)
// and vertex(next t) = vertex(h).  The C ABI checks this on the cage (it is
// then preserved by every refinement step) and uses the unfused kernels for
// cages that break it.
#include <cstdint>

#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBlockL = 256;

static inline unsigned nblocksL(int64_t n) { return (unsigned)((n + kBlockL - 1) / kBlockL); }

// kernel A: blocks [0, nbH) take one tile of parent halfedges each, the
// blocks after them refine the level's creases.
template <int RW, bool TOPO, bool UV, bool PTS, bool CREASED>
__global__ void __launch_bounds__(kBlockL)
k_level_a(LevelArgs a) {
    const int nbH = (a.H + kBlockL - 1) / kBlockL;
    if ((int)blockIdx.x >= nbH) {
        if (!TOPO) return;
        const int64_t i = (int64_t)(blockIdx.x - nbH) * kBlockL + threadIdx.x;
        if (i < a.C) crease_item(a.crIn, a.crOut, (int32_t)i);
        return;
    }
    __shared__ __align__(128) int32_t tile[kBlockL * 4 * RW];
    tile_level_a<kBlockL, RW, TOPO, UV, PTS, CREASED>(a, (int64_t)blockIdx.x * kBlockL, tile);
}

// kernel B (d >= 2): one tile of halfedges per block (face centres and edge
// midpoints)
template <int RW, bool CREASED>
__global__ void __launch_bounds__(kBlockL, 5)
k_level_b(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout) {
    tile_level_b<RW, CREASED>(L, pin, pout, (int64_t)blockIdx.x * kBlockL);
}

// kernel V (d >= 2): one thread per older vertex (a separate launch, so that
// kernel B keeps its small register footprint)
template <int RW, bool CREASED>
__global__ void __launch_bounds__(kBlockL)
k_level_v(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout, int32_t Vold) {
    const int64_t v = (int64_t)blockIdx.x * kBlockL + threadIdx.x;
    if (v < Vold) old_vertex_item<RW, CREASED>(L, pin, pout, (int32_t)v);
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
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

template <int RW, bool CREASED>
static void level_a(const Ctx& c, int d, bool topo, bool uv, const float* pin, float* pout) {
    const Level& lv = c.lv[d];
    LevelArgs a;
    a.in = c.he + (int64_t)RW * lv.heOff;
    a.out = c.he + (int64_t)RW * c.lv[d + 1].heOff;
    a.crIn = c.cr + lv.crOff;
    a.crOut = c.cr + c.lv[d + 1].crOff;
    a.pin = pin;
    a.pout = pout;
    a.H = lv.H; a.V = lv.V; a.F = lv.F; a.E = lv.E; a.C = lv.C;
    const unsigned nb = nblocksL(lv.H) + (topo ? nblocksL(lv.C) : 0u);
    c.prof->begin(c.stream, topo ? CCS_K_LEVEL_FUSED : CCS_K_FACE_POINTS, d, lv.H);
    if (topo) {
        if (RW == 4 && uv) k_level_a<RW, true, true, true, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
        else k_level_a<RW, true, false, true, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
    } else {
        k_level_a<RW, false, false, true, CREASED><<<nb, kBlockL, 0, c.stream>>>(a);
    }
    c.prof->end(c.stream);
}

template <int RW, bool CREASED>
static void level_b(const Ctx& c, int d, const float* pin, float* pout) {
    const QuadView<RW> L = quad_view_l<RW>(c, d);
    const int32_t Vold = c.lv[d - 1].V;
    // V (memory-latency bound) runs beside B (issue bound) when a second
    // stream is available: both read only kernel A's output and write
    // disjoint vertex slots
    const bool fork = c.side && c.forkEv && c.joinEv;
    cudaStream_t sv = fork ? c.side : c.stream;
    if (fork) {
        cudaEventRecord(c.forkEv, c.stream);
        cudaStreamWaitEvent(c.side, c.forkEv, 0);
    }
    c.prof->begin(sv, CCS_K_OLD_VERTICES, d, Vold);
    k_level_v<RW, CREASED><<<nblocksL(Vold), kBlockL, 0, sv>>>(L, pin, pout, Vold);
    c.prof->end(sv);
    c.prof->begin(c.stream, CCS_K_LEVEL_POINTS, d, L.H);
    k_level_b<RW, CREASED><<<nblocksL(L.H), kBlockL, 0, c.stream>>>(L, pin, pout);
    c.prof->end(c.stream);
    if (fork) {
        cudaEventRecord(c.joinEv, c.side);
        cudaStreamWaitEvent(c.stream, c.joinEv, 0);
    }
}

// Declared in ccs_forward.cu: the vertex pass of one quad level when the
// fixed-order (deterministic) sum is requested, and the cage step.
cudaError_t run_vertex_det_level(const Ctx& c, int d, const float* pin, float* pout, bool creased);
cudaError_t run_cage_step(const Ctx& c, bool topo, bool uv, const float* cagePts, float* pout, int mode, bool det);

template <int RW, bool CREASED>
static cudaError_t fused_levels(const Ctx& c, bool topo, bool uv, float* pts, bool det) {
    for (int d = 1; d < c.D; ++d) {
        const float* pin = pts + 3 * c.lv[d].ptOff;
        float* pout = pts + 3 * c.lv[d + 1].ptOff;
        level_a<RW, CREASED>(c, d, topo, uv, pin, pout);
        if (det || d == 1) {
            const cudaError_t e = run_vertex_det_level(c, d, pin, pout, CREASED);
            if (e != cudaSuccess) return e;
        } else {
            level_b<RW, CREASED>(c, d, pin, pout);
        }
    }
    return cudaGetLastError();
}

// `det` selects the one-thread-per-vertex sorted pass (k_vertex_det) at every
// depth; either way the sums follow the reference's one-thread order.
cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool det) {
    const bool creased = mode == CCS_POINTS_SCATTER;
    const bool uv = c.cage->U > 0 && c.rw == 4;
    cudaError_t e = run_cage_step(c, topo, uv, cagePts, pts + 3 * c.lv[1].ptOff, mode, true);
    if (e != cudaSuccess) return e;
    if (c.rw == 4) return creased ? fused_levels<4, true>(c, topo, uv, pts, det) : fused_levels<4, false>(c, topo, uv, pts, det);
    return creased ? fused_levels<3, true>(c, topo, false, pts, det) : fused_levels<3, false>(c, topo, false, pts, det);
}

}  // namespace ccs
