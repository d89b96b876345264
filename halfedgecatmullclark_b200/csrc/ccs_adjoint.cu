// ccs_adjoint.cu -- adjoint of the creased scatter point rule.
//
// For fixed topology and sharpness the refined points of depth d+1 are a
// linear function S_d of the points of depth d (every branch of the vertex
// rule depends only on topology and sharpness).  Per halfedge h, with
// n = face size, vp = ring valence before the boundary correction:
//
//   F[f(h)]   += P[v(h)] / n
//   E[e(h)]   += al P[v(h)] + be P[v(next h)] + ga F[f(h)]
//   Vn[v(h)]  += a P[v(h)] + bF F[f(h)] + cE E[e(h)] + dE E[e(prev h)]
//
// (coefficients in ccs_tiles.cuh).  Given g = dL/d(points of depth d+1) this
// file computes dL/d(points of depth d) += S_d^T g.
//
// Quad levels d >= 2 (cages with the twin relation, ring statistics kept):
// one pass with one thread per depth-d face, adj_face_step_tile (the
// batched path too), which completes each edge's gradient once and then adds
// the vertex terms.
// Depth 1: two halfedge-parallel passes with the forward's lane layout
// (ccs_tiles.cuh adj_quad_*):
//   1. gE[e] += the cE / dE terms, completed by the pair's larger halfedge
//      (its own side from the quad's lanes, the twin side's coefficients
//      recomputed; the twin side's vertices are this side's);
//   2. per halfedge: the face term gF + sum of bF gV + ga gE over the quad
//      (lane reduction), then the halfedge's term of its vertex
//      a gV + al gE + gF/4 + be(prev) gE(prev), summed into the vertex (a face
//      centre in the warp, the others by float atomics).
// The cage level (and cages without the twin relation) runs three gathers,
// every output slot written by one thread:
//
//   1. edge gather    (one thread per edge, run by the pair's larger
//      halfedge):  gE[e] += sum of cE / dE terms of the halfedges whose
//      vertex share reads E[e];
//   2. face gather    (one thread per face):  gF[f] += sum over the face's
//      halfedges of bF gVn[v(h)] + ga gE[e(h)];
//   3. vertex gather  (one thread per old vertex, walking its ring):
//      gP[v] += sum over outgoing h of a gVn[v] + al gE[e(h)] + gF[f(h)]/n
//               + be(prev h) gE[e(prev h)].
//
// The coefficients of a halfedge need its vertex's ring statistics.  On quad
// levels these are known from the structure for face centres and edge
// midpoints; for the older vertices the passes read the per-level table the
// topology refinement keeps (ccs_level.cu k_shape_stats / k_crease_stats).
//
// Levels run deepest first; only the level offsets are needed (no state is
// saved by the forward pass).
#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBlockA = 256;
static inline unsigned nblocksA(int64_t n) { return (unsigned)((n + kBlockA - 1) / kBlockA); }

template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_edges(View L, float* __restrict__ gNew) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.H) adj_edge_item(L, gNew, (int32_t)i);
}

template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_faces(View L, float* __restrict__ gNew) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.F) adj_face_item(L, gNew, (int32_t)i);
}

template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_vertices(View L, const float* __restrict__ gNew, float* __restrict__ gOld) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.V) adj_vertex_item(L, gNew, gOld, (int32_t)i);
}

// quad levels: two halfedge-parallel passes (ccs_tiles.cuh)
template <int RW>
__global__ void __launch_bounds__(kBlockA)
k_adj_quad_edges(QuadView<RW> L, float* __restrict__ gNew) {
    adj_quad_edge_tile<RW>(L, gNew, (int64_t)blockIdx.x * kBlockA);
}

// quad levels d >= 2, one thread per face (adj_face_step_tile).  Depth 5 of
// the headline workload: 0.364 ms with the per-halfedge tile; per face,
// 6 resident blocks of 128 (78 registers) 0.187 ms, 8 (64 registers, a
// 16-byte spill) 0.176 ms; the L2 prefetch of the records one wave ahead is
// worth 1 % (the same from 592 to 2368 blocks ahead)
static constexpr int kBlockAF = 128;
#ifndef CCS_ADJ_FQ_MIN_BLOCKS
#define CCS_ADJ_FQ_MIN_BLOCKS 8
#endif
#ifndef CCS_ADJ_FQ_PREFETCH_AHEAD
#define CCS_ADJ_FQ_PREFETCH_AHEAD 1184
#endif
template <int RW>
__global__ void __launch_bounds__(kBlockAF, CCS_ADJ_FQ_MIN_BLOCKS)
k_adj_face_step(QuadView<RW> L, const float* __restrict__ gNew, float* __restrict__ gOld) {
    chain_wait_then_release();
    const int64_t nF = (int64_t)L.H >> 2;
    if (CCS_ADJ_FQ_PREFETCH_AHEAD > 0 && threadIdx.x == 0) {
        const int64_t p0 = ((int64_t)blockIdx.x + CCS_ADJ_FQ_PREFETCH_AHEAD) * kBlockAF;
        if (p0 < nF) {
            const int64_t n = (nF - p0) < kBlockAF ? (nF - p0) : kBlockAF;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         :: "l"(L.he + (int64_t)RW * 4 * p0), "r"((uint32_t)(n * 16 * RW)) : "memory");
        }
    }
    adj_face_step_tile<RW, GradArray>(L, GradArray{gNew}, gOld, (int64_t)blockIdx.x * kBlockAF + threadIdx.x);
}

template <int RW, bool STRUCT>
__global__ void __launch_bounds__(kBlockA, 8)
k_adj_quad_points(QuadView<RW> L, const float* __restrict__ gNew, float* __restrict__ gOld) {
    adj_quad_point_tile<RW, STRUCT>(L, gNew, gOld, (int64_t)blockIdx.x * kBlockA);
}

static CageTables cage_tables_a(const DevCage& c) { return make_cage_tables(c); }

template <int RW>
static void adjoint_quad_level(const Ctx& c, const QuadView<RW>& L, float* gNew, float* gOld) {
#ifndef CCS_NO_ADJ_STEP
    if (L.d >= 2 && L.ostats) {
        c.prof->begin(c.stream, CCS_K_ADJ_STEP, L.d, L.H);
        launch_chained(k_adj_face_step<RW>, (unsigned)((((int64_t)L.H >> 2) + kBlockAF - 1) / kBlockAF),
                       kBlockAF, c.stream, L, gNew, gOld);
        c.prof->end(c.stream);
        return;
    }
#endif
    c.prof->begin(c.stream, CCS_K_ADJ_EDGES, L.d, L.H);
    k_adj_quad_edges<RW><<<nblocksA(L.H), kBlockA, 0, c.stream>>>(L, gNew);
    c.prof->end(c.stream);
    c.prof->begin(c.stream, CCS_K_ADJ_VERTICES, L.d, L.H);
    if (L.d >= 2) k_adj_quad_points<RW, true><<<nblocksA(L.H), kBlockA, 0, c.stream>>>(L, gNew, gOld);
    else k_adj_quad_points<RW, false><<<nblocksA(L.H), kBlockA, 0, c.stream>>>(L, gNew, gOld);
    c.prof->end(c.stream);
}

template <class View>
static void adjoint_level(const Ctx& c, const View& L, float* gNew, float* gOld) {
    c.prof->begin(c.stream, CCS_K_ADJ_EDGES, L.d, L.H);
    k_adj_edges<View><<<nblocksA(L.H), kBlockA, 0, c.stream>>>(L, gNew);
    c.prof->end(c.stream);
    c.prof->begin(c.stream, CCS_K_ADJ_FACES, L.d, L.F);
    k_adj_faces<View><<<nblocksA(L.F), kBlockA, 0, c.stream>>>(L, gNew);
    c.prof->end(c.stream);
    c.prof->begin(c.stream, CCS_K_ADJ_VERTICES, L.d, L.V);
    k_adj_vertices<View><<<nblocksA(L.V), kBlockA, 0, c.stream>>>(L, gNew, gOld);
    c.prof->end(c.stream);
}

// The levels' gradients start as the caller's and accumulate in `work`.  The
// finest level's are only read, and when its step runs the one-pass kernel
// (which reads its input gradients only) they are read where the caller
// holds them: only depths 1..D-1 are copied.
cudaError_t run_adjoint(const Ctx& c, const float* gradPts, float* work, float* gradCage, int64_t cumV) {
#ifndef CCS_NO_ADJ_STEP
    const bool finestInPlace = c.fusable && c.D - 1 >= 2 && stats_at(c, c.D - 1) != nullptr;
#else
    const bool finestInPlace = false;
#endif
    const int64_t copyV = finestInPlace ? c.lv[c.D].ptOff : cumV;
    cudaError_t st = cudaMemcpyAsync(work, gradPts, sizeof(float) * 3 * (size_t)copyV,
                                     cudaMemcpyDeviceToDevice, c.stream);
    if (st != cudaSuccess) return st;
    st = cudaMemsetAsync(gradCage, 0, sizeof(float) * 3 * (size_t)c.cage->V, c.stream);
    if (st != cudaSuccess) return st;
    for (int d = c.D - 1; d >= 0; --d) {
        float* gNew = (finestInPlace && d == c.D - 1) ? const_cast<float*>(gradPts) + 3 * c.lv[d + 1].ptOff
                                                      : work + 3 * c.lv[d + 1].ptOff;
        if (d == 0 && c.maps && c.maps->creasedT.rows == c.cage->V) {
            // dL/dcage = S^T dL/dP1 with the transposed map of the cage step
            c.prof->begin(c.stream, CCS_K_ADJ_CAGE_MAP, 0, c.cage->V);
            st = launch_cage_map(c.maps->creasedT, gNew, gradCage, c.stream);
            c.prof->end(c.stream);
            if (st != cudaSuccess) return st;
        } else if (d == 0) {
            CageView L;
            L.t = cage_tables_a(*c.cage);
            L.cr = c.cage->cr;
            L.V = c.cage->V; L.F = c.cage->F; L.E = c.cage->E; L.H = c.cage->H; L.C = c.cage->E;
            L.d = 0;
            adjoint_level(c, L, gNew, gradCage);
        } else {
            float* gOld = work + 3 * c.lv[d].ptOff;
            const Level& lv = c.lv[d];
            if (c.rw == 4) {
                QuadView<4> L;
                L.t = cage_tables_a(*c.cage);
                L.he = c.he + 4 * lv.heOff;
                L.cr = c.cr + lv.crOff;
                L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C; L.d = d;
                L.ostats = stats_at(c, d);
                if (c.fusable) adjoint_quad_level(c, L, gNew, gOld);
                else adjoint_level(c, L, gNew, gOld);
            } else {
                QuadView<3> L;
                L.t = cage_tables_a(*c.cage);
                L.he = c.he + 3 * lv.heOff;
                L.cr = c.cr + lv.crOff;
                L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C; L.d = d;
                L.ostats = stats_at(c, d);
                if (c.fusable) adjoint_quad_level(c, L, gNew, gOld);
                else adjoint_level(c, L, gNew, gOld);
            }
        }
    }
    return cudaGetLastError();
}

}  // namespace ccs
