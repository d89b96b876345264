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
// (coefficients below).  Given g = dL/d(points of depth d+1) this file
// computes dL/d(points of depth d) += S_d^T g as three gathers, so that
// every output slot is written by exactly one thread and the result does not
// depend on scheduling:
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
// Levels run deepest first; only the level offsets are needed (no state is
// saved by the forward pass).
#include "ccs_host.h"
#include "ccs_internal.cuh"

namespace ccs {

static constexpr int kBlockA = 256;
static constexpr int kRingCapA = 1 << 16;
static inline unsigned nblocksA(int64_t n) { return (unsigned)((n + kBlockA - 1) / kBlockA); }

struct VCoef {
    float a, bF, cE, dE;
};

// Coefficients of halfedge h's vertex share (linearisation of
// creased_vertex_share; :1872-1991 and :2496-2615).
template <class View>
__device__ __forceinline__ VCoef vertex_coef(const View& L, int32_t h) {
    const RingStats r = creased_ring(L, h);
    const int32_t prev = L.prev(h);
    const float cw = fsign(L.hsharp(h)), pcw = fsign(L.hsharp(prev));
    const float vp = r.valence;
    const bool bnd = r.fwd < 0;
    const float valence = bnd ? vp + 1.0f : vp;
    const float creaseCount = bnd ? r.creaseCount + cw : r.creaseCount;
    int branch;  // 0 corner, 1 smooth, 2 blend
    if (View::kQuad) {
        if (creaseCount >= 3.0f || valence == 2.0f) branch = 0;
        else if (creaseCount <= 1.0f) branch = 1;
        else branch = 2;
    } else {
        if (creaseCount <= 1.0f) branch = 1;
        else if (creaseCount >= 3.0f || valence == 2.0f) branch = 0;
        else branch = 2;
    }
    VCoef k{0.0f, 0.0f, 0.0f, 0.0f};
    if (branch == 0) {
        k.a = 1.0f / vp;
    } else if (branch == 1) {
        const float inv = 1.0f / (vp * vp);
        k.a = (vp - 3.0f) * inv;
        k.bF = -inv;
        k.cE = 4.0f * inv;
    } else {
        const float t = fsat(r.avgS * 0.5f);
        k.a = (1.0f - t) / vp + t * 0.25f * (cw + (bnd ? pcw : 0.0f));
        k.cE = t * 0.25f * cw;
        k.dE = bnd ? t * 0.25f * pcw : 0.0f;
    }
    return k;
}

struct ECoef {
    float al, be, ga;
};
// Coefficients of halfedge h's edge share (:1602-1648, :2194-2241)
template <class View>
__device__ __forceinline__ ECoef edge_coef(const View& L, int32_t h) {
    const float w = fsat(L.sharp(L.edge(h)));
    const float b = L.twin(h) < 0 ? 1.0f : 0.5f;
    ECoef k;
    k.al = (1.0f - w) * 0.25f + w * b * 0.5f;
    k.be = w * b * 0.5f;
    k.ga = (1.0f - w) * 0.25f;
    return k;
}

template <class View>
__device__ __forceinline__ int32_t face_size(const View& L, int32_t h) {
    if (View::kQuad) return 4;
    int32_t n = 1, guard = 0;
    for (int32_t it = L.next(h); it != h && guard < kRingCapA; it = L.next(it), ++guard) ++n;
    return n;
}

__device__ __forceinline__ void axpy3(f3& acc, float s, const float* p) {
    acc.x += s * p[0];
    acc.y += s * p[1];
    acc.z += s * p[2];
}

// 1. edge gather: gE[e] += vertex-pass terms
template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_edges(View L, float* __restrict__ gNew) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.H) return;
    const int32_t h = (int32_t)i, tw = L.twin(h);
    if (!(h > tw)) return;
    const float* gV = gNew;
    float* gE = gNew + 3 * ((int64_t)L.V + L.F);
    f3 acc = zero3();
    const int32_t sides[2] = {h, tw};
    for (int s = 0; s < (tw >= 0 ? 2 : 1); ++s) {
        const int32_t x = sides[s], nx = L.next(x);
        axpy3(acc, vertex_coef(L, x).cE, gV + 3 * (int64_t)L.vert(x));
        axpy3(acc, vertex_coef(L, nx).dE, gV + 3 * (int64_t)L.vert(nx));
    }
    float* o = gE + 3 * (int64_t)L.edge(h);
    o[0] += acc.x;
    o[1] += acc.y;
    o[2] += acc.z;
}

// 2. face gather: gF[f] += vertex-pass and edge-pass terms
template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_faces(View L, float* __restrict__ gNew) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.F) return;
    const int32_t f = (int32_t)i;
    const float* gV = gNew;
    float* gF = gNew + 3 * (int64_t)L.V;
    const float* gE = gNew + 3 * ((int64_t)L.V + L.F);
    const int32_t h0 = L.face_he(f);
    f3 acc = zero3();
    int32_t h = h0;
    int guard = 0;
    do {
        axpy3(acc, vertex_coef(L, h).bF, gV + 3 * (int64_t)L.vert(h));
        axpy3(acc, edge_coef(L, h).ga, gE + 3 * (int64_t)L.edge(h));
        h = L.next(h);
    } while (h != h0 && ++guard < kRingCapA);
    float* o = gF + 3 * (int64_t)f;
    o[0] += acc.x;
    o[1] += acc.y;
    o[2] += acc.z;
}

// 3. vertex gather: gOld[v] += all terms that read P[v]
template <class View>
__device__ __forceinline__ void adj_vertex_term(const View& L, int32_t x, const float* gVv, const float* gF,
                                                const float* gE, f3& acc) {
    axpy3(acc, vertex_coef(L, x).a, gVv);
    axpy3(acc, edge_coef(L, x).al, gE + 3 * (int64_t)L.edge(x));
    axpy3(acc, 1.0f / (float)face_size(L, x), gF + 3 * (int64_t)L.face(x));
    const int32_t p = L.prev(x);
    axpy3(acc, edge_coef(L, p).be, gE + 3 * (int64_t)L.edge(p));
}

template <class View>
__global__ void __launch_bounds__(kBlockA)
k_adj_vertices(View L, const float* __restrict__ gNew, float* __restrict__ gOld) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.V) return;
    const int32_t v = (int32_t)i;
    const float* gVv = gNew + 3 * (int64_t)v;
    const float* gF = gNew + 3 * (int64_t)L.V;
    const float* gE = gNew + 3 * ((int64_t)L.V + L.F);
    const int32_t h0 = L.vert_he(v);
    f3 acc = zero3();
    int32_t it = h0;
    int n = 0;
    do {
        adj_vertex_term(L, it, gVv, gF, gE, acc);
        it = L.prev_vertex_he(it);
    } while (it >= 0 && it != h0 && ++n < kRingCapA);
    if (it < 0) {
        n = 0;
        for (it = L.next_vertex_he(h0); it >= 0 && it != h0 && n < kRingCapA; it = L.next_vertex_he(it), ++n)
            adj_vertex_term(L, it, gVv, gF, gE, acc);
    }
    float* o = gOld + 3 * (int64_t)v;
    o[0] += acc.x;
    o[1] += acc.y;
    o[2] += acc.z;
}

static CageTables cage_tables_a(const DevCage& c) { return make_cage_tables(c); }

template <class View>
static void adjoint_level(const Ctx& c, const View& L, float* gNew, float* gOld) {
    c.prof->begin(c.stream, CCS_K_ADJOINT, L.d, L.H);
    k_adj_edges<View><<<nblocksA(L.H), kBlockA, 0, c.stream>>>(L, gNew);
    k_adj_faces<View><<<nblocksA(L.F), kBlockA, 0, c.stream>>>(L, gNew);
    k_adj_vertices<View><<<nblocksA(L.V), kBlockA, 0, c.stream>>>(L, gNew, gOld);
    c.prof->end(c.stream);
}

cudaError_t run_adjoint(const Ctx& c, const float* gradPts, float* work, float* gradCage, int64_t cumV) {
    cudaError_t st = cudaMemcpyAsync(work, gradPts, sizeof(float) * 3 * (size_t)cumV,
                                     cudaMemcpyDeviceToDevice, c.stream);
    if (st != cudaSuccess) return st;
    st = cudaMemsetAsync(gradCage, 0, sizeof(float) * 3 * (size_t)c.cage->V, c.stream);
    if (st != cudaSuccess) return st;
    for (int d = c.D - 1; d >= 0; --d) {
        float* gNew = work + 3 * c.lv[d + 1].ptOff;
        if (d == 0) {
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
                adjoint_level(c, L, gNew, gOld);
            } else {
                QuadView<3> L;
                L.t = cage_tables_a(*c.cage);
                L.he = c.he + 3 * lv.heOff;
                L.cr = c.cr + lv.crOff;
                L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C; L.d = d;
                adjoint_level(c, L, gNew, gOld);
            }
        }
    }
    return cudaGetLastError();
}

}  // namespace ccs
