// ccs_cagemap.cu -- the cage step of the atomic scatter rules as one sparse
// matrix-vector product.
//
// For a fixed cage topology and fixed crease sharpness, the points of depth 1
// are a linear map of the cage points: every face point, edge point and
// vertex point of depth 1 is a weighted sum of a few cage points (the face's
// vertices; an edge's two ends and its faces' vertices; a vertex's one-ring
// and its faces' vertices).  The weights depend only on the topology and the
// sharpness, which a subd never changes after ccs_Create_cuda, so they are
// built once on the host when the subd is created and kept on the GPU as CSR
// rows (rows in the layout of depth 1: [old vertices | faces | edges]).
//
// The builder applies the reference's cage rules symbolically, with every
// branch decided as the reference decides it (the ring statistics, the
// crease weights and the comparisons evaluated in float, in the walk order
// of the rule):
//   face point  :1437-1463   sum over the face of p / n
//   edge point  :1602-1648   lerp(0.5 lerp(v0, f, 0.5), lerp(v0, v1, 0.5) b, sat(s))
//               :1517-1548   (no creases) lerp(f / 2, lerp(w v0, w v1, 0.5), w)
//   vertex point:1872-1991   smooth first, then corner, then the crease blend
//               :1713-1756   (no creases) w (p + w s (4 e - f - 3 p))
// and accumulates the weight of each cage point in double; the weights are
// stored in float.  The map's product is the rule's value up to rounding
// (the default, float-atomic pass's tolerance), so it replaces the cage
// step of that pass only; the deterministic pass and the gather rules keep
// their own kernels, which reproduce the reference bit for bit.
//
// The transpose of the creased map (rows = cage vertices) is the cage level
// of the adjoint: dL/dcage = S^T dL/dP1, one gather per cage vertex.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ccs_host.h"

namespace ccs {

int set_last_error(int status);
int validate_cage_host(const cc_Mesh* m);

static constexpr int kBlockM = 256;
static constexpr int32_t kMapWalkCap = 1 << 16;

// out[i] = sum_k w[k] in[col[k]] for k in [rowptr[i], rowptr[i + 1]), three
// coordinates, accumulated in double.
__global__ void __launch_bounds__(kBlockM)
k_cage_map(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, const float* __restrict__ w,
           int32_t rows, const float* __restrict__ in, float* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const int32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
    double x = 0.0, y = 0.0, z = 0.0;
    for (int32_t k = b; k < e; ++k) {
        const int64_t c = 3 * (int64_t)__ldg(col + k);
        const double wk = (double)__ldg(w + k);
        x = fma(wk, (double)__ldg(in + c + 0), x);
        y = fma(wk, (double)__ldg(in + c + 1), y);
        z = fma(wk, (double)__ldg(in + c + 2), z);
    }
    out[3 * i + 0] = (float)x;
    out[3 * i + 1] = (float)y;
    out[3 * i + 2] = (float)z;
}

cudaError_t launch_cage_map(const CageMap& m, const float* in, float* out, cudaStream_t s) {
    if (m.rows <= 0) return cudaSuccess;
    k_cage_map<<<(unsigned)((m.rows + kBlockM - 1) / kBlockM), kBlockM, 0, s>>>(m.rowptr, m.col, m.w, m.rows, in,
                                                                               out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host builder
// ---------------------------------------------------------------------------
namespace {

static float satf(float x) { return std::max(0.0f, std::min(x, 1.0f)); }
static float signf_(float x) { return x < 0.0f ? -1.0f : (x > 0.0f ? 1.0f : 0.0f); }

// A row under construction: a dense accumulator over the cage vertices with
// the list of the entries it touched.
struct Acc {
    std::vector<double> val;
    std::vector<int32_t> touched;
    std::vector<uint8_t> on;
    explicit Acc(int32_t n) : val((size_t)n, 0.0), on((size_t)n, 0) {}
    void add(int32_t v, double x) {
        if (!on[(size_t)v]) {
            on[(size_t)v] = 1;
            touched.push_back(v);
        }
        val[(size_t)v] += x;
    }
    void add_row(const std::vector<std::pair<int32_t, double>>& r, double s) {
        for (const auto& kv : r) add(kv.first, s * kv.second);
    }
    // appends the row (columns in increasing order) and clears
    void flush(std::vector<int32_t>& col, std::vector<float>& w) {
        std::sort(touched.begin(), touched.end());
        for (int32_t v : touched) {
            col.push_back(v);
            w.push_back((float)val[(size_t)v]);
            val[(size_t)v] = 0.0;
            on[(size_t)v] = 0;
        }
        touched.clear();
    }
    std::vector<std::pair<int32_t, double>> take() {
        std::sort(touched.begin(), touched.end());
        std::vector<std::pair<int32_t, double>> r;
        r.reserve(touched.size());
        for (int32_t v : touched) {
            r.emplace_back(v, val[(size_t)v]);
            val[(size_t)v] = 0.0;
            on[(size_t)v] = 0;
        }
        touched.clear();
        return r;
    }
};

struct Cage {
    const cc_Mesh* m;
    int32_t twin(int32_t h) const { return m->halfedges[h].twinID; }
    int32_t next(int32_t h) const { return m->halfedges[h].nextID; }
    int32_t prev(int32_t h) const { return m->halfedges[h].prevID; }
    int32_t face(int32_t h) const { return m->halfedges[h].faceID; }
    int32_t edge(int32_t h) const { return m->halfedges[h].edgeID; }
    int32_t vert(int32_t h) const { return m->halfedges[h].vertexID; }
    float hsharp(int32_t h) const { return m->creases[edge(h)].sharpness; }
};

using Row = std::vector<std::pair<int32_t, double>>;

}  // namespace

// Builds the map of one point rule: creased (the scatter rule) or not (the
// NoCreases scatter rule).  Rows: V0 vertex points, F0 face points, E0 edge
// points of depth 1.
static void build_rows(const cc_Mesh* m, bool creased, std::vector<int32_t>& rowptr, std::vector<int32_t>& col,
                       std::vector<float>& wts) {
    const Cage c{m};
    const int32_t V = m->vertexCount, F = m->faceCount, E = m->edgeCount, H = m->halfedgeCount;
    Acc acc(V);
    // face rows: sum over the face of p / n (:1437-1463), n the face size in float
    std::vector<Row> fr((size_t)F);
    std::vector<int32_t> fh((size_t)F, -1);
    for (int32_t h = 0; h < H; ++h)
        if (fh[(size_t)c.face(h)] < 0) fh[(size_t)c.face(h)] = h;
    std::vector<float> fn((size_t)F, 0.0f);
    for (int32_t h = 0; h < H; ++h) {
        float n = 1.0f;
        int32_t guard = 0;
        for (int32_t it = c.next(h); it != h && guard < kMapWalkCap; it = c.next(it), ++guard) n += 1.0f;
        fn[(size_t)c.face(h)] = n;
    }
    for (int32_t f = 0; f < F; ++f) {
        const int32_t h0 = fh[(size_t)f];
        if (h0 < 0) continue;
        int32_t it = h0, guard = 0;
        do {
            acc.add(c.vert(it), 1.0 / (double)fn[(size_t)f]);
            it = c.next(it);
        } while (it != h0 && ++guard < kMapWalkCap);
        fr[(size_t)f] = acc.take();
    }
    // edge rows: the shares of the edge's halfedges
    std::vector<Row> er((size_t)E);
    {
        std::vector<std::vector<int32_t>> eh((size_t)E);
        for (int32_t h = 0; h < H; ++h) eh[(size_t)c.edge(h)].push_back(h);
        for (int32_t e = 0; e < E; ++e) {
            for (int32_t h : eh[(size_t)e]) {
                const bool bnd = c.twin(h) < 0;
                const int32_t v0 = c.vert(h), v1 = c.vert(c.next(h));
                double cv0, cv1, cf;
                if (creased) {                               // :1602-1648
                    const double w = (double)satf(m->creases[e].sharpness), b = bnd ? 1.0 : 0.5;
                    cv0 = (1.0 - w) * 0.25 + w * 0.5 * b;
                    cv1 = w * 0.5 * b;
                    cf = (1.0 - w) * 0.25;
                } else {                                     // :1517-1548
                    const double w = bnd ? 1.0 : 0.5;
                    cv0 = cv1 = 0.5 * w * w;
                    cf = 0.5 * (1.0 - w);
                }
                acc.add(v0, cv0);
                acc.add(v1, cv1);
                acc.add_row(fr[(size_t)c.face(h)], cf);
            }
            er[(size_t)e] = acc.take();
        }
    }
    // vertex rows: the shares of every halfedge leaving the vertex
    std::vector<std::vector<int32_t>> vh((size_t)V);
    for (int32_t h = 0; h < H; ++h) vh[(size_t)c.vert(h)].push_back(h);
    rowptr.assign((size_t)(V + F + E) + 1, 0);
    col.clear();
    wts.clear();
    for (int32_t v = 0; v < V; ++v) {
        for (int32_t h : vh[(size_t)v]) {
            double cP, cE, cEp = 0.0, cF;
            const int32_t prev = c.prev(h);
            if (creased) {                                   // :1872-1991, smooth first
                // ring statistics as the rule walks them from h (float)
                const float prevS = c.hsharp(prev);
                float avgS = prevS, creaseCount = signf_(prevS), valence = 1.0f;
                int32_t fwd, bwd, guard = 0;
                for (fwd = c.twin(prev); fwd >= 0 && fwd != h && guard < kMapWalkCap; fwd = c.twin(fwd), ++guard) {
                    const int32_t p = c.prev(fwd);
                    const float s = c.hsharp(p);
                    valence += 1.0f;
                    avgS += s;
                    creaseCount += signf_(s);
                    fwd = p;
                }
                guard = 0;
                for (bwd = c.twin(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kMapWalkCap; bwd = c.twin(bwd), ++guard) {
                    const int32_t n = c.next(bwd);
                    const float s = c.hsharp(n);
                    valence += 1.0f;
                    avgS += s;
                    creaseCount += signf_(s);
                    bwd = n;
                }
                const float cw = signf_(c.hsharp(h)), pcw = signf_(prevS);
                const double n0 = (double)valence;
                // corner = P / n; smooth = (-F + 4 E + (n - 3) P) / n^2;
                // crease = cw/4 (P + E) [+ pcw/4 (P + Ep) on a boundary]
                double crP = 0.25 * cw, crE = 0.25 * cw, crEp = 0.0;
                if (fwd < 0) {
                    creaseCount += cw;
                    valence += 1.0f;
                    crP += 0.25 * pcw;
                    crEp = 0.25 * pcw;
                }
                if (creaseCount <= 1.0f) {
                    cP = (n0 - 3.0) / (n0 * n0);
                    cE = 4.0 / (n0 * n0);
                    cF = -1.0 / (n0 * n0);
                } else if (creaseCount >= 3.0f || valence == 2.0f) {
                    cP = 1.0 / n0;
                    cE = 0.0;
                    cF = 0.0;
                } else {
                    const double t = (double)satf(avgS * 0.5f);
                    cP = (1.0 - t) / n0 + t * crP;
                    cE = t * crE;
                    cEp = t * crEp;
                    cF = 0.0;
                }
            } else {                                         // :1713-1756
                int32_t valence = 1, fwd, bwd, guard = 0;
                auto prev_vertex_he = [&](int32_t x) { return c.twin(c.prev(x)); };
                auto next_vertex_he = [&](int32_t x) { const int32_t t = c.twin(x); return t >= 0 ? c.next(t) : -1; };
                for (fwd = prev_vertex_he(h); fwd >= 0 && fwd != h && guard < kMapWalkCap; fwd = prev_vertex_he(fwd), ++guard)
                    ++valence;
                guard = 0;
                for (bwd = next_vertex_he(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kMapWalkCap;
                     bwd = next_vertex_he(bwd), ++guard)
                    ++valence;
                const double w = 1.0 / (double)valence, s = fwd < 0 ? 0.0 : 1.0;
                cP = w - 3.0 * w * w * s;
                cE = 4.0 * w * w * s;
                cF = -w * w * s;
            }
            acc.add(v, cP);
            if (cE != 0.0) acc.add_row(er[(size_t)c.edge(h)], cE);
            if (cEp != 0.0) acc.add_row(er[(size_t)c.edge(prev)], cEp);
            if (cF != 0.0) acc.add_row(fr[(size_t)c.face(h)], cF);
        }
        acc.flush(col, wts);
        rowptr[(size_t)v + 1] = (int32_t)col.size();
    }
    for (int32_t f = 0; f < F; ++f) {
        for (const auto& kv : fr[(size_t)f]) { col.push_back(kv.first); wts.push_back((float)kv.second); }
        rowptr[(size_t)(V + f) + 1] = (int32_t)col.size();
    }
    for (int32_t e = 0; e < E; ++e) {
        for (const auto& kv : er[(size_t)e]) { col.push_back(kv.first); wts.push_back((float)kv.second); }
        rowptr[(size_t)(V + F + e) + 1] = (int32_t)col.size();
    }
}

// The transpose of a map with `cols` columns.
static void transpose_rows(const std::vector<int32_t>& rowptr, const std::vector<int32_t>& col,
                           const std::vector<float>& w, int32_t cols, std::vector<int32_t>& tptr,
                           std::vector<int32_t>& tcol, std::vector<float>& tw) {
    const int32_t rows = (int32_t)rowptr.size() - 1;
    tptr.assign((size_t)cols + 1, 0);
    for (int32_t k : col) ++tptr[(size_t)k + 1];
    for (int32_t j = 0; j < cols; ++j) tptr[(size_t)j + 1] += tptr[(size_t)j];
    std::vector<int32_t> pos(tptr.begin(), tptr.end() - 1);
    tcol.assign(col.size(), 0);
    tw.assign(col.size(), 0.0f);
    for (int32_t i = 0; i < rows; ++i)
        for (int32_t k = rowptr[(size_t)i]; k < rowptr[(size_t)i + 1]; ++k) {
            const int32_t p = pos[(size_t)col[(size_t)k]]++;
            tcol[(size_t)p] = i;
            tw[(size_t)p] = w[(size_t)k];
        }
}

static bool upload_map(const std::vector<int32_t>& rowptr, const std::vector<int32_t>& col,
                       const std::vector<float>& w, CageMap* out) {
    out->rows = (int32_t)rowptr.size() - 1;
    out->nnz = (int64_t)col.size();
    if (cudaMalloc((void**)&out->rowptr, sizeof(int32_t) * rowptr.size()) != cudaSuccess ||
        cudaMalloc((void**)&out->col, sizeof(int32_t) * (col.empty() ? 1 : col.size())) != cudaSuccess ||
        cudaMalloc((void**)&out->w, sizeof(float) * (w.empty() ? 1 : w.size())) != cudaSuccess)
        return false;
    return cudaMemcpy(out->rowptr, rowptr.data(), sizeof(int32_t) * rowptr.size(), cudaMemcpyHostToDevice) ==
               cudaSuccess &&
           (col.empty() ||
            cudaMemcpy(out->col, col.data(), sizeof(int32_t) * col.size(), cudaMemcpyHostToDevice) == cudaSuccess) &&
           (w.empty() || cudaMemcpy(out->w, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice) == cudaSuccess);
}

void free_cage_map(CageMap* m) {
    if (!m) return;
    cudaFree(m->rowptr);
    cudaFree(m->col);
    cudaFree(m->w);
    *m = CageMap{};
}

int build_cage_maps(const cc_Mesh* m, CageMaps* out) {
    std::vector<int32_t> rp, col, tp, tc;
    std::vector<float> w, tw;
    build_rows(m, true, rp, col, w);
    if (!upload_map(rp, col, w, &out->creased)) return CCS_ERR_ALLOC;
    transpose_rows(rp, col, w, m->vertexCount, tp, tc, tw);
    if (!upload_map(tp, tc, tw, &out->creasedT)) return CCS_ERR_ALLOC;
    build_rows(m, false, rp, col, w);
    if (!upload_map(rp, col, w, &out->smooth)) return CCS_ERR_ALLOC;
    return CCS_OK;
}

}  // namespace ccs

// Host only (no GPU work): the cage step's sparse matrix, as built for a
// subd's default pass.  Two calls: with cap < nnz only *rows and *nnz are set.
extern "C" int ccs_CageStepMatrix_cuda(const cc_Mesh* cage, int mode, int transpose, int32_t* rows, int64_t* nnz,
                                       int32_t* rowptr, int32_t* col, float* w, int64_t cap) {
    using namespace ccs;
    if (!cage || !rows || !nnz || (mode != CCS_POINTS_SCATTER && mode != CCS_POINTS_NOCREASES_SCATTER) ||
        (transpose && mode != CCS_POINTS_SCATTER))
        return set_last_error(CCS_ERR_ARG);
    const int st = validate_cage_host(cage);
    if (st != CCS_OK) return set_last_error(st);
    std::vector<int32_t> rp, cl, tp, tc;
    std::vector<float> wt, tw;
    build_rows(cage, mode == CCS_POINTS_SCATTER, rp, cl, wt);
    if (transpose) {
        transpose_rows(rp, cl, wt, cage->vertexCount, tp, tc, tw);
        rp.swap(tp);
        cl.swap(tc);
        wt.swap(tw);
    }
    *rows = (int32_t)rp.size() - 1;
    *nnz = (int64_t)cl.size();
    if (cap >= (int64_t)cl.size() && rowptr && col && w) {
        std::memcpy(rowptr, rp.data(), sizeof(int32_t) * rp.size());
        std::memcpy(col, cl.data(), sizeof(int32_t) * cl.size());
        std::memcpy(w, wt.data(), sizeof(float) * wt.size());
    }
    return set_last_error(CCS_OK);
}
