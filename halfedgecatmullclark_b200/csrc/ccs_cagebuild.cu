// ccs_cagebuild.cu -- the halfedge cage of a polygon mesh, built on the GPU.
//
// Reproduces what the reference's OBJ converter derives from a polygon soup
// (examples/obj_to_ccm.c, LoadObj :666-752), with the same numbering:
//   * halfedges face by face in input order, next/prev cycling inside the
//     face, faceToHalfedge = the face's first corner (LoadFaceMappings
//     :312-348); uvID from the corner's texture index, 0 without one (:461-494);
//   * twins pair v0 -> v1 with v1 -> v0, -1 when unpaired (ComputeTwins
//     :142-190).  The reference sorts a hash of every directed edge; here
//     every vertex's outgoing halfedges are bucketed (counting sort: counts,
//     scan, scatter) and a halfedge looks for its twin among the bucket of
//     its end vertex.  Both need each directed edge used once; a second use,
//     and a face with two consecutive corners on one vertex, are reported
//     (CCS_ERR_ARG) instead of resolved by sort order;
//   * an edge is the larger halfedge ID of its pair, edges numbered by that
//     ID (LoadEdgeMappings :364-402): a scan of the "h > twin(h)" bits;
//   * vertexToHalfedge = the largest outgoing halfedge, or on a boundary the
//     outgoing halfedge without a twin (LoadVertexHalfedges :417-450);
//   * creases: self links, sharpness 0; every crease tag (v0, v1, s) sets the
//     sharpness of each edge whose ends are both in {v0, v1}, later tags
//     winning (ObjReadCrease :538-561, found through the two vertices'
//     buckets instead of a scan of all edges); boundary edges get 16
//     (MakeBoundariesSharp :265-279); then crease chains are linked where
//     exactly one other sharp edge meets (ComputeCreaseNeighbors :197-253).
#include <cstdint>
#include <cstring>
#include <vector>

#include "ccs_host.h"
#include "ccs_internal.cuh"
#include "ccs_scan.cuh"

namespace ccs {
namespace {

constexpr int kB = 256;
enum : int { BE_FACE = 1, BE_VERTEX = 2, BE_UV = 4, BE_DUP = 8 };

inline unsigned nblk(int64_t n, int per = kB) { return (unsigned)((n + per - 1) / per); }

// ---------------------------------------------------------------------------
// build kernels; `he` is the cc_Halfedge array as CH_WORDS int32 per record
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t& hw(int32_t* he, int32_t h, int w) { return he[(int64_t)CH_WORDS * h + w]; }
__device__ __forceinline__ int32_t hr(const int32_t* he, int32_t h, int w) { return he[(int64_t)CH_WORDS * h + w]; }

// face f: its corners' records, its first corner, and the outgoing counts
__global__ void k_faces(const int32_t* __restrict__ off, int32_t F, int32_t H, const int32_t* __restrict__ fv,
                        const int32_t* __restrict__ fu, int32_t V, int32_t U, int32_t* __restrict__ he,
                        int32_t* __restrict__ f2h, int32_t* __restrict__ count, int* err) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int32_t b = off[f], e = off[f + 1];
    if (b < 0 || e > H || e - b < 3 || (f == 0 && b != 0)) {
        atomicOr(err, BE_FACE);
        return;
    }
    f2h[f] = b;
    for (int32_t h = b; h < e; ++h) {
        const int32_t v = fv[h];
        const int32_t uv = fu ? fu[h] : 0;
        if (v < 0 || v >= V) { atomicOr(err, BE_VERTEX); continue; }
        if (v == fv[h + 1 < e ? h + 1 : b]) atomicOr(err, BE_FACE);   // a corner pair on one vertex
        if (fu && (uv < 0 || uv >= U)) atomicOr(err, BE_UV);
        hw(he, h, CH_TWIN) = -1;
        hw(he, h, CH_NEXT) = h + 1 < e ? h + 1 : b;
        hw(he, h, CH_PREV) = h > b ? h - 1 : e - 1;
        hw(he, h, CH_FACE) = (int32_t)f;
        hw(he, h, CH_EDGE) = -1;
        hw(he, h, CH_VERT) = v;
        hw(he, h, CH_UV) = uv;
        atomicAdd(count + v, 1);
    }
}

__global__ void k_bucket_fill(const int32_t* __restrict__ he, int32_t H, const int32_t* __restrict__ start,
                              int32_t* __restrict__ cursor, int32_t* __restrict__ bucket) {
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    const int32_t v = hr(he, (int32_t)h, CH_VERT);
    bucket[start[v] + atomicAdd(cursor + v, 1)] = (int32_t)h;
}

// twin of h: the halfedge leaving vertex(next h) towards vertex(h)
__global__ void k_twins(int32_t* __restrict__ he, int32_t H, const int32_t* __restrict__ start,
                        const int32_t* __restrict__ bucket, int* err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= H) return;
    const int32_t h = (int32_t)i;
    const int32_t v0 = hr(he, h, CH_VERT), v1 = hr(he, hr(he, h, CH_NEXT), CH_VERT);
    int32_t twin = -1, same = 0;
    for (int32_t k = start[v1]; k < start[v1 + 1]; ++k) {
        const int32_t g = bucket[k];
        if (hr(he, hr(he, g, CH_NEXT), CH_VERT) == v0) twin = twin < 0 ? g : twin;
    }
    for (int32_t k = start[v0]; k < start[v0 + 1]; ++k) {
        const int32_t g = bucket[k];
        same += hr(he, hr(he, g, CH_NEXT), CH_VERT) == v1;
    }
    if (same != 1) atomicOr(err, BE_DUP);
    // a halfedge from v to v (a degenerate corner pair) would be its own twin
    hw(he, h, CH_TWIN) = twin == h ? -1 : twin;
}

__global__ void k_edge_bits(const int32_t* __restrict__ he, int32_t H, int32_t* __restrict__ bits) {
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h < H) bits[h] = h > hr(he, (int32_t)h, CH_TWIN) ? 1 : 0;
}

__global__ void k_edges(int32_t* __restrict__ he, int32_t H, const int32_t* __restrict__ pre,
                        int32_t* __restrict__ e2h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= H) return;
    const int32_t h = (int32_t)i, t = hr(he, h, CH_TWIN);
    hw(he, h, CH_EDGE) = pre[h > t ? h : t];
    if (h > t) e2h[pre[h]] = h;
}

__global__ void k_v2h_max(const int32_t* __restrict__ he, int32_t H, int32_t* __restrict__ v2h) {
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h < H) atomicMax(v2h + hr(he, (int32_t)h, CH_VERT), (int32_t)h);
}

__global__ void k_v2h_boundary(const int32_t* __restrict__ he, int32_t H, int32_t* __restrict__ v2h) {
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h < H && hr(he, (int32_t)h, CH_TWIN) < 0) v2h[hr(he, (int32_t)h, CH_VERT)] = (int32_t)h;
}

// crease tag t marks (by the largest tag index) every edge with both ends in {a, b}
__global__ void k_tags(const int32_t* __restrict__ tags, int32_t T, int32_t V, const int32_t* __restrict__ he,
                       const int32_t* __restrict__ start, const int32_t* __restrict__ bucket,
                       int32_t* __restrict__ winner) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int32_t a = tags[2 * t], b = tags[2 * t + 1];
    for (int s = 0; s < 2; ++s) {
        const int32_t src = s == 0 ? a : b;
        if (src < 0 || src >= V || (s == 1 && b == a)) continue;
        for (int32_t k = start[src]; k < start[src + 1]; ++k) {
            const int32_t g = bucket[k];
            const int32_t d = hr(he, hr(he, g, CH_NEXT), CH_VERT);
            if (d == a || d == b) atomicMax(winner + hr(he, g, CH_EDGE), (int32_t)t);
        }
    }
}

__global__ void k_crease_values(cc_Crease* __restrict__ cr, int32_t E, const int32_t* __restrict__ winner,
                                const float* __restrict__ sharp, const int32_t* __restrict__ he,
                                const int32_t* __restrict__ e2h) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int32_t w = winner[e];
    float s = w >= 0 ? sharp[w] : 0.0f;
    if (hr(he, e2h[e], CH_TWIN) < 0) s = 16.0f;
    cc_Crease c;
    c.nextID = (int32_t)e;
    c.prevID = (int32_t)e;
    c.sharpness = s;
    cr[e] = c;
}

__device__ __forceinline__ int32_t next_vertex_he(const int32_t* he, int32_t h) {
    const int32_t t = hr(he, h, CH_TWIN);
    return t >= 0 ? hr(he, t, CH_NEXT) : -1;
}

// ComputeCreaseNeighbors for one sharp edge (bounded walks)
__global__ void k_crease_links(cc_Crease* __restrict__ cr, int32_t E, const int32_t* __restrict__ he,
                               const int32_t* __restrict__ e2h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E) return;
    const int32_t e = (int32_t)i;
    if (!(cr[e].sharpness > 0.0f)) return;
    const int32_t h = e2h[e], n = hr(he, h, CH_NEXT);
    auto sharp = [&](int32_t x) { return cr[hr(he, x, CH_EDGE)].sharpness; };
    int32_t cnt = 0, id = -1, it = next_vertex_he(he, h), guard = 0;
    for (; it != h && it >= 0 && guard < kWalkCap; it = next_vertex_he(he, it), ++guard) {
        if (sharp(it) > 0.0f) { id = hr(he, it, CH_EDGE); ++cnt; }
    }
    const int32_t prevID = (cnt == 1 && it == h) ? id : e;
    cnt = 0; id = -1;
    if (sharp(n) > 0.0f) { id = hr(he, n, CH_EDGE); ++cnt; }
    guard = 0;
    for (it = next_vertex_he(he, n); it != n && it >= 0 && guard < kWalkCap; it = next_vertex_he(he, it), ++guard) {
        if (sharp(it) > 0.0f && hr(he, it, CH_TWIN) != h) { id = hr(he, it, CH_EDGE); ++cnt; }
    }
    const int32_t nextID = (cnt == 1 && it == n) ? id : e;
    // only the links change; every thread reads sharpness only
    cr[e].prevID = prevID;
    cr[e].nextID = nextID;
}

// Device scratch: one allocation carved into 256-byte aligned arrays.
struct Arena {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    bool reserve(size_t bytes) {
        cap = bytes;
        return cudaMalloc(reinterpret_cast<void**>(&base), bytes ? bytes : 1) == cudaSuccess;
    }
    static size_t sz(size_t bytes) { return (bytes + 255) / 256 * 256; }
    template <class T>
    T* take(int64_t count) {
        const size_t b = sz(sizeof(T) * (size_t)(count > 0 ? count : 1));
        if (!base || used + b > cap) return nullptr;
        T* p = reinterpret_cast<T*>(base + used);
        used += b;
        return p;
    }
    ~Arena() {
        if (base) cudaFree(base);
    }
};

int build(const ccs_PolygonMesh* m, cc_Mesh** out, cudaStream_t s) {
    if (!m || !out || m->faceCount <= 0 || m->vertexCount <= 0 || m->uvCount < 0 || m->creaseTagCount < 0 ||
        !m->faceOffsets || !m->faceVertices || !m->vertexPoints || (m->uvCount > 0 && !m->uvs) ||
        (m->creaseTagCount > 0 && (!m->creaseVertices || !m->creaseSharpness)))
        return CCS_ERR_ARG;
    const int32_t F = m->faceCount, V = m->vertexCount, U = m->uvCount, T = m->creaseTagCount;
    Arena head;
    if (!head.reserve(Arena::sz(sizeof(int32_t) * ((size_t)F + 1)) + 2 * Arena::sz(16))) return CCS_ERR_ALLOC;
    int32_t* off = head.take<int32_t>(F + 1);
    int* err = head.take<int>(1);
    int32_t* total = head.take<int32_t>(2);
    if (!off || !err || !total) return CCS_ERR_ALLOC;
    if (cudaMemcpyAsync(off, m->faceOffsets, sizeof(int32_t) * ((size_t)F + 1), cudaMemcpyDefault, s) != cudaSuccess)
        return CCS_ERR_CUDA;
    int32_t H = 0;
    if (cudaMemcpyAsync(&H, off + F, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCS_ERR_CUDA;
    if (H < 3 * (int64_t)F) return CCS_ERR_ARG;

    const int64_t nTiles = scan_tiles(H > V ? H : V);
    const size_t i4 = sizeof(int32_t);
    Arena sc;
    if (!sc.reserve(Arena::sz(i4 * H) * (m->faceUvs ? 9 : 8) + Arena::sz(i4 * CH_WORDS * (size_t)H) +
                    Arena::sz(i4 * F) + 2 * Arena::sz(i4 * ((size_t)V + 1)) + 2 * Arena::sz(i4 * V) +
                    Arena::sz(i4 * nTiles) + Arena::sz(sizeof(cc_Crease) * (size_t)H) +
                    Arena::sz(i4 * 2 * (size_t)T) + Arena::sz(sizeof(float) * (size_t)T)))
        return CCS_ERR_ALLOC;
    int32_t* fv = sc.take<int32_t>(H);
    int32_t* fu = m->faceUvs ? sc.take<int32_t>(H) : nullptr;
    int32_t* he = sc.take<int32_t>((int64_t)CH_WORDS * H);
    int32_t* f2h = sc.take<int32_t>(F);
    int32_t* count = sc.take<int32_t>((int64_t)V + 1);
    int32_t* start = sc.take<int32_t>((int64_t)V + 1);
    int32_t* cursor = sc.take<int32_t>(V);
    int32_t* bucket = sc.take<int32_t>(H);
    int32_t* bits = sc.take<int32_t>(H);
    int32_t* pre = sc.take<int32_t>(H);
    int32_t* tiles = sc.take<int32_t>(nTiles);
    int32_t* e2h = sc.take<int32_t>(H);
    int32_t* v2h = sc.take<int32_t>(V);
    cc_Crease* cr = sc.take<cc_Crease>(H);
    int32_t* winner = sc.take<int32_t>(H);
    int32_t* tags = sc.take<int32_t>(2 * (int64_t)T);
    float* sharp = sc.take<float>(T);
    if (!fv || (m->faceUvs && !fu) || !he || !f2h || !count || !start || !cursor || !bucket || !bits || !pre ||
        !tiles || !e2h || !v2h || !cr || !winner || !tags || !sharp)
        return CCS_ERR_ALLOC;

    bool ok = cudaMemcpyAsync(fv, m->faceVertices, sizeof(int32_t) * (size_t)H, cudaMemcpyDefault, s) == cudaSuccess;
    if (fu) ok = ok && cudaMemcpyAsync(fu, m->faceUvs, sizeof(int32_t) * (size_t)H, cudaMemcpyDefault, s) == cudaSuccess;
    if (T > 0) {
        ok = ok && cudaMemcpyAsync(tags, m->creaseVertices, sizeof(int32_t) * 2 * (size_t)T, cudaMemcpyDefault, s) == cudaSuccess;
        ok = ok && cudaMemcpyAsync(sharp, m->creaseSharpness, sizeof(float) * (size_t)T, cudaMemcpyDefault, s) == cudaSuccess;
    }
    ok = ok && cudaMemsetAsync(err, 0, sizeof(int), s) == cudaSuccess;
    ok = ok && cudaMemsetAsync(count, 0, sizeof(int32_t) * ((size_t)V + 1), s) == cudaSuccess;
    ok = ok && cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (size_t)V, s) == cudaSuccess;
    ok = ok && cudaMemsetAsync(v2h, 0xff, sizeof(int32_t) * (size_t)V, s) == cudaSuccess;
    ok = ok && cudaMemsetAsync(winner, 0xff, sizeof(int32_t) * (size_t)H, s) == cudaSuccess;
    if (!ok) return CCS_ERR_CUDA;

    k_faces<<<nblk(F), kB, 0, s>>>(off, F, H, fv, fu, V, U, he, f2h, count, err);
    int hostErr = 0;
    if (cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCS_ERR_CUDA;
    if (hostErr) return CCS_ERR_ARG;      // every record is written and every index in range past here

    // vertex buckets of outgoing halfedges: start[v] .. start[v + 1]
    if (exclusive_scan<int32_t>(count, start, (int64_t)V + 1, tiles, total, s) != cudaSuccess) return CCS_ERR_CUDA;
    k_bucket_fill<<<nblk(H), kB, 0, s>>>(he, H, start, cursor, bucket);
    k_twins<<<nblk(H), kB, 0, s>>>(he, H, start, bucket, err);
    // edges
    k_edge_bits<<<nblk(H), kB, 0, s>>>(he, H, bits);
    if (exclusive_scan<int32_t>(bits, pre, H, tiles, total + 1, s) != cudaSuccess) return CCS_ERR_CUDA;
    k_edges<<<nblk(H), kB, 0, s>>>(he, H, pre, e2h);
    k_v2h_max<<<nblk(H), kB, 0, s>>>(he, H, v2h);
    k_v2h_boundary<<<nblk(H), kB, 0, s>>>(he, H, v2h);
    int32_t E = 0;
    if (cudaMemcpyAsync(&E, total + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCS_ERR_CUDA;
    if (hostErr) return CCS_ERR_ARG;
    // creases
    if (T > 0) k_tags<<<nblk(T), kB, 0, s>>>(tags, T, V, he, start, bucket, winner);
    k_crease_values<<<nblk(E), kB, 0, s>>>(cr, E, winner, sharp, he, e2h);
    k_crease_links<<<nblk(E), kB, 0, s>>>(cr, E, he, e2h);
    if (cudaGetLastError() != cudaSuccess) return CCS_ERR_CUDA;

    cc_Mesh* c = alloc_cage_block(V, U, H, E, F);
    if (!c) return CCS_ERR_ALLOC;
    ok = cudaMemcpyAsync(c->halfedges, he, sizeof(cc_Halfedge) * (size_t)H, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(c->creases, cr, sizeof(cc_Crease) * (size_t)E, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(c->vertexToHalfedgeIDs, v2h, sizeof(int32_t) * (size_t)V, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(c->edgeToHalfedgeIDs, e2h, sizeof(int32_t) * (size_t)E, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(c->faceToHalfedgeIDs, f2h, sizeof(int32_t) * (size_t)F, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(c->vertexPoints, m->vertexPoints, sizeof(float) * 3 * (size_t)V, cudaMemcpyDefault, s) == cudaSuccess &&
         (U == 0 || cudaMemcpyAsync(c->uvs, m->uvs, sizeof(float) * 2 * (size_t)U, cudaMemcpyDefault, s) == cudaSuccess) &&
         cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) {
        free_cage_block(c);
        return CCS_ERR_CUDA;
    }
    *out = c;
    return CCS_OK;
}

}  // namespace
}  // namespace ccs

extern "C" int ccs_BuildCage_cuda(const ccs_PolygonMesh* mesh, cc_Mesh** out, void* stream) {
    if (out) *out = nullptr;
    return ccs::set_last_error(ccs::build(mesh, out, (cudaStream_t)stream));
}
