// ccs_normals.cu -- per-halfedge normals of the finest level (a consumer of
// the refined surface).
//
// The reference computes these on the GPU in its GLSL library
// (glsl/CatmullClark_Scatter.glsl:931-960): the "fast" normal of halfedge h
// is the normalised cross product of its face's two edges at h,
//   n(h) = normalize(cross(P[v(next h)] - P[v(h)], P[v(prev h)] - P[v(h)])),
// and the smooth normal adds the fast normals of the other halfedges around
// v(h) (walking prev-vertex halfedges) and normalises the sum; on a boundary
// vertex it is the fast normal.  Here one thread per halfedge of the finest
// level; the ring walk is bounded like every walk in this library.
#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBlockN = 256;

__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return f3{fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)}; }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return f3{fsub(fmul(a.y, b.z), fmul(a.z, b.y)), fsub(fmul(a.z, b.x), fmul(a.x, b.z)),
              fsub(fmul(a.x, b.y), fmul(a.y, b.x))};
}
__device__ __forceinline__ f3 normalize3(f3 v) {
    const float r = rsqrtf(fadd(fadd(fmul(v.x, v.x), fmul(v.y, v.y)), fmul(v.z, v.z)));
    return mul3(v, r);
}

template <int RW>
__device__ __forceinline__ f3 fast_normal(const QuadView<RW>& L, const float* __restrict__ pts, int32_t h) {
    const f3 v0 = ld3(pts + 3 * (int64_t)L.vert(h));
    const f3 v1 = ld3(pts + 3 * (int64_t)L.vert(qprev(h)));
    const f3 v2 = ld3(pts + 3 * (int64_t)L.vert(qnext(h)));
    return normalize3(cross3(sub3(v2, v0), sub3(v1, v0)));
}

template <int RW, bool SMOOTH>
__global__ void __launch_bounds__(kBlockN)
k_halfedge_normals(QuadView<RW> L, const float* __restrict__ pts, float* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.H) return;
    const int32_t h = (int32_t)i;
    f3 n = fast_normal(L, pts, h);
    if (SMOOTH) {
        f3 sum = zero3();
        int32_t it = L.prev_vertex_he(h);
        int guard = 0;
        for (; it >= 0 && it != h && guard < kWalkCap; it = L.prev_vertex_he(it), ++guard)
            sum = add3(sum, fast_normal(L, pts, it));
        if (it >= 0) n = normalize3(add3(n, sum));
    }
    st3(out + 3 * i, n);
}

template <int RW>
static void launch_normals(const Ctx& c, const float* p, float* out, bool smooth) {
    const int D = c.D;
    const Level& lv = c.lv[D];
    QuadView<RW> L;
    L.t = make_cage_tables(*c.cage);
    L.he = c.he + (int64_t)RW * lv.heOff;
    L.cr = c.cr + lv.crOff;
    L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C; L.d = D;
    const unsigned nb = (unsigned)((lv.H + kBlockN - 1) / kBlockN);
    if (smooth) k_halfedge_normals<RW, true><<<nb, kBlockN, 0, c.stream>>>(L, p, out);
    else k_halfedge_normals<RW, false><<<nb, kBlockN, 0, c.stream>>>(L, p, out);
}

cudaError_t run_normals(const Ctx& c, const float* pts, float* out, bool smooth) {
    const float* p = pts + 3 * c.lv[c.D].ptOff;
    if (c.rw == 4) launch_normals<4>(c, p, out, smooth);
    else launch_normals<3>(c, p, out, smooth);
    return cudaGetLastError();
}

}  // namespace ccs
