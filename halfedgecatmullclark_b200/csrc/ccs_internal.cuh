// ccs_internal.cuh -- device-side building blocks of the refinement kernels.
//
// Everything here mirrors the arithmetic of jdupuy/HalfedgeCatmullClark's
// CatmullClark.h exactly: float operations go through __f*_rn intrinsics so
// that nvcc never contracts a*b+c into an FMA (the reference's x86-64 build
// has none), and the order of every sum and lerp is the reference's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ccs_cuda.h"
#include "ccs_host.h"

namespace ccs {

// Upper bound on the steps of any ring or face walk in device code.
static constexpr int kWalkCap = 1 << 16;

// Programmatic dependent launch, for kernels launched by launch_chained: wait
// until the previous grid in the stream has completed and its memory is
// visible (a no-op for a kernel launched the ordinary way), then let the next
// grid be launched (it fires once every block of this grid has run it, so
// the next grid's blocks, which wait in turn, only fill slots this grid has
// left).  Both must come before the kernel touches global memory.
__device__ __forceinline__ void chain_wait_then_release() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Exact float helpers (CatmullClark.h:295-392)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// x + u * (y - x)  (cc__Lerpfv, :321-327)
__device__ __forceinline__ float flerp(float x, float y, float u) { return fadd(x, fmul(u, fsub(y, x))); }
__device__ __forceinline__ float fmax_ref(float x, float y) { return x > y ? x : y; }   // :300-303
__device__ __forceinline__ float fmin_ref(float x, float y) { return x < y ? x : y; }   // :295-298
__device__ __forceinline__ float fsat(float x) { return fmax_ref(0.0f, fmin_ref(x, 1.0f)); }  // :305-308
__device__ __forceinline__ float fsign(float x) { return x < 0.0f ? -1.0f : (x > 0.0f ? 1.0f : 0.0f); }  // :310-319

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 ld3(const float* __restrict__ p) { return f3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(float* p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
__device__ __forceinline__ f3 add3(f3 a, f3 b) { return f3{fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)}; }
__device__ __forceinline__ f3 mul3(f3 a, float s) { return f3{fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)}; }
__device__ __forceinline__ f3 div3(f3 a, float s) { return f3{fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s)}; }
// x / 4 and x * 0.25 are the same correctly rounded value of x * 2^-2, so the
// reference's divisions by 4.0f are taken as multiplications.
__device__ __forceinline__ float fquarter(float x) { return __fmul_rn(x, 0.25f); }
__device__ __forceinline__ f3 quarter3(f3 a) { return f3{fquarter(a.x), fquarter(a.y), fquarter(a.z)}; }
// 1.0f / x, correctly rounded (the same value as IEEE division).
__device__ __forceinline__ float frcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ f3 lerp3(f3 a, f3 b, float u) { return f3{flerp(a.x, b.x, u), flerp(a.y, b.y, u), flerp(a.z, b.z, u)}; }
__device__ __forceinline__ f3 zero3() { return f3{0.0f, 0.0f, 0.0f}; }

// UV codec (CatmullClark.h:374-392).  The reference converts float ->
// uint32_t; its x86-64 build truncates through a signed 64-bit integer and
// keeps the low 32 bits, which this reproduces for every input.
__device__ __forceinline__ float uv_dec(uint32_t x) { return fdiv((float)(x & 0xFFFFu), 65535.0f); }
__device__ __forceinline__ uint32_t f2u32_trunc(float x) {
    if (!(x > -9.2e18f && x < 9.2e18f)) return 0u;
    return (uint32_t)(unsigned long long)__float2ll_rz(x);
}
__device__ __forceinline__ int32_t uv_enc(float u, float v) {
    const uint32_t a = f2u32_trunc(fmul(u, 65535.0f));
    const uint32_t b = f2u32_trunc(fmul(v, 65535.0f));
    return (int32_t)((a & 0xFFFFu) | ((b & 0xFFFFu) << 16));
}

// Quad-level face arithmetic (CatmullClark.h:667-689)
__device__ __forceinline__ int32_t qnext(int32_t h) { return (h & ~3) | ((h + 1) & 3); }
__device__ __forceinline__ int32_t qprev(int32_t h) { return (h & ~3) | ((h - 1) & 3); }
// 4 * x + k with two's-complement wrap, as the reference's int32 arithmetic
__device__ __forceinline__ int32_t child(int32_t x, int32_t k) { return (int32_t)((uint32_t)x * 4u + (uint32_t)k); }

// ---------------------------------------------------------------------------
// Cage counts for the O(depth) maps (CatmullClark.h:465-585)
// ---------------------------------------------------------------------------
struct CageCounts {
    int32_t V, F, E, H;
};
__device__ __forceinline__ int32_t ones32(int32_t n) { return (int32_t)~(0xFFFFFFFFu << n); }
__device__ __forceinline__ int32_t cnt_F(const CageCounts& c, int32_t d) {
    return d == 0 ? c.F : (int32_t)((uint32_t)c.H << ((d - 1) << 1));
}
__device__ __forceinline__ int32_t cnt_E(const CageCounts& c, int32_t d) {
    if (d == 0) return c.E;
    return (int32_t)(((uint32_t)c.E * 2u + (uint32_t)ones32(d) * (uint32_t)c.H) << (d - 1));
}
__device__ __forceinline__ int32_t cnt_V(const CageCounts& c, int32_t d) {
    if (d == 0) return c.V;
    const uint32_t F1 = (uint32_t)c.H, E1 = 2u * (uint32_t)c.E + (uint32_t)c.H;
    const uint32_t V1 = (uint32_t)(c.V + c.E + c.F), t = (uint32_t)ones32(d - 1);
    return (int32_t)(V1 + t * (E1 + t * F1));
}

// ---------------------------------------------------------------------------
// Level views.  A view exposes one level of the hierarchy (the cage, or
// quad level d >= 1) with the reference's accessor names.
// ---------------------------------------------------------------------------
// cc_Halfedge words (CatmullClark.h:37-45)
enum { CH_TWIN = 0, CH_NEXT, CH_PREV, CH_FACE, CH_EDGE, CH_VERT, CH_UV, CH_WORDS };

struct CageTables {
    const int32_t* __restrict__ he;    // cage cc_Halfedge records (7 words)
    const int32_t* __restrict__ v2h;
    const int32_t* __restrict__ e2h;
    const int32_t* __restrict__ f2h;
    const int32_t* __restrict__ fsz;   // cage face sizes
    const float* __restrict__ uvs;     // U x 2
    const int32_t* __restrict__ vshape;  // cage vertex ring shapes (DevCage::vshape), or null
    CageCounts n;
};

__host__ __device__ inline CageTables make_cage_tables(const DevCage& c) {
    CageTables t;
    t.he = c.he; t.v2h = c.v2h; t.e2h = c.e2h; t.f2h = c.f2h; t.fsz = c.fsz; t.uvs = c.uvs;
    t.vshape = c.vshape;
    t.n.V = c.V; t.n.F = c.F; t.n.E = c.E; t.n.H = c.H;
    return t;
}

struct CageView {
    static constexpr bool kQuad = false;
    CageTables t;
    const cc_Crease* __restrict__ cr;  // cage creases (one per edge)
    int32_t V, F, E, H, C;
    int32_t d;                         // always 0
    __device__ __forceinline__ int32_t rec(int32_t h, int w) const { return t.he[(int64_t)CH_WORDS * h + w]; }
    __device__ __forceinline__ int32_t twin(int32_t h) const { return rec(h, CH_TWIN); }
    __device__ __forceinline__ int32_t next(int32_t h) const { return rec(h, CH_NEXT); }
    __device__ __forceinline__ int32_t prev(int32_t h) const { return rec(h, CH_PREV); }
    __device__ __forceinline__ int32_t face(int32_t h) const { return rec(h, CH_FACE); }
    __device__ __forceinline__ int32_t edge(int32_t h) const { return rec(h, CH_EDGE); }
    __device__ __forceinline__ int32_t vert(int32_t h) const { return rec(h, CH_VERT); }
    __device__ __forceinline__ float sharp(int32_t e) const { return cr[e].sharpness; }       // :629-638
    __device__ __forceinline__ float hsharp(int32_t h) const { return sharp(edge(h)); }
    // twin(h) >= 0 ? next(twin(h)) : -1  (:744-749)
    __device__ __forceinline__ int32_t next_vertex_he(int32_t h) const {
        const int32_t tw = twin(h);
        return tw >= 0 ? next(tw) : -1;
    }
    __device__ __forceinline__ int32_t prev_vertex_he(int32_t h) const { return twin(prev(h)); }  // :751-756
    __device__ __forceinline__ int32_t edge_he(int32_t e) const { return t.e2h[e]; }
    __device__ __forceinline__ int32_t vert_he(int32_t v) const { return t.v2h[v]; }
    __device__ __forceinline__ int32_t face_he(int32_t f) const { return t.f2h[f]; }
};

template <int RW>
struct QuadView {
    static constexpr bool kQuad = true;
    CageTables t;
    const int32_t* __restrict__ he;    // level-d cc_Halfedge_SemiRegular records (RW words)
    const cc_Crease* __restrict__ cr;  // level-d creases
    int32_t V, F, E, H, C;
    int32_t d;
    // optional (adjoint): ring statistics of the older vertices v < V(d-1),
    // {valence, summed sharpness, crease count, boundary ? 1 : 0}
    const float4* __restrict__ ostats = nullptr;
    __device__ __forceinline__ int32_t rec(int32_t h, int w) const { return he[(int64_t)RW * h + w]; }
    __device__ __forceinline__ int32_t twin(int32_t h) const { return rec(h, 0); }
    __device__ __forceinline__ int32_t edge(int32_t h) const { return rec(h, 1); }
    __device__ __forceinline__ int32_t vert(int32_t h) const { return rec(h, 2); }
    __device__ __forceinline__ int32_t next(int32_t h) const { return qnext(h); }
    __device__ __forceinline__ int32_t prev(int32_t h) const { return qprev(h); }
    __device__ __forceinline__ int32_t face(int32_t h) const { return h >> 2; }
    // edges past the crease range never carry a crease (:1011-1021)
    __device__ __forceinline__ float sharp(int32_t e) const { return e < C ? cr[e].sharpness : 0.0f; }
    __device__ __forceinline__ float hsharp(int32_t h) const { return sharp(edge(h)); }
    __device__ __forceinline__ int32_t next_vertex_he(int32_t h) const { return qnext(twin(h)); }  // :1177-1182
    __device__ __forceinline__ int32_t prev_vertex_he(int32_t h) const { return twin(qprev(h)); }  // :1168-1175
    __device__ __forceinline__ int32_t face_he(int32_t f) const { return f << 2; }
    __device__ int32_t edge_he(int32_t e) const;
    __device__ int32_t vert_he(int32_t v) const;
};

// ccs_EdgeToHalfedgeID (CatmullClark.h:1206-1303): O(depth) walk down to the
// cage through the edge numbering of each refinement step.
__device__ __forceinline__ int32_t edge_to_he_first(const CageTables& t, int32_t e) {
    if (e >= 2 * t.n.E) {
        const int32_t h = e - 2 * t.n.E, n = t.he[(int64_t)CH_WORDS * h + CH_NEXT];
        const int32_t a = 4 * h + 1, b = 4 * n + 2;
        return a > b ? a : b;
    } else if (e & 1) {
        return 4 * t.he[(int64_t)CH_WORDS * t.e2h[e >> 1] + CH_NEXT] + 3;
    }
    return 4 * t.e2h[e >> 1] + 0;
}
__device__ __forceinline__ int32_t edge_to_he(const CageTables& t, int32_t e, int32_t d) {
    uint32_t heap = 1u;
    int32_t id = 0, hd = d;
    for (; hd > 1; --hd) {
        const int32_t Ec = cnt_E(t.n, hd - 1);
        if (e >= 2 * Ec) {
            const int32_t h = e - 2 * Ec, n = qnext(h);
            const int32_t a = 4 * h + 1, b = 4 * n + 2;
            id = a > b ? a : b;
            break;
        }
        heap = (heap << 1) | (uint32_t)(e & 1);
        e >>= 1;
    }
    if (hd == 1) id = edge_to_he_first(t, e);
    while (heap > 1u) {
        id = (heap & 1u) ? 4 * qnext(id) + 3 : 4 * id + 0;
        heap >>= 1;
    }
    return id;
}
// ccs_VertexPointToHalfedgeID (CatmullClark.h:1313-1395)
__device__ __forceinline__ int32_t vertex_to_he(const CageTables& t, int32_t v, int32_t d) {
    int32_t hd = d, stride = 0, h = 0;
    for (; hd > 1; --hd) {
        const int32_t Vc = cnt_V(t.n, hd - 1), Fc = cnt_F(t.n, hd - 1);
        if (v >= Vc + Fc) {
            h = 4 * edge_to_he(t, v - Fc - Vc, hd - 1) + 1;
            break;
        } else if (v >= Vc) {
            h = 4 * (4 * (v - Vc)) + 2;
            break;
        }
        stride += 2;
    }
    if (hd == 1) {
        if (v >= t.n.V + t.n.F) h = 4 * t.e2h[v - t.n.V - t.n.F] + 1;
        else if (v >= t.n.V) h = 4 * t.f2h[v - t.n.V] + 2;
        else h = 4 * t.v2h[v] + 0;
    }
    return h << stride;
}
template <int RW>
__device__ __forceinline__ int32_t QuadView<RW>::edge_he(int32_t e) const { return edge_to_he(t, e, d); }
template <int RW>
__device__ __forceinline__ int32_t QuadView<RW>::vert_he(int32_t v) const { return vertex_to_he(t, v, d); }

// ---------------------------------------------------------------------------
// Per-halfedge point rules (scatter form).  `pin` holds level-d points,
// `fpt`/`ept` the face / edge points of level d+1.
// ---------------------------------------------------------------------------

// Creased edge rule, one halfedge's share (:1602-1648, :2194-2241)
template <class View>
__device__ __forceinline__ f3 creased_edge_share(const View& L, int32_t h, const float* __restrict__ pin,
                                                 const float* __restrict__ fpt) {
    const int32_t tw = L.twin(h);
    const float w = fsat(L.sharp(L.edge(h)));
    const f3 F = ld3(fpt + 3 * (int64_t)L.face(h));
    const f3 v0 = ld3(pin + 3 * (int64_t)L.vert(h));
    const f3 v1 = ld3(pin + 3 * (int64_t)L.vert(L.next(h)));
    const f3 sharpP = mul3(lerp3(v0, v1, 0.5f), tw < 0 ? 1.0f : 0.5f);
    const f3 smoothP = mul3(lerp3(v0, F, 0.5f), 0.5f);
    return lerp3(smoothP, sharpP, w);
}

// Crease-free edge rule, one halfedge's share (:1517-1548, :2107-2139)
template <class View>
__device__ __forceinline__ f3 smooth_edge_share(const View& L, int32_t h, const float* __restrict__ pin,
                                                const float* __restrict__ fpt) {
    const int32_t tw = L.twin(h);
    const f3 F = ld3(fpt + 3 * (int64_t)L.face(h));
    const f3 v0 = ld3(pin + 3 * (int64_t)L.vert(h));
    const f3 v1 = ld3(pin + 3 * (int64_t)L.vert(L.next(h)));
    const float w = tw >= 0 ? 0.5f : 1.0f;
    const f3 t1 = mul3(F, 0.5f);
    const f3 t4 = lerp3(mul3(v0, w), mul3(v1, w), 0.5f);
    return lerp3(t1, t4, w);
}

// Ring statistics of the creased vertex rule seen from halfedge h
// (:1899-1936 on the cage, :2523-2566 on quad levels).
struct RingStats {
    float avgS, creaseCount, valence;
    int32_t fwd;
};
template <class View>
__device__ __forceinline__ RingStats creased_ring_walk(const View& L, int32_t h);

// On a quad level the vertex of halfedge h (child h&3 of a parent halfedge)
// is known: child 2 sits on a face centre (valence = the parent face's size,
// every incident edge crease-free), children 1 and 3 on an edge midpoint
// (valence 4, or 2 on a boundary; the only creased edges are the two halves
// e, e^1 of the parent edge).  Sharpness at depth >= 1 is +0, positive or
// NaN, so the walk's sums of these values with zeros are exactly the sums
// below.  Returns false for child 0 (an older vertex: walk its ring).
template <int RW>
__device__ __forceinline__ bool quad_ring_known(const QuadView<RW>& L, int32_t h, RingStats& r) {
    const int k = h & 3;
    if (k == 0) return false;
    if (k == 2) {
        const int32_t n = L.d == 1 ? L.t.fsz[L.t.he[(int64_t)CH_WORDS * (h >> 2) + CH_FACE]] : 4;
        r.valence = (float)n; r.creaseCount = 0.0f; r.avgS = 0.0f; r.fwd = h;
        return true;
    }
    const int32_t eh = k == 1 ? L.edge(h - 1) : L.edge(h);      // a half of the parent edge
    const bool bnd = (k == 1 ? L.twin(h - 1) : L.twin(h)) < 0;
    const float sa = L.sharp(eh), sb = L.sharp(eh ^ 1);
    const bool own = k == 3;                                     // the walk skips h's own edge
    r.valence = bnd ? 2.0f : 4.0f;
    r.avgS = (bnd && own) ? sb : fadd(sa, sb);
    r.creaseCount = (bnd && own) ? fsign(sb) : fadd(fsign(sa), fsign(sb));
    r.fwd = bnd ? -1 : h;
    return true;
}
__device__ __forceinline__ bool quad_ring_known(const CageView&, int32_t, RingStats&) { return false; }

// Child 0 (an older vertex) from precomputed whole-ring statistics: the walk
// from h sees every incident edge but, on a boundary, its own.  The
// subtraction makes avgS differ from the walk's sum by rounding only; the
// adjoint uses this, the forward passes never set ostats.
template <int RW>
__device__ __forceinline__ bool ring_from_stats(const QuadView<RW>& L, int32_t h, RingStats& r) {
    if (!L.ostats) return false;
    const float4 s = L.ostats[L.vert(h)];
    const bool bnd = s.w != 0.0f;
    const float own = L.hsharp(h);
    r.valence = s.x;
    r.avgS = bnd ? fsub(s.y, own) : s.y;
    r.creaseCount = bnd ? fsub(s.z, fsign(own)) : s.z;
    r.fwd = bnd ? -1 : h;
    return true;
}
__device__ __forceinline__ bool ring_from_stats(const CageView&, int32_t, RingStats&) { return false; }

template <class View>
__device__ __forceinline__ RingStats creased_ring(const View& L, int32_t h) {
    RingStats r;
    if (quad_ring_known(L, h, r)) return r;
    if (ring_from_stats(L, h, r)) return r;
    return creased_ring_walk(L, h);
}

template <class View>
__device__ __forceinline__ RingStats creased_ring_walk(const View& L, int32_t h) {
    RingStats r;
    const int32_t prev = L.prev(h);
    const float prevS = L.hsharp(prev);
    r.avgS = prevS;
    r.creaseCount = fsign(prevS);
    r.valence = 1.0f;
    int32_t fwd, bwd;
    // Both walks terminate on a manifold ring; the cap only bounds the work
    // on a malformed one (it never triggers on a valid mesh).
    int guard = 0;
    for (fwd = L.twin(prev); fwd >= 0 && fwd != h && guard < kWalkCap; fwd = L.twin(fwd), ++guard) {
        const int32_t p = L.prev(fwd);
        const float s = L.hsharp(p);
        r.valence = fadd(r.valence, 1.0f);
        r.avgS = fadd(r.avgS, s);
        r.creaseCount = fadd(r.creaseCount, fsign(s));
        fwd = p;
    }
    guard = 0;
    for (bwd = L.twin(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kWalkCap; bwd = L.twin(bwd), ++guard) {
        const int32_t n = L.next(bwd);
        const float s = L.hsharp(n);
        r.valence = fadd(r.valence, 1.0f);
        r.avgS = fadd(r.avgS, s);
        r.creaseCount = fadd(r.creaseCount, fsign(s));
        bwd = n;
    }
    r.fwd = fwd;
    return r;
}

// Creased vertex rule, one halfedge's share (:1872-1991 cage, smooth-first
// branch order; :2496-2615 quad levels, corner-first branch order).
template <class View>
__device__ __forceinline__ f3 creased_vertex_share(const View& L, int32_t h, const float* __restrict__ pin,
                                                   const float* __restrict__ fpt, const float* __restrict__ ept) {
    const RingStats r = creased_ring(L, h);
    const int32_t prev = L.prev(h);
    const float cw = fsign(L.hsharp(h)), pcw = fsign(L.hsharp(prev));
    const f3 E = ld3(ept + 3 * (int64_t)L.edge(h));
    const f3 F = ld3(fpt + 3 * (int64_t)L.face(h));
    const f3 P = ld3(pin + 3 * (int64_t)L.vert(h));
    float valence = r.valence, creaseCount = r.creaseCount;

    const f3 corner = mul3(P, frcp(valence));
    f3 crease = add3(mul3(P, fmul(0.25f, cw)), mul3(E, fmul(0.25f, cw)));
    f3 smooth = add3(mul3(F, -1.0f), mul3(E, 4.0f));
    smooth = add3(smooth, mul3(P, fsub(valence, 3.0f)));
    smooth = mul3(smooth, frcp(fmul(valence, valence)));
    if (r.fwd < 0) {
        creaseCount = fadd(creaseCount, cw);
        valence = fadd(valence, 1.0f);
        const f3 Ep = ld3(ept + 3 * (int64_t)L.edge(prev));
        crease = add3(crease, add3(mul3(P, fmul(0.25f, pcw)), mul3(Ep, fmul(0.25f, pcw))));
    }
    if (View::kQuad) {
        if (creaseCount >= 3.0f || valence == 2.0f) return corner;
        if (creaseCount <= 1.0f) return smooth;
    } else {
        if (creaseCount <= 1.0f) return smooth;
        if (creaseCount >= 3.0f || valence == 2.0f) return corner;
    }
    return lerp3(corner, crease, fsat(fmul(r.avgS, 0.5f)));
}

// Crease-free vertex rule, one halfedge's share (:1713-1756, :2307-2351)
template <class View>
__device__ __forceinline__ f3 smooth_vertex_share(const View& L, int32_t h, const float* __restrict__ pin,
                                                  const float* __restrict__ fpt, const float* __restrict__ ept) {
    int32_t valence = 1, fwd, bwd, guard = 0;
    RingStats known;
    if (quad_ring_known(L, h, known)) {      // the valence and boundary are all this rule uses
        valence = (int32_t)known.valence;
        fwd = known.fwd;
    } else {
        for (fwd = L.prev_vertex_he(h); fwd >= 0 && fwd != h && guard < kWalkCap; fwd = L.prev_vertex_he(fwd), ++guard)
            ++valence;
        guard = 0;
        for (bwd = L.next_vertex_he(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kWalkCap; bwd = L.next_vertex_he(bwd), ++guard)
            ++valence;
    }
    const f3 v = ld3(pin + 3 * (int64_t)L.vert(h));
    const f3 f = ld3(fpt + 3 * (int64_t)L.face(h));
    const f3 e = ld3(ept + 3 * (int64_t)L.edge(h));
    const float w = frcp((float)valence);
    const float s = fwd < 0 ? 0.0f : 1.0f;
    const float ws = fmul(w, s);
    f3 o;
    o.x = fmul(w, fadd(v.x, fmul(ws, fsub(fsub(fmul(4.0f, e.x), f.x), fmul(3.0f, v.x)))));
    o.y = fmul(w, fadd(v.y, fmul(ws, fsub(fsub(fmul(4.0f, e.y), f.y), fmul(3.0f, v.y)))));
    o.z = fmul(w, fadd(v.z, fmul(ws, fsub(fsub(fmul(4.0f, e.z), f.z), fmul(3.0f, v.z)))));
    return o;
}

}  // namespace ccs
