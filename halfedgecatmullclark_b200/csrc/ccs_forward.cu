// ccs_forward.cu -- forward refinement kernels for sm_100a.
//
// One refinement step reads depth d (the cage when d == 0) and writes depth
// d + 1 of the packed hierarchy (CatmullClark.h:136-142):
//   topology  : 4 child halfedge records per parent halfedge (+ UV codes)
//   creases   : 2 child creases per parent crease
//   points    : face points, then edge points, then vertex points.
//
// Data layout in HBM (all offsets 64-bit):
//   halfedges  cumH x {twin, edge, vertex, uv} int32 (16 B) or 12 B records
//   creases    cumC x {next, prev, sharpness} (12 B)
//   points     cumV x float3 (12 B); depth d+1 = [old vertices | faces | edges]
//
// Kernel shapes:
//   * topology: one thread per CHILD halfedge.  The four records of the
//     parent face are read as four 16-byte vector loads shared through L1 by
//     the 16 lanes that work on that face; each lane then writes its child
//     record with one 16-byte store, so a warp writes 512 contiguous bytes.
//   * face points: one thread per face.
//   * edge points: one thread per halfedge; the thread whose halfedge holds
//     its pair's larger ID adds both halves of the edge rule, so the edge
//     point is stored once, without atomics (two addends commute exactly).
//   * vertex points, scatter rule: one thread per halfedge walks the vertex
//     ring; the per-halfedge shares are summed across the warp for lanes
//     that hit the same vertex (match.any + shuffles) and one float atomic
//     per vertex and warp goes to memory.
//   * vertex points, deterministic scatter rule: one thread per vertex
//     enumerates the ring and adds the shares in increasing halfedge order
//     -- the order a single-threaded reference run applies them in.
//   * gather rule: one thread per face / edge / vertex, as the reference's
//     gather routines do.
#include <cstdio>

#include "ccs_host.h"
#include "ccs_tiles.cuh"

namespace ccs {

static constexpr int kBlock = 256;
static constexpr int kRingCap = 1 << 16;   // bound on every ring / face walk

static inline unsigned nblocks(int64_t n, int bs = kBlock) { return (unsigned)((n + bs - 1) / bs); }

// ---------------------------------------------------------------------------
// Topology + UVs, quad level (CatmullClark.h:2749-2796, :2878-2921)
// ---------------------------------------------------------------------------
template <int RW, bool TOPO, bool UV>
__global__ void __launch_bounds__(kBlock)
k_quad_topology(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                int32_t H, int32_t V, int32_t F, int32_t E) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= 4 * (int64_t)H) return;
    const int32_t h = (int32_t)(c >> 2), m = (int32_t)(c & 3);
    const int32_t f = h >> 2, k = h & 3, base = f << 2;
    int32_t tw[4], ed[4], vx[4], uv[4];
    if constexpr (RW == 4) {
        const int4* q = reinterpret_cast<const int4*>(in) + base;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int4 r = __ldg(q + i);
            tw[i] = r.x; ed[i] = r.y; vx[i] = r.z; uv[i] = r.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            tw[i] = __ldg(in + 3 * (int64_t)(base + i) + 0);
            ed[i] = __ldg(in + 3 * (int64_t)(base + i) + 1);
            vx[i] = __ldg(in + 3 * (int64_t)(base + i) + 2);
            uv[i] = 0;
        }
    }
    const int kp = (k + 3) & 3, kn = (k + 1) & 3;
    const int32_t prev = base | kp, next = base | kn;
    int32_t o_tw = 0, o_ed = 0, o_vx = 0, o_uv = 0;
    if (TOPO) {
        switch (m) {
            case 0: o_tw = child(qnext(tw[k]), 3); o_ed = 2 * ed[k] + (h > tw[k] ? 0 : 1); o_vx = vx[k]; break;
            case 1: o_tw = child(next, 2); o_ed = 2 * E + h; o_vx = V + F + ed[k]; break;
            case 2: o_tw = child(prev, 1); o_ed = 2 * E + prev; o_vx = V + f; break;
            default: o_tw = child(tw[kp], 0); o_ed = 2 * ed[kp] + (prev > tw[kp] ? 1 : 0); o_vx = V + F + ed[kp]; break;
        }
    }
    if (UV) {
        const uint32_t cu = (uint32_t)uv[k];
        const float u = uv_dec(cu), v = uv_dec(cu >> 16);
        switch (m) {
            case 0: o_uv = uv[k]; break;
            case 1: {
                const uint32_t cn = (uint32_t)uv[kn];
                o_uv = uv_enc(flerp(u, uv_dec(cn), 0.5f), flerp(v, uv_dec(cn >> 16), 0.5f));
                break;
            }
            case 2: {
                float fu = u, fv = v;
#pragma unroll
                for (int i = 1; i < 4; ++i) {
                    const uint32_t q = (uint32_t)uv[(k + i) & 3];
                    fu = fadd(fu, uv_dec(q));
                    fv = fadd(fv, uv_dec(q >> 16));
                }
                o_uv = uv_enc(fquarter(fu), fquarter(fv));
                break;
            }
            default: {
                const uint32_t cp = (uint32_t)uv[kp];
                o_uv = uv_enc(flerp(u, uv_dec(cp), 0.5f), flerp(v, uv_dec(cp >> 16), 0.5f));
                break;
            }
        }
    }
    if constexpr (RW == 4 && TOPO && UV) {
        reinterpret_cast<int4*>(out)[c] = make_int4(o_tw, o_ed, o_vx, o_uv);
    } else {
        int32_t* o = out + (int64_t)RW * c;
        if (TOPO) { o[0] = o_tw; o[1] = o_ed; o[2] = o_vx; }
        if (UV && RW == 4) o[3] = o_uv;
    }
}

// ---------------------------------------------------------------------------
// Cage topology + UVs, creases, face / edge / vertex points: thin kernels
// over the item functions of ccs_tiles.cuh (shared with the batched path).
// ---------------------------------------------------------------------------
template <int RW, bool TOPO, bool UV>
__global__ void __launch_bounds__(kBlock)
k_cage_topology(CageTables t, int32_t* __restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < 4 * (int64_t)t.n.H) cage_topology_item<RW, TOPO, UV>(t, out, c);
}

__global__ void __launch_bounds__(kBlock)
k_creases(const cc_Crease* __restrict__ in, cc_Crease* __restrict__ out, int32_t C) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < C) crease_item(in, out, (int32_t)i);
}

template <class View, bool GATHER_SEM>
__global__ void __launch_bounds__(kBlock)
k_face_points(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.F) face_point_item<View, GATHER_SEM>(L, pin, pout, (int32_t)i);
}

// face points and the cleared vertex slots of the atomic pass in one launch
// (grid over max(F, V); the two write disjoint ranges of pout)
template <class View>
__global__ void __launch_bounds__(kBlock)
k_face_points_clear(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.F) face_point_item<View, false>(L, pin, pout, (int32_t)i);
    if (i < L.V) st3(pout + 3 * i, zero3());
}

template <class View, bool CREASED>
__global__ void __launch_bounds__(kBlock)
k_edge_owner(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.H) edge_owner_item<View, CREASED>(L, pin, pout, (int32_t)i);
}

// Edge points, gather rule (:1476-1515, :1561-1600, :2065-2105, :2151-2191)
template <class View, bool CREASED>
__global__ void __launch_bounds__(kBlock)
k_edge_gather(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.E) return;
    const int32_t e = (int32_t)i;
    const float* fpt = pout + 3 * (int64_t)L.V;
    float* ept = pout + 3 * ((int64_t)L.V + L.F);
    const int32_t h = L.edge_he(e), tw = L.twin(h), n = L.next(h);
    const f3 v0 = ld3(pin + 3 * (int64_t)L.vert(h)), v1 = ld3(pin + 3 * (int64_t)L.vert(n));
    const f3 f0 = ld3(fpt + 3 * (int64_t)L.face(h));
    const f3 f1 = ld3(fpt + 3 * (int64_t)L.face(tw > 0 ? tw : 0));
    const f3 t1 = add3(v0, v1), t2 = add3(f0, f1);
    const f3 sharpP = mul3(t1, 0.5f);
    const f3 smoothP = mul3(add3(t1, t2), 0.25f);
    if (CREASED) st3(ept + 3 * (int64_t)e, lerp3(smoothP, sharpP, fsat(L.sharp(e))));
    else st3(ept + 3 * (int64_t)e, lerp3(sharpP, smoothP, tw < 0 ? 0.0f : 1.0f));
}

// Vertex points, scatter rule with warp-aggregated float atomics
template <class View, bool CREASED>
__global__ void __launch_bounds__(kBlock)
k_vertex_atomic(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    vertex_atomic_item<View, CREASED>(L, pin, pout, (int32_t)i, i < L.H);
}

// ---------------------------------------------------------------------------
// Vertex points, scatter rule summed per vertex in increasing halfedge order
// ---------------------------------------------------------------------------
template <class View, bool CREASED>
__global__ void __launch_bounds__(kBlock)
k_vertex_det(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.V) vertex_det_item<View, CREASED>(L, pin, pout, (int32_t)i);
}

// ---------------------------------------------------------------------------
// Vertex points, gather rules (:1661-1711, :1769-1869, :2254-2305, :2364-2493)
// ---------------------------------------------------------------------------
template <class View>
__global__ void __launch_bounds__(kBlock)
k_vertex_gather_smooth(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.V) return;
    const int32_t v = (int32_t)i;
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    const int32_t h = L.vert_he(v);
    const f3 P = ld3(pin + 3 * (int64_t)v);
    f3 smooth = add3(mul3(ld3(fpt + 3 * (int64_t)L.face(h)), -1.0f), mul3(ld3(ept + 3 * (int64_t)L.edge(h)), 4.0f));
    float valence = 1.0f;
    int32_t it;
    int guard = 0;
    for (it = L.prev_vertex_he(h); it >= 0 && it != h && guard < kRingCap; it = L.prev_vertex_he(it), ++guard) {
        smooth = add3(smooth, mul3(ld3(fpt + 3 * (int64_t)L.face(it)), -1.0f));
        smooth = add3(smooth, mul3(ld3(ept + 3 * (int64_t)L.edge(it)), 4.0f));
        valence = fadd(valence, 1.0f);
    }
    smooth = add3(mul3(smooth, frcp(fmul(valence, valence))), mul3(P, fsub(1.0f, fdiv(3.0f, valence))));
    st3(pout + 3 * (int64_t)v, lerp3(P, smooth, it != h ? 0.0f : 1.0f));
}

template <class View>
__global__ void __launch_bounds__(kBlock)
k_vertex_gather_creased(View L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.V) return;
    const int32_t v = (int32_t)i;
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    const int32_t h = L.vert_he(v), prev = L.prev(h);
    const float thisS = L.hsharp(h), prevS = L.hsharp(prev);
    const float cw = fsign(thisS), pcw = fsign(prevS);
    const f3 E = ld3(ept + 3 * (int64_t)L.edge(h));
    const f3 Ep = ld3(ept + 3 * (int64_t)L.edge(prev));
    const f3 Fp = ld3(fpt + 3 * (int64_t)L.face(prev));
    const f3 P = ld3(pin + 3 * (int64_t)v);
    f3 smooth = add3(mul3(Fp, -1.0f), mul3(Ep, 4.0f));
    f3 crease = add3(zero3(), mul3(Ep, pcw));
    float avgS = prevS, creaseCount = pcw, valence = 1.0f;
    int32_t fwd, bwd;
    int guard = 0;
    for (fwd = L.twin(prev); fwd >= 0 && fwd != h && guard < kRingCap; fwd = L.twin(fwd), ++guard) {
        const int32_t p = L.prev(fwd);
        const float s = L.hsharp(p), w = fsign(s);
        const f3 Ei = ld3(ept + 3 * (int64_t)L.edge(p)), Fi = ld3(fpt + 3 * (int64_t)L.face(p));
        smooth = add3(smooth, mul3(Fi, -1.0f));
        smooth = add3(smooth, mul3(Ei, 4.0f));
        valence = fadd(valence, 1.0f);
        crease = add3(crease, mul3(Ei, w));
        avgS = fadd(avgS, s);
        creaseCount = fadd(creaseCount, w);
        fwd = p;
    }
    if (View::kQuad) {   // only the quad-level gather walks back from a boundary (:2424-2451)
        guard = 0;
        for (bwd = L.twin(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kRingCap; bwd = L.twin(bwd), ++guard) {
            const int32_t nn = L.next(bwd);
            const float s = L.hsharp(nn), w = fsign(s);
            const f3 Ei = ld3(ept + 3 * (int64_t)L.edge(nn)), Fi = ld3(fpt + 3 * (int64_t)L.face(nn));
            smooth = add3(smooth, mul3(Fi, -1.0f));
            smooth = add3(smooth, mul3(Ei, 4.0f));
            valence = fadd(valence, 1.0f);
            crease = add3(crease, mul3(Ei, w));
            avgS = fadd(avgS, s);
            creaseCount = fadd(creaseCount, w);
            bwd = nn;
        }
    }
    if (fwd < 0) {
        crease = add3(crease, mul3(E, cw));
        creaseCount = fadd(creaseCount, cw);
        valence = fadd(valence, 1.0f);
    }
    smooth = add3(mul3(smooth, frcp(fmul(valence, valence))), mul3(P, fsub(1.0f, fdiv(3.0f, valence))));
    crease = add3(mul3(crease, View::kQuad ? fdiv(0.5f, creaseCount) : 0.25f), mul3(P, 0.5f));
    f3 o;
    if (creaseCount <= 1.0f) o = smooth;
    else if (creaseCount >= 3.0f || valence == 2.0f) o = P;
    else o = lerp3(P, crease, fsat(fmul(avgS, 0.5f)));
    st3(pout + 3 * (int64_t)v, o);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static CageTables cage_tables(const DevCage& c) { return make_cage_tables(c); }

static CageView cage_view(const Ctx& c) {
    CageView L;
    L.t = cage_tables(*c.cage);
    L.cr = c.cage->cr;
    L.V = c.cage->V; L.F = c.cage->F; L.E = c.cage->E; L.H = c.cage->H; L.C = c.cage->E;
    L.d = 0;
    return L;
}

template <int RW>
static QuadView<RW> quad_view(const Ctx& c, int d) {
    QuadView<RW> L;
    const Level& lv = c.lv[d];
    L.t = cage_tables(*c.cage);
    L.he = c.he + (int64_t)RW * lv.heOff;
    L.cr = c.cr + lv.crOff;
    L.V = lv.V; L.F = lv.F; L.E = lv.E; L.H = lv.H; L.C = lv.C;
    L.d = d;
    return L;
}

template <int RW, bool TOPO, bool UV>
static void launch_topology_level(const Ctx& c, int d) {
    const Level& lv = c.lv[d];
    int32_t* out = c.he + (int64_t)RW * c.lv[d + 1].heOff;
    const int64_t n = 4 * (int64_t)lv.H;
    c.prof->begin(c.stream, TOPO ? CCS_K_TOPOLOGY : CCS_K_UVS, d, lv.H);
    if (d == 0) {
        k_cage_topology<RW, TOPO, UV><<<nblocks(n), kBlock, 0, c.stream>>>(cage_tables(*c.cage), out);
    } else {
        const int32_t* in = c.he + (int64_t)RW * lv.heOff;
        k_quad_topology<RW, TOPO, UV><<<nblocks(n), kBlock, 0, c.stream>>>(in, out, lv.H, lv.V, lv.F, lv.E);
    }
    c.prof->end(c.stream);
}

cudaError_t run_topology(const Ctx& c, bool topo, bool uv) {
    for (int d = 0; d < c.D; ++d) {
        if (c.rw == 4) {
            if (topo && uv) launch_topology_level<4, true, true>(c, d);
            else if (topo) launch_topology_level<4, true, false>(c, d);
            else if (uv) launch_topology_level<4, false, true>(c, d);
        } else if (topo) {
            launch_topology_level<3, true, false>(c, d);
        }
    }
    return cudaGetLastError();
}

cudaError_t run_creases(const Ctx& c) {
    for (int d = 0; d < c.D; ++d) {
        const cc_Crease* in = d == 0 ? c.cage->cr : c.cr + c.lv[d].crOff;
        cc_Crease* out = c.cr + c.lv[d + 1].crOff;
        const int32_t C = c.lv[d].C;
        c.prof->begin(c.stream, CCS_K_CREASES, d, C);
        k_creases<<<nblocks(C), kBlock, 0, c.stream>>>(in, out, C);
        c.prof->end(c.stream);
    }
    return cudaGetLastError();
}

template <class View>
static void points_level(const Ctx& c, const View& L, const float* pin, float* pout, int mode, bool det) {
    const int d = L.d;
    const bool gather = mode == CCS_POINTS_GATHER || mode == CCS_POINTS_NOCREASES_GATHER;
    const bool creased = mode == CCS_POINTS_SCATTER || mode == CCS_POINTS_GATHER;
    c.prof->begin(c.stream, CCS_K_FACE_POINTS, d, L.H);
    if (gather) k_face_points<View, true><<<nblocks(L.F), kBlock, 0, c.stream>>>(L, pin, pout);
    else k_face_points<View, false><<<nblocks(L.F), kBlock, 0, c.stream>>>(L, pin, pout);
    c.prof->end(c.stream);

    c.prof->begin(c.stream, CCS_K_EDGE_POINTS, d, L.H);
    if (gather) {
        if (creased) k_edge_gather<View, true><<<nblocks(L.E), kBlock, 0, c.stream>>>(L, pin, pout);
        else k_edge_gather<View, false><<<nblocks(L.E), kBlock, 0, c.stream>>>(L, pin, pout);
    } else {
        if (creased) k_edge_owner<View, true><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, pin, pout);
        else k_edge_owner<View, false><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, pin, pout);
    }
    c.prof->end(c.stream);

    if (gather) {
        c.prof->begin(c.stream, CCS_K_VERTEX_POINTS, d, L.H);
        if (creased) k_vertex_gather_creased<View><<<nblocks(L.V), kBlock, 0, c.stream>>>(L, pin, pout);
        else k_vertex_gather_smooth<View><<<nblocks(L.V), kBlock, 0, c.stream>>>(L, pin, pout);
        c.prof->end(c.stream);
    } else if (det) {
        c.prof->begin(c.stream, CCS_K_VERTEX_POINTS, d, L.H);
        if (creased) k_vertex_det<View, true><<<nblocks(L.V), kBlock, 0, c.stream>>>(L, pin, pout);
        else k_vertex_det<View, false><<<nblocks(L.V), kBlock, 0, c.stream>>>(L, pin, pout);
        c.prof->end(c.stream);
    } else {
        c.prof->begin(c.stream, CCS_K_CLEAR, d, L.V);
        cudaMemsetAsync(pout, 0, sizeof(float) * 3 * (size_t)L.V, c.stream);
        c.prof->end(c.stream);
        c.prof->begin(c.stream, CCS_K_VERTEX_POINTS, d, L.H);
        if (creased) k_vertex_atomic<View, true><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, pin, pout);
        else k_vertex_atomic<View, false><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, pin, pout);
        c.prof->end(c.stream);
    }
}

// The cage step of the fused pipeline: topology (+UV) and creases of depth 1
// on `topoStream` (the points do not read them), and the cage's face, edge
// and vertex points on the subd's stream -- for the atomic scatter, face
// points and the cleared vertex slots in one launch.
cudaError_t run_cage_step(const Ctx& c, bool topo, bool uv, const float* cagePts, float* pout, int mode, bool det,
                          cudaStream_t topoStream) {
    if (topo) {
        Ctx ct = c;
        ct.stream = topoStream ? topoStream : c.stream;
        if (c.rw == 4) {
            if (uv) launch_topology_level<4, true, true>(ct, 0);
            else launch_topology_level<4, true, false>(ct, 0);
        } else {
            launch_topology_level<3, true, false>(ct, 0);
        }
        const int32_t C = c.lv[0].C;
        c.prof->begin(ct.stream, CCS_K_CREASES, 0, C);
        k_creases<<<nblocks(C), kBlock, 0, ct.stream>>>(c.cage->cr, c.cr + c.lv[1].crOff, C);
        c.prof->end(ct.stream);
    }
    const bool atomic = !det && (mode == CCS_POINTS_SCATTER || mode == CCS_POINTS_NOCREASES_SCATTER);
    if (!atomic) {
        points_level(c, cage_view(c), cagePts, pout, mode, det);
        return cudaGetLastError();
    }
    const bool creased = mode == CCS_POINTS_SCATTER;
    if (c.maps) {
        // every point of depth 1 as one sparse product of the cage points
        const CageMap& m = creased ? c.maps->creased : c.maps->smooth;
        c.prof->begin(c.stream, CCS_K_CAGE_MAP, 0, m.rows);
        const cudaError_t e = launch_cage_map(m, cagePts, pout, c.stream);
        c.prof->end(c.stream);
        return e;
    }
    const CageView L = cage_view(c);
    c.prof->begin(c.stream, CCS_K_FACE_POINTS, 0, L.H);
    k_face_points_clear<CageView><<<nblocks(L.F > L.V ? L.F : L.V), kBlock, 0, c.stream>>>(L, cagePts, pout);
    c.prof->end(c.stream);
    c.prof->begin(c.stream, CCS_K_EDGE_POINTS, 0, L.H);
    if (creased) k_edge_owner<CageView, true><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, cagePts, pout);
    else k_edge_owner<CageView, false><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, cagePts, pout);
    c.prof->end(c.stream);
    c.prof->begin(c.stream, CCS_K_VERTEX_POINTS, 0, L.H);
    if (creased) k_vertex_atomic<CageView, true><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, cagePts, pout);
    else k_vertex_atomic<CageView, false><<<nblocks(L.H), kBlock, 0, c.stream>>>(L, cagePts, pout);
    c.prof->end(c.stream);
    return cudaGetLastError();
}

// Vertex pass of quad level d, summed per vertex in increasing halfedge order.
cudaError_t run_vertex_det_level(const Ctx& c, int d, const float* pin, float* pout, bool creased) {
    c.prof->begin(c.stream, CCS_K_VERTEX_POINTS, d, c.lv[d].H);
    const unsigned nb = nblocks(c.lv[d].V);
    if (c.rw == 4) {
        const QuadView<4> L = quad_view<4>(c, d);
        if (creased) k_vertex_det<QuadView<4>, true><<<nb, kBlock, 0, c.stream>>>(L, pin, pout);
        else k_vertex_det<QuadView<4>, false><<<nb, kBlock, 0, c.stream>>>(L, pin, pout);
    } else {
        const QuadView<3> L = quad_view<3>(c, d);
        if (creased) k_vertex_det<QuadView<3>, true><<<nb, kBlock, 0, c.stream>>>(L, pin, pout);
        else k_vertex_det<QuadView<3>, false><<<nb, kBlock, 0, c.stream>>>(L, pin, pout);
    }
    c.prof->end(c.stream);
    return cudaGetLastError();
}

cudaError_t run_points(const Ctx& c, const float* cagePts, float* pts, int mode, bool det) {
    for (int d = 0; d < c.D; ++d) {
        float* pout = pts + 3 * c.lv[d + 1].ptOff;
        if (d == 0) {
            points_level(c, cage_view(c), cagePts, pout, mode, det);
        } else {
            const float* pin = pts + 3 * c.lv[d].ptOff;
            if (c.rw == 4) points_level(c, quad_view<4>(c, d), pin, pout, mode, det);
            else points_level(c, quad_view<3>(c, d), pin, pout, mode, det);
        }
    }
    return cudaGetLastError();
}

}  // namespace ccs
