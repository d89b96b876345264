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
//      - clears the vertex slots the atomics of kernel B accumulate into;
//      - extra blocks refine the creases of the level.
//   B  (one thread per halfedge)
//      - edge point: both halves of the edge rule (its own face point is
//        rebuilt from the quad's lanes, the twin face's point is read from
//        kernel A's output); the pair's larger halfedge stores it;
//      - vertex point share (ring walk for valence / crease statistics),
//        summed across lanes of the warp that hit the same vertex, one float
//        atomic per vertex and warp.
//
// Both kernels evaluate every float expression in the reference's order, so
// topology, creases, UVs, face and edge points are bit-identical to the
// reference; vertex points differ only by the order of the atomic sums.
//
// Twin relation used by B: for a twin pair (h, t), vertex(t) = vertex(next h)
// and vertex(next t) = vertex(h).  The C ABI checks this on the cage (it is
// then preserved by every refinement step) and uses the unfused kernels for
// cages that break it.
#include <cstdint>

#include "ccs_host.h"
#include "ccs_internal.cuh"

namespace ccs {

static constexpr int kBlockL = 256;

static inline unsigned nblocksL(int64_t n) { return (unsigned)((n + kBlockL - 1) / kBlockL); }

// Exact x / 65535 for an integer x in [0, 65535]: reciprocal product plus one
// FMA correction (checked exhaustively against IEEE division).
__device__ __forceinline__ float uv_dec_fast(uint32_t x) {
    const float a = (float)(x & 0xFFFFu);
    const float inv = 0x1.0001p-16f;
    const float q = __fmul_rn(a, inv);
    const float r = __fmaf_rn(-q, 65535.0f, a);
    return __fmaf_rn(r, inv, q);
}
// float -> uint32 as the reference's x86-64 build converts (see uv_enc)
__device__ __forceinline__ uint32_t f2u32_fast(float x) {
    if (x >= -2147483648.0f && x < 2147483648.0f) return (uint32_t)__float2int_rz(x);
    return f2u32_trunc(x);
}
__device__ __forceinline__ int32_t uv_enc_fast(float u, float v) {
    const uint32_t a = f2u32_fast(fmul(u, 65535.0f));
    const uint32_t b = f2u32_fast(fmul(v, 65535.0f));
    return (int32_t)((a & 0xFFFFu) | ((b & 0xFFFFu) << 16));
}

__device__ __forceinline__ void bulk_store_tile(void* gdst, const void* ssrc, uint32_t bytes) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(gdst), "r"(s), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__device__ __forceinline__ f3 shfl3(f3 v, int src) {
    return f3{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
              __shfl_sync(0xffffffffu, v.z, src)};
}

// Face point of the quad held by lanes qb..qb+3, in halfedge order:
// ((0 + p0/4) + p1/4) + p2/4) + p3/4   (CatmullClark.h:2032-2052)
__device__ __forceinline__ f3 quad_face_point(f3 p, int qb) {
    f3 acc = zero3();
#pragma unroll
    for (int i = 0; i < 4; ++i) acc = add3(acc, quarter3(shfl3(p, qb + i)));
    return acc;
}

struct LevelArgs {
    const int32_t* __restrict__ in;     // depth-d records (RW words)
    int32_t* __restrict__ out;          // depth-(d+1) records
    const cc_Crease* __restrict__ crIn; // depth-d creases
    cc_Crease* __restrict__ crOut;      // depth-(d+1) creases
    const float* __restrict__ pin;      // depth-d points
    float* __restrict__ pout;           // depth-(d+1) points
    int32_t H, V, F, E, C;              // depth-d counts
    int zeroV;                          // clear the old-vertex slots (atomic path)
};

// ---------------------------------------------------------------------------
// kernel A
// ---------------------------------------------------------------------------
template <int RW, bool TOPO, bool UV, bool PTS>
__global__ void __launch_bounds__(kBlockL)
k_level_a(LevelArgs a) {
    const int nbH = (a.H + kBlockL - 1) / kBlockL;
    if ((int)blockIdx.x >= nbH) {
        // crease refinement (CatmullClark.h:2992-3026)
        if (!TOPO) return;
        const int64_t i = (int64_t)(blockIdx.x - nbH) * kBlockL + threadIdx.x;
        if (i >= a.C) return;
        const int32_t e = (int32_t)i;
        const cc_Crease me = a.crIn[e];
        const int32_t nx = me.nextID, pv = me.prevID;
        const cc_Crease cn = a.crIn[nx], cp = a.crIn[pv];
        const bool t1 = cn.prevID == e && nx != e;
        const bool t2 = cp.nextID == e && pv != e;
        const float thisS = fmul(3.0f, me.sharpness);
        cc_Crease x, y;
        x.nextID = 2 * e + 1;
        y.nextID = 2 * nx + (t1 ? 0 : 1);
        x.prevID = 2 * pv + (t2 ? 1 : 0);
        y.prevID = 2 * e + 0;
        x.sharpness = fmax_ref(0.0f, fsub(fquarter(fadd(cp.sharpness, thisS)), 1.0f));
        y.sharpness = fmax_ref(0.0f, fsub(fquarter(fadd(thisS, cn.sharpness)), 1.0f));
        a.crOut[2 * i + 0] = x;
        a.crOut[2 * i + 1] = y;
        return;
    }
    __shared__ __align__(128) int32_t tile[kBlockL * 4 * RW];
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = (int64_t)blockIdx.x * kBlockL + tid;
    const bool valid = h64 < a.H;
    const int32_t h = (int32_t)h64;
    const int k = lane & 3, qb = lane & ~3;
    int32_t tw = 0, ed = 0, vx = 0, uv = 0;
    if (valid) {
        if constexpr (RW == 4) {
            const int4 r = __ldg(reinterpret_cast<const int4*>(a.in) + h);
            tw = r.x; ed = r.y; vx = r.z; uv = r.w;
        } else {
            tw = __ldg(a.in + 3 * h64 + 0);
            ed = __ldg(a.in + 3 * h64 + 1);
            vx = __ldg(a.in + 3 * h64 + 2);
        }
    }
    const int ln = qb | ((k + 1) & 3), lp = qb | ((k + 3) & 3), lo = qb | ((k + 2) & 3);
    const int32_t prev = (h & ~3) | ((k + 3) & 3), next = (h & ~3) | ((k + 1) & 3), f = h >> 2;
    if (TOPO) {
        const int32_t ptw = __shfl_sync(0xffffffffu, tw, lp);
        const int32_t ped = __shfl_sync(0xffffffffu, ed, lp);
        int32_t uvc[4] = {uv, 0, 0, 0};
        if (UV) {
            const float u = uv_dec_fast((uint32_t)uv), v = uv_dec_fast((uint32_t)uv >> 16);
            const float un = __shfl_sync(0xffffffffu, u, ln), vn = __shfl_sync(0xffffffffu, v, ln);
            const float uo = __shfl_sync(0xffffffffu, u, lo), vo = __shfl_sync(0xffffffffu, v, lo);
            const float up = __shfl_sync(0xffffffffu, u, lp), vp = __shfl_sync(0xffffffffu, v, lp);
            uvc[1] = uv_enc_fast(flerp(u, un, 0.5f), flerp(v, vn, 0.5f));
            uvc[2] = uv_enc_fast(fquarter(fadd(fadd(fadd(u, un), uo), up)),
                                 fquarter(fadd(fadd(fadd(v, vn), vo), vp)));
            uvc[3] = uv_enc_fast(flerp(u, up, 0.5f), flerp(v, vp, 0.5f));
        }
        int32_t* t = tile + tid * 4 * RW;
        const int32_t c_tw[4] = {child(qnext(tw), 3), child(next, 2), child(prev, 1), child(ptw, 0)};
        const int32_t c_ed[4] = {2 * ed + (h > tw ? 0 : 1), 2 * a.E + h, 2 * a.E + prev,
                                 2 * ped + (prev > ptw ? 1 : 0)};
        const int32_t c_vx[4] = {vx, a.V + a.F + ed, a.V + f, a.V + a.F + ped};
        if constexpr (RW == 4) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
                reinterpret_cast<int4*>(t)[m] = make_int4(c_tw[m], c_ed[m], c_vx[m], UV ? uvc[m] : 0);
        } else {
#pragma unroll
            for (int m = 0; m < 4; ++m) { t[3 * m] = c_tw[m]; t[3 * m + 1] = c_ed[m]; t[3 * m + 2] = c_vx[m]; }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (PTS) {
        const f3 p = valid ? ld3(a.pin + 3 * (int64_t)vx) : zero3();
        const f3 Fp = quad_face_point(p, qb);
        if (valid && k == 0) st3(a.pout + 3 * ((int64_t)a.V + f), Fp);
        if (a.zeroV && h64 < a.V) st3(a.pout + 3 * h64, zero3());
    }
    if (TOPO) {
        __syncthreads();
        if (tid == 0) {
            const int64_t h0 = (int64_t)blockIdx.x * kBlockL;
            const int64_t n = (a.H - h0) < kBlockL ? (a.H - h0) : kBlockL;
            bulk_store_tile(a.out + 4 * RW * h0, tile, (uint32_t)(n * 16 * RW));
        }
    }
}

// ---------------------------------------------------------------------------
// kernel B
// ---------------------------------------------------------------------------
template <int RW, bool CREASED, bool VERTEX>
__global__ void __launch_bounds__(kBlockL)
k_level_b(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = (int64_t)blockIdx.x * kBlockL + tid;
    const bool valid = h64 < L.H;
    const int32_t h = (int32_t)h64;
    const int k = lane & 3, qb = lane & ~3;
    const float* fpt = pout + 3 * (int64_t)L.V;
    float* ept = pout + 3 * ((int64_t)L.V + L.F);
    int32_t tw = -1, ed = 0, vx = 0;
    if (valid) {
        if constexpr (RW == 4) {
            const int4 r = __ldg(reinterpret_cast<const int4*>(L.he) + h);
            tw = r.x; ed = r.y; vx = r.z;
        } else {
            tw = __ldg(L.he + 3 * h64 + 0);
            ed = __ldg(L.he + 3 * h64 + 1);
            vx = __ldg(L.he + 3 * h64 + 2);
        }
    }
    const f3 p = valid ? ld3(pin + 3 * (int64_t)vx) : zero3();
    const f3 Fh = quad_face_point(p, qb);
    const f3 pn = shfl3(p, qb | ((k + 1) & 3));
    // ---- edge point ---------------------------------------------------------
    f3 Eh = zero3();
    if (valid) {
        f3 sh_h, sh_t = zero3();
        if (CREASED) {
            const float w = fsat(L.sharp(ed));
            const f3 sharpP = mul3(lerp3(p, pn, 0.5f), tw < 0 ? 1.0f : 0.5f);
            const f3 smoothP = mul3(lerp3(p, Fh, 0.5f), 0.5f);
            sh_h = lerp3(smoothP, sharpP, w);
            if (tw >= 0) {
                const f3 Ft = ld3(fpt + 3 * (int64_t)(tw >> 2));
                const f3 sharpT = mul3(lerp3(pn, p, 0.5f), 0.5f);
                const f3 smoothT = mul3(lerp3(pn, Ft, 0.5f), 0.5f);
                sh_t = lerp3(smoothT, sharpT, w);
            }
        } else {
            const float wh = tw >= 0 ? 0.5f : 1.0f;
            sh_h = lerp3(mul3(Fh, 0.5f), lerp3(mul3(p, wh), mul3(pn, wh), 0.5f), wh);
            if (tw >= 0) {
                const f3 Ft = ld3(fpt + 3 * (int64_t)(tw >> 2));
                sh_t = lerp3(mul3(Ft, 0.5f), lerp3(mul3(pn, 0.5f), mul3(p, 0.5f), 0.5f), 0.5f);
            }
        }
        if (tw < 0) Eh = add3(zero3(), sh_h);
        else if (h > tw) Eh = add3(add3(zero3(), sh_t), sh_h);   // lower halfedge ID first
        else Eh = add3(add3(zero3(), sh_h), sh_t);
        if (h > tw) st3(ept + 3 * (int64_t)ed, Eh);
    }
    if (!VERTEX) return;
    // ---- vertex point share ---------------------------------------------------
    const f3 Ep = shfl3(Eh, qb | ((k + 3) & 3));     // edge point of prev(h)
    const int32_t ped = __shfl_sync(0xffffffffu, ed, qb | ((k + 3) & 3));
    const int32_t ptw = __shfl_sync(0xffffffffu, tw, qb | ((k + 3) & 3));
    int32_t key = -1 - lane;
    f3 s = zero3();
    if (valid) {
        key = vx;
        // Ring statistics of vertex(h) as the reference's walk from h finds
        // them (:2523-2566).  At a refined level the vertex of child k of a
        // parent halfedge is known: k = 2 is a face centre (valence = parent
        // face size, all edges crease-free), k = 1 and 3 are edge midpoints
        // (valence 4, or 2 on a boundary; the creased edges are the two halves
        // e and e^1 of the parent edge), k = 0 is an older vertex that needs
        // the walk.  Sharpness at depth >= 1 is +0 or positive, so sums with
        // the crease-free edges' zeros are exact in any order.
        float vpre, cpre, avgS;
        bool bnd;
        if (k == 2) {
            vpre = L.d == 1 ? (float)L.t.fsz[L.t.he[(int64_t)CH_WORDS * (h >> 2) + CH_FACE]] : 4.0f;
            cpre = 0.0f; avgS = 0.0f; bnd = false;
        } else if (k == 1) {
            const float sa = L.sharp(ped), sb = L.sharp(ped ^ 1);
            bnd = ptw < 0;
            vpre = bnd ? 2.0f : 4.0f;
            avgS = fadd(sa, sb);
            cpre = fadd(fsign(sa), fsign(sb));
        } else if (k == 3) {
            const float sa = L.sharp(ed), sb = L.sharp(ed ^ 1);
            bnd = tw < 0;
            vpre = bnd ? 2.0f : 4.0f;
            avgS = bnd ? sb : fadd(sa, sb);
            cpre = bnd ? fsign(sb) : fadd(fsign(sa), fsign(sb));
        } else if (CREASED) {
            const RingStats r = creased_ring(L, h);
            vpre = r.valence; cpre = r.creaseCount; avgS = r.avgS; bnd = r.fwd < 0;
        } else {
            int32_t valence = 1, fwd, bwd, guard = 0;
            for (fwd = L.prev_vertex_he(h); fwd >= 0 && fwd != h && guard < kWalkCap; fwd = L.prev_vertex_he(fwd), ++guard) ++valence;
            guard = 0;
            for (bwd = L.next_vertex_he(h); fwd < 0 && bwd >= 0 && bwd != h && guard < kWalkCap; bwd = L.next_vertex_he(bwd), ++guard) ++valence;
            vpre = (float)valence; cpre = 0.0f; avgS = 0.0f; bnd = fwd < 0;
        }
        if (CREASED) {
            const float cw = fsign(L.sharp(ed)), pcw = fsign(L.sharp(ped));
            float valence = vpre, creaseCount = cpre;
            const f3 corner = mul3(p, frcp(valence));
            f3 crease = add3(mul3(p, fmul(0.25f, cw)), mul3(Eh, fmul(0.25f, cw)));
            f3 smooth = add3(mul3(Fh, -1.0f), mul3(Eh, 4.0f));
            smooth = add3(smooth, mul3(p, fsub(valence, 3.0f)));
            smooth = mul3(smooth, frcp(fmul(valence, valence)));
            if (bnd) {
                creaseCount = fadd(creaseCount, cw);
                valence = fadd(valence, 1.0f);
                crease = add3(crease, add3(mul3(p, fmul(0.25f, pcw)), mul3(Ep, fmul(0.25f, pcw))));
            }
            if (creaseCount >= 3.0f || valence == 2.0f) s = corner;
            else if (creaseCount <= 1.0f) s = smooth;
            else s = lerp3(corner, crease, fsat(fmul(avgS, 0.5f)));
        } else {
            const float w = frcp(vpre);
            const float ws = fmul(w, bnd ? 0.0f : 1.0f);
            s.x = fmul(w, fadd(p.x, fmul(ws, fsub(fsub(fmul(4.0f, Eh.x), Fh.x), fmul(3.0f, p.x)))));
            s.y = fmul(w, fadd(p.y, fmul(ws, fsub(fsub(fmul(4.0f, Eh.y), Fh.y), fmul(3.0f, p.y)))));
            s.z = fmul(w, fadd(p.z, fmul(ws, fsub(fsub(fmul(4.0f, Eh.z), Fh.z), fmul(3.0f, p.z)))));
        }
    }
    const unsigned full = 0xffffffffu;
    const unsigned grp = __match_any_sync(full, key);
    const int n = __popc(grp);
    const int maxn = (int)__reduce_max_sync(full, (unsigned)n);
    f3 acc = zero3();
    for (int i = 0; i < maxn; ++i) {
        const int src = i < n ? (int)__fns(grp, 0, i + 1) : lane;
        const f3 t = shfl3(s, src);
        if (i < n) acc = add3(acc, t);
    }
    if (valid && lane == __ffs(grp) - 1) {
        float* o = pout + 3 * (int64_t)vx;
        atomicAdd(o + 0, acc.x);
        atomicAdd(o + 1, acc.y);
        atomicAdd(o + 2, acc.z);
    }
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

template <int RW>
static void level_a(const Ctx& c, int d, bool topo, bool uv, const float* pin, float* pout, bool zeroV) {
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
    const unsigned nb = nblocksL(lv.H) + (topo ? nblocksL(lv.C) : 0u);
    c.prof->begin(c.stream, topo ? CCS_K_LEVEL_FUSED : CCS_K_FACE_POINTS, d, lv.H);
    if (topo) {
        if (RW == 4 && uv) k_level_a<RW, true, true, true><<<nb, kBlockL, 0, c.stream>>>(a);
        else k_level_a<RW, true, false, true><<<nb, kBlockL, 0, c.stream>>>(a);
    } else {
        k_level_a<RW, false, false, true><<<nb, kBlockL, 0, c.stream>>>(a);
    }
    c.prof->end(c.stream);
}

template <int RW>
static void level_b(const Ctx& c, int d, bool creased, bool vertex, const float* pin, float* pout) {
    const QuadView<RW> L = quad_view_l<RW>(c, d);
    c.prof->begin(c.stream, vertex ? CCS_K_LEVEL_POINTS : CCS_K_EDGE_POINTS, d, L.H);
    const unsigned nb = nblocksL(L.H);
    if (creased) {
        if (vertex) k_level_b<RW, true, true><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
        else k_level_b<RW, true, false><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    } else {
        if (vertex) k_level_b<RW, false, true><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
        else k_level_b<RW, false, false><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    }
    c.prof->end(c.stream);
}

// Declared in ccs_forward.cu: the vertex pass of one quad level when the
// fixed-order (deterministic) sum is requested.
cudaError_t run_vertex_det_level(const Ctx& c, int d, const float* pin, float* pout, bool creased);
cudaError_t run_cage_step(const Ctx& c, bool topo, bool uv, const float* cagePts, float* pout, int mode, bool det);

cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool det) {
    const bool creased = mode == CCS_POINTS_SCATTER;
    const bool uv = c.cage->U > 0 && c.rw == 4;
    cudaError_t e = run_cage_step(c, topo, uv, cagePts, pts + 3 * c.lv[1].ptOff, mode, det);
    if (e != cudaSuccess) return e;
    for (int d = 1; d < c.D; ++d) {
        const float* pin = pts + 3 * c.lv[d].ptOff;
        float* pout = pts + 3 * c.lv[d + 1].ptOff;
        if (c.rw == 4) {
            level_a<4>(c, d, topo, uv, pin, pout, !det);
            level_b<4>(c, d, creased, !det, pin, pout);
        } else {
            level_a<3>(c, d, topo, false, pin, pout, !det);
            level_b<3>(c, d, creased, !det, pin, pout);
        }
        if (det) {
            e = run_vertex_det_level(c, d, pin, pout, creased);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaGetLastError();
}

}  // namespace ccs
