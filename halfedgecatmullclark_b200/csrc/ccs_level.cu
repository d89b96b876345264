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
//      - clears the vertex slots the atomics of kernel B accumulate into;
//      - extra blocks refine the creases of the level.
//   B  (one thread per halfedge)
//      - vertex point share of its halfedge: face and edge points come from
//        kernel A's output, the ring statistics from the known structure of
//        refined levels (face centres and edge midpoints need no walk);
//      - shares of the same vertex are summed inside the warp where the
//        structure puts them together (a face centre's 4 shares: plain
//        store, no atomic; an edge midpoint's 2 shares per side: one atomic
//        triple), other shares go to memory with one float atomic triple.
//
// Both kernels evaluate every float expression in the reference's order, so
// topology, creases, UVs, face and edge points are bit-identical to the
// reference; vertex points differ only by the order of the atomic sums.
//
// Twin relation used by A: for a twin pair (h, t), vertex(t) = vertex(next h)
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
__device__ __forceinline__ f3 shfl_xor3(f3 v, int m) {
    return f3{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m),
              __shfl_xor_sync(0xffffffffu, v.z, m)};
}

// Face point of the quad held by lanes qb..qb+3, in halfedge order:
// ((0 + p0/4) + p1/4) + p2/4) + p3/4   (CatmullClark.h:2032-2052)
__device__ __forceinline__ f3 quad_face_point(f3 p, int qb) {
    f3 acc = zero3();
#pragma unroll
    for (int i = 0; i < 4; ++i) acc = add3(acc, quarter3(shfl3(p, qb + i)));
    return acc;
}

// One halfedge's share of its edge point: v0 = its vertex, v1 = the next
// vertex, F = its face point (creased rule :2194-2241, plain rule :2107-2139).
template <bool CREASED>
__device__ __forceinline__ f3 edge_share(f3 v0, f3 v1, f3 F, bool boundary, float w) {
    if (CREASED) {
        const f3 sharpP = mul3(lerp3(v0, v1, 0.5f), boundary ? 1.0f : 0.5f);
        const f3 smoothP = mul3(lerp3(v0, F, 0.5f), 0.5f);
        return lerp3(smoothP, sharpP, w);
    }
    const float wh = boundary ? 1.0f : 0.5f;
    return lerp3(mul3(F, 0.5f), lerp3(mul3(v0, wh), mul3(v1, wh), 0.5f), wh);
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
template <int RW, bool TOPO, bool UV, bool PTS, bool CREASED>
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
        const f3 pn = shfl3(p, ln);
        if (valid && k == 0) st3(a.pout + 3 * ((int64_t)a.V + f), Fp);
        if (a.zeroV && h64 < a.V) st3(a.pout + 3 * h64, zero3());
        // edge point, by the pair's larger halfedge; the smaller one's share
        // is added first, as a one-thread reference run adds it
        if (valid && h > tw) {
            const float w = CREASED ? fsat(ed < a.C ? a.crIn[ed].sharpness : 0.0f) : 0.0f;
            const f3 sh_h = edge_share<CREASED>(p, pn, Fp, tw < 0, w);
            f3 E;
            if (tw >= 0) {
                const int32_t tb = tw & ~3;
                f3 Ft = zero3();
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int32_t tv = __ldg(a.in + (int64_t)RW * (tb + i) + 2);
                    Ft = add3(Ft, quarter3(ld3(a.pin + 3 * (int64_t)tv)));
                }
                const f3 sh_t = edge_share<CREASED>(pn, p, Ft, false, w);
                E = add3(add3(zero3(), sh_t), sh_h);
            } else {
                E = add3(zero3(), sh_h);
            }
            st3(a.pout + 3 * ((int64_t)a.V + a.F + ed), E);
        }
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
__device__ __forceinline__ void atomic_add3(float* o, f3 v) {
    atomicAdd(o + 0, v.x);
    atomicAdd(o + 1, v.y);
    atomicAdd(o + 2, v.z);
}

// STRUCT: depth >= 2, where a 16-lane group holds the 16 children of one
// parent quad face, so a face centre's 4 shares sit in lanes 2, 6, 10, 14 and
// an edge midpoint's shares from this face in lanes 4j+1 and 4(j+1 mod 4)+3.
template <int RW, bool CREASED, bool STRUCT>
__global__ void __launch_bounds__(kBlockL)
k_level_b(QuadView<RW> L, const float* __restrict__ pin, float* __restrict__ pout) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = (int64_t)blockIdx.x * kBlockL + tid;
    const bool valid = h64 < L.H;
    const int32_t h = (int32_t)h64;
    const int k = lane & 3, qb = lane & ~3, lp = qb | ((k + 3) & 3);
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
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
    f3 p = zero3(), Fh = zero3(), Eh = zero3();
    if (valid) {
        p = ld3(pin + 3 * (int64_t)vx);
        Fh = ld3(fpt + 3 * (int64_t)(h >> 2));
        Eh = ld3(ept + 3 * (int64_t)ed);
    }
    const f3 Ep = shfl3(Eh, lp);                         // edge point of prev(h)
    const int32_t ped = __shfl_sync(0xffffffffu, ed, lp);
    const int32_t ptw = __shfl_sync(0xffffffffu, tw, lp);
    f3 s = zero3();
    if (valid) {
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
        } else if (k != 0) {
            const int32_t eh = k == 1 ? ped : ed;        // one half of the parent edge
            const float sa = L.sharp(eh), sb = L.sharp(eh ^ 1);
            bnd = (k == 1 ? ptw : tw) < 0;
            vpre = bnd ? 2.0f : 4.0f;
            const bool own = k == 3;                     // the walk from h skips its own edge
            avgS = (bnd && own) ? sb : fadd(sa, sb);
            cpre = (bnd && own) ? fsign(sb) : fadd(fsign(sa), fsign(sb));
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
            // vertex rule, corner-first branch order of quad levels (:2567-2607)
            const float cw = fsign(L.sharp(ed)), pcw = fsign(L.sharp(ped));
            const float valence = bnd ? fadd(vpre, 1.0f) : vpre;
            const float creaseCount = bnd ? fadd(cpre, cw) : cpre;
            if (creaseCount >= 3.0f || valence == 2.0f) {
                s = mul3(p, frcp(vpre));
            } else if (creaseCount <= 1.0f) {
                f3 smooth = add3(mul3(Fh, -1.0f), mul3(Eh, 4.0f));
                smooth = add3(smooth, mul3(p, fsub(vpre, 3.0f)));
                s = mul3(smooth, frcp(fmul(vpre, vpre)));
            } else {
                const f3 corner = mul3(p, frcp(vpre));
                f3 crease = add3(mul3(p, fmul(0.25f, cw)), mul3(Eh, fmul(0.25f, cw)));
                if (bnd) crease = add3(crease, add3(mul3(p, fmul(0.25f, pcw)), mul3(Ep, fmul(0.25f, pcw))));
                s = lerp3(corner, crease, fsat(fmul(avgS, 0.5f)));
            }
        } else {
            // crease-free vertex rule (:2307-2351)
            const float w = frcp(vpre);
            const float ws = fmul(w, bnd ? 0.0f : 1.0f);
            s.x = fmul(w, fadd(p.x, fmul(ws, fsub(fsub(fmul(4.0f, Eh.x), Fh.x), fmul(3.0f, p.x)))));
            s.y = fmul(w, fadd(p.y, fmul(ws, fsub(fsub(fmul(4.0f, Eh.y), Fh.y), fmul(3.0f, p.y)))));
            s.z = fmul(w, fadd(p.z, fmul(ws, fsub(fsub(fmul(4.0f, Eh.z), Fh.z), fmul(3.0f, p.z)))));
        }
    }
    float* o = pout + 3 * (int64_t)vx;
    if (STRUCT) {
        const f3 u = add3(s, shfl_xor3(s, 4));
        const f3 fsum = add3(u, shfl_xor3(u, 8));       // (s2 + s6) + (s10 + s14)
        const int partner = (lane & ~15) | ((((lane >> 2) + 1) & 3) << 2) | 3;
        const f3 pe = shfl3(s, partner);
        if (valid) {
            if (k == 2) {
                if ((lane & 15) == 2) st3(o, fsum);     // all 4 shares of this vertex
            } else if (k == 1) {
                atomic_add3(o, add3(s, pe));
            } else if (k == 0) {
                atomic_add3(o, s);
            }
        }
    } else if (valid) {
        atomic_add3(o, s);
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

template <int RW, bool CREASED>
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
    c.prof->begin(c.stream, CCS_K_LEVEL_POINTS, d, L.H);
    const unsigned nb = nblocksL(L.H);
    if (d >= 2) k_level_b<RW, CREASED, true><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    else k_level_b<RW, CREASED, false><<<nb, kBlockL, 0, c.stream>>>(L, pin, pout);
    c.prof->end(c.stream);
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
        level_a<RW, CREASED>(c, d, topo, uv, pin, pout, !det);
        if (det) {
            const cudaError_t e = run_vertex_det_level(c, d, pin, pout, CREASED);
            if (e != cudaSuccess) return e;
        } else {
            level_b<RW, CREASED>(c, d, pin, pout);
        }
    }
    return cudaGetLastError();
}

cudaError_t run_fused(const Ctx& c, bool topo, const float* cagePts, float* pts, int mode, bool det) {
    const bool creased = mode == CCS_POINTS_SCATTER;
    const bool uv = c.cage->U > 0 && c.rw == 4;
    cudaError_t e = run_cage_step(c, topo, uv, cagePts, pts + 3 * c.lv[1].ptOff, mode, det);
    if (e != cudaSuccess) return e;
    if (c.rw == 4) return creased ? fused_levels<4, true>(c, topo, uv, pts, det) : fused_levels<4, false>(c, topo, uv, pts, det);
    return creased ? fused_levels<3, true>(c, topo, false, pts, det) : fused_levels<3, false>(c, topo, false, pts, det);
}

}  // namespace ccs
