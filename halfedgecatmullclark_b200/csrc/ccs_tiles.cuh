// ccs_tiles.cuh -- per-tile / per-item bodies of the refinement kernels.
//
// The single-mesh kernels (ccs_forward.cu, ccs_level.cu, ccs_adjoint.cu)
// and the persistent batched kernels (ccs_batch.cu) run these same device
// functions; a kernel only decides which tile or item a block or thread
// takes.  See ccs_level.cu for the design of the two quad-level kernels.
#pragma once

#include <cstdint>

#include "ccs_internal.cuh"

namespace ccs {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
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

// One thread writes `bytes` of shared memory to global memory through the
// TMA engine (no multicast) and waits until the shared source has been read.
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
__device__ __forceinline__ void atomic_add3(float* o, f3 v) {
    atomicAdd(o + 0, v.x);
    atomicAdd(o + 1, v.y);
    atomicAdd(o + 2, v.z);
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

// ---------------------------------------------------------------------------
// creases (CatmullClark.h:2950-2983, :2992-3026): item = parent crease
// ---------------------------------------------------------------------------
__device__ __forceinline__ void crease_item(const cc_Crease* __restrict__ in, cc_Crease* __restrict__ out,
                                            int32_t e) {
    const cc_Crease me = in[e];
    const int32_t nx = me.nextID, pv = me.prevID;
    const cc_Crease cn = in[nx], cp = in[pv];
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
    out[2 * (int64_t)e + 0] = x;
    out[2 * (int64_t)e + 1] = y;
}

// ---------------------------------------------------------------------------
// quad level, kernel A body: one tile of BLOCK parent halfedges [h0, h0+BLOCK)
// ---------------------------------------------------------------------------
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

// `tile` is BLOCK * 4 * RW ints of shared memory; every thread of the block
// must call this with the same h0.
template <int BLOCK, int RW, bool TOPO, bool UV, bool PTS, bool CREASED>
__device__ __forceinline__ void tile_level_a(const LevelArgs& a, int64_t h0, int32_t* tile) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = h0 + tid;
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
            const int64_t n = (a.H - h0) < BLOCK ? (a.H - h0) : BLOCK;
            bulk_store_tile(a.out + 4 * RW * h0, tile, (uint32_t)(n * 16 * RW));
        }
    }
}

// ---------------------------------------------------------------------------
// quad level, kernel B body: vertex shares of halfedges [h0, h0 + blockDim)
// ---------------------------------------------------------------------------
// STRUCT: depth >= 2, where a 16-lane group holds the 16 children of one
// parent quad face, so a face centre's 4 shares sit in lanes 2, 6, 10, 14 and
// an edge midpoint's shares from this face in lanes 4j+1 and 4(j+1 mod 4)+3.
template <int RW, bool CREASED, bool STRUCT>
__device__ __forceinline__ void tile_level_b(const QuadView<RW>& L, const float* __restrict__ pin,
                                             float* __restrict__ pout, int64_t h0) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = h0 + tid;
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
// cage level items (n-gon faces; CatmullClark.h:1437-1463, :1602-1648,
// :1872-1991, :2693-2740, :2825-2869)
// ---------------------------------------------------------------------------
// item = child halfedge c (4 per cage halfedge)
template <int RW, bool TOPO, bool UV>
__device__ __forceinline__ void cage_topology_item(const CageTables& t, int32_t* __restrict__ out, int64_t c) {
    const int32_t h = (int32_t)(c >> 2), m = (int32_t)(c & 3);
    const int32_t* r = t.he + (int64_t)CH_WORDS * h;
    const int32_t twin = r[CH_TWIN], next = r[CH_NEXT], prev = r[CH_PREV];
    const int32_t* rp = t.he + (int64_t)CH_WORDS * prev;
    int32_t o_tw = 0, o_ed = 0, o_vx = 0, o_uv = 0;
    if (TOPO) {
        const int32_t V = t.n.V, F = t.n.F, E = t.n.E;
        switch (m) {
            case 0: {
                const int32_t twinNext = twin >= 0 ? t.he[(int64_t)CH_WORDS * twin + CH_NEXT] : -1;
                o_tw = child(twinNext, 3); o_ed = 2 * r[CH_EDGE] + (h > twin ? 0 : 1); o_vx = r[CH_VERT];
                break;
            }
            case 1: o_tw = child(next, 2); o_ed = 2 * E + h; o_vx = V + F + r[CH_EDGE]; break;
            case 2: o_tw = child(prev, 1); o_ed = 2 * E + prev; o_vx = V + r[CH_FACE]; break;
            default: {
                const int32_t pt = rp[CH_TWIN], pe = rp[CH_EDGE];
                o_tw = child(pt, 0); o_ed = 2 * pe + (prev > pt ? 1 : 0); o_vx = V + F + pe;
                break;
            }
        }
    }
    if (UV) {
        const float* uvh = t.uvs + 2 * (int64_t)r[CH_UV];
        const float u = uvh[0], v = uvh[1];
        switch (m) {
            case 0: o_uv = uv_enc(u, v); break;
            case 1: {
                const float* q = t.uvs + 2 * (int64_t)t.he[(int64_t)CH_WORDS * next + CH_UV];
                o_uv = uv_enc(flerp(u, q[0], 0.5f), flerp(v, q[1], 0.5f));
                break;
            }
            case 2: {
                float fu = u, fv = v;
                int32_t n = 1, guard = 0;
                for (int32_t it = next; it != h && guard < kWalkCap; it = t.he[(int64_t)CH_WORDS * it + CH_NEXT], ++guard) {
                    const float* q = t.uvs + 2 * (int64_t)t.he[(int64_t)CH_WORDS * it + CH_UV];
                    fu = fadd(fu, q[0]);
                    fv = fadd(fv, q[1]);
                    ++n;
                }
                o_uv = uv_enc(fdiv(fu, (float)n), fdiv(fv, (float)n));
                break;
            }
            default: {
                const float* q = t.uvs + 2 * (int64_t)rp[CH_UV];
                o_uv = uv_enc(flerp(u, q[0], 0.5f), flerp(v, q[1], 0.5f));
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

// item = face f.  GATHER_SEM: sum then scale (gather routines); otherwise
// each vertex adds p / n in halfedge order (scatter routines).
template <class View, bool GATHER_SEM>
__device__ __forceinline__ void face_point_item(const View& L, const float* __restrict__ pin,
                                                float* __restrict__ pout, int32_t f) {
    float* fp = pout + 3 * ((int64_t)L.V + f);
    if constexpr (View::kQuad) {
        f3 p[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) p[k] = ld3(pin + 3 * (int64_t)L.vert(4 * f + k));
        if (GATHER_SEM) {
            f3 acc = add3(add3(add3(p[0], p[1]), p[2]), p[3]);
            st3(fp, mul3(acc, 0.25f));
        } else {
            f3 acc = zero3();
#pragma unroll
            for (int k = 0; k < 4; ++k) acc = add3(acc, quarter3(p[k]));
            st3(fp, acc);
        }
    } else {
        const int32_t h0 = L.face_he(f);
        float n = 1.0f;
        int guard = 0;
        for (int32_t it = L.next(h0); it != h0 && guard < kWalkCap; it = L.next(it), ++guard) n = fadd(n, 1.0f);
        if (GATHER_SEM) {
            f3 acc = ld3(pin + 3 * (int64_t)L.vert(h0));
            guard = 0;
            for (int32_t it = L.next(h0); it != h0 && guard < kWalkCap; it = L.next(it), ++guard)
                acc = add3(acc, ld3(pin + 3 * (int64_t)L.vert(it)));
            st3(fp, mul3(acc, frcp(n)));
        } else {
            f3 acc = add3(zero3(), div3(ld3(pin + 3 * (int64_t)L.vert(h0)), n));
            guard = 0;
            for (int32_t it = L.next(h0); it != h0 && guard < kWalkCap; it = L.next(it), ++guard)
                acc = add3(acc, div3(ld3(pin + 3 * (int64_t)L.vert(it)), n));
            st3(fp, acc);
        }
    }
}

template <class View, bool CREASED>
__device__ __forceinline__ f3 edge_share_of(const View& L, int32_t h, const float* pin, const float* fpt) {
    if (CREASED) return creased_edge_share(L, h, pin, fpt);
    return smooth_edge_share(L, h, pin, fpt);
}

// item = halfedge h; the pair's larger halfedge stores the edge point
template <class View, bool CREASED>
__device__ __forceinline__ void edge_owner_item(const View& L, const float* __restrict__ pin,
                                                float* __restrict__ pout, int32_t h) {
    const int32_t tw = L.twin(h);
    if (!(h > tw)) return;   // the pair's smaller halfedge defers to its twin
    const float* fpt = pout + 3 * (int64_t)L.V;
    float* ept = pout + 3 * ((int64_t)L.V + L.F);
    f3 acc = add3(zero3(), edge_share_of<View, CREASED>(L, tw >= 0 ? tw : h, pin, fpt));
    if (tw >= 0) acc = add3(acc, edge_share_of<View, CREASED>(L, h, pin, fpt));
    st3(ept + 3 * (int64_t)L.edge(h), acc);
}

template <class View, bool CREASED>
__device__ __forceinline__ f3 vertex_share_of(const View& L, int32_t h, const float* pin, const float* fpt,
                                              const float* ept) {
    if (CREASED) return creased_vertex_share(L, h, pin, fpt, ept);
    return smooth_vertex_share(L, h, pin, fpt, ept);
}

// item = halfedge h; warp-collective (every lane of the warp must call it),
// lanes with valid == false contribute nothing
template <class View, bool CREASED>
__device__ __forceinline__ void vertex_atomic_item(const View& L, const float* __restrict__ pin,
                                                   float* __restrict__ pout, int32_t h, bool valid) {
    const int lane = threadIdx.x & 31;
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    int32_t v = -1 - lane;           // distinct keys for lanes without work
    f3 s = zero3();
    if (valid) {
        v = L.vert(h);
        s = vertex_share_of<View, CREASED>(L, h, pin, fpt, ept);
    }
    const unsigned full = 0xffffffffu;
    const unsigned grp = __match_any_sync(full, v);
    const int n = __popc(grp);
    const int maxn = (int)__reduce_max_sync(full, (unsigned)n);
    f3 acc = zero3();
    for (int k = 0; k < maxn; ++k) {
        const int src = k < n ? (int)__fns(grp, 0, k + 1) : lane;
        const f3 t = shfl3(s, src);
        if (k < n) acc = add3(acc, t);
    }
    if (valid && lane == __ffs(grp) - 1) atomic_add3(pout + 3 * (int64_t)v, acc);
}

// ---------------------------------------------------------------------------
// adjoint of the creased scatter rule (see ccs_adjoint.cu): three gathers
// ---------------------------------------------------------------------------
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
    for (int32_t it = L.next(h); it != h && guard < kWalkCap; it = L.next(it), ++guard) ++n;
    return n;
}

__device__ __forceinline__ void axpy3(f3& acc, float s, const float* p) {
    acc.x += s * p[0];
    acc.y += s * p[1];
    acc.z += s * p[2];
}

// 1. edge gather: gE[e] += vertex-pass terms
template <class View>
__device__ __forceinline__ void adj_edge_item(const View& L, float* __restrict__ gNew, int32_t h) {
    const int32_t tw = L.twin(h);
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
__device__ __forceinline__ void adj_face_item(const View& L, float* __restrict__ gNew, int32_t f) {
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
    } while (h != h0 && ++guard < kWalkCap);
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
__device__ __forceinline__ void adj_vertex_item(const View& L, const float* __restrict__ gNew,
                                                float* __restrict__ gOld, int32_t v) {
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
    } while (it >= 0 && it != h0 && ++n < kWalkCap);
    if (it < 0) {
        n = 0;
        for (it = L.next_vertex_he(h0); it >= 0 && it != h0 && n < kWalkCap; it = L.next_vertex_he(it), ++n)
            adj_vertex_term(L, it, gVv, gF, gE, acc);
    }
    float* o = gOld + 3 * (int64_t)v;
    o[0] += acc.x;
    o[1] += acc.y;
    o[2] += acc.z;
}


}  // namespace ccs
