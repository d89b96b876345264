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

// The same copy issued without the wait, and one box of a 128-byte swizzled
// child tile (1024-byte aligned in shared memory) to row `row` of the tensor
// `tmap` describes (TMA tensor store, no multicast; rows past the tensor's end
// are not written): the issuing thread must call bulk_wait_read() before the
// block ends (or reuses the tile).
__device__ __forceinline__ void bulk_store_tile_async(void* gdst, const void* ssrc, uint32_t bytes) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 :: "l"(gdst), "r"(s), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void tensor_store_tile_async(const void* tmap, const void* ssrc, int32_t row) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                 :: "l"(tmap), "r"(0), "r"(row), "r"(s) : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// `nrows` rows of a 128-byte swizzled child tile, stored as consecutive boxes
// of kChildBoxRows rows (4 KB apart, each 1024-byte aligned) to rows [row0,
// row0 + nrows) of a child-record map with `limit` rows: boxes that start
// past the end are skipped, one that runs past it is clipped by the copy.
// The issuing thread calls bulk_wait_read() before the tile is reused or the
// block ends.
__device__ __forceinline__ void tensor_store_rows_async(const void* tmap, const void* tile, int32_t row0, int nrows,
                                                        int32_t limit) {
    for (int b = 0; b < nrows; b += kChildBoxRows) {
        if (row0 + b >= limit) break;
        tensor_store_tile_async(tmap, static_cast<const char*>(tile) + 128 * b, row0 + b);
    }
}

__device__ __forceinline__ f3 shfl3(f3 v, int src) {
    return f3{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
              __shfl_sync(0xffffffffu, v.z, src)};
}
__device__ __forceinline__ f3 shfl_xor3(f3 v, int m) {
    return f3{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m),
              __shfl_xor_sync(0xffffffffu, v.z, m)};
}
// A 12-byte point as one 8-byte vector atomic (the aligned pair) and one
// scalar atomic: two reductions instead of three (vector float atomics are
// native from sm_90 on).
__device__ __forceinline__ void atomic_add3(float* o, f3 v) {
    if ((reinterpret_cast<uintptr_t>(o) & 7u) == 0) {
        atomicAdd(reinterpret_cast<float2*>(o), make_float2(v.x, v.y));
        atomicAdd(o + 2, v.z);
    } else {
        atomicAdd(o, v.x);
        atomicAdd(reinterpret_cast<float2*>(o + 1), make_float2(v.y, v.z));
    }
}

// Face point of the quad held by lanes qb..qb+3, in halfedge order,
// ((0 + p0/4) + p1/4) + p2/4) + p3/4 (CatmullClark.h:2032-2052), from the
// lanes' quartered points p4 = p / 4 (x / 4 is exact, so shuffling quarters
// gives the same terms).  Fewer instructions than quad_face_point_next: the
// points-only step (issue-bound) gains from it, the step with the topology
// (bound by its dependent loads) measured slower with it.
__device__ __forceinline__ f3 quad_face_point4(f3 p4, int qb) {
    const f3 q0 = shfl3(p4, qb), q1 = shfl3(p4, qb + 1), q2 = shfl3(p4, qb + 2), q3 = shfl3(p4, qb + 3);
    return add3(add3(add3(add3(zero3(), q0), q1), q2), q3);
}
// The same face point, and in `pn` the point of the next lane of the quad
// (taken from the face point's shuffles, none of its own).
__device__ __forceinline__ f3 quad_face_point_next(f3 p, int qb, int k, f3& pn) {
    const f3 q0 = shfl3(p, qb), q1 = shfl3(p, qb + 1), q2 = shfl3(p, qb + 2), q3 = shfl3(p, qb + 3);
    pn = k == 0 ? q1 : (k == 1 ? q2 : (k == 2 ? q3 : q0));
    return add3(add3(add3(add3(zero3(), quarter3(q0)), quarter3(q1)), quarter3(q2)), quarter3(q3));
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

// edge_share with a shortcut for an uncreased edge of the creased rule: with
// w = 0 the rule's lerp(smoothP, sharpP, 0) = smoothP + 0 * (sharpP - smoothP)
// is smoothP bit for bit unless a coordinate of smoothP is a zero (the sign
// of a zero sum can differ), which takes the full rule.
template <bool CREASED>
__device__ __forceinline__ f3 edge_share_fast(f3 v0, f3 v1, f3 F, bool boundary, float w) {
    if (CREASED && w == 0.0f) {
        const f3 sm = mul3(lerp3(v0, F, 0.5f), 0.5f);
        if (sm.x != 0.0f && sm.y != 0.0f && sm.z != 0.0f) return sm;
    }
    return edge_share<CREASED>(v0, v1, F, boundary, w);
}

// ---------------------------------------------------------------------------
// creases (CatmullClark.h:2950-2983, :2992-3026): item = parent crease
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 crease_item(const cc_Crease* __restrict__ in, cc_Crease* __restrict__ out,
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
    return make_float2(x.sharpness, y.sharpness);
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
    int zeroV = 0;                      // clear the vertex slots the atomic pass accumulates into
    float* __restrict__ zeroNext = nullptr;  // floats to clear for the next level's accumulation
    int64_t zeroNextN = 0;
    const float4* __restrict__ ostats = nullptr;  // older vertices' ring statistics (tile_level_ab)
    // crease half of depth d+1's ring statistics, added by the crease items
    // (the shape half must already be there); null = not kept
    float4* __restrict__ statsNext = nullptr;
    CageTables t;
    int32_t d = 0;
};

// Crease item e of depth d >= 1 that made children 2e, 2e+1 of sharpness
// `s`: each child's sharpness and sign go to the ring statistics of its end
// that is a depth-d vertex (crease_stats_item's rule, located without depth
// d+1's records).  Child 0 of halfedge h runs along half 2 e(h) + (h > twin
// ? 0 : 1) of e(h) from vertex(h); so with h0 = a halfedge of e, half b0 =
// (h0 > twin(h0) ? 0 : 1) ends at vertex(h0) and the other half at
// vertex(next h0).
template <int RW>
__device__ __forceinline__ void crease_stats_next(const LevelArgs& a, int32_t e, float2 s) {
    if (s.x == 0.0f && s.y == 0.0f) return;
    const int32_t h0 = edge_to_he(a.t, e, a.d);
    const int32_t tw0 = __ldg(a.in + (int64_t)RW * h0 + 0);
    const int32_t v0 = __ldg(a.in + (int64_t)RW * h0 + 2);
    const int32_t v1 = __ldg(a.in + (int64_t)RW * qnext(h0) + 2);
    const int b0 = h0 > tw0 ? 0 : 1;
    if (s.x != 0.0f) {
        float* o = reinterpret_cast<float*>(a.statsNext + (b0 == 0 ? v0 : v1));
        atomicAdd(o + 1, s.x);
        atomicAdd(o + 2, fsign(s.x));
    }
    if (s.y != 0.0f) {
        float* o = reinterpret_cast<float*>(a.statsNext + (b0 == 1 ? v0 : v1));
        atomicAdd(o + 1, s.y);
        atomicAdd(o + 2, fsign(s.y));
    }
}

// One parent record (twin, edge, vertex, uv); zeros past the level's end.
struct ARec {
    int32_t tw, ed, vx, uv;
};
// The four records of quad face f (RW = 3: three 16-byte loads of the 48
// bytes; the fourth word is then 0)
template <int RW>
__device__ __forceinline__ void load_face_records(const int32_t* __restrict__ in, int64_t f, int4 (&r)[4]) {
    const int4* q = reinterpret_cast<const int4*>(in + (int64_t)RW * 4 * f);
    if constexpr (RW == 4) {
#pragma unroll
        for (int k = 0; k < 4; ++k) r[k] = __ldg(q + k);
    } else {
        const int4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        r[0] = make_int4(a.x, a.y, a.z, 0); r[1] = make_int4(a.w, b.x, b.y, 0);
        r[2] = make_int4(b.z, b.w, c.x, 0); r[3] = make_int4(c.y, c.z, c.w, 0);
    }
}
template <int RW>
__device__ __forceinline__ ARec load_arec(const int32_t* __restrict__ in, int64_t h64, int64_t H) {
    ARec r{0, 0, 0, 0};
    if (h64 < H) {
        if constexpr (RW == 4) {
            const int4 q = __ldg(reinterpret_cast<const int4*>(in) + h64);
            r.tw = q.x; r.ed = q.y; r.vx = q.z; r.uv = q.w;
        } else {
            r.tw = __ldg(in + 3 * h64 + 0);
            r.ed = __ldg(in + 3 * h64 + 1);
            r.vx = __ldg(in + 3 * h64 + 2);
        }
    }
    return r;
}

// Writes a thread's four child records to its 16 * RW-byte slot of the shared
// tile with 16-byte stores free of bank conflicts.  RW = 4: the slots are 64
// bytes apart, so lanes start at different children (lane pair u of each
// quarter-warp at child u): the eight stores of a quarter-warp then cover
// the 32 banks once.  RW = 3: the three 16-byte words of 48-byte slots are
// conflict-free as they are (48 / 16 = 3 is odd).
template <int RW, bool UV>
__device__ __forceinline__ void put_children(int32_t* tile, int tid, int lane, const int32_t (&tw)[4],
                                             const int32_t (&ed)[4], const int32_t (&vx)[4],
                                             const int32_t (&uv)[4]) {
    int4* t4 = reinterpret_cast<int4*>(tile) + tid * RW;
    if constexpr (RW == 4) {
        int4 r0 = make_int4(tw[0], ed[0], vx[0], UV ? uv[0] : 0);
        int4 r1 = make_int4(tw[1], ed[1], vx[1], UV ? uv[1] : 0);
        int4 r2 = make_int4(tw[2], ed[2], vx[2], UV ? uv[2] : 0);
        int4 r3 = make_int4(tw[3], ed[3], vx[3], UV ? uv[3] : 0);
        const int r = (lane >> 1) & 3;
        if (r & 1) { const int4 x = r0; r0 = r1; r1 = r2; r2 = r3; r3 = x; }
        if (r & 2) { int4 x = r0; r0 = r2; r2 = x; x = r1; r1 = r3; r3 = x; }
        t4[r] = r0;
        t4[(r + 1) & 3] = r1;
        t4[(r + 2) & 3] = r2;
        t4[(r + 3) & 3] = r3;
    } else {
        t4[0] = make_int4(tw[0], ed[0], vx[0], tw[1]);
        t4[1] = make_int4(ed[1], vx[1], tw[2], ed[2]);
        t4[2] = make_int4(vx[2], tw[3], ed[3], vx[3]);
    }
}

// `tile` is BLOCK * 4 * RW ints of shared memory; every thread of the block
// must call this with the same h0, and `rec` = its parent record.  The child
// records go out through the shared tile and one bulk store per block (each
// thread's own 16-byte vector stores, measured, ran 17% slower at depth 5).
template <int BLOCK, int RW, bool TOPO, bool UV, bool PTS, bool CREASED>
__device__ __forceinline__ void tile_level_a_rec(const LevelArgs& a, int64_t h0, int32_t* tile, ARec rec) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = h0 + tid;
    const bool valid = h64 < a.H;
    const int32_t h = (int32_t)h64;
    const int k = lane & 3, qb = lane & ~3;
    const int32_t tw = rec.tw, ed = rec.ed, vx = rec.vx, uv = rec.uv;
    const int ln = qb | ((k + 1) & 3), lp = qb | ((k + 3) & 3), lo = qb | ((k + 2) & 3);
    const int32_t prev = (h & ~3) | ((k + 3) & 3), next = (h & ~3) | ((k + 1) & 3), f = h >> 2;
    int32_t c_tw[4] = {0, 0, 0, 0}, c_ed[4] = {0, 0, 0, 0}, c_vx[4] = {0, 0, 0, 0}, uvc[4] = {uv, 0, 0, 0};
    if (TOPO) {
        const int32_t ptw = __shfl_sync(0xffffffffu, tw, lp);
        const int32_t ped = __shfl_sync(0xffffffffu, ed, lp);
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
        c_tw[0] = child(qnext(tw), 3); c_tw[1] = child(next, 2); c_tw[2] = child(prev, 1); c_tw[3] = child(ptw, 0);
        c_ed[0] = 2 * ed + (h > tw ? 0 : 1); c_ed[1] = 2 * a.E + h; c_ed[2] = 2 * a.E + prev;
        c_ed[3] = 2 * ped + (prev > ptw ? 1 : 0);
        c_vx[0] = vx; c_vx[1] = a.V + a.F + ed; c_vx[2] = a.V + f; c_vx[3] = a.V + a.F + ped;
    }
    if (PTS) {
        const f3 p = valid ? ld3(a.pin + 3 * (int64_t)vx) : zero3();
        f3 pn;
        const f3 Fp = quad_face_point_next(p, qb, k, pn);
        if (valid && k == 0) st3(a.pout + 3 * ((int64_t)a.V + f), Fp);
        if (a.zeroV && h64 < a.V) st3(a.pout + 3 * h64, zero3());
        // edge point, by the pair's larger halfedge; the smaller one's share
        // is added first, as a one-thread reference run adds it
        if (valid && h > tw) {
            const float w = CREASED ? fsat(ed < a.C ? a.crIn[ed].sharpness : 0.0f) : 0.0f;
            const f3 sh_h = edge_share<CREASED>(p, pn, Fp, tw < 0, w);
            f3 E;
            if (tw >= 0) {
                // the twin quad's face point, in its halfedge order; by the
                // twin relation vertex(t) = vertex(next h) and vertex(next t)
                // = vertex(h), so only its other two vertices are read
                const int32_t tb = tw & ~3, kt = tw & 3;
                f3 q[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i == kt) q[i] = pn;
                    else if (i == ((kt + 1) & 3)) q[i] = p;
                    else q[i] = ld3(a.pin + 3 * (int64_t)__ldg(a.in + (int64_t)RW * (tb + i) + 2));
                }
                f3 Ft = zero3();
#pragma unroll
                for (int i = 0; i < 4; ++i) Ft = add3(Ft, quarter3(q[i]));
                const f3 sh_t = edge_share<CREASED>(pn, p, Ft, false, w);
                E = add3(add3(zero3(), sh_t), sh_h);
            } else {
                E = add3(zero3(), sh_h);
            }
            st3(a.pout + 3 * ((int64_t)a.V + a.F + ed), E);
        }
    }
    if (TOPO) {
        put_children<RW, UV>(tile, tid, lane, c_tw, c_ed, c_vx, uvc);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            const int64_t n = (a.H - h0) < BLOCK ? (a.H - h0) : BLOCK;
            bulk_store_tile(a.out + 4 * RW * h0, tile, (uint32_t)(n * 16 * RW));
        }
    }
}

template <int BLOCK, int RW, bool TOPO, bool UV, bool PTS, bool CREASED>
__device__ __forceinline__ void tile_level_a(const LevelArgs& a, int64_t h0, int32_t* tile) {
    tile_level_a_rec<BLOCK, RW, TOPO, UV, PTS, CREASED>(a, h0, tile, load_arec<RW>(a.in, h0 + threadIdx.x, a.H));
}

// ---------------------------------------------------------------------------
// Vertex rule of quad levels for one halfedge's share (creased rule in the
// corner-first branch order :2567-2607, crease-free rule :2307-2351), given
// the ring statistics the reference's walk from that halfedge finds
// (:2523-2566): vpre = valence before the boundary adjustment, cpre = crease
// count, avgS = summed sharpness, bnd = the walk met a boundary; cw / pcw =
// crease signs of the halfedge's edge and of its prev's edge, Ep = edge
// point of its prev's edge (read on a boundary only).
// ---------------------------------------------------------------------------
template <bool CREASED>
__device__ __forceinline__ f3 quad_vertex_rule(f3 p, f3 F, f3 E, f3 Ep, float vpre, float cpre, float avgS,
                                               bool bnd, float cw, float pcw) {
    f3 s;
    if (CREASED) {
        const float valence = bnd ? fadd(vpre, 1.0f) : vpre;
        const float creaseCount = bnd ? fadd(cpre, cw) : cpre;
        if (creaseCount >= 3.0f || valence == 2.0f) {
            s = mul3(p, frcp(vpre));
        } else if (creaseCount <= 1.0f) {
            f3 smooth = add3(mul3(F, -1.0f), mul3(E, 4.0f));
            smooth = add3(smooth, mul3(p, fsub(vpre, 3.0f)));
            s = mul3(smooth, frcp(fmul(vpre, vpre)));
        } else {
            const f3 corner = mul3(p, frcp(vpre));
            f3 crease = add3(mul3(p, fmul(0.25f, cw)), mul3(E, fmul(0.25f, cw)));
            if (bnd) crease = add3(crease, add3(mul3(p, fmul(0.25f, pcw)), mul3(Ep, fmul(0.25f, pcw))));
            s = lerp3(corner, crease, fsat(fmul(avgS, 0.5f)));
        }
    } else {
        const float w = frcp(vpre);
        const float ws = fmul(w, bnd ? 0.0f : 1.0f);
        s.x = fmul(w, fadd(p.x, fmul(ws, fsub(fsub(fmul(4.0f, E.x), F.x), fmul(3.0f, p.x)))));
        s.y = fmul(w, fadd(p.y, fmul(ws, fsub(fsub(fmul(4.0f, E.y), F.y), fmul(3.0f, p.y)))));
        s.z = fmul(w, fadd(p.z, fmul(ws, fsub(fsub(fmul(4.0f, E.z), F.z), fmul(3.0f, p.z)))));
    }
    return s;
}

__device__ __forceinline__ f3 shfl_down3(f3 v, int d) {
    return f3{__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d),
              __shfl_down_sync(0xffffffffu, v.z, d)};
}

// Order two (id, share) pairs by id.
__device__ __forceinline__ void order2(int32_t& ia, f3& sa, int32_t& ib, f3& sb) {
    if (ib < ia) {
        const int32_t ti = ia; ia = ib; ib = ti;
        const f3 ts = sa; sa = sb; sb = ts;
    }
}

// ---------------------------------------------------------------------------
// quad level d >= 1, kernel B body of the default pass: vertex points of
// depth d+1 from the halfedges [h0, h0 + blockDim) of depth d, accumulated
// with float atomics into slots kernel A cleared.
// ---------------------------------------------------------------------------
// One thread per halfedge h (child k = h & 3 of a parent halfedge).  Ring
// statistics without walks: a face centre (k = 2) and an edge midpoint
// (k = 1, 3) from the refined structure, an older vertex (k = 0) from the
// per-level table L.ostats (one walk per vertex when the topology was
// refined).  STRUCT (depth >= 2, a 16-lane group holds the children of one
// parent quad): a face centre's four shares are summed in lanes 2, 6, 10, 14
// in increasing halfedge order and stored (no atomic); an edge midpoint's two
// shares on this side go out as one atomic triple (two per interior vertex:
// the two additions commute, so the result does not depend on their order);
// an older vertex's shares as one atomic triple each.  Depth 1 (children of
// n-gons): one atomic triple per halfedge.
template <int RW, bool CREASED, bool STRUCT>
__device__ __forceinline__ void tile_level_b(const QuadView<RW>& L, const float* __restrict__ pin,
                                             float* __restrict__ pout, int64_t h0) {
    const unsigned full = 0xffffffffu;
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
    float4 st = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (valid) {
        p = ld3(pin + 3 * (int64_t)vx);
        Fh = ld3(fpt + 3 * (int64_t)(h >> 2));
        Eh = ld3(ept + 3 * (int64_t)ed);
        if (k == 0 && L.ostats) st = L.ostats[vx];
    }
    const f3 Ep = shfl3(Eh, lp);                      // edge point of prev(h)'s edge
    const int32_t ped = __shfl_sync(full, ed, lp);
    const int32_t ptw = __shfl_sync(full, tw, lp);
    f3 s = zero3();
    if (valid) {
        float vpre, cpre = 0.0f, avgS = 0.0f;
        bool bnd = false;
        if (k == 2) {
            vpre = L.d == 1 ? (float)L.t.fsz[L.t.he[(int64_t)CH_WORDS * (h >> 2) + CH_FACE]] : 4.0f;
        } else if (k != 0) {
            const int32_t eh = k == 1 ? ped : ed;        // one half of the parent edge
            bnd = (k == 1 ? ptw : tw) < 0;
            vpre = bnd ? 2.0f : 4.0f;
            if (CREASED) {
                const float sa = L.sharp(eh), sb = L.sharp(eh ^ 1);
                const bool own = k == 3;                 // the walk from h skips its own edge
                avgS = (bnd && own) ? sb : fadd(sa, sb);
                cpre = (bnd && own) ? fsign(sb) : fadd(fsign(sa), fsign(sb));
            }
        } else if (L.ostats) {
            // whole-ring statistics; on a boundary the walk from h skips h's own edge
            bnd = st.w != 0.0f;
            vpre = st.x;
            if (CREASED) {
                const float own = L.sharp(ed);
                avgS = bnd ? fsub(st.y, own) : st.y;
                cpre = bnd ? fsub(st.z, fsign(own)) : st.z;
            }
        } else {
            const RingStats r = creased_ring_walk(L, h);
            vpre = r.valence; cpre = r.creaseCount; avgS = r.avgS; bnd = r.fwd < 0;
        }
        s = quad_vertex_rule<CREASED>(p, Fh, Eh, Ep, vpre, cpre, avgS, bnd,
                                      CREASED ? fsign(L.sharp(ed)) : 0.0f, CREASED ? fsign(L.sharp(ped)) : 0.0f);
    }
    float* o = pout + 3 * (int64_t)vx;
    if (STRUCT) {
        const f3 s4 = shfl_down3(s, 4), s8 = shfl_down3(s, 8), s12 = shfl_down3(s, 12);
        const int partner = (lane & ~15) | ((((lane >> 2) + 1) & 3) << 2) | 3;
        const f3 sA2 = shfl3(s, partner);
        if (!valid) return;
        if ((lane & 15) == 2) {
            st3(o, add3(add3(add3(add3(zero3(), s), s4), s8), s12));
        } else if (k == 1) {
            // the pair in increasing halfedge order: child 3 of next(g) is
            // below child 1 of g only when next(g) wraps to the face's first
            atomic_add3(o, (lane & 12) == 12 ? add3(sA2, s) : add3(s, sA2));
        } else if (k == 0) {
            atomic_add3(o, s);
        }
    } else if (valid) {
        atomic_add3(o, s);
    }
}

// ---------------------------------------------------------------------------
// quad level d >= 2, one pass for the whole default step d -> d+1: kernel A's
// body (child records, face and edge points) and the default vertex pass's
// body (tile_level_b with STRUCT) over the same tile of depth-d halfedges.
// ---------------------------------------------------------------------------
// The vertex share of halfedge h needs its face point (the quad's lanes), its
// own edge point and that of prev(h) (a lane of the quad), its vertex point
// and the ring statistics; only the last come from memory (the older
// vertices' table `ostats`; face centres and edge midpoints from the
// structure).  So every halfedge evaluates its own edge point, not only the
// pair's owner.  At depth d >= 2 the twin of child 1 or 2 is child 2 or 1 of
// a sibling quad in the same 16-lane group, whose face point is read from
// that quad's lanes; the twin of child 0 is child 3 of its quad and the twin
// of child 3 is child 0 (CatmullClark.h:2778-2781), and that quad's face
// point is rebuilt: its vertices are vertex(h) and vertex(next h) (the twin
// relation) and the two others, read from its records, summed in its
// halfedge order.  Both halves evaluate (0 + share(smaller halfedge)) +
// share(larger halfedge), so both hold the owner's value bit for bit; the
// owner stores it.
// The vertex slots [0, V) of depth d+1 must be zero on entry; the tile also
// clears its share of `zeroNext` (the slots the next level accumulates into).
// Requires BLOCK a multiple of 32 and h0 a multiple of 16.
// TMAP (16-byte records, BLOCK = 256): the child records go out through TMA
// tensor stores of `tmap` (rows of 128 bytes = the children of two parent
// halfedges, kChildBoxRows rows a box) from a 128-byte swizzled tile
// (1024-byte aligned): 16-byte chunk
// c of row r sits at chunk c ^ (r & 7), which also spreads every
// quarter-warp's stores over the 32 banks.
template <int BLOCK, int RW, bool TOPO, bool UV, bool CREASED, bool TMAP = false, int EARLY = 0>
__device__ __forceinline__ void tile_level_ab(const LevelArgs& a, int64_t h0, int32_t* tile, int64_t zeroStride,
                                              const void* tmap = nullptr) {
    static_assert(!TMAP || (RW == 4 && BLOCK == 256), "tensor-store tiles are 256 sixteen-byte records wide");
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t h64 = h0 + tid;
    const bool valid = h64 < a.H;
    const int32_t h = (int32_t)h64;
    const ARec rec = load_arec<RW>(a.in, h64, a.H);
    const int k = lane & 3, qb = lane & ~3, j = (lane >> 2) & 3;
    const int32_t tw = rec.tw, ed = rec.ed, vx = rec.vx;
    const int ln = qb | ((k + 1) & 3), lp = qb | ((k + 3) & 3);
    const int32_t f = h >> 2;
    const int32_t ptw = __shfl_sync(full, tw, lp);
    const int32_t ped = __shfl_sync(full, ed, lp);

    // child records through the shared tile and one bulk store (EARLY = 1:
    // issued after the record's gathers, 2: before them -- both before the
    // points, with the wait left to the end; 0: after the points)
    auto child_records = [&]() {
        const int lo = qb | ((k + 2) & 3);
        const int32_t prev = (h & ~3) | ((k + 3) & 3), next = (h & ~3) | ((k + 1) & 3);
        int32_t c_tw[4], c_ed[4], c_vx[4], uvc[4] = {rec.uv, 0, 0, 0};
        if (UV) {
            const float u = uv_dec_fast((uint32_t)rec.uv), v = uv_dec_fast((uint32_t)rec.uv >> 16);
            const float un = __shfl_sync(full, u, ln), vn = __shfl_sync(full, v, ln);
            const float uo = __shfl_sync(full, u, lo), vo = __shfl_sync(full, v, lo);
            const float up = __shfl_sync(full, u, lp), vp = __shfl_sync(full, v, lp);
            uvc[1] = uv_enc_fast(flerp(u, un, 0.5f), flerp(v, vn, 0.5f));
            uvc[2] = uv_enc_fast(fquarter(fadd(fadd(fadd(u, un), uo), up)),
                                 fquarter(fadd(fadd(fadd(v, vn), vo), vp)));
            uvc[3] = uv_enc_fast(flerp(u, up, 0.5f), flerp(v, vp, 0.5f));
        }
        c_tw[0] = child(qnext(tw), 3); c_tw[1] = child(next, 2); c_tw[2] = child(prev, 1); c_tw[3] = child(ptw, 0);
        c_ed[0] = 2 * ed + (h > tw ? 0 : 1); c_ed[1] = 2 * a.E + h; c_ed[2] = 2 * a.E + prev;
        c_ed[3] = 2 * ped + (prev > ptw ? 1 : 0);
        c_vx[0] = vx; c_vx[1] = a.V + a.F + ed; c_vx[2] = a.V + f; c_vx[3] = a.V + a.F + ped;
        if constexpr (TMAP) {
            const int r = tid >> 1, sw = r & 7, cb = (tid & 1) << 2;
            int4* row = reinterpret_cast<int4*>(tile) + 8 * r;
#pragma unroll
            for (int m = 0; m < 4; ++m) row[(cb + m) ^ sw] = make_int4(c_tw[m], c_ed[m], c_vx[m], UV ? uvc[m] : 0);
        } else {
            put_children<RW, UV>(tile, tid, lane, c_tw, c_ed, c_vx, uvc);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            if constexpr (TMAP) {
                tensor_store_rows_async(tmap, tile, (int32_t)(h0 >> 1), BLOCK / 2, (int32_t)(a.H >> 1));
                if (EARLY == 0) bulk_wait_read();
            } else {
                const int64_t n = (a.H - h0) < BLOCK ? (a.H - h0) : BLOCK;
                if (EARLY != 0) bulk_store_tile_async(a.out + 4 * RW * h0, tile, (uint32_t)(n * 16 * RW));
                else bulk_store_tile(a.out + 4 * RW * h0, tile, (uint32_t)(n * 16 * RW));
            }
        }
    };

    if constexpr (TOPO && EARLY == 2) child_records();

    // every load that needs only the record, issued before any is used
    const int sibK = k == 1 ? ((((j + 1) & 3) << 2) | 2) : ((((j + 3) & 3) << 2) | 1);
    const bool inner = (k == 1 || k == 2) && tw == ((h & ~15) | sibK);
    const bool gatherTwin = valid && tw >= 0 && !inner;
    const f3 p = valid ? ld3(a.pin + 3 * (int64_t)vx) : zero3();
    const float sOwn = CREASED ? (valid && ed < a.C ? a.crIn[ed].sharpness : 0.0f) : 0.0f;
    float sOther = 0.0f;                                 // the other half of the parent edge (k = 1, 3)
    if (CREASED && valid && (k & 1)) {
        const int32_t eo = (k == 1 ? ped : ed) ^ 1;
        sOther = eo < a.C ? a.crIn[eo].sharpness : 0.0f;
    }
    const float4 st = (valid && k == 0) ? a.ostats[vx] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // the twin quad's two vertices other than vertex(h) and vertex(next h):
    // qF at position 2, qX at position 1 (child 0's twin) or 3 (child 3's)
    f3 qF = zero3(), qX = zero3();
    if (gatherTwin) {
        const int32_t vX = __ldg(a.in + (int64_t)RW * ((tw & ~3) + (k == 0 ? 1 : 3)) + 2);
        const int32_t vF = __ldg(a.in + (int64_t)RW * ((tw & ~3) + 2) + 2);
        qF = ld3(a.pin + 3 * (int64_t)vF);
        qX = ld3(a.pin + 3 * (int64_t)vX);
    }

    // EARLY = 1: the child records go out while those loads are in flight
    if constexpr (TOPO && EARLY == 1) child_records();

    // face point, and the next vertex's point from its shuffles
    f3 pn, Fp;
    if constexpr (TOPO) {
        Fp = quad_face_point_next(p, qb, k, pn);
    } else {
        Fp = quad_face_point4(quarter3(p), qb);
        pn = shfl3(p, ln);
    }
    if (valid && k == 0) st3(a.pout + 3 * ((int64_t)a.V + f), Fp);
    const f3 Fsib = shfl3(Fp, (lane & ~15) | sibK);      // a sibling quad's face point
    // edge point of h's edge, by both halves
    f3 E = zero3();
    if (valid) {
        const float w = CREASED ? fsat(sOwn) : 0.0f;
        const f3 sh_h = edge_share_fast<CREASED>(p, pn, Fp, tw < 0, w);
        if (tw >= 0) {
            f3 Ft;
            if (gatherTwin) {
                // the twin quad in position order: child 0's twin quad
                // (v(h), qX, qF, v(next h)), child 3's (v(next h), v(h), qF, qX)
                const f3 p4 = quarter3(p), pn4 = quarter3(pn), qX4 = quarter3(qX), qF4 = quarter3(qF);
                const bool c0 = k == 0;
                Ft = add3(add3(add3(add3(zero3(), c0 ? p4 : pn4), c0 ? qX4 : p4), qF4), c0 ? pn4 : qX4);
            } else {
                Ft = Fsib;
            }
            const f3 sh_t = edge_share_fast<CREASED>(pn, p, Ft, false, w);
            // (0 + a) + b and (0 + b) + a are the same float (x + y = y + x;
            // 0 + x differs from x only for x = -0, which both orders turn
            // into +0), so the points-only step skips the owner-order select
            if constexpr (TOPO) E = h > tw ? add3(add3(zero3(), sh_t), sh_h) : add3(add3(zero3(), sh_h), sh_t);
            else E = add3(add3(zero3(), sh_h), sh_t);
        } else {
            E = add3(zero3(), sh_h);
        }
        if (h > tw) st3(a.pout + 3 * ((int64_t)a.V + a.F + ed), E);
    }

    // vertex share of h (tile_level_b, STRUCT)
    const f3 Ep = shfl3(E, lp);
    const float sPrev = __shfl_sync(full, sOwn, lp);
    f3 s = zero3();
    if (valid) {
        float vpre, cpre = 0.0f, avgS = 0.0f;
        bool bnd = false;
        if (k == 2) {
            vpre = 4.0f;
        } else if (k != 0) {
            bnd = (k == 1 ? ptw : tw) < 0;
            vpre = bnd ? 2.0f : 4.0f;
            if (CREASED) {
                const float sa = k == 1 ? sPrev : sOwn;  // this side's half of the parent edge
                const bool own = k == 3;                 // the walk from h skips its own edge
                avgS = (bnd && own) ? sOther : fadd(sa, sOther);
                cpre = (bnd && own) ? fsign(sOther) : fadd(fsign(sa), fsign(sOther));
            }
        } else {
            bnd = st.w != 0.0f;
            vpre = st.x;
            if (CREASED) {
                avgS = bnd ? fsub(st.y, sOwn) : st.y;
                cpre = bnd ? fsub(st.z, fsign(sOwn)) : st.z;
            }
        }
        s = quad_vertex_rule<CREASED>(p, Fp, E, Ep, vpre, cpre, avgS, bnd, CREASED ? fsign(sOwn) : 0.0f,
                                      CREASED ? fsign(sPrev) : 0.0f);
    }
    {
        float* o = a.pout + 3 * (int64_t)vx;
        const f3 s4 = shfl_down3(s, 4), s8 = shfl_down3(s, 8), s12 = shfl_down3(s, 12);
        const int partner = (lane & ~15) | ((((lane >> 2) + 1) & 3) << 2) | 3;
        const f3 sA2 = shfl3(s, partner);
        if (valid) {
            if ((lane & 15) == 2) {
                st3(o, add3(add3(add3(add3(zero3(), s), s4), s8), s12));
            } else if (k == 1) {
                atomic_add3(o, (lane & 12) == 12 ? add3(sA2, s) : add3(s, sA2));
            } else if (k == 0) {
                atomic_add3(o, s);
            }
        }
    }

    // clear this thread's share of the next level's accumulation slots
    for (int64_t i = h64; i < a.zeroNextN; i += zeroStride) a.zeroNext[i] = 0.0f;

    if constexpr (TOPO && EARLY == 0) child_records();
    if constexpr (TOPO && EARLY != 0) {
        if (tid == 0) bulk_wait_read();
    }
}

// The points of the step d -> d+1 for depth-d face f (k_level_fq's body; r =
// its four records, valid = f is a face of the level; every lane of the warp
// calls it): face point, inner edge j, the two outer edge points it owns,
// the four vertex shares (see k_level_fq in ccs_level.cu).
// VERTS = false: face and edge points only (kernel A of the exact pass; no
// ring statistics read, no vertex slot touched).
template <int RW, bool CREASED, bool VERTS = true>
__device__ __forceinline__ void fq_points(const LevelArgs& a, int64_t f, bool valid, const int4 (&r)[4]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, qb = lane & ~3, j = lane & 3;
    const int ln = qb | ((j + 1) & 3), lp = qb | ((j + 3) & 3);
    const int32_t h0 = (int32_t)(4 * f);
    const int32_t tw0 = r[0].x, e0 = r[0].y, C = r[0].z;  // (j, 0): C_j -> M_j
    const int32_t e1 = r[1].y, Mj = r[1].z;               // (j, 1): M_j -> Z, inner edge j
    const int32_t Z = r[2].z;                             // (j, 2): Z -> M_{j-1}
    const int32_t tw3 = r[3].x, e3 = r[3].y, Mp = r[3].z; // (j, 3): M_{j-1} -> C_j
    // across parent edge j: the far vertex of (j, 0)'s twin quad and that
    // quad's centre; across parent edge j-1: the far vertex of (j, 3)'s
    int32_t vX0 = 0, vF0 = 0, vX3 = 0;
    if (valid && tw0 >= 0) {
        vX0 = __ldg(a.in + (int64_t)RW * ((tw0 & ~3) + 1) + 2);
        // the centre of parent quad T is vertex V(d-1) + T (the face points
        // follow the older vertices), and Z - G = V(d-1): no record read
        // (depth 5 of the headline workload: points-only step 0.221 -> 0.217 ms)
        vF0 = Z - (int32_t)(f >> 2) + (tw0 >> 4);
    }
    if (valid && tw3 >= 0) vX3 = __ldg(a.in + (int64_t)RW * ((tw3 & ~3) + 3) + 2);
    f3 pC = zero3(), pM = zero3(), pZ = zero3(), pMp = zero3(), qX0 = zero3(), qF0 = zero3(), qX3 = zero3();
    float4 st = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float s0 = 0.0f, s1 = 0.0f, s3 = 0.0f;
    if (valid) {
        pC = ld3(a.pin + 3 * (int64_t)C);
        pM = ld3(a.pin + 3 * (int64_t)Mj);
        pZ = ld3(a.pin + 3 * (int64_t)Z);
        pMp = ld3(a.pin + 3 * (int64_t)Mp);
        if (VERTS) st = a.ostats[C];
        if (CREASED) {
            s0 = e0 < a.C ? __ldg(&a.crIn[e0].sharpness) : 0.0f;
            s1 = e1 < a.C ? __ldg(&a.crIn[e1].sharpness) : 0.0f;
            s3 = e3 < a.C ? __ldg(&a.crIn[e3].sharpness) : 0.0f;
        }
        if (tw0 >= 0) {
            qX0 = ld3(a.pin + 3 * (int64_t)vX0);
            qF0 = ld3(a.pin + 3 * (int64_t)vF0);
        }
        if (tw3 >= 0) qX3 = ld3(a.pin + 3 * (int64_t)vX3);
    }
    // the other half of parent edge j is (j+1, 3), of parent edge j-1 is
    // (j-1, 0); the edge of (j, 2) is inner edge j-1
    const float s3n = __shfl_sync(full, s3, ln), s0p = __shfl_sync(full, s0, lp), s1p = __shfl_sync(full, s1, lp);

    // face point
    const f3 F = add3(add3(add3(add3(zero3(), quarter3(pC)), quarter3(pM)), quarter3(pZ)), quarter3(pMp));
    if (valid) st3(a.pout + 3 * ((int64_t)a.V + f), F);
    const int64_t eOut = (int64_t)a.V + a.F;
    // inner edge j: (j, 1) and its twin (j+1, 2), with the next lane's face point
    const f3 Fn = shfl3(F, ln);
    f3 I;
    {
        const float w = CREASED ? fsat(s1) : 0.0f;
        I = add3(add3(zero3(), edge_share_fast<CREASED>(pM, pZ, F, false, w)),
                 edge_share_fast<CREASED>(pZ, pM, Fn, false, w));
        if (valid) st3(a.pout + 3 * (eOut + e1), I);
    }
    const f3 Ip = shfl3(I, lp);                            // inner edge j-1
    // (j, 0): C_j -> M_j, half of parent edge j
    f3 Eo0;
    {
        const float w = CREASED ? fsat(s0) : 0.0f;
        const f3 sh = edge_share_fast<CREASED>(pC, pM, F, tw0 < 0, w);
        if (tw0 >= 0) {
            const f3 Ft = add3(add3(add3(add3(zero3(), quarter3(pC)), quarter3(qX0)), quarter3(qF0)), quarter3(pM));
            Eo0 = add3(add3(zero3(), sh), edge_share_fast<CREASED>(pM, pC, Ft, false, w));
        } else {
            Eo0 = add3(zero3(), sh);
        }
        if (valid && h0 > tw0) st3(a.pout + 3 * (eOut + e0), Eo0);
    }
    // (j, 3): M_{j-1} -> C_j, half of parent edge j-1, whose twin quad's
    // centre the previous lane read
    const f3 qFp = shfl3(qF0, lp);
    f3 Eo3;
    {
        const float w = CREASED ? fsat(s3) : 0.0f;
        const f3 sh = edge_share_fast<CREASED>(pMp, pC, F, tw3 < 0, w);
        if (tw3 >= 0) {
            const f3 Ft = add3(add3(add3(add3(zero3(), quarter3(pC)), quarter3(pMp)), quarter3(qFp)), quarter3(qX3));
            Eo3 = add3(add3(zero3(), sh), edge_share_fast<CREASED>(pC, pMp, Ft, false, w));
        } else {
            Eo3 = add3(zero3(), sh);
        }
        if (valid && h0 + 3 > tw3) st3(a.pout + 3 * (eOut + e3), Eo3);
    }
    if constexpr (!VERTS) return;
    // vertex shares (tile_level_b's rules)
    {   // (j, 0): the corner; on a boundary the walk from it skips its own edge
        const bool bnd = st.w != 0.0f;
        const float avgS = CREASED ? (bnd ? fsub(st.y, s0) : st.y) : 0.0f;
        const float cpre = CREASED ? (bnd ? fsub(st.z, fsign(s0)) : st.z) : 0.0f;
        const f3 s = quad_vertex_rule<CREASED>(pC, F, Eo0, Eo3, st.x, cpre, avgS, bnd,
                                               CREASED ? fsign(s0) : 0.0f, CREASED ? fsign(s3) : 0.0f);
        if (a.d >= 3) {
            // From depth 3 the parent quads G = 4 F' + j' of a grandparent face F'
            // fill a 16-lane group (lane = 16 (F' & 1) + 4 j' + j), and parent
            // quad j''s corners are F''s corner j', its midpoints j' and j'-1
            // and its centre.  So the centre's four shares (corner 2 of every
            // parent quad) are all in the group: summed and stored, no atomic;
            // midpoint j' is corner 1 of quad j' and corner 3 of quad j'+1:
            // one atomic for the pair.  Half the corner atomics go (depth 5 of the
            // headline workload: full step 0.412 -> 0.382 ms, points-only
            // 0.218 -> 0.199 ms).
            const int jq = (lane >> 2) & 3;
            const f3 t1 = add3(s, shfl_xor3(s, 4));
            const f3 t2 = add3(t1, shfl_xor3(t1, 8));
            const f3 pr = shfl3(s, (lane & 16) | (((jq + 1) & 3) << 2) | 3);
            if (valid) {
                float* o = a.pout + 3 * (int64_t)C;
                if (j == 0) atomic_add3(o, s);
                else if (j == 1) atomic_add3(o, add3(s, pr));
                else if (j == 2 && jq == 0) st3(o, t2);
            }
        } else if (valid) {
            atomic_add3(a.pout + 3 * (int64_t)C, s);
        }
    }
    f3 sM3;
    {   // (j, 3): midpoint M_{j-1}; the walk from it skips its own edge
        const bool bnd = tw3 < 0;
        const float avgS = CREASED ? (bnd ? s0p : fadd(s3, s0p)) : 0.0f;
        const float cpre = CREASED ? (bnd ? fsign(s0p) : fadd(fsign(s3), fsign(s0p))) : 0.0f;
        sM3 = quad_vertex_rule<CREASED>(pMp, F, Eo3, Ip, bnd ? 2.0f : 4.0f, cpre, avgS, bnd,
                                        CREASED ? fsign(s3) : 0.0f, CREASED ? fsign(s1p) : 0.0f);
    }
    {   // (j, 1): midpoint M_j, added with the next lane's (j+1, 3) share
        const bool bnd = tw0 < 0;
        const float avgS = CREASED ? fadd(s0, s3n) : 0.0f;
        const float cpre = CREASED ? fadd(fsign(s0), fsign(s3n)) : 0.0f;
        const f3 s = quad_vertex_rule<CREASED>(pM, F, I, Eo0, bnd ? 2.0f : 4.0f, cpre, avgS, bnd,
                                               CREASED ? fsign(s1) : 0.0f, CREASED ? fsign(s0) : 0.0f);
        const f3 pair = add3(s, shfl3(sM3, ln));
        if (a.d >= 3) {
            // From depth 3 parent edges 1 and 2 of a parent quad are inner edges
            // of its grandparent face: their twins are parent edges 2 and 1 of
            // the neighbouring parent quads in the same 16-lane group, so the
            // midpoint's two pairs meet here and are stored by one lane (depth
            // 5 of the headline workload: full step 0.373 -> 0.369 ms,
            // points-only 0.199 -> 0.195 ms).
            const int jq = (lane >> 2) & 3;
            const int tq = j == 1 ? ((jq + 1) & 3) : ((jq + 3) & 3);
            const f3 other = shfl3(pair, (lane & 16) | (tq << 2) | (j == 1 ? 2 : 1));
            if (valid) {
                if (j == 1) st3(a.pout + 3 * (int64_t)Mj, add3(pair, other));
                else if (j != 2) atomic_add3(a.pout + 3 * (int64_t)Mj, pair);
            }
        } else if (valid) {
            atomic_add3(a.pout + 3 * (int64_t)Mj, pair);
        }
    }
    {   // (j, 2): the centre, summed by lane 0 of the quad in face order
        const f3 s = quad_vertex_rule<CREASED>(pZ, F, Ip, I, 4.0f, 0.0f, 0.0f, false,
                                               CREASED ? fsign(s1p) : 0.0f, CREASED ? fsign(s1) : 0.0f);
        const f3 a1 = shfl3(s, qb + 1), a2 = shfl3(s, qb + 2), a3 = shfl3(s, qb + 3);
        if (valid && j == 0) st3(a.pout + 3 * (int64_t)Z, add3(add3(add3(add3(zero3(), s), a1), a2), a3));
    }
}

// ---------------------------------------------------------------------------
// quad level d >= 2, kernel B body of the exact (deterministic) pass:
// face-centre and edge-midpoint vertex points of depth d+1 from the
// halfedges [h0, h0 + blockDim) of depth d.
// ---------------------------------------------------------------------------
// Exact vertex pass at depth d >= 2, one thread per depth-d face f = 4 g + j
// (face j of the parent quad g; lane j of a quad of lanes, the layout of
// fq_points).  Face j has halfedges (j, k) = 4 f + k at the corner C_j
// (k = 0), the midpoint M_j of parent edge j (k = 1), the centre Z of g
// (k = 2) and M_{j-1} (k = 3).  The thread evaluates the shares of (j, 1),
// (j, 2) and (j, 3) from kernel A's face and edge points:
//   Z: its four shares are the (j, 2) of the quad's lanes, summed by lane 0
//      in increasing halfedge order;
//   M_j (valence 4, or 2 on a boundary; its only creased edges are the two
//      halves e, e^1 of parent edge j): its shares are (j, 1) and (j+1, 3)
//      here, and child 1 of t = twin(g) and child 3 of next(t) across the
//      parent edge.  The thread of the pair's owner (g > t, or t < 0) sums
//      all of them: the twin side's two shares are rebuilt from face and
//      edge points alone, since their ring statistics equal this side's;
//   C_j: an older vertex.  With GRAND (d >= 3, g = 4 G + J a child of the
//      grandparent face G) the corners that are G's centre (j = 2) or the
//      midpoint of G's edge J (j = 1 of quad J, j = 3 of quad J+1) are
//      summed here too, by the statistics and arithmetic of
//      old_vertex_item: the centre's four members (child 0 of the lanes
//      j = 2) by the lane of quad 0, the midpoint's four by the j = 1 lane
//      of the pair's owner (G's halfedge > its twin T, or no twin), the
//      twin side's two (child 0 of faces 4 T + 1 and 4 next(T) + 3) rebuilt.
//      Corners older than G go to old_vertex_item (vertex ids below V(d-2)).
// Every vertex is summed by one thread in increasing halfedge order, starting
// from zero, so the result is bit-identical to the reference's one-thread
// scatter loop (:2496-2615) and needs neither atomics nor cleared slots.
// Sharpness at depth >= 1 is +0 or positive, so the structural sums of
// sharpness equal the walk's, zeros and order notwithstanding (a sum is read
// only where two terms are nonzero).
// Requires f0 and blockDim to be multiples of 32 (the quad's lanes agree on
// validity: the face count is a multiple of 4 at depth >= 2; with GRAND a
// multiple of 16).
template <int RW, bool CREASED, bool GRAND>
__device__ __forceinline__ void tile_face_exact(const QuadView<RW>& L, const float* __restrict__ pin,
                                                float* __restrict__ pout, int64_t f0) {
    const int64_t nF = (int64_t)L.H >> 2;
    const int64_t f = f0 + threadIdx.x;
    const bool valid = f < nF;
    const int lane = threadIdx.x & 31, qb = lane & ~3, j = lane & 3;
    const int ln = qb | ((j + 1) & 3), lp = qb | ((j + 3) & 3);
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    int4 r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = make_int4(-1, 0, 0, 0);
    if (valid) load_face_records<RW>(L.he, f, r);
    const int32_t tw0 = r[0].x, e0 = r[0].y, C = r[0].z;   // (j, 0): a half of parent edge j
    const int32_t e1 = r[1].y, Mj = r[1].z;                // (j, 1): inner edge j
    const int32_t e2 = r[2].y, Z = r[2].z;                 // (j, 2): inner edge j-1
    const int32_t tw3 = r[3].x, e3 = r[3].y, Mp = r[3].z;  // (j, 3): a half of parent edge j-1
    const int32_t g = (int32_t)(f >> 2);
    const bool own = (e0 & 1) == 0;                        // g owns parent edge j (g > t, or t < 0)
    const bool twinSide = own && tw0 >= 0;
    // child 0 of g: twin = 4 next(t) + 3, so next(t) and t are depth-d faces
    const int32_t tn = tw0 >> 2, t = qprev(tn);
    const int32_t eB1 = e1 - (int32_t)f + t;               // edge of child 1 of t: 2 E(d-1) + t
    // GRAND, lane j = 1: C = M_J of G's halfedge g.  (j, 3)'s twin is child 0
    // of face 4 next(T) + 3; child 0 of face 4 T + 1 has the edge
    // 2 (2 E(d-2) + T) + (T > next(T) ? 0 : 1), where 2 E(d-2) + g = e0 >> 1
    const int32_t gT = qprev(tw3 >> 4);
    const bool ownC = GRAND && j == 1 && (tw3 < 0 || g > gT);
    const bool twinC = ownC && tw3 >= 0;
    const int32_t eT1 = 2 * ((e0 >> 1) - g + gT) + ((gT & 3) == 3 ? 0 : 1);
    f3 pM = zero3(), pZ = zero3(), pMp = zero3(), F = zero3(), E0 = zero3(), E1 = zero3(), E3 = zero3();
    f3 FB1 = zero3(), FB2 = zero3(), EB1 = zero3();
    float s0 = 0.0f, s0x = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f, s3x = 0.0f;
    if (valid) {
        pM = ld3(pin + 3 * (int64_t)Mj);
        pZ = ld3(pin + 3 * (int64_t)Z);
        pMp = ld3(pin + 3 * (int64_t)Mp);
        F = ld3(fpt + 3 * f);
        E0 = ld3(ept + 3 * (int64_t)e0);
        E1 = ld3(ept + 3 * (int64_t)e1);
        E3 = ld3(ept + 3 * (int64_t)e3);
        if (CREASED) {
            s0 = L.sharp(e0); s0x = L.sharp(e0 ^ 1); s1 = L.sharp(e1); s2 = L.sharp(e2);
            s3 = L.sharp(e3); s3x = L.sharp(e3 ^ 1);
        }
        if (twinSide) {
            FB1 = ld3(fpt + 3 * (int64_t)t);
            FB2 = ld3(fpt + 3 * (int64_t)tn);
            EB1 = ld3(ept + 3 * (int64_t)eB1);
        }
    }
    const f3 E2 = shfl3(E1, lp);                           // inner edge j-1 is the previous lane's
    // (j, 1) at M_j: the halves of its parent edge are e0 and e0 ^ 1
    const bool bnd1 = tw0 < 0;
    const float vpre1 = bnd1 ? 2.0f : 4.0f;
    const float avgS1 = CREASED ? fadd(s0, s0x) : 0.0f;
    const float cpre1 = CREASED ? fadd(fsign(s0), fsign(s0x)) : 0.0f;
    const f3 sh1 = quad_vertex_rule<CREASED>(pM, F, E1, E0, vpre1, cpre1, avgS1, bnd1, fsign(s1), fsign(s0));
    // (j, 2) at the centre
    const f3 sh2 = quad_vertex_rule<CREASED>(pZ, F, E2, E1, 4.0f, 0.0f, 0.0f, false, fsign(s2), fsign(s1));
    // (j, 3) at M_{j-1}: on a boundary the walk from it skips its own edge
    const bool bnd3 = tw3 < 0;
    const float avgS3 = CREASED ? (bnd3 ? s3x : fadd(s3, s3x)) : 0.0f;
    const float cpre3 = CREASED ? (bnd3 ? fsign(s3x) : fadd(fsign(s3), fsign(s3x))) : 0.0f;
    const f3 sh3 = quad_vertex_rule<CREASED>(pMp, F, E3, E2, bnd3 ? 2.0f : 4.0f, cpre3, avgS3, bnd3, fsign(s3),
                                             fsign(s2));
    const f3 c1 = shfl3(sh2, qb + 1), c2 = shfl3(sh2, qb + 2), c3 = shfl3(sh2, qb + 3);
    f3 sA2 = shfl3(sh3, ln);                               // (j+1, 3), also at M_j
    if (valid && j == 0) st3(pout + 3 * (int64_t)Z, add3(add3(add3(add3(zero3(), sh2), c1), c2), c3));
    if (valid && own) {
        int32_t iA1 = (int32_t)(4 * f + 1), iA2 = (int32_t)(4 * (f - j + ((j + 1) & 3)) + 3);
        f3 sA1 = sh1;
        order2(iA1, sA1, iA2, sA2);
        f3 acc;
        if (!twinSide) {
            acc = add3(add3(zero3(), sA1), sA2);
        } else {
            // child 1 of t, and child 3 of next(t), the twin of (j, 0) (edge e0, point E0)
            f3 b1 = quad_vertex_rule<CREASED>(pM, FB1, EB1, zero3(), vpre1, cpre1, avgS1, false,
                                              CREASED ? fsign(L.sharp(eB1)) : 0.0f, 0.0f);
            f3 b2 = quad_vertex_rule<CREASED>(pM, FB2, E0, zero3(), vpre1, cpre1, avgS1, false, fsign(s0), 0.0f);
            int32_t iB1 = 4 * t + 1, iB2 = 4 * tn + 3;
            order2(iB1, b1, iB2, b2);
            // merge the two ordered pairs
            order2(iA1, sA1, iB1, b1);                    // smallest in A1
            order2(iA2, sA2, iB2, b2);                    // largest in B2
            order2(iA2, sA2, iB1, b1);
            acc = add3(add3(add3(add3(zero3(), sA1), sA2), b1), b2);
        }
        st3(pout + 3 * (int64_t)Mj, acc);
    }
    if (GRAND) {
        // a third round of gathers, after the midpoints' registers are free
        f3 pC = zero3(), FT1 = zero3(), FT2 = zero3(), ET1 = zero3();
        float sT1 = 0.0f;
        if (valid && (j == 2 || ownC)) pC = ld3(pin + 3 * (int64_t)C);
        if (valid && twinC) {
            FT1 = ld3(fpt + 3 * (int64_t)(4 * gT + 1));
            FT2 = ld3(fpt + 3 * (int64_t)(tw3 >> 2));
            ET1 = ld3(ept + 3 * (int64_t)eT1);
            if (CREASED) sT1 = L.sharp(eT1);
        }
        const int gl = lane & ~15, J = (lane >> 2) & 3;
        // G's centre: members child 0 of the lanes j = 2, in quad order
        const float z0 = __shfl_sync(0xffffffffu, s0, gl | 2), z1 = __shfl_sync(0xffffffffu, s0, gl | 6);
        const float z2 = __shfl_sync(0xffffffffu, s0, gl | 10), z3 = __shfl_sync(0xffffffffu, s0, gl | 14);
        const float totZ = CREASED ? fadd(fadd(fadd(fadd(0.0f, z0), z1), z2), z3) : 0.0f;
        const float cntZ = CREASED ? fadd(fadd(fadd(fadd(0.0f, fsign(z0)), fsign(z1)), fsign(z2)), fsign(z3)) : 0.0f;
        const f3 shZ = quad_vertex_rule<CREASED>(pC, F, E0, zero3(), 4.0f, cntZ, totZ, false, fsign(s0), 0.0f);
        const f3 zs1 = shfl3(shZ, gl | 6), zs2 = shfl3(shZ, gl | 10), zs3 = shfl3(shZ, gl | 14);
        // G's midpoint of edge J: the second local member is child 0 of the
        // lane j = 3 of quad J+1 (face 4 next(g) + 3)
        const int l2 = gl | (((J + 1) & 3) << 2) | 3;
        const f3 F2 = shfl3(F, l2), E02 = shfl3(E0, l2);
        const float s02 = __shfl_sync(0xffffffffu, s0, l2);
        if (valid && j == 2 && J == 0)
            st3(pout + 3 * (int64_t)C, add3(add3(add3(add3(zero3(), shZ), zs1), zs2), zs3));
        if (ownC && valid) {
            int32_t i1 = 4 * (int32_t)f, i2 = 4 * (4 * qnext(g) + 3);
            f3 a1, a2, acc;
            if (!twinC) {
                // boundary: members child 0 of f and of face 4 next(g) + 3; the
                // ring's edge without a member is (j, 3)'s, the prev edge of
                // the second member is f's own (their twins share it)
                const float cA = CREASED ? fadd(fsign(s3), fsign(s02)) : 0.0f;
                const float aA = CREASED ? fadd(s3, s02) : 0.0f;
                const float cB = CREASED ? fadd(fsign(s3), fsign(s0)) : 0.0f;
                const float aB = CREASED ? fadd(s3, s0) : 0.0f;
                a1 = quad_vertex_rule<CREASED>(pC, F, E0, CREASED ? E3 : zero3(), 2.0f, cA, aA, true, fsign(s0),
                                               fsign(s3));
                a2 = quad_vertex_rule<CREASED>(pC, F2, E02, CREASED ? E0 : zero3(), 2.0f, cB, aB, true,
                                               fsign(s02), fsign(s0));
                order2(i1, a1, i2, a2);
                acc = add3(add3(zero3(), a1), a2);
            } else {
                // interior: the twin side's members child 0 of faces 4 T + 1
                // (edge eT1) and 4 next(T) + 3 (the twin of (j, 3), edge e3)
                const float tot = CREASED ? fadd(fadd(fadd(s0, s02), sT1), s3) : 0.0f;
                const float cnt = CREASED ? fadd(fadd(fadd(fsign(s0), fsign(s02)), fsign(sT1)), fsign(s3)) : 0.0f;
                a1 = quad_vertex_rule<CREASED>(pC, F, E0, zero3(), 4.0f, cnt, tot, false, fsign(s0), 0.0f);
                a2 = quad_vertex_rule<CREASED>(pC, F2, E02, zero3(), 4.0f, cnt, tot, false, fsign(s02), 0.0f);
                f3 b1 = quad_vertex_rule<CREASED>(pC, FT1, ET1, zero3(), 4.0f, cnt, tot, false, fsign(sT1), 0.0f);
                f3 b2 = quad_vertex_rule<CREASED>(pC, FT2, E3, zero3(), 4.0f, cnt, tot, false, fsign(s3), 0.0f);
                int32_t i3 = 4 * (4 * gT + 1), i4 = tw3;
                order2(i1, a1, i2, a2);
                order2(i3, b1, i4, b2);
                order2(i1, a1, i3, b1);                    // smallest in a1
                order2(i2, a2, i4, b2);                    // largest in b2
                order2(i2, a2, i3, b1);
                acc = add3(add3(add3(add3(zero3(), a1), a2), b1), b2);
            }
            st3(pout + 3 * (int64_t)C, acc);
        }
    }
}

// ---------------------------------------------------------------------------
// quad level d >= 2: vertex point of an older vertex v < V(d-1).  Its ring
// members are child-0 halfedges; one thread walks the ring once, gathers the
// statistics every member's own walk would find (the valence and crease count
// of the whole ring; the summed sharpness of the ring, or on a boundary of
// the ring without the member's own edge -- the sum only matters when the
// count is 2, where it has at most two nonzero terms and is order-free),
// and sums the shares in increasing halfedge order.  Rings longer than
// kRingRegs members take the generic sorted path.
// ---------------------------------------------------------------------------
static constexpr int kRingRegs = 8;

template <class View, bool CREASED>
__device__ __forceinline__ f3 vertex_share_of(const View& L, int32_t h, const float* pin, const float* fpt,
                                              const float* ept);

// Shares of the ring of h0 summed in increasing halfedge order, any view.
template <class View, bool CREASED>
__device__ f3 ring_sorted_sum(const View& L, int32_t h0, const float* __restrict__ pin,
                              const float* __restrict__ fpt, const float* __restrict__ ept) {
    constexpr int kMax = 24;
    int32_t ring[kMax];
    int n = 0;
    int32_t it = h0;
    do {
        if (n < kMax) ring[n] = it;
        ++n;
        it = L.prev_vertex_he(it);
    } while (it >= 0 && it != h0 && n < kWalkCap);
    if (it < 0) {
        for (it = L.next_vertex_he(h0); it >= 0 && it != h0 && n < kWalkCap; it = L.next_vertex_he(it)) {
            if (n < kMax) ring[n] = it;
            ++n;
        }
    }
    f3 acc = zero3();
    if (n <= kMax) {
        for (int a = 1; a < n; ++a) {            // insertion sort, n is small
            const int32_t x = ring[a];
            int b = a - 1;
            while (b >= 0 && ring[b] > x) { ring[b + 1] = ring[b]; --b; }
            ring[b + 1] = x;
        }
        for (int a = 0; a < n; ++a) acc = add3(acc, vertex_share_of<View, CREASED>(L, ring[a], pin, fpt, ept));
    } else {
        // rare high valence: pick ring members in increasing order by walks
        int32_t last = -1;
        for (int a = 0; a < n; ++a) {
            int32_t best = 0x7fffffff;
            int32_t w = h0;
            int steps = 0;
            do {
                if (w > last && w < best) best = w;
                w = L.prev_vertex_he(w);
            } while (w >= 0 && w != h0 && ++steps < kWalkCap);
            if (w < 0) {
                steps = 0;
                for (w = L.next_vertex_he(h0); w >= 0 && w != h0 && steps < kWalkCap; w = L.next_vertex_he(w), ++steps)
                    if (w > last && w < best) best = w;
            }
            acc = add3(acc, vertex_share_of<View, CREASED>(L, best, pin, fpt, ept));
            last = best;
        }
    }
    return acc;
}

template <int RW, bool CREASED>
__device__ __forceinline__ void old_vertex_item(const QuadView<RW>& L, const float* __restrict__ pin,
                                                float* __restrict__ pout, int32_t v) {
    constexpr int M = kRingRegs;
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    const int32_t h0 = L.vert_he(v);
    int32_t id[M], eo[M], ep[M];      // member, its edge, the edge of its prev
    // forward: x -> twin(prev(x)); edge(prev(x)) is the next member's edge
    int32_t x = h0, ex = L.edge(h0);
    bool run = true;
    int n = 0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        id[i] = 0x7fffffff; eo[i] = 0; ep[i] = 0;
        if (run) {
            id[i] = x; eo[i] = ex;
            const int32_t pr = qprev(x);
            ex = L.edge(pr);
            ep[i] = ex;
            x = L.twin(pr);
            n = i + 1;
            run = x >= 0 && x != h0;
        }
    }
    const bool bnd = x < 0;
    const int32_t eEnd = ex;          // on a boundary: the ring's last edge, no member's own
    bool over = run;
    if (bnd) {
        // backward: b = twin(c), next member next(b); edge(prev(next(b))) = edge(b) = edge(c)
        int32_t b = L.twin(h0), pe = eo[0];
#pragma unroll
        for (int i = 1; i < M; ++i) {
            if (i >= n && b >= 0) {
                const int32_t c = qnext(b);
                id[i] = c; ep[i] = pe;
                eo[i] = L.edge(c);
                pe = eo[i];
                b = L.twin(c);
                n = i + 1;
            }
        }
        over = b >= 0;
    }
    float* o = pout + 3 * (int64_t)v;
    if (over) {
        st3(o, ring_sorted_sum<QuadView<RW>, CREASED>(L, h0, pin, fpt, ept));
        return;
    }
    // sort the members by halfedge id (odd-even transposition; empty slots hold INT_MAX)
#pragma unroll
    for (int r = 0; r < M; ++r) {
#pragma unroll
        for (int i = r & 1; i + 1 < M; i += 2) {
            if (id[i + 1] < id[i]) {
                int32_t t = id[i]; id[i] = id[i + 1]; id[i + 1] = t;
                t = eo[i]; eo[i] = eo[i + 1]; eo[i + 1] = t;
                t = ep[i]; ep[i] = ep[i + 1]; ep[i + 1] = t;
            }
        }
    }
    const f3 p = ld3(pin + 3 * (int64_t)v);
    const float vpre = (float)n;
    float sh[M];
    float tot = 0.0f, cnt = 0.0f;
    if (CREASED) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            sh[i] = i < n ? L.sharp(eo[i]) : 0.0f;
            tot = fadd(tot, sh[i]);
            cnt = fadd(cnt, fsign(sh[i]));
        }
    }
    const float sEnd = (CREASED && bnd) ? L.sharp(eEnd) : 0.0f;
    f3 acc = zero3();
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i < n) {
            const f3 F = ld3(fpt + 3 * (int64_t)(id[i] >> 2));
            const f3 E = ld3(ept + 3 * (int64_t)eo[i]);
            f3 s;
            if (CREASED) {
                float avgS = tot, cpre = cnt, pcw = 0.0f;
                f3 Ep = zero3();
                if (bnd) {
                    avgS = sEnd;
                    cpre = fsign(sEnd);
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        if (m != i && m < n) { avgS = fadd(avgS, sh[m]); cpre = fadd(cpre, fsign(sh[m])); }
                    }
                    pcw = fsign(L.sharp(ep[i]));
                    Ep = ld3(ept + 3 * (int64_t)ep[i]);
                }
                s = quad_vertex_rule<true>(p, F, E, Ep, vpre, cpre, avgS, bnd, fsign(sh[i]), pcw);
            } else {
                s = quad_vertex_rule<false>(p, F, E, zero3(), vpre, 0.0f, 0.0f, bnd, 0.0f, 0.0f);
            }
            acc = add3(acc, s);
        }
    }
    st3(o, acc);
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

// item = vertex v: its shares summed in increasing halfedge order, which is
// the reference's one-thread scatter order (any view, any depth)
template <class View, bool CREASED>
__device__ __forceinline__ void vertex_det_item(const View& L, const float* __restrict__ pin,
                                                float* __restrict__ pout, int32_t v) {
    const float* fpt = pout + 3 * (int64_t)L.V;
    const float* ept = pout + 3 * ((int64_t)L.V + L.F);
    st3(pout + 3 * (int64_t)v, ring_sorted_sum<View, CREASED>(L, L.vert_he(v), pin, fpt, ept));
}

// ---------------------------------------------------------------------------
// adjoint of the creased scatter rule (see ccs_adjoint.cu): three gathers
// ---------------------------------------------------------------------------
// Ring statistics of an older vertex v < V(d-1) of quad level d, {valence,
// summed sharpness and crease count of every incident edge, boundary} for
// ring_from_stats, without walking the level: the valence and boundary of
// an older vertex are those it was created with (refinement keeps a
// vertex's ring), and its creased edges are found from the crease side.
//
// Valence (outgoing halfedges) and boundary of vertex v < V(d-1) at quad
// level d >= 1, from the vertex numbering and the cage alone: a face centre
// of a level >= 1 quad has 4 (interior); of a cage face, the face's size; an
// edge midpoint 4, or 2 when its edge descends from a cage boundary edge
// (edges created inside faces are interior); a cage vertex its cage ring.
__device__ __forceinline__ void old_vertex_shape(const CageTables& t, int32_t v, int32_t d, int32_t& valence,
                                                 bool& bnd) {
    for (int32_t hd = d; hd > 1; --hd) {
        const int32_t Vc = cnt_V(t.n, hd - 1), Fc = cnt_F(t.n, hd - 1);
        if (v >= Vc + Fc) {                          // midpoint of edge e of level hd - 1
            int32_t e = v - Vc - Fc, j = hd - 1;
            for (; j >= 1 && e < 2 * cnt_E(t.n, j - 1); --j) e >>= 1;
            bnd = j == 0 && t.he[(int64_t)CH_WORDS * t.e2h[e] + CH_TWIN] < 0;
            valence = bnd ? 2 : 4;
            return;
        }
        if (v >= Vc) { valence = 4; bnd = false; return; }
    }
    const CageCounts& n = t.n;
    if (v >= n.V + n.F) {                            // midpoint of a cage edge
        bnd = t.he[(int64_t)CH_WORDS * t.e2h[v - n.V - n.F] + CH_TWIN] < 0;
        valence = bnd ? 2 : 4;
        return;
    }
    if (v >= n.V) { valence = t.fsz[v - n.V]; bnd = false; return; }
    if (t.vshape) {                                  // a cage vertex, its shape kept
        const int32_t x = t.vshape[v];
        valence = x & 0x3FFFFFFF;
        bnd = (x >> 30) & 1;
        return;
    }
    // a cage vertex: its ring in the cage (twin(prev h) forward, next(twin h) back)
    const int32_t h0 = t.v2h[v];
    int32_t cntv = 1, x = h0, guard = 0;
    auto tw = [&](int32_t h) { return t.he[(int64_t)CH_WORDS * h + CH_TWIN]; };
    for (x = tw(t.he[(int64_t)CH_WORDS * h0 + CH_PREV]); x >= 0 && x != h0 && guard < kWalkCap;
         x = tw(t.he[(int64_t)CH_WORDS * x + CH_PREV]), ++guard)
        ++cntv;
    if (x < 0) {
        guard = 0;
        for (int32_t y = tw(h0); y >= 0 && guard < kWalkCap; ++guard) {
            y = t.he[(int64_t)CH_WORDS * y + CH_NEXT];
            ++cntv;
            y = tw(y);
        }
    }
    valence = cntv;
    bnd = x < 0;
}

// item = older vertex v: {valence, 0, 0, boundary}; the crease pass adds the
// summed sharpness and crease count
__device__ __forceinline__ void shape_stats_item(const CageTables& t, int32_t d, float4* __restrict__ out,
                                                 int32_t v) {
    int32_t valence;
    bool bnd;
    old_vertex_shape(t, v, d, valence, bnd);
    out[v] = make_float4((float)valence, 0.0f, 0.0f, bnd ? 1.0f : 0.0f);
}

// item = crease (edge) c < C of quad level d with nonzero sharpness: one end
// of c is an older vertex (an end of the parent edge), the other the parent
// edge's midpoint; the older end's statistics take its sharpness and sign.
template <int RW>
__device__ __forceinline__ void crease_stats_item(const QuadView<RW>& L, int32_t Vold, float4* __restrict__ out,
                                                  int32_t c) {
    const float s = L.cr[c].sharpness;
    if (s == 0.0f) return;
    const int32_t h = edge_to_he(L.t, c, L.d);
    const int32_t v0 = L.vert(h), v1 = L.vert(qnext(h));
    float* o = reinterpret_cast<float*>(out + (v0 < Vold ? v0 : v1));
    atomicAdd(o + 1, s);
    atomicAdd(o + 2, fsign(s));
}

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

// ---------------------------------------------------------------------------
// adjoint of a quad level (d >= 1) in two halfedge-parallel passes with the
// forward's lane structure (a face's 4 halfedges in 4 adjacent lanes); needs
// the twin relation vertex(twin h) = vertex(next h).
// ---------------------------------------------------------------------------
// Coefficients of the quad-level vertex rule from its ring statistics
// (vertex_coef's formulas, corner-first branch order).
__device__ __forceinline__ VCoef coef_from_stats(float vp, float cpre, float avgS, bool bnd, float cw, float pcw) {
    const float valence = bnd ? vp + 1.0f : vp;
    const float creaseCount = bnd ? cpre + cw : cpre;
    VCoef k{0.0f, 0.0f, 0.0f, 0.0f};
    if (creaseCount >= 3.0f || valence == 2.0f) {
        k.a = 1.0f / vp;
    } else if (creaseCount <= 1.0f) {
        const float inv = 1.0f / (vp * vp);
        k.a = (vp - 3.0f) * inv;
        k.bF = -inv;
        k.cE = 4.0f * inv;
    } else {
        const float t = fsat(avgS * 0.5f);
        k.a = (1.0f - t) / vp + t * 0.25f * (cw + (bnd ? pcw : 0.0f));
        k.cE = t * 0.25f * cw;
        k.dE = bnd ? t * 0.25f * pcw : 0.0f;
    }
    return k;
}

// The vertex coefficients of halfedge h from its own record (tw, ed), its
// prev lane's (ptw, ped) and, for child 0, its older vertex's statistics `st`
// -- what vertex_coef finds by reading the level.
template <int RW>
__device__ __forceinline__ VCoef lane_vertex_coef(const QuadView<RW>& L, int32_t h, int32_t tw, int32_t ed,
                                                  int32_t ptw, int32_t ped, const float4& st) {
    const int k = h & 3;
    float vp, cpre = 0.0f, avgS = 0.0f;
    bool bnd = false;
    if (k == 2) {
        vp = L.d == 1 ? (float)L.t.fsz[L.t.he[(int64_t)CH_WORDS * (h >> 2) + CH_FACE]] : 4.0f;
    } else if (k != 0) {
        const int32_t eh = k == 1 ? ped : ed;
        const float sa = L.sharp(eh), sb = L.sharp(eh ^ 1);
        bnd = (k == 1 ? ptw : tw) < 0;
        vp = bnd ? 2.0f : 4.0f;
        const bool own = k == 3;
        avgS = (bnd && own) ? sb : sa + sb;
        cpre = (bnd && own) ? fsign(sb) : fsign(sa) + fsign(sb);
    } else if (L.ostats) {
        bnd = st.w != 0.0f;
        vp = st.x;
        const float own = L.sharp(ed);
        avgS = bnd ? st.y - own : st.y;
        cpre = bnd ? st.z - fsign(own) : st.z;
    } else {
        const RingStats r = creased_ring_walk(L, h);
        vp = r.valence; cpre = r.creaseCount; avgS = r.avgS; bnd = r.fwd < 0;
    }
    return coef_from_stats(vp, cpre, avgS, bnd, fsign(L.sharp(ed)), fsign(L.sharp(ped)));
}

// A lane's record of a quad level: twin, edge, vertex (one 16-byte load for
// 4-word records).
template <int RW>
__device__ __forceinline__ void lane_record(const QuadView<RW>& L, int64_t h64, int32_t& tw, int32_t& ed,
                                            int32_t& vx) {
    if constexpr (RW == 4) {
        const int4 r = __ldg(reinterpret_cast<const int4*>(L.he) + h64);
        tw = r.x; ed = r.y; vx = r.z;
    } else {
        tw = __ldg(L.he + 3 * h64 + 0);
        ed = __ldg(L.he + 3 * h64 + 1);
        vx = __ldg(L.he + 3 * h64 + 2);
    }
}
// Pass 1, tile of halfedges [h0, h0 + blockDim): each halfedge adds its
// side's terms cE(h) gV[v(h)] + dE(next h) gV[v(next h)] to gE[e] (next h is
// the quad's next lane) with one float atomic triple.
template <int RW>
__device__ __forceinline__ void adj_quad_edge_tile(const QuadView<RW>& L, float* __restrict__ gNew, int64_t h0) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, k = lane & 3, qb = lane & ~3, ln = qb | ((k + 1) & 3);
    const int lp = qb | ((k + 3) & 3);
    const int64_t h64 = h0 + threadIdx.x;
    const bool valid = h64 < L.H;
    const int32_t h = (int32_t)h64;
    const float* gV = gNew;
    float* gE = gNew + 3 * ((int64_t)L.V + L.F);
    int32_t tw = -1, ed = 0, vx = 0;
    float4 st = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    f3 g = zero3();
    if (valid) {
        lane_record(L, h64, tw, ed, vx);
        g = ld3(gV + 3 * (int64_t)vx);
        if (k == 0 && L.ostats) st = L.ostats[vx];
    }
    const int32_t ped = __shfl_sync(full, ed, lp), ptw = __shfl_sync(full, tw, lp);
    VCoef kc{0.0f, 0.0f, 0.0f, 0.0f};
    if (valid) kc = lane_vertex_coef(L, h, tw, ed, ptw, ped, st);
    const float dEn = __shfl_sync(full, kc.dE, ln);
    const f3 gn = shfl3(g, ln);
    if (valid) atomic_add3(gE + 3 * (int64_t)ed, add3(mul3(g, kc.cE), mul3(gn, dEn)));
}

// Pass 2, tile of halfedges: the face's gradient gF[f] + sum over its
// halfedges of bF gV[v] + ga gE[e] (reduced over the quad's lanes), then
// each halfedge's term of its vertex a gV[v] + al gE[e] + gF/4 + be(prev h)
// gE[e(prev h)], summed into gOld[v]: STRUCT (depth >= 2) a face centre's
// four terms in the warp (one writer), an edge midpoint's two per side and
// an older vertex's one by float atomics; depth 1 all by atomics.
template <int RW, bool STRUCT>
__device__ __forceinline__ void adj_quad_point_tile(const QuadView<RW>& L, const float* __restrict__ gNew,
                                                    float* __restrict__ gOld, int64_t h0) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, k = lane & 3, qb = lane & ~3, lp = qb | ((k + 3) & 3);
    const int64_t h64 = h0 + threadIdx.x;
    const bool valid = h64 < L.H;
    const int32_t h = (int32_t)h64;
    const float* gV = gNew;
    const float* gF = gNew + 3 * (int64_t)L.V;
    const float* gE = gNew + 3 * ((int64_t)L.V + L.F);
    int32_t tw = -1, ed = 0, vx = 0;
    float4 st = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    f3 gv = zero3(), ge = zero3(), gf = zero3();
    if (valid) {
        lane_record(L, h64, tw, ed, vx);
        gv = ld3(gV + 3 * (int64_t)vx);
        ge = ld3(gE + 3 * (int64_t)ed);
        if (k == 0) {
            gf = ld3(gF + 3 * (int64_t)(h >> 2));
            if (L.ostats) st = L.ostats[vx];
        }
    }
    const int32_t ped = __shfl_sync(full, ed, lp), ptw = __shfl_sync(full, tw, lp);
    VCoef kc{0.0f, 0.0f, 0.0f, 0.0f};
    ECoef ke{0.0f, 0.0f, 0.0f};
    if (valid) {
        kc = lane_vertex_coef(L, h, tw, ed, ptw, ped, st);
        const float w = fsat(L.sharp(ed)), b = tw < 0 ? 1.0f : 0.5f;    // edge_coef
        ke.al = (1.0f - w) * 0.25f + w * b * 0.5f;
        ke.be = w * b * 0.5f;
        ke.ga = (1.0f - w) * 0.25f;
    }
    f3 ft = add3(mul3(gv, kc.bF), mul3(ge, ke.ga));
    ft = add3(ft, shfl_xor3(ft, 1));
    ft = add3(ft, shfl_xor3(ft, 2));
    const f3 gFt = add3(shfl3(gf, qb), ft);
    const float bep = __shfl_sync(full, ke.be, lp);
    const f3 gep = shfl3(ge, lp);
    f3 s = add3(add3(mul3(gv, kc.a), mul3(ge, ke.al)), add3(mul3(gFt, 0.25f), mul3(gep, bep)));
    float* o = gOld + 3 * (int64_t)vx;
    if (STRUCT) {
        const f3 s4 = shfl_down3(s, 4), s8 = shfl_down3(s, 8), s12 = shfl_down3(s, 12);
        const int partner = (lane & ~15) | ((((lane >> 2) + 1) & 3) << 2) | 3;
        const f3 sA2 = shfl3(s, partner);
        if (!valid) return;
        if ((lane & 15) == 2) {
            const f3 t = add3(add3(s, s4), add3(s8, s12));
            o[0] += t.x;
            o[1] += t.y;
            o[2] += t.z;
        } else if (k == 1) {
            atomic_add3(o, add3(s, sA2));
        } else if (k == 0) {
            atomic_add3(o, s);
        }
    } else if (valid) {
        atomic_add3(o, s);
    }
}

// One pass for a quad level d >= 2 of the adjoint: the two-pass form's edge
// gradient (pass 1) is completed whole where it is needed instead of
// accumulated by atomics, and the vertex terms (pass 2) follow in the same
// thread.  For halfedge h with twin t:
//   gEt[e(h)] = gE[e] + cE(h) gV[v(h)] + dE(next h) gV[v(next h)]      (own side)
//                     + cE(t) gV[v(t)] + dE(next t) gV[v(next t)]      (twin t)
// with v(t) = v(next h), v(next t) = v(h).  The twin side (at depth >= 2 the
// twins of children 0, 1, 2, 3 of parent halfedge g are children 3, 2, 1, 0:
// CatmullClark.h:2778-2781):
//   * inside the parent quad (children 1, 2): the sibling face's own side;
//   * across a parent edge, child 0 of g (twin t = child 3 of next(twin g)):
//     cE(t) at the parent edge's midpoint, an interior vertex of valence 4
//     whose only creased edges are the parent edge's two halves; dE(next t)
//     at the older vertex v(h), non-zero only on a boundary in the crease
//     branch (the only case that reads next t's edge);
//   * child 3 of g (twin t = child 0 of twin(prev g)): cE(t) at the older
//     vertex v(next h) (its statistics, the boundary correction with t's
//     edge, which is h's); dE(next t) = 0, at the interior midpoint of
//     prev(g)'s edge.
// The vertex coefficients are lane_vertex_coef's with the statistics it
// would read known from the structure: child 2 sits at a face centre
// (valence 4), children 1 and 3 at edge midpoints whose creased edges are the
// halves of one parent edge, child 0 at an older vertex (its statistics).
// gE is read, not written.
// Where the adjoint step reads the gradients of depth d+1's points (index =
// the point's slot in the level: [vertices | faces | edges]): an array, or,
// for the finest level of a fitting loss, the difference P - T of the
// level's points and its target, formed as it is read.
struct GradArray {
    const float* __restrict__ g;
    __device__ __forceinline__ f3 at(int64_t i) const { return ld3(g + 3 * i); }
};
struct GradDistance {
    const float* __restrict__ p;
    const float* __restrict__ t;
    __device__ __forceinline__ f3 at(int64_t i) const {
        const f3 a = ld3(p + 3 * i), b = ld3(t + 3 * i);
        return f3{fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)};
    }
};

// The pass runs one thread per depth-d face: lane j of a quad of lanes
// takes face j of a parent quad (the structure k_level_fq relies on: face j
// runs C_j, M_j, Z, M_{j-1}; inner edge j = (j, 1) | (j+1, 2); the halves of
// parent edge j are (j, 0) and (j+1, 3)).  The terms above, per halfedge k
// of the face: coefficients kc(k), ke(k) and own(k) =
// cE(k) gV[v(k)] + dE(k+1) gV[v(k+1)]; the edge gradients
//   gEt(0) = gE + own(0) + cE(t) gV[M_j] + dE(next t) gV[C_j]  (across parent edge j)
//   gEt(1) = gE + own(1) + own(2) of the next lane              (inner edge j)
//   gEt(2) = gEt(1) of the previous lane                        (inner edge j-1)
//   gEt(3) = gE + own(3) + cB gV[C_j]                           (across parent edge j-1)
// then the face gradient gF + sum_k (bF(k) gV[v(k)] + ga(k) gEt(k)) and the
// four vertex terms a gV + al gEt + gF/4 + be(prev) gEt(prev): the corner's
// and midpoint M_j's pair (with the next lane's (j+1, 3) term) by float
// atomics, the centre's four by lane 0 of the quad.  Every coefficient and
// edge term is evaluated once per face (a layout with one halfedge per lane
// evaluates most of them in several lanes), with 15 shuffles per face.
__device__ __forceinline__ ECoef ecoef_of(float s, bool bnd) {
    const float w = fsat(s), b = bnd ? 1.0f : 0.5f;
    return ECoef{(1.0f - w) * 0.25f + w * b * 0.5f, w * b * 0.5f, (1.0f - w) * 0.25f};
}
template <int RW, class GradIn>
__device__ __forceinline__ void adj_face_step_tile(const QuadView<RW>& L, const GradIn gin,
                                                   float* __restrict__ gOld, int64_t f) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, qb = lane & ~3, j = lane & 3;
    const int ln = qb | ((j + 1) & 3), lp = qb | ((j + 3) & 3);
    const bool valid = f < ((int64_t)L.H >> 2);            // the four lanes of a quad agree
    const int64_t fBase = L.V, eBase = (int64_t)L.V + L.F;
    int4 r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = make_int4(-1, 0, 0, 0);
    if (valid) load_face_records<RW>(L.he, f, r);
    const int32_t tw0 = r[0].x, e0 = r[0].y, C = r[0].z;
    const int32_t e1 = r[1].y, Mj = r[1].z, Z = r[2].z;
    const int32_t tw3 = r[3].x, e3 = r[3].y, Mp = r[3].z;
    f3 gC = zero3(), gM = zero3(), gZ = zero3(), gMp = zero3(), ge0 = zero3(), ge1 = zero3(), ge3 = zero3(),
       gf = zero3();
    float4 st = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float s0 = 0.0f, s1 = 0.0f, s3 = 0.0f;
    if (valid) {
        gC = gin.at(C); gM = gin.at(Mj); gZ = gin.at(Z); gMp = gin.at(Mp);
        ge0 = gin.at(eBase + e0); ge1 = gin.at(eBase + e1); ge3 = gin.at(eBase + e3);
        gf = gin.at(fBase + f);
        st = L.ostats[C];
        s0 = L.sharp(e0); s1 = L.sharp(e1); s3 = L.sharp(e3);
    }
    // the other half of parent edge j is (j+1, 3), of parent edge j-1 is
    // (j-1, 0); the edge of (j, 2) is inner edge j-1
    const float s3n = __shfl_sync(full, s3, ln), s0p = __shfl_sync(full, s0, lp), s1p = __shfl_sync(full, s1, lp);
    const bool obnd = st.w != 0.0f;                      // the older vertex C_j's ring is open
    // vertex coefficients (lane_vertex_coef's cases) and edge coefficients
    const VCoef k0 = coef_from_stats(st.x, obnd ? st.z - fsign(s0) : st.z, obnd ? st.y - s0 : st.y, obnd,
                                     fsign(s0), fsign(s3));
    const VCoef k1 = coef_from_stats(tw0 < 0 ? 2.0f : 4.0f, fsign(s0) + fsign(s3n), s0 + s3n, tw0 < 0,
                                     fsign(s1), fsign(s0));
    const VCoef k2 = coef_from_stats(4.0f, 0.0f, 0.0f, false, fsign(s1p), fsign(s1));
    const VCoef k3 = coef_from_stats(tw3 < 0 ? 2.0f : 4.0f, tw3 < 0 ? fsign(s0p) : fsign(s3) + fsign(s0p),
                                     tw3 < 0 ? s0p : s3 + s0p, tw3 < 0, fsign(s3), fsign(s1p));
    const ECoef q0 = ecoef_of(s0, tw0 < 0), q1 = ecoef_of(s1, false), q2 = ecoef_of(s1p, false),
                q3 = ecoef_of(s3, tw3 < 0);
    // the edge gradients
    const f3 own2 = add3(mul3(gZ, k2.cE), mul3(gMp, k3.dE));
    f3 gEt1 = add3(add3(ge1, add3(mul3(gM, k1.cE), mul3(gZ, k2.dE))), shfl3(own2, ln));
    f3 gEt0 = add3(ge0, add3(mul3(gC, k0.cE), mul3(gM, k1.dE)));
    if (tw0 >= 0) {
        // cE(t) at the midpoint (interior, valence 4); dE(next t) at C_j,
        // non-zero only on an open ring in the crease branch
        const VCoef ct = coef_from_stats(4.0f, fsign(s0) + fsign(s3n), s0 + s3n, false, fsign(s0), 0.0f);
        float dEt = 0.0f;
        const float valence = obnd ? st.x + 1.0f : st.x;
        if (valid && obnd && !(st.z >= 3.0f || valence == 2.0f) && !(st.z <= 1.0f) && s0 != 0.0f) {
            const float sn = L.sharp(L.edge(tw0 & ~3));  // next(t) = child 0 of t's quad
            dEt = fsat((st.y - sn) * 0.5f) * 0.25f * fsign(s0);
        }
        gEt0 = add3(gEt0, add3(mul3(gM, ct.cE), mul3(gC, dEt)));
    }
    f3 gEt3 = add3(ge3, add3(mul3(gMp, k3.cE), mul3(gC, k0.dE)));
    if (tw3 >= 0) {
        // cE(t) at C_j seen from t, whose edge is (j, 3)'s
        const float cB = coef_from_stats(st.x, obnd ? st.z - fsign(s3) : st.z, obnd ? st.y - s3 : st.y, obnd,
                                         fsign(s3), 0.0f).cE;
        gEt3 = add3(gEt3, mul3(gC, cB));
    }
    const f3 gEt2 = shfl3(gEt1, lp);
    // the face gradient, then the four vertex terms
    f3 gFt = add3(gf, add3(mul3(gC, k0.bF), mul3(gEt0, q0.ga)));
    gFt = add3(gFt, add3(mul3(gM, k1.bF), mul3(gEt1, q1.ga)));
    gFt = add3(gFt, add3(mul3(gZ, k2.bF), mul3(gEt2, q2.ga)));
    gFt = add3(gFt, add3(mul3(gMp, k3.bF), mul3(gEt3, q3.ga)));
    const f3 gF4 = mul3(gFt, 0.25f);
    const f3 t0 = add3(add3(mul3(gC, k0.a), mul3(gEt0, q0.al)), add3(gF4, mul3(gEt3, q3.be)));
    const f3 t1 = add3(add3(mul3(gM, k1.a), mul3(gEt1, q1.al)), add3(gF4, mul3(gEt0, q0.be)));
    const f3 t2 = add3(add3(mul3(gZ, k2.a), mul3(gEt2, q2.al)), add3(gF4, mul3(gEt1, q1.be)));
    const f3 t3 = add3(add3(mul3(gMp, k3.a), mul3(gEt3, q3.al)), add3(gF4, mul3(gEt2, q2.be)));
    const f3 t3n = shfl3(t3, ln);
    const f3 c1 = shfl3(t2, qb + 1), c2 = shfl3(t2, qb + 2), c3 = shfl3(t2, qb + 3);
    // from depth 3, the corners shared inside a grandparent's 16-lane group
    // (fq_points): the grandparent centre's four terms added by one lane (no
    // other thread touches its slot), a grandparent midpoint's pair by one
    // atomic (depth 5 of the headline workload: 0.176 -> 0.171 ms)
    const bool agg = L.d >= 3;
    const int jq = (lane >> 2) & 3;
    const f3 u1 = add3(t0, shfl_xor3(t0, 4));
    const f3 u2 = add3(u1, shfl_xor3(u1, 8));
    const f3 pr = shfl3(t0, (lane & 16) | (((jq + 1) & 3) << 2) | 3);
    if (!valid) return;
    if (!agg || j == 0) {
        atomic_add3(gOld + 3 * (int64_t)C, t0);
    } else if (j == 1) {
        atomic_add3(gOld + 3 * (int64_t)C, add3(t0, pr));
    } else if (j == 2 && jq == 0) {
        float* o = gOld + 3 * (int64_t)C;
        o[0] += u2.x;
        o[1] += u2.y;
        o[2] += u2.z;
    }
    // (the midpoints of the grandparent's inner edges summed in the group as
    // fq_points does: 0.171 -> 0.176 ms here, so one atomic per pair)
    atomic_add3(gOld + 3 * (int64_t)Mj, add3(t1, t3n));
    if (j == 0) {
        const f3 t = add3(add3(t2, c1), add3(c2, c3));
        float* o = gOld + 3 * (int64_t)Z;
        o[0] += t.x;
        o[1] += t.y;
        o[2] += t.z;
    }
}


}  // namespace ccs
