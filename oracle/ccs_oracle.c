/*
 * ccs_oracle.c -- CPU oracle for Catmull-Clark halfedge refinement.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The CUDA library in halfedgecatmullclark_b200/ never links or calls it.
 *
 * It restates, as plain sequential C, the refinement rules of
 * jdupuy/HalfedgeCatmullClark's CatmullClark.h.  Each routine names the
 * reference lines it follows.  Floating-point expressions keep the
 * reference's operation order (build with -ffp-contract=off) so that the
 * FP32 build reproduces a single-threaded run of the reference bit for bit.
 *
 * The file is compiled twice:
 *   OR_REAL=float   -> liboracle32.so : the FP32 oracle
 *   OR_REAL=double  -> liboracle64.so : FP64 oracle of the same rule (points
 *                      in double; topology and crease sharpness are the FP32
 *                      values, so only point arithmetic differs).
 *
 * Parity pins: tests/test_oracle_pin.py compares this oracle with the
 * reference itself compiled from its sources into oracle/_ref/ (see
 * oracle/Makefile) and with the fixtures under tests/golden/.
 *
 * Beyond the reference, it holds the transposed (adjoint) point rules used
 * to check the CUDA adjoint; the reference has no adjoint.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>

#ifndef OR_REAL
#define OR_REAL float
#endif
typedef OR_REAL real;

/* ------------------------------------------------------------------------ */
/* Data layout (CatmullClark.h:17-71, :136-142)                              */
/* ------------------------------------------------------------------------ */
typedef struct { int32_t next, prev; float sharpness; } or_crease;          /* cc_Crease :30-34 */
typedef struct { int32_t twin, next, prev, face, edge, vertex, uv; } or_he; /* cc_Halfedge :37-45 */

typedef struct {
    int32_t V, U, H, E, F;
    const int32_t *v2h, *e2h, *f2h;
    const or_he *he;
    const or_crease *cr;
    const float *uvs;                /* U x 2 */
} or_cage;

/* A refined hierarchy: halfedge records of `stride` int32 words each
 * (4 = {twin, edge, vertex, uv}, 3 = no UV slot; :48-55), creases, points. */
typedef struct {
    const or_cage *cage;
    int32_t D;
    int32_t stride;
    int32_t *he;
    or_crease *cr;
    real *pts;                       /* sum_V x 3 */
} or_subd;

/* ------------------------------------------------------------------------ */
/* int32 arithmetic with the reference's wrap-around (two's complement)       */
/* ------------------------------------------------------------------------ */
static int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
static int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static int32_t wshl(int32_t a, int32_t s) { return (int32_t)((uint32_t)a << s); }
static int32_t ones(int32_t n) { return (int32_t)~(0xFFFFFFFFu << n); } /* 2^n - 1, :505 */

/* Count algebra: CatmullClark.h:465-585 */
int32_t or_H_at(const or_cage *c, int32_t d) { return wshl(c->H, d << 1); }           /* :523-528 */
int32_t or_C_at(const or_cage *c, int32_t d) { return wshl(c->E, d); }                /* :540-545 */
int32_t or_F_at(const or_cage *c, int32_t d)                                          /* :465-480 */
{
    return d == 0 ? c->F : wshl(c->H, (d - 1) << 1);
}
int32_t or_E_at(const or_cage *c, int32_t d)                                          /* :494-511 */
{
    if (d == 0) return c->E;
    return wshl(wadd(c->E << 1, wmul(ones(d), c->H)), d - 1);
}
int32_t or_V_at(const or_cage *c, int32_t d)                                          /* :563-585 */
{
    if (d == 0) return c->V;
    {
        const int32_t F1 = c->H, E1 = wadd(2 * c->E, c->H), V1 = c->V + c->E + c->F;
        const int32_t t = ones(d - 1);
        return wadd(V1, wmul(t, wadd(E1, wmul(t, F1))));
    }
}

/* Cumulative counts: CatmullClark.h:815-936 */
int32_t or_cumH(const or_cage *c, int32_t d)                                          /* :846-855 */
{
    const int32_t H1 = wshl(c->H, 2);
    return wmul(H1, ones(d << 1)) / 3;
}
int32_t or_cumC(const or_cage *c, int32_t d)                                          /* :873-882 */
{
    return wmul(wshl(c->E, 1), ones(d));
}
int32_t or_cumE(const or_cage *c, int32_t d)                                          /* :815-826 */
{
    const int32_t H1 = wshl(c->H, 2), E1 = wadd(wshl(c->E, 1), c->H), A = ones(d);
    return wmul(A, wsub(wadd(6 * E1, wmul(A, H1)), H1)) / 6;
}
int32_t or_cumV(const or_cage *c, int32_t d)                                          /* :897-912 */
{
    const int32_t F1 = c->H, E1 = wadd(2 * c->E, c->H), V1 = c->V + c->E + c->F;
    const int32_t A = ones(d);
    const int32_t B = (int32_t)((~(0xFFFFFFFFu << (d << 1))) / 3u);
    return wadd(wadd(wmul(A, wsub(E1, wshl(F1, 1))), wmul(B, F1)),
                wmul(d, wadd(wsub(F1, E1), V1)));
}
int32_t or_cumF(const or_cage *c, int32_t d) { return or_cumH(c, d) >> 2; }          /* :815-818 */

/* ------------------------------------------------------------------------ */
/* Scalar helpers (CatmullClark.h:295-392)                                   */
/* ------------------------------------------------------------------------ */
static real maxr(real x, real y) { return x > y ? x : y; }                   /* :300-303 */
static real minr(real x, real y) { return x < y ? x : y; }                   /* :295-298 */
static real satr(real x) { return maxr((real)0, minr(x, (real)1)); }         /* :305-308 */
static real signr(real x) { return x < 0 ? (real)-1 : (x > 0 ? (real)1 : (real)0); } /* :310-319 */
static float maxf(float x, float y) { return x > y ? x : y; }

static void lerp3(real *o, const real *x, const real *y, real u)           /* :321-338 */
{
    int i;
    for (i = 0; i < 3; ++i) o[i] = x[i] + u * (y[i] - x[i]);
}
static void mul3(real *o, const real *x, real y) { int i; for (i = 0; i < 3; ++i) o[i] = x[i] * y; }
static void add3(real *o, const real *x, const real *y) { int i; for (i = 0; i < 3; ++i) o[i] = x[i] + y[i]; }

/* UV codec (:374-392).  The float -> uint32 conversion follows what the
 * reference's x86-64 build does: truncate through a signed 64-bit integer. */
static float uv_decode1(uint32_t x) { return (float)(x & 0xFFFFu) / 65535.0f; }
static uint32_t f2u32(float x)
{
    if (!(x > -9.2e18f && x < 9.2e18f)) return 0u;
    return (uint32_t)(int64_t)x;
}
static int32_t uv_encode(float u, float v)
{
    const uint32_t a = f2u32(u * 65535.0f), b = f2u32(v * 65535.0f);
    return (int32_t)((a & 0xFFFFu) | ((b & 0xFFFFu) << 16));
}

/* Quad-level face arithmetic (:667-689) */
static int32_t qnext(int32_t h) { return (h & ~3) | ((h + 1) & 3); }
static int32_t qprev(int32_t h) { return (h & ~3) | ((h - 1) & 3); }

/* ------------------------------------------------------------------------ */
/* Accessors into the refined hierarchy (:986-1161)                          */
/* ------------------------------------------------------------------------ */
static int32_t *HE(const or_subd *s, int32_t d, int32_t h)                 /* :1064-1072 */
{
    return s->he + ((size_t)or_cumH(s->cage, d - 1) + (size_t)h) * (size_t)s->stride;
}
static const or_crease *CR(const or_subd *s, int32_t d, int32_t e)         /* :995-1003 */
{
    return &s->cr[(size_t)or_cumC(s->cage, d - 1) + (size_t)e];
}
static real *PT(const or_subd *s, int32_t d, int32_t v)                    /* :1154-1161 */
{
    return s->pts + 3 * ((size_t)or_cumV(s->cage, d - 1) + (size_t)v);
}
static float sharp_at(const or_subd *s, int32_t d, int32_t e)              /* :1011-1021 */
{
    return e < or_C_at(s->cage, d) ? CR(s, d, e)->sharpness : 0.0f;
}
static int32_t twin_at(const or_subd *s, int32_t d, int32_t h) { return HE(s, d, h)[0]; }
static int32_t edge_at(const or_subd *s, int32_t d, int32_t h) { return HE(s, d, h)[1]; }
static int32_t vert_at(const or_subd *s, int32_t d, int32_t h) { return HE(s, d, h)[2]; }

/* ------------------------------------------------------------------------ */
/* Halfedge refinement (:2693-2812)                                          */
/* ------------------------------------------------------------------------ */
static void write_children(int32_t *o, int32_t S, int32_t h, int32_t twin, int32_t prev,
                           int32_t next, int32_t face, int32_t edge, int32_t vert,
                           int32_t prevEdge, int32_t prevTwin, int32_t twinNext,
                           int32_t V, int32_t E, int32_t F)
{
    o[0 * S + 0] = wadd(wmul(4, twinNext), 3);
    o[1 * S + 0] = wadd(wmul(4, next), 2);
    o[2 * S + 0] = wadd(wmul(4, prev), 1);
    o[3 * S + 0] = wmul(4, prevTwin);
    o[0 * S + 1] = 2 * edge + (h > twin ? 0 : 1);
    o[1 * S + 1] = 2 * E + h;
    o[2 * S + 1] = 2 * E + prev;
    o[3 * S + 1] = 2 * prevEdge + (prev > prevTwin ? 1 : 0);
    o[0 * S + 2] = vert;
    o[1 * S + 2] = V + F + edge;
    o[2 * S + 2] = V + face;
    o[3 * S + 2] = V + F + prevEdge;
}

void or_refine_halfedges(or_subd *s)                                        /* :2803-2812 */
{
    const or_cage *c = s->cage;
    int32_t h, d;

    /* cage level, :2693-2740 */
    for (h = 0; h < c->H; ++h) {
        const or_he *r = &c->he[h];
        const int32_t twinNext = r->twin >= 0 ? c->he[r->twin].next : -1;
        write_children(s->he + (size_t)4 * h * s->stride, s->stride, h, r->twin, r->prev,
                       r->next, r->face, r->edge, r->vertex, c->he[r->prev].edge,
                       c->he[r->prev].twin, twinNext, c->V, c->E, c->F);
    }
    /* quad levels, :2749-2796 */
    for (d = 1; d < s->D; ++d) {
        const int32_t Hd = or_H_at(c, d), V = or_V_at(c, d), E = or_E_at(c, d), F = or_F_at(c, d);
        int32_t *out = s->he + (size_t)or_cumH(c, d) * s->stride;
        for (h = 0; h < Hd; ++h) {
            const int32_t twin = twin_at(s, d, h), prev = qprev(h);
            write_children(out + (size_t)4 * h * s->stride, s->stride, h, twin, prev, qnext(h),
                           h >> 2, edge_at(s, d, h), vert_at(s, d, h), edge_at(s, d, prev),
                           twin_at(s, d, prev), qnext(twin), V, E, F);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Crease refinement (:2950-3042)                                            */
/* ------------------------------------------------------------------------ */
static void refine_crease(or_crease *out, int32_t e, const or_crease *in)
{
    const or_crease *me = &in[e];
    const int32_t nx = me->next, pv = me->prev;
    const int t1 = in[nx].prev == e && nx != e;
    const int t2 = in[pv].next == e && pv != e;
    const float thisS = 3.0f * me->sharpness;
    const float nextS = in[nx].sharpness, prevS = in[pv].sharpness;

    out[0].next = 2 * e + 1;
    out[1].next = 2 * nx + (t1 ? 0 : 1);
    out[0].prev = 2 * pv + (t2 ? 1 : 0);
    out[1].prev = 2 * e + 0;
    out[0].sharpness = maxf(0.0f, (prevS + thisS) / 4.0f - 1.0f);
    out[1].sharpness = maxf(0.0f, (thisS + nextS) / 4.0f - 1.0f);
}

void or_refine_creases(or_subd *s)                                          /* :3033-3042 */
{
    const or_cage *c = s->cage;
    int32_t e, d;

    for (e = 0; e < c->E; ++e) refine_crease(&s->cr[2 * (size_t)e], e, c->cr);  /* :2950-2983 */
    for (d = 1; d < s->D; ++d) {                                                 /* :2992-3026 */
        const int32_t Cd = or_C_at(c, d);
        const or_crease *in = &s->cr[or_cumC(c, d - 1)];
        or_crease *out = &s->cr[or_cumC(c, d)];
        for (e = 0; e < Cd; ++e) refine_crease(&out[2 * (size_t)e], e, in);
    }
}

/* ------------------------------------------------------------------------ */
/* UV refinement (:2825-2939)                                                */
/* ------------------------------------------------------------------------ */
void or_refine_uvs(or_subd *s)
{
    const or_cage *c = s->cage;
    const int32_t S = s->stride;
    int32_t h, d;

    if (c->U <= 0 || S < 4) return;                                          /* :2930 */
    for (h = 0; h < c->H; ++h) {                                             /* :2825-2869 */
        const or_he *r = &c->he[h];
        const float *uv = &c->uvs[2 * (size_t)r->uv];
        const float *nu = &c->uvs[2 * (size_t)c->he[r->next].uv];
        const float *pu = &c->uvs[2 * (size_t)c->he[r->prev].uv];
        float fu = uv[0], fv = uv[1], eu, ev, pu_, pv_;
        int32_t m = 1, it;
        int32_t *o = s->he + (size_t)4 * h * S;

        eu = uv[0] + 0.5f * (nu[0] - uv[0]);
        ev = uv[1] + 0.5f * (nu[1] - uv[1]);
        pu_ = uv[0] + 0.5f * (pu[0] - uv[0]);
        pv_ = uv[1] + 0.5f * (pu[1] - uv[1]);
        for (it = r->next; it != h; it = c->he[it].next) {
            const float *q = &c->uvs[2 * (size_t)c->he[it].uv];
            fu += q[0];
            fv += q[1];
            ++m;
        }
        fu /= (float)m;
        fv /= (float)m;
        o[0 * S + 3] = uv_encode(uv[0], uv[1]);
        o[1 * S + 3] = uv_encode(eu, ev);
        o[2 * S + 3] = uv_encode(fu, fv);
        o[3 * S + 3] = uv_encode(pu_, pv_);
    }
    for (d = 1; d < s->D; ++d) {                                             /* :2878-2921 */
        const int32_t Hd = or_H_at(c, d);
        int32_t *out = s->he + (size_t)or_cumH(c, d) * S;
        for (h = 0; h < Hd; ++h) {
            const uint32_t code = (uint32_t)HE(s, d, h)[3];
            const uint32_t cn = (uint32_t)HE(s, d, qnext(h))[3];
            const uint32_t cp = (uint32_t)HE(s, d, qprev(h))[3];
            const float u = uv_decode1(code), v = uv_decode1(code >> 16);
            const float nu = uv_decode1(cn), nv = uv_decode1(cn >> 16);
            const float pu = uv_decode1(cp), pv = uv_decode1(cp >> 16);
            float fu = u, fv = v;
            int32_t it;
            int32_t *o = out + (size_t)4 * h * S;

            for (it = qnext(h); it != h; it = qnext(it)) {
                const uint32_t q = (uint32_t)HE(s, d, it)[3];
                fu += uv_decode1(q);
                fv += uv_decode1(q >> 16);
            }
            fu /= 4.0f;
            fv /= 4.0f;
            o[0 * S + 3] = (int32_t)code;
            o[1 * S + 3] = uv_encode(u + 0.5f * (nu - u), v + 0.5f * (nv - v));
            o[2 * S + 3] = uv_encode(fu, fv);
            o[3 * S + 3] = uv_encode(u + 0.5f * (pu - u), v + 0.5f * (pv - v));
        }
    }
}

void or_refine_topology(or_subd *s)                                         /* :3051-3058 */
{
    or_refine_halfedges(s);
    or_refine_creases(s);
    or_refine_uvs(s);
}

/* ------------------------------------------------------------------------ */
/* Per-level view used by the point rules: a level is either the cage        */
/* (d == 0) or quad level d of the hierarchy.                                */
/* ------------------------------------------------------------------------ */
typedef struct {
    const or_subd *s;
    int32_t d;
    int32_t V, F, E, H, C;
    const real *old;      /* V x 3 : level-d points                      */
    real *out;            /* V_{d+1} x 3 : [old vertices | faces | edges] */
} lvl;

static void lvl_init(lvl *L, const or_subd *s, int32_t d, const real *cagePts)
{
    const or_cage *c = s->cage;
    L->s = s;
    L->d = d;
    L->V = or_V_at(c, d);
    L->F = or_F_at(c, d);
    L->E = or_E_at(c, d);
    L->H = or_H_at(c, d);
    L->C = or_C_at(c, d);
    L->old = d == 0 ? cagePts : PT(s, d, 0);
    L->out = s->pts + 3 * (size_t)or_cumV(c, d);
}
static int32_t L_twin(const lvl *L, int32_t h) { return L->d ? twin_at(L->s, L->d, h) : L->s->cage->he[h].twin; }
static int32_t L_next(const lvl *L, int32_t h) { return L->d ? qnext(h) : L->s->cage->he[h].next; }
static int32_t L_prev(const lvl *L, int32_t h) { return L->d ? qprev(h) : L->s->cage->he[h].prev; }
static int32_t L_face(const lvl *L, int32_t h) { return L->d ? (h >> 2) : L->s->cage->he[h].face; }
static int32_t L_edge(const lvl *L, int32_t h) { return L->d ? edge_at(L->s, L->d, h) : L->s->cage->he[h].edge; }
static int32_t L_vert(const lvl *L, int32_t h) { return L->d ? vert_at(L->s, L->d, h) : L->s->cage->he[h].vertex; }
static real L_esharp(const lvl *L, int32_t e)
{
    return (real)(L->d ? sharp_at(L->s, L->d, e) : L->s->cage->cr[e].sharpness);
}
static real L_hsharp(const lvl *L, int32_t h) { return L_esharp(L, L_edge(L, h)); }
static const real *L_pt(const lvl *L, int32_t v) { return &L->old[3 * (size_t)v]; }
static real *L_fpt(const lvl *L, int32_t f) { return &L->out[3 * ((size_t)L->V + f)]; }
static real *L_ept(const lvl *L, int32_t e) { return &L->out[3 * ((size_t)L->V + L->F + e)]; }
static real *L_vpt(const lvl *L, int32_t v) { return &L->out[3 * (size_t)v]; }
/* (twin(h) >= 0 ? next(twin(h)) : -1) on the cage (:744-749); the quad
 * levels apply next to the twin unconditionally (:1168-1175). */
static int32_t L_next_vertex_he(const lvl *L, int32_t h)
{
    const int32_t t = L_twin(L, h);
    if (L->d) return qnext(t);
    return t >= 0 ? L->s->cage->he[t].next : -1;
}
static int32_t L_prev_vertex_he(const lvl *L, int32_t h) { return L_twin(L, L_prev(L, h)); }

/* ------------------------------------------------------------------------ */
/* Scatter point rules (:1437-1463, :1517-1548, :1602-1648, :1713-1756,      */
/* :1872-1991, :2032-2052, :2107-2139, :2194-2241, :2307-2351, :2496-2615). */
/* Loops run in halfedge order, i.e. the order a one-thread reference run    */
/* applies its atomics in.                                                   */
/* ------------------------------------------------------------------------ */
static void face_points_scatter(const lvl *L)
{
    int32_t h, i;
    for (h = 0; h < L->H; ++h) {
        const real *p = L_pt(L, L_vert(L, h));
        real *f = L_fpt(L, L_face(L, h));
        if (L->d == 0) {                                                     /* :1437-1463 */
            float n = 1.0f;
            int32_t it;
            for (it = L_next(L, h); it != h; it = L_next(L, it)) ++n;
            for (i = 0; i < 3; ++i) f[i] += p[i] / (real)n;
        } else {                                                             /* :2032-2052 */
            for (i = 0; i < 3; ++i) f[i] += p[i] / (real)4.0f;
        }
    }
}

static void creased_edge_points_scatter(const lvl *L)                       /* :1602-1648, :2194-2241 */
{
    int32_t h, i;
    for (h = 0; h < L->H; ++h) {
        const int32_t twin = L_twin(L, h), e = L_edge(L, h);
        const real w = satr(L_esharp(L, e));
        const real *f = L_fpt(L, L_face(L, h));
        const real *v0 = L_pt(L, L_vert(L, h)), *v1 = L_pt(L, L_vert(L, L_next(L, h)));
        real tmp[3], sharp[3], smooth[3], aw[3];
        lerp3(tmp, v0, v1, (real)0.5f);
        mul3(sharp, tmp, twin < 0 ? (real)1.0f : (real)0.5f);
        lerp3(tmp, v0, f, (real)0.5f);
        mul3(smooth, tmp, (real)0.5f);
        lerp3(aw, smooth, sharp, w);
        for (i = 0; i < 3; ++i) L_ept(L, e)[i] += aw[i];
    }
}

static void edge_points_scatter(const lvl *L)                               /* :1517-1548, :2107-2139 */
{
    int32_t h, i;
    for (h = 0; h < L->H; ++h) {
        const int32_t twin = L_twin(L, h), e = L_edge(L, h);
        const real *f = L_fpt(L, L_face(L, h));
        const real *v0 = L_pt(L, L_vert(L, h)), *v1 = L_pt(L, L_vert(L, L_next(L, h)));
        const real w = twin >= 0 ? (real)0.5f : (real)1.0f;
        real t1[3], t2[3], t3[3], t4[3], aw[3];
        mul3(t1, f, (real)0.5f);
        mul3(t2, v0, w);
        mul3(t3, v1, w);
        lerp3(t4, t2, t3, (real)0.5f);
        lerp3(aw, t1, t4, w);
        for (i = 0; i < 3; ++i) L_ept(L, e)[i] += aw[i];
    }
}

/* Ring statistics of the creased vertex rule as seen from halfedge h
 * (:1899-1936 on the cage, :2523-2566 on quad levels). */
typedef struct { real avgS, creaseCount, valence; int32_t fwd; } ring_stats;

static ring_stats creased_ring(const lvl *L, int32_t h)
{
    ring_stats r;
    const int32_t prev = L_prev(L, h);
    const real prevS = L_hsharp(L, prev);
    int32_t fwd, bwd;

    r.avgS = prevS;
    r.creaseCount = signr(prevS);
    r.valence = 1;
    for (fwd = L_twin(L, prev); fwd >= 0 && fwd != h; fwd = L_twin(L, fwd)) {
        const int32_t p = L_prev(L, fwd);
        const real s = L_hsharp(L, p);
        ++r.valence;
        r.avgS += s;
        r.creaseCount += signr(s);
        fwd = p;
    }
    for (bwd = L_twin(L, h); fwd < 0 && bwd >= 0 && bwd != h; bwd = L_twin(L, bwd)) {
        const int32_t n = L_next(L, bwd);
        const real s = L_hsharp(L, n);
        ++r.valence;
        r.avgS += s;
        r.creaseCount += signr(s);
        bwd = n;
    }
    r.fwd = fwd;
    return r;
}

/* Contribution of halfedge h to its vertex under the creased scatter rule.
 * cornerFirst selects the branch order of the quad levels (:2598-2607);
 * the cage uses smooth-first (:1974-1983). */
static void creased_vertex_contrib(const lvl *L, int32_t h, int cornerFirst, real *aw)
{
    const ring_stats r = creased_ring(L, h);
    const int32_t prev = L_prev(L, h);
    const real thisS = L_hsharp(L, h), prevS = L_hsharp(L, prev);
    const real cw = signr(thisS), pcw = signr(prevS);
    const real *E = L_ept(L, L_edge(L, h)), *Ep = L_ept(L, L_edge(L, prev));
    const real *F = L_fpt(L, L_face(L, h)), *P = L_pt(L, L_vert(L, h));
    real corner[3], smooth[3], crease[3], t1[3], t2[3];
    real valence = r.valence, creaseCount = r.creaseCount;
    const real avgS = r.avgS;

    mul3(corner, P, (real)1.0f / valence);
    mul3(t1, P, (real)0.25f * cw);
    mul3(t2, E, (real)0.25f * cw);
    add3(crease, t1, t2);
    mul3(t1, F, (real)-1.0f);
    mul3(t2, E, (real)+4.0f);
    add3(smooth, t1, t2);
    mul3(t1, P, valence - (real)3.0f);
    add3(smooth, smooth, t1);
    mul3(smooth, smooth, (real)1.0f / (valence * valence));
    if (r.fwd < 0) {
        creaseCount += cw;
        ++valence;
        mul3(t1, P, (real)0.25f * pcw);
        mul3(t2, Ep, (real)0.25f * pcw);
        add3(t1, t1, t2);
        add3(crease, crease, t1);
    }
    if (cornerFirst) {
        if (creaseCount >= (real)3.0f || valence == (real)2.0f) memcpy(aw, corner, sizeof corner);
        else if (creaseCount <= (real)1.0f) memcpy(aw, smooth, sizeof smooth);
        else lerp3(aw, corner, crease, satr(avgS * (real)0.5f));
    } else {
        if (creaseCount <= (real)1.0f) memcpy(aw, smooth, sizeof smooth);
        else if (creaseCount >= (real)3.0f || valence == (real)2.0f) memcpy(aw, corner, sizeof corner);
        else lerp3(aw, corner, crease, satr(avgS * (real)0.5f));
    }
}

static void creased_vertex_points_scatter(const lvl *L)
{
    int32_t h, i;
    real aw[3];
    for (h = 0; h < L->H; ++h) {
        creased_vertex_contrib(L, h, L->d > 0, aw);
        for (i = 0; i < 3; ++i) L_vpt(L, L_vert(L, h))[i] += aw[i];
    }
}

static void vertex_points_scatter(const lvl *L)                             /* :1713-1756, :2307-2351 */
{
    int32_t h, i;
    for (h = 0; h < L->H; ++h) {
        const int32_t v = L_vert(L, h), e = L_edge(L, h), f = L_face(L, h);
        int32_t valence = 1, fwd, bwd;
        for (fwd = L_prev_vertex_he(L, h); fwd >= 0 && fwd != h; fwd = L_prev_vertex_he(L, fwd)) ++valence;
        for (bwd = L_next_vertex_he(L, h); fwd < 0 && bwd >= 0 && bwd != h; bwd = L_next_vertex_he(L, bwd)) ++valence;
        for (i = 0; i < 3; ++i) {
            const real w = (real)1.0f / (real)valence;
            const real pv = L_pt(L, v)[i], pf = L_fpt(L, f)[i], pe = L_ept(L, e)[i];
            const real s = fwd < 0 ? (real)0.0f : (real)1.0f;
            L_vpt(L, v)[i] += w * (pv + w * s * ((real)4.0f * pe - pf - (real)3.0f * pv));
        }
    }
}

static void clear_points(or_subd *s)                                        /* :2623-2629 */
{
    memset(s->pts, 0, sizeof(real) * 3 * (size_t)or_cumV(s->cage, s->D));
}

void or_refine_points_scatter(or_subd *s, const real *cagePts)             /* :2631-2643 */
{
    int32_t d;
    clear_points(s);
    for (d = 0; d < s->D; ++d) {
        lvl L;
        lvl_init(&L, s, d, cagePts);
        face_points_scatter(&L);
        creased_edge_points_scatter(&L);
        creased_vertex_points_scatter(&L);
    }
}

/* One step d -> d+1 of the scatter rules (the loop body of :2631-2643 or
 * :2645-2657) on the level-d points already in s->pts (d = 0: cagePts):
 * level d+1's rows are cleared and recomputed.  With it a test holds one
 * step of a float-atomic pass to the reference's arithmetic, on the level-d
 * points that pass produced itself. */
void or_step_points_scatter(or_subd *s, int32_t d, int32_t creased, const real *cagePts)
{
    lvl L;
    lvl_init(&L, s, d, cagePts);
    memset(L.out, 0, sizeof(real) * 3 * (size_t)or_V_at(s->cage, d + 1));
    face_points_scatter(&L);
    if (creased) {
        creased_edge_points_scatter(&L);
        creased_vertex_points_scatter(&L);
    } else {
        edge_points_scatter(&L);
        vertex_points_scatter(&L);
    }
}

void or_refine_points_nocreases_scatter(or_subd *s, const real *cagePts)   /* :2645-2657 */
{
    int32_t d;
    clear_points(s);
    for (d = 0; d < s->D; ++d) {
        lvl L;
        lvl_init(&L, s, d, cagePts);
        face_points_scatter(&L);
        edge_points_scatter(&L);
        vertex_points_scatter(&L);
    }
}

/* ------------------------------------------------------------------------ */
/* O(depth) maps used by the gather rules (:1206-1395)                        */
/* ------------------------------------------------------------------------ */
static int32_t edge_to_he_first(const or_cage *c, int32_t e)               /* :1206-1227 */
{
    if (e >= 2 * c->E) {
        const int32_t h = e - 2 * c->E, n = c->he[h].next;
        const int32_t a = 4 * h + 1, b = 4 * n + 2;
        return a > b ? a : b;
    } else if (e & 1) {
        return 4 * c->he[c->e2h[e >> 1]].next + 3;
    }
    return 4 * c->e2h[e >> 1] + 0;
}

int32_t or_edge_to_halfedge(const or_cage *c, int32_t e, int32_t d)        /* :1229-1303 */
{
    uint32_t heap = 1u;
    int32_t id = 0, hd = d;
    for (; hd > 1; --hd) {
        const int32_t Ec = or_E_at(c, hd - 1);
        if (e >= 2 * Ec) {
            const int32_t h = e - 2 * Ec, n = qnext(h);
            const int32_t a = 4 * h + 1, b = 4 * n + 2;
            id = a > b ? a : b;
            break;
        }
        heap = (heap << 1) | (uint32_t)(e & 1);
        e >>= 1;
    }
    if (hd == 1) id = edge_to_he_first(c, e);
    while (heap > 1u) {
        id = (heap & 1u) ? 4 * qnext(id) + 3 : 4 * id + 0;
        heap >>= 1;
    }
    return id;
}

static int32_t vertex_to_he_first(const or_cage *c, int32_t v)             /* :1313-1333 */
{
    if (v >= c->V + c->F) return 4 * c->e2h[v - c->V - c->F] + 1;
    if (v >= c->V) return 4 * c->f2h[v - c->V] + 2;
    return 4 * c->v2h[v] + 0;
}

int32_t or_vertex_to_halfedge(const or_cage *c, int32_t v, int32_t d)      /* :1335-1395 */
{
    int32_t hd = d, stride = 0, h = 0;
    for (; hd > 1; --hd) {
        const int32_t Vc = or_V_at(c, hd - 1), Fc = or_F_at(c, hd - 1);
        if (v >= Vc + Fc) {
            h = 4 * or_edge_to_halfedge(c, v - Fc - Vc, hd - 1) + 1;
            break;
        } else if (v >= Vc) {
            h = 4 * (4 * (v - Vc)) + 2;
            break;
        }
        stride += 2;
    }
    if (hd == 1) h = vertex_to_he_first(c, v);
    return h << stride;
}

/* Level-generic edge / vertex -> halfedge lookups for the gather rules. */
static int32_t L_edge_he(const lvl *L, int32_t e)
{
    return L->d ? or_edge_to_halfedge(L->s->cage, e, L->d) : L->s->cage->e2h[e];
}
static int32_t L_vert_he(const lvl *L, int32_t v)
{
    return L->d ? or_vertex_to_halfedge(L->s->cage, v, L->d) : L->s->cage->v2h[v];
}

/* ------------------------------------------------------------------------ */
/* Gather point rules (:1408-1435, :1476-1515, :1561-1600, :1661-1711,       */
/* :1769-1869, :2004-2030, :2065-2105, :2151-2191, :2254-2305, :2364-2493)  */
/* ------------------------------------------------------------------------ */
static void face_points_gather(const lvl *L)
{
    int32_t f;
    for (f = 0; f < L->F; ++f) {
        const int32_t h = L->d ? 4 * f : L->s->cage->f2h[f];
        real acc[3];
        float n = 1.0f;
        int32_t it;
        memcpy(acc, L_pt(L, L_vert(L, h)), sizeof acc);
        for (it = L_next(L, h); it != h; it = L_next(L, it)) {
            add3(acc, acc, L_pt(L, L_vert(L, it)));
            ++n;
        }
        mul3(L_fpt(L, f), acc, L->d ? (real)0.25f : (real)(1.0f / n));
    }
}

static void edge_points_gather(const lvl *L, int creased)
{
    int32_t e;
    for (e = 0; e < L->E; ++e) {
        const int32_t h = L_edge_he(L, e), twin = L_twin(L, h), n = L_next(L, h);
        const real w = creased ? satr(L_esharp(L, e)) : (twin < 0 ? (real)0 : (real)1);
        const real *v0 = L_pt(L, L_vert(L, h)), *v1 = L_pt(L, L_vert(L, n));
        const real *f0 = L_fpt(L, L_face(L, h)), *f1 = L_fpt(L, L_face(L, twin > 0 ? twin : 0));
        real t1[3], t2[3], sharp[3], smooth[3];
        add3(t1, v0, v1);
        add3(t2, f0, f1);
        mul3(sharp, t1, (real)0.5f);
        add3(smooth, t1, t2);
        mul3(smooth, smooth, (real)0.25f);
        if (creased) lerp3(L_ept(L, e), smooth, sharp, w);                     /* :1561-1600, :2151-2191 */
        else lerp3(L_ept(L, e), sharp, smooth, w);                              /* :1476-1515, :2065-2105 */
    }
}

static void vertex_points_gather(const lvl *L)                              /* :1661-1711, :2254-2305 */
{
    int32_t v;
    for (v = 0; v < L->V; ++v) {
        const int32_t h = L_vert_he(L, v);
        const real *E = L_ept(L, L_edge(L, h)), *F = L_fpt(L, L_face(L, h)), *P = L_pt(L, v);
        real smooth[3], t1[3], t2[3];
        real valence = 1;
        int32_t it;
        mul3(t1, F, (real)-1.0f);
        mul3(t2, E, (real)+4.0f);
        add3(smooth, t1, t2);
        for (it = L_prev_vertex_he(L, h); it >= 0 && it != h; it = L_prev_vertex_he(L, it)) {
            mul3(t1, L_fpt(L, L_face(L, it)), (real)-1.0f);
            mul3(t2, L_ept(L, L_edge(L, it)), (real)+4.0f);
            add3(smooth, smooth, t1);
            add3(smooth, smooth, t2);
            ++valence;
        }
        mul3(t1, smooth, (real)1.0f / (valence * valence));
        mul3(t2, P, (real)1.0f - (real)3.0f / valence);
        add3(smooth, t1, t2);
        lerp3(L_vpt(L, v), P, smooth, it != h ? (real)0.0f : (real)1.0f);
    }
}

static void creased_vertex_points_gather(const lvl *L)                      /* :1769-1869, :2364-2493 */
{
    int32_t v;
    for (v = 0; v < L->V; ++v) {
        const int32_t h = L_vert_he(L, v), e = L_edge(L, h), prev = L_prev(L, h);
        const real thisS = L_hsharp(L, h), prevS = L_hsharp(L, prev);
        const real cw = signr(thisS), pcw = signr(prevS);
        const real *E = L_ept(L, e), *Ep = L_ept(L, L_edge(L, prev));
        const real *Fp = L_fpt(L, L_face(L, prev)), *P = L_pt(L, v);
        real smooth[3], crease[3] = {0, 0, 0}, t1[3], t2[3];
        real avgS = prevS, creaseCount = pcw, valence = 1;
        int32_t fwd, bwd;

        mul3(t1, Fp, (real)-1.0f);
        mul3(t2, Ep, (real)+4.0f);
        add3(smooth, t1, t2);
        mul3(t1, Ep, pcw);
        add3(crease, crease, t1);
        for (fwd = L_twin(L, prev); fwd >= 0 && fwd != h; fwd = L_twin(L, fwd)) {
            const int32_t p = L_prev(L, fwd);
            const real s = L_hsharp(L, p), w = signr(s);
            const real *Ei = L_ept(L, L_edge(L, p)), *Fi = L_fpt(L, L_face(L, p));
            mul3(t1, Fi, (real)-1.0f);
            mul3(t2, Ei, (real)+4.0f);
            add3(smooth, smooth, t1);
            add3(smooth, smooth, t2);
            ++valence;
            mul3(t1, Ei, w);
            add3(crease, crease, t1);
            avgS += s;
            creaseCount += w;
            fwd = p;
        }
        /* the quad-level gather also walks backwards from a boundary
         * (:2424-2451); the cage gather does not (:1799-1827) */
        for (bwd = L_twin(L, h); L->d && fwd < 0 && bwd >= 0 && bwd != h; bwd = L_twin(L, bwd)) {
            const int32_t n = L_next(L, bwd);
            const real s = L_hsharp(L, n), w = signr(s);
            const real *Ei = L_ept(L, L_edge(L, n)), *Fi = L_fpt(L, L_face(L, n));
            mul3(t1, Fi, (real)-1.0f);
            mul3(t2, Ei, (real)+4.0f);
            add3(smooth, smooth, t1);
            add3(smooth, smooth, t2);
            ++valence;
            mul3(t1, Ei, w);
            add3(crease, crease, t1);
            avgS += s;
            creaseCount += w;
            bwd = n;
        }
        if (fwd < 0) {
            mul3(t1, E, cw);
            add3(crease, crease, t1);
            creaseCount += cw;
            ++valence;
        }
        mul3(t1, smooth, (real)1.0f / (valence * valence));
        mul3(t2, P, (real)1.0f - (real)3.0f / valence);
        add3(smooth, t1, t2);
        mul3(t1, crease, L->d ? (real)0.5f / creaseCount : (real)0.25f);
        mul3(t2, P, (real)0.5f);
        add3(crease, t1, t2);
        if (creaseCount <= (real)1.0f) memcpy(L_vpt(L, v), smooth, sizeof smooth);
        else if (creaseCount >= (real)3.0f || valence == (real)2.0f) memcpy(L_vpt(L, v), P, 3 * sizeof(real));
        else lerp3(L_vpt(L, v), P, crease, satr(avgS * (real)0.5f));
    }
}

void or_refine_points_gather(or_subd *s, const real *cagePts)              /* :2659-2670 */
{
    int32_t d;
    for (d = 0; d < s->D; ++d) {
        lvl L;
        lvl_init(&L, s, d, cagePts);
        face_points_gather(&L);
        edge_points_gather(&L, 1);
        creased_vertex_points_gather(&L);
    }
}

void or_refine_points_nocreases_gather(or_subd *s, const real *cagePts)    /* :2672-2683 */
{
    int32_t d;
    for (d = 0; d < s->D; ++d) {
        lvl L;
        lvl_init(&L, s, d, cagePts);
        face_points_gather(&L);
        edge_points_gather(&L, 0);
        vertex_points_gather(&L);
    }
}

/* ------------------------------------------------------------------------ */
/* Adjoint of the creased scatter rule (no reference counterpart).           */
/*                                                                           */
/* For fixed topology and sharpness, level d+1 points are linear in level d  */
/* points.  Per halfedge h (n = face size, vp = valence before the boundary  */
/* correction, bnd = walk hit a boundary):                                   */
/*   F[f]   += P[v(h)] / n                                                   */
/*   E[e(h)]+= al P[v(h)] + be P[v(next h)] + ga F[f(h)]                     */
/*            al = (1-w)/4 + w*b/2, be = w*b/2, ga = (1-w)/4,                */
/*            w = sat(s_e), b = 1 on a boundary edge else 1/2                */
/*   V'[v]  += a P[v] + bF F[f(h)] + cE E[e(h)] + dE E[e(prev h)]            */
/*            corner: a = 1/vp; smooth: a = (vp-3)/vp^2, bF = -1/vp^2,       */
/*            cE = 4/vp^2; crease blend t: a = (1-t)/vp + t/4 (cw + bnd pcw), */
/*            cE = t cw/4, dE = t bnd pcw/4.                                  */
/* The adjoint applies the transposes in reverse pass order.                */
/* ------------------------------------------------------------------------ */
typedef struct { real a, bF, cE, dE; } vcoef;

static vcoef creased_vertex_coef(const lvl *L, int32_t h)
{
    const ring_stats r = creased_ring(L, h);
    const int32_t prev = L_prev(L, h);
    const real cw = signr(L_hsharp(L, h)), pcw = signr(L_hsharp(L, prev));
    const real vp = r.valence;
    const int bnd = r.fwd < 0;
    const real valence = bnd ? vp + 1 : vp;
    const real creaseCount = bnd ? r.creaseCount + cw : r.creaseCount;
    const int cornerFirst = L->d > 0;
    vcoef k = {0, 0, 0, 0};
    int branch; /* 0 corner, 1 smooth, 2 blend */

    if (cornerFirst) {
        if (creaseCount >= 3 || valence == 2) branch = 0;
        else if (creaseCount <= 1) branch = 1;
        else branch = 2;
    } else {
        if (creaseCount <= 1) branch = 1;
        else if (creaseCount >= 3 || valence == 2) branch = 0;
        else branch = 2;
    }
    if (branch == 0) {
        k.a = (real)1 / vp;
    } else if (branch == 1) {
        k.a = (vp - 3) / (vp * vp);
        k.bF = (real)-1 / (vp * vp);
        k.cE = (real)4 / (vp * vp);
    } else {
        const real t = satr(r.avgS * (real)0.5f);
        k.a = (1 - t) / vp + t * (real)0.25f * (cw + (bnd ? pcw : 0));
        k.cE = t * (real)0.25f * cw;
        k.dE = bnd ? t * (real)0.25f * pcw : 0;
    }
    return k;
}

static int32_t L_face_size(const lvl *L, int32_t h)
{
    int32_t n = 1, it;
    if (L->d) return 4;
    for (it = L_next(L, h); it != h; it = L_next(L, it)) ++n;
    return n;
}

/* gOld (V_d x 3) += S_d^T gNew, where gNew (V_{d+1} x 3) is modified in place
 * (its face and edge parts accumulate the vertex-pass and edge-pass terms). */
static void adjoint_level(const lvl *L, real *gNew, real *gOld)
{
    real *gF = gNew + 3 * (size_t)L->V;
    real *gE = gNew + 3 * ((size_t)L->V + L->F);
    int32_t h, i;

    for (h = 0; h < L->H; ++h) {                          /* vertex pass^T */
        const vcoef k = creased_vertex_coef(L, h);
        const int32_t v = L_vert(L, h), f = L_face(L, h);
        const int32_t e = L_edge(L, h), ep = L_edge(L, L_prev(L, h));
        for (i = 0; i < 3; ++i) {
            const real g = gNew[3 * (size_t)v + i];
            gOld[3 * (size_t)v + i] += k.a * g;
            gF[3 * (size_t)f + i] += k.bF * g;
            gE[3 * (size_t)e + i] += k.cE * g;
            gE[3 * (size_t)ep + i] += k.dE * g;
        }
    }
    for (h = 0; h < L->H; ++h) {                          /* edge pass^T */
        const int32_t e = L_edge(L, h), f = L_face(L, h);
        const int32_t v0 = L_vert(L, h), v1 = L_vert(L, L_next(L, h));
        const real w = satr(L_esharp(L, e));
        const real b = L_twin(L, h) < 0 ? (real)1 : (real)0.5f;
        const real al = (1 - w) * (real)0.25f + w * b * (real)0.5f;
        const real be = w * b * (real)0.5f, ga = (1 - w) * (real)0.25f;
        for (i = 0; i < 3; ++i) {
            const real g = gE[3 * (size_t)e + i];
            gOld[3 * (size_t)v0 + i] += al * g;
            gOld[3 * (size_t)v1 + i] += be * g;
            gF[3 * (size_t)f + i] += ga * g;
        }
    }
    for (h = 0; h < L->H; ++h) {                          /* face pass^T */
        const int32_t f = L_face(L, h), v = L_vert(L, h);
        const real inv = (real)1 / (real)L_face_size(L, h);
        for (i = 0; i < 3; ++i) gOld[3 * (size_t)v + i] += gF[3 * (size_t)f + i] * inv;
    }
}

/* grad (sum_V x 3, one slot per refined point of every level) -> gCage
 * (V0 x 3).  `work` must hold sum_V x 3 reals; it receives the total
 * gradient w.r.t. each level's points. */
void or_adjoint_points_scatter(const or_subd *s, const real *grad, real *work, real *gCage)
{
    const or_cage *c = s->cage;
    int32_t d;
    memcpy(work, grad, sizeof(real) * 3 * (size_t)or_cumV(c, s->D));
    memset(gCage, 0, sizeof(real) * 3 * (size_t)c->V);
    for (d = s->D - 1; d >= 0; --d) {
        lvl L;
        or_subd tmp = *s;
        tmp.pts = work;
        lvl_init(&L, &tmp, d, NULL);
        adjoint_level(&L, work + 3 * (size_t)or_cumV(c, d),
                      d == 0 ? gCage : work + 3 * (size_t)or_cumV(c, d - 1));
    }
}

/* Ring valence of a cage halfedge's vertex, exported for test diagnostics. */
int32_t or_cage_valence(const or_cage *c, int32_t h)
{
    or_subd s;
    lvl L;
    memset(&s, 0, sizeof s);
    s.cage = c;
    memset(&L, 0, sizeof L);
    L.s = &s;
    return (int32_t)creased_ring(&L, h).valence;
}

int32_t or_real_size(void) { return (int32_t)sizeof(real); }
