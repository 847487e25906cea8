/*
 * or_feat.c -- CPU restatement of the 1D feature / boundary pass (TEST INFRASTRUCTURE ONLY;
 * see vsdmo_oracle.h).
 *
 * Feature vertices (the boundary of a flat mesh, the feature lines of a surface) slide along
 * curves fitted to their feature neighbours:
 *   calcOptFeatureVec / k_calcOptFeatureVec (dmo/DMOCommon.h:130-180): a feature vertex is
 *     optimised when it has exactly two feature ring vertices and the angle between them at
 *     the vertex is >= 160 degrees;
 *   computeLocalSurface1d (dmo/Surface1D.cu:8-82): frame t2 = n x (n x r) (r: to the LAST
 *     feature ring vertex in ring order, n the vertex normal or +z on flat meshes), axes
 *     (t2, n), least-squares v = a u^2 over the vertex and its feature ring vertices;
 *   localSurfaceEstimation1d (dmo/Surface1D.h:52-93): the point u of the vertex's curve (of its
 *     nearest initial vertex) blended by inverse squared distance with its projections onto
 *     the curves of the ring's feature vertices that have exactly two feature neighbours;
 *   k_optimizeHierarchical1DFlat (dmo/DMOTriFlatImplCub.h:159-330), k_optimizeHierarchical1D
 *     (dmo/DMOTriImplCub.h:205-380, dmo/DMOQuadImplCub.h:219-400): 8 candidates along u per
 *     level, half-extent grid_scale x the largest ring distance shrinking by 2/7, the lowest
 *     candidate index on ties, move on strict improvement, write when the last level's best
 *     beats the current position's quality (surfaces: the unsigned ring quality).
 * Ring quality: flat meshes the 2D mean ratio (or_q_tri2d_mean_ratio_*), surface triangles the
 * fraction key of the surface search (sign |n_t|^2 / L^2 against the nearest initial vertex's
 * normal), quads meanRatioMetricQuad with the 0.7 normal rule. Open fans for boundary vertices.
 *
 * f32: the product's operation order (estimate accumulated as sum p_i w_i, scaled by 1 / sum w
 * at the end); f64: the same formulas in double, with decision margins.
 */
#include "vsdmo_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPSF 1.19209e-07f
#define NQ 8
#define LS1F 12   /* floats per 1D curve: p0[3] a, e0[3] 0, e1[3] 0 */
#define MAXR 64

extern const int* or__he_rowptr(const or_mesh* m);
extern const int* or__he(const or_mesh* m);
extern int or__fk(const or_mesh* m);
extern const uint8_t* or__isB1(const or_mesh* m);
extern const int* or__hf_rowptr(const or_mesh* m);
extern const int* or__hf(const or_mesh* m);

static inline float d3f(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static inline double d3d(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void crossf(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline void crossd(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
}

static int nfree_of(const or_mesh* m) { return or_mesh_info(m, OR_I_NSURF) - or_mesh_info(m, OR_I_NFEATURE); }

void or_feature_flags(const or_mesh* m, const float* X, int32_t* fdeg, uint8_t* opt) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFree = nfree_of(m);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    for (int v = 0; v < nS; ++v) {
        int cnt = 0, a = -1, b = -1;
        for (int i = rp[v]; i < rp[v + 1]; ++i) {
            const int d = he[4 * i];
            if (d >= nFree) {
                if (cnt == 0) a = d; else if (cnt == 1) b = d;
                ++cnt;
            }
        }
        fdeg[v] = cnt;
        opt[v] = 0;
        if (v >= nFree && cnt == 2) {
            const float* p0 = X + 3 * (size_t)v;
            float u[3], w[3];
            for (int c = 0; c < 3; ++c) { u[c] = X[3 * (size_t)a + c] - p0[c]; w[c] = X[3 * (size_t)b + c] - p0[c]; }
            const float dot = d3f(u, w);
            const float len = sqrtf(d3f(u, u) * d3f(w, w));
            /* a float angle, as in the reference (DMOCommon.h:157-158) */
            const float ang = (float)(180.0 / 3.14159265358979323846 * (double)acosf(dot / len));
            opt[v] = ang >= 160.f;
        }
    }
}

/* ---- curve fits ----------------------------------------------------------------------- */
void or_surface_fit_1d_f32(const or_mesh* m, const float* X, const float* vn, float* LS1) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFree = nfree_of(m);
    const int flat = or_mesh_info(m, OR_I_IS_FLAT);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    memset(LS1, 0, sizeof(float) * LS1F * (size_t)nS);
    for (int v = nFree; v < nS; ++v) {
        const float* c = X + 3 * (size_t)v;
        int last = -1;
        for (int i = rp[v]; i < rp[v + 1]; ++i) if (he[4 * i] >= nFree) last = he[4 * i];
        if (last < 0) continue;
        float n[3] = { 0.f, 0.f, 1.f };
        if (!flat) { n[0] = vn[3 * (size_t)v]; n[1] = vn[3 * (size_t)v + 1]; n[2] = vn[3 * (size_t)v + 2]; }
        float r[3] = { X[3 * (size_t)last] - c[0], X[3 * (size_t)last + 1] - c[1], X[3 * (size_t)last + 2] - c[2] };
        float cr[3];
        crossf(n, r, cr);
        if (sqrtf(d3f(cr, cr)) < 10.f * EPSF) { r[0] = n[0]; r[1] = n[2]; r[2] = -n[1]; }
        float t1[3], t2[3];
        crossf(n, r, t1);
        crossf(n, t1, t2);
        float ln = sqrtf(d3f(n, n)), l1 = sqrtf(d3f(t1, t1)), l2 = sqrtf(d3f(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] /= ln; t1[a] /= l1; t2[a] /= l2; }
        float ATA = 0.f, ATb = 0.f;
        for (int i = rp[v] - 1; i < rp[v + 1]; ++i) {
            const int nb = i < rp[v] ? v : he[4 * i];
            if (i >= rp[v] && nb < nFree) continue;
            float p[3] = { X[3 * (size_t)nb] - c[0], X[3 * (size_t)nb + 1] - c[1], X[3 * (size_t)nb + 2] - c[2] };
            const float u = d3f(t2, p), w = d3f(n, p);
            ATb += (u * u) * w;
            ATA += ((u * u) * u) * u;
        }
        float* o = LS1 + LS1F * (size_t)v;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = ATb / ATA;
        o[4] = t2[0]; o[5] = t2[1]; o[6] = t2[2];
        o[8] = n[0]; o[9] = n[1]; o[10] = n[2];
    }
}

void or_surface_fit_1d_f64(const or_mesh* m, const double* X, const double* vn, double* LS1) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFree = nfree_of(m);
    const int flat = or_mesh_info(m, OR_I_IS_FLAT);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    memset(LS1, 0, sizeof(double) * LS1F * (size_t)nS);
    for (int v = nFree; v < nS; ++v) {
        const double* c = X + 3 * (size_t)v;
        int last = -1;
        for (int i = rp[v]; i < rp[v + 1]; ++i) if (he[4 * i] >= nFree) last = he[4 * i];
        if (last < 0) continue;
        double n[3] = { 0.0, 0.0, 1.0 };
        if (!flat) { n[0] = vn[3 * (size_t)v]; n[1] = vn[3 * (size_t)v + 1]; n[2] = vn[3 * (size_t)v + 2]; }
        double r[3] = { X[3 * (size_t)last] - c[0], X[3 * (size_t)last + 1] - c[1], X[3 * (size_t)last + 2] - c[2] };
        double cr[3];
        crossd(n, r, cr);
        if (sqrt(d3d(cr, cr)) < 10.0 * EPSF) { r[0] = n[0]; r[1] = n[2]; r[2] = -n[1]; }
        double t1[3], t2[3];
        crossd(n, r, t1);
        crossd(n, t1, t2);
        double ln = sqrt(d3d(n, n)), l1 = sqrt(d3d(t1, t1)), l2 = sqrt(d3d(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] /= ln; t1[a] /= l1; t2[a] /= l2; }
        double ATA = 0.0, ATb = 0.0;
        for (int i = rp[v]; i < rp[v + 1]; ++i) {
            const int nb = he[4 * i];
            if (nb < nFree) continue;
            double p[3] = { X[3 * (size_t)nb] - c[0], X[3 * (size_t)nb + 1] - c[1], X[3 * (size_t)nb + 2] - c[2] };
            const double u = d3d(t2, p), w = d3d(n, p);
            ATb += u * u * w;
            ATA += u * u * u * u;
        }
        double* o = LS1 + LS1F * (size_t)v;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = ATb / ATA;
        o[4] = t2[0]; o[5] = t2[1]; o[6] = t2[2];
        o[8] = n[0]; o[9] = n[1]; o[10] = n[2];
    }
}

/* ---- ring qualities ---------------------------------------------------------------------- */
float or_q_quad_f32(const float* p0, const float* p1, const float* p2, const float* p3, const float* n);
double or_q_quad_f64(const double* p0, const double* p1, const double* p2, const double* p3, const double* n);
float or_q_tri2d_mean_ratio_f32(const float* p0, const float* p1, const float* p2);
double or_q_tri2d_mean_ratio_f64(const double* p0, const double* p1, const double* p2);

/* mode 0: flat (2D mean ratio), 1: surface triangles (fraction key, n == NULL unsigned),
   2: surface quads; k elements, ring holds k + 1 points (tri) or 2k + 1 (quad) */
static float ringq32(int mode, int k, const float* ring, const float* p, const float* n) {
    if (mode == 0) {
        float q = FLT_MAX;
        for (int i = 0; i < k; ++i) q = fminf(q, or_q_tri2d_mean_ratio_f32(p, ring + 3 * i, ring + 3 * (i + 1)));
        return q;
    }
    if (mode == 1) {
        float N = 0.f, D = 1.f;
        for (int i = 0; i < k; ++i) {
            const float* a = ring + 3 * i; const float* b = ring + 3 * (i + 1);
            float e0[3] = { a[0] - p[0], a[1] - p[1], a[2] - p[2] };
            float e1[3] = { b[0] - p[0], b[1] - p[1], b[2] - p[2] };
            float e2[3] = { b[0] - a[0], b[1] - a[1], b[2] - a[2] };
            float l = (d3f(e0, e0) + d3f(e1, e1)) + d3f(e2, e2);
            float nt[3];
            crossf(e0, e1, nt);
            float a2 = d3f(nt, nt), num = a2;
            if (n) { float dn = d3f(nt, n); num = dn > 0.f ? a2 : (dn < 0.f ? -a2 : 0.f); }
            float den = l * l;
            if (i == 0) { N = num; D = den; continue; }
            if (num * D < N * den) { N = num; D = den; }
        }
        return N / D;
    }
    float q = 0.f;
    for (int i = 0; i < k; ++i) {
        float v = or_q_quad_f32(p, ring + 6 * i, ring + 6 * i + 3, ring + 6 * i + 6, n);
        q = i == 0 ? v : fminf(q, v);
    }
    return q;
}

static double ringq64(int mode, int k, const double* ring, const double* p, const double* n) {
    double q = DBL_MAX;
    const int crit = or__criterion();
    for (int i = 0; i < k; ++i) {
        double v;
        if (mode == 0 && crit != OR_MEAN_RATIO)
            v = crit == OR_MAX_ANGLE ? or_q_tri2d_max_angle_f64(p, ring + 3 * i, ring + 3 * (i + 1))
                                     : or_q_tri2d_min_angle_f64(p, ring + 3 * i, ring + 3 * (i + 1));
        else if (mode == 1 && crit != OR_MEAN_RATIO)
            v = or_q_tri3d_angle_f64(p, ring + 3 * i, ring + 3 * (i + 1), n, crit == OR_MAX_ANGLE);
        else if (mode == 0) v = or_q_tri2d_mean_ratio_f64(p, ring + 3 * i, ring + 3 * (i + 1));
        else if (mode == 1) {
            const double* a = ring + 3 * i; const double* b = ring + 3 * (i + 1);
            double e0[3] = { a[0] - p[0], a[1] - p[1], a[2] - p[2] };
            double e1[3] = { b[0] - p[0], b[1] - p[1], b[2] - p[2] };
            double e2[3] = { b[0] - a[0], b[1] - a[1], b[2] - a[2] };
            double l = d3d(e0, e0) + d3d(e1, e1) + d3d(e2, e2);
            double nt[3];
            crossd(e0, e1, nt);
            double a2 = d3d(nt, nt), num = a2;
            if (n) { double dn = d3d(nt, n); num = dn > 0.0 ? a2 : (dn < 0.0 ? -a2 : 0.0); }
            v = num / (l * l);
        } else v = or_q_quad_f64(p, ring + 6 * i, ring + 6 * i + 3, ring + 6 * i + 6, n);
        q = fmin(q, v);
    }
    return q;
}

/* ---- the 1D search ------------------------------------------------------------------------- */
typedef struct {
    const or_mesh* m;
    const void* X0; const void* LS1; const int32_t* nn; const void* vn; const int32_t* fdeg; const uint8_t* opt;
    int nFree, mode;
} feat_ctx;

static int ring_mode(const or_mesh* m) {
    if (or__hf_rowptr(m)) return 3;          /* boundary of a volume mesh: its ring of tets / halfhexes */
    if (or_mesh_info(m, OR_I_IS_FLAT)) return 0;
    return or__fk(m) == 3 ? 1 : 2;
}

/* mode 3: the vertex's ring of tets / halfhexes (or_vring.c) */
/* collects the quality ring (returns the element count), the extent and the surf neighbours */
#define COLLECT(T, SQRT, FABS, FMAX)                                                                       \
    const int* rp = or__he_rowptr(C->m);                                                                  \
    const int* he = or__he(C->m);                                                                         \
    const int fk = or__fk(C->m);                                                                          \
    const int b = rp[v], k = rp[v + 1] - b;                                                               \
    const T* c0 = X + 3 * (size_t)v;                                                                      \
    T ring[3 * (2 * MAXR + 1)];                                                                           \
    int surf[MAXR], ns = 0;                                                                               \
    T md = -FLT_MAX;                                                                                      \
    for (int i = 0; i < k; ++i) {                                                                         \
        const int t = he[4 * (b + i)];                                                                    \
        const int t2 = he[4 * he[4 * (b + i) + 3]];                                                       \
        const int slot = fk == 3 ? i : 2 * i;                                                             \
        for (int a = 0; a < 3; ++a) ring[3 * slot + a] = X[3 * (size_t)t + a];                             \
        T dx = FABS(c0[0] - X[3 * (size_t)t]), dy = FABS(c0[1] - X[3 * (size_t)t + 1]),                  \
          dz = FABS(c0[2] - X[3 * (size_t)t + 2]);                                                         \
        md = FMAX(md, SQRT((dx * dx + dy * dy) + dz * dz));                                                \
        if (fk == 4) {                                                                                    \
            for (int a = 0; a < 3; ++a) ring[3 * (slot + 1) + a] = X[3 * (size_t)t2 + a];                  \
            dx = FABS(c0[0] - X[3 * (size_t)t2]); dy = FABS(c0[1] - X[3 * (size_t)t2 + 1]);               \
            dz = FABS(c0[2] - X[3 * (size_t)t2 + 2]);                                                     \
            md = FMAX(md, SQRT((dx * dx + dy * dy) + dz * dz));                                            \
        }                                                                                                 \
        if (t >= C->nFree && C->fdeg[t] == 2) surf[ns++] = t;                                              \
    }                                                                                                     \
    const int closed = !or__isB1(C->m)[v];                                                                \
    int ne;                                                                                               \
    if (fk == 3) { ne = closed ? k : k - 1; if (closed) for (int a = 0; a < 3; ++a) ring[3 * k + a] = ring[a]; } \
    else { ne = closed ? k : k - 1; if (closed) for (int a = 0; a < 3; ++a) ring[3 * (2 * k) + a] = ring[a]; }

static void est1d_32(const feat_ctx* C, int v, const int* surf, int ns, float u, float* out) {
    const float* X0 = (const float*)C->X0;
    const float* LS = (const float*)C->LS1;
    const float* L = LS + LS1F * (size_t)C->nn[v];
    const float w = (L[3] * u) * u;
    float pw[3];
    for (int a = 0; a < 3; ++a) pw[a] = (L[a] + u * L[4 + a]) + w * L[8 + a];
    const float* x0 = X0 + 3 * (size_t)C->nn[v];
    float d[3] = { x0[0] - pw[0], x0[1] - pw[1], x0[2] - pw[2] };
    float id = 1.0f / (d3f(d, d) + EPSF);
    float isum = id;
    float acc[3] = { pw[0] * id, pw[1] * id, pw[2] * id };
    for (int i = 0; i < ns; ++i) {
        const int nnN = C->nn[surf[i]];
        const float* xn = X0 + 3 * (size_t)nnN;
        float e[3] = { xn[0] - pw[0], xn[1] - pw[1], xn[2] - pw[2] };
        const float idn = 1.0f / (d3f(e, e) + EPSF);
        isum = isum + idn;
        const float* Ln = LS + LS1F * (size_t)nnN;
        float q[3] = { pw[0] - Ln[0], pw[1] - Ln[1], pw[2] - Ln[2] };
        const float lu = d3f(q, Ln + 4);
        const float lw = (Ln[3] * lu) * lu;
        for (int a = 0; a < 3; ++a) acc[a] = acc[a] + ((Ln[a] + lu * Ln[4 + a]) + lw * Ln[8 + a]) * idn;
    }
    const float inv = 1.0f / isum;
    out[0] = acc[0] * inv; out[1] = acc[1] * inv; out[2] = acc[2] * inv;
}

static void feat_vertex_32(const feat_ctx* C, float* X, int v, float gs) {
    if (!C->opt[v]) return;
    COLLECT(float, sqrtf, fabsf, fmaxf)
    if (k > MAXR) return;
    or_vring32 R = { 0 };
    if (C->mode == 3) {
        if (!or__vring32_init(&R, C->m, X, v)) { or__vring32_free(&R); return; }
        md = R.md;
    }
#define RQ(P, N) (C->mode == 3 ? or__vring32_key(&R, P) : ringq32(C->mode, ne, ring, P, N))
    const float* LS = (const float*)C->LS1;
    const float* L = LS + LS1F * (size_t)C->nn[v];
    float q[3] = { c0[0] - L[0], c0[1] - L[1], c0[2] - L[2] };
    float cu = d3f(q, L + 4);
    const float* nv = (C->mode == 1 || C->mode == 2) ? (const float*)C->vn + 3 * (size_t)C->nn[v] : NULL;
    float cur[3] = { c0[0], c0[1], c0[2] };
    const float aff = 1.f / (float)(NQ - 1);
    float ds = gs, lastMax = -FLT_MAX;
    for (int d = 0; d < 3; ++d) {
        const float uMax = ds * md, uMin = -ds * md;
        float best = 0.f, bu = 0.f;
        int bi = -1;
        for (int i = 0; i < NQ; ++i) {
            const float u = cu + aff * ((float)i * uMin + (float)(NQ - 1 - i) * uMax);
            float p[3];
            est1d_32(C, v, surf, ns, u, p);
            const float qv = RQ(p, nv);
            if (bi < 0 || qv > best) { best = qv; bi = i; bu = u; }
        }
        const float qLast = RQ(cur, nv);
        if (qLast < best) {
            est1d_32(C, v, surf, ns, bu, cur);
            cu = bu;
        }
        lastMax = best;
        ds = ds * (2.f / (float)(NQ - 1));
    }
    const float qOld = RQ(c0, NULL);
#undef RQ
    if (qOld < lastMax) { X[3 * (size_t)v] = cur[0]; X[3 * (size_t)v + 1] = cur[1]; X[3 * (size_t)v + 2] = cur[2]; }
    or__vring32_free(&R);
}

void or_dmo_1d_f32(const or_mesh* m, float* X, const float* X0, const float* LS1, const int32_t* nn, const float* vn,
                   const int32_t* fdeg, const uint8_t* opt, int v0, int v1, float gs, int nthreads) {
    feat_ctx C = { m, X0, LS1, nn, vn, fdeg, opt, nfree_of(m), ring_mode(m) };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) feat_vertex_32(&C, X, v, gs);
}

static void est1d_64(const feat_ctx* C, int v, const int* surf, int ns, double u, double* out) {
    const double* X0 = (const double*)C->X0;
    const double* LS = (const double*)C->LS1;
    const double* L = LS + LS1F * (size_t)C->nn[v];
    const double w = L[3] * u * u;
    double pw[3];
    for (int a = 0; a < 3; ++a) pw[a] = L[a] + u * L[4 + a] + w * L[8 + a];
    const double* x0 = X0 + 3 * (size_t)C->nn[v];
    double d[3] = { x0[0] - pw[0], x0[1] - pw[1], x0[2] - pw[2] };
    double id = 1.0 / (d3d(d, d) + EPSF);
    double isum = id;
    double acc[3] = { pw[0] * id, pw[1] * id, pw[2] * id };
    for (int i = 0; i < ns; ++i) {
        const int nnN = C->nn[surf[i]];
        const double* xn = X0 + 3 * (size_t)nnN;
        double e[3] = { xn[0] - pw[0], xn[1] - pw[1], xn[2] - pw[2] };
        const double idn = 1.0 / (d3d(e, e) + EPSF);
        isum += idn;
        const double* Ln = LS + LS1F * (size_t)nnN;
        double q[3] = { pw[0] - Ln[0], pw[1] - Ln[1], pw[2] - Ln[2] };
        const double lu = d3d(q, Ln + 4);
        const double lw = Ln[3] * lu * lu;
        for (int a = 0; a < 3; ++a) acc[a] += (Ln[a] + lu * Ln[4 + a] + lw * Ln[8 + a]) * idn;
    }
    for (int a = 0; a < 3; ++a) out[a] = acc[a] / isum;
}

static void feat_vertex_64(const feat_ctx* C, double* X, int v, double gs, double* margin) {
    if (margin) *margin = DBL_MAX;
    if (!C->opt[v]) return;
    COLLECT(double, sqrt, fabs, fmax)
    if (k > MAXR) return;
    if (C->mode == 3) md = or__vring64_extent(C->m, X, v);
#define RQ(P, N) (C->mode == 3 ? or__vring64_q(C->m, X, v, P) : ringq64(C->mode, ne, ring, P, N))
    const double* LS = (const double*)C->LS1;
    const double* L = LS + LS1F * (size_t)C->nn[v];
    double q[3] = { c0[0] - L[0], c0[1] - L[1], c0[2] - L[2] };
    double cu = d3d(q, L + 4);
    const double* nv = (C->mode == 1 || C->mode == 2) ? (const double*)C->vn + 3 * (size_t)C->nn[v] : NULL;
    double cur[3] = { c0[0], c0[1], c0[2] };
    const double aff = 1.0 / (NQ - 1);
    double ds = gs, lastMax = -DBL_MAX, mg = DBL_MAX;
    for (int d = 0; d < 3; ++d) {
        const double uMax = ds * md, uMin = -ds * md;
        double best = -DBL_MAX, second = -DBL_MAX, bu = 0.0;
        for (int i = 0; i < NQ; ++i) {
            const double u = cu + aff * (i * uMin + (NQ - 1 - i) * uMax);
            double p[3];
            est1d_64(C, v, surf, ns, u, p);
            const double qv = RQ(p, nv);
            if (qv > best) { second = best; best = qv; bu = u; }
            else if ((C->mode != 3 || qv < best) && qv > second) second = qv;
        }
        const double qLast = RQ(cur, nv);
        mg = fmin(mg, best - second);
        mg = fmin(mg, C->mode == 3 ? or__gap64(best, qLast) : fabs(best - qLast));
        if (qLast < best) { est1d_64(C, v, surf, ns, bu, cur); cu = bu; }
        lastMax = best;
        ds = ds * (2.0 / (NQ - 1));
    }
    const double qOld = RQ(c0, NULL);
#undef RQ
    mg = fmin(mg, C->mode == 3 ? or__gap64(lastMax, qOld) : fabs(lastMax - qOld));
    if (qOld < lastMax) { X[3 * (size_t)v] = cur[0]; X[3 * (size_t)v + 1] = cur[1]; X[3 * (size_t)v + 2] = cur[2]; }
    if (margin) *margin = mg;
}

void or_dmo_1d_f64(const or_mesh* m, double* X, const double* X0, const double* LS1, const int32_t* nn,
                   const double* vn, const int32_t* fdeg, const uint8_t* opt, int v0, int v1, double gs, double* margin,
                   int nthreads) {
    feat_ctx C = { m, X0, LS1, nn, vn, fdeg, opt, nfree_of(m), ring_mode(m) };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) feat_vertex_64(&C, X, v, gs, margin ? margin + (v - v0) : NULL);
}
