/*
 * or_hex.c -- CPU restatement of the reference's hexahedral interior DMO (TEST INFRASTRUCTURE
 * ONLY; see vsdmo_oracle.h).
 *
 * f64 functions restate the reference literally, in double:
 *   shapeMetricHex                          dmo/DMOQualityHex.h:54-71 (corners read as
 *                                           4 5 6 7 0 1 2 3; 9 sub-tetrahedra from
 *                                           hex_edges / hex_principal_axes / hex_subtets,
 *                                           dmo/DMOQualityUtil.h:100-150; 0 when a sub-tet
 *                                           determinant or Frobenius norm is below EPSILON)
 *   qualityShapeMRMHex                      dmo/DMOQualityHex.h:75-96 (ring minimum)
 *   k_optimizeHierarchicalInnerHex<128>     dmo/DMOHexImplCub.h:21-137: extent = per-axis
 *                                           MINIMUM ring distance, 128 threads x 4
 *                                           candidates, per-thread maxima carried across
 *                                           levels, block arg-max with the lowest thread on
 *                                           ties, absolute-coordinate candidates
 *
 * f32 functions restate the product's arithmetic (written independently of the product):
 * ring coordinates relative to the vertex scaled by 2^-e (e from frexpf of the largest
 * per-axis ring distance); with the candidate p as corner 0, sub-tets 1, 2, 3, 6 do not depend
 * on p, and sub-tets 0, 4, 5, 7, 8 have a determinant affine in p (s = c + g.p) and a Frobenius
 * term quadratic in p (A = C + m.p + alpha |p|^2, alpha 1 or 3); the metric min_j cbrt(s^2)/A is
 * compared through s^2 / A^3 as a fraction; the 128 virtual threads of the reference block
 * are kept (lane l of a warp owns virtual threads 4l .. 4l+3).
 */
#include "vsdmo_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern const int* or__hf_rowptr(const or_mesh* m);
extern const int* or__hf(const or_mesh* m);
extern const int* or__elems(const or_mesh* m);
extern const int* or__col(const or_mesh* m, int which);

#define NQ 8
#define DEPTH 3
#define HEX_EPS 1.19209e-07f

/* ======================================================================================== */
/* f64 literal                                                                               */
/* ======================================================================================== */
static double det3d(const double* a, const double* b, const double* c) {
    double x[3] = { b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0] };
    return a[0] * x[0] + a[1] * x[1] + a[2] * x[2];
}

static double nrm2d(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

/* shapeMetricHex of corners v[0..7] */
double or_q_hex_f64(const double v[8][3]) {
    const double* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    double L[12][3], X[3][3];
    for (int a = 0; a < 3; ++a) {
        L[0][a] = P[1][a] - P[0][a]; L[4][a] = P[4][a] - P[0][a]; L[8][a] = P[5][a] - P[4][a];
        L[1][a] = P[2][a] - P[1][a]; L[5][a] = P[5][a] - P[1][a]; L[9][a] = P[6][a] - P[5][a];
        L[2][a] = P[3][a] - P[2][a]; L[6][a] = P[6][a] - P[2][a]; L[10][a] = P[7][a] - P[6][a];
        L[3][a] = P[3][a] - P[0][a]; L[7][a] = P[7][a] - P[3][a]; L[11][a] = P[7][a] - P[4][a];
        X[0][a] = (P[1][a] - P[0][a]) + (P[2][a] - P[3][a]) + (P[5][a] - P[4][a]) + (P[6][a] - P[7][a]);
        X[1][a] = (P[3][a] - P[0][a]) + (P[2][a] - P[1][a]) + (P[7][a] - P[4][a]) + (P[6][a] - P[5][a]);
        X[2][a] = (P[4][a] - P[0][a]) + (P[5][a] - P[1][a]) + (P[6][a] - P[2][a]) + (P[7][a] - P[3][a]);
    }
    /* hex_subtets: (index, sign) triples */
    static const int T[9][3] = { { 0, 3, 4 }, { 1, 0, 5 }, { 2, 1, 6 }, { 3, 2, 7 }, { 11, 8, 4 },
                                 { 8, 9, 5 }, { 9, 10, 6 }, { 10, 11, 7 }, { 0, 1, 2 } };
    static const int S[9][3] = { { 1, 1, 1 }, { 1, -1, 1 }, { 1, -1, 1 }, { -1, -1, 1 }, { 1, 1, -1 },
                                 { -1, 1, -1 }, { -1, 1, -1 }, { -1, -1, -1 }, { 1, 1, 1 } };
    double ret = 1e30;
    for (int i = 0; i < 9; ++i) {
        double e[3][3];
        for (int j = 0; j < 3; ++j)
            for (int a = 0; a < 3; ++a) e[j][a] = S[i][j] * (i == 8 ? X[T[i][j]][a] : L[T[i][j]][a]);
        double sj = det3d(e[0], e[1], e[2]);
        double Aj = nrm2d(e[0]) + nrm2d(e[1]) + nrm2d(e[2]);
        if (sj < (double)HEX_EPS || Aj < (double)HEX_EPS) return 0.0;
        double r = cbrt(sj * sj) / Aj;
        if (r < ret) ret = r;
    }
    return 3.0 * ret;
}

typedef double (*hex_metric64)(const double v[8][3]);

static double ring_hex64(int k, const double* ring, const double* p, hex_metric64 metric) {
    double q = DBL_MAX;
    for (int h = 0; h < k; ++h) {
        double v[8][3];
        for (int a = 0; a < 3; ++a) v[0][a] = p[a];
        for (int c = 0; c < 7; ++c)
            for (int a = 0; a < 3; ++a) v[1 + c][a] = ring[21 * h + 3 * c + a];
        double x = metric(v);
        q = fmin(q, x);
    }
    return q;
}

static void hex_vertex_f64(const or_mesh* m, double* X, int v, double gs, double* margin, hex_metric64 metric) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    const int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) { if (margin) *margin = DBL_MAX; return; }
    double* ring = (double*)malloc(sizeof(double) * 21 * (size_t)k);
    const double c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    double minD[3] = { DBL_MAX, DBL_MAX, DBL_MAX };
    for (int h = 0; h < k; ++h)
        for (int c = 0; c < 7; ++c) {
            const int u = hf[7 * (b + h) + c];
            for (int a = 0; a < 3; ++a) {
                ring[21 * h + 3 * c + a] = X[3 * u + a];
                minD[a] = fmin(minD[a], fabs(X[3 * u + a] - c0[a]));
            }
        }
    double curr[3] = { c0[0], c0[1], c0[2] };
    double qMax[128], pMax[128][3];
    for (int t = 0; t < 128; ++t) { qMax[t] = -FLT_MAX; pMax[t][0] = pMax[t][1] = pMax[t][2] = 0.0; }
    const double aff = 1.0 / (NQ - 1);
    double ds = gs, mg = DBL_MAX;
    int key = 0;
    for (int d = 0; d < DEPTH; ++d) {
        double gmax[3], gmin[3];
        for (int a = 0; a < 3; ++a) { gmax[a] = curr[a] + ds * minD[a]; gmin[a] = curr[a] - ds * minD[a]; }
        const double qLast = ring_hex64(k, ring, curr, metric);
        double best = -DBL_MAX, second = -DBL_MAX, carried = -DBL_MAX;
        for (int t = 0; t < 128; ++t) carried = fmax(carried, qMax[t]);
        for (int t = 0; t < 128; ++t)
            for (int idx = 4 * t; idx < 4 * t + 4; ++idx) {
                const int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
                double p[3];
                p[0] = aff * (i * gmin[0] + (NQ - 1 - i) * gmax[0]);
                p[1] = aff * (j * gmin[1] + (NQ - 1 - j) * gmax[1]);
                p[2] = aff * (kk * gmin[2] + (NQ - 1 - kk) * gmax[2]);
                const double q = ring_hex64(k, ring, p, metric);
                if (q > best) { second = best; best = q; }
                else if (q < best && q > second) second = q;   /* exact ties: see or__gap64 */
                if (q > qMax[t]) { qMax[t] = q; pMax[t][0] = p[0]; pMax[t][1] = p[1]; pMax[t][2] = p[2]; }
            }
        key = 0;
        for (int t = 1; t < 128; ++t) if (qMax[t] > qMax[key]) key = t;
        mg = fmin(mg, best - second);
        if (carried > -DBL_MAX && best != carried) mg = fmin(mg, fabs(best - carried));
        mg = fmin(mg, or__gap64(qMax[key], qLast));
        if (qLast < qMax[key]) { curr[0] = pMax[key][0]; curr[1] = pMax[key][1]; curr[2] = pMax[key][2]; }
        ds = ds * (2.0 / (NQ - 1));
    }
    const double qOld = ring_hex64(k, ring, c0, metric);
    mg = fmin(mg, or__gap64(qMax[key], qOld));
    if (qOld < qMax[key]) { X[3 * v] = curr[0]; X[3 * v + 1] = curr[1]; X[3 * v + 2] = curr[2]; }
    if (margin) *margin = mg;
    free(ring);
}

void or_dmo_hex_f64(const or_mesh* m, double* X, int v0, int v1, double gs, double* margin, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int v = v0; v < v1; ++v) hex_vertex_f64(m, X, v, gs, margin ? margin + (v - v0) : NULL, or_q_hex_f64);
}

/* ======================================================================================== */
/* f32: the product's arithmetic                                                             */
/* ======================================================================================== */
static inline float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static inline void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline void sub3(const float* a, const float* b, float* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
static inline void add3(const float* a, const float* b, float* o) { o[0] = a[0] + b[0]; o[1] = a[1] + b[1]; o[2] = a[2] + b[2]; }
static inline void neg3(const float* a, float* o) { o[0] = -a[0]; o[1] = -a[1]; o[2] = -a[2]; }

/* per halfhex: constant part (N, D, zero) + 5 candidate-dependent sub-tets, each
 * { gx, gy, gz, c, mx, my, mz, C } (alpha = 1 for sub-tets 0, 5, 7 and 3 for 4, 8) */
typedef struct { float N, D; int zero; float co[5][8]; } hexco;
static const float HEX_ALPHA[5] = { 1.f, 3.f, 1.f, 1.f, 3.f };

/* the key's fraction update: zero flag, first-initialises, strict cross-multiplied compare */
static inline void frac_min(float s, float A, float es, float ea, float* N, float* D, int* first, int* zero) {
    if (s < es || A < ea) { *zero = 1; return; }
    const float num = s * s, den = (A * A) * A;
    if (*first) { *N = num; *D = den; *first = 0; return; }
    if (num * *D < *N * den) { *N = num; *D = den; }
}

void or_hex_coeffs_f32(const float r[7][3], float es, float ea, float* out /* 43 floats */) {
    /* v0 = p, v1..v7 = r[0..6] */
    const float* v1 = r[0]; const float* v2 = r[1]; const float* v3 = r[2]; const float* v4 = r[3];
    const float* v5 = r[4]; const float* v6 = r[5]; const float* v7 = r[6];
    float L0[3], L1[3], L2[3], L3[3], L5[3], L6[3], L7[3], L9[3], L10[3];
    sub3(v5, v4, L0); sub3(v6, v5, L1); sub3(v7, v6, L2); sub3(v7, v4, L3); sub3(v1, v5, L5);
    sub3(v2, v6, L6); sub3(v3, v7, L7); sub3(v2, v1, L9); sub3(v3, v2, L10);
    float N = 0.f, D = 1.f;
    int first = 1, zero = 0;
    /* constant sub-tets 1 (L1, -L0, L5), 2 (L2, -L1, L6), 3 (-L3, -L2, L7), 6 (-L9, L10, -L6) */
    float e[4][3][3];
    memcpy(e[0][0], L1, 12); neg3(L0, e[0][1]); memcpy(e[0][2], L5, 12);
    memcpy(e[1][0], L2, 12); neg3(L1, e[1][1]); memcpy(e[1][2], L6, 12);
    neg3(L3, e[2][0]); neg3(L2, e[2][1]); memcpy(e[2][2], L7, 12);
    neg3(L9, e[3][0]); memcpy(e[3][1], L10, 12); neg3(L6, e[3][2]);
    for (int i = 0; i < 4; ++i) {
        float x[3];
        cross3(e[i][1], e[i][2], x);
        const float s = dot3(e[i][0], x);
        const float A = (dot3(e[i][0], e[i][0]) + dot3(e[i][1], e[i][1])) + dot3(e[i][2], e[i][2]);
        frac_min(s, A, es, ea, &N, &D, &first, &zero);
    }
    out[0] = N; out[1] = D; out[2] = zero ? 1.f : 0.f;
    float* co = out + 3;
    float g[3], t1[3], t2[3], t3[3];
    /* sub 0: det = (p - v4) . (L0 x L3); A = (|L0|^2 + |L3|^2) + |v4|^2 - 2 v4.p + |p|^2 */
    cross3(L0, L3, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -dot3(v4, g);
    co[4] = -2.f * v4[0]; co[5] = -2.f * v4[1]; co[6] = -2.f * v4[2];
    co[7] = (dot3(L0, L0) + dot3(L3, L3)) + dot3(v4, v4);
    co += 8;
    /* sub 4: (v3 - p, v1 - p, v4 - p): det = a.(b x c) - p.((b x c + c x a) + a x b) */
    cross3(v1, v4, t1); cross3(v4, v3, t2); cross3(v3, v1, t3);
    co[0] = -((t1[0] + t2[0]) + t3[0]); co[1] = -((t1[1] + t2[1]) + t3[1]); co[2] = -((t1[2] + t2[2]) + t3[2]);
    co[3] = dot3(v3, t1);
    co[4] = -2.f * ((v3[0] + v1[0]) + v4[0]); co[5] = -2.f * ((v3[1] + v1[1]) + v4[1]); co[6] = -2.f * ((v3[2] + v1[2]) + v4[2]);
    co[7] = (dot3(v3, v3) + dot3(v1, v1)) + dot3(v4, v4);
    co += 8;
    /* sub 5: (p - v1, L9, -L5): det = (p - v1) . (L9 x -L5) */
    float mL5[3];
    neg3(L5, mL5);
    cross3(L9, mL5, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -dot3(v1, g);
    co[4] = -2.f * v1[0]; co[5] = -2.f * v1[1]; co[6] = -2.f * v1[2];
    co[7] = dot3(v1, v1) + (dot3(L9, L9) + dot3(L5, L5));
    co += 8;
    /* sub 7: (-L10, p - v3, -L7): det = (p - v3) . (L7 x L10) */
    cross3(L7, L10, g);
    co[0] = g[0]; co[1] = g[1]; co[2] = g[2]; co[3] = -dot3(v3, g);
    co[4] = -2.f * v3[0]; co[5] = -2.f * v3[1]; co[6] = -2.f * v3[2];
    co[7] = dot3(v3, v3) + (dot3(L10, L10) + dot3(L7, L7));
    co += 8;
    /* sub 8: (Q0 - p, Q1 - p, Q2 + p) */
    float Q0[3], Q1[3], Q2[3], a1[3], a2[3], a3[3];
    for (int a = 0; a < 3; ++a) {
        Q0[a] = ((v5[a] - v4[a]) + (v6[a] - v7[a])) + (v1[a] + (v2[a] - v3[a]));
        Q1[a] = ((v7[a] - v4[a]) + (v6[a] - v5[a])) + (v3[a] + (v2[a] - v1[a]));
        Q2[a] = ((v1[a] - v5[a]) + (v2[a] - v6[a])) + ((v3[a] - v7[a]) - v4[a]);
    }
    cross3(Q0, Q1, a1); cross3(Q2, Q0, a2); cross3(Q1, Q2, a3);
    co[0] = (a1[0] - a2[0]) - a3[0]; co[1] = (a1[1] - a2[1]) - a3[1]; co[2] = (a1[2] - a2[2]) - a3[2];
    co[3] = dot3(Q0, a3);
    co[4] = 2.f * ((Q2[0] - Q0[0]) - Q1[0]); co[5] = 2.f * ((Q2[1] - Q0[1]) - Q1[1]); co[6] = 2.f * ((Q2[2] - Q0[2]) - Q1[2]);
    co[7] = (dot3(Q0, Q0) + dot3(Q1, Q1)) + dot3(Q2, Q2);
}

/* ring key at p = (x, y, z): s = fmaf(gx, x, fmaf(gy, y, fmaf(gz, z, c))),
 * A = ((C + fmaf(mz, z, a z z)) + fmaf(my, y, a y y)) + fmaf(mx, x, a x x) */
static float hex_key32(int k, const float* co, float x, float y, float z, float es, float ea) {
    const float t1[3] = { x * x, y * y, z * z };
    const float t3[3] = { (3.f * x) * x, (3.f * y) * y, (3.f * z) * z };
    float N = 0.f, D = 1.f;
    int first = 1, zero = 0;
    for (int h = 0; h < k; ++h) {
        const float* c = co + 43 * h;
        if (c[2] != 0.f) zero = 1;
        else if (first) { N = c[0]; D = c[1]; first = 0; }
        else if (c[0] * D < N * c[1]) { N = c[0]; D = c[1]; }
        for (int j = 0; j < 5; ++j) {
            const float* q = c + 3 + 8 * j;
            const float* t = HEX_ALPHA[j] == 1.f ? t1 : t3;
            const float s = fmaf(q[0], x, fmaf(q[1], y, fmaf(q[2], z, q[3])));
            const float A = ((q[7] + fmaf(q[6], z, t[2])) + fmaf(q[5], y, t[1])) + fmaf(q[4], x, t[0]);
            frac_min(s, A, es, ea, &N, &D, &first, &zero);
        }
    }
    return zero ? 0.f : N / D;
}

float or__hex_key_f32(int k, const float* co, float x, float y, float z, float es, float ea) {
    return hex_key32(k, co, x, y, z, es, ea);
}

static inline float grid_offset(int i) { return (float)(NQ - 1 - 2 * i) / (float)(NQ - 1); }

static void hex_vertex_f32(const or_mesh* m, float* X, int v, float gs) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    const int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    const float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float mx[3] = { 0.f, 0.f, 0.f }, mn[3] = { FLT_MAX, FLT_MAX, FLT_MAX };
    for (int h = 0; h < k; ++h)
        for (int c = 0; c < 7; ++c) {
            const int u = hf[7 * (b + h) + c];
            for (int a = 0; a < 3; ++a) {
                const float d = fabsf(X[3 * u + a] - c0[a]);
                mx[a] = fmaxf(mx[a], d);
                mn[a] = fminf(mn[a], d);
            }
        }
    const float mm = fmaxf(mx[0], fmaxf(mx[1], mx[2]));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;
    int ex;
    (void)frexpf(mm, &ex);
    const float es = ldexpf(HEX_EPS, -3 * ex), ea = ldexpf(HEX_EPS, -2 * ex);
    float* co = (float*)malloc(sizeof(float) * 43 * (size_t)k);
    for (int h = 0; h < k; ++h) {
        float r[7][3];
        for (int c = 0; c < 7; ++c) {
            const int u = hf[7 * (b + h) + c];
            for (int a = 0; a < 3; ++a) r[c][a] = ldexpf(X[3 * u + a] - c0[a], -ex);
        }
        or_hex_coeffs_f32(r, es, ea, co + 43 * h);
    }
    const float S[3] = { ldexpf(mn[0], -ex), ldexpf(mn[1], -ex), ldexpf(mn[2], -ex) };
    float qMax[128], pMax[128][3];
    for (int t = 0; t < 128; ++t) { qMax[t] = -FLT_MAX; pMax[t][0] = pMax[t][1] = pMax[t][2] = 0.f; }
    float dx = 0.f, dy = 0.f, dz = 0.f;
    float ds = gs;
    int key = 0;
    for (int d = 0; d < DEPTH; ++d) {
        const float Sx = ds * S[0], Sy = ds * S[1], Sz = ds * S[2];
        const float qLast = hex_key32(k, co, dx, dy, dz, es, ea);
        for (int t = 0; t < 128; ++t)
            for (int idx = 4 * t; idx < 4 * t + 4; ++idx) {
                const int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
                const float x = fmaf(grid_offset(i), Sx, dx), y = fmaf(grid_offset(j), Sy, dy), z = fmaf(grid_offset(kk), Sz, dz);
                const float q = hex_key32(k, co, x, y, z, es, ea);
                if (q > qMax[t]) { qMax[t] = q; pMax[t][0] = x; pMax[t][1] = y; pMax[t][2] = z; }
            }
        key = 0;
        for (int t = 1; t < 128; ++t) if (qMax[t] > qMax[key]) key = t;
        if (qLast < qMax[key]) { dx = pMax[key][0]; dy = pMax[key][1]; dz = pMax[key][2]; }
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    const float qOld = hex_key32(k, co, 0.f, 0.f, 0.f, es, ea);
    if (qOld < qMax[key]) {
        X[3 * v] = c0[0] + ldexpf(dx, ex);
        X[3 * v + 1] = c0[1] + ldexpf(dy, ex);
        X[3 * v + 2] = c0[2] + ldexpf(dz, ex);
    }
    free(co);
}

void or_dmo_hex_f32(const or_mesh* m, float* X, int v0, int v1, float gs, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int v = v0; v < v1; ++v) hex_vertex_f32(m, X, v, gs);
}

/* shapeMetricHex in float with the reference's operation order and cbrtf */
float or_q_hex_f32(const float v[8][3]) {
    const float* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    float L[12][3], Xa[3][3];
    for (int a = 0; a < 3; ++a) {
        L[0][a] = P[1][a] - P[0][a]; L[4][a] = P[4][a] - P[0][a]; L[8][a] = P[5][a] - P[4][a];
        L[1][a] = P[2][a] - P[1][a]; L[5][a] = P[5][a] - P[1][a]; L[9][a] = P[6][a] - P[5][a];
        L[2][a] = P[3][a] - P[2][a]; L[6][a] = P[6][a] - P[2][a]; L[10][a] = P[7][a] - P[6][a];
        L[3][a] = P[3][a] - P[0][a]; L[7][a] = P[7][a] - P[3][a]; L[11][a] = P[7][a] - P[4][a];
        Xa[0][a] = (((P[1][a] - P[0][a]) + (P[2][a] - P[3][a])) + (P[5][a] - P[4][a])) + (P[6][a] - P[7][a]);
        Xa[1][a] = (((P[3][a] - P[0][a]) + (P[2][a] - P[1][a])) + (P[7][a] - P[4][a])) + (P[6][a] - P[5][a]);
        Xa[2][a] = (((P[4][a] - P[0][a]) + (P[5][a] - P[1][a])) + (P[6][a] - P[2][a])) + (P[7][a] - P[3][a]);
    }
    static const int T[9][3] = { { 0, 3, 4 }, { 1, 0, 5 }, { 2, 1, 6 }, { 3, 2, 7 }, { 11, 8, 4 },
                                 { 8, 9, 5 }, { 9, 10, 6 }, { 10, 11, 7 }, { 0, 1, 2 } };
    static const int S[9][3] = { { 1, 1, 1 }, { 1, -1, 1 }, { 1, -1, 1 }, { -1, -1, 1 }, { 1, 1, -1 },
                                 { -1, 1, -1 }, { -1, 1, -1 }, { -1, -1, -1 }, { 1, 1, 1 } };
    float ret = 1e30f;
    for (int i = 0; i < 9; ++i) {
        float e[3][3];
        for (int j = 0; j < 3; ++j)
            for (int a = 0; a < 3; ++a) {
                const float val = i == 8 ? Xa[T[i][j]][a] : L[T[i][j]][a];
                e[j][a] = S[i][j] < 0 ? -val : val;
            }
        float x[3];
        cross3(e[1], e[2], x);
        const float sj = dot3(e[0], x);
        const float Aj = (dot3(e[0], e[0]) + dot3(e[1], e[1])) + dot3(e[2], e[2]);
        if (sj < HEX_EPS || Aj < HEX_EPS) return 0.f;
        ret = fminf(ret, cbrtf(sj * sj) / Aj);
    }
    return 3.f * ret;
}

void or_hex_qualities_f64(const or_mesh* m, const double* X, double* q) {
    const int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    for (int e = 0; e < nE; ++e) {
        double v[8][3];
        for (int c = 0; c < 8; ++c)
            for (int a = 0; a < 3; ++a) v[c][a] = X[3 * (size_t)el[8 * e + c] + a];
        q[e] = or_q_hex_f64(v);
    }
}

void or_hex_qualities_f32(const or_mesh* m, const float* X, float* q) {
    const int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    for (int e = 0; e < nE; ++e) {
        float v[8][3];
        for (int c = 0; c < 8; ++c)
            for (int a = 0; a < 3; ++a) v[c][a] = X[3 * (size_t)el[8 * e + c] + a];
        q[e] = or_q_hex_f32(v);
    }
}

static void hex_hist(const or_mesh* m, const float* X, float* q, double* mn, double* mean) {
    const int nE = or_mesh_info(m, OR_I_NE);
    or_hex_qualities_f32(m, X, q);
    double a = DBL_MAX, s = 0.0;
    for (int i = 0; i < nE; ++i) { a = fmin(a, q[i]); s += q[i]; }
    *mn = a;
    *mean = s / nE;
}

void or_optimize_hex_f32(const or_mesh* m, float* X, int n_iter, float gs, int nthreads, double* min_hist,
                         double* mean_hist) {
    const int nc = or_mesh_info(m, OR_I_NCOL_INNER);
    const int* off = or__col(m, 2);
    float* q = (float*)malloc(sizeof(float) * (size_t)or_mesh_info(m, OR_I_NE));
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) or_dmo_hex_f32(m, X, off[c], off[c + 1], gs, nthreads);
        double mn, mean;
        hex_hist(m, X, q, &mn, &mean);
        if (min_hist) min_hist[it] = mn;
        if (mean_hist) mean_hist[it] = mean;
    }
    free(q);
}

void or_optimize_hex_f64(const or_mesh* m, double* X, int n_iter, double gs, int nthreads, double* min_hist,
                         double* mean_hist) {
    const int nc = or_mesh_info(m, OR_I_NCOL_INNER);
    const int* off = or__col(m, 2);
    const int nE = or_mesh_info(m, OR_I_NE);
    double* q = (double*)malloc(sizeof(double) * (size_t)nE);
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) or_dmo_hex_f64(m, X, off[c], off[c + 1], gs, NULL, nthreads);
        or_hex_qualities_f64(m, X, q);
        double a = DBL_MAX, s = 0.0;
        for (int i = 0; i < nE; ++i) { a = fmin(a, q[i]); s += q[i]; }
        if (min_hist) min_hist[it] = a;
        if (mean_hist) mean_hist[it] = s / nE;
    }
    free(q);
}

/* ======================================================================================== */
/* condition-number quality of hexahedra (an addition to the reference's criteria)            */
/* ======================================================================================== */
/* Corner Jacobians of the hex read in the reference's order P = v4 v5 v6 v7 v0 v1 v2 v3:
 * c0 (P1-P0, P3-P0, P4-P0), c1 (P2-P1, P0-P1, P5-P1), c2 (P3-P2, P1-P2, P6-P2),
 * c3 (P0-P3, P2-P3, P7-P3), c4 (P7-P4, P5-P4, P0-P4), c5 (P4-P5, P6-P5, P1-P5),
 * c6 (P5-P6, P7-P6, P2-P6), c7 (P6-P7, P4-P7, P3-P7); corner quality 3 det A /
 * (|A|_F |adj A|_F) (the inverse condition number, signed; 0 for a degenerate corner); element
 * quality = minimum over the corners. f64: literally; f32: the product's arithmetic (the key
 * det |det| / (|A|_F^2 |adj A|_F^2) in the search, the ring scaled as for the shape metric). */
static const int HC_CORNER[8][4] = { { 0, 1, 3, 4 }, { 1, 2, 0, 5 }, { 2, 3, 1, 6 }, { 3, 0, 2, 7 },
                                     { 4, 7, 5, 0 }, { 5, 4, 6, 1 }, { 6, 5, 7, 2 }, { 7, 6, 4, 3 } };

double or_q_hex_cond_f64(const double v[8][3]) {
    const double* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    double q = DBL_MAX;
    for (int c = 0; c < 8; ++c) {
        double e[3][3];
        for (int j = 0; j < 3; ++j)
            for (int a = 0; a < 3; ++a) e[j][a] = P[HC_CORNER[c][j + 1]][a] - P[HC_CORNER[c][0]][a];
        const double det = det3d(e[0], e[1], e[2]);
        double x[3][3];
        for (int j = 0; j < 3; ++j) {
            const double* u = e[(j + 1) % 3]; const double* w = e[(j + 2) % 3];
            x[j][0] = u[1] * w[2] - u[2] * w[1]; x[j][1] = u[2] * w[0] - u[0] * w[2]; x[j][2] = u[0] * w[1] - u[1] * w[0];
        }
        const double F2 = nrm2d(e[0]) + nrm2d(e[1]) + nrm2d(e[2]);
        const double G2 = nrm2d(x[0]) + nrm2d(x[1]) + nrm2d(x[2]);
        const double qc = F2 * G2 > 0.0 ? 3.0 * det / sqrt(F2 * G2) : 0.0;
        q = fmin(q, qc);
    }
    return q;
}

/* f32: fixed operation order */
static void hcf_cross(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static float hcf_dot(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static void hcf_corner(const float* o, const float* a, const float* b, const float* c, float* det, float* den) {
    const float e1[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] };
    const float e2[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] };
    const float e3[3] = { c[0] - o[0], c[1] - o[1], c[2] - o[2] };
    float x[3], y[3], z[3];
    hcf_cross(e2, e3, x);
    *det = hcf_dot(e1, x);
    const float F2 = (hcf_dot(e1, e1) + hcf_dot(e2, e2)) + hcf_dot(e3, e3);
    hcf_cross(e3, e1, y);
    hcf_cross(e1, e2, z);
    const float G2 = (hcf_dot(x, x) + hcf_dot(y, y)) + hcf_dot(z, z);
    *den = F2 * G2;
}
static float hcf_key(const float* o, const float* a, const float* b, const float* c) {
    float det, den;
    hcf_corner(o, a, b, c, &det, &den);
    return den > 0.f ? (det * fabsf(det)) / den : 0.f;
}
static float hcf_quality(const float* o, const float* a, const float* b, const float* c) {
    float det, den;
    hcf_corner(o, a, b, c, &det, &den);
    return den > 0.f ? (3.f * det) / sqrtf(den) : 0.f;
}

float or_q_hex_cond_f32(const float v[8][3]) {
    const float* P[8] = { v[4], v[5], v[6], v[7], v[0], v[1], v[2], v[3] };
    float q = hcf_quality(P[0], P[1], P[3], P[4]);
    for (int c = 1; c < 8; ++c)
        q = fminf(q, hcf_quality(P[HC_CORNER[c][0]], P[HC_CORNER[c][1]], P[HC_CORNER[c][2]], P[HC_CORNER[c][3]]));
    return q;
}

/* halfhex (p, r0..r6): P4 = p, P5..P7 = r0..r2, P0..P3 = r3..r6 */
static float hcf_const_key(const float (*r)[3]) {
    float k = hcf_key(r[4], r[5], r[3], r[0]);
    k = fminf(k, hcf_key(r[5], r[6], r[4], r[1]));
    k = fminf(k, hcf_key(r[6], r[3], r[5], r[2]));
    k = fminf(k, hcf_key(r[1], r[0], r[2], r[5]));
    return k;
}
static float hcf_halfhex_key(const float (*r)[3], float ck, const float* p) {
    float k = fminf(ck, hcf_key(p, r[2], r[0], r[3]));
    k = fminf(k, hcf_key(r[3], r[4], r[6], p));
    k = fminf(k, hcf_key(r[0], p, r[1], r[4]));
    k = fminf(k, hcf_key(r[2], r[1], p, r[6]));
    return k;
}
static float hcf_ring_key(int k, const float* R, const float* CK, const float* p) {
    float q = FLT_MAX;
    for (int h = 0; h < k; ++h) q = fminf(q, hcf_halfhex_key((const float(*)[3])(R + 21 * h), CK[h], p));
    return q;
}

static void hex_cond_vertex_f32(const or_mesh* m, float* X, int v, float gs) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    const int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    const float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float mx[3] = { 0.f, 0.f, 0.f }, mn[3] = { FLT_MAX, FLT_MAX, FLT_MAX };
    for (int h = 0; h < k; ++h)
        for (int c = 0; c < 7; ++c) {
            const int u = hf[7 * (b + h) + c];
            for (int a = 0; a < 3; ++a) {
                const float d = fabsf(X[3 * u + a] - c0[a]);
                mx[a] = fmaxf(mx[a], d);
                mn[a] = fminf(mn[a], d);
            }
        }
    const float mm = fmaxf(mx[0], fmaxf(mx[1], mx[2]));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return;
    int ex;
    (void)frexpf(mm, &ex);
    float* R = (float*)malloc(sizeof(float) * 21 * (size_t)k);
    float* CK = (float*)malloc(sizeof(float) * (size_t)k);
    for (int h = 0; h < k; ++h) {
        for (int c = 0; c < 7; ++c) {
            const int u = hf[7 * (b + h) + c];
            for (int a = 0; a < 3; ++a) R[21 * h + 3 * c + a] = ldexpf(X[3 * u + a] - c0[a], -ex);
        }
        CK[h] = hcf_const_key((const float(*)[3])(R + 21 * h));
    }
    const float S[3] = { ldexpf(mn[0], -ex), ldexpf(mn[1], -ex), ldexpf(mn[2], -ex) };
    float qMax[128], pMax[128][3];
    for (int t = 0; t < 128; ++t) { qMax[t] = -FLT_MAX; pMax[t][0] = pMax[t][1] = pMax[t][2] = 0.f; }
    float d[3] = { 0.f, 0.f, 0.f };
    float ds = gs;
    int key = 0;
    for (int lv = 0; lv < DEPTH; ++lv) {
        const float Sx = ds * S[0], Sy = ds * S[1], Sz = ds * S[2];
        const float qLast = hcf_ring_key(k, R, CK, d);
        for (int t = 0; t < 128; ++t)
            for (int idx = 4 * t; idx < 4 * t + 4; ++idx) {
                const int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
                const float p[3] = { fmaf(grid_offset(i), Sx, d[0]), fmaf(grid_offset(j), Sy, d[1]),
                                     fmaf(grid_offset(kk), Sz, d[2]) };
                const float q = hcf_ring_key(k, R, CK, p);
                if (q > qMax[t]) { qMax[t] = q; pMax[t][0] = p[0]; pMax[t][1] = p[1]; pMax[t][2] = p[2]; }
            }
        key = 0;
        for (int t = 1; t < 128; ++t) if (qMax[t] > qMax[key]) key = t;
        if (qLast < qMax[key]) { d[0] = pMax[key][0]; d[1] = pMax[key][1]; d[2] = pMax[key][2]; }
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    const float z0[3] = { 0.f, 0.f, 0.f };
    const float qOld = hcf_ring_key(k, R, CK, z0);
    if (qOld < qMax[key]) {
        X[3 * v] = c0[0] + ldexpf(d[0], ex);
        X[3 * v + 1] = c0[1] + ldexpf(d[1], ex);
        X[3 * v + 2] = c0[2] + ldexpf(d[2], ex);
    }
    free(R); free(CK);
}

void or_dmo_hex_cond_f32(const or_mesh* m, float* X, int v0, int v1, float gs, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int v = v0; v < v1; ++v) hex_cond_vertex_f32(m, X, v, gs);
}

void or_dmo_hex_cond_f64(const or_mesh* m, double* X, int v0, int v1, double gs, double* margin, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int v = v0; v < v1; ++v) hex_vertex_f64(m, X, v, gs, margin ? margin + (v - v0) : NULL, or_q_hex_cond_f64);
}

void or_hex_cond_qualities_f64(const or_mesh* m, const double* X, double* q) {
    const int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    for (int e = 0; e < nE; ++e) {
        double v[8][3];
        for (int c = 0; c < 8; ++c)
            for (int a = 0; a < 3; ++a) v[c][a] = X[3 * (size_t)el[8 * e + c] + a];
        q[e] = or_q_hex_cond_f64(v);
    }
}

void or_hex_cond_qualities_f32(const or_mesh* m, const float* X, float* q) {
    const int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    for (int e = 0; e < nE; ++e) {
        float v[8][3];
        for (int c = 0; c < 8; ++c)
            for (int a = 0; a < 3; ++a) v[c][a] = X[3 * (size_t)el[8 * e + c] + a];
        q[e] = or_q_hex_cond_f32(v);
    }
}
