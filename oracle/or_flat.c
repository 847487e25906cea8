/*
 * or_flat.c -- CPU restatement of the 2D (flat) DMO with a general grid, for triangle and quad
 * meshes, as used by the batched optimiser (TEST INFRASTRUCTURE ONLY; see vsdmo_oracle.h).
 *
 * The search is k_optimizeHierarchical2DFlat (dmo/DMOTriFlatImplCub.h:24-152) generalised to
 * N candidates per axis: N*N/2 virtual threads, thread t owning (t / N, t % N) and
 * (t / N + N/2, t % N); a thread's value is the larger of its two keys and its position the
 * first candidate's only when that key is strictly larger (the reference's p2-on-tie); the
 * winner is the first thread with the largest value; the half-extent starts at grid_scale x
 * the per-axis ring extent and shrinks by 2/(N-1) per level. N = 8 with 3 levels is the
 * reference kernel (and or_dmo_tri2d_f32 bit for bit).
 *
 * Ring elements: triangles (p, r_i, r_i+1) of the closed fan; quads (p, r_i, next(r_i), r_i+1)
 * with the reference's quad mean ratio against the +z normal (meanRatioMetricQuad(p, n),
 * dmo/DMOQualityQuad.h:30-50): -1 when a corner turns clockwise, else 2 (A1 + A2) / sum |e|^2.
 * The reference has no flat-quad optimiser; this is its 2D specialisation.
 *
 * f32 arithmetic (the product's): coordinates relative to the vertex scaled by 2^-e;
 * triangle area and quad corner cross products affine in the candidate, edge sums
 * quadratic; triangles keyed by the fraction A / L (negative area: the most negative area),
 * quads by (c1 + c2) / l (any negative corner: -1).
 */
#include "vsdmo_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern const int* or__he_rowptr(const or_mesh* m);
extern const int* or__he(const or_mesh* m);
extern int or__fk(const or_mesh* m);

/* triangle (p, a, b): A = K0 x + K1 y + K2, L = K5 + K3 x + K4 y + 2 |p|^2 */
static void tri_co(const float* a, const float* b, float* K) {
    const float ux = b[0] - a[0], uy = b[1] - a[1];
    K[0] = -uy; K[1] = ux;
    K[2] = a[0] * uy - a[1] * ux;
    K[3] = -2.0f * (a[0] + b[0]); K[4] = -2.0f * (a[1] + b[1]);
    K[5] = ((a[0] * a[0] + a[1] * a[1]) + (b[0] * b[0] + b[1] * b[1])) + (ux * ux + uy * uy);
}

/* quad (p, a, b, c): c1 = K0 x + K1 y + K2, c2 = K3 x + K4 y + K5, l = K8 + K6 x + K7 y + 2 |p|^2 */
static void quad_co(const float* a, const float* b, const float* c, float* K) {
    const float e1x = b[0] - a[0], e1y = b[1] - a[1];
    const float fx = b[0] - c[0], fy = b[1] - c[1];
    const float gx = c[0] - b[0], gy = c[1] - b[1];
    K[0] = -e1y; K[1] = e1x; K[2] = e1y * a[0] - e1x * a[1];
    K[3] = fy; K[4] = -fx; K[5] = c[1] * fx - c[0] * fy;
    K[6] = -2.0f * (a[0] + c[0]); K[7] = -2.0f * (a[1] + c[1]);
    K[8] = (((a[0] * a[0] + a[1] * a[1]) + (e1x * e1x + e1y * e1y)) + (gx * gx + gy * gy)) + (c[0] * c[0] + c[1] * c[1]);
}

static float key_tri(int k, const float* K, float x, float y) {
    const float tx = (2.0f * x) * x, ty = (2.0f * y) * y;
    float N = 0.f, D = 1.f, amin = 0.f;
    for (int t = 0; t < k; ++t) {
        const float* c = K + 6 * t;
        const float A = fmaf(c[1], y, fmaf(c[0], x, c[2]));
        const float L = (c[5] + fmaf(c[3], x, tx)) + fmaf(c[4], y, ty);
        if (t == 0) { N = A; D = L; amin = A; continue; }
        if (A * D < N * L) { N = A; D = L; }
        amin = fminf(amin, A);
    }
    return amin < 0.f ? amin : N / D;
}

static float key_quad(int k, const float* K, float x, float y) {
    const float tx = (2.0f * x) * x, ty = (2.0f * y) * y;
    float N = 0.f, D = 1.f;
    int neg = 0;
    for (int t = 0; t < k; ++t) {
        const float* c = K + 9 * t;
        const float c1 = fmaf(c[1], y, fmaf(c[0], x, c[2]));
        const float c2 = fmaf(c[4], y, fmaf(c[3], x, c[5]));
        const float l = (c[8] + fmaf(c[6], x, tx)) + fmaf(c[7], y, ty);
        if (c1 < 0.f || c2 < 0.f) neg = 1;
        const float num = c1 + c2;
        if (t == 0) { N = num; D = l; continue; }
        if (num * D < N * l) { N = num; D = l; }
    }
    return neg ? -1.f : N / D;
}

static inline float offset_n(int i, int n) { return (float)(n - 1 - 2 * i) / (float)(n - 1); }

static void flat_vertex_f32(const or_mesh* m, float* X, int v, float gs, int nq, int depth) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    const int fk = or__fk(m);
    const int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    const float c0[2] = { X[3 * v], X[3 * v + 1] };
    const int nr = fk == 3 ? k : 2 * k;
    float* r = (float*)malloc(sizeof(float) * 2 * ((size_t)nr + 1));
    float* K = (float*)malloc(sizeof(float) * 9 * (size_t)k);
    float md[2] = { 0.f, 0.f };
    for (int i = 0; i < k; ++i) {
        const int u = he[4 * (b + i)];
        const int slot = fk == 3 ? i : 2 * i;
        for (int a = 0; a < 2; ++a) { const float d = X[3 * u + a] - c0[a]; r[2 * slot + a] = d; md[a] = fmaxf(md[a], fabsf(d)); }
        if (fk == 4) {
            const int u2 = he[4 * he[4 * (b + i) + 3]];
            for (int a = 0; a < 2; ++a) { const float d = X[3 * u2 + a] - c0[a]; r[2 * (slot + 1) + a] = d; md[a] = fmaxf(md[a], fabsf(d)); }
        }
    }
    const float mm = fmaxf(md[0], md[1]);
    if (!(mm > 0.f) || !(mm < FLT_MAX)) { free(r); free(K); return; }
    int ex;
    (void)frexpf(mm, &ex);
    for (int i = 0; i < 2 * nr; ++i) r[i] = ldexpf(r[i], -ex);
    r[2 * nr] = r[0]; r[2 * nr + 1] = r[1];
    md[0] = ldexpf(md[0], -ex); md[1] = ldexpf(md[1], -ex);
    for (int t = 0; t < k; ++t) {
        if (fk == 3) tri_co(r + 2 * t, r + 2 * t + 2, K + 6 * t);
        else quad_co(r + 4 * t, r + 4 * t + 2, r + 4 * t + 4, K + 9 * t);
    }
    float dlt[2] = { 0.f, 0.f };
    const float qOld = fk == 3 ? key_tri(k, K, 0.f, 0.f) : key_quad(k, K, 0.f, 0.f);
    float qLast = qOld, lastMax = -FLT_MAX;
    float ds = gs;
    const int nvt = nq * nq / 2;
    for (int d = 0; d < depth; ++d) {
        float xs[8], ys[8];
        const float Sx = ds * md[0], Sy = ds * md[1];
        for (int i = 0; i < nq; ++i) { const float o = offset_n(i, nq); xs[i] = fmaf(o, Sx, dlt[0]); ys[i] = fmaf(o, Sy, dlt[1]); }
        float bv = 0.f, bx = 0.f, by = 0.f;
        int bt = -1;
        for (int t = 0; t < nvt; ++t) {
            const int i1 = t / nq, j1 = t % nq, i2 = i1 + nq / 2;
            const float q1 = fk == 3 ? key_tri(k, K, xs[i1], ys[j1]) : key_quad(k, K, xs[i1], ys[j1]);
            const float q2 = fk == 3 ? key_tri(k, K, xs[i2], ys[j1]) : key_quad(k, K, xs[i2], ys[j1]);
            float val = q1;
            if (q2 > q1) val = q2;
            if (bt < 0 || val > bv) {
                bv = val; bt = t;
                bx = q1 > q2 ? xs[i1] : xs[i2];
                by = ys[j1];
            }
        }
        if (qLast < bv) { dlt[0] = bx; dlt[1] = by; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0f / (float)(nq - 1));
    }
    if (qOld < lastMax) {
        X[3 * v] = c0[0] + ldexpf(dlt[0], ex);
        X[3 * v + 1] = c0[1] + ldexpf(dlt[1], ex);
    }
    free(r); free(K);
}

void or_dmo_flat_f32(const or_mesh* m, float* X, int v0, int v1, float gs, int nq, int depth, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) flat_vertex_f32(m, X, v, gs, nq, depth);
}

/* ---- f64 literal: quads with meanRatioMetricQuad(p, +z) --------------------------------- */
static double q_quad64(const double* p0, const double* p1, const double* p2, const double* p3) {
    double e[4][3];
    for (int a = 0; a < 2; ++a) { e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p1[a]; e[2][a] = p3[a] - p2[a]; e[3][a] = p0[a] - p3[a]; }
    for (int i = 0; i < 4; ++i) e[i][2] = 0.0;
    const double l = (e[0][0] * e[0][0] + e[0][1] * e[0][1]) + (e[1][0] * e[1][0] + e[1][1] * e[1][1]) +
                     (e[2][0] * e[2][0] + e[2][1] * e[2][1]) + (e[3][0] * e[3][0] + e[3][1] * e[3][1]);
    /* c1 = e1 x (-e0), c2 = e3 x (-e2): z components only */
    const double c1 = e[1][0] * (-e[0][1]) - e[1][1] * (-e[0][0]);
    const double c2 = e[3][0] * (-e[2][1]) - e[3][1] * (-e[2][0]);
    const double a1 = fabs(c1), a2 = fabs(c2);
    const double d1 = c1 / a1, d2 = c2 / a2;    /* +1 / -1 (NaN for a degenerate corner) */
    if (d1 < 0.7 || d2 < 0.7) return -1.0;
    return 2.0 * (a1 + a2) / l;
}

static double ring_quad64(int k, const double* ring, const double* p) {
    double q = DBL_MAX;
    for (int i = 0; i < k; ++i) q = fmin(q, q_quad64(p, ring + 6 * i, ring + 6 * i + 3, ring + 6 * i + 6));
    return q;
}

static void quad2d_vertex_f64(const or_mesh* m, double* X, int v, double gs, double* margin) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    const int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) { if (margin) *margin = DBL_MAX; return; }
    double* ring = (double*)malloc(sizeof(double) * 3 * (2 * (size_t)k + 1));
    double md[2] = { 0.0, 0.0 };
    const double p0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    for (int i = 0; i < k; ++i) {
        const int u = he[4 * (b + i)], u2 = he[4 * he[4 * (b + i) + 3]];
        for (int a = 0; a < 3; ++a) { ring[6 * i + a] = X[3 * u + a]; ring[6 * i + 3 + a] = X[3 * u2 + a]; }
        for (int a = 0; a < 2; ++a) {
            md[a] = fmax(md[a], fabs(X[3 * u + a] - p0[a]));
            md[a] = fmax(md[a], fabs(X[3 * u2 + a] - p0[a]));
        }
    }
    for (int a = 0; a < 3; ++a) ring[6 * k + a] = ring[a];
    double cur[3] = { p0[0], p0[1], p0[2] };
    const double aff = 1.0 / 7.0;
    double ds = gs, lastMax = -DBL_MAX, mg = DBL_MAX;
    double qLast = ring_quad64(k, ring, cur);
    const double qOld = qLast;
    for (int d = 0; d < 3; ++d) {
        double gmax[2] = { cur[0] + ds * md[0], cur[1] + ds * md[1] }, gmin[2] = { cur[0] - ds * md[0], cur[1] - ds * md[1] };
        double bv = -DBL_MAX, best = -DBL_MAX, second = -DBL_MAX, bp[2] = { 0, 0 };
        int bt = -1;
        for (int t = 0; t < 32; ++t) {
            const int i1 = t / 8, j1 = t % 8, i2 = i1 + 4;
            const double y = aff * (j1 * gmin[1] + (7 - j1) * gmax[1]);
            const double x1 = aff * (i1 * gmin[0] + (7 - i1) * gmax[0]), x2 = aff * (i2 * gmin[0] + (7 - i2) * gmax[0]);
            const double P1[3] = { x1, y, cur[2] }, P2[3] = { x2, y, cur[2] };
            const double q1 = ring_quad64(k, ring, P1), q2 = ring_quad64(k, ring, P2);
            const double qs[2] = { q1, q2 };
            for (int s = 0; s < 2; ++s) { if (qs[s] > best) { second = best; best = qs[s]; } else if (qs[s] > second) second = qs[s]; }
            const double val = q2 > q1 ? q2 : q1;
            if (bt < 0 || val > bv) { bv = val; bt = t; bp[0] = q1 > q2 ? x1 : x2; bp[1] = y; }
        }
        mg = fmin(mg, best - second);
        mg = fmin(mg, fabs(bv - qLast));
        if (qLast < bv) { cur[0] = bp[0]; cur[1] = bp[1]; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0 / 7.0);
    }
    mg = fmin(mg, fabs(lastMax - qOld));
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; }
    if (margin) *margin = mg;
    free(ring);
}

void or_dmo_quad2d_f64(const or_mesh* m, double* X, int v0, int v1, double gs, double* margin, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) quad2d_vertex_f64(m, X, v, gs, margin ? margin + (v - v0) : NULL);
}

/* quality of a flat quad (meanRatioMetricQuad(p, +z)) in float, for the batched statistics */
float or_q_quad2d_f32(const float* p0, const float* p1, const float* p2, const float* p3) {
    const float e0x = p1[0] - p0[0], e0y = p1[1] - p0[1], e1x = p2[0] - p1[0], e1y = p2[1] - p1[1];
    const float e2x = p3[0] - p2[0], e2y = p3[1] - p2[1], e3x = p0[0] - p3[0], e3y = p0[1] - p3[1];
    const float l = (((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y)) + (e3x * e3x + e3y * e3y);
    const float c1 = e1x * (-e0y) - e1y * (-e0x);
    const float c2 = e3x * (-e2y) - e3y * (-e2x);
    if (c1 < 0.f || c2 < 0.f) return -1.f;
    return (2.f * (c1 + c2)) / l;
}

double or_q_quad2d_f64(const double* p0, const double* p1, const double* p2, const double* p3) {
    return q_quad64(p0, p1, p2, p3);
}
