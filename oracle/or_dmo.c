/*
 * or_dmo.c -- CPU restatement of the reference DMO grid search and quality metrics
 * (TEST INFRASTRUCTURE ONLY; see vsdmo_oracle.h).
 *
 * f64 functions restate the reference kernels literally, in double:
 *   k_optimizeHierarchicalInnerTet   dmo/DMOTetImplCub.h:21-137
 *   k_optimizeHierarchical2DFlat     dmo/DMOTriFlatImplCub.h:24-152
 *   meanRatioMetricTet / ring        dmo/DMOQualityTet.h:119-162
 *   meanRatioMetricTri2D / ring      dmo/DMOQualityTri.h:243-257, 297-311
 *   DMO_NQ = 8, DMO_DEPTH = 3        dmo/DMOConfig.h:4-6
 *   doIteration (fix-boundary mode)  dmo/DMOTet.cu:128-170, dmo/DMOTriFlat.cu:129-166
 *
 * f32 functions restate the same search with the product's float arithmetic, written
 * independently of the product so that the CUDA result can be compared bit for bit:
 *   - ring coordinates relative to the vertex, scaled by the power of two that brings the
 *     largest per-axis extent into [0.5, 1) (exact, so it changes no rounding);
 *   - per element: determinant affine in the candidate, det = d0 - n.p, and the sum of
 *     squared edge lengths quadratic in it, L = C - 2 s.p + k|p|^2, evaluated with fmaf in
 *     a fixed association (x, then y, then z);
 *   - the ring minimum of the mean ratio compared through the monotone transform
 *     det^2 / L^3 (tet) or A / L (triangle), kept as a fraction num/den and compared by
 *     cross-multiplication; a ring with an inverted element is keyed by its most negative
 *     determinant / area (the reference returns the negative volume / area there);
 *   - per level the best candidate is the largest key with the lowest linear candidate
 *     index (x fastest), moved to only if strictly better than the current position.
 * Compile with -ffp-contract=off so that only the written fmaf calls fuse.
 */
#include "vsdmo_oracle.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern const int* or__hf_rowptr(const or_mesh* m);
extern const int* or__hf(const or_mesh* m);
extern const int* or__he_rowptr(const or_mesh* m);
extern const int* or__he(const or_mesh* m);
extern const int* or__elems(const or_mesh* m);
extern const int* or__col(const or_mesh* m, int which);

#define NQ 8
#define DEPTH 3

/* ======================================================================================= */
/* reference metrics                                                                        */
/* ======================================================================================= */

double or_q_tet_mean_ratio_f64(const double* p0, const double* p1, const double* p2, const double* p3) {
    double e[6][3];
    for (int a = 0; a < 3; ++a) { e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p0[a]; e[2][a] = p3[a] - p0[a]; }
    double cx = e[1][1] * e[2][2] - e[1][2] * e[2][1];
    double cy = e[1][2] * e[2][0] - e[1][0] * e[2][2];
    double cz = e[1][0] * e[2][1] - e[1][1] * e[2][0];
    double volume = (1.0 / 6.0) * (e[0][0] * cx + e[0][1] * cy + e[0][2] * cz);
    if (volume < 0.0) return volume;
    double mu = cbrt(volume * volume);
    for (int a = 0; a < 3; ++a) { e[3][a] = p2[a] - p1[a]; e[4][a] = p3[a] - p1[a]; e[5][a] = p3[a] - p2[a]; }
    double l = 0.0;
    for (int i = 0; i < 6; ++i) l += e[i][0] * e[i][0] + e[i][1] * e[i][1] + e[i][2] * e[i][2];
    return 12.0 * cbrt(9.0) * mu / l;
}

float or_q_tet_mean_ratio_f32(const float* p0, const float* p1, const float* p2, const float* p3) {
    float e[6][3];
    for (int a = 0; a < 3; ++a) { e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p0[a]; e[2][a] = p3[a] - p0[a]; }
    float cx = e[1][1] * e[2][2] - e[1][2] * e[2][1];
    float cy = e[1][2] * e[2][0] - e[1][0] * e[2][2];
    float cz = e[1][0] * e[2][1] - e[1][1] * e[2][0];
    float volume = (1.f / 6.f) * ((e[0][0] * cx + e[0][1] * cy) + e[0][2] * cz);
    if (volume < 0.f) return volume;
    float mu = cbrtf(volume * volume);
    for (int a = 0; a < 3; ++a) { e[3][a] = p2[a] - p1[a]; e[4][a] = p3[a] - p1[a]; e[5][a] = p3[a] - p2[a]; }
    float l = 0.f;
    for (int i = 0; i < 6; ++i) l += (e[i][0] * e[i][0] + e[i][1] * e[i][1]) + e[i][2] * e[i][2];
    const float cbrtf9 = 2.0800838230519f;
    return ((12.f * cbrtf9) * mu) / l;
}

double or_q_tri2d_mean_ratio_f64(const double* p0, const double* p1, const double* p2) {
    const double* p[3] = { p0, p1, p2 };
    double e[3][2], l = 0.0;
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3;
        e[i][0] = p[j][0] - p[i][0]; e[i][1] = p[j][1] - p[i][1];
        l += e[i][0] * e[i][0] + e[i][1] * e[i][1];
    }
    double area = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    if (area < 0.0) return area;
    return 2.0 * sqrt(3.0) * area / l;
}

float or_q_tri2d_mean_ratio_f32(const float* p0, const float* p1, const float* p2) {
    const float* p[3] = { p0, p1, p2 };
    float e[3][2], el[3];
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3;
        e[i][0] = p[j][0] - p[i][0]; e[i][1] = p[j][1] - p[i][1];
        el[i] = e[i][0] * e[i][0] + e[i][1] * e[i][1];
    }
    float l = (el[0] + el[1]) + el[2];
    float area = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    if (area < 0.f) return area;
    return ((2.f * sqrtf(3.f)) * area) / l;
}

void or_element_qualities_f64(const or_mesh* m, const double* xyz, double* q) {
    int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    if (or__hf_rowptr(m)) {
        for (int t = 0; t < nE; ++t) {
            const int* v = el + 4 * t;
            q[t] = or_q_tet_mean_ratio_f64(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3]);
        }
    } else {
        for (int t = 0; t < nE; ++t) {
            const int* v = el + 3 * t;
            q[t] = or_q_tri2d_mean_ratio_f64(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2]);
        }
    }
}

void or_element_qualities_f32(const or_mesh* m, const float* xyz, float* q) {
    int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    if (or__hf_rowptr(m)) {
        for (int t = 0; t < nE; ++t) {
            const int* v = el + 4 * t;
            q[t] = or_q_tet_mean_ratio_f32(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3]);
        }
    } else {
        for (int t = 0; t < nE; ++t) {
            const int* v = el + 3 * t;
            q[t] = or_q_tri2d_mean_ratio_f32(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2]);
        }
    }
}

/* ======================================================================================= */
/* f64: literal restatement of the reference kernels                                        */
/* ======================================================================================= */

typedef double (*tet_metric64)(const double*, const double*, const double*, const double*);
typedef double (*tri_metric64)(const double*, const double*, const double*);

static double ring_q_tet_f64(int k, const double* ring, const double* p, tet_metric64 metric) {
    double q = DBL_MAX;
    for (int t = 0; t < k; ++t) {
        double v = metric(p, ring + 9 * t, ring + 9 * t + 3, ring + 9 * t + 6);
        q = fmin(q, v);
    }
    return q;
}

static void tet_vertex_f64(const or_mesh* m, double* X, int v, double gs, double* margin, tet_metric64 metric) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    double* ring = (double*)malloc(sizeof(double) * 9 * (size_t)k);
    double p0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    double md[3] = { -DBL_MAX, -DBL_MAX, -DBL_MAX };
    for (int t = 0; t < k; ++t) for (int j = 0; j < 3; ++j) {
        int u = hf[3 * (b + t) + j];
        for (int a = 0; a < 3; ++a) {
            ring[9 * t + 3 * j + a] = X[3 * u + a];
            md[a] = fmax(md[a], fabs(X[3 * u + a] - p0[a]));
        }
    }
    const double aff = 1.0 / (NQ - 1);
    double ds = gs;
    double cur[3] = { p0[0], p0[1], p0[2] };
    double qMax[128], pMax[128][3];
    for (int t = 0; t < 128; ++t) { qMax[t] = -DBL_MAX; pMax[t][0] = pMax[t][1] = pMax[t][2] = 0.0; }
    int w = 0;
    double mg = DBL_MAX;
    for (int d = 0; d < DEPTH; ++d) {
        double gmax[3], gmin[3];
        for (int a = 0; a < 3; ++a) { gmax[a] = cur[a] + ds * md[a]; gmin[a] = cur[a] - ds * md[a]; }
        double qLast = ring_q_tet_f64(k, ring, cur, metric);
        double best = -DBL_MAX, second = -DBL_MAX;
        for (int t = 0; t < 128; ++t) {
            for (int idx = 4 * t; idx < 4 * t + 4; ++idx) {
                int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
                double p[3];
                p[0] = aff * (i * gmin[0] + (NQ - 1 - i) * gmax[0]);
                p[1] = aff * (j * gmin[1] + (NQ - 1 - j) * gmax[1]);
                p[2] = aff * (kk * gmin[2] + (NQ - 1 - kk) * gmax[2]);
                double q = ring_q_tet_f64(k, ring, p, metric);
                if (q > best) { second = best; best = q; } else if (q > second) second = q;
                if (q > qMax[t]) { qMax[t] = q; pMax[t][0] = p[0]; pMax[t][1] = p[1]; pMax[t][2] = p[2]; }
            }
        }
        w = 0;
        for (int t = 1; t < 128; ++t) if (qMax[t] > qMax[w]) w = t;
        /* decision margins of this level: best vs runner-up, best vs current position */
        mg = fmin(mg, best - second);
        mg = fmin(mg, fabs(best - qLast));
        if (qLast < qMax[w]) { cur[0] = pMax[w][0]; cur[1] = pMax[w][1]; cur[2] = pMax[w][2]; }
        ds = ds * (2.0 / (NQ - 1));
    }
    double qOld = ring_q_tet_f64(k, ring, p0, metric);
    mg = fmin(mg, fabs(qMax[w] - qOld));
    if (qOld < qMax[w]) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    if (margin) *margin = mg;
    free(ring);
}

static double ring_q_tri2d_f64(int n1, const double* ring, const double* p, tri_metric64 metric) {
    double q = DBL_MAX;
    for (int i = 0; i < n1 - 1; ++i) q = fmin(q, metric(p, ring + 3 * i, ring + 3 * (i + 1)));
    return q;
}

static void tri2d_vertex_f64(const or_mesh* m, double* X, int v, double gs, double* margin, tri_metric64 metric) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    double* ring = (double*)malloc(sizeof(double) * 3 * ((size_t)k + 1));
    double p0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    double md[3] = { -DBL_MAX, -DBL_MAX, -DBL_MAX };
    for (int i = 0; i < k; ++i) {
        int u = he[4 * (b + i)];
        for (int a = 0; a < 3; ++a) { ring[3 * i + a] = X[3 * u + a]; md[a] = fmax(md[a], fabs(X[3 * u + a] - p0[a])); }
    }
    for (int a = 0; a < 3; ++a) ring[3 * k + a] = ring[a];
    int n1 = k + 1;
    const double aff = 1.0 / (NQ - 1);
    double ds = gs;
    double cur[3] = { p0[0], p0[1], p0[2] };
    double lastMax = -DBL_MAX, mg = DBL_MAX;
    for (int d = 0; d < DEPTH; ++d) {
        double gmax[2], gmin[2];
        for (int a = 0; a < 2; ++a) { gmax[a] = cur[a] + ds * md[a]; gmin[a] = cur[a] - ds * md[a]; }
        double qLast = ring_q_tri2d_f64(n1, ring, cur, metric);
        double val[32], pp[32][2];
        double best = -DBL_MAX, second = -DBL_MAX;
        for (int t = 0; t < 32; ++t) {
            int i1 = t / NQ, j1 = t % NQ, i2 = i1 + 4;
            double p1[3] = { aff * (i1 * gmin[0] + (NQ - 1 - i1) * gmax[0]), aff * (j1 * gmin[1] + (NQ - 1 - j1) * gmax[1]), cur[2] };
            double p2[3] = { aff * (i2 * gmin[0] + (NQ - 1 - i2) * gmax[0]), aff * (j1 * gmin[1] + (NQ - 1 - j1) * gmax[1]), cur[2] };
            double q1 = ring_q_tri2d_f64(n1, ring, p1, metric), q2 = ring_q_tri2d_f64(n1, ring, p2, metric);
            val[t] = q1; if (q2 > q1) val[t] = q2;
            if (q1 > q2) { pp[t][0] = p1[0]; pp[t][1] = p1[1]; } else { pp[t][0] = p2[0]; pp[t][1] = p2[1]; }
            double qs[2] = { q1, q2 };
            for (int s = 0; s < 2; ++s) { if (qs[s] > best) { second = best; best = qs[s]; } else if (qs[s] > second) second = qs[s]; }
        }
        int w = 0;
        for (int t = 1; t < 32; ++t) if (val[t] > val[w]) w = t;
        mg = fmin(mg, best - second);
        mg = fmin(mg, fabs(best - qLast));
        if (qLast < val[w]) { cur[0] = pp[w][0]; cur[1] = pp[w][1]; }
        lastMax = val[w];
        ds = ds * (2.0 / (NQ - 1));
    }
    double qOld = ring_q_tri2d_f64(n1, ring, p0, metric);
    mg = fmin(mg, fabs(lastMax - qOld));
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; }
    if (margin) *margin = mg;
    free(ring);
}

void or_dmo_tet_f64(const or_mesh* m, double* xyz, int v0, int v1, double gs, double* margin, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) tet_vertex_f64(m, xyz, v, gs, margin ? margin + (v - v0) : NULL, or_q_tet_mean_ratio_f64);
}

void or_dmo_tri2d_f64(const or_mesh* m, double* xyz, int v0, int v1, double gs, double* margin, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) tri2d_vertex_f64(m, xyz, v, gs, margin ? margin + (v - v0) : NULL, or_q_tri2d_mean_ratio_f64);
}

/* literal float restatement of k_optimizeHierarchicalInnerTet (the reference's own FP32
 * arithmetic with cbrtf per element): the CPU baseline that bench.py times.                  */
static float ring_q_tet_ref32(int k, const float* ring, const float* p) {
    float q = FLT_MAX;
    for (int t = 0; t < k; ++t) q = fminf(q, or_q_tet_mean_ratio_f32(p, ring + 9 * t, ring + 9 * t + 3, ring + 9 * t + 6));
    return q;
}

static void tet_vertex_ref32(const or_mesh* m, float* X, int v, float gs) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    float* ring = (float*)malloc(sizeof(float) * 9 * (size_t)k);
    float p0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float md[3] = { -FLT_MAX, -FLT_MAX, -FLT_MAX };
    for (int t = 0; t < k; ++t) for (int j = 0; j < 3; ++j) {
        int u = hf[3 * (b + t) + j];
        for (int a = 0; a < 3; ++a) { ring[9 * t + 3 * j + a] = X[3 * u + a]; md[a] = fmaxf(md[a], fabsf(X[3 * u + a] - p0[a])); }
    }
    const float aff = 1.f / (float)(NQ - 1);
    float ds = gs, cur[3] = { p0[0], p0[1], p0[2] };
    float qMax[128], pMax[128][3];
    for (int t = 0; t < 128; ++t) { qMax[t] = -FLT_MAX; pMax[t][0] = pMax[t][1] = pMax[t][2] = 0.f; }
    int w = 0;
    for (int d = 0; d < DEPTH; ++d) {
        float gmax[3], gmin[3];
        for (int a = 0; a < 3; ++a) { gmax[a] = cur[a] + ds * md[a]; gmin[a] = cur[a] - ds * md[a]; }
        float qLast = ring_q_tet_ref32(k, ring, cur);
        for (int t = 0; t < 128; ++t)
            for (int idx = 4 * t; idx < 4 * t + 4; ++idx) {
                int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
                float p[3] = { aff * (i * gmin[0] + (NQ - 1 - i) * gmax[0]), aff * (j * gmin[1] + (NQ - 1 - j) * gmax[1]),
                               aff * (kk * gmin[2] + (NQ - 1 - kk) * gmax[2]) };
                float q = ring_q_tet_ref32(k, ring, p);
                if (q > qMax[t]) { qMax[t] = q; pMax[t][0] = p[0]; pMax[t][1] = p[1]; pMax[t][2] = p[2]; }
            }
        w = 0;
        for (int t = 1; t < 128; ++t) if (qMax[t] > qMax[w]) w = t;
        if (qLast < qMax[w]) { cur[0] = pMax[w][0]; cur[1] = pMax[w][1]; cur[2] = pMax[w][2]; }
        ds = ds * (2.f / (NQ - 1));
    }
    float qOld = ring_q_tet_ref32(k, ring, p0);
    if (qOld < qMax[w]) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    free(ring);
}

void or_dmo_tet_ref32(const or_mesh* m, float* xyz, int v0, int v1, float gs, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) tet_vertex_ref32(m, xyz, v, gs);
}

/* ======================================================================================= */
/* f32: the product's arithmetic                                                            */
/* ======================================================================================= */

static inline float grid_offset(int i) { return (float)(NQ - 1 - 2 * i) / (float)(NQ - 1); }

/* per tet: (nn.x, nn.y, nn.z, d0) and (m.x, m.y, m.z, C) from scaled a, b, c */
static void tet_coeffs(const float* a, const float* b, const float* c, float* K) {
    float ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
    float wx = c[0] - a[0], wy = c[1] - a[1], wz = c[2] - a[2];
    float vx = c[0] - b[0], vy = c[1] - b[1], vz = c[2] - b[2];
    float nx = uy * wz - uz * wy;
    float ny = uz * wx - ux * wz;
    float nz = ux * wy - uy * wx;
    float d0 = (a[0] * nx + a[1] * ny) + a[2] * nz;
    float sx = (a[0] + b[0]) + c[0], sy = (a[1] + b[1]) + c[1], sz = (a[2] + b[2]) + c[2];
    float a2 = (a[0] * a[0] + a[1] * a[1]) + a[2] * a[2];
    float b2 = (b[0] * b[0] + b[1] * b[1]) + b[2] * b[2];
    float c2 = (c[0] * c[0] + c[1] * c[1]) + c[2] * c[2];
    float u2 = (ux * ux + uy * uy) + uz * uz;
    float w2 = (wx * wx + wy * wy) + wz * wz;
    float v2 = (vx * vx + vy * vy) + vz * vz;
    K[0] = -nx; K[1] = -ny; K[2] = -nz; K[3] = d0;
    K[4] = -2.0f * sx; K[5] = -2.0f * sy; K[6] = -2.0f * sz;
    K[7] = ((((a2 + b2) + c2) + u2) + w2) + v2;
}

static float tet_key(int k, const float* K, float x, float y, float z) {
    float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    float N = 0.f, D = 1.f, dmin = 0.f;
    for (int t = 0; t < k; ++t) {
        const float* c = K + 8 * t;
        float detA = fmaf(c[0], x, c[3]);
        float LA = c[7] + fmaf(c[4], x, tx);
        float detB = fmaf(c[1], y, detA);
        float LB = LA + fmaf(c[5], y, ty);
        float det = fmaf(c[2], z, detB);
        float L = LB + fmaf(c[6], z, tz);
        float num = det * det;
        float den = (L * L) * L;
        if (t == 0) { N = num; D = den; dmin = det; continue; }
        if (num * D < N * den) { N = num; D = den; }
        dmin = fminf(dmin, det);
    }
    return dmin < 0.f ? dmin : N / D;
}

static void tet_vertex_f32(const or_mesh* m, float* X, int v, float gs) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float* r = (float*)malloc(sizeof(float) * 9 * (size_t)k);
    float* K = (float*)malloc(sizeof(float) * 8 * (size_t)k);
    float md[3] = { 0.f, 0.f, 0.f };
    for (int t = 0; t < k; ++t) for (int j = 0; j < 3; ++j) {
        int u = hf[3 * (b + t) + j];
        for (int a = 0; a < 3; ++a) {
            float d = X[3 * u + a] - c0[a];
            r[9 * t + 3 * j + a] = d;
            md[a] = fmaxf(md[a], fabsf(d));
        }
    }
    float mm = fmaxf(md[0], fmaxf(md[1], md[2]));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) { free(r); free(K); return; }
    int ex; (void)frexpf(mm, &ex);
    for (int i = 0; i < 9 * k; ++i) r[i] = ldexpf(r[i], -ex);
    for (int a = 0; a < 3; ++a) md[a] = ldexpf(md[a], -ex);
    for (int t = 0; t < k; ++t) tet_coeffs(r + 9 * t, r + 9 * t + 3, r + 9 * t + 6, K + 8 * t);
    float dlt[3] = { 0.f, 0.f, 0.f };
    float qLast = tet_key(k, K, 0.f, 0.f, 0.f);
    int moved = 0;
    float ds = gs;
    for (int d = 0; d < DEPTH; ++d) {
        float xs[NQ], ys[NQ], zs[NQ];
        float Sx = ds * md[0], Sy = ds * md[1], Sz = ds * md[2];
        for (int i = 0; i < NQ; ++i) {
            float o = grid_offset(i);
            xs[i] = fmaf(o, Sx, dlt[0]); ys[i] = fmaf(o, Sy, dlt[1]); zs[i] = fmaf(o, Sz, dlt[2]);
        }
        float best = -FLT_MAX; int bi = -1;
        for (int idx = 0; idx < NQ * NQ * NQ; ++idx) {
            int i = idx % NQ, j = (idx / NQ) % NQ, kk = idx / (NQ * NQ);
            float q = tet_key(k, K, xs[i], ys[j], zs[kk]);
            if (q > best) { best = q; bi = idx; }
        }
        if (bi >= 0 && qLast < best) {
            dlt[0] = xs[bi % NQ]; dlt[1] = ys[(bi / NQ) % NQ]; dlt[2] = zs[bi / (NQ * NQ)];
            qLast = best; moved = 1;
        }
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    if (moved) {
        X[3 * v] = c0[0] + ldexpf(dlt[0], ex);
        X[3 * v + 1] = c0[1] + ldexpf(dlt[1], ex);
        X[3 * v + 2] = c0[2] + ldexpf(dlt[2], ex);
    }
    free(r); free(K);
}

/* ---- learned reduced search (the product's addition; restated from its design) ---------- */
/* The network's displacement y (units of the largest per-axis ring extent) centres a grid of
 * rn^3 candidates per level, rdepth levels, offsets (rn-1-2i)/(rn-1), first half-extent
 * grid_scale * rscale * the per-axis extent, shrinking by 2/(rn-1); the proposal is clamped to
 * +-grid_scale * extent per axis. Keys: the ring minimum of the per-tet keys (det if negative,
 * else det^2 / L^3) for the current position and the proposal, the ordered fraction minimum
 * (tet_key) for the grid candidates; the best candidate of a level (largest key, lowest index
 * on ties) becomes the centre when it beats the best so far. The vertex moves when the best
 * beats the key of its current position; otherwise it is queued for the plain search.
 * With rn = 4 the candidates are ranked by the ordered fraction minimum over the 8 tets of
 * smallest per-tet key at the level's centre (picked by the order key of the float with the
 * tet index in its low 5 bits, ties to the lower tet), and the best-ranked candidate counts
 * with its ring minimum of the per-tet keys. */
static float tet_key_piecemin(int k, const float* K, float x, float y, float z) {
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    float m = FLT_MAX;
    for (int t = 0; t < k; ++t) {
        const float* c = K + 8 * t;
        const float det = fmaf(c[2], z, fmaf(c[1], y, fmaf(c[0], x, c[3])));
        const float L = ((c[7] + fmaf(c[4], x, tx)) + fmaf(c[5], y, ty)) + fmaf(c[6], z, tz);
        m = fminf(m, det < 0.f ? det : (det * det) / ((L * L) * L));
    }
    return m;
}

#define LEARNED_CRIT 8

static float tet_piece_key_at(const float* c, float x, float y, float z) {
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    const float det = fmaf(c[2], z, fmaf(c[1], y, fmaf(c[0], x, c[3])));
    const float L = ((c[7] + fmaf(c[4], x, tx)) + fmaf(c[5], y, ty)) + fmaf(c[6], z, tz);
    return det < 0.f ? det : (det * det) / ((L * L) * L);
}

/* float order as unsigned order, the low 5 bits replaced by t & 31 */
static uint32_t tet_order_key(float key, int t) {
    uint32_t b;
    memcpy(&b, &key, sizeof b);
    const uint32_t o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return (o & ~31u) | (uint32_t)(t & 31);
}

/* the min(LEARNED_CRIT, k) tets of smallest (order key, tet) at (x, y, z) */
static int learned_critical(int k, const float* K, float x, float y, float z, int* crit) {
    const int nt = k < LEARNED_CRIT ? k : LEARNED_CRIT;
    for (int r = 0; r < nt; ++r) {
        uint32_t best = 0xffffffffu;
        int bt = -1;
        for (int t = 0; t < k; ++t) {
            int used = 0;
            for (int q = 0; q < r; ++q) used |= crit[q] == t;
            if (used) continue;
            const uint32_t kt = tet_order_key(tet_piece_key_at(K + 8 * t, x, y, z), t);
            if (bt < 0 || kt < best) { best = kt; bt = t; }
        }
        crit[r] = bt;
    }
    return nt;
}

/* tet_key over the tets crit[0 .. nt) in that order */
static float tet_key_subset(const int* crit, int nt, const float* K, float x, float y, float z) {
    const float tx = (3.0f * x) * x, ty = (3.0f * y) * y, tz = (3.0f * z) * z;
    float N = 0.f, D = 1.f, dmin = 0.f;
    for (int r = 0; r < nt; ++r) {
        const float* c = K + 8 * crit[r];
        const float det = fmaf(c[2], z, fmaf(c[1], y, fmaf(c[0], x, c[3])));
        const float L = ((c[7] + fmaf(c[4], x, tx)) + fmaf(c[5], y, ty)) + fmaf(c[6], z, tz);
        const float n = det * det, d = (L * L) * L;
        if (r == 0) { N = n; D = d; dmin = det; continue; }
        if (n * D < N * d) { N = n; D = d; }
        dmin = fminf(dmin, det);
    }
    return dmin < 0.f ? dmin : N / D;
}

static int tet_learned_vertex_f32(const or_mesh* m, float* X, int v, const float* yv, float gs, int rn, int rdepth,
                                  float rscale) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return 0;
    float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float* r = (float*)malloc(sizeof(float) * 9 * (size_t)k);
    float* K = (float*)malloc(sizeof(float) * 8 * (size_t)k);
    float md[3] = { 0.f, 0.f, 0.f };
    for (int t = 0; t < k; ++t) for (int j = 0; j < 3; ++j) {
        int u = hf[3 * (b + t) + j];
        for (int a = 0; a < 3; ++a) {
            float d = X[3 * u + a] - c0[a];
            r[9 * t + 3 * j + a] = d;
            md[a] = fmaxf(md[a], fabsf(d));
        }
    }
    float mm = fmaxf(md[0], fmaxf(md[1], md[2]));
    if (!(mm > 0.f) || !(mm < FLT_MAX)) { free(r); free(K); return 0; }
    int ex; (void)frexpf(mm, &ex);
    for (int i = 0; i < 9 * k; ++i) r[i] = ldexpf(r[i], -ex);
    for (int a = 0; a < 3; ++a) md[a] = ldexpf(md[a], -ex);
    for (int t = 0; t < k; ++t) tet_coeffs(r + 9 * t, r + 9 * t + 3, r + 9 * t + 6, K + 8 * t);
    const float q0 = tet_key_piecemin(k, K, 0.f, 0.f, 0.f);
    const float mms = fmaxf(md[0], fmaxf(md[1], md[2]));
    float p[3] = { yv[0] * mms, yv[1] * mms, yv[2] * mms };
    const int have = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
    float best = -FLT_MAX, c[3] = { 0.f, 0.f, 0.f };
    if (have) {
        for (int a = 0; a < 3; ++a) { const float bnd = gs * md[a]; p[a] = fminf(fmaxf(p[a], -bnd), bnd); c[a] = p[a]; }
        best = tet_key_piecemin(k, K, p[0], p[1], p[2]);
        float rr[3] = { gs * rscale * md[0], gs * rscale * md[1], gs * rscale * md[2] };
        const int nc = rn * rn * rn;
        for (int level = 0; level < rdepth; ++level) {
            float bk = -FLT_MAX;
            int bi = -1;
            int crit[LEARNED_CRIT], nt = 0;
            if (rn == 4) nt = learned_critical(k, K, c[0], c[1], c[2], crit);
            for (int ci = 0; ci < nc; ++ci) {
                const int ix = ci % rn, iy = (ci / rn) % rn, iz = ci / (rn * rn);
                const float x = fmaf((float)(rn - 1 - 2 * ix) / (float)(rn - 1), rr[0], c[0]);
                const float y = fmaf((float)(rn - 1 - 2 * iy) / (float)(rn - 1), rr[1], c[1]);
                const float z = fmaf((float)(rn - 1 - 2 * iz) / (float)(rn - 1), rr[2], c[2]);
                const float q = rn == 4 ? tet_key_subset(crit, nt, K, x, y, z) : tet_key(k, K, x, y, z);
                if (bi < 0 || q > bk) { bk = q; bi = ci; }
            }
            if (rn == 4 && bk > best) {
                const int ix = bi % rn, iy = (bi / rn) % rn, iz = bi / (rn * rn);
                bk = tet_key_piecemin(k, K, fmaf((float)(rn - 1 - 2 * ix) / (float)(rn - 1), rr[0], c[0]),
                                      fmaf((float)(rn - 1 - 2 * iy) / (float)(rn - 1), rr[1], c[1]),
                                      fmaf((float)(rn - 1 - 2 * iz) / (float)(rn - 1), rr[2], c[2]));
            }
            if (bk > best) {
                const int ix = bi % rn, iy = (bi / rn) % rn, iz = bi / (rn * rn);
                const float n0 = fmaf((float)(rn - 1 - 2 * ix) / (float)(rn - 1), rr[0], c[0]);
                const float n1 = fmaf((float)(rn - 1 - 2 * iy) / (float)(rn - 1), rr[1], c[1]);
                const float n2 = fmaf((float)(rn - 1 - 2 * iz) / (float)(rn - 1), rr[2], c[2]);
                c[0] = n0; c[1] = n1; c[2] = n2;
                best = bk;
            }
            const float sh = 2.0f / (float)(rn - 1);
            rr[0] *= sh; rr[1] *= sh; rr[2] *= sh;
        }
    }
    int moved = 0;
    if (have && best > q0) {
        X[3 * v] = c0[0] + ldexpf(c[0], ex);
        X[3 * v + 1] = c0[1] + ldexpf(c[1], ex);
        X[3 * v + 2] = c0[2] + ldexpf(c[2], ex);
        moved = 1;
    }
    free(r); free(K);
    return moved;
}

/* one colour class [v0, v1) of the learned mode: the reduced search with proposals Y
 * [(v1 - v0) x ldy], then the plain search (tet_vertex_f32) of the vertices it did not move;
 * queued[i] = 1 for those */
void or_dmo_tet_learned_f32(const or_mesh* m, float* X, int v0, int v1, const float* Y, int ldy, float gs, int rn,
                            int rdepth, float rscale, uint8_t* queued, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) {
        const int mv = tet_learned_vertex_f32(m, X, v, Y + (size_t)(v - v0) * ldy, gs, rn, rdepth, rscale);
        if (queued) queued[v - v0] = (uint8_t)!mv;
        if (!mv) tet_vertex_f32(m, X, v, gs);
    }
}

/* per triangle (p, a, b): (nA.x, nA.y, A0, m.x, m.y, C) */
static void tri_coeffs(const float* a, const float* b, float* K) {
    float ux = b[0] - a[0], uy = b[1] - a[1];
    K[0] = -uy; K[1] = ux;
    K[2] = a[0] * uy - a[1] * ux;
    K[3] = -2.0f * (a[0] + b[0]); K[4] = -2.0f * (a[1] + b[1]);
    K[5] = ((a[0] * a[0] + a[1] * a[1]) + (b[0] * b[0] + b[1] * b[1])) + (ux * ux + uy * uy);
}

static float tri_key(int k, const float* K, float x, float y) {
    float tx = (2.0f * x) * x, ty = (2.0f * y) * y;
    float N = 0.f, D = 1.f, amin = 0.f;
    for (int t = 0; t < k; ++t) {
        const float* c = K + 6 * t;
        float A = fmaf(c[1], y, fmaf(c[0], x, c[2]));
        float L = (c[5] + fmaf(c[3], x, tx)) + fmaf(c[4], y, ty);
        if (t == 0) { N = A; D = L; amin = A; continue; }
        if (A * D < N * L) { N = A; D = L; }
        amin = fminf(amin, A);
    }
    return amin < 0.f ? amin : N / D;
}

static void tri2d_vertex_f32(const or_mesh* m, float* X, int v, float gs) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float* r = (float*)malloc(sizeof(float) * 2 * ((size_t)k + 1));
    float* K = (float*)malloc(sizeof(float) * 6 * (size_t)k);
    float md[2] = { 0.f, 0.f };
    for (int i = 0; i < k; ++i) {
        int u = he[4 * (b + i)];
        for (int a = 0; a < 2; ++a) { float d = X[3 * u + a] - c0[a]; r[2 * i + a] = d; md[a] = fmaxf(md[a], fabsf(d)); }
    }
    float mm = fmaxf(md[0], md[1]);
    if (!(mm > 0.f) || !(mm < FLT_MAX)) { free(r); free(K); return; }
    int ex; (void)frexpf(mm, &ex);
    for (int i = 0; i < 2 * k; ++i) r[i] = ldexpf(r[i], -ex);
    r[2 * k] = r[0]; r[2 * k + 1] = r[1];
    md[0] = ldexpf(md[0], -ex); md[1] = ldexpf(md[1], -ex);
    for (int t = 0; t < k; ++t) tri_coeffs(r + 2 * t, r + 2 * t + 2, K + 6 * t);
    float dlt[2] = { 0.f, 0.f };
    float qOld = tri_key(k, K, 0.f, 0.f);
    float qLast = qOld, lastMax = -FLT_MAX;
    float ds = gs;
    for (int d = 0; d < DEPTH; ++d) {
        float xs[NQ], ys[NQ];
        float Sx = ds * md[0], Sy = ds * md[1];
        for (int i = 0; i < NQ; ++i) { float o = grid_offset(i); xs[i] = fmaf(o, Sx, dlt[0]); ys[i] = fmaf(o, Sy, dlt[1]); }
        float bv = 0.f; int bt = -1; float bx = 0.f, by = 0.f;
        for (int t = 0; t < 32; ++t) {
            int i1 = t / NQ, j1 = t % NQ, i2 = i1 + 4;
            float q1 = tri_key(k, K, xs[i1], ys[j1]);
            float q2 = tri_key(k, K, xs[i2], ys[j1]);
            float val = q1; if (q2 > q1) val = q2;
            if (bt < 0 || val > bv) {
                bv = val; bt = t;
                if (q1 > q2) { bx = xs[i1]; by = ys[j1]; } else { bx = xs[i2]; by = ys[j1]; }
            }
        }
        if (qLast < bv) { dlt[0] = bx; dlt[1] = by; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    if (qOld < lastMax) {
        X[3 * v] = c0[0] + ldexpf(dlt[0], ex);
        X[3 * v + 1] = c0[1] + ldexpf(dlt[1], ex);
    }
    free(r); free(K);
}

void or_dmo_tet_f32(const or_mesh* m, float* xyz, int v0, int v1, float gs, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) tet_vertex_f32(m, xyz, v, gs);
}

void or_dmo_tri2d_f32(const or_mesh* m, float* xyz, int v0, int v1, float gs, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int v = v0; v < v1; ++v) tri2d_vertex_f32(m, xyz, v, gs);
}

/* ======================================================================================= */
/* optimisation loops (fix-boundary mode)                                                   */
/* ======================================================================================= */

static void stats_f64(const double* q, int n, double* mn, double* mean) {
    double a = DBL_MAX, s = 0.0;
    for (int i = 0; i < n; ++i) { a = fmin(a, q[i]); s += q[i]; }
    *mn = a; *mean = s / n;
}

void or_optimize_f32(const or_mesh* m, float* xyz, int n_iter, float gs, int nthreads, double* min_hist, double* mean_hist) {
    int isTet = or__hf_rowptr(m) != NULL;
    int nE = or_mesh_info(m, OR_I_NE);
    int nc = isTet ? or_mesh_info(m, OR_I_NCOL_INNER) : or_mesh_info(m, OR_I_NCOL_FREE);
    const int* off = isTet ? or__col(m, 2) : or__col(m, 0);
    float* q = (float*)malloc(sizeof(float) * (size_t)nE);
    double* qd = (double*)malloc(sizeof(double) * (size_t)nE);
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) {
            if (isTet) or_dmo_tet_f32(m, xyz, off[c], off[c + 1], gs, nthreads);
            else or_dmo_tri2d_f32(m, xyz, off[c], off[c + 1], gs, nthreads);
        }
        if (min_hist || mean_hist) {
            or_element_qualities_f32(m, xyz, q);
            for (int i = 0; i < nE; ++i) qd[i] = q[i];
            double mn, mean; stats_f64(qd, nE, &mn, &mean);
            if (min_hist) min_hist[it] = mn;
            if (mean_hist) mean_hist[it] = mean;
        }
    }
    free(q); free(qd);
}

void or_optimize_f64(const or_mesh* m, double* xyz, int n_iter, double gs, int nthreads, double* min_hist, double* mean_hist) {
    int isTet = or__hf_rowptr(m) != NULL;
    int nE = or_mesh_info(m, OR_I_NE);
    int nc = isTet ? or_mesh_info(m, OR_I_NCOL_INNER) : or_mesh_info(m, OR_I_NCOL_FREE);
    const int* off = isTet ? or__col(m, 2) : or__col(m, 0);
    double* q = (double*)malloc(sizeof(double) * (size_t)nE);
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) {
            if (isTet) or_dmo_tet_f64(m, xyz, off[c], off[c + 1], gs, NULL, nthreads);
            else or_dmo_tri2d_f64(m, xyz, off[c], off[c + 1], gs, NULL, nthreads);
        }
        if (min_hist || mean_hist) {
            or_element_qualities_f64(m, xyz, q);
            double mn, mean; stats_f64(q, nE, &mn, &mean);
            if (min_hist) min_hist[it] = mn;
            if (mean_hist) mean_hist[it] = mean;
        }
    }
    free(q);
}


/* ======================================================================================= */
/* angle criteria (MIN_ANGLE / MAX_ANGLE), literal in double                                */
/* minAngleMetricTri2D / maxAngleMetricTri2D (dmo/DMOQualityTri.h:10-29,124-144),            */
/* minAngleMetricTet / maxAngleMetricTet (dmo/DMOQualityTet.h:10-37,62-91), calcAngle        */
/* (dmo/DMOQualityUtil.h:30-50): angles by acos of dot / sqrt(|u|^2 |v|^2).                  */
/* ======================================================================================= */

static double calc_angle(const double* u, const double* v, int dim) {
    double d = 0.0, uu = 0.0, vv = 0.0;
    for (int a = 0; a < dim; ++a) { d += u[a] * v[a]; uu += u[a] * u[a]; vv += v[a] * v[a]; }
    return acos(d / sqrt(uu * vv));
}

static double tri2d_angle64(const double* p0, const double* p1, const double* p2, int max_angle) {
    const double e0[2] = { p1[0] - p0[0], p1[1] - p0[1] }, e1[2] = { p2[0] - p1[0], p2[1] - p1[1] };
    const double area = e0[0] * e1[1] - e0[1] * e1[0];
    if (area < 0.0) return area;
    const double a0[2] = { p0[0] - p1[0], p0[1] - p1[1] }, a1[2] = { p2[0] - p1[0], p2[1] - p1[1] };
    const double b0[2] = { p1[0] - p2[0], p1[1] - p2[1] }, b1[2] = { p0[0] - p2[0], p0[1] - p2[1] };
    const double c0[2] = { p2[0] - p0[0], p2[1] - p0[1] }, c1[2] = { p1[0] - p0[0], p1[1] - p0[1] };
    const double a = calc_angle(a0, a1, 2), b = calc_angle(b0, b1, 2), c = calc_angle(c0, c1, 2);
    if (max_angle) return 1.0 - fmax(fmax(a, b), c) / M_PI;
    return 3.0 * fmin(fmin(a, b), c) / M_PI;
}
/* minAngleMetricTri(p, n) / maxAngleMetricTri(p, n) (dmo/DMOQualityTri.h:50-71,166-189); n == NULL:
 * the unsigned metric (minAngleMetricTri(p), :31-47) */
double or_q_tri3d_angle_f64(const double* p0, const double* p1, const double* p2, const double* n, int max_angle) {
    double a0[3], a1[3], b0[3], b1[3], c0[3], c1[3], e0[3], e1[3];
    for (int i = 0; i < 3; ++i) {
        a0[i] = p0[i] - p1[i]; a1[i] = p2[i] - p1[i];
        b0[i] = p1[i] - p2[i]; b1[i] = p0[i] - p2[i];
        c0[i] = p2[i] - p0[i]; c1[i] = p1[i] - p0[i];
        e0[i] = p1[i] - p0[i]; e1[i] = p2[i] - p1[i];
    }
    const double a = calc_angle(a0, a1, 3), b = calc_angle(b0, b1, 3), c = calc_angle(c0, c1, 3);
    double q = max_angle ? 1.0 - fmax(fmax(a, b), c) / M_PI : 3.0 * fmin(fmin(a, b), c) / M_PI;
    if (n) {
        const double t[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
        const double len = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        if ((t[0] / len) * n[0] + (t[1] / len) * n[1] + (t[2] / len) * n[2] < 0.0) q = -q;
    }
    return q;
}

/* the quality criterion of the surface, 1D and boundary restatements (OR_MEAN_RATIO,
 * OR_MIN_ANGLE, OR_MAX_ANGLE); process-wide test state, set before the calls it governs */
static int g_criterion = 0;
void or_set_criterion(int c) { g_criterion = c; }
int or__criterion(void) { return g_criterion; }

double or_q_tri2d_min_angle_f64(const double* p0, const double* p1, const double* p2) { return tri2d_angle64(p0, p1, p2, 0); }
double or_q_tri2d_max_angle_f64(const double* p0, const double* p1, const double* p2) { return tri2d_angle64(p0, p1, p2, 1); }

static void cross64(const double* u, const double* v, double* o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
}

static double tet_angle64(const double* p0, const double* p1, const double* p2, const double* p3, int max_angle) {
    double e[6][3], n[4][3];
    for (int a = 0; a < 3; ++a) {
        e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p0[a]; e[2][a] = p3[a] - p0[a];
        e[3][a] = p2[a] - p1[a]; e[4][a] = p3[a] - p1[a]; e[5][a] = p3[a] - p2[a];
    }
    double x[3];
    cross64(e[1], e[2], x);
    const double vol = (e[0][0] * x[0] + e[0][1] * x[1] + e[0][2] * x[2]) / 6.0;
    if (vol < 0.0) return vol;
    cross64(e[0], e[2], n[0]); cross64(e[3], e[4], n[1]); cross64(e[1], e[0], n[2]); cross64(e[2], e[1], n[3]);
    for (int i = 0; i < 4; ++i) {
        const double l = sqrt(n[i][0] * n[i][0] + n[i][1] * n[i][1] + n[i][2] * n[i][2]);
        for (int a = 0; a < 3; ++a) n[i][a] /= l;
    }
    const int P[6][2] = { { 0, 1 }, { 0, 2 }, { 0, 3 }, { 1, 2 }, { 1, 3 }, { 2, 3 } };
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int q = 0; q < 6; ++q) {
        const double m[3] = { -n[P[q][0]][0], -n[P[q][0]][1], -n[P[q][0]][2] };
        const double ang = calc_angle(m, n[P[q][1]], 3);
        mn = fmin(mn, ang); mx = fmax(mx, ang);
    }
    if (max_angle) return 1.0 - mx / M_PI;
    return 3.0 * mn / M_PI;
}
double or_q_tet_min_angle_f64(const double* p0, const double* p1, const double* p2, const double* p3) { return tet_angle64(p0, p1, p2, p3, 0); }
double or_q_tet_max_angle_f64(const double* p0, const double* p1, const double* p2, const double* p3) { return tet_angle64(p0, p1, p2, p3, 1); }

void or_dmo_angle_f64(const or_mesh* m, double* xyz, int v0, int v1, double gs, int max_angle, double* margin, int nthreads) {
    const int tet = or__hf_rowptr(m) != NULL;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) {
        double* mg = margin ? margin + (v - v0) : NULL;
        if (tet) tet_vertex_f64(m, xyz, v, gs, mg, max_angle ? or_q_tet_max_angle_f64 : or_q_tet_min_angle_f64);
        else tri2d_vertex_f64(m, xyz, v, gs, mg, max_angle ? or_q_tri2d_max_angle_f64 : or_q_tri2d_min_angle_f64);
    }
}

void or_angle_qualities_f64(const or_mesh* m, const double* xyz, int max_angle, double* q) {
    const int nE = or_mesh_info(m, OR_I_NE);
    const int* el = or__elems(m);
    for (int t = 0; t < nE; ++t) {
        if (or__hf_rowptr(m)) {
            const int* v = el + 4 * t;
            q[t] = tet_angle64(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], xyz + 3 * v[3], max_angle);
        } else {
            const int* v = el + 3 * t;
            q[t] = tri2d_angle64(xyz + 3 * v[0], xyz + 3 * v[1], xyz + 3 * v[2], max_angle);
        }
    }
}

/* the f32 tet ring key for the boundary-surface passes (or_surf.c, or_feat.c) */
void or__tet_coeffs_f32(const float* a, const float* b, const float* c, float* K) { tet_coeffs(a, b, c, K); }
float or__tet_key_f32(int k, const float* K, float x, float y, float z) { return tet_key(k, K, x, y, z); }
