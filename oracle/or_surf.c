/*
 * or_surf.c -- CPU restatement of the reference's surface DMO (TEST INFRASTRUCTURE ONLY;
 * see vsdmo_oracle.h).
 *
 * f64 functions restate the reference literally, in double:
 *   computeLocalCoordinates                 dmo/surfaceP/Surface.h:66-93
 *   computeLocalSurface1 / 2 (quadric fit)  dmo/surfaceP/Surface.cu:11-104 with the 3x3 normal
 *                                           equations solved by LU with partial pivoting (the
 *                                           reference calls cublasSgetrf/getrsBatched,
 *                                           Surface.h:144-168; the published LAPACK algorithm is
 *                                           restated, the library's internals are not used)
 *   localSurfaceEstimationWithFeature       dmo/SurfaceEstimation.h:122-197 (surfaces without
 *                                           feature vertices)
 *   k_optimizeHierarchical2D (tri)          dmo/DMOTriImplCub.h:26-201
 *   k_optimizeHierarchical2D (quad)         dmo/DMOQuadImplCub.h:24-209
 *   meanRatioMetricTri(p, n) / (p)          dmo/DMOQualityTri.h:260-293
 *   meanRatioMetricQuad(p, n) / (p)         dmo/DMOQualityQuad.h:13-50
 *   k_updateNearestNeighbor                 dmo/DMOCommon.cu:11-42
 *   updateNormals                           mesh/DMOMeshTri.h:62-71 (k_calcFaceNormals /
 *                                           k_calcVertexNormals, mesh/MeshGPUCommon.cu:363-434)
 *   DMOTriClass / DMOQuadClass::doIteration dmo/DMOTri.cu:129-165, dmo/DMOQuad.cu:125-162
 *
 * f32 functions restate the same with the product's float arithmetic (written independently
 * of the product): projections with explicit operation order, the blended position
 * accumulated as sum(p_i w_i) * (1 / sum w_i), the signed triangle mean ratio compared as
 * sign(n_t . n) |n_t|^2 / L^2 (monotone in the reference value q = 2 sqrt3 sign |n_t| / L) by
 * cross-multiplication, quads evaluated with the reference formula.
 */
#include "vsdmo_oracle.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

extern const int* or__he_rowptr(const or_mesh* m);
extern const int* or__he(const or_mesh* m);
extern const int* or__col(const or_mesh* m, int which);
extern const int* or__faces(const or_mesh* m);
extern int or__fk(const or_mesh* m);

#define NQ 8
#define DEPTH 3
#define EPS 1.19209e-07f
#define LSF 16   /* floats per local surface: p0[3] a, e0[3] b, e1[3] c, e2[3] numPoints */

/* ======================================================================================== */
/* normals (reference order)                                                                 */
/* ======================================================================================== */
void or_surface_normals_f32(const or_mesh* m, const float* X, float* fn, float* vn) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nF = or_mesh_info(m, OR_I_NTRIS), fk = or__fk(m);
    const int* F = or__faces(m);
    for (int t = 0; t < nF; ++t) {
        const float* p0 = X + 3 * (size_t)F[fk * t];
        const float* p1 = X + 3 * (size_t)F[fk * t + 1];
        const float* p2 = X + 3 * (size_t)F[fk * t + (fk == 4 ? 3 : 2)];
        float e0[3] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
        float e1[3] = { p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2] };
        float n[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
        float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        fn[3 * t] = n[0] / len; fn[3 * t + 1] = n[1] / len; fn[3 * t + 2] = n[2] / len;
    }
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    for (int v = 0; v < nS; ++v) {
        float n[3] = { 0.f, 0.f, 0.f };
        for (int i = rp[v]; i < rp[v + 1]; ++i) {
            int f = he[4 * i + 2];
            if (f != -1) { n[0] += fn[3 * f]; n[1] += fn[3 * f + 1]; n[2] += fn[3 * f + 2]; }
        }
        float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        vn[3 * v] = n[0] / len; vn[3 * v + 1] = n[1] / len; vn[3 * v + 2] = n[2] / len;
    }
}

/* ======================================================================================== */
/* quadric fit                                                                               */
/* ======================================================================================== */
static inline float dot3f(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static inline double dot3d(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* LU with partial pivoting of a 3x3 system (row-major A), float; returns x in b */
static void solve3_f32(float A[3][3], float b[3]) {
    for (int k = 0; k < 3; ++k) {
        int p = k;
        for (int i = k + 1; i < 3; ++i) if (fabsf(A[i][k]) > fabsf(A[p][k])) p = i;
        if (p != k) {
            for (int j = 0; j < 3; ++j) { float t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
            float t = b[k]; b[k] = b[p]; b[p] = t;
        }
        for (int i = k + 1; i < 3; ++i) {
            float f = A[i][k] / A[k][k];
            for (int j = k + 1; j < 3; ++j) A[i][j] = A[i][j] - f * A[k][j];
            b[i] = b[i] - f * b[k];
        }
    }
    b[2] = b[2] / A[2][2];
    b[1] = (b[1] - A[1][2] * b[2]) / A[1][1];
    b[0] = ((b[0] - A[0][1] * b[1]) - A[0][2] * b[2]) / A[0][0];
}

static void solve3_f64(double A[3][3], double b[3]) {
    for (int k = 0; k < 3; ++k) {
        int p = k;
        for (int i = k + 1; i < 3; ++i) if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
        if (p != k) {
            for (int j = 0; j < 3; ++j) { double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        for (int i = k + 1; i < 3; ++i) {
            double f = A[i][k] / A[k][k];
            for (int j = k + 1; j < 3; ++j) A[i][j] -= f * A[k][j];
            b[i] -= f * b[k];
        }
    }
    b[2] = b[2] / A[2][2];
    b[1] = (b[1] - A[1][2] * b[2]) / A[1][1];
    b[0] = (b[0] - A[0][1] * b[1] - A[0][2] * b[2]) / A[0][0];
}

/* the fit's points after the centre: the 1-ring (halfedge targets in row order), and with
 * ring == 2 then the ring vertices of each 1-ring vertex in row order, each vertex once, the
 * centre excluded; at most 62 */
static int fit_ids(const or_mesh* m, int v, int ring, int* ids) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int nb = 0;
    for (int i = rp[v]; i < rp[v + 1] && nb < 62; ++i) ids[nb++] = he[4 * i];
    if (ring == 2) {
        const int n1 = nb;
        for (int i = 0; i < n1 && nb < 62; ++i) {
            const int u = ids[i];
            for (int j = rp[u]; j < rp[u + 1] && nb < 62; ++j) {
                const int w = he[4 * j];
                int seen = w == v;
                for (int a = 0; a < nb && !seen; ++a) seen = ids[a] == w;
                if (!seen) ids[nb++] = w;
            }
        }
    }
    return nb;
}

/* returns number of vertices whose frame failed the orthonormality check */
int or_surface_fit_ring_f32(const or_mesh* m, const float* X, const float* vn, float* LS, int ring) {
    const int nS = or_mesh_info(m, OR_I_NSURF);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int bad = 0;
    for (int v = 0; v < nS; ++v) {
        const float* c = X + 3 * (size_t)v;
        int b = rp[v];
        float P[64][3];
        int np = 0, ids[62];
        const int nb = fit_ids(m, v, ring, ids);
        P[np][0] = c[0]; P[np][1] = c[1]; P[np][2] = c[2]; np++;
        for (int i = 0; i < nb; ++i) { const float* q = X + 3 * (size_t)ids[i]; P[np][0] = q[0]; P[np][1] = q[1]; P[np][2] = q[2]; np++; }
        if (np == 5) { for (int a = 0; a < 3; ++a) P[np][a] = 0.5f * (P[2][a] + P[3][a]); np++; }
        /* frame */
        float n[3] = { vn[3 * v], vn[3 * v + 1], vn[3 * v + 2] };
        const float* q0 = X + 3 * (size_t)he[4 * b];
        float rv[3] = { q0[0] - c[0], q0[1] - c[1], q0[2] - c[2] };
        float cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        if (sqrtf(dot3f(cr, cr)) < 10.f * EPS) { rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1]; }
        float t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        float t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        float ln = sqrtf(dot3f(n, n)), l1 = sqrtf(dot3f(t1, t1)), l2 = sqrtf(dot3f(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] = n[a] / ln; t1[a] = t1[a] / l1; t2[a] = t2[a] / l2; }
        float x12[3] = { t1[1] * t2[2] - t1[2] * t2[1], t1[2] * t2[0] - t1[0] * t2[2], t1[0] * t2[1] - t1[1] * t2[0] };
        if (!(fabsf(dot3f(x12, n) - 1.f) <= 10.f * EPS)) bad++;
        float M00 = 0.f, M01 = 0.f, M11 = 0.f, M12 = 0.f, M22 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f;
        for (int i = 0; i < np; ++i) {
            float p[3] = { P[i][0] - c[0], P[i][1] - c[1], P[i][2] - c[2] };
            float u = dot3f(t1, p), vv = dot3f(t2, p), w = dot3f(n, p);
            float uu = u * u, uv = u * vv, v2 = vv * vv;
            r0 = r0 + uu * w; r1 = r1 + uv * w; r2 = r2 + v2 * w;
            M00 = M00 + uu * uu; M01 = M01 + uu * uv; M11 = M11 + uu * v2; M12 = M12 + uv * v2; M22 = M22 + v2 * v2;
        }
        float A[3][3] = { { M00, M01, M11 }, { M01, M11, M12 }, { M11, M12, M22 } };
        float s[3] = { r0, r1, r2 };
        solve3_f32(A, s);
        if (np <= 4) { s[0] = s[1] = s[2] = 0.f; }
        for (int a = 0; a < 3; ++a) if (s[a] != s[a]) s[a] = 0.f;
        float* o = LS + LSF * (size_t)v;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = s[0];
        o[4] = t1[0]; o[5] = t1[1]; o[6] = t1[2]; o[7] = s[1];
        o[8] = t2[0]; o[9] = t2[1]; o[10] = t2[2]; o[11] = s[2];
        o[12] = n[0]; o[13] = n[1]; o[14] = n[2]; o[15] = (float)np;
    }
    return bad;
}

int or_surface_fit_ring_f64(const or_mesh* m, const double* X, const double* vn, double* LS, int ring) {
    const int nS = or_mesh_info(m, OR_I_NSURF);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int bad = 0;
    for (int v = 0; v < nS; ++v) {
        const double* c = X + 3 * (size_t)v;
        int b = rp[v];
        double P[64][3];
        int np = 0, ids[62];
        const int nb = fit_ids(m, v, ring, ids);
        P[np][0] = c[0]; P[np][1] = c[1]; P[np][2] = c[2]; np++;
        for (int i = 0; i < nb; ++i) { const double* q = X + 3 * (size_t)ids[i]; P[np][0] = q[0]; P[np][1] = q[1]; P[np][2] = q[2]; np++; }
        if (np == 5) { for (int a = 0; a < 3; ++a) P[np][a] = 0.5 * (P[2][a] + P[3][a]); np++; }
        double n[3] = { vn[3 * v], vn[3 * v + 1], vn[3 * v + 2] };
        const double* q0 = X + 3 * (size_t)he[4 * b];
        double rv[3] = { q0[0] - c[0], q0[1] - c[1], q0[2] - c[2] };
        double cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        if (sqrt(dot3d(cr, cr)) < 10.0 * EPS) { rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1]; }
        double t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        double t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        double ln = sqrt(dot3d(n, n)), l1 = sqrt(dot3d(t1, t1)), l2 = sqrt(dot3d(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] /= ln; t1[a] /= l1; t2[a] /= l2; }
        double x12[3] = { t1[1] * t2[2] - t1[2] * t2[1], t1[2] * t2[0] - t1[0] * t2[2], t1[0] * t2[1] - t1[1] * t2[0] };
        if (!(fabs(dot3d(x12, n) - 1.0) <= 10.0 * EPS)) bad++;
        double M[9] = { 0 }, r[3] = { 0 };
        for (int i = 0; i < np; ++i) {
            double p[3] = { P[i][0] - c[0], P[i][1] - c[1], P[i][2] - c[2] };
            double u = dot3d(t1, p), vv = dot3d(t2, p), w = dot3d(n, p);
            r[0] += u * u * w; r[1] += u * vv * w; r[2] += vv * vv * w;
            M[0] += u * u * u * u; M[1] += u * u * u * vv; M[4] += u * u * vv * vv; M[2] += u * u * vv * vv;
            M[5] += u * vv * vv * vv; M[8] += vv * vv * vv * vv;
        }
        double A[3][3] = { { M[0], M[1], M[2] }, { M[1], M[4], M[5] }, { M[2], M[5], M[8] } };
        solve3_f64(A, r);
        if (np <= 4) { r[0] = r[1] = r[2] = 0.0; }
        for (int a = 0; a < 3; ++a) if (r[a] != r[a]) r[a] = 0.0;
        double* o = LS + LSF * (size_t)v;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = r[0];
        o[4] = t1[0]; o[5] = t1[1]; o[6] = t1[2]; o[7] = r[1];
        o[8] = t2[0]; o[9] = t2[1]; o[10] = t2[2]; o[11] = r[2];
        o[12] = n[0]; o[13] = n[1]; o[14] = n[2]; o[15] = (double)np;
    }
    return bad;
}

int or_surface_fit_f32(const or_mesh* m, const float* X, const float* vn, float* LS) {
    return or_surface_fit_ring_f32(m, X, vn, LS, 1);
}
int or_surface_fit_f64(const or_mesh* m, const double* X, const double* vn, double* LS) {
    return or_surface_fit_ring_f64(m, X, vn, LS, 1);
}

/* ======================================================================================== */
/* per-sector surfaces of feature vertices (SurfaceFeature.h:79-106, SurfaceFeature.cu:12-221)*/
/* ======================================================================================== */
#define TABLE_SIZE 20
#define MAX_NEIGHBORS 40

/* sector neighbour lists of every feature vertex: nb[s*MAX_NEIGHBORS + i], nnb[s];
 * returns the number of sectors or -1 (valence beyond the reference's table / list sizes) */
static int feature_sectors(const or_mesh* m, int32_t* rowptr, int32_t* table, int* nb, int* nnb, int cap) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFeat = or_mesh_info(m, OR_I_NFEATURE), nFree = nS - nFeat;
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    extern const uint8_t* or__isFeat(const or_mesh* m);
    extern const uint8_t* or__isB1(const or_mesh* m);
    const uint8_t* isB1 = or__isB1(m);
    rowptr[0] = 0;
    for (int idx = 0; idx < nFeat; ++idx) {
        int vid = nFree + idx, b = rp[vid], e = rp[vid + 1];
        if (e - b > TABLE_SIZE) return -1;
        int sid = 0;
        for (int i = b + 1; i < e; ++i) if (he[4 * i] >= nFree) ++sid;
        if (!isB1[vid]) ++sid;
        rowptr[idx + 1] = rowptr[idx] + sid;
    }
    if (rowptr[nFeat] > cap) return -1;
    for (int i = 0; i < nFeat * TABLE_SIZE; ++i) table[i] = -1;
    for (int idx = 0; idx < nFeat; ++idx) {
        int vid = nFree + idx, b = rp[vid], e = rp[vid + 1];
        int sid = 0, nn = 0, last = 1, lastHE = b, vindex = 1;
        int* T = table + TABLE_SIZE * idx;
        T[0] = 0;
        for (int i = b + 1; i < e; ++i) {
            int vdst = he[4 * i];
            int* L = nb + MAX_NEIGHBORS * (size_t)(rowptr[idx] + sid);
            if (last) { nn = 0; L[nn++] = vid; L[nn++] = he[4 * lastHE]; }
            if (vdst >= nFree) {
                T[vindex] = sid; L[nn++] = vdst; nnb[rowptr[idx] + sid] = nn; ++sid; nn = 0; last = 1;
            } else {
                if (nn >= MAX_NEIGHBORS) return -1;
                T[vindex] = sid; L[nn++] = vdst; last = 0;
            }
            ++lastHE; ++vindex;
        }
        if (!isB1[vid]) {
            int* L = nb + MAX_NEIGHBORS * (size_t)(rowptr[idx] + sid);
            if (last) { nn = 0; L[nn++] = vid; L[nn++] = he[4 * lastHE]; }
            L[nn++] = he[4 * b];
            nnb[rowptr[idx] + sid] = nn;
        }
    }
    return rowptr[nFeat];
}

/* face normal of the halfedge vid -> target (last match, SurfaceFeature.cu:36-40) */
static int face_of(const or_mesh* m, int vid, int target) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int f = -1;
    for (int i = rp[vid]; i < rp[vid + 1]; ++i) if (he[4 * i] == target) f = he[4 * i + 2];
    return f;
}

int or_feature_surfaces_f32(const or_mesh* m, const float* X, const float* fn, int32_t* rowptr, int32_t* table,
                            float* LS, int cap) {
    int* nb = (int*)calloc((size_t)(cap > 0 ? cap : 1) * MAX_NEIGHBORS, sizeof(int));
    int* nnb = (int*)calloc((size_t)(cap > 0 ? cap : 1), sizeof(int));
    int ns = feature_sectors(m, rowptr, table, nb, nnb, cap);
    for (int s_ = 0; s_ < ns; ++s_) {
        const int* L = nb + MAX_NEIGHBORS * (size_t)s_;
        int np = nnb[s_];
        const int vid = L[0];
        const float* c = X + 3 * (size_t)vid;
        float P[MAX_NEIGHBORS + 1][3];
        for (int i = 0; i < np; ++i) for (int a = 0; a < 3; ++a) P[i][a] = X[3 * (size_t)L[i] + a];
        if (np == 5) { for (int a = 0; a < 3; ++a) P[np][a] = 0.5f * (P[2][a] + P[3][a]); np++; }
        int f = face_of(m, vid, L[1]);
        float n[3] = { fn[3 * f], fn[3 * f + 1], fn[3 * f + 2] };
        const float* q0 = X + 3 * (size_t)L[1];
        float rv[3] = { q0[0] - c[0], q0[1] - c[1], q0[2] - c[2] };
        float cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        if (sqrtf(dot3f(cr, cr)) < 10.f * EPS) { rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1]; }
        float t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        float t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        float ln = sqrtf(dot3f(n, n)), l1 = sqrtf(dot3f(t1, t1)), l2 = sqrtf(dot3f(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] = n[a] / ln; t1[a] = t1[a] / l1; t2[a] = t2[a] / l2; }
        float M00 = 0.f, M01 = 0.f, M11 = 0.f, M12 = 0.f, M22 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f;
        for (int i = 0; i < np; ++i) {
            float p[3] = { P[i][0] - c[0], P[i][1] - c[1], P[i][2] - c[2] };
            float u = dot3f(t1, p), vv = dot3f(t2, p), w = dot3f(n, p);
            float uu = u * u, uv = u * vv, v2 = vv * vv;
            r0 = r0 + uu * w; r1 = r1 + uv * w; r2 = r2 + v2 * w;
            M00 = M00 + uu * uu; M01 = M01 + uu * uv; M11 = M11 + uu * v2; M12 = M12 + uv * v2; M22 = M22 + v2 * v2;
        }
        float A[3][3] = { { M00, M01, M11 }, { M01, M11, M12 }, { M11, M12, M22 } };
        float sv[3] = { r0, r1, r2 };
        solve3_f32(A, sv);
        if (np <= 4) { sv[0] = sv[1] = sv[2] = 0.f; }
        for (int a = 0; a < 3; ++a) if (sv[a] != sv[a]) sv[a] = 0.f;
        float* o = LS + LSF * (size_t)s_;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = sv[0];
        o[4] = t1[0]; o[5] = t1[1]; o[6] = t1[2]; o[7] = sv[1];
        o[8] = t2[0]; o[9] = t2[1]; o[10] = t2[2]; o[11] = sv[2];
        o[12] = n[0]; o[13] = n[1]; o[14] = n[2]; o[15] = (float)np;
    }
    free(nb); free(nnb);
    return ns;
}

int or_feature_surfaces_f64(const or_mesh* m, const double* X, const double* fn, int32_t* rowptr, int32_t* table,
                            double* LS, int cap) {
    int* nb = (int*)calloc((size_t)(cap > 0 ? cap : 1) * MAX_NEIGHBORS, sizeof(int));
    int* nnb = (int*)calloc((size_t)(cap > 0 ? cap : 1), sizeof(int));
    int ns = feature_sectors(m, rowptr, table, nb, nnb, cap);
    for (int s_ = 0; s_ < ns; ++s_) {
        const int* L = nb + MAX_NEIGHBORS * (size_t)s_;
        int np = nnb[s_];
        const int vid = L[0];
        const double* c = X + 3 * (size_t)vid;
        double P[MAX_NEIGHBORS + 1][3];
        for (int i = 0; i < np; ++i) for (int a = 0; a < 3; ++a) P[i][a] = X[3 * (size_t)L[i] + a];
        if (np == 5) { for (int a = 0; a < 3; ++a) P[np][a] = 0.5 * (P[2][a] + P[3][a]); np++; }
        int f = face_of(m, vid, L[1]);
        double n[3] = { fn[3 * f], fn[3 * f + 1], fn[3 * f + 2] };
        const double* q0 = X + 3 * (size_t)L[1];
        double rv[3] = { q0[0] - c[0], q0[1] - c[1], q0[2] - c[2] };
        double cr[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        if (sqrt(dot3d(cr, cr)) < 10.0 * EPS) { rv[0] = n[0]; rv[1] = n[2]; rv[2] = -n[1]; }
        double t1[3] = { n[1] * rv[2] - n[2] * rv[1], n[2] * rv[0] - n[0] * rv[2], n[0] * rv[1] - n[1] * rv[0] };
        double t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
        double ln = sqrt(dot3d(n, n)), l1 = sqrt(dot3d(t1, t1)), l2 = sqrt(dot3d(t2, t2));
        for (int a = 0; a < 3; ++a) { n[a] /= ln; t1[a] /= l1; t2[a] /= l2; }
        double M[9] = { 0 }, r[3] = { 0 };
        for (int i = 0; i < np; ++i) {
            double p[3] = { P[i][0] - c[0], P[i][1] - c[1], P[i][2] - c[2] };
            double u = dot3d(t1, p), vv = dot3d(t2, p), w = dot3d(n, p);
            r[0] += u * u * w; r[1] += u * vv * w; r[2] += vv * vv * w;
            M[0] += u * u * u * u; M[1] += u * u * u * vv; M[4] += u * u * vv * vv; M[2] += u * u * vv * vv;
            M[5] += u * vv * vv * vv; M[8] += vv * vv * vv * vv;
        }
        double A[3][3] = { { M[0], M[1], M[2] }, { M[1], M[4], M[5] }, { M[2], M[5], M[8] } };
        solve3_f64(A, r);
        if (np <= 4) { r[0] = r[1] = r[2] = 0.0; }
        for (int a = 0; a < 3; ++a) if (r[a] != r[a]) r[a] = 0.0;
        double* o = LS + LSF * (size_t)s_;
        o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = r[0];
        o[4] = t1[0]; o[5] = t1[1]; o[6] = t1[2]; o[7] = r[1];
        o[8] = t2[0]; o[9] = t2[1]; o[10] = t2[2]; o[11] = r[2];
        o[12] = n[0]; o[13] = n[1]; o[14] = n[2]; o[15] = (double)np;
    }
    free(nb); free(nnb);
    return ns;
}

/* ======================================================================================== */
/* nearest initial vertex (k_updateNearestNeighbor)                                          */
/* ======================================================================================== */
void or_update_nn_f32(const or_mesh* m, const float* X, const float* X0, int32_t* nn) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFree = nS - or_mesh_info(m, OR_I_NFEATURE);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    for (int v = 0; v < nS; ++v) {
        const float* p = X + 3 * (size_t)v;
        int vh = nn[v];
        const float* pi = X0 + 3 * (size_t)vh;
        float dd[3] = { p[0] - pi[0], p[1] - pi[1], p[2] - pi[2] };
        float sd = dot3f(dd, dd);
        int vnew;
        const int fv = v >= nFree;
        do {
            vnew = vh;
            int b = rp[vnew], e = rp[vnew + 1];
            for (int i = b; i < e; ++i) {
                int d = he[4 * i];
                if (fv != (d >= nFree)) continue;
                const float* q = X0 + 3 * (size_t)d;
                float ee[3] = { p[0] - q[0], p[1] - q[1], p[2] - q[2] };
                float s2 = dot3f(ee, ee);
                if (s2 < sd) { sd = s2; vh = d; }
            }
        } while (vnew != vh);
        nn[v] = vnew;
    }
}

void or_update_nn_f64(const or_mesh* m, const double* X, const double* X0, int32_t* nn) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nFree = nS - or_mesh_info(m, OR_I_NFEATURE);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    for (int v = 0; v < nS; ++v) {
        const double* p = X + 3 * (size_t)v;
        int vh = nn[v];
        const double* pi = X0 + 3 * (size_t)vh;
        double dd[3] = { p[0] - pi[0], p[1] - pi[1], p[2] - pi[2] };
        double sd = dot3d(dd, dd);
        int vnew;
        const int fv = v >= nFree;
        do {
            vnew = vh;
            int b = rp[vnew], e = rp[vnew + 1];
            for (int i = b; i < e; ++i) {
                int d = he[4 * i];
                if (fv != (d >= nFree)) continue;
                const double* q = X0 + 3 * (size_t)d;
                double ee[3] = { p[0] - q[0], p[1] - q[1], p[2] - q[2] };
                double s2 = dot3d(ee, ee);
                if (s2 < sd) { sd = s2; vh = d; }
            }
        } while (vnew != vh);
        nn[v] = vnew;
    }
}

/* ======================================================================================== */
/* element metrics                                                                           */
/* ======================================================================================== */
/* meanRatioMetricTri(p) unsigned (DMOQualityTri.h:260-272) */
double or_q_tri3d_f64(const double* p0, const double* p1, const double* p2) {
    double e0[3], e1[3], e2[3];
    for (int a = 0; a < 3; ++a) { e0[a] = p1[a] - p0[a]; e1[a] = p2[a] - p0[a]; e2[a] = p2[a] - p1[a]; }
    double l = dot3d(e0, e0) + dot3d(e1, e1) + dot3d(e2, e2);
    double c[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
    return 2.0 * sqrt(3.0) * sqrt(dot3d(c, c)) / l;
}

float or_q_tri3d_f32(const float* p0, const float* p1, const float* p2) {
    float e0[3], e1[3], e2[3];
    for (int a = 0; a < 3; ++a) { e0[a] = p1[a] - p0[a]; e1[a] = p2[a] - p0[a]; e2[a] = p2[a] - p1[a]; }
    float l = (dot3f(e0, e0) + dot3f(e1, e1)) + dot3f(e2, e2);
    float c[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
    return ((2.f * sqrtf(3.f)) * sqrtf(dot3f(c, c))) / l;
}

/* meanRatioMetricQuad(p) / (p, n) (DMOQualityQuad.h:13-50); n == NULL: unsigned variant */
/* condition-number quality of a quad (an addition; or_set_criterion(OR_CONDITION)): per corner
 * with edges e1, e2 to its neighbours 2 det / (|e1|^2 + |e2|^2), det = (e1 x e2) . n, or
 * |e1 x e2| without n; the smallest corner */
static double qcond_corner64(const double* o, const double* a, const double* b, const double* n) {
    const double e1[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] }, e2[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] };
    const double c[3] = { e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0] };
    const double F2 = dot3d(e1, e1) + dot3d(e2, e2);
    const double det = n ? dot3d(c, n) : sqrt(dot3d(c, c));
    return F2 > 0.0 ? 2.0 * det / F2 : 0.0;
}
static float qcond_corner32(const float* o, const float* a, const float* b, const float* n) {
    const float e1[3] = { a[0] - o[0], a[1] - o[1], a[2] - o[2] }, e2[3] = { b[0] - o[0], b[1] - o[1], b[2] - o[2] };
    const float c[3] = { e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0] };
    const float F2 = dot3f(e1, e1) + dot3f(e2, e2);
    const float det = n ? dot3f(c, n) : sqrtf(dot3f(c, c));
    return F2 > 0.f ? (2.f * det) / F2 : 0.f;
}

double or_q_quad_f64(const double* p0, const double* p1, const double* p2, const double* p3, const double* n) {
    if (or__criterion() == OR_CONDITION)
        return fmin(fmin(qcond_corner64(p0, p1, p3, n), qcond_corner64(p1, p2, p0, n)),
                    fmin(qcond_corner64(p2, p3, p1, n), qcond_corner64(p3, p0, p2, n)));
    double e[4][3];
    for (int a = 0; a < 3; ++a) { e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p1[a]; e[2][a] = p3[a] - p2[a]; e[3][a] = p0[a] - p3[a]; }
    double l = dot3d(e[0], e[0]) + dot3d(e[1], e[1]) + dot3d(e[2], e[2]) + dot3d(e[3], e[3]);
    double m0[3] = { -e[0][0], -e[0][1], -e[0][2] }, m2[3] = { -e[2][0], -e[2][1], -e[2][2] };
    double c1[3] = { e[1][1] * m0[2] - e[1][2] * m0[1], e[1][2] * m0[0] - e[1][0] * m0[2], e[1][0] * m0[1] - e[1][1] * m0[0] };
    double c2[3] = { e[3][1] * m2[2] - e[3][2] * m2[1], e[3][2] * m2[0] - e[3][0] * m2[2], e[3][0] * m2[1] - e[3][1] * m2[0] };
    double a1 = sqrt(dot3d(c1, c1)), a2 = sqrt(dot3d(c2, c2));
    if (n) {
        double d1 = (c1[0] / a1) * n[0] + (c1[1] / a1) * n[1] + (c1[2] / a1) * n[2];
        double d2 = (c2[0] / a2) * n[0] + (c2[1] / a2) * n[1] + (c2[2] / a2) * n[2];
        if (d1 < 0.7 || d2 < 0.7) return -1.0;
    }
    return 2.0 * (a1 + a2) / l;
}

float or_q_quad_f32(const float* p0, const float* p1, const float* p2, const float* p3, const float* n) {
    if (or__criterion() == OR_CONDITION) {
        float q = qcond_corner32(p0, p1, p3, n);
        q = fminf(q, qcond_corner32(p1, p2, p0, n));
        q = fminf(q, qcond_corner32(p2, p3, p1, n));
        return fminf(q, qcond_corner32(p3, p0, p2, n));
    }
    float e[4][3];
    for (int a = 0; a < 3; ++a) { e[0][a] = p1[a] - p0[a]; e[1][a] = p2[a] - p1[a]; e[2][a] = p3[a] - p2[a]; e[3][a] = p0[a] - p3[a]; }
    float l = ((dot3f(e[0], e[0]) + dot3f(e[1], e[1])) + dot3f(e[2], e[2])) + dot3f(e[3], e[3]);
    float m0[3] = { -e[0][0], -e[0][1], -e[0][2] }, m2[3] = { -e[2][0], -e[2][1], -e[2][2] };
    float c1[3] = { e[1][1] * m0[2] - e[1][2] * m0[1], e[1][2] * m0[0] - e[1][0] * m0[2], e[1][0] * m0[1] - e[1][1] * m0[0] };
    float c2[3] = { e[3][1] * m2[2] - e[3][2] * m2[1], e[3][2] * m2[0] - e[3][0] * m2[2], e[3][0] * m2[1] - e[3][1] * m2[0] };
    float a1 = sqrtf(dot3f(c1, c1)), a2 = sqrtf(dot3f(c2, c2));
    if (n) {
        float d1 = dot3f(c1, n) / a1, d2 = dot3f(c2, n) / a2;
        if (d1 < 0.7f || d2 < 0.7f) return -1.f;
    }
    return (2.f * (a1 + a2)) / l;
}

/* ======================================================================================== */
/* f64: literal restatement of the surface kernels                                          */
/* ======================================================================================== */
typedef struct {
    const or_mesh* m;
    const double* X0;   /* initial positions */
    const double* LS;   /* local surfaces of the initial positions */
    const int32_t* nn;  /* nearest initial vertex */
    const double* vn;   /* current vertex normals */
    /* feature vertices' sector surfaces (NULL: the mesh has none) and the positions the sector
       of a feature neighbour is chosen from (the positions at the start of the colour class) */
    const int32_t* frow; const int32_t* ftab; const double* FS; const double* Xs;
} surf64;

/* sector surface of feature vertex f seen from vertex v: the sector of f's halfedge whose target
   is closest to v (localSurfaceEstimationWithFeature, dmo/SurfaceEstimation.h:150-172) */
static int sector_of(const or_mesh* m, const int32_t* frow, const int32_t* ftab, int f, int nFree, const double* Xs64,
                     const float* Xs32, int v) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int arg = 0, idx = 0;
    if (Xs64) {
        double best = DBL_MAX;
        const double* pv = Xs64 + 3 * (size_t)v;
        for (int i = rp[f]; i < rp[f + 1]; ++i, ++idx) {
            const double* t = Xs64 + 3 * (size_t)he[4 * i];
            double d[3] = { t[0] - pv[0], t[1] - pv[1], t[2] - pv[2] };
            double s = dot3d(d, d);
            if (s < best) { best = s; arg = idx; }
        }
    } else {
        float best = FLT_MAX;
        const float* pv = Xs32 + 3 * (size_t)v;
        for (int i = rp[f]; i < rp[f + 1]; ++i, ++idx) {
            const float* t = Xs32 + 3 * (size_t)he[4 * i];
            float d[3] = { t[0] - pv[0], t[1] - pv[1], t[2] - pv[2] };
            float s = dot3f(d, d);
            if (s < best) { best = s; arg = idx; }
        }
    }
    return frow[f - nFree] + ftab[TABLE_SIZE * (f - nFree) + arg];
}

static inline double poly64(const double* L, double u, double v) { return L[3] * u * u + L[7] * u * v + L[11] * v * v; }

static void est64(const surf64* S, int v, double u, double vv, double* out) {
    const int* rp = or__he_rowptr(S->m);
    const int* he = or__he(S->m);
    const double* L = S->LS + LSF * (size_t)S->nn[v];
    double w = poly64(L, u, vv);
    double pw[3];
    for (int a = 0; a < 3; ++a) pw[a] = L[a] + u * L[4 + a] + vv * L[8 + a] + w * L[12 + a];
    double d[3]; const double* x0 = S->X0 + 3 * (size_t)S->nn[v];
    for (int a = 0; a < 3; ++a) d[a] = x0[a] - pw[a];
    double ids[64], ps[64][3];
    int k = 0;
    ids[0] = 1.0 / (dot3d(d, d) + EPS);
    double isum = ids[0];
    ps[0][0] = pw[0]; ps[0][1] = pw[1]; ps[0][2] = pw[2];
    for (int i = rp[v]; i < rp[v + 1] && k < 62; ++i) {
        int vN = he[4 * i];
        int nnN = S->nn[vN];
        const double* xn = S->X0 + 3 * (size_t)nnN;
        for (int a = 0; a < 3; ++a) d[a] = xn[a] - pw[a];
        ++k;
        ids[k] = 1.0 / (dot3d(d, d) + EPS);
        isum += ids[k];
        const int nFree = or_mesh_info(S->m, OR_I_NSURF) - or_mesh_info(S->m, OR_I_NFEATURE);
        const double* Ln = S->LS + LSF * (size_t)S->nn[vN];
        if (S->FS && nnN >= nFree) Ln = S->FS + LSF * (size_t)sector_of(S->m, S->frow, S->ftab, nnN, nFree, S->Xs, NULL, v);
        double q[3] = { pw[0] - Ln[0], pw[1] - Ln[1], pw[2] - Ln[2] };
        double lu = q[0] * Ln[4] + q[1] * Ln[5] + q[2] * Ln[6];
        double lv = q[0] * Ln[8] + q[1] * Ln[9] + q[2] * Ln[10];
        double lw = poly64(Ln, lu, lv);
        for (int a = 0; a < 3; ++a) ps[k][a] = Ln[a] + lu * Ln[4 + a] + lv * Ln[8 + a] + lw * Ln[12 + a];
    }
    double inv = 1.0 / isum;
    out[0] = out[1] = out[2] = 0.0;
    for (int i = 0; i <= k; ++i) for (int a = 0; a < 3; ++a) out[a] += ps[i][a] * ids[i] * inv;
}

/* ring quality: fk == 3 closed triangle fan, fk == 4 quad pairs; n == NULL: unsigned */
static double ring64(int fk, int k, const double* ring, const double* p, const double* n) {
    double q = DBL_MAX;
    for (int i = 0; i < k; ++i) {
        double v;
        const int crit = or__criterion();
        if (fk == 3 && crit != OR_MEAN_RATIO) {
            v = or_q_tri3d_angle_f64(p, ring + 3 * i, ring + 3 * (i + 1), n, crit == OR_MAX_ANGLE);
        } else if (fk == 3) {
            const double* a = ring + 3 * i; const double* b = ring + 3 * (i + 1);
            double e0[3], e1[3], e2[3];
            for (int c = 0; c < 3; ++c) { e0[c] = a[c] - p[c]; e1[c] = b[c] - p[c]; e2[c] = b[c] - a[c]; }
            double l = dot3d(e0, e0) + dot3d(e1, e1) + dot3d(e2, e2);
            double nt[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
            double len = sqrt(dot3d(nt, nt));
            double area = len;
            if (n) {
                double nd = (nt[0] / len) * n[0] + (nt[1] / len) * n[1] + (nt[2] / len) * n[2];
                double sg = nd > 0.0 ? 1.0 : (nd < 0.0 ? -1.0 : 0.0);
                area = len * sg;
            }
            v = 2.0 * sqrt(3.0) * area / l;
        } else {
            v = or_q_quad_f64(p, ring + 6 * i, ring + 6 * i + 3, ring + 6 * i + 6, n);
        }
        q = fmin(q, v);
    }
    return q;
}

static void surf_vertex_f64(const surf64* S, double* X, int v, double gs, double* margin) {
    const or_mesh* m = S->m;
    const int fk = or__fk(m);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    double* ring = (double*)malloc(sizeof(double) * 3 * (2 * (size_t)k + 2));
    double cur[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    double p0[3] = { cur[0], cur[1], cur[2] };
    double md = -DBL_MAX;
    for (int i = 0; i < k; ++i) {
        const double* t = X + 3 * (size_t)he[4 * (b + i)];
        if (fk == 3) {
            for (int a = 0; a < 3; ++a) ring[3 * i + a] = t[a];
        } else {
            const double* t2 = X + 3 * (size_t)he[4 * he[4 * (b + i) + 3]];
            for (int a = 0; a < 3; ++a) { ring[6 * i + a] = t[a]; ring[6 * i + 3 + a] = t2[a]; }
            double d2[3] = { t2[0] - cur[0], t2[1] - cur[1], t2[2] - cur[2] };
            md = fmax(md, sqrt(dot3d(d2, d2)));
        }
        double d[3] = { t[0] - cur[0], t[1] - cur[1], t[2] - cur[2] };
        md = fmax(md, sqrt(dot3d(d, d)));
    }
    if (fk == 3) for (int a = 0; a < 3; ++a) ring[3 * k + a] = ring[a];
    else for (int a = 0; a < 3; ++a) ring[6 * k + a] = ring[a];
    const int nnv = S->nn[v];
    const double* L = S->LS + LSF * (size_t)nnv;
    const double* n = S->vn + 3 * (size_t)nnv;
    double dl[3] = { cur[0] - L[0], cur[1] - L[1], cur[2] - L[2] };
    double cu = dl[0] * L[4] + dl[1] * L[5] + dl[2] * L[6];
    double cv = dl[0] * L[8] + dl[1] * L[9] + dl[2] * L[10];
    const double aff = 1.0 / (NQ - 1);
    double ds = gs, lastMax = -DBL_MAX, mg = DBL_MAX;
    /* the quad condition number has a corner that does not touch the vertex (the diagonal
       one): exact ties at its value are structural (or__gap64) */
    const int ties = or__criterion() == OR_CONDITION;
    for (int d = 0; d < DEPTH; ++d) {
        double uMax = ds * md, uMin = -ds * md;
        double val[32], uvs[32][2];
        double best = -DBL_MAX, second = -DBL_MAX;
        for (int t = 0; t < 32; ++t) {
            int i1 = t / NQ, j1 = t % NQ, i2 = i1 + 4;
            double u1 = cu + aff * (i1 * uMin + (NQ - 1 - i1) * uMax);
            double v1 = cv + aff * (j1 * uMin + (NQ - 1 - j1) * uMax);
            double u2 = cu + aff * (i2 * uMin + (NQ - 1 - i2) * uMax);
            double pw1[3], pw2[3];
            est64(S, v, u1, v1, pw1);
            est64(S, v, u2, v1, pw2);
            double q1 = ring64(fk, k, ring, pw1, n), q2 = ring64(fk, k, ring, pw2, n);
            val[t] = q1; uvs[t][0] = u1; uvs[t][1] = v1;
            if (q2 > q1) { val[t] = q2; uvs[t][0] = u2; }
            double qs[2] = { q1, q2 };
            for (int s = 0; s < 2; ++s) {
                if (qs[s] > best) { second = best; best = qs[s]; }
                else if ((!ties || qs[s] < best) && qs[s] > second) second = qs[s];
            }
        }
        double qLast = ring64(fk, k, ring, cur, n);
        int w = 0;
        for (int t = 1; t < 32; ++t) if (val[t] > val[w]) w = t;
        mg = fmin(mg, best - second);
        mg = fmin(mg, ties ? or__gap64(best, qLast) : fabs(best - qLast));
        if (qLast < val[w]) {
            est64(S, v, uvs[w][0], uvs[w][1], cur);
            cu = uvs[w][0]; cv = uvs[w][1];
        }
        lastMax = val[w];
        ds = ds * (2.0 / (NQ - 1));
    }
    double qOld = ring64(fk, k, ring, p0, NULL);
    mg = fmin(mg, ties ? or__gap64(lastMax, qOld) : fabs(lastMax - qOld));
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    if (margin) *margin = mg;
    free(ring);
}

void or_dmo_surf_feat_f64(const or_mesh* m, double* X, const double* X0, const double* LS, const int32_t* nn,
                          const double* vn, const int32_t* frow, const int32_t* ftab, const double* FS, int v0, int v1,
                          double gs, double* margin, int nthreads) {
    const int nS = or_mesh_info(m, OR_I_NSURF);
    double* Xs = FS ? (double*)malloc(sizeof(double) * 3 * (size_t)nS) : NULL;
    if (Xs) memcpy(Xs, X, sizeof(double) * 3 * (size_t)nS);
    surf64 S = { m, X0, LS, nn, vn, frow, ftab, FS, Xs };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) surf_vertex_f64(&S, X, v, gs, margin ? margin + (v - v0) : NULL);
    free(Xs);
}

void or_dmo_surf_f64(const or_mesh* m, double* X, const double* X0, const double* LS, const int32_t* nn,
                     const double* vn, int v0, int v1, double gs, double* margin, int nthreads) {
    surf64 S = { m, X0, LS, nn, vn, NULL, NULL, NULL, NULL };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) surf_vertex_f64(&S, X, v, gs, margin ? margin + (v - v0) : NULL);
}

/* ======================================================================================== */
/* f32: the product's arithmetic                                                             */
/* ======================================================================================== */
typedef struct {
    const or_mesh* m;
    const float* X0;
    const float* LS;
    const int32_t* nn;
    const float* vn;
    const int32_t* frow; const int32_t* ftab; const float* FS; const float* Xs;
} surf32;

static inline float poly32(const float* L, float u, float v) { return (((L[3] * u) * u) + ((L[7] * u) * v)) + ((L[11] * v) * v); }

static void est32(const surf32* S, int v, float u, float vv, float* out) {
    const int* rp = or__he_rowptr(S->m);
    const int* he = or__he(S->m);
    const float* L = S->LS + LSF * (size_t)S->nn[v];
    float w = poly32(L, u, vv);
    float pw[3];
    for (int a = 0; a < 3; ++a) pw[a] = ((L[a] + u * L[4 + a]) + vv * L[8 + a]) + w * L[12 + a];
    const float* x0 = S->X0 + 3 * (size_t)S->nn[v];
    float d[3] = { x0[0] - pw[0], x0[1] - pw[1], x0[2] - pw[2] };
    float id = 1.0f / (dot3f(d, d) + EPS);
    float isum = id;
    float acc[3] = { pw[0] * id, pw[1] * id, pw[2] * id };
    for (int i = rp[v]; i < rp[v + 1]; ++i) {
        int vN = he[4 * i];
        const float* xn = S->X0 + 3 * (size_t)S->nn[vN];
        float dn[3] = { xn[0] - pw[0], xn[1] - pw[1], xn[2] - pw[2] };
        float idn = 1.0f / (dot3f(dn, dn) + EPS);
        isum = isum + idn;
        const int nnN = S->nn[vN];
        const int nFree = or_mesh_info(S->m, OR_I_NSURF) - or_mesh_info(S->m, OR_I_NFEATURE);
        const float* Ln = S->LS + LSF * (size_t)nnN;
        if (S->FS && nnN >= nFree) Ln = S->FS + LSF * (size_t)sector_of(S->m, S->frow, S->ftab, nnN, nFree, NULL, S->Xs, v);
        float q[3] = { pw[0] - Ln[0], pw[1] - Ln[1], pw[2] - Ln[2] };
        float lu = dot3f(q, Ln + 4), lv = dot3f(q, Ln + 8);
        float lw = poly32(Ln, lu, lv);
        for (int a = 0; a < 3; ++a) {
            float p2 = ((Ln[a] + lu * Ln[4 + a]) + lv * Ln[8 + a]) + lw * Ln[12 + a];
            acc[a] = acc[a] + p2 * idn;
        }
    }
    float inv = 1.0f / isum;
    out[0] = acc[0] * inv; out[1] = acc[1] * inv; out[2] = acc[2] * inv;
}

/* ring key: triangles -> sign |nt|^2 / L^2 (or |nt|^2 / L^2 unsigned) as a fraction; quads -> q */
static float ring32(int fk, int k, const float* ring, const float* p, const float* n) {
    if (fk == 3) {
        float N = 0.f, D = 1.f;
        for (int i = 0; i < k; ++i) {
            const float* a = ring + 3 * i; const float* b = ring + 3 * (i + 1);
            float e0[3] = { a[0] - p[0], a[1] - p[1], a[2] - p[2] };
            float e1[3] = { b[0] - p[0], b[1] - p[1], b[2] - p[2] };
            float e2[3] = { b[0] - a[0], b[1] - a[1], b[2] - a[2] };
            float l = (dot3f(e0, e0) + dot3f(e1, e1)) + dot3f(e2, e2);
            float nt[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
            float a2 = dot3f(nt, nt);
            float num = a2;
            if (n) { float dn = dot3f(nt, n); num = dn > 0.f ? a2 : (dn < 0.f ? -a2 : 0.f); }
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

static inline float grid_offset(int i) { return (float)(NQ - 1 - 2 * i) / (float)(NQ - 1); }

static void surf_vertex_f32(const surf32* S, float* X, int v, float gs) {
    const or_mesh* m = S->m;
    const int fk = or__fk(m);
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    int b = rp[v], k = rp[v + 1] - b;
    if (k <= 0) return;
    float* ring = (float*)malloc(sizeof(float) * 3 * (2 * (size_t)k + 2));
    float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float cur[3] = { c0[0], c0[1], c0[2] };
    float md = 0.f;
    for (int i = 0; i < k; ++i) {
        const float* t = X + 3 * (size_t)he[4 * (b + i)];
        float d[3] = { t[0] - c0[0], t[1] - c0[1], t[2] - c0[2] };
        md = fmaxf(md, sqrtf(dot3f(d, d)));
        if (fk == 3) {
            for (int a = 0; a < 3; ++a) ring[3 * i + a] = t[a];
        } else {
            const float* t2 = X + 3 * (size_t)he[4 * he[4 * (b + i) + 3]];
            for (int a = 0; a < 3; ++a) { ring[6 * i + a] = t[a]; ring[6 * i + 3 + a] = t2[a]; }
            float d2[3] = { t2[0] - c0[0], t2[1] - c0[1], t2[2] - c0[2] };
            md = fmaxf(md, sqrtf(dot3f(d2, d2)));
        }
    }
    if (fk == 3) for (int a = 0; a < 3; ++a) ring[3 * k + a] = ring[a];
    else for (int a = 0; a < 3; ++a) ring[6 * k + a] = ring[a];
    const int nnv = S->nn[v];
    const float* L = S->LS + LSF * (size_t)nnv;
    const float* n = S->vn + 3 * (size_t)nnv;
    float dl[3] = { c0[0] - L[0], c0[1] - L[1], c0[2] - L[2] };
    float cu = dot3f(dl, L + 4), cv = dot3f(dl, L + 8);
    float qLast = ring32(fk, k, ring, c0, n);
    const float qOld = ring32(fk, k, ring, c0, NULL);
    float ds = gs, lastMax = -FLT_MAX;
    for (int d = 0; d < DEPTH; ++d) {
        float S_ = ds * md;
        float us[NQ], vs[NQ];
        for (int i = 0; i < NQ; ++i) { us[i] = fmaf(grid_offset(i), S_, cu); vs[i] = fmaf(grid_offset(i), S_, cv); }
        float bv = 0.f, bu = 0.f, bvv = 0.f, bp[3] = { 0.f, 0.f, 0.f };
        int bt = -1;
        for (int t = 0; t < 32; ++t) {
            int i1 = t >> 3, j1 = t & 7, i2 = i1 + 4;
            float pw1[3], pw2[3];
            est32(S, v, us[i1], vs[j1], pw1);
            est32(S, v, us[i2], vs[j1], pw2);
            float q1 = ring32(fk, k, ring, pw1, n), q2 = ring32(fk, k, ring, pw2, n);
            float val = q1; int second = 0;
            if (q2 > q1) { val = q2; second = 1; }
            if (bt < 0 || val > bv) {
                bv = val; bt = t;
                bu = second ? us[i2] : us[i1]; bvv = vs[j1];
                const float* pp = second ? pw2 : pw1;
                bp[0] = pp[0]; bp[1] = pp[1]; bp[2] = pp[2];
            }
        }
        if (qLast < bv) { cur[0] = bp[0]; cur[1] = bp[1]; cur[2] = bp[2]; cu = bu; cv = bvv; qLast = bv; }
        lastMax = bv;
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    free(ring);
}

void or_dmo_surf_feat_f32(const or_mesh* m, float* X, const float* X0, const float* LS, const int32_t* nn,
                          const float* vn, const int32_t* frow, const int32_t* ftab, const float* FS, int v0, int v1,
                          float gs, int nthreads) {
    const int nS = or_mesh_info(m, OR_I_NSURF);
    float* Xs = FS ? (float*)malloc(sizeof(float) * 3 * (size_t)nS) : NULL;
    if (Xs) memcpy(Xs, X, sizeof(float) * 3 * (size_t)nS);
    surf32 S = { m, X0, LS, nn, vn, frow, ftab, FS, Xs };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) surf_vertex_f32(&S, X, v, gs);
    free(Xs);
}

void or_dmo_surf_f32(const or_mesh* m, float* X, const float* X0, const float* LS, const int32_t* nn,
                     const float* vn, int v0, int v1, float gs, int nthreads) {
    surf32 S = { m, X0, LS, nn, vn, NULL, NULL, NULL, NULL };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) surf_vertex_f32(&S, X, v, gs);
}

/* ======================================================================================== */
/* surface element qualities + optimisation loops                                            */
/* ======================================================================================== */
void or_surface_qualities_f64(const or_mesh* m, const double* X, double* q) {
    const int nF = or_mesh_info(m, OR_I_NTRIS), fk = or__fk(m);
    const int* F = or__faces(m);
    for (int t = 0; t < nF; ++t) {
        const int* f = F + fk * (size_t)t;
        const int crit = or__criterion();
        if (fk == 3 && crit != OR_MEAN_RATIO)
            q[t] = or_q_tri3d_angle_f64(X + 3 * f[0], X + 3 * f[1], X + 3 * f[2], NULL, crit == OR_MAX_ANGLE);
        else
            q[t] = fk == 3 ? or_q_tri3d_f64(X + 3 * f[0], X + 3 * f[1], X + 3 * f[2])
                           : or_q_quad_f64(X + 3 * f[0], X + 3 * f[1], X + 3 * f[2], X + 3 * f[3], NULL);
    }
}

void or_surface_qualities_f32(const or_mesh* m, const float* X, float* q) {
    const int nF = or_mesh_info(m, OR_I_NTRIS), fk = or__fk(m);
    const int* F = or__faces(m);
    for (int t = 0; t < nF; ++t) {
        const int* f = F + fk * (size_t)t;
        q[t] = fk == 3 ? or_q_tri3d_f32(X + 3 * f[0], X + 3 * f[1], X + 3 * f[2])
                       : or_q_quad_f32(X + 3 * f[0], X + 3 * f[1], X + 3 * f[2], X + 3 * f[3], NULL);
    }
}

void or_optimize_surf_f32(const or_mesh* m, float* X, int n_iter, float gs, int nthreads,
                          double* min_hist, double* mean_hist) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nF = or_mesh_info(m, OR_I_NTRIS);
    const int nc = or_mesh_info(m, OR_I_NCOL_FREE);
    const int* off = or__col(m, 0);
    float* X0 = (float*)malloc(sizeof(float) * 3 * (size_t)nS);
    float* fn = (float*)malloc(sizeof(float) * 3 * (size_t)nF);
    float* vn = (float*)malloc(sizeof(float) * 3 * (size_t)nS);
    float* LS = (float*)malloc(sizeof(float) * LSF * (size_t)nS);
    int32_t* nn = (int32_t*)malloc(sizeof(int32_t) * (size_t)nS);
    float* q = (float*)malloc(sizeof(float) * (size_t)nF);
    memcpy(X0, X, sizeof(float) * 3 * (size_t)nS);
    or_surface_normals_f32(m, X, fn, vn);
    or_surface_fit_f32(m, X, vn, LS);
    for (int i = 0; i < nS; ++i) nn[i] = i;
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) or_dmo_surf_f32(m, X, X0, LS, nn, vn, off[c], off[c + 1], gs, nthreads);
        or_update_nn_f32(m, X, X0, nn);
        or_surface_normals_f32(m, X, fn, vn);
        if (min_hist || mean_hist) {
            or_surface_qualities_f32(m, X, q);
            double mn = DBL_MAX, s = 0.0;
            for (int i = 0; i < nF; ++i) { mn = fmin(mn, q[i]); s += q[i]; }
            if (min_hist) min_hist[it] = mn;
            if (mean_hist) mean_hist[it] = s / nF;
        }
    }
    free(X0); free(fn); free(vn); free(LS); free(nn); free(q);
}

static void normals_f64(const or_mesh* m, const double* X, double* fn, double* vn) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nF = or_mesh_info(m, OR_I_NTRIS), fk = or__fk(m);
    const int* F = or__faces(m);
    for (int t = 0; t < nF; ++t) {
        const double* p0 = X + 3 * (size_t)F[fk * t];
        const double* p1 = X + 3 * (size_t)F[fk * t + 1];
        const double* p2 = X + 3 * (size_t)F[fk * t + (fk == 4 ? 3 : 2)];
        double e0[3] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
        double e1[3] = { p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2] };
        double n[3] = { e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0] };
        double len = sqrt(dot3d(n, n));
        for (int a = 0; a < 3; ++a) fn[3 * t + a] = n[a] / len;
    }
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    for (int v = 0; v < nS; ++v) {
        double n[3] = { 0, 0, 0 };
        for (int i = rp[v]; i < rp[v + 1]; ++i) {
            int f = he[4 * i + 2];
            if (f != -1) for (int a = 0; a < 3; ++a) n[a] += fn[3 * f + a];
        }
        double len = sqrt(dot3d(n, n));
        for (int a = 0; a < 3; ++a) vn[3 * v + a] = n[a] / len;
    }
}

/* face and vertex normals in double (MeshGPUCommon.cu:363-434), for the f64 iteration loops */
void or_surface_normals_f64(const or_mesh* m, const double* X, double* fn, double* vn) { normals_f64(m, X, fn, vn); }

void or_optimize_surf_f64(const or_mesh* m, double* X, int n_iter, double gs, int nthreads,
                          double* min_hist, double* mean_hist) {
    const int nS = or_mesh_info(m, OR_I_NSURF), nF = or_mesh_info(m, OR_I_NTRIS);
    const int nc = or_mesh_info(m, OR_I_NCOL_FREE);
    const int* off = or__col(m, 0);
    double* X0 = (double*)malloc(sizeof(double) * 3 * (size_t)nS);
    double* fn = (double*)malloc(sizeof(double) * 3 * (size_t)nF);
    double* vn = (double*)malloc(sizeof(double) * 3 * (size_t)nS);
    double* LS = (double*)malloc(sizeof(double) * LSF * (size_t)nS);
    int32_t* nn = (int32_t*)malloc(sizeof(int32_t) * (size_t)nS);
    double* q = (double*)malloc(sizeof(double) * (size_t)nF);
    memcpy(X0, X, sizeof(double) * 3 * (size_t)nS);
    normals_f64(m, X, fn, vn);
    or_surface_fit_f64(m, X, vn, LS);
    for (int i = 0; i < nS; ++i) nn[i] = i;
    for (int it = 0; it < n_iter; ++it) {
        for (int c = 0; c < nc; ++c) or_dmo_surf_f64(m, X, X0, LS, nn, vn, off[c], off[c + 1], gs, NULL, nthreads);
        or_update_nn_f64(m, X, X0, nn);
        normals_f64(m, X, fn, vn);
        if (min_hist || mean_hist) {
            or_surface_qualities_f64(m, X, q);
            double mn = DBL_MAX, s = 0.0;
            for (int i = 0; i < nF; ++i) { mn = fmin(mn, q[i]); s += q[i]; }
            if (min_hist) min_hist[it] = mn;
            if (mean_hist) mean_hist[it] = s / nF;
        }
    }
    free(X0); free(fn); free(vn); free(LS); free(nn); free(q);
}

/* ======================================================================================== */
/* sample grids of the surface views (dmo/DMOCommon.cu:73-150, dmo/DMOCommon.h:196-276)     */
/* ======================================================================================== */
void or_surface_points_f32(const or_mesh* m, const float* X, const float* X0, const float* LS, const int32_t* nn,
                           int vid, int nu, int nv, float gs, int estimate_mode, float* out) {
    const int* rp = or__he_rowptr(m);
    const int* he = or__he(m);
    surf32 S = { m, X0, LS, nn, NULL };
    const float* c0 = X + 3 * (size_t)vid;
    float md = -FLT_MAX;
    for (int i = rp[vid]; i < rp[vid + 1]; ++i) {
        const float* t = X + 3 * (size_t)he[4 * i];
        float d[3] = { t[0] - c0[0], t[1] - c0[1], t[2] - c0[2] };
        md = fmaxf(md, sqrtf(dot3f(d, d)));
    }
    const float* L = LS + LSF * (size_t)nn[vid];
    float q[3] = { c0[0] - L[0], c0[1] - L[1], c0[2] - L[2] };
    const float cu = dot3f(q, L + 4), cv = dot3f(q, L + 8);
    float uMax = gs * md, uMin = -gs * md, vMax = gs * md, vMin = -gs * md;
    if (!estimate_mode) { uMin *= 2.f; uMax *= 2.f; vMin *= 2.f; vMax *= 2.f; }
    const float afU = 1.f / (float)(nu - 1), afV = 1.f / (float)(nv - 1);
    for (int idx = 0; idx < nu * nv; ++idx) {
        const int j = idx % nu, i = idx / nu;
        const float u = cu + afU * ((float)i * uMin + (float)(nu - 1 - i) * uMax);
        const float v = cv + afV * ((float)j * vMin + (float)(nv - 1 - j) * vMax);
        float* o = out + 3 * (size_t)idx;
        if (estimate_mode) {
            est32(&S, vid, u, v, o);
        } else {
            const float w = poly32(L, u, v);
            for (int a = 0; a < 3; ++a) o[a] = ((L[a] + u * L[4 + a]) + v * L[8 + a]) + w * L[12 + a];
        }
    }
}


/* ======================================================================================== */
/* boundary-surface pass of volume meshes (k_optimizeHierarchical2DTet, dmo/DMOTetImplCub.h:  */
/* 142-325; k_optimizeHierarchical2DHex, dmo/DMOHexImplCub.h:142-317): the surface search of   */
/* the free boundary vertices judged by their ring of tets / halfhexes (or_vring.c)            */
/* ======================================================================================== */
extern const int* or__hf_rowptr(const or_mesh* m);

static void vol_surf_vertex_f32(const surf32* S, float* X, int v, float gs) {
    const or_mesh* m = S->m;
    or_vring32 R;
    if (!or__vring32_init(&R, m, X, v)) { or__vring32_free(&R); return; }
    const float md = R.md;
    float c0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    float cur[3] = { c0[0], c0[1], c0[2] };
    const float* L = S->LS + LSF * (size_t)S->nn[v];
    float dl[3] = { c0[0] - L[0], c0[1] - L[1], c0[2] - L[2] };
    float cu = dot3f(dl, L + 4), cv = dot3f(dl, L + 8);
    const float qOld = or__vring32_key(&R, c0);
    float ds = gs, lastMax = -FLT_MAX;
    for (int d = 0; d < DEPTH; ++d) {
        float S_ = ds * md;
        float us[NQ], vs[NQ];
        for (int i = 0; i < NQ; ++i) { us[i] = fmaf(grid_offset(i), S_, cu); vs[i] = fmaf(grid_offset(i), S_, cv); }
        float bv = 0.f, bu = 0.f, bvv = 0.f, bp[3] = { 0.f, 0.f, 0.f };
        int bt = -1;
        for (int t = 0; t < 32; ++t) {
            int i1 = t >> 3, j1 = t & 7, i2 = i1 + 4;
            float pw1[3], pw2[3];
            est32(S, v, us[i1], vs[j1], pw1);
            est32(S, v, us[i2], vs[j1], pw2);
            float q1 = or__vring32_key(&R, pw1), q2 = or__vring32_key(&R, pw2);
            float val = q1; int second = 0;
            if (q2 > q1) { val = q2; second = 1; }
            if (bt < 0 || val > bv) {
                bv = val; bt = t;
                bu = second ? us[i2] : us[i1]; bvv = vs[j1];
                const float* pp = second ? pw2 : pw1;
                bp[0] = pp[0]; bp[1] = pp[1]; bp[2] = pp[2];
            }
        }
        const float qLast = or__vring32_key(&R, cur);
        if (qLast < bv) { cur[0] = bp[0]; cur[1] = bp[1]; cur[2] = bp[2]; cu = bu; cv = bvv; }
        lastMax = bv;
        ds = ds * (2.0f / (float)(NQ - 1));
    }
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    or__vring32_free(&R);
}

void or_dmo_vol_surf_f32(const or_mesh* m, float* X, const float* X0, const float* LS, const int32_t* nn,
                         const int32_t* frow, const int32_t* ftab, const float* FS, int v0, int v1, float gs,
                         int nthreads) {
    const int nS = or_mesh_info(m, OR_I_NSURF);
    float* Xs = FS ? (float*)malloc(sizeof(float) * 3 * (size_t)or_mesh_info(m, OR_I_NV)) : NULL;
    if (Xs) memcpy(Xs, X, sizeof(float) * 3 * (size_t)or_mesh_info(m, OR_I_NV));
    (void)nS;
    surf32 S = { m, X0, LS, nn, NULL, frow, ftab, FS, Xs };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) vol_surf_vertex_f32(&S, X, v, gs);
    free(Xs);
}

static void vol_surf_vertex_f64(const surf64* S, double* X, int v, double gs, double* margin) {
    const or_mesh* m = S->m;
    const int* rp = or__hf_rowptr(m);
    if (rp[v + 1] - rp[v] <= 0) { if (margin) *margin = DBL_MAX; return; }
    double p0[3] = { X[3 * v], X[3 * v + 1], X[3 * v + 2] };
    double cur[3] = { p0[0], p0[1], p0[2] };
    const double md = or__vring64_extent(m, X, v);
    const double* L = S->LS + LSF * (size_t)S->nn[v];
    double dl[3] = { p0[0] - L[0], p0[1] - L[1], p0[2] - L[2] };
    double cu = dot3d(dl, L + 4), cv = dot3d(dl, L + 8);
    const double aff = 1.0 / (NQ - 1);
    double ds = gs, lastMax = -DBL_MAX, mg = DBL_MAX;
    for (int d = 0; d < DEPTH; ++d) {
        double uMax = ds * md, uMin = -ds * md;
        double val[32], uvs[32][2], pts[32][3];
        double best = -DBL_MAX, second = -DBL_MAX;
        for (int t = 0; t < 32; ++t) {
            int i1 = t / NQ, j1 = t % NQ, i2 = i1 + 4;
            double u1 = cu + aff * (i1 * uMin + (NQ - 1 - i1) * uMax);
            double v1 = cv + aff * (j1 * uMin + (NQ - 1 - j1) * uMax);
            double u2 = cu + aff * (i2 * uMin + (NQ - 1 - i2) * uMax);
            double pw1[3], pw2[3];
            est64(S, v, u1, v1, pw1);
            est64(S, v, u2, v1, pw2);
            double q1 = or__vring64_q(m, X, v, pw1), q2 = or__vring64_q(m, X, v, pw2);
            val[t] = q1; uvs[t][0] = u1; uvs[t][1] = v1;
            for (int a = 0; a < 3; ++a) pts[t][a] = pw1[a];
            if (q2 > q1) { val[t] = q2; uvs[t][0] = u2; for (int a = 0; a < 3; ++a) pts[t][a] = pw2[a]; }
            double qs[2] = { q1, q2 };
            for (int s_ = 0; s_ < 2; ++s_) {
                if (qs[s_] > best) { second = best; best = qs[s_]; }
                else if (qs[s_] < best && qs[s_] > second) second = qs[s_];
            }
        }
        double qLast = or__vring64_q(m, X, v, cur);
        int w = 0;
        for (int t = 1; t < 32; ++t) if (val[t] > val[w]) w = t;
        mg = fmin(mg, best - second);
        mg = fmin(mg, or__gap64(best, qLast));
        if (qLast < val[w]) { for (int a = 0; a < 3; ++a) cur[a] = pts[w][a]; cu = uvs[w][0]; cv = uvs[w][1]; }
        lastMax = val[w];
        ds = ds * (2.0 / (NQ - 1));
    }
    double qOld = or__vring64_q(m, X, v, p0);
    mg = fmin(mg, or__gap64(lastMax, qOld));
    if (qOld < lastMax) { X[3 * v] = cur[0]; X[3 * v + 1] = cur[1]; X[3 * v + 2] = cur[2]; }
    if (margin) *margin = mg;
}

void or_dmo_vol_surf_f64(const or_mesh* m, double* X, const double* X0, const double* LS, const int32_t* nn,
                         const int32_t* frow, const int32_t* ftab, const double* FS, int v0, int v1, double gs,
                         double* margin, int nthreads) {
    double* Xs = FS ? (double*)malloc(sizeof(double) * 3 * (size_t)or_mesh_info(m, OR_I_NV)) : NULL;
    if (Xs) memcpy(Xs, X, sizeof(double) * 3 * (size_t)or_mesh_info(m, OR_I_NV));
    surf64 S = { m, X0, LS, nn, NULL, frow, ftab, FS, Xs };
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int v = v0; v < v1; ++v) vol_surf_vertex_f64(&S, X, v, gs, margin ? margin + (v - v0) : NULL);
    free(Xs);
}
