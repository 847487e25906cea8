/*
 * or_vring.c -- the volume ring of a boundary vertex for the boundary passes of tet and hex
 * meshes (TEST INFRASTRUCTURE ONLY; see vsdmo_oracle.h).
 *
 * f32 (the product's arithmetic, written independently of it): the ring relative to the vertex,
 * scaled by 2^-e (e from frexpf of the largest per-axis ring distance), turned into per-element
 * coefficients once (tets: the 8 of or_dmo.c's tet key; halfhexes: the 43 of or_hex.c's hex
 * key); the key of a candidate p is that of (p - c0) 2^-e.
 * f64 (the reference literally): the ring minimum of the element metric with p as the vertex
 * (qualityTetRing / qualityHexRing, dmo/DMOQualityTet.h:165-177, dmo/DMOQualityHex.h:75-112), tets
 * under the criterion of or_set_criterion (mean ratio, min or max angle).
 * Grid extent: tets the LARGEST Euclidean distance to a ring point (dmo/DMOTetImplCub.h:246,
 * 455), hexes the SMALLEST (dmo/DMOHexImplCub.h:246, 448).
 */
#include "vsdmo_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>

extern const int* or__hf_rowptr(const or_mesh* m);
extern const int* or__hf(const or_mesh* m);
extern int or__type(const or_mesh* m);
void or__tet_coeffs_f32(const float* a, const float* b, const float* c, float* K);
float or__tet_key_f32(int k, const float* K, float x, float y, float z);
float or__hex_key_f32(int k, const float* co, float x, float y, float z, float es, float ea);
double or_q_tet_mean_ratio_f64(const double* p0, const double* p1, const double* p2, const double* p3);

#define HEX_EPS 1.19209e-07f

static int npts(int hex) { return hex ? 7 : 3; }

int or__vring32_init(or_vring32* R, const or_mesh* m, const float* X, int v) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    const int hex = or__type(m) == OR_HEX, np = npts(hex);
    const int b = rp[v], k = rp[v + 1] - b;
    R->hex = hex; R->k = k; R->co = NULL;
    R->c0[0] = X[3 * (size_t)v]; R->c0[1] = X[3 * (size_t)v + 1]; R->c0[2] = X[3 * (size_t)v + 2];
    if (k <= 0) return 0;
    float mm = 0.f, me = hex ? FLT_MAX : -FLT_MAX;
    for (int t = 0; t < k; ++t)
        for (int j = 0; j < np; ++j) {
            const float* q = X + 3 * (size_t)hf[np * (b + t) + j];
            const float d[3] = { q[0] - R->c0[0], q[1] - R->c0[1], q[2] - R->c0[2] };
            mm = fmaxf(mm, fmaxf(fabsf(d[0]), fmaxf(fabsf(d[1]), fabsf(d[2]))));
            const float e = sqrtf((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
            me = hex ? fminf(me, e) : fmaxf(me, e);
        }
    R->md = me;
    if (!(mm > 0.f) || !(mm < FLT_MAX)) return 0;
    (void)frexpf(mm, &R->ex);
    R->es = ldexpf(HEX_EPS, -3 * R->ex);
    R->ea = ldexpf(HEX_EPS, -2 * R->ex);
    R->co = (float*)malloc(sizeof(float) * (hex ? 43 : 8) * (size_t)k);
    for (int t = 0; t < k; ++t) {
        float r[7][3];
        for (int j = 0; j < np; ++j) {
            const float* q = X + 3 * (size_t)hf[np * (b + t) + j];
            for (int a = 0; a < 3; ++a) r[j][a] = ldexpf(q[a] - R->c0[a], -R->ex);
        }
        if (hex) or_hex_coeffs_f32((const float(*)[3])r, R->es, R->ea, R->co + 43 * t);
        else or__tet_coeffs_f32(r[0], r[1], r[2], R->co + 8 * t);
    }
    return 1;
}

float or__vring32_key(const or_vring32* R, const float* p) {
    const float x = ldexpf(p[0] - R->c0[0], -R->ex), y = ldexpf(p[1] - R->c0[1], -R->ex),
                z = ldexpf(p[2] - R->c0[2], -R->ex);
    return R->hex ? or__hex_key_f32(R->k, R->co, x, y, z, R->es, R->ea) : or__tet_key_f32(R->k, R->co, x, y, z);
}

void or__vring32_free(or_vring32* R) { free(R->co); R->co = NULL; }

double or__vring64_q(const or_mesh* m, const double* X, int v, const double* p) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    double q = DBL_MAX;
    if (or__type(m) == OR_HEX) {
        for (int i = rp[v]; i < rp[v + 1]; ++i) {
            double c[8][3];
            for (int a = 0; a < 3; ++a) c[0][a] = p[a];
            for (int j = 0; j < 7; ++j)
                for (int a = 0; a < 3; ++a) c[1 + j][a] = X[3 * (size_t)hf[7 * i + j] + a];
            q = fmin(q, or_q_hex_f64((const double(*)[3])c));
        }
        return q;
    }
    const int crit = or__criterion();
    double (*metric)(const double*, const double*, const double*, const double*) =
        crit == OR_MIN_ANGLE ? or_q_tet_min_angle_f64 : (crit == OR_MAX_ANGLE ? or_q_tet_max_angle_f64 : or_q_tet_mean_ratio_f64);
    for (int i = rp[v]; i < rp[v + 1]; ++i)
        q = fmin(q, metric(p, X + 3 * (size_t)hf[3 * i], X + 3 * (size_t)hf[3 * i + 1], X + 3 * (size_t)hf[3 * i + 2]));
    return q;
}

double or__vring64_extent(const or_mesh* m, const double* X, int v) {
    const int* rp = or__hf_rowptr(m);
    const int* hf = or__hf(m);
    const int hex = or__type(m) == OR_HEX, np = npts(hex);
    const double* c0 = X + 3 * (size_t)v;
    double me = hex ? DBL_MAX : -DBL_MAX;
    for (int i = rp[v]; i < rp[v + 1]; ++i)
        for (int j = 0; j < np; ++j) {
            const double* q = X + 3 * (size_t)hf[np * i + j];
            const double d[3] = { q[0] - c0[0], q[1] - c0[1], q[2] - c0[2] };
            const double e = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            me = hex ? fmin(me, e) : fmax(me, e);
        }
    return me;
}

/* decision margin of a comparison of two ring values: under the shape metrics an exact tie in
 * double is structural (the ring minimum of both is a part that does not depend on the candidate
 * -- a halfhex's constant sub-tets, or 0), and the f32 keys tie exactly too, so it decides
 * nothing. Under the angle criteria an exact tie is not safe: the dihedral angle at a ring edge
 * that lies on the line a boundary vertex slides along is constant along the line, but its float
 * evaluations at two positions differ in the last bits, so the float search can decide either
 * way -- such a comparison has no margin. */
double or__gap64(double a, double b) {
    if (a != b) return fabs(a - b);
    const int c = or__criterion();
    return c == OR_MIN_ANGLE || c == OR_MAX_ANGLE ? 0.0 : DBL_MAX;
}
