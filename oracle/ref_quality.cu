/* The reference's own element quality functions, compiled from its headers as they lie
 * (VSDMO/src/dmo/DMOQuality.h -> DMOQualityTri.h, DMOQualityQuad.h, DMOQualityTet.h,
 * DMOQualityHex.h, DMOQualityUtil.h) into oracle/_ref/libref_quality.so by `make ref`.
 *
 * TEST INFRASTRUCTURE ONLY: the GPU tests evaluate these functions on the same elements as the
 * oracle's restatements and the library's element qualities, which pins both to the reference's
 * arithmetic. Nothing in the library calls this file.
 *
 * One thread per item; each item is an element given by its corner positions (3 floats each;
 * a 2D triangle reads x and y) and, for the normal-signed surface metrics, a normal. */
#include "dmo/DMOQuality.h"
#include <cuda_runtime.h>

namespace {

using DMO::QualityCriterium;

enum RefFn {
    RQ_TET = 0,     // DMO::qualityTet(p[4], crit)                 DMOQualityTet.h:181
    RQ_HEX = 1,     // DMO::qualityHex(p[8], crit)                 DMOQualityHex.h:120
    RQ_QUAD = 2,    // DMO::qualityQuad(p[4], crit)                DMOQualityQuad.h:124
    RQ_TRI = 3,     // DMO::qualityTri(p[3], crit)                 DMOQualityTri.h:410
    RQ_TRI2D = 4,   // DMO::qualityTri2D(Vec2f p[3], crit)         DMOQualityTri.h:395
    RQ_TRI_N = 5,   // mean ratio / min / max angle with normal    DMOQualityTri.h:50,166,276
    RQ_QUAD_N = 6,  // DMO::meanRatioMetricQuad(p[4], n)           DMOQualityQuad.h:30
};

__host__ __device__ int corners_of(int fn) {
    return fn == RQ_HEX ? 8 : (fn == RQ_TET || fn == RQ_QUAD || fn == RQ_QUAD_N) ? 4 : 3;
}

__global__ void k_ref_quality(int fn, int crit, const float* pts, const float* nrm, int n, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = corners_of(fn);
    const float* e = pts + (long)i * 3 * k;
    Vec3f p[8];
    for (int c = 0; c < k; ++c) p[c] = Vec3f(e[3 * c], e[3 * c + 1], e[3 * c + 2]);
    const QualityCriterium q = static_cast<QualityCriterium>(crit);
    float r = 0.f;
    switch (fn) {
    case RQ_TET: r = DMO::qualityTet(p, q); break;
    case RQ_HEX: r = DMO::qualityHex(p, q); break;
    case RQ_QUAD: r = DMO::qualityQuad(p, q); break;
    case RQ_TRI: r = DMO::qualityTri(p, q); break;
    case RQ_TRI2D: {
        Vec2f p2[3];
        for (int c = 0; c < 3; ++c) p2[c] = Vec2f(p[c].x, p[c].y);
        r = DMO::qualityTri2D(p2, q);
        break;
    }
    case RQ_TRI_N: {
        const Vec3f nv(nrm[3L * i], nrm[3L * i + 1], nrm[3L * i + 2]);
        if (q == QualityCriterium::MIN_ANGLE) r = DMO::minAngleMetricTri(p, nv);
        else if (q == QualityCriterium::MAX_ANGLE) r = DMO::maxAngleMetricTri(p, nv);
        else r = DMO::meanRatioMetricTri(p, nv);
        break;
    }
    case RQ_QUAD_N: {
        const Vec3f nv(nrm[3L * i], nrm[3L * i + 1], nrm[3L * i + 2]);
        r = DMO::meanRatioMetricQuad(p, nv);
        break;
    }
    default: r = nanf("");
    }
    out[i] = r;
}

}  // namespace

/* Evaluates reference function `fn` (RefFn) with criterion `crit` (the reference's
 * QualityCriterium value: 0 mean ratio, 4 min angle, 6 max angle) on n items. pts: host array of
 * n x corners x 3 floats; nrm: host array of n x 3 floats (RQ_TRI_N, RQ_QUAD_N; else unused, may
 * be null); out: host array of n floats. Returns a cudaError_t value (0 on success). */
extern "C" int refq_eval(int fn, int crit, const float* pts, const float* nrm, int n, float* out) {
    if (n <= 0) return 0;
    if (fn < RQ_TET || fn > RQ_QUAD_N) return (int)cudaErrorInvalidValue;
    const size_t np = (size_t)n * 3 * corners_of(fn);
    float *dp = nullptr, *dn = nullptr, *dq = nullptr;
    cudaError_t e = cudaMalloc(&dp, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&dn, (size_t)n * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&dq, (size_t)n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(dp, pts, np * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nrm) e = cudaMemcpy(dn, nrm, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !nrm) e = cudaMemset(dn, 0, (size_t)n * 3 * sizeof(float));
    if (e == cudaSuccess) {
        k_ref_quality<<<(n + 127) / 128, 128>>>(fn, crit, dp, dn, n, dq);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dq, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dp);
    cudaFree(dn);
    cudaFree(dq);
    return (int)e;
}
