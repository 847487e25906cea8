/* The reference's own mesh build and DMO, run as a checker (TEST INFRASTRUCTURE ONLY).
 *
 * `make -C oracle ref` compiles the reference's translation units where they lie
 * (VSDMO/src/mesh/{MeshGPUCommon,MeshTriGPU,MeshTetGPU,MeshQuadGPU,MeshHexGPU,SortUtil,
 * VertexColoring,CopyUtil}.cu, VSDMO/src/dmo/{DMOTet,DMOTri,DMOTriFlat,DMOQuad,DMOHex,DMOCommon,
 * Surface1D}.cu, dmo/surfaceP/{Surface,SurfaceFeature}.cu, Timer.cpp) with the forced-include
 * prelude ref_prelude_vsdmo.h, and links them with this file into oracle/_ref/libref_vsdmo.so.
 * The tests compare the library with it; nothing in the library links it.
 *
 * Colouring seam. The reference colours with the closed cusparseScsrcolor
 * (mesh/VertexColoring.cu:128-153) and keeps its own Jones-Plassmann-Luby colouring beside it
 * (color_jpl(start, n, ...), VertexColoring.cu:107-125, priorities n - i). VertexColoring.cu is
 * compiled with its color_cuSPARSE renamed to refvs_cusparse_colouring, and the color_cuSPARSE
 * defined below calls the reference's color_jpl(0, n, ...) instead, or the renamed cuSPARSE
 * colouring, or the rounds of the reference's k_color_jpl_kernel with the library's hashed
 * priorities (refvs_set_colouring). Every other line that runs is the reference's.
 *
 * Meshes are created the way the reference's file parsers fill them (io/ParserOFF.cu:47-84,
 * io/ParserTetGen.cu:49-110, io/ParserHex.cu:152-237), then MeshXxxGPU::init() and the DMOMeshXxx
 * constructor run as in the factories (mesh/MeshFactory.cu). Array ids, kinds and formats are the
 * library's (VSDMO_A_*, elem types TRI 0 / QUAD 1 / TET 2 / HEX 3), so outputs compare directly.
 * The reference writes progress to std::cout; the calls here discard it. CUDA errors inside the
 * reference end the process (its gpuErrchk calls exit). */
#include "mesh/MeshTriGPU.h"
#include "mesh/MeshTetGPU.h"
#include "mesh/MeshQuadGPU.h"
#include "mesh/MeshHexGPU.h"
#include "mesh/DMOMeshTri.h"
#include "mesh/DMOMeshTet.h"
#include "mesh/DMOMeshQuad.h"
#include "mesh/DMOMeshHex.h"
#include "mesh/VertexColoring.h"
#include "dmo/DMOTet.h"
#include "dmo/DMOTri.h"
#include "dmo/DMOTriFlat.h"
#include "dmo/DMOQuad.h"
#include "dmo/DMOHex.h"
#include "dmo/DMOCommon.h"
#include "dmo/DMOTetImplCub.h"
#include "dmo/DMOTriFlatImplCub.h"
#include "dmo/DMOHexImplCub.h"
#include "dmo/DMOTriImplCub.h"
#include "dmo/DMOQuadImplCub.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <sstream>
#include <vector>

void refvs_cusparse_colouring(int nVertices, int* rowPtr, int* colInd, device_vector<int>& colors, int nnz);
// the reference's JPL round kernel (mesh/VertexColoring.cu:76-105), defined there
__global__ void k_color_jpl_kernel(int start, int nVertices, int c, int* rowPtr, int* colInd, ArrayView<int> randoms,
                                   ArrayView<int> colors);

namespace {
// 0: the reference's color_jpl (priorities n - i); 1: cusparseScsrcolor; 2: the reference's JPL
// rounds with the library's hashed priorities (seed g_seed); 3: the library's default colouring
// with those priorities (the smallest colour free among the higher-priority neighbours)
int g_colouring = 0;
uint32_t g_seed = 1;

uint32_t hashed_priority(uint32_t i, uint32_t seed) {  // the library's default priorities
    uint32_t h = i + seed * 0x9E3779B9u;
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// color_jpl(0, n, ...) (VertexColoring.cu:107-125) with other priorities: the same rounds of the
// reference's kernel, the same count of uncoloured vertices after each
void jpl_with_priorities(int n, int* rowPtr, int* colInd, device_vector<int>& colors) {
    std::vector<int> pr(n);
    // unsigned order as signed ints: flip the sign bit (the kernel compares ints)
    for (int i = 0; i < n; ++i) pr[i] = (int)(hashed_priority((uint32_t)i, g_seed) ^ 0x80000000u);
    device_vector<int> randoms(pr.begin(), pr.end());
    thrust::fill(colors.begin(), colors.end(), -1);
    for (int c = 0; c < n; c++) {
        const int nt = 256;
        k_color_jpl_kernel<<<getBlockCount(n, nt), nt>>>(0, n, c, rowPtr, colInd, randoms, colors);
        gpuErrchk(cudaPeekAtLastError());
        gpuErrchk(cudaDeviceSynchronize());
        if ((int)thrust::count(colors.begin(), colors.end(), -1) == 0) break;
    }
}


// The greedy colouring in descending priority order: each vertex takes the smallest colour that
// none of its already coloured (higher-priority) neighbours has -- the colours the library's JPL
// rounds assign by default, computed here sequentially on the host.
void first_fit_with_priorities(int n, int* rowPtr, int* colInd, device_vector<int>& colors, int nnz) {
    std::vector<int> rp(n + 1), ci(std::max(nnz, 1)), order(n), col(n, -1);
    gpuErrchk(cudaMemcpy(rp.data(), rowPtr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    if (nnz > 0) gpuErrchk(cudaMemcpy(ci.data(), colInd, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> pr(n);
    for (int i = 0; i < n; ++i) { pr[i] = hashed_priority((uint32_t)i, g_seed); order[i] = i; }
    std::sort(order.begin(), order.end(), [&](int a, int b) { return pr[a] > pr[b]; });
    std::vector<char> used;
    for (int i : order) {
        used.assign((size_t)(rp[i + 1] - rp[i]) + 2, 0);
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
            const int j = ci[e];
            if (j != i && col[j] >= 0 && col[j] < (int)used.size()) used[col[j]] = 1;
        }
        int c = 0;
        while (used[c]) ++c;
        col[i] = c;
    }
    thrust::copy(col.begin(), col.end(), colors.begin());
}
}  // namespace

void color_cuSPARSE(int nVertices, int* rowPtr, int* colInd, device_vector<int>& colors, int nnz) {
    if (g_colouring == 1) refvs_cusparse_colouring(nVertices, rowPtr, colInd, colors, nnz);
    else if (g_colouring == 2) jpl_with_priorities(nVertices, rowPtr, colInd, colors);
    else if (g_colouring == 3) first_fit_with_priorities(nVertices, rowPtr, colInd, colors, nnz);
    else color_jpl(0, nVertices, rowPtr, colInd, colors);
}

namespace {

enum { TRI = 0, QUAD = 1, TET = 2, HEX = 3 };
enum { A_XYZ, A_NEW_OF_OLD, A_ELEMS, A_SURF_TRIS, A_HE_ROWPTR, A_HALFEDGES, A_HF_ROWPTR, A_HALFFACES,
       A_COL_FREE, A_COL_FEATURE, A_COL_INNER, A_IS_BOUNDARY1D, A_IS_FEATURE, A_IS_BOUNDARY2D,
       A_FACE_NORMALS, A_VERTEX_NORMALS };
enum { I_NV, I_NE, I_NSURF, I_NFEATURE, I_NTRIS, I_NHE, I_NCOLFREE, I_NCOLFEATURE, I_NCOLINNER,
       I_MAXHE, I_MAXELEMS, I_ISFLAT };

struct Quiet {  // discards std::cout for the lifetime of the object
    std::ostringstream sink;
    std::streambuf* old;
    Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

// The reference's surface optimiser classes, unchanged, with read access to the state their
// constructors build (initial positions, local surfaces, nearest initial vertices) and one colour
// launch of their free-vertex kernel exactly as their doIteration issues it
// (dmo/DMOTri.cu:132-138, dmo/DMOQuad.cu:130-138). A derived class sees the protected members.
template <class Base, class MeshT, int RING_FACTOR>
struct SurfaceProbe : Base {
    SurfaceProbe(MeshT& m, QualityCriterium c, float gs, int n) : Base(m, c, gs, n) {}
    void state(float* x0, float* ls, int* nn) {
        const int nS = this->dmo_mesh.nVerticesSurf;
        cudaMemcpy(x0, raw_pointer_cast(this->vertexPointsInit.data()), sizeof(Vec3f) * nS, cudaMemcpyDeviceToHost);
        static_assert(sizeof(SurfLS::localSurface) == 16 * sizeof(float), "localSurface layout");
        cudaMemcpy(ls, raw_pointer_cast(this->localSurfacesInit.data()), sizeof(SurfLS::localSurface) * nS,
                   cudaMemcpyDeviceToHost);
        cudaMemcpy(nn, raw_pointer_cast(this->nearestNeighbors.data()), sizeof(int) * nS, cudaMemcpyDeviceToHost);
    }
    int colour(int cid) {
        MeshT& m = this->dmo_mesh;
        if (cid < 0 || cid >= m.nColorsFree) return -1;
        const int ring = RING_FACTOR * m.maxNumHalfedges + 1;
        const int dyn = ring * 3 * sizeof(float) + m.maxNumHalfedges * sizeof(int);
        DMOImplCub::k_optimizeHierarchical2D<DMO_NQ * DMO_NQ / 2, USE_SURF_OF_NN>
            <<<m.colorOffsetsFree[cid + 1] - m.colorOffsetsFree[cid], DMO_NQ * DMO_NQ / 2, dyn>>>(
                m.colorOffsetsFree[cid], m.colorOffsetsFree[cid + 1], m.d_mesh, this->affineFactor,
                this->qualityCriterium, this->gridScale, raw_pointer_cast(this->vertexPointsInit.data()),
                raw_pointer_cast(this->localSurfacesInit.data()), raw_pointer_cast(this->nearestNeighbors.data()),
                raw(this->table), raw(this->surfacesRowPtr), raw(this->localSurfacesFeatureInit), ring);
        const cudaError_t e = cudaDeviceSynchronize();
        return e == cudaSuccess ? 0 : (int)e;
    }
};
using TriProbe = SurfaceProbe<DMO::DMOTriClass, DMOMeshTri, 1>;
using QuadProbe = SurfaceProbe<DMO::DMOQuadClass, DMOMeshQuad, 2>;

struct RefMesh {
    int kind = TRI;
    int nE = 0;
    std::shared_ptr<DMOMeshTri> tri;
    std::shared_ptr<DMOMeshQuad> quad;
    std::shared_ptr<DMOMeshTet> tet;
    std::shared_ptr<DMOMeshHex> hex;
    DMOMeshBase* base = nullptr;
    std::unique_ptr<DMO::DMOBaseClass> opt;
    float* d_qual = nullptr;
    ~RefMesh() {
        opt.reset();
        if (d_qual) cudaFree(d_qual);
    }
};

std::vector<Vec3f> points_of(const float* xyz, int n) {
    std::vector<Vec3f> p(n);
    for (int i = 0; i < n; ++i) p[i] = Vec3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return p;
}

template <class E>
std::vector<E> elems_of(const int* el, int n) {
    std::vector<E> e(n);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < E::numVertices; ++c) e[i].data[c] = el[(long)E::numVertices * i + c];
    return e;
}

int device_int(const int* p) {
    int v = 0;
    cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
    return v;
}

long copy_out(void* out, const void* dev, long count, size_t elem) {
    if (out && count > 0) cudaMemcpy(out, dev, count * elem, cudaMemcpyDeviceToHost);
    return count;
}

long copy_host(void* out, const host_vector<int>& v) {
    if (out) std::memcpy(out, v.data(), sizeof(int) * v.size());
    return (long)v.size();
}

long copy_flags(void* out, const bool* dev, long n) {  // bool -> uint8
    if (out && n > 0) {
        std::vector<char> b(n);
        cudaMemcpy(b.data(), dev, n, cudaMemcpyDeviceToHost);
        for (long i = 0; i < n; ++i) static_cast<uint8_t*>(out)[i] = b[i] ? 1 : 0;
    }
    return n;
}

}  // namespace

extern "C" {

/* 0: colour with the reference's color_jpl (default); 1: with cusparseScsrcolor; 2: with the
 * reference's JPL rounds and the library's hashed priorities of color_seed `seed`; 3: with the
 * library's default colouring for that seed (the greedy colouring in priority order). */
void refvs_set_colouring(int mode, uint32_t seed) {
    g_colouring = mode;
    g_seed = seed;
}

/* Builds a mesh of `kind` from host arrays as the reference's parsers and factories do.
 * Returns a handle, or null when the kind is unknown. */
void* refvs_mesh_create(int kind, const float* xyz, int nV, const int* elems, int nE) {
    Quiet q;
    auto r = std::make_unique<RefMesh>();
    r->kind = kind;
    r->nE = nE;
    std::vector<Vec3f> pts = points_of(xyz, nV);
    if (kind == TRI || kind == QUAD) {
        bool nonZeroZ = false;  // io/ParserOFF.cu:53-67
        for (int i = 0; i < nV; ++i) nonZeroZ |= xyz[3 * i + 2] != 0.f;
        if (kind == TRI) {
            MeshTriGPU m;
            m.setNumVerticesSurf(nV);
            m.setVertexPoints(pts, nonZeroZ);
            m.setNumTriangles(nE);
            std::vector<Triangle> e = elems_of<Triangle>(elems, nE);
            m.setTriangles(e);
            m.init();
            r->tri = std::make_shared<DMOMeshTri>(m);
            r->base = r->tri.get();
        } else {
            MeshQuadGPU m;
            m.setNumVerticesSurf(nV);
            m.setVertexPoints(pts, nonZeroZ);
            m.setNumQuads(nE);
            std::vector<Quad> e = elems_of<Quad>(elems, nE);
            m.setQuads(e);
            m.init();
            r->quad = std::make_shared<DMOMeshQuad>(m);
            r->base = r->quad.get();
        }
    } else if (kind == TET) {
        MeshTetGPU m;  // io/ParserTetGen.cu:49-110, no boundary markers
        m.setNumVertices(nV);
        m.setVertexPoints(pts);
        m.setNumTetrahedra(nE);
        std::vector<Tetrahedron> e = elems_of<Tetrahedron>(elems, nE);
        m.setTetrahedra(e);
        m.init();
        r->tet = std::make_shared<DMOMeshTet>(m);
        r->base = r->tet.get();
    } else if (kind == HEX) {
        MeshHexGPU m;  // io/ParserHex.cu:152-237
        m.setNumVertices(nV);
        m.setNumHexahedra(nE);
        m.setVertexPoints(pts);
        std::vector<Hexahedron> e = elems_of<Hexahedron>(elems, nE);
        m.setHexahedra(e);
        m.init();
        r->hex = std::make_shared<DMOMeshHex>(m);
        r->base = r->hex.get();
    } else {
        return nullptr;
    }
    cudaDeviceSynchronize();
    return r.release();
}

void refvs_mesh_destroy(void* h) {
    Quiet q;
    delete static_cast<RefMesh*>(h);
}

/* The library's mesh info items (nV, nE, nSurf, nFeature, nTris, nHE, nColorsFree,
 * nColorsFeature, nColorsInner, maxNumHalfedges, maxNumTetrahedra, isFlat). */
int refvs_mesh_info(void* h, int item) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    DMOMeshBase& b = *r.base;
    switch (item) {
    case I_NV: return b.nVertices;
    case I_NE: return r.nE;
    case I_NSURF: return b.nVerticesSurf;
    case I_NFEATURE: return b.nVerticesFeature;
    case I_NTRIS: return r.tet ? r.tet->nTriangles : r.hex ? r.hex->nQuads : r.tri ? r.tri->nTriangles : r.quad->nQuads;
    case I_NHE: return b.nHalfedges;
    case I_NCOLFREE: return b.nColorsFree;
    case I_NCOLFEATURE: return b.nColorsFeature;
    case I_NCOLINNER: return r.tet ? r.tet->nColorsInner : r.hex ? r.hex->nColorsInner : 0;
    case I_MAXHE: return b.maxNumHalfedges;
    case I_MAXELEMS: return r.tet ? r.tet->maxNumTetrahedra : r.hex ? r.hex->maxNumHexahedra : 0;
    case I_ISFLAT: return b.isFlat_ ? 1 : 0;
    default: return -1;
    }
}

/* Copies array `aid` (int32, float or uint8 as the library's VSDMO_A_* of the same id) to host
 * memory `out` when it is not null; returns the number of items (-1: not available). */
long refvs_mesh_array(void* h, int aid, void* out) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    DMOMeshBase& b = *r.base;
    const int nV = b.nVertices, nS = b.nVerticesSurf;
    const int nTris = refvs_mesh_info(h, I_NTRIS);
    switch (aid) {
    case A_XYZ: return copy_out(out, b.vertexPoints.get(), nV, sizeof(Vec3f)) * 3;
    case A_ELEMS:
        if (r.tet) return copy_out(out, r.tet->tetrahedra.get(), r.nE, sizeof(Tetrahedron)) * 4;
        if (r.hex) return copy_out(out, r.hex->hexahedra.get(), r.nE, sizeof(Hexahedron)) * 8;
        if (r.tri) return copy_out(out, r.tri->triangles.get(), r.nE, sizeof(Triangle)) * 3;
        return copy_out(out, r.quad->quads.get(), r.nE, sizeof(Quad)) * 4;
    case A_SURF_TRIS:
        if (r.tet || r.tri) {
            DMOMeshBaseTri* t = r.tet ? static_cast<DMOMeshBaseTri*>(r.tet.get()) : r.tri.get();
            return copy_out(out, t->triangles.get(), nTris, sizeof(Triangle)) * 3;
        } else {
            DMOMeshBaseQuad* t = r.hex ? static_cast<DMOMeshBaseQuad*>(r.hex.get()) : r.quad.get();
            return copy_out(out, t->quads.get(), nTris, sizeof(Quad)) * 4;
        }
    case A_HE_ROWPTR: return copy_out(out, b.halfedges.rowPtr_, nS + 1, sizeof(int));
    case A_HALFEDGES: return copy_out(out, b.halfedges.values_, b.nHalfedges, sizeof(Halfedge)) * 4;
    case A_HF_ROWPTR:
        if (r.tet) return copy_out(out, r.tet->halffaces.rowPtr_, nV + 1, sizeof(int));
        if (r.hex) return copy_out(out, r.hex->halfhexes.rowPtr_, nV + 1, sizeof(int));
        return -1;
    case A_HALFFACES:
        if (r.tet) {
            const long n = device_int(r.tet->halffaces.rowPtr_ + nV);
            return copy_out(out, r.tet->halffaces.values_, n, sizeof(Halfface)) * 3;
        }
        if (r.hex) {
            const long n = device_int(r.hex->halfhexes.rowPtr_ + nV);
            return copy_out(out, r.hex->halfhexes.values_, n, sizeof(Halfhex)) * 7;
        }
        return -1;
    case A_COL_FREE: return copy_host(out, b.colorOffsetsFree);
    case A_COL_FEATURE: return copy_host(out, b.colorOffsetsFeature);
    case A_COL_INNER:
        if (r.tet) return copy_host(out, r.tet->colorOffsetsInner);
        if (r.hex) return copy_host(out, r.hex->colorOffsetsInner);
        return 0;
    case A_IS_BOUNDARY1D: return copy_flags(out, b.vertexIsBoundary1D.get(), nS);
    case A_IS_FEATURE: return copy_flags(out, b.vertexIsFeature.get(), nS);
    case A_IS_BOUNDARY2D:
        if (r.tet) return copy_flags(out, r.tet->vertexIsBoundary2D.get(), nV);
        if (r.hex) return copy_flags(out, r.hex->vertexIsBoundary2D.get(), nV);
        return -1;
    case A_FACE_NORMALS: return copy_out(out, b.faceNormals.get(), nTris, sizeof(Vec3f)) * 3;
    case A_VERTEX_NORMALS: return copy_out(out, b.vertexNormals.get(), nS, sizeof(Vec3f)) * 3;
    default: return -1;
    }
}

/* Overwrites the positions (internal order, nVertices x 3 floats from host memory). */
void refvs_set_positions(void* h, const float* xyz) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    cudaMemcpy(r.base->vertexPoints.get(), xyz, sizeof(Vec3f) * r.base->nVertices, cudaMemcpyHostToDevice);
}

/* One colour launch of the interior search with the reference's launch shape and dynamic shared
 * memory (dmo/DMOTet.cu:129-136 k_optimizeHierarchicalInnerTet<128>, dmo/DMOHex.cu:132-150
 * k_optimizeHierarchicalInnerHex<128>) or, for a flat triangle mesh, of the free-vertex search
 * (dmo/DMOTriFlat.cu:131-138 k_optimizeHierarchical2DFlat<32>). Mean ratio quality. */
int refvs_colour_launch(void* h, int cid, float grid_scale) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    const float affine = 1.f / (DMO_NQ - 1);
    const QualityCriterium q = QualityCriterium::MEAN_RATIO;
    if (r.tet) {
        const host_vector<int>& co = r.tet->colorOffsetsInner;
        if (cid < 0 || cid + 1 >= (int)co.size()) return -1;
        const int dyn = r.tet->maxNumTetrahedra * 3 * 3 * sizeof(float);
        DMOImplCub::k_optimizeHierarchicalInnerTet<128><<<co[cid + 1] - co[cid], 128, dyn>>>(
            co[cid], co[cid + 1], r.tet->d_mesh, affine, q, grid_scale);
    } else if (r.hex) {
        const host_vector<int>& co = r.hex->colorOffsetsInner;
        if (cid < 0 || cid + 1 >= (int)co.size()) return -1;
        const int dyn = r.hex->maxNumHexahedra * 7 * 3 * sizeof(float);
        DMOImplCub::k_optimizeHierarchicalInnerHex<128><<<co[cid + 1] - co[cid], 128, dyn>>>(
            co[cid], co[cid + 1], r.hex->d_mesh, affine, q, grid_scale);
    } else if (r.tri && r.tri->isFlat_) {
        const host_vector<int>& co = r.tri->colorOffsetsFree;
        if (cid < 0 || cid + 1 >= (int)co.size()) return -1;
        const int dyn = (r.tri->maxNumHalfedges + 1) * 3 * sizeof(float) + r.tri->maxNumHalfedges * sizeof(int);
        DMOImplCub::k_optimizeHierarchical2DFlat<DMO_NQ * DMO_NQ / 2><<<co[cid + 1] - co[cid], DMO_NQ * DMO_NQ / 2, dyn>>>(
            co[cid], co[cid + 1], r.tri->d_mesh, affine, q, grid_scale);
    } else {
        return -1;
    }
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

/* n_iter sweeps over every colour of refvs_colour_launch, each launch followed by a device
 * synchronisation as in the reference's doIteration; *ms receives the time of the sweeps
 * (CUDA events). This is the reference's interior search as its host loop runs it with the
 * surface passes off (boundary vertices fixed). */
int refvs_colour_sweeps(void* h, int n_iter, float grid_scale, float* ms) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    const int nc = r.tet ? r.tet->nColorsInner : r.hex ? r.hex->nColorsInner : r.base->nColorsFree;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int st = 0;
    for (int it = 0; it < n_iter && st == 0; ++it)
        for (int c = 0; c < nc && st == 0; ++c) st = refvs_colour_launch(h, c, grid_scale);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

/* The reference's optimiser class for the mesh (DMOTetClass, DMOTriFlatClass for a flat
 * triangle mesh, DMOTriClass, DMOQuadClass, DMOHexClass) with criterion `crit` (the reference's
 * QualityCriterium value), grid scale and iteration count, as DMO::DMOXxxClass(mesh, crit,
 * grid_scale, n_iter). Returns 0 on success. */
int refvs_opt_create(void* h, int crit, float grid_scale, int n_iter) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    Quiet q;
    const QualityCriterium c = static_cast<QualityCriterium>(crit);
    try {
        r.opt.reset();
        if (r.tet) r.opt.reset(new DMO::DMOTetClass(*r.tet, c, grid_scale, n_iter));
        else if (r.hex) r.opt.reset(new DMO::DMOHexClass(*r.hex, c, grid_scale, n_iter));
        else if (r.quad) r.opt.reset(new QuadProbe(*r.quad, c, grid_scale, n_iter));
        else if (r.tri->isFlat_) r.opt.reset(new DMO::DMOTriFlatClass(*r.tri, c, grid_scale, n_iter));
        else r.opt.reset(new TriProbe(*r.tri, c, grid_scale, n_iter));
    } catch (...) {
        return -1;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

/* n calls of the optimiser's doIteration(); 0 on success, -1 when the reference threw (its
 * monotonicity check). */
int refvs_opt_iterate(void* h, int n) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    if (!r.opt) return -3;
    Quiet q;
    try {
        for (int i = 0; i < n; ++i) r.opt->doIteration();
    } catch (...) {
        return -1;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

/* Surface optimisers (DMOTriClass, DMOQuadClass): the state their constructor built, per surface
 * vertex: initial position (3 floats), local surface (16 floats: p0, ei[0..2], a, b, c and the
 * int numPoints, the reference's localSurface) and nearest initial vertex. */
int refvs_opt_surface_state(void* h, float* x0, float* ls, int* nn) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    if (auto* t = dynamic_cast<TriProbe*>(r.opt.get())) { t->state(x0, ls, nn); return 0; }
    if (auto* q = dynamic_cast<QuadProbe*>(r.opt.get())) { q->state(x0, ls, nn); return 0; }
    return -3;
}

/* One colour launch of a surface optimiser's free-vertex kernel as its doIteration issues it. */
int refvs_opt_surface_colour(void* h, int cid) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    if (auto* t = dynamic_cast<TriProbe*>(r.opt.get())) return t->colour(cid);
    if (auto* q = dynamic_cast<QuadProbe*>(r.opt.get())) return q->colour(cid);
    return -3;
}

/* The optimiser's getQuality(): the minimum element quality after the last iteration. */
float refvs_opt_quality(void* h) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    return r.opt ? r.opt->getQuality() : 0.f;
}

/* The optimiser's getElementQualities() into host memory (one float per element). */
int refvs_opt_element_qualities(void* h, float* out) {
    RefMesh& r = *static_cast<RefMesh*>(h);
    if (!r.opt) return -3;
    if (!r.d_qual && cudaMalloc(&r.d_qual, sizeof(float) * (r.nE > 0 ? r.nE : 1)) != cudaSuccess) return -2;
    r.opt->getElementQualities(r.d_qual);
    return cudaMemcpy(out, r.d_qual, sizeof(float) * r.nE, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -2;
}

}  // extern "C"
