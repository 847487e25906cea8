// DMO.hpp -- C++ host API with the reference's class names, over the C ABI of vsdmo.h.
//
// Mirrors the interface a user of DanielZint/VolumeSurfaceDiscreteMeshOptimization calls:
//   DMOMeshTri/Quad/Tet/HexFactory::create          mesh/MeshFactory.h:17-40 (arrays, files, boundaries)
//   writeOFF / writeTetgen / writeHex               io/FileWriter.h
//   DMOMeshTri / DMOMeshQuad / DMOMeshTet           mesh/DMOMeshTri.h:81-94, mesh/DMOMeshQuad.h,
//                                                   mesh/DMOMeshTet.h:145-198
//   DMO::QualityCriterium                           dmo/DMOQualityUtil.h:10-18
//   DMO::DMOBaseClass, DMOTetClass, DMOTriFlatClass dmo/DMOBase.h:23-88, dmo/DMOTet.h:21-62,
//                                                   dmo/DMOTriFlat.h:19-51
//   DMO::DMOTriClass, DMOQuadClass (surfaces)       dmo/DMOTri.h, dmo/DMOQuad.h
//   DMOMeshHex, DMO::DMOHexClass                    mesh/DMOMeshHex.h, dmo/DMOHex.h
// Header-only; link against libvsdmo.so. Errors surface as DMO::Error exceptions carrying the
// vsdmo_status (the reference exits through gpuErrchk or throws 1 instead).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <cstdint>

#include "../vsdmo.h"

namespace DMO {

struct Error : std::runtime_error {
    vsdmo_status status;
    Error(vsdmo_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(vsdmo_status s) {
    if (s != VSDMO_OK) throw Error(s, std::string(vsdmo_status_string(s)) + ": " + vsdmo_last_error());
}

enum class QualityCriterium { MEAN_RATIO = 0, AREA, RIGHT_ANGLE, JACOBIAN, MIN_ANGLE, RADIUS_RATIO, MAX_ANGLE, CONDITION };

// Owns a device mesh (connectivity, colouring, positions) built from host or device arrays.
class DMOMesh {
public:
    DMOMesh(int elemType, const float* xyz, int nVertices, const int32_t* elems, int nElems,
            int memSpace = VSDMO_HOST, uint32_t colorSeed = 1, void* cudaStream = nullptr) {
        check(vsdmo_mesh_create(elemType, xyz, nVertices, elems, nElems, memSpace, colorSeed, cudaStream, &h_));
        nVertices_ = vsdmo_mesh_info(h_, VSDMO_I_NV);
        nVerticesSurf = vsdmo_mesh_info(h_, VSDMO_I_NSURF);
        nVerticesFeature = vsdmo_mesh_info(h_, VSDMO_I_NFEATURE);
        nColorsFree = vsdmo_mesh_info(h_, VSDMO_I_NCOL_FREE);
        nColorsFeature = vsdmo_mesh_info(h_, VSDMO_I_NCOL_FEATURE);
        nColorsInner = vsdmo_mesh_info(h_, VSDMO_I_NCOL_INNER);
        maxNumHalfedges = vsdmo_mesh_info(h_, VSDMO_I_MAX_HE);
        maxNumTetrahedra = vsdmo_mesh_info(h_, VSDMO_I_MAX_TETS);
    }
    // adopts a handle made by vsdmo_mesh_create_from_file / vsdmo_mesh_create_surface
    explicit DMOMesh(vsdmo_mesh_t adopted) : h_(adopted) {
        nVertices_ = vsdmo_mesh_info(h_, VSDMO_I_NV);
        nVerticesSurf = vsdmo_mesh_info(h_, VSDMO_I_NSURF);
        nVerticesFeature = vsdmo_mesh_info(h_, VSDMO_I_NFEATURE);
        nColorsFree = vsdmo_mesh_info(h_, VSDMO_I_NCOL_FREE);
        nColorsFeature = vsdmo_mesh_info(h_, VSDMO_I_NCOL_FEATURE);
        nColorsInner = vsdmo_mesh_info(h_, VSDMO_I_NCOL_INNER);
        maxNumHalfedges = vsdmo_mesh_info(h_, VSDMO_I_MAX_HE);
        maxNumTetrahedra = vsdmo_mesh_info(h_, VSDMO_I_MAX_TETS);
    }
    DMOMesh(const DMOMesh&) = delete;
    DMOMesh& operator=(const DMOMesh&) = delete;
    virtual ~DMOMesh() { vsdmo_mesh_destroy(h_); }
    // writes the current positions in the caller's numbering (io/FileWriter.cu)
    void write(const std::string& filename, int format = VSDMO_FMT_AUTO) const {
        check(vsdmo_mesh_write_file(h_, filename.c_str(), format));
    }

    vsdmo_mesh_t handle() const { return h_; }
    int nVertices() const { return nVertices_; }
    std::vector<float> getVertexPoints(bool originalOrder = true) const {
        std::vector<float> out(3 * (size_t)nVertices_);
        check(vsdmo_mesh_get_positions(h_, out.data(), originalOrder ? 1 : 0, VSDMO_HOST));
        return out;
    }
    std::vector<int32_t> permutation() const {
        std::vector<int32_t> p(nVertices_);
        check(vsdmo_mesh_permutation(h_, p.data()));
        return p;
    }

    int nVerticesSurf = 0, nVerticesFeature = 0;
    int nColorsFree = 0, nColorsFeature = 0, nColorsInner = 0;
    int maxNumHalfedges = 0, maxNumTetrahedra = 0;

private:
    vsdmo_mesh_t h_ = nullptr;
    int nVertices_ = 0;
};

class DMOMeshTri : public DMOMesh {
public:
    explicit DMOMeshTri(vsdmo_mesh_t adopted) : DMOMesh(adopted) {}
    DMOMeshTri(int nVS, int nT, const float* points, const int32_t* tris, int memSpace = VSDMO_HOST)
        : DMOMesh(VSDMO_TRI, points, nVS, tris, nT, memSpace) {}
};

class DMOMeshQuad : public DMOMesh {
public:
    explicit DMOMeshQuad(vsdmo_mesh_t adopted) : DMOMesh(adopted) {}
    DMOMeshQuad(int nVS, int nQ, const float* points, const int32_t* quads, int memSpace = VSDMO_HOST)
        : DMOMesh(VSDMO_QUAD, points, nVS, quads, nQ, memSpace) {}
};

class DMOMeshTet : public DMOMesh {
public:
    explicit DMOMeshTet(vsdmo_mesh_t adopted) : DMOMesh(adopted) {}
    DMOMeshTet(int nV, int nT, const float* points, const int32_t* tets, int memSpace = VSDMO_HOST)
        : DMOMesh(VSDMO_TET, points, nV, tets, nT, memSpace) {}
};

class DMOMeshHex : public DMOMesh {
public:
    explicit DMOMeshHex(vsdmo_mesh_t adopted) : DMOMesh(adopted) {}
    DMOMeshHex(int nV, int nH, const float* points, const int32_t* hexes, int memSpace = VSDMO_HOST)
        : DMOMesh(VSDMO_HEX, points, nV, hexes, nH, memSpace) {}
};

namespace detail {
// nullptr when the file cannot be opened or parsed (the reference's factories return nullptr)
template <class M>
std::shared_ptr<M> from_file(const std::string& filename, int expect) {
    vsdmo_mesh_t h = nullptr;
    const vsdmo_status st = vsdmo_mesh_create_from_file(filename.c_str(), VSDMO_FMT_AUTO, 1, nullptr, &h);
    if (st == VSDMO_E_IO) return nullptr;
    check(st);
    if (vsdmo_mesh_info(h, VSDMO_I_ELEM_TYPE) != expect) {
        vsdmo_mesh_destroy(h);
        throw Error(VSDMO_E_ARG, filename + " holds another element type");
    }
    return std::make_shared<M>(h);
}
template <class M>
std::shared_ptr<M> surface_of(const DMOMesh& volume) {
    vsdmo_mesh_t h = nullptr;
    check(vsdmo_mesh_create_surface(volume.handle(), 1, nullptr, &h));
    return std::make_shared<M>(h);
}
}  // namespace detail

struct DMOMeshTriFactory {
    static std::shared_ptr<DMOMeshTri> create(const std::string& filename) {
        return detail::from_file<DMOMeshTri>(filename, VSDMO_TRI);
    }
    static std::shared_ptr<DMOMeshTri> create(const DMOMeshTet& tetmesh) { return detail::surface_of<DMOMeshTri>(tetmesh); }
    static std::shared_ptr<DMOMeshTri> create(int nVS, int nT, const float* points, const int32_t* tris,
                                              int memSpace = VSDMO_HOST) {
        return std::make_shared<DMOMeshTri>(nVS, nT, points, tris, memSpace);
    }
};

struct DMOMeshQuadFactory {
    static std::shared_ptr<DMOMeshQuad> create(const std::string& filename) {
        return detail::from_file<DMOMeshQuad>(filename, VSDMO_QUAD);
    }
    static std::shared_ptr<DMOMeshQuad> create(const DMOMeshHex& hexmesh) { return detail::surface_of<DMOMeshQuad>(hexmesh); }
    static std::shared_ptr<DMOMeshQuad> create(int nVS, int nQ, const float* points, const int32_t* quads,
                                               int memSpace = VSDMO_HOST) {
        return std::make_shared<DMOMeshQuad>(nVS, nQ, points, quads, memSpace);
    }
};

struct DMOMeshHexFactory {
    static std::shared_ptr<DMOMeshHex> create(const std::string& filename) {
        return detail::from_file<DMOMeshHex>(filename, VSDMO_HEX);
    }
    static std::shared_ptr<DMOMeshHex> create(int nV, int nH, const float* points, const int32_t* hexes,
                                              int memSpace = VSDMO_HOST) {
        return std::make_shared<DMOMeshHex>(nV, nH, points, hexes, memSpace);
    }
};

struct DMOMeshTetFactory {
    static std::shared_ptr<DMOMeshTet> create(const std::string& filename) {
        return detail::from_file<DMOMeshTet>(filename, VSDMO_TET);
    }
    static std::shared_ptr<DMOMeshTet> create(int nV, int nT, const float* points, const int32_t* tets,
                                              int memSpace = VSDMO_HOST) {
        return std::make_shared<DMOMeshTet>(nV, nT, points, tets, memSpace);
    }
};

// io/FileWriter.h names
inline void writeOFF(const std::string& filename, const DMOMeshTri& mesh) { mesh.write(filename + ".off", VSDMO_FMT_OFF); }
inline void writeOFF(const std::string& filename, const DMOMeshQuad& mesh) { mesh.write(filename + ".off", VSDMO_FMT_OFF); }
inline void writeTetgen(const std::string& filename, const DMOMeshTet& mesh) { mesh.write(filename, VSDMO_FMT_TETGEN); }
inline void writeHex(const std::string& filename, const DMOMeshHex& mesh) { mesh.write(filename + ".mesh", VSDMO_FMT_MEDIT); }

class DMOBaseClass {
public:
    DMOBaseClass(DMOMesh& mesh, QualityCriterium q, float gridScale, int n_iter, int flat, bool fixBoundary)
        : mesh_(mesh) {
        vsdmo_params p;
        check(vsdmo_params_default(VSDMO_TET, &p));
        p.quality = (int)q;
        p.grid_scale = gridScale;
        p.n_iter = n_iter;
        p.flat = flat;
        p.fix_boundary = fixBoundary ? 1 : 0;
        check(vsdmo_opt_create(mesh.handle(), &p, &h_));
    }
    DMOBaseClass(const DMOBaseClass&) = delete;
    DMOBaseClass& operator=(const DMOBaseClass&) = delete;
    virtual ~DMOBaseClass() { vsdmo_opt_destroy(h_); }

    void optimize() { check(vsdmo_opt_optimize(h_)); }
    void doIteration() { check(vsdmo_opt_iterate(h_, 1)); }
    bool isDone() const { return vsdmo_opt_is_done(h_) != 0; }
    float getQuality() const {
        float q = 0.f;
        check(vsdmo_opt_get_quality(h_, &q));
        return q;
    }
    float findMinimumQuality() const {
        float q = 0.f;
        check(vsdmo_opt_find_min_quality(h_, &q, nullptr));
        return q;
    }
    void displayQualityGPU(int n_cols = 10) { check(vsdmo_opt_display_quality(h_, n_cols)); }
    // device pointer to nElements floats, like the reference's getElementQualities(void*)
    void getElementQualities(void* outFloatBuffer) { check(vsdmo_opt_element_qualities(h_, (float*)outFloatBuffer, VSDMO_DEVICE)); }
    void getQualityHistogram(std::vector<int>& vec, int n_cols) {
        vec.resize(n_cols);
        check(vsdmo_opt_quality_histogram(h_, vec.data(), n_cols));
    }
    vsdmo_opt_t handle() const { return h_; }

protected:
    DMOMesh& mesh_;
    vsdmo_opt_t h_ = nullptr;
};

class DMOTetClass : public DMOBaseClass {
public:
    DMOTetClass(DMOMeshTet& mesh, QualityCriterium q = QualityCriterium::MEAN_RATIO, float gridScale = 0.5f,
                int n_iter = 30, bool fixBoundary = true)
        : DMOBaseClass(mesh, q, gridScale, n_iter, -1, fixBoundary) {}
};

class DMOTriFlatClass : public DMOBaseClass {
public:
    DMOTriFlatClass(DMOMeshTri& mesh, QualityCriterium q = QualityCriterium::MEAN_RATIO, float gridScale = 0.5f,
                    int n_iter = 30, bool fixBoundary = true)
        : DMOBaseClass(mesh, q, gridScale, n_iter, 1, fixBoundary) {}
};

// interior hex DMO (dmo/DMOHex.h), boundary fixed
class DMOHexClass : public DMOBaseClass {
public:
    DMOHexClass(DMOMeshHex& mesh, QualityCriterium q = QualityCriterium::MEAN_RATIO, float gridScale = 0.5f,
                int n_iter = 30, bool fixBoundary = true)
        : DMOBaseClass(mesh, q, gridScale, n_iter, -1, fixBoundary) {}
};

// surface triangle DMO (meshes without feature vertices)
class DMOTriClass : public DMOBaseClass {
public:
    DMOTriClass(DMOMeshTri& mesh, QualityCriterium q = QualityCriterium::MEAN_RATIO, float gridScale = 0.5f,
                int n_iter = 30)
        : DMOBaseClass(mesh, q, gridScale, n_iter, 0, true) {}
};

// surface quad DMO (meshes without feature vertices)
class DMOQuadClass : public DMOBaseClass {
public:
    DMOQuadClass(DMOMeshQuad& mesh, QualityCriterium q = QualityCriterium::MEAN_RATIO, float gridScale = 0.5f,
                 int n_iter = 30)
        : DMOBaseClass(mesh, q, gridScale, n_iter, 0, true) {}
};

}  // namespace DMO
