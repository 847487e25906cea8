// vsdmo_internal.cuh -- shared declarations of the CUDA implementation behind include/vsdmo.h.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <stdexcept>
#include <utility>

#include "../../include/vsdmo.h"

namespace vsdmo {

// Internal error: carries a status code to the C ABI boundary (capi.cu), where it is
// turned into a return value; nothing escapes the library as an exception.
struct Error : std::runtime_error {
    vsdmo_status status;
    Error(vsdmo_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define VSDMO_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            throw ::vsdmo::Error(e_ == cudaErrorMemoryAllocation ? VSDMO_E_NOMEM           \
                                                                 : VSDMO_E_CUDA,           \
                                 std::string(#call) + ": " + cudaGetErrorString(e_));      \
        }                                                                                  \
    } while (0)

#define VSDMO_CHECK_LAUNCH() VSDMO_CUDA(cudaGetLastError())

// The library's stream-ordered memory pool on the current device (created on first use). It
// keeps up to 8 GiB of freed memory cached across stream synchronisations, where the default
// pool hands it back to the driver at every synchronisation and the next build maps it again
// (measured: mesh build of the 48^3 tet cube 9-88 ms with the default pool, 5 ms with this one).
cudaMemPool_t device_pool();

// Stream-ordered device buffer (allocated from device_pool() / cudaFreeAsync on the owning
// stream).
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(size_t count, cudaStream_t st) { alloc(count, st); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count, cudaStream_t st) {
        release();
        s = st;
        n = count;
        if (count) VSDMO_CUDA(cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), device_pool(), st));
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    void zero() { if (n) VSDMO_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void fill_bytes(int v) { if (n) VSDMO_CUDA(cudaMemsetAsync(p, v, n * sizeof(T), s)); }
    std::vector<T> to_host() const {
        std::vector<T> h(n);
        if (n) {
            VSDMO_CUDA(cudaMemcpyAsync(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
            VSDMO_CUDA(cudaStreamSynchronize(s));
        }
        return h;
    }
    T* get() const { return p; }
};

template <class T>
inline T read_scalar(const T* dptr, cudaStream_t s) {
    T v;
    VSDMO_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(T), cudaMemcpyDeviceToHost, s));
    VSDMO_CUDA(cudaStreamSynchronize(s));
    return v;
}

inline int grid_for(long n, int block, int cap = 148 * 32) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// ---- primitives (prim.cu) --------------------------------------------------------------
// exclusive prefix sum of n ints (in may alias out); returns nothing, total written to
// *d_total if non-null.
void exclusive_scan(const int* d_in, int* d_out, long n, int* d_total, cudaStream_t s);
// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the keys.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, long n, int bits, cudaStream_t s);
// Stable compaction: out[j] = i for the flagged positions i, in increasing order; returns count.
int compact_flags(const uint8_t* d_flags, long n, int* d_out_index, cudaStream_t s);
// stable partition of [0, n) into d_order: indices with (flag != 0) == first_value first, then
// the rest, each in index order; returns the number of the first group (one host read)
int stable_partition_flags(const uint8_t* d_flags, long n, int first_value, int* d_order, cudaStream_t s);
// CSR (rows 0..K-1) of the distinct (key, value) pairs, each row's values ascending: the same
// arrays as a stable sort by (key, value) followed by dropping repeats. d_rowptr holds K + 1
// ints, d_col at least n.
// stable sort of [0, n) by d_keys (values in [0, K)): d_order receives the original indices in
// (key, index) order, d_keys the keys in that order and d_rowptr (K + 1 ints) the row starts,
// the same arrays as radix_sort_pairs over (keys, 0..n-1) followed by rowptr_from_sorted. For
// keys whose rows are short (a vertex's elements or halfedges): each row is ordered by one warp
// in time quadratic in its length; above SHORT_ROW_MAX entries in a row, by the radix sort.
// Returns the longest row (one host read).
int stable_sort_short_rows(uint32_t* d_keys, uint32_t* d_order, long n, int K, int* d_rowptr, cudaStream_t s);
void csr_unique_from_pairs(const uint32_t* d_keys, const uint32_t* d_vals, long n, int K, int* d_rowptr, int* d_col,
                           cudaStream_t s);
// CSR offsets [K+1] from n keys already sorted ascending (keys < K).
void rowptr_from_sorted(const uint32_t* d_sorted_keys, long n, int K, int* d_rowptr, cudaStream_t s);
// Rows longer than this are not ordered by one warp's quadratic scans: stable_sort_short_rows and
// csr_unique_from_pairs switch to radix sorts, and the tet face pairing rejects the mesh
// (VSDMO_E_VALENCE). The kernels' ring budgets (at most 512 elements around a vertex) stay far below.
constexpr int SHORT_ROW_MAX = 4096;
// longest row of a CSR row pointer d_rowptr[0..K] (one host read)
int longest_row(const int* d_rowptr, long K, cudaStream_t s);
int bits_for(uint32_t maxval);

// ---- mesh (mesh_build.cu) ----------------------------------------------------------------
struct Mesh {
    int type = VSDMO_TRI;   // vsdmo_elem_type
    int k = 3;              // vertices per element
    int fk = 3;             // vertices per surface face: 3 (triangles, tet boundary) or 4 (quads)
    int nV = 0, nE = 0;
    int nSurf = 0, nFeature = 0, nTris = 0, nHE = 0;
    int nColFree = 0, nColFeature = 0, nColInner = 0;
    int maxHE = 0, maxTets = 0, isFlat = 0;
    uint32_t seed = 1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    DBuf<float4> pos;         // [nV] xyz + pad, internal numbering (the optimiser's state)
    DBuf<int> new_of_old;     // [nV]
    DBuf<int> elems;          // [nE*k]
    DBuf<int> tris;           // [nTris*fk] surface faces
    DBuf<int> he_rowptr;      // [nSurf+1]
    DBuf<int4> he;            // [nHE] target, opposite, face, next
    DBuf<int> hf_rowptr;      // [nV+1]
    DBuf<int4> hf;            // [4nT] v0, v1, v2, tet
    DBuf<int4> hh;            // hex: [8nH x 2] the other seven corners of each halfhex (+ -1)
    DBuf<uint8_t> isB1, isFeat, isB2;
    DBuf<float> fn, vn;       // [nTris*3], [nSurf*3]; quad normals from corners 0, 1, 3
    std::vector<int> col_free, col_feature, col_inner;  // host copies of colour offsets
    DBuf<int> d_col_free, d_col_feature, d_col_inner;

    void sync() const { VSDMO_CUDA(cudaStreamSynchronize(stream)); }
};

// Builds connectivity + colouring from device arrays xyz [nV*3] and elems [nE*k].
void build_mesh(Mesh& m, const float* d_xyz, const int* d_elems);

// Normals of the surface (reference k_calcFaceNormals / k_calcVertexNormals).
void update_normals(const Mesh& m, cudaStream_t s);

// ---- DMO kernels (dmo_kernels.cu) ---------------------------------------------------------
struct DmoLaunch {
    int v0, v1;          // vertex range of one colour class
    float grid_scale;
    int depth;
};
// dirty (optional): active-set flags [nV], see k_dmo_tet; skipped (optional): skip counter
void launch_mark_rings(const Mesh& m, int v0, int v1, uint8_t* dirty, cudaStream_t s);
void launch_dmo_tet(const Mesh& m, const DmoLaunch& L, cudaStream_t s, uint8_t* dirty = nullptr,
                    unsigned long long* skipped = nullptr);
void launch_dmo_tri2d(const Mesh& m, const DmoLaunch& L, cudaStream_t s);
int dmo_tet_max_ring();      // largest halfface row the tet kernel accepts
void launch_dmo_hex(const Mesh& m, const DmoLaunch& L, cudaStream_t s);
int dmo_hex_max_ring();      // largest halfhex row the hex kernel accepts
void prepare_dmo_kernels();
int dmo_tri2d_max_ring();    // largest halfedge row the 2D kernel accepts

// ---- learned proposal (tet; dmo_kernels.cu) ----------------------------------------------------
// distinct ring vertices of [v0, v1) (first occurrence in the halfface row, at most 32):
// nb [(v - v0) * 32 + a], nbn [v - v0]
void launch_tet_neighbours(const Mesh& m, int v0, int v1, int* nb, int* nbn, cudaStream_t s);
// network inputs of vertices [v0, v1) from the neighbour table (whose first vertex is nb_base):
// FP32 rows [n x 96] and / or BF16 packed operand rows, ring extent and old position per
// vertex (any output may be null)
void launch_tet_features(const Mesh& m, int v0, int v1, const int* nb, const int* nbn, int nb_base, float* feats,
                         uint8_t* packed, float* scale, float4* old, cudaStream_t s);
// displacement of [v0, v1) since launch_tet_features, in units of the ring extent
void launch_tet_targets(const Mesh& m, int v0, int v1, const float* scale, const float4* old, float* targets,
                        cudaStream_t s);
// reduced grid around the network's proposal (Y [n x ldy], first 3 columns), plain fallback;
// counters [4], dirty: optional active-set flags
// fb_list [colour size] / fb_count [2]: the fallback queue (its length and a block counter,
// both zero between launches: the fallback kernel leaves them so)
void launch_dmo_tet_learned(const Mesh& m, const DmoLaunch& L, const float* Y, int ldy, int rn, int rdepth,
                            float rscale, unsigned long long* counters, uint8_t* dirty, int* fb_list, int* fb_count,
                            cudaStream_t s);

// ---- surface DMO (surf_kernels.cu) ----------------------------------------------------------
// Local quadric surfaces LS [4 nSurf] float4 fitted to pos with the mesh's vertex normals.
// hex interiors under the condition-number quality (hex_cond.cu)
void launch_dmo_hex_cond(const Mesh& m, const DmoLaunch& L, cudaStream_t s);
int dmo_hex_cond_max_ring();
void prepare_hex_cond_kernels();
// ring: 1 = centre + 1-ring (the reference), 2 = centre + 1-ring + 2-ring
void launch_surface_fit(const Mesh& m, const float4* pos, float4* LS, int ring, cudaStream_t s);
// nn [nSurf]: nearest initial vertex of every surface vertex, walked from its previous value.
void launch_update_nn(const Mesh& m, const float4* X0, int* nn, cudaStream_t s);
struct IterStats;
// Sector surfaces of the feature vertices (per-sector quadrics) and the positions the sector of
// a feature neighbour is chosen from (a copy of the positions taken at the start of the colour).
struct SectorSurfaces {
    const int* srow;      // [nFeature + 1]
    const int* stab;      // [nFeature x 20]
    const float4* FS;     // [4 per sector]
    const float4* Xs;     // [nSurf]
};
// One colour class of free surface vertices (triangles when m.fk == 3, quads when 4); sec:
// null for meshes without feature vertices.
void launch_dmo_surf(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS, const int* nn,
                     const SectorSurfaces* sec, int crit, cudaStream_t s);
// Feature vertices: fdeg, the 1D-pass flags and the curves LS1 [3 nSurf] from the current
// positions and vertex normals (flat: +z).
void init_feature_state(const Mesh& m, int flat, float4* LS1, int* fdeg, uint8_t* opt, cudaStream_t s);
// per-sector surfaces; returns the sector count (VSDMO_E_VALENCE beyond the table sizes)
int build_sectors(const Mesh& m, DBuf<int>& srow, DBuf<int>& stab, DBuf<float4>& FS, cudaStream_t s);
// Boundary passes of a tet or hex mesh (run only while the last minimum quality is positive):
// one colour class of free boundary vertices on their surfaces, one of feature vertices on their
// curves, each judged by the vertex's volume ring.
// crit: criterion_of(kind) (tets only; hex rings use the shape metric)
void launch_dmo_surf_vol(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS, const int* nn,
                         const SectorSurfaces* sec, int crit, const IterStats* gate_stats, const int* gate_iter,
                         cudaStream_t s);
// list (optional): the vertices of the class, L.v0 .. L.v1 then index the list instead of the
// vertices (the movable feature vertices of the class; the others would return at once)
void launch_dmo_1d_vol(const Mesh& m, const DmoLaunch& L, const float4* X0, const float4* LS1, const int* nn,
                       const int* fdeg, const uint8_t* opt, int crit, const IterStats* gate_stats, const int* gate_iter,
                       cudaStream_t s, const int* list = nullptr);
int surf_vol_max_ring(int elem_type);
void prepare_surf_kernels();
// One colour class of feature vertices: mode 0 flat (gated on the last minimum quality being
// positive when gate_stats is set), 1 surface triangles, 2 surface quads.
void launch_dmo_1d(const Mesh& m, int mode, const DmoLaunch& L, const float4* X0, const float4* LS1, const int* nn,
                   const int* fdeg, const uint8_t* opt, int crit, const IterStats* gate_stats, const int* gate_iter,
                   cudaStream_t s, const int* list = nullptr);
int dmo_surf_max_ring();     // largest halfedge row the surface kernel accepts
// nu x nv samples of vertex vid's own surface (estimate_mode 0) or of the blended estimate (1)
void launch_surface_samples(const Mesh& m, int estimate_mode, int vid, int nu, int nv, float grid_scale,
                            const float4* X0, const float4* LS, const int* nn, float* out, cudaStream_t s);

// Element metric used by the quality kernels.
enum MetricKind { MK_TRI2D = 0, MK_TRI3D = 1, MK_QUAD = 2, MK_TET = 3, MK_HEX = 4, MK_QUAD2D = 5,
                  MK_TRI2D_MINA = 6, MK_TRI2D_MAXA = 7, MK_TET_MINA = 8, MK_TET_MAXA = 9,
                  MK_TRI3D_MINA = 10, MK_TRI3D_MAXA = 11, MK_HEX_COND = 12, MK_QUAD_COND = 13 };
// ring criterion of the surface, 1D and boundary passes: 0 mean ratio, 1 min angle, 2 max angle,
// 3 condition number
inline int criterion_of(int kind) {
    if (kind == MK_TRI2D_MINA || kind == MK_TET_MINA || kind == MK_TRI3D_MINA) return 1;
    if (kind == MK_TRI2D_MAXA || kind == MK_TET_MAXA || kind == MK_TRI3D_MAXA) return 2;
    if (kind == MK_HEX_COND || kind == MK_QUAD_COND) return 3;
    return 0;
}

// ---- angle criteria (angle.cu) ------------------------------------------------------------
// one colour class with MIN_ANGLE (max_angle = false) or MAX_ANGLE for tet interiors and flat
// triangle meshes
void launch_dmo_angle(const Mesh& m, const DmoLaunch& L, bool max_angle, cudaStream_t s);
int dmo_angle_max_ring(int elem_type);
void prepare_angle_kernels();

// Per-iteration statistics written by the quality kernel.
struct IterStats {
    float min_q;
    int fail_count;
    double sum_q;
};
// Element qualities (reference formulas) -> min / sum into stats[*d_iter], monotonicity check
// against min of the previous slot (or init_min for slot 0), then ++*d_iter.
void launch_quality_stats(const Mesh& m, int kind, IterStats* d_stats, int* d_iter, float* d_partial_min,
                          double* d_partial_sum, int* d_partial_fail, unsigned* d_done, int check_monotone,
                          cudaStream_t s);
void launch_element_qualities(const Mesh& m, int kind, float* d_out, cudaStream_t s);
void launch_quality_histogram(const Mesh& m, int kind, int* d_counts, int n_cols, cudaStream_t s);
int quality_stats_blocks();

// ---- allocation-free quality reduction (noalloc.cu) -----------------------------------------
long noalloc_max_elements();
void quality_reduce_noalloc(int k, const float* d_xyz, int n_vertices, const int* d_elems, long n_elems,
                            float threshold, float* d_min, double* d_sum, int* d_below, cudaStream_t s);

}  // namespace vsdmo
