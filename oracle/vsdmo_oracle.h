/*
 * vsdmo_oracle.h -- CPU restatement of the reference DMO path (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the checker for the CUDA product in
 * volumesurfacediscretemeshoptimization_b200/. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it. Nothing in the product links
 * or calls it.
 *
 * Parity status: PARTIAL PIN. The reference repository ships no tests, no golden vectors and
 * no sample meshes, and its live colouring is the closed cusparseScsrcolor. The restatement
 * is pinned by (a) known-answer cases the reference's formulas fix exactly (regular
 * simplices / unit cube = quality 1, flipped elements return their signed volume/area,
 * unperturbed structured meshes are fixed points), (b) golden fixtures produced by this
 * restatement and committed under tests/golden/, and (c) the reference's own element quality
 * functions (dmo/DMOQuality.h compiled unmodified into oracle/_ref/ by the Makefile target
 * `ref`, through ref_quality.cu): every element metric restated here matches them on the GPU
 * within FP32 rounding (tests/test_gpu_reference_metrics.py). See the file header of each .c
 * file for the reference lines each function follows.
 *
 * Two arithmetic modes of the DMO grid search are provided:
 *   *_f64 : the reference kernels' algorithm and formulas (mean ratio with cbrt, candidate
 *           grid in absolute coordinates, per-thread carried maxima) evaluated in double;
 *   *_f32 : the product's float arithmetic (local, power-of-two scaled coordinates, affine
 *           per-element determinant and quadratic edge-length sums, ring minimum kept as a
 *           fraction), written independently here so the GPU result can be checked bitwise.
 */
#ifndef VSDMO_ORACLE_H
#define VSDMO_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { OR_TRI = 0, OR_QUAD = 1, OR_TET = 2, OR_HEX = 3 };

/* array ids for or_mesh_array / or_mesh_array_len (same ids as the product's C ABI) */
enum {
    OR_A_XYZ = 0,          /* float [nV*3] permuted positions                       */
    OR_A_NEW_OF_OLD = 1,   /* int   [nV]                                            */
    OR_A_ELEMS = 2,        /* int   [nE*k] remapped elements                        */
    OR_A_SURF_TRIS = 3,    /* int   [nTris*3] surface triangles (tet: boundary)      */
    OR_A_HE_ROWPTR = 4,    /* int   [nSurf+1]                                       */
    OR_A_HALFEDGES = 5,    /* int   [nHE*4] target, opposite, face, next            */
    OR_A_HF_ROWPTR = 6,    /* int   [nV+1]  (tet)                                   */
    OR_A_HALFFACES = 7,    /* int   [4nT*3] (tet)                                   */
    OR_A_COL_FREE = 8,     /* int   [nColorsFree+1]                                 */
    OR_A_COL_FEATURE = 9,  /* int   [nColorsFeature+1]                              */
    OR_A_COL_INNER = 10,   /* int   [nColorsInner+1]                                */
    OR_A_IS_BOUNDARY1D = 11, /* uint8 [nSurf]                                       */
    OR_A_IS_FEATURE = 12,  /* uint8 [nSurf]                                         */
    OR_A_IS_BOUNDARY2D = 13, /* uint8 [nV] (tet)                                    */
    OR_A_FACE_NORMALS = 14,  /* float [nTris*3]                                     */
    OR_A_VERTEX_NORMALS = 15,/* float [nSurf*3]                                     */
    OR_A_COUNT
};

typedef struct or_mesh or_mesh;

/* counts: nV, nE, nSurf, nFeature, nTris, nHE, nColorsFree, nColorsFeature, nColorsInner,
 *         maxNumHalfedges, maxNumTetrahedra, isFlat */
enum { OR_I_NV = 0, OR_I_NE, OR_I_NSURF, OR_I_NFEATURE, OR_I_NTRIS, OR_I_NHE,
       OR_I_NCOL_FREE, OR_I_NCOL_FEATURE, OR_I_NCOL_INNER, OR_I_MAX_HE, OR_I_MAX_TETS,
       OR_I_IS_FLAT, OR_I_COUNT };

/* Build connectivity + colouring for a tri (OR_TRI), quad (OR_QUAD), tet (OR_TET) or hex
 * (OR_HEX) mesh; for hex meshes the halfface arrays hold halfhexes (7 ints each).
 * Returns NULL on invalid input (err set to a message). */
or_mesh* or_mesh_build(int elem_type, int nV, const float* xyz, int nE, const int32_t* elems,
                       uint32_t color_seed, char* err, int err_len);
void     or_mesh_free(or_mesh* m);
int      or_mesh_info(const or_mesh* m, int which);
long     or_mesh_array_len(const or_mesh* m, int id);          /* elements of the array   */
int      or_mesh_array(const or_mesh* m, int id, void* out);    /* copies; 0 on success    */

/* JPL colouring of a CSR graph: the smallest colour free among the coloured neighbours with the
 * seeded priorities (default), the round as colour with OR_COLOR_ROUNDS in the seed, or the
 * round with the reference's priorities n - i when seed == OR_COLOR_REFERENCE; returns the
 * number of colours. */
#define OR_COLOR_REFERENCE 0xFFFFFFFFu
#define OR_COLOR_ROUNDS 0x80000000u
int      or_color_jpl(int n, const int32_t* rowptr, const int32_t* col, uint32_t seed, int32_t* colors);
uint32_t or_priority(uint32_t i, uint32_t seed);

/* ---- DMO grid search (one colour class = vertex range [v0, v1)) ---------------------- */
/* tet inner vertices: reference k_optimizeHierarchicalInnerTet                           */
void or_dmo_tet_f32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nthreads);
void or_dmo_tet_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale,
                    double* margin, int nthreads);
/* the reference kernel's own float arithmetic (cbrtf per element): CPU baseline            */
void or_dmo_tet_ref32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nthreads);
/* flat triangle free vertices: reference k_optimizeHierarchical2DFlat                     */
void or_dmo_tri2d_f32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nthreads);
void or_dmo_tri2d_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale,
                      double* margin, int nthreads);

/* ---- element quality (reference formulas) ------------------------------------------- */
double or_q_tet_mean_ratio_f64(const double* p0, const double* p1, const double* p2, const double* p3);
float  or_q_tet_mean_ratio_f32(const float* p0, const float* p1, const float* p2, const float* p3);
double or_q_tri2d_mean_ratio_f64(const double* p0, const double* p1, const double* p2);
float  or_q_tri2d_mean_ratio_f32(const float* p0, const float* p1, const float* p2);
/* per-element quality of the whole mesh (elements in the mesh's internal numbering)      */
void   or_element_qualities_f64(const or_mesh* m, const double* xyz, double* q);
void   or_element_qualities_f32(const or_mesh* m, const float* xyz, float* q);

/* Full optimisation loop (reference doIteration, fix-boundary mode): n_iter iterations,
 * colours in order; writes min quality after each iteration to min_hist (may be NULL).  */
void or_optimize_f32(const or_mesh* m, float* xyz, int n_iter, float grid_scale, int nthreads,
                     double* min_hist, double* mean_hist);
void or_optimize_f64(const or_mesh* m, double* xyz, int n_iter, double grid_scale, int nthreads,
                     double* min_hist, double* mean_hist);

/* ---- angle criteria (MIN_ANGLE / MAX_ANGLE), literal in double (or_dmo.c) ---------------- */
/* learned mode, one colour class: reduced search around the proposals Y [(v1-v0) x ldy], plain
 * search for the vertices it does not move (queued[i] = 1) */
void or_dmo_tet_learned_f32(const or_mesh* m, float* xyz, int v0, int v1, const float* Y, int ldy, float grid_scale,
                            int rn, int rdepth, float rscale, uint8_t* queued, int nthreads);
double or_q_tri2d_min_angle_f64(const double* p0, const double* p1, const double* p2);
double or_q_tri3d_angle_f64(const double* p0, const double* p1, const double* p2, const double* n, int max_angle);
/* criterion of the f64 surface / 1D / boundary restatements and of or_surface_qualities_f64:
 * OR_MEAN_RATIO (default), OR_MIN_ANGLE or OR_MAX_ANGLE, OR_CONDITION for quads (process-wide
 * test state) */
enum { OR_MEAN_RATIO = 0, OR_MIN_ANGLE = 4, OR_MAX_ANGLE = 6, OR_CONDITION = 7 };
void or_set_criterion(int criterion);
int  or__criterion(void);
double or_q_tri2d_max_angle_f64(const double* p0, const double* p1, const double* p2);
double or_q_tet_min_angle_f64(const double* p0, const double* p1, const double* p2, const double* p3);
double or_q_tet_max_angle_f64(const double* p0, const double* p1, const double* p2, const double* p3);
/* one colour class (tet interior or flat triangles) with the reference search and the angle metric */
void or_dmo_angle_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale, int max_angle, double* margin,
                      int nthreads);
void or_angle_qualities_f64(const or_mesh* m, const double* xyz, int max_angle, double* q);

/* ---- flat tri / quad meshes with a general grid (or_flat.c, the batched optimiser) ------ */
void or_dmo_flat_f32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nq, int depth, int nthreads);
void or_dmo_quad2d_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale, double* margin, int nthreads);
float  or_q_quad2d_f32(const float* p0, const float* p1, const float* p2, const float* p3);
double or_q_quad2d_f64(const double* p0, const double* p1, const double* p2, const double* p3);

/* ---- 1D feature / boundary pass (or_feat.c) ---------------------------------------------- */
/* fdeg [nSurf]: feature ring vertices of every surface vertex; opt [nSurf]: feature vertices the
 * pass moves (two feature neighbours at >= 160 degrees) */
void or_feature_flags(const or_mesh* m, const float* xyz, int32_t* fdeg, uint8_t* opt);
/* curves [nSurf x 12] (p0[3] a, e0[3] 0, e1[3] 0) of the feature vertices (zeros elsewhere) */
void or_surface_fit_1d_f32(const or_mesh* m, const float* xyz, const float* vertex_normals, float* curves);
void or_surface_fit_1d_f64(const or_mesh* m, const double* xyz, const double* vertex_normals, double* curves);
/* one feature colour class [v0, v1) */
void or_dmo_1d_f32(const or_mesh* m, float* xyz, const float* xyz_init, const float* curves, const int32_t* nearest,
                   const float* vertex_normals, const int32_t* fdeg, const uint8_t* opt, int v0, int v1,
                   float grid_scale, int nthreads);
void or_dmo_1d_f64(const or_mesh* m, double* xyz, const double* xyz_init, const double* curves, const int32_t* nearest,
                   const double* vertex_normals, const int32_t* fdeg, const uint8_t* opt, int v0, int v1,
                   double grid_scale, double* margin, int nthreads);

/* ---- hexahedra (or_hex.c) ------------------------------------------------------------- */
/* shapeMetricHex of corners v[0..7] (literal f64 / reference-order f32 with cbrtf) */
double or_q_hex_f64(const double v[8][3]);
float  or_q_hex_f32(const float v[8][3]);
/* one colour class of interior hex vertices: f64 = the reference kernel literally (margin per
 * vertex: smallest gap between competing keys), f32 = the product's arithmetic */
void or_dmo_hex_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale, double* margin, int nthreads);
void or_dmo_hex_f32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nthreads);
void or_hex_qualities_f64(const or_mesh* m, const double* xyz, double* q);
void or_hex_qualities_f32(const or_mesh* m, const float* xyz, float* q);
void or_optimize_hex_f32(const or_mesh* m, float* xyz, int n_iter, float grid_scale, int nthreads,
                         double* min_hist, double* mean_hist);
void or_optimize_hex_f64(const or_mesh* m, double* xyz, int n_iter, double grid_scale, int nthreads,
                         double* min_hist, double* mean_hist);
/* condition-number quality of hexahedra (an addition): corner inverse condition numbers,
 * element minimum; search of one colour class of interior hex vertices under it */
double or_q_hex_cond_f64(const double v[8][3]);
float  or_q_hex_cond_f32(const float v[8][3]);
void or_dmo_hex_cond_f32(const or_mesh* m, float* xyz, int v0, int v1, float grid_scale, int nthreads);
void or_dmo_hex_cond_f64(const or_mesh* m, double* xyz, int v0, int v1, double grid_scale, double* margin,
                         int nthreads);
void or_hex_cond_qualities_f64(const or_mesh* m, const double* xyz, double* q);
void or_hex_cond_qualities_f32(const or_mesh* m, const float* xyz, float* q);
/* per-halfhex coefficients of the product arithmetic (43 floats, see or_hex.c) */
void or_hex_coeffs_f32(const float r[7][3], float eps_s, float eps_a, float* out);

/* ---- surfaces (tri / quad meshes without feature vertices) ----------------------------- */
/* local surfaces: 16 values per surface vertex: p0[3] a, e0[3] b, e1[3] c, e2[3] numPoints  */
void or_surface_normals_f32(const or_mesh* m, const float* xyz, float* face_normals, float* vertex_normals);
void or_surface_normals_f64(const or_mesh* m, const double* xyz, double* face_normals, double* vertex_normals);
int  or_surface_fit_f32(const or_mesh* m, const float* xyz, const float* vertex_normals, float* local_surfaces);
int  or_surface_fit_f64(const or_mesh* m, const double* xyz, const double* vertex_normals, double* local_surfaces);
/* ring 1: the fits above (centre + 1-ring, the reference); ring 2: centre + 1-ring + 2-ring */
int  or_surface_fit_ring_f32(const or_mesh* m, const float* xyz, const float* vertex_normals, float* local_surfaces,
                             int ring);
int  or_surface_fit_ring_f64(const or_mesh* m, const double* xyz, const double* vertex_normals, double* local_surfaces,
                             int ring);
/* per-sector surfaces of feature vertices: rowptr [nFeature+1], table [nFeature*20] (sector of
 * each halfedge of a feature vertex, -1 unused), local_surfaces [cap*16]; returns the sector
 * count, -1 when a feature vertex exceeds 20 halfedges / 40 sector points or cap is too small */
int  or_feature_surfaces_f32(const or_mesh* m, const float* xyz, const float* face_normals, int32_t* rowptr,
                             int32_t* table, float* local_surfaces, int cap);
int  or_feature_surfaces_f64(const or_mesh* m, const double* xyz, const double* face_normals, int32_t* rowptr,
                             int32_t* table, double* local_surfaces, int cap);
void or_update_nn_f32(const or_mesh* m, const float* xyz, const float* xyz_init, int32_t* nearest);
void or_update_nn_f64(const or_mesh* m, const double* xyz, const double* xyz_init, int32_t* nearest);
void or_dmo_surf_f32(const or_mesh* m, float* xyz, const float* xyz_init, const float* local_surfaces,
                     const int32_t* nearest, const float* vertex_normals, int v0, int v1, float grid_scale, int nthreads);
void or_dmo_surf_f64(const or_mesh* m, double* xyz, const double* xyz_init, const double* local_surfaces,
                     const int32_t* nearest, const double* vertex_normals, int v0, int v1, double grid_scale,
                     double* margin, int nthreads);
/* the free-vertex surface search on meshes with feature vertices: the ring's feature neighbours
 * project onto the sector surface (rowptr / table / surfaces of or_feature_surfaces_*) of the
 * halfedge whose target is nearest to the vertex, nearest by the positions at the start of the
 * colour class */
void or_dmo_surf_feat_f32(const or_mesh* m, float* xyz, const float* xyz_init, const float* local_surfaces,
                          const int32_t* nearest, const float* vertex_normals, const int32_t* rowptr,
                          const int32_t* table, const float* sector_surfaces, int v0, int v1, float grid_scale,
                          int nthreads);
void or_dmo_surf_feat_f64(const or_mesh* m, double* xyz, const double* xyz_init, const double* local_surfaces,
                          const int32_t* nearest, const double* vertex_normals, const int32_t* rowptr,
                          const int32_t* table, const double* sector_surfaces, int v0, int v1, double grid_scale,
                          double* margin, int nthreads);
/* boundary-surface pass of a tet or hex mesh: one colour class of free boundary vertices, the
 * surface search judged by the vertex's ring of tets / halfhexes (sector data may be NULL) */
void or_dmo_vol_surf_f32(const or_mesh* m, float* xyz, const float* xyz_init, const float* local_surfaces,
                         const int32_t* nearest, const int32_t* rowptr, const int32_t* table,
                         const float* sector_surfaces, int v0, int v1, float grid_scale, int nthreads);
void or_dmo_vol_surf_f64(const or_mesh* m, double* xyz, const double* xyz_init, const double* local_surfaces,
                         const int32_t* nearest, const int32_t* rowptr, const int32_t* table,
                         const double* sector_surfaces, int v0, int v1, double grid_scale, double* margin,
                         int nthreads);
/* the volume ring of a boundary vertex (or_vring.c; internal to the oracle) */
typedef struct { int hex, k, ex; float es, ea, md; float* co; float c0[3]; } or_vring32;
int    or__vring32_init(or_vring32* R, const or_mesh* m, const float* xyz, int v);  /* 0: degenerate */
float  or__vring32_key(const or_vring32* R, const float* p);
void   or__vring32_free(or_vring32* R);
double or__vring64_q(const or_mesh* m, const double* xyz, int v, const double* p);
double or__vring64_extent(const or_mesh* m, const double* xyz, int v);
double or__gap64(double a, double b);
void or_surface_qualities_f32(const or_mesh* m, const float* xyz, float* q);
void or_surface_qualities_f64(const or_mesh* m, const double* xyz, double* q);
void or_optimize_surf_f32(const or_mesh* m, float* xyz, int n_iter, float grid_scale, int nthreads,
                          double* min_hist, double* mean_hist);
void or_optimize_surf_f64(const or_mesh* m, double* xyz, int n_iter, double grid_scale, int nthreads,
                          double* min_hist, double* mean_hist);
/* nu x nv samples of vertex vid's own surface (estimate_mode 0) or of the blended estimate (1) */
void or_surface_points_f32(const or_mesh* m, const float* xyz, const float* xyz_init, const float* local_surfaces,
                           const int32_t* nearest, int vid, int nu, int nv, float grid_scale, int estimate_mode, float* out);
float  or_q_tri3d_f32(const float* p0, const float* p1, const float* p2);
double or_q_tri3d_f64(const double* p0, const double* p1, const double* p2);
float  or_q_quad_f32(const float* p0, const float* p1, const float* p2, const float* p3, const float* n);
double or_q_quad_f64(const double* p0, const double* p1, const double* p2, const double* p3, const double* n);

#ifdef __cplusplus
}
#endif
#endif
