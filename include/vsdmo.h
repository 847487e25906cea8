/*
 * vsdmo.h -- C ABI of the B200 discrete mesh optimisation (DMO) engine.
 *
 * This is the drop-in boundary for the reference's C++ mesh/optimizer API
 * (DanielZint/VolumeSurfaceDiscreteMeshOptimization). Every entry point below names the
 * reference interface it replaces (path:line inside that project). The C++ classes with the
 * reference's names live in include/vsdmo/DMO.hpp and call only these functions.
 *
 * Conventions
 *   - Every call returns a vsdmo_status and never exits, throws or traps. A failed call
 *     leaves a message for vsdmo_last_error() (thread-local).
 *   - Handles are bound to the CUDA stream given at creation; calls on one handle are not
 *     thread-safe. Distinct handles may be used from different host threads.
 *   - The library owns everything it allocates. Caller pointers are borrowed for the
 *     duration of the call. mem_space says whether a caller pointer is host or device memory.
 *   - Vertex positions are float[3] per vertex (AoS, like the reference's Vec3f), element
 *     indices int32 with 3 (tri), 4 (quad, tet) or 8 (hex) entries per element.
 *   - The build reorders vertices exactly as the reference does (boundary / free / feature
 *     partitions, each sorted by colour); vsdmo_mesh_permutation() returns new_of_old and
 *     vsdmo_mesh_get_positions(..., original_order=1, ...) undoes it.
 */
#ifndef VSDMO_H
#define VSDMO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define VSDMO_API __declspec(dllexport)
#else
#define VSDMO_API __attribute__((visibility("default")))
#endif

typedef enum vsdmo_status {
    VSDMO_OK = 0,
    VSDMO_E_ARG = 1,          /* invalid argument / size / null pointer                */
    VSDMO_E_CUDA = 2,         /* CUDA runtime error                                    */
    VSDMO_E_NONMANIFOLD = 3,  /* element list is not a manifold mesh                  */
    VSDMO_E_VALENCE = 4,      /* a one-ring exceeds the kernels' shared-memory budget  */
    VSDMO_E_MONOTONE = 5,     /* an element's quality fell below the last minimum      */
    VSDMO_E_TIMEOUT = 6,      /* a bounded device-side wait gave up                    */
    VSDMO_E_NAN = 7,          /* non-finite coordinates                                */
    VSDMO_E_NOMEM = 8,        /* device allocation failed                              */
    VSDMO_E_UNSUPPORTED = 9,  /* combination of element type / options not supported   */
    VSDMO_E_IO = 10           /* a mesh file could not be opened, parsed or written     */
} vsdmo_status;

typedef enum vsdmo_elem_type {
    VSDMO_TRI = 0,   /* triangle surface or flat 2D mesh  (DMOMeshTri,  mesh/DMOMeshTri.h:81-94)  */
    VSDMO_QUAD = 1,  /* quad surface                      (DMOMeshQuad, mesh/DMOMeshQuad.h)      */
    VSDMO_TET = 2,   /* tetrahedral volume                (DMOMeshTet,  mesh/DMOMeshTet.h:145-198) */
    VSDMO_HEX = 3    /* hexahedral volume                 (DMOMeshHex,  mesh/DMOMeshHex.h)       */
} vsdmo_elem_type;

/* Same numbering as the reference's DMO::QualityCriterium (dmo/DMOQualityUtil.h:10-18). */
typedef enum vsdmo_quality {
    VSDMO_MEAN_RATIO = 0,
    VSDMO_AREA = 1,
    VSDMO_RIGHT_ANGLE = 2,
    VSDMO_JACOBIAN = 3,
    VSDMO_MIN_ANGLE = 4,
    VSDMO_RADIUS_RATIO = 5,
    VSDMO_MAX_ANGLE = 6,
    VSDMO_CONDITION = 7        /* hex meshes and quad surfaces: inverse condition number of the */
                               /* corner Jacobians (an addition; the reference judges hexes by   */
                               /* shapeMetricHex and quads by meanRatioMetricQuad)               */
} vsdmo_quality;

typedef enum vsdmo_mem_space { VSDMO_HOST = 0, VSDMO_DEVICE = 1 } vsdmo_mem_space;

/* ids for vsdmo_mesh_array / vsdmo_mesh_array_len (internal numbering, for golden tests) */
typedef enum vsdmo_array_id {
    VSDMO_A_XYZ = 0,             /* float [nV*3]      positions, internal order                */
    VSDMO_A_NEW_OF_OLD = 1,      /* int32 [nV]        new index of every input vertex          */
    VSDMO_A_ELEMS = 2,           /* int32 [nE*k]      elements, internal vertex numbering      */
    VSDMO_A_SURF_TRIS = 3,       /* int32 [nTris*fk]  surface faces, fk = 4 for quad meshes else 3 */
    VSDMO_A_HE_ROWPTR = 4,       /* int32 [nSurf+1]   halfedge CSR, CCW fan per vertex         */
    VSDMO_A_HALFEDGES = 5,       /* int32 [nHE*4]     {target, opposite, face, next}           */
    VSDMO_A_HF_ROWPTR = 6,       /* int32 [nV+1]      halfface CSR (tet)                       */
    VSDMO_A_HALFFACES = 7,       /* int32 [4nT*3]     face opposite to the vertex, oriented;   */
                                 /*       hex: [8nH*7] the other corners of each halfhex      */
    VSDMO_A_COL_FREE = 8,        /* int32 [nColorsFree+1]    colour offsets, free surface      */
    VSDMO_A_COL_FEATURE = 9,     /* int32 [nColorsFeature+1] colour offsets, feature vertices  */
    VSDMO_A_COL_INNER = 10,      /* int32 [nColorsInner+1]   colour offsets, volume interior   */
    VSDMO_A_IS_BOUNDARY1D = 11,  /* uint8 [nSurf]                                              */
    VSDMO_A_IS_FEATURE = 12,     /* uint8 [nSurf]                                              */
    VSDMO_A_IS_BOUNDARY2D = 13,  /* uint8 [nV] (tet)                                           */
    VSDMO_A_FACE_NORMALS = 14,   /* float [nTris*3]                                            */
    VSDMO_A_VERTEX_NORMALS = 15  /* float [nSurf*3]                                            */
} vsdmo_array_id;

/* ids for vsdmo_mesh_info */
typedef enum vsdmo_info_id {
    VSDMO_I_NV = 0, VSDMO_I_NE, VSDMO_I_NSURF, VSDMO_I_NFEATURE, VSDMO_I_NTRIS, VSDMO_I_NHE,
    VSDMO_I_NCOL_FREE, VSDMO_I_NCOL_FEATURE, VSDMO_I_NCOL_INNER, VSDMO_I_MAX_HE,
    VSDMO_I_MAX_TETS, VSDMO_I_IS_FLAT, VSDMO_I_ELEM_TYPE, VSDMO_I_COUNT
} vsdmo_info_id;

typedef struct vsdmo_mesh_s* vsdmo_mesh_t;
typedef struct vsdmo_opt_s* vsdmo_opt_t;
typedef struct vsdmo_model_s* vsdmo_model_t;

/* Optimiser parameters. Defaults (vsdmo_params_default) follow the reference constructors:
 * DMOTetClass(mesh, MEAN_RATIO, 0.5f, 30)  dmo/DMOTet.h:24,
 * DMOTriFlatClass(mesh, MIN_ANGLE, 0.5f, 30) dmo/DMOTriFlat.h:25 (the default here is
 * MEAN_RATIO for every element type; MIN_ANGLE / MAX_ANGLE run on tet and triangle meshes),
 * DMO_NQ = 8, DMO_DEPTH = 3 (dmo/DMOConfig.h:4-6). */
typedef struct vsdmo_params {
    int   quality;        /* vsdmo_quality                                                  */
    float grid_scale;     /* initial half-extent factor (0.5)                               */
    int   n_iter;         /* iterations run by vsdmo_opt_optimize (30)                      */
    int   grid_n;         /* candidates per axis: 8; flat tri / quad meshes also take 4     */
    int   depth;          /* refinement levels; 1..4 (3)                                    */
    int   fix_boundary;   /* 1: surface and feature passes are skipped (volume / flat runs  */
                          /*    with the boundary held fixed); 0: reference behaviour       */
    int   flat;           /* tri / quad meshes: -1 = from the mesh (all z == 0), 0 = surface, */
                          /*    1 = 2D                                                      */
    int   use_graph;      /* 1: each iteration is replayed from a captured CUDA graph       */
    int   check_monotone; /* 1: per-element check against the last minimum (reference       */
                          /*    k_updateCurrentQualities, dmo/DMOTet.cu:55-67)              */
    int   active_set;     /* tet: 1 = skip a vertex whose last search found no improvement   */
                          /*    while none of its ring vertices moved since (the result is   */
                          /*    the same with or without skipping); 0 = search every vertex  */
    int   fit_ring;       /* local quadric surfaces: 1 = fitted over the vertex and its       */
                          /*    1-ring (dmo/surfaceP/Surface.cu:11-104, the reference), 2 =    */
                          /*    over its 2-ring as well (an addition; at most 63 points)      */
} vsdmo_params;

/* ---- library --------------------------------------------------------------------------- */
VSDMO_API const char* vsdmo_version(void);
VSDMO_API const char* vsdmo_last_error(void);
VSDMO_API const char* vsdmo_status_string(vsdmo_status s);
VSDMO_API vsdmo_status vsdmo_params_default(int elem_type, vsdmo_params* out);

/* ---- meshes ---------------------------------------------------------------------------- */
/* Replaces DMOMeshTriFactory::create(int nVS, int nT, CudaArray<Vec3f>&, CudaArray<Triangle>&)
 * (mesh/MeshFactory.cu:15-31), DMOMeshTetFactory::create (mesh/MeshFactory.cu:45-55, minus the
 * file parsing) and the MeshTetGPU::init / MeshTriGPU::init builds they run
 * (mesh/MeshTetGPU.cu:35-42, mesh/MeshTriGPU.cu:37-50). Colouring (the reference's live
 * colouring is cusparseScsrcolor, VertexColoring.cu:128-153) runs the rounds of the reference's
 * JPL rule (VertexColoring.cu:76-105) with priorities hashed from color_seed; by default a vertex
 * takes the smallest colour none of its higher-priority neighbours has (the greedy colouring in
 * priority order: 11 classes on the 48^3 tet cube where round colours give 33). Two values
 * select the reference's own rule, colour = round:
 *   VSDMO_COLOR_ROUNDS | s  round colours, priorities hashed from s (the low 31 bits);
 *   VSDMO_COLOR_REFERENCE   round colours with the reference's priorities n - i for local
 *                           index i of the n vertices coloured together (VertexColoring.cu:107-125). */
#define VSDMO_COLOR_ROUNDS 0x80000000u
#define VSDMO_COLOR_REFERENCE 0xFFFFFFFFu
VSDMO_API vsdmo_status vsdmo_mesh_create(int elem_type, const float* xyz, int n_vertices,
                                         const int32_t* elems, int n_elems, int mem_space,
                                         uint32_t color_seed, void* cuda_stream, vsdmo_mesh_t* out);
/* Replaces the DMOMeshTri / DMOMeshTet destructors (mesh/DMOMeshBase.h:132-142). While
 * optimisers created on the mesh are alive the release is deferred to the destruction of the
 * last of them (the reference's DMO classes hold a reference to their mesh). */
VSDMO_API void vsdmo_mesh_destroy(vsdmo_mesh_t mesh);
/* Counts the reference keeps as public members of DMOMeshBase / DMOMeshTet
 * (mesh/DMOMeshBase.h:80-94, mesh/DMOMeshTet.h:145-151): nVertices, nVerticesSurf, ...   */
VSDMO_API int vsdmo_mesh_info(vsdmo_mesh_t mesh, int which);
VSDMO_API long vsdmo_mesh_array_len(vsdmo_mesh_t mesh, int array_id);
/* Copies an internal array to host memory (the reference exposes them as device_ptr members
 * of DMOMeshBase / DMOMeshTet, mesh/DMOMeshBase.h:97-105, mesh/DMOMeshTet.h:153-155). */
VSDMO_API vsdmo_status vsdmo_mesh_array(vsdmo_mesh_t mesh, int array_id, void* host_out);
/* new_of_old[nV]: the vertex permutation applied by the build (sortVerticesByBoundary2D,
 * sortSurfVerticesByFeature, sort*RangeByColor: mesh/MeshTetGPU.cu:241-295,
 * mesh/MeshTriGPU.cu:597-671). */
VSDMO_API vsdmo_status vsdmo_mesh_permutation(vsdmo_mesh_t mesh, int32_t* host_new_of_old);
/* Reads positions (DMOMeshBase::getVertexPoints, mesh/DMOMeshBase.h:146-148); with
 * original_order = 1 they come back in the caller's input numbering. */
VSDMO_API vsdmo_status vsdmo_mesh_get_positions(vsdmo_mesh_t mesh, float* xyz, int original_order,
                                                int mem_space);
/* Overwrites positions (internal or input numbering); used to restart an optimisation.
 * With a device source the copy is queued on the handle's stream and the call returns
 * without waiting; with a host source it returns after the copy. */
VSDMO_API vsdmo_status vsdmo_mesh_set_positions(vsdmo_mesh_t mesh, const float* xyz, int original_order,
                                                int mem_space);

/* ---- mesh files -------------------------------------------------------------------------- */
/* Formats of the reference's parsers and writers (io/ParserOFF.cu, io/ParserTetGen.cu,
 * io/ParserHex.cu, io/FileWriter.cu): OFF (triangles or quads, decided by the first face),
 * TetGen (<base>.node + <base>.ele, 0- or 1-based by the first node's number; attributes and
 * boundary markers are read and not used), Medit .mesh (Vertices + Triangles / Quadrilaterals
 * / Tetrahedra / Hexahedra, 1-based; hexahedra swap their two faces on reading and writing
 * like the reference, so file order 0..7 = the library's 4 5 6 7 0 1 2 3). AUTO picks the
 * format from the extension (.off, .mesh, .node / .ele, or a base name whose .node exists). */
typedef enum vsdmo_file_format {
    VSDMO_FMT_AUTO = 0, VSDMO_FMT_OFF = 1, VSDMO_FMT_TETGEN = 2, VSDMO_FMT_MEDIT = 3
} vsdmo_file_format;
/* Parses a file on the host (no device work). Call once with xyz = elems = NULL for the
 * sizes, then with host buffers of 3 n_vertices floats and k n_elements ints. */
VSDMO_API vsdmo_status vsdmo_file_read(const char* path, int format, int* elem_type, int* n_vertices, int* n_elements,
                                       float* xyz, int32_t* elems);
/* Writes host arrays (floats with 9 significant digits: a written mesh reads back bit for bit;
 * the reference prints 6). TetGen writes 0-based <base>.node and <base>.ele. */
VSDMO_API vsdmo_status vsdmo_file_write(const char* path, int format, int elem_type, const float* xyz, int n_vertices,
                                        const int32_t* elems, int n_elements);
/* DMOMeshTriFactory / DMOMeshQuadFactory / DMOMeshTetFactory / DMOMeshHexFactory::create(
 * filename) (mesh/MeshFactory.cu:3-13,45-55,60-70,101-111): read, then vsdmo_mesh_create.
 * VSDMO_E_IO (message in vsdmo_last_error) where the reference returns nullptr. */
VSDMO_API vsdmo_status vsdmo_mesh_create_from_file(const char* path, int format, uint32_t color_seed, void* cuda_stream,
                                                   vsdmo_mesh_t* out);
/* writeOFF / writeTetgen / writeHex (io/FileWriter.cu:12-147) with the current positions, in
 * the caller's vertex numbering and element order (the reference writes its internal order). */
VSDMO_API vsdmo_status vsdmo_mesh_write_file(vsdmo_mesh_t mesh, const char* path, int format);
/* DMOMeshTriFactory::create(DMOMeshTet&) / DMOMeshQuadFactory::create(DMOMeshHex&)
 * (mesh/MeshFactory.cu:33-41,91-99): a new tri / quad mesh of a volume mesh's boundary faces
 * and surface vertices (the volume's first nSurf vertices in its internal numbering). */
VSDMO_API vsdmo_status vsdmo_mesh_create_surface(vsdmo_mesh_t volume, uint32_t color_seed, void* cuda_stream,
                                                 vsdmo_mesh_t* out);

/* ---- optimiser ------------------------------------------------------------------------- */
/* Replaces DMOTetClass / DMOTriFlatClass / DMOTriClass / DMOQuadClass construction + init()
 * (dmo/DMOTet.cu:82-125, dmo/DMOTriFlat.cu:84-126, dmo/DMOTri.cu:80-126, dmo/DMOQuad.cu:78-123).
 * Tri and quad meshes that are not flat (or flat = 0) get the surface optimiser (feature
 * vertices: sector surfaces for their neighbours; with fix_boundary = 0 they slide along their
 * feature curves, the reference's k_optimizeHierarchical1D). Flat triangle meshes with
 * fix_boundary = 0 slide their boundary vertices (k_optimizeHierarchical1DFlat). Flat quad meshes get the 2D
 * search of DMOTriFlatClass with the quad mean ratio against +z (meanRatioMetricQuad(p, n),
 * dmo/DMOQualityQuad.h:30-50; the reference has no flat-quad class). Hex meshes get the
 * interior search of DMOHexClass (dmo/DMOHex.cu, k_optimizeHierarchicalInnerHex). Tet and hex
 * meshes with fix_boundary = 0 add the boundary passes of DMOTetClass / DMOHexClass::doIteration
 * (dmo/DMOTet.cu:128-170, dmo/DMOHex.cu:131-185): free boundary vertices on their local
 * surfaces and feature vertices on their curves, judged by their volume rings, while the last
 * minimum quality is positive. */
VSDMO_API vsdmo_status vsdmo_opt_create(vsdmo_mesh_t mesh, const vsdmo_params* params, vsdmo_opt_t* out);
VSDMO_API void vsdmo_opt_destroy(vsdmo_opt_t opt);
/* n_iter calls of doIteration() (dmo/DMOTet.cu:128-170, dmo/DMOTriFlat.cu:129-166,
 * dmo/DMOTri.cu:129-165, dmo/DMOQuad.cu:125-162). */
VSDMO_API vsdmo_status vsdmo_opt_iterate(vsdmo_opt_t opt, int n_iter);
/* Restarts the optimiser from the mesh's current positions: iteration count back to 0 and
 * the initial minimum quality re-evaluated (the reference constructs a new DMO object for
 * that, dmo/DMOTet.cu:82-125). Use after vsdmo_mesh_set_positions. */
VSDMO_API vsdmo_status vsdmo_opt_restart(vsdmo_opt_t opt);
/* DMOBaseClass::optimize() (dmo/DMOBase.h:44-52): iterate until isDone(). */
VSDMO_API vsdmo_status vsdmo_opt_optimize(vsdmo_opt_t opt);
/* DMOTetClass::isDone() (dmo/DMOTet.h:26). */
VSDMO_API int vsdmo_opt_is_done(vsdmo_opt_t opt);
VSDMO_API int vsdmo_opt_iterations_done(vsdmo_opt_t opt);
/* DMOBaseClass::getQuality() (dmo/DMOBase.h:41): minimum quality after the last iteration. */
VSDMO_API vsdmo_status vsdmo_opt_get_quality(vsdmo_opt_t opt, float* last_min_quality);
/* DMOTetClass::findMinimumQuality() (dmo/DMOTet.cu:214-221), plus the mean quality. */
VSDMO_API vsdmo_status vsdmo_opt_find_min_quality(vsdmo_opt_t opt, float* min_q, double* mean_q);
/* DMOTetClass::getElementQualities(void*) (dmo/DMOTet.cu:235-240): one float per element in
 * the internal element order. */
VSDMO_API vsdmo_status vsdmo_opt_element_qualities(vsdmo_opt_t opt, float* out, int mem_space);
/* DMOTetClass::getQualityHistogram (dmo/DMOTet.cu:202-212): n_cols bins of [0,1). */
VSDMO_API vsdmo_status vsdmo_opt_quality_histogram(vsdmo_opt_t opt, int32_t* host_counts, int n_cols);
/* DMOTetClass::displayQualityGPU (dmo/DMOTet.cu:188-200): prints the histogram table. */
VSDMO_API vsdmo_status vsdmo_opt_display_quality(vsdmo_opt_t opt, int n_cols);
/* Minimum and mean quality recorded after each completed iteration (the reference prints
 * "it,q_min" lines, dmo/DMOTet.cu:167). Returns the count in *n (at most cap). */
VSDMO_API vsdmo_status vsdmo_opt_history(vsdmo_opt_t opt, float* min_q, double* mean_q, int cap, int* n);
/* One launch of the grid-search kernel over colour class `color` of the inner (tet) or free
 * (tri / quad) partition -- a single step of doIteration's colour loop, for parity tests and
 * per-kernel timing. Asynchronous: it returns once the launch is queued on the stream. */
VSDMO_API vsdmo_status vsdmo_opt_run_color(vsdmo_opt_t opt, int color);
/* Number of kernel launches one iteration issues: the colour launches, the quality kernel
 * and, for surface optimisers, the nearest-neighbour walk and the two normal kernels. */
VSDMO_API int vsdmo_opt_launches_per_iteration(vsdmo_opt_t opt);
/* Surface optimisers (tri / quad surface meshes): copies to host memory, in the internal
 * vertex numbering, the state the reference keeps as DMOTriClass / DMOQuadClass members
 * (dmo/DMOTri.cu:95-112): vertexPointsInit as xyz_init [nSurf*3], localSurfacesInit as
 * local_surfaces [nSurf*16] (p0[3] a, t1[3] b, t2[3] c, n[3] numPoints) and nearestNeighbors
 * as nearest [nSurf]. Any output may be NULL. VSDMO_E_ARG for other optimisers. */
VSDMO_API vsdmo_status vsdmo_opt_surface_state(vsdmo_opt_t opt, float* xyz_init, float* local_surfaces,
                                               int32_t* nearest);

/* Waits for all work queued on the handle's stream. */
VSDMO_API vsdmo_status vsdmo_mesh_sync(vsdmo_mesh_t mesh);

/* ---- allocation-free quality reduction ------------------------------------------------- */
/* No counterpart in the reference: an addition for callers that cannot allocate device
 * memory -- an engine that hands this library a fixed arena and forbids further cudaMalloc,
 * or code running where cudaMalloc / cudaFree are not allowed or would stall the device.
 * Computes, over the n_elems elements of a mesh the caller holds on the device
 * (d_xyz: float[3] per vertex, d_elems: 4 (VSDMO_TET) or 3 (VSDMO_TRI with flat = 1) int32 per
 * element), the minimum element quality (mean ratio, the formula of vsdmo_opt_find_min_quality),
 * the double-precision sum of the qualities and the number of elements whose quality is below
 * `threshold`, written to the caller's device pointers d_min / d_sum / d_below.
 *   - Allocates nothing: the per-block partial results live in a fixed 20,736-byte
 *     __device__ array inside the library that every GPU loading the library holds until the
 *     process exits. At most 8,388,608 elements per call; larger meshes are rejected with
 *     VSDMO_E_ARG. All pointers must be device memory of the current device (VSDMO_E_ARG).
 *   - An element with an index outside [0, n_vertices) is skipped before any of its corners
 *     is read; when there is one, the results are *d_below = -1 and a NaN minimum and sum (the
 *     call is asynchronous, so the check is reported through the results, not the status).
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 *     with that device current; make that first call before any stream capture.
 *   - Asynchronous on cuda_stream (NULL = legacy default stream); results are valid after the
 *     stream is synchronised.
 *   - Every call shares the array: calls that overlap on the GPU (other streams, other host
 *     threads) race and must be serialised by the caller. Each call clears the part that must
 *     start at zero. */
VSDMO_API vsdmo_status vsdmo_quality_reduce_noalloc(int elem_type, int flat, const float* d_xyz, int n_vertices,
                                                    const int32_t* d_elems, int n_elems, float threshold,
                                                    float* d_min, double* d_sum, int32_t* d_below, void* cuda_stream);

/* ---- learned proposal (tet meshes) ----------------------------------------------------- */
/* No counterpart in the reference. A small network (96 -> 128 -> 128 -> 128 -> 3, ReLU, BF16
 * weights and activations, FP32 accumulation, run and trained by the library's own tcgen05
 * tensor-core kernels) maps the one-ring of an inner vertex -- up to 32 distinct ring
 * vertices in first-occurrence order of its halfface row, relative to the vertex and divided
 * by the ring's largest per-axis extent -- to the displacement plain DMO picks for it, in the
 * same units. In learned mode an optimiser searches a reduced grid around that proposal and
 * runs the full plain search whenever the reduced one does not raise the vertex's ring
 * minimum, so every move is one the plain search would accept and the minimum quality stays
 * monotone. Parameters: one flat FP32 array of vsdmo_model_num_params() values
 * (W1 [128x96] b1 W2 [128x128] b2 W3 [128x128] b3 W4 [16x128] b4 [16]; rows 3..15 of W4 and
 * b4 are padding and stay zero). */
VSDMO_API int vsdmo_model_num_params(void);
/* He-uniform weights from seed, zero biases; runs on cuda_stream (NULL: a stream of its own). */
VSDMO_API vsdmo_status vsdmo_model_create(uint64_t seed, void* cuda_stream, vsdmo_model_t* out);
VSDMO_API void vsdmo_model_destroy(vsdmo_model_t model);
VSDMO_API vsdmo_status vsdmo_model_get_params(vsdmo_model_t model, float* host_params);
VSDMO_API vsdmo_status vsdmo_model_set_params(vsdmo_model_t model, const float* host_params);
/* out [n x 3] = network(feats [n x 96]); host or device arrays. */
VSDMO_API vsdmo_status vsdmo_model_forward(vsdmo_model_t model, const float* feats, long n, float* out, int mem_space);
/* Mean squared error of one batch (n a multiple of 128, host arrays) and its gradient with
 * respect to every parameter (grads: host, vsdmo_model_num_params() values). */
VSDMO_API vsdmo_status vsdmo_model_gradients(vsdmo_model_t model, const float* feats, const float* targets, int n,
                                             float* loss, float* grads);
/* Adam (lr, betas 0.9 / 0.999) on `steps` batches of `batch` rows (a multiple of 128) drawn
 * with replacement from the n_rows pairs (feats [n_rows x 96], targets [n_rows x 3], host or
 * device); loss_history (host, may be NULL) receives each step's mean squared error. */
VSDMO_API vsdmo_status vsdmo_model_train(vsdmo_model_t model, const float* feats, const float* targets, long n_rows,
                                         int mem_space, int steps, int batch, float lr, uint64_t seed,
                                         float* loss_history);
/* Runs n_iter plain iterations of a tet optimiser (outside its iteration history: call
 * vsdmo_opt_restart afterwards) and writes one training pair per vertex update into the
 * DEVICE arrays feats [capacity x 96] and targets [capacity x 3]; *n_out = pairs written. */
VSDMO_API vsdmo_status vsdmo_opt_collect_pairs(vsdmo_opt_t opt, int n_iter, float* feats, float* targets,
                                               long capacity, long* n_out);
/* Learned mode for a tet optimiser (model = NULL switches it off): reduced grid of
 * reduced_n^3 candidates per level (2..8), reduced_depth levels (1..4), first half-extent
 * reduced_scale x grid_scale x the ring's per-axis extent (0 < reduced_scale <= 1; each
 * further level shrinks it by 2 / (reduced_n - 1)). The model must stay alive while the
 * optimiser uses it. */
VSDMO_API vsdmo_status vsdmo_opt_set_model(vsdmo_opt_t opt, vsdmo_model_t model, int reduced_n, int reduced_depth,
                                           float reduced_scale);
/* Network proposals [n x 3] (host) of colour class `color` at the current positions, computed
 * by the fused inference kernel the learned search uses (for tests and inspection). */
VSDMO_API vsdmo_status vsdmo_opt_proposals(vsdmo_opt_t opt, int color, float* out);
/* When the learned mode runs the network (no counterpart in the reference, which has no
 * learned mode). Iterations before once_after (counted from the last restart; all of them
 * when once_after = -1, the default) run it before every colour class, from the positions
 * that class sees. Iterations from once_after on run it once for all interior vertices, from
 * the positions at the start of the iteration: one launch instead of one per class, but a
 * class's proposals do not see the moves of the classes before it in the same iteration,
 * which costs fallbacks while vertices still move far. The reduced search and the fallback
 * always evaluate the current ring, so the minimum quality stays monotone either way. */
VSDMO_API vsdmo_status vsdmo_opt_set_proposal_schedule(vsdmo_opt_t opt, int once_after);
/* Counters since vsdmo_opt_set_model / vsdmo_opt_restart: [0] vertex updates accepted from the
 * reduced search, [1] fallbacks to the plain search, [2] fallbacks that moved the vertex,
 * [3] vertices skipped by the active set (plain and learned mode). */
VSDMO_API vsdmo_status vsdmo_opt_learned_counters(vsdmo_opt_t opt, unsigned long long* counters4);
/* TEST-ONLY: the tensor-core GEMM alone, D [M x N] = bf16(A) [M x K] . bf16(B) [N x K]^T in
 * FP32, host arrays; N in {16, 32, 64, 96, 128}, K a multiple of 32. It allocates and
 * synchronises per call; no product path uses it. */
VSDMO_API vsdmo_status vsdmo_debug_gemm_bf16(const float* A, const float* B, int M, int N, int K, float* D);
/* TEST-ONLY: lowers the limit of the bounded device waits that report VSDMO_E_TIMEOUT -- the
 * colour-class waits of the batched iteration, the stage waits of the tensor-core GEMM and the
 * weight / MMA waits of the proposal inference -- on the current device, so that a test can make
 * them expire. ns = 0 makes the GEMM and inference waits expire at once and a batch colour wait
 * as soon as it is entered (a colour class still being searched); ns < 0 restores the default of
 * 1 s; above 1 s is refused (VSDMO_E_ARG). The
 * waits that let copies and MMAs in flight land after an expiry keep 1 s. Synchronises the
 * device; call it with none of the library's work in flight. */
VSDMO_API vsdmo_status vsdmo_debug_set_wait_limit_ns(int64_t ns);

/* Feature-vertex state of an optimiser with feature vertices (surfaces with features, flat
 * meshes with sliding boundaries), internal numbering: curves [nSurf x 12] (p0[3] a, e0[3] 0,
 * e1[3] 0; computeLocalSurface1d, dmo/Surface1D.cu:41-82), fdeg [nSurf] (feature ring
 * vertices), flags [nSurf] (the 1D pass moves the vertex; calcOptFeatureVec,
 * dmo/DMOCommon.h:130-180); surfaces only: sector_rowptr [nFeature + 1], sector_table
 * [nFeature x 20], sector_surfaces [n_sectors x 16] (initLocalSurfacesFeature,
 * dmo/surfaceP/SurfaceFeature.h:79-106). Any output may be NULL. */
VSDMO_API vsdmo_status vsdmo_opt_feature_state(vsdmo_opt_t opt, float* curves, int32_t* fdeg, uint8_t* flags,
                                               int32_t* sector_rowptr, int32_t* sector_table, float* sector_surfaces,
                                               int* n_sectors);
/* The GUI's surface views as sample grids (DMOTriClass / DMOQuadClass::getLocalSurfacePoints
 * and getEstimateLocalSurfacePoints, dmo/DMOTri.cu:169-183, kernels dmo/DMOCommon.cu:73-150,
 * dmo/DMOCommon.h:196-276): nu x nv points (xyz, sample i nu + j) around surface vertex vid
 * (internal numbering) in the frame of its nearest initial vertex's local surface; local: the
 * quadric itself over twice the search extent; estimate: the blended projection over the
 * ring's surfaces that the search evaluates. out: 3 nu nv floats, host or device. Surface
 * optimisers only; feature_sid is for per-sector surfaces of feature vertices, which the
 * surface optimiser does not accept yet (ignored). */
VSDMO_API vsdmo_status vsdmo_opt_local_surface_points(vsdmo_opt_t opt, int vid, int nu, int nv, float* out, int mem_space,
                                                      int feature_sid);
VSDMO_API vsdmo_status vsdmo_opt_estimate_surface_points(vsdmo_opt_t opt, int vid, int nu, int nv, float* out,
                                                         int mem_space);

/* ---- batched flat meshes ------------------------------------------------------------------ */
/* Many independent flat (z = 0) tri and quad meshes optimised together: one persistent launch
 * per iteration takes (mesh, colour class, vertex chunk) work items in colour-major order, each
 * mesh with its own grid (4 or 8 candidates per axis), refinement levels (1..4) and lanes per
 * vertex (8, 16 or 32); iterations are replayed from a captured CUDA graph. The search per
 * vertex is that of DMOTriFlatClass (dmo/DMOTriFlatImplCub.h:24-152, the reference runs one
 * mesh per process). The reference has no batched mode: this replaces a loop over
 * DMOTriFlatClass objects, one per mesh.
 *
 * n_meshes meshes; elem_types [n] (VSDMO_TRI or VSDMO_QUAD), n_vertices [n], n_elements [n]
 * (host arrays); xyz: every mesh's vertices concatenated, float [sum n_vertices x 3];
 * elems: every mesh's element list concatenated, int32 [sum k n_elements] with MESH-LOCAL
 * vertex ids; mem_space applies to xyz and elems. Each mesh is built (connectivity and
 * colouring) as vsdmo_mesh_create would with color_seed. Initial configuration: 8 / 3 / 32. */
typedef struct vsdmo_batch_s* vsdmo_batch_t;
VSDMO_API vsdmo_status vsdmo_batch_create(int n_meshes, const int32_t* elem_types, const int32_t* n_vertices,
                                          const int32_t* n_elements, const float* xyz, const int32_t* elems,
                                          int mem_space, uint32_t color_seed, void* cuda_stream,
                                          vsdmo_batch_t* out);
VSDMO_API void vsdmo_batch_destroy(vsdmo_batch_t batch);
/* Queues n_iter iterations (graph replays) and waits for them; VSDMO_E_TIMEOUT when a
 * colour-class wait of the persistent kernel expired (positions then are not a full
 * iteration's result). */
VSDMO_API vsdmo_status vsdmo_batch_iterate(vsdmo_batch_t batch, int n_iter);
/* Queues n_iter iterations and returns without waiting (vsdmo_batch_sync waits and reports). */
VSDMO_API vsdmo_status vsdmo_batch_iterate_async(vsdmo_batch_t batch, int n_iter);
VSDMO_API vsdmo_status vsdmo_batch_sync(vsdmo_batch_t batch);
/* Iteration count back to 0 and the per-mesh statistics of slot 0 from the current positions. */
VSDMO_API vsdmo_status vsdmo_batch_restart(vsdmo_batch_t batch);
/* Per-mesh statistics after `iteration` iterations since the restart (0 = at the restart):
 * minimum and mean element quality, elements below the previous minimum; any output may be NULL. */
VSDMO_API vsdmo_status vsdmo_batch_stats(vsdmo_batch_t batch, int iteration, float* min_q, double* mean_q,
                                         int32_t* below_prev_min);
/* Positions in the input numbering (concatenated, float [sum n_vertices x 3]). */
VSDMO_API vsdmo_status vsdmo_batch_get_positions(vsdmo_batch_t batch, float* xyz, int mem_space);
VSDMO_API vsdmo_status vsdmo_batch_set_positions(vsdmo_batch_t batch, const float* xyz, int mem_space);
/* Per-mesh search configuration, host arrays [n_meshes]. */
VSDMO_API vsdmo_status vsdmo_batch_get_config(vsdmo_batch_t batch, int32_t* grid_n, int32_t* depth, int32_t* lanes);
VSDMO_API vsdmo_status vsdmo_batch_set_config(vsdmo_batch_t batch, const int32_t* grid_n, const int32_t* depth,
                                              const int32_t* lanes);
/* Autotuner: per size bucket (free vertices < 2,000 / < 10,000 / more) the configuration with
 * the least device time to reach, within 1e-4, the mean and minimum quality that 8 / 3 / 32
 * reaches in probe_iters iterations. Positions are left as they were. The report (one line per
 * bucket) is written to `report` (truncated to report_len bytes, may be NULL). */
VSDMO_API vsdmo_status vsdmo_batch_autotune(vsdmo_batch_t batch, int probe_iters, char* report, int report_len);
/* Counts: 0 meshes, 1 vertices, 2 work items per iteration, 3 colour classes (all meshes),
 * 4 iterations since the restart, 5 CTAs of the persistent launch, 6 largest halfedge row. */
VSDMO_API long vsdmo_batch_info(vsdmo_batch_t batch, int which);
/* Mesh m's layout in the batch: out8 = {first vertex, vertices, elements, vertices per
 * element, colour classes, first free vertex (mesh-local), end of the free vertices,
 * first halfedge}. */
VSDMO_API vsdmo_status vsdmo_batch_mesh_info(vsdmo_batch_t batch, int mesh, int32_t* out8);

#ifdef __cplusplus
}
#endif
#endif /* VSDMO_H */
