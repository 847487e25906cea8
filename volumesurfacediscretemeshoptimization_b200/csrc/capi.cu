// capi.cu -- the extern "C" boundary declared in include/vsdmo.h.
//
// Mesh handles own the device mesh (Mesh, mesh_build.cu); optimiser handles own the
// per-iteration statistics and a CUDA graph of one doIteration(): every colour launch of the
// grid search followed by the fused quality / monotonicity kernel (dmo/DMOTet.cu:128-170,
// dmo/DMOTriFlat.cu:129-166 issue the same steps with a cudaDeviceSynchronize after each).
// Surface optimisers (dmo/DMOTri.cu:129-165, dmo/DMOQuad.cu:125-162) also own the initial
// positions, the local surfaces and the nearest-neighbour map, and their iteration adds the
// nearest-neighbour walk and the normal update after the colour launches.
#include "capi_internal.cuh"
#include <cstring>
#include <cmath>
#include <algorithm>
#include <memory>
#include <iostream>
#include <sstream>

namespace {

__global__ void k_pack_xyz(const float4* pos, int n, const int* new_of_old, float* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float4 p = pos[new_of_old ? new_of_old[i] : i];
        out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
    }
}

__global__ void k_unpack_xyz(float4* pos, int n, const int* new_of_old, const float* in) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int d = new_of_old ? new_of_old[i] : (int)i;
        float4 p = pos[d];
        p.x = in[3 * i]; p.y = in[3 * i + 1]; p.z = in[3 * i + 2];
        pos[d] = p;
    }
}

__global__ void k_pack_hf(const int4* hf, long n, int* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int4 h = hf[i];
        out[3 * i] = h.x; out[3 * i + 1] = h.y; out[3 * i + 2] = h.z;
    }
}

__global__ void k_pack_hh(const int4* hh, long n, int* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int4 a = hh[2 * i], b = hh[2 * i + 1];
        int* o = out + 7 * i;
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z;
    }
}

void copy_in(void* dst, const void* src, size_t bytes, int mem_space, cudaStream_t s) {
    VSDMO_CUDA(cudaMemcpyAsync(dst, src, bytes, mem_space == VSDMO_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
}

void launch_color(vsdmo_opt_s* o, int c, cudaStream_t s) {
    const Mesh& m = o->mesh->m;
    DmoLaunch L{o->ranges[c].first, o->ranges[c].second, o->p.grid_scale, o->p.depth};
    if (o->mode == MODE_TET && o->model) {
        // learned proposal: ring features + network (one fused tensor-core kernel) -> reduced
        // grid around the proposal -> plain search for the vertices it did not improve
        const int n = L.v1 - L.v0;
        const float* Y = o->ws.Y.p;
        if (o->proposals_once) Y = o->Yall.p + (size_t)(L.v0 - o->nb_base) * mlp::OUTP;
        else o->model->m.infer_tet(m.pos.p, o->nb.p, o->nbn.p, o->nb_base, L.v0, n, o->ws.Y.p, mlp::OUTP, s);
        launch_dmo_tet_learned(m, L, Y, mlp::OUTP, o->reduced_n, o->reduced_depth, o->reduced_scale,
                               o->counters.p, o->dirty.p, o->fb_list.p, o->fb_count.p, s);
    } else if (o->mode == MODE_TET) {
        launch_dmo_tet(m, L, s, o->dirty.p, o->dirty.p ? o->counters.p + 3 : nullptr);
    } else if (o->mode == MODE_HEX) {
        if (o->kind == MK_HEX_COND) launch_dmo_hex_cond(m, L, s);
        else launch_dmo_hex(m, L, s);
    }
    else if (o->mode == MODE_TRI2D) launch_dmo_tri2d(m, L, s);
    else if (o->mode == MODE_FLAT) launch_dmo_flat(m, L, o->p.grid_n, 32, s);
    else if (o->mode == MODE_ANGLE) launch_dmo_angle(m, L, o->p.quality == VSDMO_MAX_ANGLE, s);
    else {
        SectorSurfaces sec{o->srow.p, o->stab.p, o->FS.p, o->Xs.p};
        if (o->feat) VSDMO_CUDA(cudaMemcpyAsync(o->Xs.p, m.pos.p, sizeof(float4) * m.nSurf, cudaMemcpyDeviceToDevice, s));
        launch_dmo_surf(m, L, o->X0.p, o->LS.p, o->nn.p, o->feat ? &sec : nullptr, criterion_of(o->kind), s);
    }
}

}  // namespace

// ring-vertex table of the inner (tet) range, built once: the topology never changes
void vsdmo_opt_s::ensure_neighbours() {
    if (nb.p) return;
    const Mesh& m = mesh->m;
    const int n = m.nV - m.nSurf;
    nb_base = m.nSurf;
    nb.alloc((size_t)std::max(n, 1) * 32, m.stream);
    nbn.alloc(std::max(n, 1), m.stream);
    launch_tet_neighbours(m, m.nSurf, m.nV, nb.p, nbn.p, m.stream);
}

namespace {

void run_iteration_body(vsdmo_opt_s* o, cudaStream_t s) {
    const Mesh& m = o->mesh->m;
    // proposals of every colour class from the positions at the start of the iteration
    if (o->mode == MODE_TET && o->model && o->proposals_once)
        o->model->m.infer_tet(m.pos.p, o->nb.p, o->nbn.p, o->nb_base, o->nb_base, m.nV - o->nb_base, o->Yall.p,
                              mlp::OUTP, s);
    for (int c = 0; c < (int)o->ranges.size(); ++c) launch_color(o, c, s);
    if (o->volsurf) {
        // boundary passes of a volume mesh, only while the last minimum quality is positive
        // (DMOTetClass::doIteration, dmo/DMOTet.cu:128-170; DMOHexClass::doIteration,
        // dmo/DMOHex.cu:131-185): free boundary classes on their surfaces, feature classes on
        // their curves
        SectorSurfaces sec{o->srow.p, o->stab.p, o->FS.p, o->Xs.p};
        for (const auto& r : o->sranges) {
            DmoLaunch L{r.first, r.second, o->p.grid_scale, o->p.depth};
            if (o->feat) VSDMO_CUDA(cudaMemcpyAsync(o->Xs.p, m.pos.p, sizeof(float4) * m.nSurf, cudaMemcpyDeviceToDevice, s));
            launch_dmo_surf_vol(m, L, o->X0.p, o->LS.p, o->nn.p, o->feat ? &sec : nullptr, criterion_of(o->kind),
                                o->stats.p, o->d_iter.p, s);
        }
        if (o->pass1d)
            for (const auto& r : o->fmranges) {
                DmoLaunch L{r.first, r.second, o->p.grid_scale, o->p.depth};
                launch_dmo_1d_vol(m, L, o->X0.p, o->LS1.p, o->nn.p, o->fdeg.p, o->fopt.p, criterion_of(o->kind),
                                  o->stats.p, o->d_iter.p, s, o->fmove.p);
            }
        launch_mark_rings(m, 0, m.nSurf, o->dirty.p, s);
        launch_update_nn(m, o->X0.p, o->nn.p, s);
        update_normals(m, s);
    } else if (o->pass1d) {
        // feature vertices along their curves (flat meshes: only while the last minimum quality is
        // positive, dmo/DMOTriFlat.cu:140)
        const int mode = o->slide ? 0 : (m.fk == 3 ? 1 : 2);
        for (const auto& r : o->fmranges) {
            DmoLaunch L{r.first, r.second, o->p.grid_scale, o->p.depth};
            launch_dmo_1d(m, mode, L, o->X0.p, o->LS1.p, o->nn.p, o->fdeg.p, o->fopt.p, criterion_of(o->kind),
                          o->slide ? o->stats.p : nullptr, o->slide ? o->d_iter.p : nullptr, s, o->fmove.p);
        }
    }
    if (o->mode == MODE_SURF || o->slide) launch_update_nn(m, o->X0.p, o->nn.p, s);
    if (o->mode == MODE_SURF) update_normals(m, s);
    launch_quality_stats(m, o->kind, o->stats.p, o->d_iter.p, o->pmin.p, o->psum.p, o->pfail.p, o->done.p,
                         o->p.check_monotone ? 1 : 0, s);
}

__global__ void k_surface_state(const float4* pos, int nS, float4* X0, int* nn) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nS; i += gridDim.x * blockDim.x) {
        X0[i] = pos[i];
        nn[i] = i;
    }
}

// The 1D pass only moves the feature vertices whose flag is set (two feature ring vertices at
// 160 degrees or more); the others return at once. Their ids, class by class, let the pass
// launch one warp per movable vertex and skip classes without any. Returns whether the set
// changed (the launch sizes of captured iterations then no longer hold).
bool build_feature_movers(vsdmo_opt_s* o) {
    const Mesh& m = o->mesh->m;
    cudaStream_t s = m.stream;
    const int nFree = m.nSurf - m.nFeature;
    std::vector<uint8_t> flags(std::max(m.nFeature, 1));
    if (m.nFeature > 0)
        VSDMO_CUDA(cudaMemcpyAsync(flags.data(), o->fopt.p + nFree, m.nFeature, cudaMemcpyDeviceToHost, s));
    VSDMO_CUDA(cudaStreamSynchronize(s));
    std::vector<int> ids;
    o->fmranges.clear();
    for (const auto& r : o->franges) {
        const int b = (int)ids.size();
        for (int v = r.first; v < r.second; ++v)
            if (flags[v - nFree]) ids.push_back(v);
        if ((int)ids.size() > b) o->fmranges.push_back({b, (int)ids.size()});
    }
    if (o->fmove.p && ids == o->fmove_ids) return false;
    o->fmove_ids = ids;
    o->fmove.alloc(std::max<size_t>(ids.size(), 1), s);
    if (!ids.empty())
        VSDMO_CUDA(cudaMemcpyAsync(o->fmove.p, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice, s));
    VSDMO_CUDA(cudaStreamSynchronize(s));
    return true;
}

// initial positions, normals, local surfaces and nn = identity from the current positions
// (the constructor of DMOTriClass / DMOQuadClass, dmo/DMOTri.cu:80-126)
// With feature vertices also their curves and 1D flags (computeLocalSurfaces1d,
// calcOptFeatureVec) and, on surfaces, the per-sector surfaces (initLocalSurfacesFeature).
void init_surface_state(vsdmo_opt_s* o) {
    const Mesh& m = o->mesh->m;
    cudaStream_t s = m.stream;
    const bool surfaces = o->mode == MODE_SURF || o->volsurf;
    if (!o->X0.p) {
        o->X0.alloc(m.nSurf, s);
        o->nn.alloc(m.nSurf, s);
        if (surfaces) o->LS.alloc(4L * m.nSurf, s);
    }
    k_surface_state<<<grid_for(m.nSurf, 256), 256, 0, s>>>(m.pos.p, m.nSurf, o->X0.p, o->nn.p);
    VSDMO_CHECK_LAUNCH();
    if (surfaces) {
        update_normals(m, s);
        launch_surface_fit(m, o->X0.p, o->LS.p, o->p.fit_ring, s);
    }
    if (o->feat) {
        if (!o->LS1.p) {
            o->LS1.alloc(3L * m.nSurf, s);
            o->fdeg.alloc(m.nSurf, s);
            o->fopt.alloc(m.nSurf, s);
        }
        init_feature_state(m, o->slide ? 1 : 0, o->LS1.p, o->fdeg.p, o->fopt.p, s);
        bool changed = build_feature_movers(o);
        if (surfaces) {
            const void* before[3] = { o->srow.p, o->stab.p, o->FS.p };
            const int ns = o->nsect;
            o->nsect = build_sectors(m, o->srow, o->stab, o->FS, s);
            changed |= o->srow.p != before[0] || o->stab.p != before[1] || o->FS.p != before[2] || o->nsect != ns;
            if (!o->Xs.p) o->Xs.alloc(m.nSurf, s);
        }
        // captured iterations hold the movers' launch sizes and the sector buffers' addresses;
        // a restart from the same positions usually rebuilds both unchanged and keeps them
        if (changed) o->drop_graphs();
    }
}

void ensure_capacity(vsdmo_opt_s* o, int need) {
    if (need + 1 <= o->capacity) return;
    cudaStream_t s = o->mesh->m.stream;
    int cap = std::max(need + 1, std::max(2 * o->capacity, 256));
    DBuf<IterStats> ns(cap, s);
    ns.zero();
    if (o->stats.p)
        VSDMO_CUDA(cudaMemcpyAsync(ns.p, o->stats.p, sizeof(IterStats) * o->capacity, cudaMemcpyDeviceToDevice, s));
    o->stats = std::move(ns);
    o->capacity = cap;
    o->drop_graphs();
}

void ensure_graph(vsdmo_opt_s* o) {
    const int slot = o->proposals_once;
    if (o->exec[slot] || !o->p.use_graph) return;
    cudaStream_t s = o->mesh->m.stream;
    VSDMO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        run_iteration_body(o, s);
    } catch (...) {
        cudaGraph_t g;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    VSDMO_CUDA(cudaStreamEndCapture(s, &o->graph[slot]));
    VSDMO_CUDA(cudaGraphInstantiate(&o->exec[slot], o->graph[slot], 0));
}

std::vector<IterStats> read_stats(vsdmo_opt_s* o, int from, int count) {
    std::vector<IterStats> h(count);
    if (count > 0) {
        VSDMO_CUDA(cudaMemcpyAsync(h.data(), o->stats.p + from, sizeof(IterStats) * count, cudaMemcpyDeviceToHost, o->mesh->m.stream));
        VSDMO_CUDA(cudaStreamSynchronize(o->mesh->m.stream));
    }
    return h;
}

}  // namespace

extern "C" {

VSDMO_API const char* vsdmo_version(void) { return "vsdmo-b200 0.1.0 (sm_100a)"; }

VSDMO_API const char* vsdmo_last_error(void) { return g_last_error.c_str(); }

VSDMO_API const char* vsdmo_status_string(vsdmo_status s) {
    switch (s) {
    case VSDMO_OK: return "ok";
    case VSDMO_E_ARG: return "invalid argument";
    case VSDMO_E_CUDA: return "CUDA error";
    case VSDMO_E_NONMANIFOLD: return "non-manifold mesh";
    case VSDMO_E_VALENCE: return "one-ring too large";
    case VSDMO_E_MONOTONE: return "quality decreased";
    case VSDMO_E_TIMEOUT: return "device wait timed out";
    case VSDMO_E_NAN: return "non-finite coordinates";
    case VSDMO_E_NOMEM: return "out of memory";
    case VSDMO_E_UNSUPPORTED: return "unsupported";
    case VSDMO_E_IO: return "mesh file error";
    }
    return "unknown status";
}

VSDMO_API vsdmo_status vsdmo_params_default(int elem_type, vsdmo_params* out) {
    if (!out) return fail(VSDMO_E_ARG, "null params");
    if (elem_type < VSDMO_TRI || elem_type > VSDMO_HEX) return fail(VSDMO_E_ARG, "bad element type");
    out->quality = VSDMO_MEAN_RATIO;
    out->grid_scale = 0.5f;
    out->n_iter = 30;
    out->grid_n = 8;
    out->depth = 3;
    out->fix_boundary = 1;
    out->flat = -1;
    out->use_graph = 1;
    out->check_monotone = 1;
    out->active_set = 0;
    out->fit_ring = 1;
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_mesh_create(int elem_type, const float* xyz, int n_vertices, const int32_t* elems,
                                         int n_elems, int mem_space, uint32_t color_seed, void* cuda_stream,
                                         vsdmo_mesh_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    if (elem_type != VSDMO_TRI && elem_type != VSDMO_TET && elem_type != VSDMO_QUAD && elem_type != VSDMO_HEX)
        return fail(VSDMO_E_ARG, "bad element type");
    if (!xyz || !elems || n_vertices <= 0 || n_elems <= 0) return fail(VSDMO_E_ARG, "empty mesh or null arrays");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    const int k = elem_type == VSDMO_TRI ? 3 : elem_type == VSDMO_HEX ? 8 : 4;
    if ((long)n_elems * k > (long)INT32_MAX / 2 || (long)n_vertices * 4 > (long)INT32_MAX)
        return fail(VSDMO_E_ARG, "mesh too large for 32-bit indices");
    std::unique_ptr<vsdmo_mesh_s> h(new vsdmo_mesh_s);
    vsdmo_status st = guarded([&] {
        Mesh& m = h->m;
        m.type = elem_type;
        m.k = k;
        m.nV = n_vertices;
        m.nE = n_elems;
        m.seed = color_seed;
        if (cuda_stream) {
            m.stream = (cudaStream_t)cuda_stream;
        } else {
            VSDMO_CUDA(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
            m.own_stream = true;
        }
        DBuf<float> dx(3L * n_vertices, m.stream);
        DBuf<int> de((long)n_elems * k, m.stream);
        copy_in(dx.p, xyz, sizeof(float) * 3L * n_vertices, mem_space, m.stream);
        copy_in(de.p, elems, sizeof(int) * (long)n_elems * k, mem_space, m.stream);
        build_mesh(m, dx.p, de.p);
        m.sync();
    });
    if (st != VSDMO_OK) {
        if (h->m.own_stream && h->m.stream) {
            cudaStream_t s = h->m.stream;
            h.reset();
            cudaStreamDestroy(s);
        }
        return st;
    }
    *out = h.release();
    return VSDMO_OK;
}

namespace {
void release_mesh(vsdmo_mesh_t mesh) {
    cudaStream_t s = mesh->m.stream;
    bool own = mesh->m.own_stream;
    cudaStreamSynchronize(s);
    delete mesh;
    if (own) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
}
}  // namespace

VSDMO_API void vsdmo_mesh_destroy(vsdmo_mesh_t mesh) {
    if (!mesh) return;
    // optimisers still hold the mesh: it is released with the last of them
    if (mesh->n_opts > 0) {
        mesh->destroy_requested = true;
        return;
    }
    release_mesh(mesh);
}

VSDMO_API vsdmo_status vsdmo_mesh_sync(vsdmo_mesh_t mesh) {
    if (!mesh) return fail(VSDMO_E_ARG, "null mesh");
    return guarded([&] { mesh->m.sync(); });
}

VSDMO_API int vsdmo_mesh_info(vsdmo_mesh_t mesh, int which) {
    if (!mesh) return -1;
    const Mesh& m = mesh->m;
    switch (which) {
    case VSDMO_I_NV: return m.nV;
    case VSDMO_I_NE: return m.nE;
    case VSDMO_I_NSURF: return m.nSurf;
    case VSDMO_I_NFEATURE: return m.nFeature;
    case VSDMO_I_NTRIS: return m.nTris;
    case VSDMO_I_NHE: return m.nHE;
    case VSDMO_I_NCOL_FREE: return m.nColFree;
    case VSDMO_I_NCOL_FEATURE: return m.nColFeature;
    case VSDMO_I_NCOL_INNER: return m.nColInner;
    case VSDMO_I_MAX_HE: return m.maxHE;
    case VSDMO_I_MAX_TETS: return m.maxTets;
    case VSDMO_I_IS_FLAT: return m.isFlat;
    case VSDMO_I_ELEM_TYPE: return m.type;
    default: return -1;
    }
}

VSDMO_API long vsdmo_mesh_array_len(vsdmo_mesh_t mesh, int id) {
    if (!mesh) return -1;
    const Mesh& m = mesh->m;
    switch (id) {
    case VSDMO_A_XYZ: return 3L * m.nV;
    case VSDMO_A_NEW_OF_OLD: return m.nV;
    case VSDMO_A_ELEMS: return (long)m.nE * m.k;
    case VSDMO_A_SURF_TRIS: return (long)m.fk * m.nTris;
    case VSDMO_A_HE_ROWPTR: return m.he_rowptr.p ? m.nSurf + 1L : 0;
    case VSDMO_A_HALFEDGES: return 4L * m.nHE;
    case VSDMO_A_HF_ROWPTR: return m.hf_rowptr.p ? m.nV + 1L : 0;
    case VSDMO_A_HALFFACES: return m.hf.p ? 12L * m.nE : (m.hh.p ? 56L * m.nE : 0);
    case VSDMO_A_COL_FREE: return (long)m.col_free.size();
    case VSDMO_A_COL_FEATURE: return (long)m.col_feature.size();
    case VSDMO_A_COL_INNER: return (long)m.col_inner.size();
    case VSDMO_A_IS_BOUNDARY1D: return m.isB1.p ? m.nSurf : 0;
    case VSDMO_A_IS_FEATURE: return m.isFeat.p ? m.nSurf : 0;
    case VSDMO_A_IS_BOUNDARY2D: return m.isB2.p ? m.nV : 0;
    case VSDMO_A_FACE_NORMALS: return m.fn.p ? 3L * m.nTris : 0;
    case VSDMO_A_VERTEX_NORMALS: return m.vn.p ? 3L * m.nSurf : 0;
    default: return -1;
    }
}

VSDMO_API vsdmo_status vsdmo_mesh_array(vsdmo_mesh_t mesh, int id, void* host_out) {
    if (!mesh || !host_out) return fail(VSDMO_E_ARG, "null argument");
    long n = vsdmo_mesh_array_len(mesh, id);
    if (n < 0) return fail(VSDMO_E_ARG, "bad array id");
    if (n == 0) return VSDMO_OK;
    return guarded([&] {
        Mesh& m = mesh->m;
        cudaStream_t s = m.stream;
        auto d2h = [&](const void* src, size_t bytes) {
            VSDMO_CUDA(cudaMemcpyAsync(host_out, src, bytes, cudaMemcpyDeviceToHost, s));
            VSDMO_CUDA(cudaStreamSynchronize(s));
        };
        switch (id) {
        case VSDMO_A_XYZ: {
            DBuf<float> t(3L * m.nV, s);
            k_pack_xyz<<<grid_for(m.nV, 256), 256, 0, s>>>(m.pos.p, m.nV, nullptr, t.p);
            VSDMO_CHECK_LAUNCH();
            d2h(t.p, sizeof(float) * 3L * m.nV);
            break;
        }
        case VSDMO_A_NEW_OF_OLD: d2h(m.new_of_old.p, sizeof(int) * n); break;
        case VSDMO_A_ELEMS: d2h(m.elems.p, sizeof(int) * n); break;
        case VSDMO_A_SURF_TRIS: d2h(m.tris.p, sizeof(int) * n); break;
        case VSDMO_A_HE_ROWPTR: d2h(m.he_rowptr.p, sizeof(int) * n); break;
        case VSDMO_A_HALFEDGES: d2h(m.he.p, sizeof(int) * n); break;
        case VSDMO_A_HF_ROWPTR: d2h(m.hf_rowptr.p, sizeof(int) * n); break;
        case VSDMO_A_HALFFACES: {
            DBuf<int> t(n, s);
            if (m.hf.p) k_pack_hf<<<grid_for(n / 3, 256), 256, 0, s>>>(m.hf.p, n / 3, t.p);
            else k_pack_hh<<<grid_for(n / 7, 256), 256, 0, s>>>(m.hh.p, n / 7, t.p);
            VSDMO_CHECK_LAUNCH();
            d2h(t.p, sizeof(int) * n);
            break;
        }
        case VSDMO_A_COL_FREE: std::memcpy(host_out, m.col_free.data(), sizeof(int) * n); break;
        case VSDMO_A_COL_FEATURE: std::memcpy(host_out, m.col_feature.data(), sizeof(int) * n); break;
        case VSDMO_A_COL_INNER: std::memcpy(host_out, m.col_inner.data(), sizeof(int) * n); break;
        case VSDMO_A_IS_BOUNDARY1D: d2h(m.isB1.p, n); break;
        case VSDMO_A_IS_FEATURE: d2h(m.isFeat.p, n); break;
        case VSDMO_A_IS_BOUNDARY2D: d2h(m.isB2.p, n); break;
        case VSDMO_A_FACE_NORMALS: d2h(m.fn.p, sizeof(float) * n); break;
        case VSDMO_A_VERTEX_NORMALS: d2h(m.vn.p, sizeof(float) * n); break;
        }
    });
}

VSDMO_API vsdmo_status vsdmo_mesh_permutation(vsdmo_mesh_t mesh, int32_t* host_new_of_old) {
    return vsdmo_mesh_array(mesh, VSDMO_A_NEW_OF_OLD, host_new_of_old);
}

VSDMO_API vsdmo_status vsdmo_mesh_get_positions(vsdmo_mesh_t mesh, float* xyz, int original_order, int mem_space) {
    if (!mesh || !xyz) return fail(VSDMO_E_ARG, "null argument");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        Mesh& m = mesh->m;
        cudaStream_t s = m.stream;
        const int* map = original_order ? m.new_of_old.p : nullptr;
        if (mem_space == VSDMO_DEVICE) {
            k_pack_xyz<<<grid_for(m.nV, 256), 256, 0, s>>>(m.pos.p, m.nV, map, xyz);
            VSDMO_CHECK_LAUNCH();
            m.sync();
        } else {
            DBuf<float> t(3L * m.nV, s);
            k_pack_xyz<<<grid_for(m.nV, 256), 256, 0, s>>>(m.pos.p, m.nV, map, t.p);
            VSDMO_CHECK_LAUNCH();
            VSDMO_CUDA(cudaMemcpyAsync(xyz, t.p, sizeof(float) * 3L * m.nV, cudaMemcpyDeviceToHost, s));
            m.sync();
        }
    });
}

VSDMO_API vsdmo_status vsdmo_mesh_set_positions(vsdmo_mesh_t mesh, const float* xyz, int original_order, int mem_space) {
    if (!mesh || !xyz) return fail(VSDMO_E_ARG, "null argument");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        Mesh& m = mesh->m;
        cudaStream_t s = m.stream;
        const int* map = original_order ? m.new_of_old.p : nullptr;
        DBuf<float> t;
        const float* src = xyz;
        if (mem_space == VSDMO_HOST) {
            t.alloc(3L * m.nV, s);
            VSDMO_CUDA(cudaMemcpyAsync(t.p, xyz, sizeof(float) * 3L * m.nV, cudaMemcpyHostToDevice, s));
            src = t.p;
        }
        k_unpack_xyz<<<grid_for(m.nV, 256), 256, 0, s>>>(m.pos.p, m.nV, map, src);
        VSDMO_CHECK_LAUNCH();
        if (mem_space == VSDMO_HOST) m.sync();  // the caller's host buffer may be reused on return
    });
}

namespace {
vsdmo_status surface_points(vsdmo_opt_t o, int estimate_mode, int vid, int nu, int nv, float* out, int mem_space) {
    if (!o || !out) return fail(VSDMO_E_ARG, "null argument");
    if (o->mode != MODE_SURF && !o->volsurf) return fail(VSDMO_E_ARG, "not a surface optimiser");
    const Mesh& m = o->mesh->m;
    if (vid < 0 || vid >= m.nSurf) return fail(VSDMO_E_ARG, "vid must be a surface vertex (internal numbering)");
    if (nu < 2 || nv < 2 || (long)nu * nv > (1L << 24)) return fail(VSDMO_E_ARG, "nu, nv must be >= 2 (at most 2^24 samples)");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        cudaStream_t s = m.stream;
        const size_t n = 3 * (size_t)nu * nv;
        if (mem_space == VSDMO_DEVICE) {
            launch_surface_samples(m, estimate_mode, vid, nu, nv, o->p.grid_scale, o->X0.p, o->LS.p, o->nn.p, out, s);
            m.sync();
            return;
        }
        DBuf<float> d(n, s);
        launch_surface_samples(m, estimate_mode, vid, nu, nv, o->p.grid_scale, o->X0.p, o->LS.p, o->nn.p, d.p, s);
        VSDMO_CUDA(cudaMemcpyAsync(out, d.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
        m.sync();
    });
}
}  // namespace

VSDMO_API vsdmo_status vsdmo_opt_local_surface_points(vsdmo_opt_t opt, int vid, int nu, int nv, float* out, int mem_space,
                                                      int feature_sid) {
    (void)feature_sid;   // meshes with feature vertices are not accepted by the surface optimiser yet
    return surface_points(opt, 0, vid, nu, nv, out, mem_space);
}

VSDMO_API vsdmo_status vsdmo_opt_estimate_surface_points(vsdmo_opt_t opt, int vid, int nu, int nv, float* out,
                                                         int mem_space) {
    return surface_points(opt, 1, vid, nu, nv, out, mem_space);
}

VSDMO_API vsdmo_status vsdmo_opt_create(vsdmo_mesh_t mesh, const vsdmo_params* params, vsdmo_opt_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    if (!mesh) return fail(VSDMO_E_ARG, "null mesh");
    vsdmo_params p;
    if (params) p = *params; else vsdmo_params_default(mesh->m.type, &p);
    const Mesh& m = mesh->m;
    const bool angle = p.quality == VSDMO_MIN_ANGLE || p.quality == VSDMO_MAX_ANGLE;
    const bool cond = p.quality == VSDMO_CONDITION;
    const bool flat2d = (m.type == VSDMO_TRI || m.type == VSDMO_QUAD) && (p.flat < 0 ? m.isFlat : p.flat);
    if (p.quality != VSDMO_MEAN_RATIO && !angle && !(cond && (m.type == VSDMO_HEX || (m.type == VSDMO_QUAD && !flat2d))))
        return fail(VSDMO_E_UNSUPPORTED, "MEAN_RATIO, MIN_ANGLE and MAX_ANGLE are implemented, and CONDITION for hex "
                                         "meshes and quad surfaces");
    if (p.grid_n != 8 && !(flat2d && p.grid_n == 4))
        return fail(VSDMO_E_UNSUPPORTED, "only an 8-point grid per axis is implemented (4 or 8 for flat meshes)");
    if (flat2d && p.grid_n == 4 && p.depth > 4) return fail(VSDMO_E_ARG, "depth must be in 1..4 with a 4-point grid");
    if (p.depth < 1 || p.depth > 8) return fail(VSDMO_E_ARG, "depth must be in 1..8");
    if (!(p.grid_scale > 0.f) || !std::isfinite(p.grid_scale)) return fail(VSDMO_E_ARG, "grid_scale must be positive");
    if (p.n_iter < 0) return fail(VSDMO_E_ARG, "n_iter must be >= 0");
    if (p.fit_ring != 1 && p.fit_ring != 2) return fail(VSDMO_E_ARG, "fit_ring must be 1 or 2");
    std::unique_ptr<vsdmo_opt_s> o(new vsdmo_opt_s);
    o->mesh = mesh;
    o->p = p;
    if (angle) {
        // angle criteria (dmo/DMOQualityTri.h:10-237, dmo/DMOQualityTet.h:10-115): tet meshes
        // (interior search; boundary passes with fix_boundary = 0), flat triangle meshes (interior
        // search; sliding boundary with fix_boundary = 0) and triangle surfaces; 8-point grid
        const bool tet = m.type == VSDMO_TET, tri = m.type == VSDMO_TRI;
        if (!(tet || tri) || p.grid_n != 8)
            return fail(VSDMO_E_UNSUPPORTED, "angle criteria are implemented for tet and triangle meshes with an "
                                             "8-point grid");
        const bool mx = p.quality == VSDMO_MAX_ANGLE;
        if (tri && !flat2d) {
            if (m.maxHE > dmo_surf_max_ring()) return fail(VSDMO_E_VALENCE, "a vertex has more halfedges than the kernel's ring budget");
            o->mode = MODE_SURF;
            o->kind = mx ? MK_TRI3D_MAXA : MK_TRI3D_MINA;
            for (int c = 0; c < m.nColFree; ++c) o->ranges.push_back({m.col_free[c], m.col_free[c + 1]});
            if (m.nFeature > 0) {
                o->feat = true;
                o->pass1d = !p.fix_boundary;
                for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
            }
        } else {
            if ((tet ? m.maxTets : m.maxHE) > dmo_angle_max_ring(m.type))
                return fail(VSDMO_E_VALENCE, "a vertex's ring exceeds the angle kernel's budget");
            o->mode = MODE_ANGLE;
            o->kind = tet ? (mx ? MK_TET_MAXA : MK_TET_MINA) : (mx ? MK_TRI2D_MAXA : MK_TRI2D_MINA);
            if (tet) for (int c = 0; c < m.nColInner; ++c) o->ranges.push_back({m.col_inner[c], m.col_inner[c + 1]});
            else for (int c = 0; c < m.nColFree; ++c) o->ranges.push_back({m.col_free[c], m.col_free[c + 1]});
            if (!p.fix_boundary && tet) {
                if (m.maxTets > surf_vol_max_ring(VSDMO_TET) || m.maxHE > dmo_surf_max_ring())
                    return fail(VSDMO_E_VALENCE, "a boundary vertex's ring exceeds the boundary kernels' budget");
                o->volsurf = true;
                for (int c = 0; c < m.nColFree; ++c) o->sranges.push_back({m.col_free[c], m.col_free[c + 1]});
                if (m.nFeature > 0) {
                    o->feat = o->pass1d = true;
                    for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
                }
            } else if (!p.fix_boundary && m.nFeature > 0) {
                if (m.maxHE > dmo_surf_max_ring()) return fail(VSDMO_E_VALENCE, "a vertex has more halfedges than the kernel's ring budget");
                o->slide = o->feat = o->pass1d = true;
                for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
            }
        }
    } else if (m.type == VSDMO_TET) {
        if (m.maxTets > dmo_tet_max_ring()) return fail(VSDMO_E_VALENCE, "a vertex has more tetrahedra than the kernel's ring budget");
        o->mode = MODE_TET;
        o->kind = MK_TET;
        for (int c = 0; c < m.nColInner; ++c) o->ranges.push_back({m.col_inner[c], m.col_inner[c + 1]});
        if (!p.fix_boundary) {
            // the boundary vertices move on the boundary surface (and feature vertices on their
            // feature curves) after the interior classes, like DMOTetClass
            if (m.maxTets > surf_vol_max_ring(VSDMO_TET) || m.maxHE > dmo_surf_max_ring())
                return fail(VSDMO_E_VALENCE, "a boundary vertex's ring exceeds the boundary kernels' budget");
            o->volsurf = true;
            for (int c = 0; c < m.nColFree; ++c) o->sranges.push_back({m.col_free[c], m.col_free[c + 1]});
            if (m.nFeature > 0) {
                o->feat = o->pass1d = true;
                for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
            }
        }
    } else if (m.type == VSDMO_HEX) {
        if (m.maxTets > (cond ? dmo_hex_cond_max_ring() : dmo_hex_max_ring()))
            return fail(VSDMO_E_VALENCE, "a vertex has more hexahedra than the kernel's ring budget");
        if (cond && !p.fix_boundary)
            return fail(VSDMO_E_UNSUPPORTED, "the boundary passes of hex meshes use the shape metric; set fix_boundary=1 "
                                             "with CONDITION");
        o->mode = MODE_HEX;
        o->kind = cond ? MK_HEX_COND : MK_HEX;
        for (int c = 0; c < m.nColInner; ++c) o->ranges.push_back({m.col_inner[c], m.col_inner[c + 1]});
        if (!p.fix_boundary) {
            // boundary and feature passes after the interior classes, like DMOHexClass
            if (m.maxTets > surf_vol_max_ring(VSDMO_HEX) || m.maxHE > dmo_surf_max_ring())
                return fail(VSDMO_E_VALENCE, "a boundary vertex's ring exceeds the boundary kernels' budget");
            o->volsurf = true;
            for (int c = 0; c < m.nColFree; ++c) o->sranges.push_back({m.col_free[c], m.col_free[c + 1]});
            if (m.nFeature > 0) {
                o->feat = o->pass1d = true;
                for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
            }
        }
    } else if (m.type == VSDMO_TRI && flat2d && p.grid_n == 8) {
        if (m.maxHE > dmo_tri2d_max_ring() || (!p.fix_boundary && m.maxHE > dmo_surf_max_ring()))
            return fail(VSDMO_E_VALENCE, "a vertex has more halfedges than the kernel's ring budget");
        o->mode = MODE_TRI2D;
        o->kind = MK_TRI2D;
        for (int c = 0; c < m.nColFree; ++c) o->ranges.push_back({m.col_free[c], m.col_free[c + 1]});
        if (!p.fix_boundary && m.nFeature > 0) {
            // boundary vertices slide along their boundary curves (DMOTriFlatClass::doIteration)
            o->slide = o->feat = o->pass1d = true;
            for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
        }
    } else if (flat2d) {
        // flat quads (any grid) and flat triangles with a 4-point grid: the general 2D search
        if (!p.fix_boundary) return fail(VSDMO_E_UNSUPPORTED, "sliding boundary vertices are not implemented yet; set fix_boundary=1");
        if (m.maxHE > flat_max_ring()) return fail(VSDMO_E_VALENCE, "a vertex has more halfedges than the kernel's ring budget");
        o->mode = MODE_FLAT;
        o->kind = m.type == VSDMO_QUAD ? MK_QUAD2D : MK_TRI2D;
        for (int c = 0; c < m.nColFree; ++c) o->ranges.push_back({m.col_free[c], m.col_free[c + 1]});
    } else if (m.type == VSDMO_TRI || m.type == VSDMO_QUAD) {
        if (m.maxHE > dmo_surf_max_ring()) return fail(VSDMO_E_VALENCE, "a vertex has more halfedges than the kernel's ring budget");
        o->mode = MODE_SURF;
        o->kind = m.type == VSDMO_QUAD ? (cond ? MK_QUAD_COND : MK_QUAD) : MK_TRI3D;
        for (int c = 0; c < m.nColFree; ++c) o->ranges.push_back({m.col_free[c], m.col_free[c + 1]});
        if (m.nFeature > 0) {
            // feature neighbours project onto their sector surfaces; the feature vertices themselves
            // slide along their feature curves unless fix_boundary holds them
            o->feat = true;
            o->pass1d = !p.fix_boundary;
            for (int c = 0; c < m.nColFeature; ++c) o->franges.push_back({m.col_feature[c], m.col_feature[c + 1]});
        }
    } else {
        return fail(VSDMO_E_UNSUPPORTED, "element type not supported");
    }
    vsdmo_status st = guarded([&] {
        cudaStream_t s = m.stream;
        o->d_iter.alloc(1, s); o->d_iter.zero();
        o->pmin.alloc(quality_stats_blocks(), s);
        o->psum.alloc(quality_stats_blocks(), s);
        o->pfail.alloc(quality_stats_blocks(), s);
        o->done.alloc(1, s); o->done.zero();
        prepare_dmo_kernels();
        if (o->mode == MODE_ANGLE) prepare_angle_kernels();
        if (o->kind == MK_HEX_COND) prepare_hex_cond_kernels();
        if (o->volsurf) prepare_surf_kernels();
        if (o->mode == MODE_SURF || o->slide || o->volsurf) init_surface_state(o.get());
        o->counters.alloc(4, s);
        o->counters.zero();
        if (o->mode == MODE_TET && p.active_set) {
            o->dirty.alloc(m.nV, s);
            o->dirty.fill_bytes(1);
        }
        ensure_capacity(o.get(), std::min(std::max(p.n_iter, 1), 4096));
        launch_quality_stats(m, o->kind, o->stats.p, o->d_iter.p, o->pmin.p, o->psum.p, o->pfail.p, o->done.p, -1, s);
        auto h = read_stats(o.get(), 0, 1);
        o->last_min = h[0].min_q;
    });
    if (st != VSDMO_OK) return st;
    ++mesh->n_opts;
    *out = o.release();
    return VSDMO_OK;
}

VSDMO_API void vsdmo_opt_destroy(vsdmo_opt_t opt) {
    if (!opt) return;
    vsdmo_mesh_s* mesh = opt->mesh;
    cudaStreamSynchronize(mesh->m.stream);
    delete opt;
    if (--mesh->n_opts == 0 && mesh->destroy_requested) release_mesh(mesh);
}

VSDMO_API vsdmo_status vsdmo_opt_iterate(vsdmo_opt_t o, int n_iter) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (n_iter < 0) return fail(VSDMO_E_ARG, "n_iter < 0");
    if (n_iter == 0) return VSDMO_OK;
    int failures = 0;
    vsdmo_status st = guarded([&] {
        cudaStream_t s = o->mesh->m.stream;
        ensure_capacity(o, o->iters_done + n_iter);
        for (int i = 0; i < n_iter; ++i) {
            o->proposals_once = (o->model && o->once_after >= 0 && o->iters_done + i >= o->once_after) ? 1 : 0;
            ensure_graph(o);
            if (o->exec[o->proposals_once]) VSDMO_CUDA(cudaGraphLaunch(o->exec[o->proposals_once], s));
            else run_iteration_body(o, s);
        }
        auto h = read_stats(o, o->iters_done + 1, n_iter);
        for (auto& x : h) failures += x.fail_count;
        o->iters_done += n_iter;
        o->last_min = h.back().min_q;
        // an expired network wait is reported after the iterations are counted: they ran, and
        // every move was evaluated on the current ring whatever the proposals held
        if (o->model) o->model->m.check(s);
    });
    if (st != VSDMO_OK) return st;
    if (failures) return fail(VSDMO_E_MONOTONE, "minimum quality decreased during the iteration");
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_opt_restart(vsdmo_opt_t o) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        o->iters_done = 0;
        o->d_iter.zero();
        if (o->mode == MODE_SURF || o->slide || o->volsurf) init_surface_state(o);
        o->counters.zero();
        if (o->fb_count.p) o->fb_count.zero();
        if (o->dirty.p) o->dirty.fill_bytes(1);
        launch_quality_stats(m, o->kind, o->stats.p, o->d_iter.p, o->pmin.p, o->psum.p, o->pfail.p, o->done.p, -1,
                             m.stream);
        auto h = read_stats(o, 0, 1);
        o->last_min = h[0].min_q;
    });
}

VSDMO_API vsdmo_status vsdmo_opt_optimize(vsdmo_opt_t o) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    int left = o->p.n_iter - o->iters_done;
    if (left <= 0) return VSDMO_OK;
    return vsdmo_opt_iterate(o, left);
}

VSDMO_API int vsdmo_opt_is_done(vsdmo_opt_t o) { return o ? (o->iters_done >= o->p.n_iter) : 1; }

VSDMO_API int vsdmo_opt_iterations_done(vsdmo_opt_t o) { return o ? o->iters_done : -1; }

VSDMO_API int vsdmo_opt_launches_per_iteration(vsdmo_opt_t o) {
    if (!o) return -1;
    // colour launches + quality kernel (+ nearest-neighbour walk and two normal kernels)
    return (int)o->ranges.size() + 1 + (o->mode == MODE_SURF || o->volsurf ? 3 : 0) + (o->slide ? 1 : 0) +
           (o->volsurf && o->dirty.p ? 1 : 0) +
           (o->pass1d ? (int)o->fmranges.size() : 0) + (int)o->sranges.size();
}

VSDMO_API vsdmo_status vsdmo_opt_feature_state(vsdmo_opt_t o, float* curves, int32_t* fdeg, uint8_t* flags,
                                               int32_t* sector_rowptr, int32_t* sector_table, float* sector_surfaces,
                                               int* n_sectors) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (!o->feat) return fail(VSDMO_E_ARG, "the optimiser has no feature vertices");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        if (n_sectors) *n_sectors = o->nsect;
        if (curves) VSDMO_CUDA(cudaMemcpyAsync(curves, o->LS1.p, sizeof(float4) * 3L * m.nSurf, cudaMemcpyDeviceToHost, s));
        if (fdeg) VSDMO_CUDA(cudaMemcpyAsync(fdeg, o->fdeg.p, sizeof(int) * m.nSurf, cudaMemcpyDeviceToHost, s));
        if (flags) VSDMO_CUDA(cudaMemcpyAsync(flags, o->fopt.p, m.nSurf, cudaMemcpyDeviceToHost, s));
        if (o->nsect > 0) {
            if (sector_rowptr) VSDMO_CUDA(cudaMemcpyAsync(sector_rowptr, o->srow.p, sizeof(int) * (m.nFeature + 1), cudaMemcpyDeviceToHost, s));
            if (sector_table) VSDMO_CUDA(cudaMemcpyAsync(sector_table, o->stab.p, sizeof(int) * 20L * m.nFeature, cudaMemcpyDeviceToHost, s));
            if (sector_surfaces) VSDMO_CUDA(cudaMemcpyAsync(sector_surfaces, o->FS.p, sizeof(float4) * 4L * o->nsect, cudaMemcpyDeviceToHost, s));
        }
        m.sync();
    });
}

VSDMO_API vsdmo_status vsdmo_opt_surface_state(vsdmo_opt_t o, float* xyz_init, float* local_surfaces,
                                               int32_t* nearest) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (o->mode != MODE_SURF && !o->slide && !o->volsurf) return fail(VSDMO_E_ARG, "not a surface optimiser");
    if (local_surfaces && !o->LS.p) return fail(VSDMO_E_ARG, "this optimiser has no local surfaces");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        const int nS = m.nSurf;
        if (xyz_init) {
            DBuf<float> t(3L * nS, s);
            k_pack_xyz<<<grid_for(nS, 256), 256, 0, s>>>(o->X0.p, nS, nullptr, t.p);
            VSDMO_CHECK_LAUNCH();
            VSDMO_CUDA(cudaMemcpyAsync(xyz_init, t.p, sizeof(float) * 3L * nS, cudaMemcpyDeviceToHost, s));
            m.sync();
        }
        if (local_surfaces)
            VSDMO_CUDA(cudaMemcpyAsync(local_surfaces, o->LS.p, sizeof(float4) * 4L * nS, cudaMemcpyDeviceToHost, s));
        if (nearest) VSDMO_CUDA(cudaMemcpyAsync(nearest, o->nn.p, sizeof(int) * nS, cudaMemcpyDeviceToHost, s));
        m.sync();
    });
}

VSDMO_API vsdmo_status vsdmo_opt_get_quality(vsdmo_opt_t o, float* q) {
    if (!o || !q) return fail(VSDMO_E_ARG, "null argument");
    *q = o->last_min;
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_opt_element_qualities(vsdmo_opt_t o, float* out, int mem_space) {
    if (!o || !out) return fail(VSDMO_E_ARG, "null argument");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        if (mem_space == VSDMO_DEVICE) {
            launch_element_qualities(m, o->kind, out, s);
            m.sync();
        } else {
            DBuf<float> t(m.nE, s);
            launch_element_qualities(m, o->kind, t.p, s);
            VSDMO_CUDA(cudaMemcpyAsync(out, t.p, sizeof(float) * m.nE, cudaMemcpyDeviceToHost, s));
            m.sync();
        }
    });
}

VSDMO_API vsdmo_status vsdmo_opt_find_min_quality(vsdmo_opt_t o, float* min_q, double* mean_q) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    std::vector<float> q;
    vsdmo_status st = guarded([&] {
        const Mesh& m = o->mesh->m;
        DBuf<float> t(m.nE, m.stream);
        launch_element_qualities(m, o->kind, t.p, m.stream);
        q = t.to_host();
    });
    if (st != VSDMO_OK) return st;
    float mn = INFINITY;
    double sm = 0.0;
    for (float x : q) { mn = std::min(mn, x); sm += x; }
    if (min_q) *min_q = mn;
    if (mean_q) *mean_q = q.empty() ? 0.0 : sm / (double)q.size();
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_opt_quality_histogram(vsdmo_opt_t o, int32_t* host_counts, int n_cols) {
    if (!o || !host_counts || n_cols <= 0) return fail(VSDMO_E_ARG, "bad argument");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        DBuf<int> c(n_cols, m.stream);
        c.zero();
        launch_quality_histogram(m, o->kind, c.p, n_cols, m.stream);
        auto h = c.to_host();
        std::memcpy(host_counts, h.data(), sizeof(int) * n_cols);
    });
}

VSDMO_API vsdmo_status vsdmo_opt_display_quality(vsdmo_opt_t o, int n_cols) {
    if (n_cols <= 0) n_cols = 10;
    std::vector<int32_t> c(n_cols);
    vsdmo_status st = vsdmo_opt_quality_histogram(o, c.data(), n_cols);
    if (st != VSDMO_OK) return st;
    float mn;
    st = vsdmo_opt_find_min_quality(o, &mn, nullptr);
    if (st != VSDMO_OK) return st;
    // table layout of DMOBaseClass::printFormattedQuality (dmo/DMOBase.h:61-87)
    int maxnum = *std::max_element(c.begin(), c.end());
    int maxlen = std::max((int)std::log10(std::max(maxnum, 1)) + 1, 5);
    std::ostringstream os;
    os << "interval ";
    for (int i = 0; i < n_cols; ++i) {
        std::string si = std::to_string((float)i / (float)n_cols).substr(0, 4);
        os << si;
        for (int j = 0; j < maxlen - (int)si.size(); ++j) os << " |";
    }
    os << "\namount   ";
    for (int i = 0; i < n_cols; ++i) {
        std::string sn = std::to_string(c[i]);
        os << sn;
        for (int j = 0; j < maxlen - (int)sn.size(); ++j) os << " ";
        os << "|";
    }
    os << "\nq_min = " << mn << "\n";
    std::cout << os.str() << std::flush;
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_opt_history(vsdmo_opt_t o, float* min_q, double* mean_q, int cap, int* n) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    std::vector<IterStats> h;
    vsdmo_status st = guarded([&] { h = read_stats(o, 0, o->iters_done + 1); });
    if (st != VSDMO_OK) return st;
    const int cnt = std::min(cap, (int)h.size());
    const double nE = (double)o->mesh->m.nE;
    for (int i = 0; i < cnt; ++i) {
        if (min_q) min_q[i] = h[i].min_q;
        if (mean_q) mean_q[i] = h[i].sum_q / nE;
    }
    if (n) *n = cnt;
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_opt_run_color(vsdmo_opt_t o, int color) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (color < 0 || color >= (int)o->ranges.size()) return fail(VSDMO_E_ARG, "colour out of range");
    return guarded([&] { launch_color(o, color, o->mesh->m.stream); });
}

VSDMO_API vsdmo_status vsdmo_quality_reduce_noalloc(int elem_type, int flat, const float* d_xyz, int n_vertices,
                                                    const int32_t* d_elems, int n_elems, float threshold, float* d_min,
                                                    double* d_sum, int32_t* d_below, void* cuda_stream) {
    if (elem_type != VSDMO_TET && !(elem_type == VSDMO_TRI && flat))
        return fail(VSDMO_E_UNSUPPORTED, "the no-alloc reduction covers tetrahedra and flat triangles");
    if (!d_xyz || !d_elems || !d_min || !d_sum || !d_below) return fail(VSDMO_E_ARG, "null pointer");
    if (n_vertices <= 0 || n_elems <= 0) return fail(VSDMO_E_ARG, "empty mesh");
    if ((long)n_elems > noalloc_max_elements())
        return fail(VSDMO_E_ARG, "n_elems " + std::to_string(n_elems) + " exceeds the no-alloc limit of " +
                                     std::to_string(noalloc_max_elements()) + " elements per call");
    return guarded([&] {
        quality_reduce_noalloc(elem_type == VSDMO_TET ? 4 : 3, d_xyz, n_vertices, d_elems, n_elems, threshold, d_min,
                               d_sum, d_below, (cudaStream_t)cuda_stream);
    });
}

}  // extern "C"
