// capi_internal.cuh -- handle structures and error plumbing shared by the C-ABI files.
#pragma once
#include "vsdmo_internal.cuh"
#include "mlp.cuh"
#include "batch.cuh"
#include <memory>
#include <string>

using namespace vsdmo;

struct vsdmo_mesh_s {
    Mesh m;
    int n_opts = 0;                 // optimisers that reference this mesh
    bool destroy_requested = false; // vsdmo_mesh_destroy came while optimisers were alive
};

enum OptMode { MODE_TET = 0, MODE_TRI2D = 1, MODE_SURF = 2, MODE_HEX = 3, MODE_FLAT = 4, MODE_ANGLE = 5 };

struct vsdmo_opt_s {
    vsdmo_mesh_s* mesh = nullptr;
    vsdmo_params p{};
    int iters_done = 0;
    int capacity = 0;
    int mode = MODE_TET;
    int kind = MK_TET;                         // element metric of the quality kernels
    std::vector<std::pair<int, int>> ranges;  // colour classes in launch order
    // feature / boundary pass: slide = flat triangles with sliding boundary vertices; feat = the
    // mesh has feature vertices (surface: sector surfaces always, the 1D pass unless fix_boundary)
    bool slide = false, feat = false, pass1d = false;
    bool volsurf = false;                      // tet / hex mesh with its boundary passes (fix_boundary = 0)
    std::vector<std::pair<int, int>> sranges;  // free boundary colour classes of a tet mesh
    DBuf<float4> LS1;                          // curves of the feature vertices [3 nSurf]
    DBuf<int> fdeg;                            // feature ring vertices [nSurf]
    DBuf<uint8_t> fopt;                        // the 1D pass moves the vertex [nSurf]
    DBuf<int> srow, stab;                      // sector rows [nFeature + 1], table [nFeature x 20]
    DBuf<float4> FS;                           // sector surfaces [4 per sector]
    DBuf<float4> Xs;                           // positions at the start of a colour class [nSurf]
    int nsect = 0;
    std::vector<std::pair<int, int>> franges;  // feature colour classes
    // movable feature vertices (the 1D pass moves them, fopt set), class by class: fmove holds
    // their ids, fmranges[c] the range of class c in it (rebuilt with the flags)
    DBuf<int> fmove;
    std::vector<int> fmove_ids;                // host copy of fmove
    std::vector<std::pair<int, int>> fmranges;
    DBuf<float4> X0;                           // surface mode: initial surface positions [nSurf]
    DBuf<float4> LS;                           // local surfaces [4 nSurf]
    DBuf<int> nn;                              // nearest initial vertex [nSurf]
    DBuf<IterStats> stats;
    DBuf<int> d_iter;
    DBuf<float> pmin;
    DBuf<double> psum;
    DBuf<int> pfail;
    DBuf<unsigned> done;
    // captured iterations: [0] the default body, [1] the body with one network launch for all
    // colour classes (learned mode, proposals_once)
    cudaGraph_t graph[2] = { nullptr, nullptr };
    cudaGraphExec_t exec[2] = { nullptr, nullptr };
    void drop_graphs() {
        for (int i = 0; i < 2; ++i) {
            if (exec[i]) { cudaGraphExecDestroy(exec[i]); exec[i] = nullptr; }
            if (graph[i]) { cudaGraphDestroy(graph[i]); graph[i] = nullptr; }
        }
    }
    float last_min = 0.f;
    // learned proposal (tet): model, feature rows of one colour class, proposals, counters
    struct vsdmo_model_s* model = nullptr;
    int reduced_n = 4, reduced_depth = 2;
    float reduced_scale = 2.0f / 7.0f;
    mlp::Workspace ws;
    DBuf<unsigned long long> counters;    // [0] reduced accepted, [1] fallback, [2] fallback moved, [3] skipped
    DBuf<uint8_t> dirty;                  // active-set flags [nV] (params.active_set)
    DBuf<int> nb, nbn;                    // ring vertices of the inner range [32 per vertex], counts
    DBuf<int> fb_list, fb_count;          // fallback queue of one colour class: entries, {length, blocks done}
    int proposals_once = 0;               // body being run or captured: 1 = one network launch for all colours
    int once_after = -1;                  // iterations from this one on (since the restart) use it; -1 never
    DBuf<float> Yall;                     // its proposals [inner vertices x OUTP]
    int nb_base = 0;
    void ensure_neighbours();
    bool collect = false;
    ~vsdmo_opt_s() { drop_graphs(); }
};

inline thread_local std::string g_last_error;

inline vsdmo_status fail(vsdmo_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

template <class F>
inline vsdmo_status guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return VSDMO_OK;
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(VSDMO_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(VSDMO_E_CUDA, e.what());
    }
}

struct vsdmo_model_s {
    mlp::Model m;
    mlp::Workspace ws;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
};
