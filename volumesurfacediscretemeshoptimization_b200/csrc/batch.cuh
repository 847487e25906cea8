// batch.cuh -- the batched multi-mesh optimiser (batch.cu): many flat triangle / quad meshes
// concatenated into one vertex space and iterated by one persistent launch per iteration.
#pragma once
#include "vsdmo_internal.cuh"
#include <string>
#include <vector>

namespace vsdmo {

// one work item: a chunk [v0, v1) of colour class `color` of mesh `mesh` (batch vertex ids)
struct BatchItem {
    int mesh, color, v0, v1;
};

// per-mesh search parameters as the kernel reads them
struct BatchMeshDev {
    int fk;        // 3 triangles, 4 quads
    int nq;        // candidates per axis (4 or 8)
    int depth;     // refinement levels (1..4)
    int lanes;     // lanes per vertex (8, 16 or 32)
    int col_base;  // first entry of this mesh in the per-(mesh, colour) arrays
    int n_elems;
    long el_off;   // first element index (x fk) in the concatenated element array
};

struct BatchStats {
    float min_q;
    int fail_count;   // elements below the previous iteration's minimum (monotonicity check)
    double sum_q;
};

struct BatchConfig {
    int nq, depth, lanes;
};

struct BatchMeshHost {
    int fk = 3, nV = 0, nE = 0;
    int v_off = 0, he_off = 0, col_base = 0, n_colors = 0;
    long el_off = 0;
    std::vector<int> col;          // colour offsets of the free vertices, mesh-local ids
};

// one input mesh: device arrays xyz [nV x 3], elems [nE x k] with mesh-local vertex ids
struct MeshInput {
    int elem_type, nV, nE;
    const float* d_xyz;
    const int* d_elems;
};

// single-mesh flat search (triangles or quads, N candidates per axis, `lanes` lanes per vertex)
void launch_dmo_flat(const Mesh& m, const DmoLaunch& L, int nq, int lanes, cudaStream_t s);
int flat_max_ring();
void prepare_flat_kernels();

struct Batch {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    float grid_scale = 0.5f;
    int maxk = 1;
    long nV = 0;
    std::vector<BatchMeshHost> hm;
    std::vector<BatchConfig> cfg;
    DBuf<float4> pos;            // [nV] internal numbering, mesh after mesh
    DBuf<int> old_to_batch;      // [nV] input (concatenated) vertex id -> batch vertex id
    DBuf<int> rowptr;            // [nV + 1] halfedge rows (batch halfedge ids)
    DBuf<int4> he;               // target, opposite, face, next (batch ids)
    DBuf<int> el;                // elements, batch vertex ids
    DBuf<int> csize, done, head, err, d_iter;
    DBuf<BatchMeshDev> d_meshes;
    DBuf<BatchItem> d_items;
    DBuf<BatchStats> stats;      // [(iterations + 1) x meshes]
    int n_items = 0;
    bool items_dirty = true;
    int blocks = 0;
    int iters_done = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~Batch();
    void build(const std::vector<MeshInput>& inputs, uint32_t seed);
    void set_configs(const std::vector<BatchConfig>& c);
    void restart();
    void iterate(int n);          // enqueues n graph replays
    void check_errors();          // synchronises; throws on an expired wait
    std::vector<BatchStats> read_stats(int slot) const;
    std::vector<std::string> autotune(int probe_iters);
    void get_positions(float* d_xyz_out) const;        // input numbering, [nV x 3]
    void set_positions(const float* d_xyz_in);
    int n_colors_total() const;

   private:
    void upload_meshes();
    void invalidate_graph();
    std::vector<BatchItem> make_items(const std::vector<int>& sel) const;
    void ensure_items();
    void ensure_stats(int iters);
    void ensure_launch_setup();
    void launch_iteration(const BatchItem* d_it, int n, bool with_stats, cudaStream_t s);
    void quality(BatchStats* out, int* d_it, int init, cudaStream_t s) const;
};

// limit of the colour-class waits of the batched iteration on the current device (test-only lowering)
void batch_set_wait_limit(unsigned long long ns);

}  // namespace vsdmo
