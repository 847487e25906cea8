// capi_batch.cu -- the extern "C" entry points of the batched flat-mesh optimiser (batch.cu).
#include "capi_internal.cuh"
#include <cstring>
#include <string>

struct vsdmo_batch_s {
    Batch b;
};

namespace {

void copy_in_b(void* dst, const void* src, size_t bytes, int mem_space, cudaStream_t s) {
    VSDMO_CUDA(cudaMemcpyAsync(dst, src, bytes, mem_space == VSDMO_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
}

}  // namespace

VSDMO_API vsdmo_status vsdmo_batch_create(int n_meshes, const int32_t* elem_types, const int32_t* n_vertices,
                                          const int32_t* n_elements, const float* xyz, const int32_t* elems,
                                          int mem_space, uint32_t color_seed, void* cuda_stream, vsdmo_batch_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    if (n_meshes <= 0 || !elem_types || !n_vertices || !n_elements || !xyz || !elems)
        return fail(VSDMO_E_ARG, "empty batch or null arrays");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    long vtot = 0, itot = 0;
    for (int i = 0; i < n_meshes; ++i) {
        if (elem_types[i] != VSDMO_TRI && elem_types[i] != VSDMO_QUAD)
            return fail(VSDMO_E_ARG, "batched meshes must be VSDMO_TRI or VSDMO_QUAD");
        if (n_vertices[i] <= 0 || n_elements[i] <= 0) return fail(VSDMO_E_ARG, "empty mesh in the batch");
        vtot += n_vertices[i];
        itot += (long)n_elements[i] * (elem_types[i] == VSDMO_TRI ? 3 : 4);
    }
    if (vtot > (long)INT32_MAX / 4 || itot > (long)INT32_MAX / 2) return fail(VSDMO_E_ARG, "batch too large for 32-bit indices");
    std::unique_ptr<vsdmo_batch_s> h(new vsdmo_batch_s);
    vsdmo_status st = guarded([&] {
        Batch& b = h->b;
        if (cuda_stream) {
            b.stream = (cudaStream_t)cuda_stream;
        } else {
            VSDMO_CUDA(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
            b.own_stream = true;
        }
        DBuf<float> dx(3L * vtot, b.stream);
        DBuf<int> de(itot, b.stream);
        copy_in_b(dx.p, xyz, sizeof(float) * 3L * vtot, mem_space, b.stream);
        copy_in_b(de.p, elems, sizeof(int) * itot, mem_space, b.stream);
        std::vector<MeshInput> in(n_meshes);
        long vo = 0, io = 0;
        for (int i = 0; i < n_meshes; ++i) {
            in[i] = MeshInput{elem_types[i], n_vertices[i], n_elements[i], dx.p + 3 * vo, de.p + io};
            vo += n_vertices[i];
            io += (long)n_elements[i] * (elem_types[i] == VSDMO_TRI ? 3 : 4);
        }
        b.build(in, color_seed);
        b.restart();
    });
    if (st != VSDMO_OK) {
        if (h->b.own_stream && h->b.stream) {
            cudaStream_t s = h->b.stream;
            h.reset();
            cudaStreamDestroy(s);
        }
        return st;
    }
    *out = h.release();
    return VSDMO_OK;
}

VSDMO_API void vsdmo_batch_destroy(vsdmo_batch_t batch) {
    if (!batch) return;
    const bool own = batch->b.own_stream;
    cudaStream_t s = batch->b.stream;
    if (s) cudaStreamSynchronize(s);
    delete batch;
    if (own && s) cudaStreamDestroy(s);
}

VSDMO_API vsdmo_status vsdmo_batch_iterate_async(vsdmo_batch_t batch, int n_iter) {
    if (!batch || n_iter < 0) return fail(VSDMO_E_ARG, "null batch or negative n_iter");
    return guarded([&] { if (n_iter) batch->b.iterate(n_iter); });
}

VSDMO_API vsdmo_status vsdmo_batch_sync(vsdmo_batch_t batch) {
    if (!batch) return fail(VSDMO_E_ARG, "null batch");
    return guarded([&] { batch->b.check_errors(); });
}

VSDMO_API vsdmo_status vsdmo_batch_iterate(vsdmo_batch_t batch, int n_iter) {
    const vsdmo_status st = vsdmo_batch_iterate_async(batch, n_iter);
    if (st != VSDMO_OK) return st;
    return vsdmo_batch_sync(batch);
}

VSDMO_API vsdmo_status vsdmo_batch_restart(vsdmo_batch_t batch) {
    if (!batch) return fail(VSDMO_E_ARG, "null batch");
    return guarded([&] { batch->b.restart(); });
}

VSDMO_API vsdmo_status vsdmo_batch_stats(vsdmo_batch_t batch, int iteration, float* min_q, double* mean_q,
                                         int32_t* below_prev_min) {
    if (!batch) return fail(VSDMO_E_ARG, "null batch");
    if (iteration < 0 || iteration > batch->b.iters_done) return fail(VSDMO_E_ARG, "no statistics for that iteration");
    return guarded([&] {
        const std::vector<BatchStats> st = batch->b.read_stats(iteration);
        for (size_t i = 0; i < st.size(); ++i) {
            if (min_q) min_q[i] = st[i].min_q;
            if (mean_q) mean_q[i] = st[i].sum_q / std::max(batch->b.hm[i].nE, 1);
            if (below_prev_min) below_prev_min[i] = st[i].fail_count;
        }
    });
}

VSDMO_API vsdmo_status vsdmo_batch_get_positions(vsdmo_batch_t batch, float* xyz, int mem_space) {
    if (!batch || !xyz) return fail(VSDMO_E_ARG, "null argument");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        Batch& b = batch->b;
        if (mem_space == VSDMO_DEVICE) {
            b.get_positions(xyz);
            return;
        }
        DBuf<float> t(3L * b.nV, b.stream);
        b.get_positions(t.p);
        VSDMO_CUDA(cudaMemcpyAsync(xyz, t.p, sizeof(float) * 3L * b.nV, cudaMemcpyDeviceToHost, b.stream));
        VSDMO_CUDA(cudaStreamSynchronize(b.stream));
    });
}

VSDMO_API vsdmo_status vsdmo_batch_set_positions(vsdmo_batch_t batch, const float* xyz, int mem_space) {
    if (!batch || !xyz) return fail(VSDMO_E_ARG, "null argument");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        Batch& b = batch->b;
        if (mem_space == VSDMO_DEVICE) {
            b.set_positions(xyz);
            return;
        }
        DBuf<float> t(3L * b.nV, b.stream);
        VSDMO_CUDA(cudaMemcpyAsync(t.p, xyz, sizeof(float) * 3L * b.nV, cudaMemcpyHostToDevice, b.stream));
        b.set_positions(t.p);
        VSDMO_CUDA(cudaStreamSynchronize(b.stream));   // the caller's host buffer may be reused on return
    });
}

VSDMO_API vsdmo_status vsdmo_batch_get_config(vsdmo_batch_t batch, int32_t* grid_n, int32_t* depth, int32_t* lanes) {
    if (!batch) return fail(VSDMO_E_ARG, "null batch");
    const std::vector<BatchConfig>& c = batch->b.cfg;
    for (size_t i = 0; i < c.size(); ++i) {
        if (grid_n) grid_n[i] = c[i].nq;
        if (depth) depth[i] = c[i].depth;
        if (lanes) lanes[i] = c[i].lanes;
    }
    return VSDMO_OK;
}

VSDMO_API vsdmo_status vsdmo_batch_set_config(vsdmo_batch_t batch, const int32_t* grid_n, const int32_t* depth,
                                              const int32_t* lanes) {
    if (!batch || !grid_n || !depth || !lanes) return fail(VSDMO_E_ARG, "null argument");
    return guarded([&] {
        std::vector<BatchConfig> c(batch->b.hm.size());
        for (size_t i = 0; i < c.size(); ++i) c[i] = BatchConfig{grid_n[i], depth[i], lanes[i]};
        batch->b.set_configs(c);
    });
}

VSDMO_API vsdmo_status vsdmo_batch_autotune(vsdmo_batch_t batch, int probe_iters, char* report, int report_len) {
    if (!batch) return fail(VSDMO_E_ARG, "null batch");
    return guarded([&] {
        const std::vector<std::string> lines = batch->b.autotune(probe_iters);
        if (report && report_len > 0) {
            std::string all;
            for (const std::string& l : lines) all += l + "\n";
            const size_t n = std::min(all.size(), (size_t)report_len - 1);
            std::memcpy(report, all.data(), n);
            report[n] = 0;
        }
    });
}

VSDMO_API long vsdmo_batch_info(vsdmo_batch_t batch, int which) {
    if (!batch) return -1;
    const Batch& b = batch->b;
    switch (which) {
    case 0: return (long)b.hm.size();
    case 1: return b.nV;
    case 2: {
        long n = 0;
        for (size_t i = 0; i < b.hm.size(); ++i) {
            const int chunk = 8 * (32 / b.cfg[i].lanes);
            for (int c = 0; c < b.hm[i].n_colors; ++c) n += (b.hm[i].col[c + 1] - b.hm[i].col[c] + chunk - 1) / chunk;
        }
        return n;
    }
    case 3: return b.n_colors_total();
    case 4: return b.iters_done;
    case 5: return b.blocks;
    case 6: return b.maxk;
    default: return -1;
    }
}

VSDMO_API vsdmo_status vsdmo_batch_mesh_info(vsdmo_batch_t batch, int mesh, int32_t* out8) {
    if (!batch || !out8) return fail(VSDMO_E_ARG, "null argument");
    if (mesh < 0 || mesh >= (int)batch->b.hm.size()) return fail(VSDMO_E_ARG, "mesh index out of range");
    const BatchMeshHost& h = batch->b.hm[mesh];
    out8[0] = h.v_off;
    out8[1] = h.nV;
    out8[2] = h.nE;
    out8[3] = h.fk;
    out8[4] = h.n_colors;
    out8[5] = h.col.empty() ? 0 : h.col.front();
    out8[6] = h.col.empty() ? 0 : h.col.back();
    out8[7] = h.he_off;
    return VSDMO_OK;
}
