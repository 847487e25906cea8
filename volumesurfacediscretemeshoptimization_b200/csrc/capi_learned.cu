// capi_learned.cu -- C ABI of the learned proposal: the network handle (create, parameters,
// forward, gradients, training), training-pair collection from plain DMO, and the switch that
// puts a tet optimiser into learned mode. None of this has a counterpart in the reference.
#include "capi_internal.cuh"
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

namespace {

void copy_in_rows(DBuf<float>& dst, const float* src, size_t count, int mem_space, cudaStream_t s) {
    dst.alloc(count, s);
    VSDMO_CUDA(cudaMemcpyAsync(dst.p, src, sizeof(float) * count,
                               mem_space == VSDMO_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
}

}  // namespace

extern "C" {

VSDMO_API vsdmo_status vsdmo_debug_gemm_bf16(const float* A, const float* B, int M, int N, int K, float* D) {
    if (!A || !B || !D || M <= 0 || K <= 0 || K % 32) return fail(VSDMO_E_ARG, "need M > 0, K a multiple of 32");
    return guarded([&] {
        cudaStream_t s;
        VSDMO_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            mlp::prepare(s);
            mlp::debug_gemm(A, B, M, N, K, D, s);
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        VSDMO_CUDA(cudaStreamSynchronize(s));
        cudaStreamDestroy(s);
    });
}

VSDMO_API vsdmo_status vsdmo_debug_set_wait_limit_ns(int64_t ns) {
    if (ns > 1000000000ll) return fail(VSDMO_E_ARG, "the wait limit can only be lowered (at most 1e9 ns)");
    const unsigned long long lim = ns < 0 ? 1000000000ull : (unsigned long long)ns;
    return guarded([&] {
        mlp::set_wait_limit(lim);
        batch_set_wait_limit(lim);
    });
}

VSDMO_API int vsdmo_model_num_params(void) { return mlp::N_PARAMS; }

VSDMO_API vsdmo_status vsdmo_model_create(uint64_t seed, void* cuda_stream, vsdmo_model_t* out) {
    if (!out) return fail(VSDMO_E_ARG, "null output handle");
    *out = nullptr;
    std::unique_ptr<vsdmo_model_s> h(new vsdmo_model_s);
    vsdmo_status st = guarded([&] {
        if (cuda_stream) {
            h->stream = (cudaStream_t)cuda_stream;
        } else {
            VSDMO_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
            h->own_stream = true;
        }
        mlp::prepare(h->stream);
        h->m.init(seed, h->stream);
    });
    if (st != VSDMO_OK) {
        if (h->own_stream && h->stream) {
            cudaStream_t s = h->stream;
            h.reset();
            cudaStreamDestroy(s);
        }
        return st;
    }
    *out = h.release();
    return VSDMO_OK;
}

VSDMO_API void vsdmo_model_destroy(vsdmo_model_t m) {
    if (!m) return;
    cudaStream_t s = m->stream;
    const bool own = m->own_stream;
    cudaStreamSynchronize(s);
    delete m;
    if (own) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
}

VSDMO_API vsdmo_status vsdmo_model_get_params(vsdmo_model_t m, float* host) {
    if (!m || !host) return fail(VSDMO_E_ARG, "null argument");
    return guarded([&] { m->m.get_params(host); });
}

VSDMO_API vsdmo_status vsdmo_model_set_params(vsdmo_model_t m, const float* host) {
    if (!m || !host) return fail(VSDMO_E_ARG, "null argument");
    return guarded([&] { m->m.set_params(host); });
}

VSDMO_API vsdmo_status vsdmo_model_forward(vsdmo_model_t m, const float* feats, long n, float* out, int mem_space) {
    if (!m || !feats || !out || n <= 0) return fail(VSDMO_E_ARG, "bad argument");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        cudaStream_t s = m->stream;
        DBuf<float> f;
        copy_in_rows(f, feats, (size_t)n * mlp::IN, mem_space, s);
        m->ws.ensure(n, false, s);
        m->m.gather(m->ws, f.p, nullptr, nullptr, (int)n, (int)n, false, s);
        m->m.forward(m->ws, (int)n, false, s);
        m->m.check(s);
        std::vector<float> y = m->ws.Y.to_host();
        std::vector<float> o((size_t)n * mlp::OUT);
        for (long r = 0; r < n; ++r)
            for (int j = 0; j < mlp::OUT; ++j) o[(size_t)r * mlp::OUT + j] = y[(size_t)r * mlp::OUTP + j];
        if (mem_space == VSDMO_DEVICE)
            VSDMO_CUDA(cudaMemcpyAsync(out, o.data(), sizeof(float) * o.size(), cudaMemcpyHostToDevice, s));
        else
            std::memcpy(out, o.data(), sizeof(float) * o.size());
        VSDMO_CUDA(cudaStreamSynchronize(s));
    });
}

VSDMO_API vsdmo_status vsdmo_model_gradients(vsdmo_model_t m, const float* feats, const float* targets, int n,
                                             float* loss, float* grads) {
    if (!m || !feats || !targets || n <= 0 || n % 128) return fail(VSDMO_E_ARG, "n must be a positive multiple of 128");
    return guarded([&] {
        cudaStream_t s = m->stream;
        DBuf<float> f, t;
        copy_in_rows(f, feats, (size_t)n * mlp::IN, VSDMO_HOST, s);
        copy_in_rows(t, targets, (size_t)n * mlp::OUT, VSDMO_HOST, s);
        m->ws.ensure(n, true, s);
        m->m.gather(m->ws, f.p, t.p, nullptr, n, n, true, s);
        m->m.forward(m->ws, n, true, s);
        m->m.backward(m->ws, n, s);
        m->m.check(s);
        if (loss) *loss = read_scalar(m->ws.loss.p, s) / (3.f * (float)n);
        if (grads) {
            VSDMO_CUDA(cudaMemcpyAsync(grads, m->m.grads.p, sizeof(float) * mlp::N_PARAMS, cudaMemcpyDeviceToHost, s));
            VSDMO_CUDA(cudaStreamSynchronize(s));
        }
    });
}

VSDMO_API vsdmo_status vsdmo_model_train(vsdmo_model_t m, const float* feats, const float* targets, long n_rows,
                                         int mem_space, int steps, int batch, float lr, uint64_t seed,
                                         float* loss_history) {
    if (!m || !feats || !targets || n_rows <= 0 || steps < 0) return fail(VSDMO_E_ARG, "bad argument");
    if (batch <= 0 || batch % 128) return fail(VSDMO_E_ARG, "batch must be a positive multiple of 128");
    if (mem_space != VSDMO_HOST && mem_space != VSDMO_DEVICE) return fail(VSDMO_E_ARG, "bad mem_space");
    return guarded([&] {
        cudaStream_t s = m->stream;
        DBuf<float> fh, th;
        const float* df = feats;
        const float* dt = targets;
        if (mem_space == VSDMO_HOST) {
            copy_in_rows(fh, feats, (size_t)n_rows * mlp::IN, VSDMO_HOST, s);
            copy_in_rows(th, targets, (size_t)n_rows * mlp::OUT, VSDMO_HOST, s);
            df = fh.p;
            dt = th.p;
        }
        m->ws.ensure(batch, true, s);
        DBuf<float> hist(std::max(steps, 1), s);
        std::mt19937_64 g(seed);
        std::uniform_int_distribution<long> pick(0, n_rows - 1);
        std::vector<int> idx(batch);
        DBuf<int> didx[2] = { DBuf<int>(batch, s), DBuf<int>(batch, s) };
        for (int it = 0; it < steps; ++it) {
            for (int i = 0; i < batch; ++i) idx[i] = (int)pick(g);
            DBuf<int>& d = didx[it & 1];
            VSDMO_CUDA(cudaMemcpyAsync(d.p, idx.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, s));
            m->m.gather(m->ws, df, dt, d.p, batch, batch, true, s);
            m->m.forward(m->ws, batch, true, s);
            m->m.backward(m->ws, batch, s);
            m->m.adam(lr, s);
            VSDMO_CUDA(cudaMemcpyAsync(hist.p + it, m->ws.loss.p, sizeof(float), cudaMemcpyDeviceToDevice, s));
        }
        m->m.check(s);
        if (loss_history && steps > 0) {
            std::vector<float> h = hist.to_host();
            for (int i = 0; i < steps; ++i) loss_history[i] = h[i] / (3.f * (float)batch);
        }
        VSDMO_CUDA(cudaStreamSynchronize(s));
    });
}

VSDMO_API vsdmo_status vsdmo_opt_set_model(vsdmo_opt_t o, vsdmo_model_t model, int reduced_n, int reduced_depth,
                                           float reduced_scale) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (model && o->mode != MODE_TET) return fail(VSDMO_E_UNSUPPORTED, "the learned proposal is implemented for tet meshes");
    if (model && (reduced_n < 2 || reduced_n > 8 || reduced_depth < 1 || reduced_depth > 4))
        return fail(VSDMO_E_ARG, "reduced grid: 2..8 points per axis, 1..4 levels");
    if (model && !(reduced_scale > 0.f && reduced_scale <= 1.f)) return fail(VSDMO_E_ARG, "reduced_scale must be in (0, 1]");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        o->model = model;
        o->reduced_n = reduced_n;
        o->reduced_depth = reduced_depth;
        o->reduced_scale = reduced_scale;
        if (model) {
            int maxn = 1;
            for (auto& r : o->ranges) maxn = std::max(maxn, r.second - r.first);
            o->ws.ensure(maxn, false, s);
            o->ensure_neighbours();
            if (!o->fb_list.p || (int)o->fb_list.n < maxn) o->fb_list.alloc(maxn, s);
            if (!o->fb_count.p) o->fb_count.alloc(2, s);
            o->fb_count.zero();
        }
        o->counters.zero();
        // the captured iteration changes
        o->drop_graphs();
        m.sync();
    });
}

VSDMO_API vsdmo_status vsdmo_opt_set_proposal_schedule(vsdmo_opt_t o, int once_after) {
    if (!o) return fail(VSDMO_E_ARG, "null optimiser");
    if (o->mode != MODE_TET) return fail(VSDMO_E_UNSUPPORTED, "the learned proposal is implemented for tet meshes");
    if (once_after < -1) return fail(VSDMO_E_ARG, "once_after must be -1 or an iteration index >= 0");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        o->once_after = once_after;
        if (once_after >= 0 && !o->Yall.p) o->Yall.alloc((size_t)std::max(m.nV - m.nSurf, 1) * mlp::OUTP, m.stream);
        if (once_after >= 0) o->ensure_neighbours();
        m.sync();
    });
}

VSDMO_API vsdmo_status vsdmo_opt_proposals(vsdmo_opt_t o, int color, float* out) {
    if (!o || !out) return fail(VSDMO_E_ARG, "null argument");
    if (!o->model) return fail(VSDMO_E_ARG, "no model set");
    if (color < 0 || color >= (int)o->ranges.size()) return fail(VSDMO_E_ARG, "colour out of range");
    return guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        const int v0 = o->ranges[color].first, n = o->ranges[color].second - v0;
        o->model->m.infer_tet(m.pos.p, o->nb.p, o->nbn.p, o->nb_base, v0, n, o->ws.Y.p, mlp::OUTP, s);
        o->model->m.check(s);
        std::vector<float> y((size_t)n * mlp::OUTP);
        VSDMO_CUDA(cudaMemcpyAsync(y.data(), o->ws.Y.p, sizeof(float) * y.size(), cudaMemcpyDeviceToHost, s));
        VSDMO_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < 3; ++j) out[(size_t)i * 3 + j] = y[(size_t)i * mlp::OUTP + j];
    });
}

VSDMO_API vsdmo_status vsdmo_opt_learned_counters(vsdmo_opt_t o, unsigned long long* out4) {
    if (!o || !out4) return fail(VSDMO_E_ARG, "null argument");
    return guarded([&] {
        std::vector<unsigned long long> h = o->counters.to_host();
        for (int i = 0; i < 4; ++i) out4[i] = h[i];
    });
}

VSDMO_API vsdmo_status vsdmo_opt_collect_pairs(vsdmo_opt_t o, int n_iter, float* feats, float* targets, long capacity,
                                               long* n_out) {
    if (!o || !feats || !targets || capacity <= 0 || n_iter < 0) return fail(VSDMO_E_ARG, "bad argument");
    if (o->mode != MODE_TET) return fail(VSDMO_E_UNSUPPORTED, "training pairs are collected from tet meshes");
    long rows = 0;
    vsdmo_status st = guarded([&] {
        const Mesh& m = o->mesh->m;
        cudaStream_t s = m.stream;
        int maxn = 1;
        for (auto& r : o->ranges) maxn = std::max(maxn, r.second - r.first);
        DBuf<float> scale(maxn, s);
        DBuf<float4> old(maxn, s);
        o->ensure_neighbours();
        for (int it = 0; it < n_iter && rows < capacity; ++it) {
            for (auto& r : o->ranges) {
                const int n = (int)std::min<long>(r.second - r.first, capacity - rows);
                if (n <= 0) break;
                launch_tet_features(m, r.first, r.first + n, o->nb.p, o->nbn.p, o->nb_base, feats + rows * mlp::IN,
                                    nullptr, scale.p, old.p, s);
                DmoLaunch L{r.first, r.second, o->p.grid_scale, o->p.depth};
                launch_dmo_tet(m, L, s);
                launch_tet_targets(m, r.first, r.first + n, scale.p, old.p, targets + rows * mlp::OUT, s);
                rows += n;
            }
        }
        m.sync();
    });
    if (n_out) *n_out = rows;
    return st;
}

}  // extern "C"
