// prim.cu -- device-wide primitives used by the connectivity build: exclusive scan, stable
// LSD radix sort of (key, value) pairs, stable compaction and CSR offsets. These replace the
// thrust::sort_by_key / remove_if / inclusive_scan calls of the reference's mesh build
// (e.g. mesh/MeshTriGPU.cu:142,162-170, mesh/MeshTetGPU.cu:125) and k_find_first_n
// (mesh/SortUtil.cu:3-35). The build runs once per mesh; these kernels are HBM-bound.
#include "vsdmo_internal.cuh"
#include <mutex>

namespace vsdmo {

namespace {
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr unsigned FULL = 0xffffffffu;

__global__ void k_scan_tiles(const int* in, int* out, long n, int* block_sums) {
    __shared__ int warp_sum[SCAN_THREADS / 32];
    const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        s += v[i];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < SCAN_THREADS / 32 ? warp_sum[lane] : 0;
        int u = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL, u, o);
            if (lane >= o) u += y;
        }
        if (lane < SCAN_THREADS / 32) warp_sum[lane] = u - t;  // exclusive
        if (lane == SCAN_THREADS / 32 - 1) block_sums[blockIdx.x] = u;
    }
    __syncthreads();
    int run = warp_sum[w] + (x - s);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

__global__ void k_scan_add(int* out, long n, const int* block_offs) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] += block_offs[i / SCAN_TILE];
}

constexpr int RS_THREADS = 256;
constexpr int RS_ROUNDS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void k_radix_hist(const uint32_t* keys, long n, int shift, int* counts, int nTiles) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ROUNDS; ++r) {
        long idx = base + (long)r * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1);
    }
    __syncthreads();
    counts[(long)threadIdx.x * nTiles + blockIdx.x] = h[threadIdx.x];
}

// One tile of RS_TILE pairs: the stable rank of every pair within the tile, computed 256 pairs at
// a time (a warp match per digit, warp counts, a running base per digit), places the pair in
// shared memory in tile-local digit order; then consecutive threads write consecutive pairs of
// a digit run to consecutive global positions (the tile's run of digit d starts at its global
// offset offs[d * nTiles + tile]), so the writes coalesce.
__global__ void __launch_bounds__(RS_THREADS)
k_radix_scatter(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, long n, int shift,
                const int* offs, int nTiles) {
    __shared__ uint32_t sk[RS_TILE], sv[RS_TILE];
    __shared__ int gbase[256], lstart[256], run[256];
    __shared__ int wcnt[RS_WARPS][257];
    __shared__ int wsum[RS_WARPS];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const long tile = (long)blockIdx.x * RS_TILE;
    const int tile_n = (int)min((long)RS_TILE, n - tile);
    // the tile's count of digit tid, from the scanned (digit-major) offsets
    const long idx = (long)tid * nTiles + blockIdx.x;
    const int g = offs[idx];
    const int next = (idx + 1 < 256L * nTiles) ? offs[idx + 1] : (int)n;
    const int cnt = next - g;
    gbase[tid] = g;
    // exclusive scan of the counts over the digits: the tile-local run starts
    int x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    int before = 0;
#pragma unroll
    for (int i = 0; i < RS_WARPS; ++i) before += i < w ? wsum[i] : 0;
    lstart[tid] = before + x - cnt;
    run[tid] = before + x - cnt;
    __syncthreads();
    for (int r = 0; r < RS_ROUNDS; ++r) {
        for (int j = tid; j < RS_WARPS * 257; j += RS_THREADS) (&wcnt[0][0])[j] = 0;
        __syncthreads();
        const long i = tile + (long)r * RS_THREADS + tid;
        const bool valid = i < n;
        const uint32_t k = valid ? kin[i] : 0u;
        const uint32_t v = valid ? vin[i] : 0u;
        const int d = valid ? (int)((k >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(FULL, d);
        const int rank = __popc(peers & lt);
        if (lane == __ffs(peers) - 1) wcnt[w][d] = __popc(peers);
        __syncthreads();
        {
            int s = run[tid];
#pragma unroll
            for (int ww = 0; ww < RS_WARPS; ++ww) {
                const int t = wcnt[ww][tid];
                wcnt[ww][tid] = s;
                s += t;
            }
            run[tid] = s;
        }
        __syncthreads();
        if (valid) {
            const int p = wcnt[w][d] + rank;
            sk[p] = k;
            sv[p] = v;
        }
        __syncthreads();
    }
    for (int j = tid; j < tile_n; j += RS_THREADS) {
        const uint32_t k = sk[j];
        const int d = (int)((k >> shift) & 255u);
        const int p = gbase[d] + (j - lstart[d]);
        kout[p] = k;
        vout[p] = sv[j];
    }
}

__global__ void k_flags_to_int(const uint8_t* f, int* o, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        o[i] = f[i] ? 1 : 0;
}

__global__ void k_compact_scatter(const uint8_t* f, const int* pos, long n, int* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (f[i]) out[pos[i]] = (int)i;
}

// flag == first ? 1 : 0
__global__ void k_match_to_int(const uint8_t* f, int first, int* o, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        o[i] = ((f[i] != 0) == (first != 0)) ? 1 : 0;
}

// stable partition: matching index i goes to pos[i], the others after the *total matching
// ones, in index order (i - pos[i] non-matching indices precede i)
__global__ void k_partition_scatter(const uint8_t* f, int first, const int* pos, const int* total, long n,
                                    int* out) {
    const int nm = *total;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const bool match = (f[i] != 0) == (first != 0);
        out[match ? pos[i] : nm + (int)(i - pos[i])] = (int)i;
    }
}

__global__ void k_count_keys(const uint32_t* keys, long n, int* counts) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        atomicAdd(&counts[keys[i]], 1);
}
// ---- CSR of the distinct pairs ------------------------------------------------------------------
// bucket the values by key: each pair takes the next free slot of its key's row (the order
// inside a row is arbitrary; k_row_unique makes the row canonical)
__global__ void k_bucket_scatter(const uint32_t* keys, const uint32_t* vals, long n, int* cursor, uint32_t* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[atomicAdd(&cursor[keys[i]], 1)] = vals[i];
}

// one warp per row (grid-stride over rows): the row's distinct values in ascending order to
// out[rs[r] ...] and their number to u[r]. A value is kept at its first occurrence in the row,
// and its place is the number of kept values below it. Rows are short (the edges of one
// vertex's ring), so the quadratic scans cost less than sorting the rows.
__global__ void k_row_unique(const int* rs, const uint32_t* v, long K, uint8_t* keep, uint32_t* out, int* u) {
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < K; r += nw) {
        const int b = rs[r], n = rs[r + 1] - b;
        for (int i = lane; i < n; i += 32) {
            const uint32_t x = v[b + i];
            bool first = true;
            for (int j = 0; j < i && first; ++j) first = v[b + j] != x;
            keep[b + i] = first ? 1 : 0;
        }
        __syncwarp();
        int cnt = 0;
        for (int i = lane; i < n; i += 32) {
            if (!keep[b + i]) continue;
            const uint32_t x = v[b + i];
            int rank = 0;
            for (int j = 0; j < n; ++j) rank += (keep[b + j] && v[b + j] < x) ? 1 : 0;
            out[b + rank] = x;
            ++cnt;
        }
        cnt = __reduce_add_sync(FULL, cnt);
        if (lane == 0) u[r] = cnt;
        __syncwarp();
    }
}

// one warp per row: the distinct values of row r to col[rowptr[r] ...]
__global__ void k_row_copy(const int* rs, const int* rowptr, const uint32_t* src, long K, int* col) {
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < K; r += nw) {
        const int b = rs[r], o = rowptr[r], n = rowptr[r + 1] - o;
        for (int j = lane; j < n; j += 32) col[o + j] = (int)src[b + j];
    }
}

// bucket the indices [0, n) by key (arbitrary order inside a row)
__global__ void k_bucket_index(const uint32_t* keys, long n, int* cursor, uint32_t* out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[atomicAdd(&cursor[keys[i]], 1)] = (uint32_t)i;
}

// one warp per row (grid-stride): the row's indices in ascending order (each placed by the
// number of smaller indices in the row: they are distinct), and the row's key beside each
__global__ void k_row_order(const int* rs, const uint32_t* idx, long K, uint32_t* order, uint32_t* keys) {
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long r = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < K; r += nw) {
        const int b = rs[r], n = rs[r + 1] - b;
        for (int i = lane; i < n; i += 32) {
            const uint32_t x = idx[b + i];
            int k = 0;
            for (int j = 0; j < n; ++j) k += idx[b + j] < x ? 1 : 0;
            order[b + k] = x;
            keys[b + i] = (uint32_t)r;
        }
    }
}

// the longest row of a CSR row pointer rs[0..K] to *out (atomic maximum; *out starts at 0)
__global__ void k_longest_row(const int* rs, long K, int* out) {
    int m = 0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < K; r += (long)gridDim.x * blockDim.x)
        m = max(m, rs[r + 1] - rs[r]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m > 0) atomicMax(out, m);
}

__global__ void k_iota_u32(uint32_t* a, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        a[i] = (uint32_t)i;
}

// in (key, value)-sorted pairs: 1 where a pair differs from the one before it, counted per key
__global__ void k_flag_distinct(const uint32_t* k, const uint32_t* v, long n, uint8_t* flag, int* per_key) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const bool d = i == 0 || k[i] != k[i - 1] || v[i] != v[i - 1];
        flag[i] = d ? 1 : 0;
        if (d) atomicAdd(&per_key[k[i]], 1);
    }
}

__global__ void k_gather_col(const uint32_t* v, const int* idx, long n, int* col) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        col[i] = (int)v[idx[i]];
}

}  // namespace

int longest_row(const int* d_rowptr, long K, cudaStream_t s) {
    if (K <= 0) return 0;
    DBuf<int> m(1, s);
    m.zero();
    k_longest_row<<<grid_for(K, 256), 256, 0, s>>>(d_rowptr, K, m.p);
    VSDMO_CHECK_LAUNCH();
    return read_scalar(m.p, s);
}

int bits_for(uint32_t maxval) {
    int b = 1;
    while (b < 32 && (maxval >> b) != 0u) ++b;
    return b;
}

void exclusive_scan(const int* d_in, int* d_out, long n, int* d_total, cudaStream_t s) {
    if (n <= 0) {
        if (d_total) VSDMO_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int), s));
        return;
    }
    long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    DBuf<int> sums(nb, s);
    k_scan_tiles<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(d_in, d_out, n, sums.p);
    VSDMO_CHECK_LAUNCH();
    if (nb > 1) {
        exclusive_scan(sums.p, sums.p, nb, d_total, s);
        k_scan_add<<<grid_for(n, 256), 256, 0, s>>>(d_out, n, sums.p);
        VSDMO_CHECK_LAUNCH();
    } else if (d_total) {
        VSDMO_CUDA(cudaMemcpyAsync(d_total, sums.p, sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
}

void radix_sort_pairs(uint32_t* keys, uint32_t* vals, long n, int bits, cudaStream_t s) {
    if (n <= 1 || bits <= 0) return;
    const int nTiles = (int)((n + RS_TILE - 1) / RS_TILE);
    DBuf<uint32_t> k2(n, s), v2(n, s);
    DBuf<int> counts((long)256 * nTiles, s);
    uint32_t *ka = keys, *va = vals, *kb = k2.p, *vb = v2.p;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += 8, ++passes) {
        k_radix_hist<<<nTiles, RS_THREADS, 0, s>>>(ka, n, shift, counts.p, nTiles);
        VSDMO_CHECK_LAUNCH();
        exclusive_scan(counts.p, counts.p, (long)256 * nTiles, nullptr, s);
        k_radix_scatter<<<nTiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, counts.p, nTiles);
        VSDMO_CHECK_LAUNCH();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        VSDMO_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        VSDMO_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    }
}

int compact_flags(const uint8_t* d_flags, long n, int* d_out_index, cudaStream_t s) {
    if (n <= 0) return 0;
    DBuf<int> pos(n, s), tot(1, s);
    k_flags_to_int<<<grid_for(n, 256), 256, 0, s>>>(d_flags, pos.p, n);
    VSDMO_CHECK_LAUNCH();
    exclusive_scan(pos.p, pos.p, n, tot.p, s);
    k_compact_scatter<<<grid_for(n, 256), 256, 0, s>>>(d_flags, pos.p, n, d_out_index);
    VSDMO_CHECK_LAUNCH();
    return read_scalar(tot.p, s);
}

int stable_partition_flags(const uint8_t* d_flags, long n, int first_value, int* d_order, cudaStream_t s) {
    if (n <= 0) return 0;
    DBuf<int> pos(n, s), tot(1, s);
    k_match_to_int<<<grid_for(n, 256), 256, 0, s>>>(d_flags, first_value, pos.p, n);
    VSDMO_CHECK_LAUNCH();
    exclusive_scan(pos.p, pos.p, n, tot.p, s);
    k_partition_scatter<<<grid_for(n, 256), 256, 0, s>>>(d_flags, first_value, pos.p, tot.p, n, d_order);
    VSDMO_CHECK_LAUNCH();
    return read_scalar(tot.p, s);
}

void rowptr_from_sorted(const uint32_t* d_sorted_keys, long n, int K, int* d_rowptr, cudaStream_t s) {
    DBuf<int> counts((long)K + 1, s);
    counts.zero();
    if (n > 0) {
        k_count_keys<<<grid_for(n, 256), 256, 0, s>>>(d_sorted_keys, n, counts.p);
        VSDMO_CHECK_LAUNCH();
    }
    exclusive_scan(counts.p, d_rowptr, (long)K + 1, nullptr, s);
}

void csr_unique_from_pairs(const uint32_t* d_keys, const uint32_t* d_vals, long n, int K, int* d_rowptr, int* d_col,
                           cudaStream_t s) {
    if (K <= 0) {
        VSDMO_CUDA(cudaMemsetAsync(d_rowptr, 0, sizeof(int), s));
        return;
    }
    const long cap = std::max(n, 1L);
    DBuf<int> counts(K, s), rs((long)K + 1, s), cursor(K, s), u(K, s);
    DBuf<uint32_t> bucket(cap, s), uniq(cap, s);
    DBuf<uint8_t> keep(cap, s);
    counts.zero();
    if (n > 0) {
        k_count_keys<<<grid_for(n, 256), 256, 0, s>>>(d_keys, n, counts.p);
        VSDMO_CHECK_LAUNCH();
    }
    exclusive_scan(counts.p, rs.p, K, rs.p + K, s);
    if (n > 0 && longest_row(rs.p, K, s) > SHORT_ROW_MAX) {
        // a row too long for one warp's quadratic scans: the same CSR from two stable radix sorts
        // (by value, then by key) and the first pair of every run of equal pairs
        DBuf<uint32_t> kk(n, s), vv(n, s);
        DBuf<int> idx(n, s);
        VSDMO_CUDA(cudaMemcpyAsync(kk.p, d_keys, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        VSDMO_CUDA(cudaMemcpyAsync(vv.p, d_vals, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        radix_sort_pairs(vv.p, kk.p, n, 32, s);
        radix_sort_pairs(kk.p, vv.p, n, bits_for((uint32_t)(K > 1 ? K - 1 : 1)), s);
        u.zero();
        k_flag_distinct<<<grid_for(n, 256), 256, 0, s>>>(kk.p, vv.p, n, keep.p, u.p);
        VSDMO_CHECK_LAUNCH();
        exclusive_scan(u.p, d_rowptr, K, d_rowptr + K, s);
        const int nu = compact_flags(keep.p, n, idx.p, s);
        if (nu > 0) {
            k_gather_col<<<grid_for(nu, 256), 256, 0, s>>>(vv.p, idx.p, nu, d_col);
            VSDMO_CHECK_LAUNCH();
        }
        return;
    }
    VSDMO_CUDA(cudaMemcpyAsync(cursor.p, rs.p, sizeof(int) * K, cudaMemcpyDeviceToDevice, s));
    if (n > 0) {
        k_bucket_scatter<<<grid_for(n, 256), 256, 0, s>>>(d_keys, d_vals, n, cursor.p, bucket.p);
        VSDMO_CHECK_LAUNCH();
    }
    k_row_unique<<<grid_for((long)K * 32, 256), 256, 0, s>>>(rs.p, bucket.p, K, keep.p, uniq.p, u.p);
    VSDMO_CHECK_LAUNCH();
    exclusive_scan(u.p, d_rowptr, K, d_rowptr + K, s);
    k_row_copy<<<grid_for((long)K * 32, 256), 256, 0, s>>>(rs.p, d_rowptr, uniq.p, K, d_col);
    VSDMO_CHECK_LAUNCH();
}

int stable_sort_short_rows(uint32_t* d_keys, uint32_t* d_order, long n, int K, int* d_rowptr, cudaStream_t s) {
    if (K <= 0) return 0;
    DBuf<int> counts(K, s), cursor(K, s);
    DBuf<uint32_t> bucket(std::max(n, 1L), s);
    counts.zero();
    if (n > 0) {
        k_count_keys<<<grid_for(n, 256), 256, 0, s>>>(d_keys, n, counts.p);
        VSDMO_CHECK_LAUNCH();
    }
    exclusive_scan(counts.p, d_rowptr, K, d_rowptr + K, s);
    if (n <= 0) return 0;
    const int longest = longest_row(d_rowptr, K, s);
    if (longest > SHORT_ROW_MAX) {
        // a row too long for one warp's quadratic scan: the stable radix sort gives the same arrays
        k_iota_u32<<<grid_for(n, 256), 256, 0, s>>>(d_order, n);
        VSDMO_CHECK_LAUNCH();
        radix_sort_pairs(d_keys, d_order, n, bits_for((uint32_t)(K > 1 ? K - 1 : 1)), s);
        return longest;
    }
    VSDMO_CUDA(cudaMemcpyAsync(cursor.p, d_rowptr, sizeof(int) * K, cudaMemcpyDeviceToDevice, s));
    k_bucket_index<<<grid_for(n, 256), 256, 0, s>>>(d_keys, n, cursor.p, bucket.p);
    VSDMO_CHECK_LAUNCH();
    k_row_order<<<grid_for((long)K * 32, 256), 256, 0, s>>>(d_rowptr, bucket.p, K, d_order, d_keys);
    VSDMO_CHECK_LAUNCH();
    return longest;
}

cudaMemPool_t device_pool() {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    VSDMO_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        VSDMO_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = 8ull << 30;
        VSDMO_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[dev] = pool;
    }
    return pools[dev];
}

}  // namespace vsdmo
