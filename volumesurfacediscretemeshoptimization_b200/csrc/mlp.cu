// mlp.cu -- the learned proposal network: a 96 -> 128 -> 128 -> 128 -> 3 ReLU MLP in BF16 with
// FP32 accumulation, trained and evaluated by the tcgen05 GEMM of tc_gemm.cuh.
//
// The network has no counterpart in the reference. It maps the one-ring of an inner vertex
// (up to 32 neighbour positions relative to the vertex, divided by the ring's largest per-axis
// extent, padded with zeros: 96 inputs) to the displacement plain DMO chose for that vertex,
// in the same units. Every layer is one GEMM launch, Z = H . W^T, with a fused epilogue:
//
//   forward   H_l = relu(Z_l + b_l) -> BF16, written packed as the next layer's A operand and,
//             for training, transposed as the weight-gradient GEMM's operand;
//             Y = Z_4 + b_4 in FP32;
//   loss      dY = 2 (Y - T) / (3B) (mean squared error), BF16, both layouts;
//   backward  dH_l = dZ_{l+1} . W_{l+1} (B operand = packed W^T), dZ_l = dH_l * [H_l > 0];
//             dW_l = dZ_l^T . H_{l-1} with the batch as K, split over CTAs (FP32 partials
//             summed in a fixed order, so gradients are deterministic); bias gradients from
//             per-warp column sums;
//   update    Adam on FP32 master weights, then the BF16 packed copies (W and W^T) rebuilt.
//
// Parameters live in one flat FP32 array: W1 [128x96] b1 [128] W2 [128x128] b2 W3 [128x128] b3
// W4 [16x128] b4 [16] (rows 3..15 of W4 and b4 stay zero: the output is padded to the
// smallest tensor-core N).
#include "vsdmo_internal.cuh"
#include "mlp.cuh"
#include "tc_gemm.cuh"
#include <cmath>
#include <cstring>
#include <random>

namespace vsdmo {
namespace mlp {

using tc::pk_off;
using tc::pk_bytes;

namespace {

enum Epi { EPI_RAW = 0, EPI_HIDDEN = 1, EPI_OUT = 2, EPI_DRELU = 3 };

struct GemmParams {
    const uint8_t* A;        // packed [Mpad x K]
    const uint8_t* B;        // packed [N x K]
    int K;                   // columns (multiple of 32)
    int chunks_per_part;     // split-K: chunks per blockIdx.y
    int M;                   // valid rows
    int Mtot;                // rows of the tile grid (multiple of 128): K of transposed outputs
    int* err;
    const float* bias;       // [N] (hidden / out)
    uint8_t* out;            // packed bf16 [Mpad x N]  (hidden / drelu)
    uint8_t* outT;           // packed bf16 [N x Mtot]  (optional)
    float* outf;             // fp32 outputs (raw: [parts][Mtot x N], out: [M x ldo])
    int ldo;
    int nvalid;              // columns written by EPI_OUT
    const uint8_t* H;        // packed bf16 forward activation [Mpad x N] (drelu mask)
    float* dbias;            // drelu: per-warp column sums [Mtot/32 x N]
};

__device__ __forceinline__ void store_bf16x8(uint8_t* base, size_t off, const float* v) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16_rn(v[i]);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(h);
}

template <int N, int EPI>
struct Epilogue {
    const GemmParams& p;
    int mt, part;
    __device__ void operator()(int row, int c0, float* v) {
        const long m = (long)mt * 128 + row;
        const bool valid = m < p.M;
        if (EPI == EPI_RAW) {
            float* o = p.outf + ((size_t)part * p.Mtot + m) * N + c0;
#pragma unroll
            for (int i = 0; i < 16; ++i) o[i] = v[i];
        } else if (EPI == EPI_HIDDEN) {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = valid ? fmaxf(v[i] + p.bias[c0 + i], 0.f) : 0.f;
            store_bf16x8(p.out, pk_off(m, c0, N), v);
            store_bf16x8(p.out, pk_off(m, c0 + 8, N), v + 8);
            if (p.outT) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    *reinterpret_cast<__nv_bfloat16*>(p.outT + pk_off(c0 + i, (int)m, p.Mtot)) = __float2bfloat16_rn(v[i]);
            }
        } else if (EPI == EPI_OUT) {
            if (valid) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i < p.nvalid) p.outf[(size_t)m * p.ldo + c0 + i] = v[i] + p.bias[c0 + i];
            }
        } else {  // EPI_DRELU
            const uint4 h0 = *reinterpret_cast<const uint4*>(p.H + pk_off(m, c0, N));
            const uint4 h1 = *reinterpret_cast<const uint4*>(p.H + pk_off(m, c0 + 8, N));
            const __nv_bfloat16* hb0 = reinterpret_cast<const __nv_bfloat16*>(&h0);
            const __nv_bfloat16* hb1 = reinterpret_cast<const __nv_bfloat16*>(&h1);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float h = __bfloat162float(i < 8 ? hb0[i] : hb1[i - 8]);
                v[i] = (valid && h > 0.f) ? v[i] : 0.f;
            }
            float q[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) q[i] = __bfloat162float(__float2bfloat16_rn(v[i]));
            store_bf16x8(p.out, pk_off(m, c0, N), v);
            store_bf16x8(p.out, pk_off(m, c0 + 8, N), v + 8);
            if (p.outT) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    *reinterpret_cast<__nv_bfloat16*>(p.outT + pk_off(c0 + i, (int)m, p.Mtot)) = __float2bfloat16_rn(v[i]);
            }
            // bias gradient: column sums of the (BF16-rounded) dZ over this warp's 32 rows
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float s = q[i];
#pragma unroll
                for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                q[i] = s;
            }
            if ((threadIdx.x & 31) == 0) {
                const int wrow = mt * 4 + (threadIdx.x >> 5);
#pragma unroll
                for (int i = 0; i < 16; ++i) p.dbias[(size_t)wrow * N + c0 + i] = q[i];
            }
        }
    }
};

template <int N, int EPI>
__global__ void __launch_bounds__(tc::GEMM_THREADS) k_gemm(GemmParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int mt = blockIdx.x, part = blockIdx.y;
    const int kA = p.K / tc::CHUNK_K;
    const int c0 = part * p.chunks_per_part;
    const int c1 = min(kA, c0 + p.chunks_per_part);
    if (c0 >= c1) return;
    Epilogue<N, EPI> e{p, mt, part};
    tc::gemm_tile<N>(p.A + (size_t)mt * kA * tc::CHUNK_BYTES, p.B, kA, c0, c1, smem, p.err, e);
}

// launch; the shared-memory limit of every instantiation is raised once by prepare()
template <int N, int EPI>
void launch_gemm(const GemmParams& p, int m_tiles, int parts, cudaStream_t s) {
    k_gemm<N, EPI><<<dim3(m_tiles, parts), tc::GEMM_THREADS, tc::gemm_smem_bytes<N>(), s>>>(p);
    VSDMO_CHECK_LAUNCH();
}

// ---- parameter handling -------------------------------------------------------------------------
__global__ void k_pack_matrix(const float* __restrict__ W, int rows, int cols, int ld, uint8_t* __restrict__ out,
                              int K, int transpose) {
    // out = packed bf16 of W [rows x cols] (transpose = 0: rows x K, K >= cols, zero padded;
    // transpose = 1: cols x K, K >= rows)
    const long n = (long)rows * cols;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        const __nv_bfloat16 h = __float2bfloat16_rn(W[(size_t)r * ld + c]);
        if (!transpose) *reinterpret_cast<__nv_bfloat16*>(out + pk_off(r, c, K)) = h;
        else *reinterpret_cast<__nv_bfloat16*>(out + pk_off(c, r, K)) = h;
    }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// zero the padded output rows 3..15 of W4 and b4
__global__ void k_mask_out(float* params) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < (OUTP - OUT) * HID) params[OFF_W4 + OUT * HID + i] = 0.f;
    if (i < OUTP - OUT) params[OFF_B4 + OUT + i] = 0.f;
}

// sum of split-K partials [parts][rows x cols] into dst (row-major rows x cols, or transposed)
__global__ void k_reduce_parts(const float* __restrict__ part, int parts, int rows, int cols, int part_rows,
                               float* __restrict__ dst, int transpose, int dst_cols) {
    const int n = rows * cols;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = i / cols, c = i % cols;
        float s = 0.f;
        for (int q = 0; q < parts; ++q) s += part[((size_t)q * part_rows + r) * cols + c];
        if (!transpose) dst[(size_t)r * dst_cols + c] = s;
        else dst[(size_t)c * dst_cols + r] = s;
    }
}

// bias gradient: sum of per-warp column sums [nw x N] (first `valid` columns)
__global__ void k_reduce_bias(const float* __restrict__ wsum, int nw, int N, int valid, float* __restrict__ dst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    float s = 0.f;
    for (int q = 0; q < nw; ++q) s += wsum[(size_t)q * N + c];
    dst[c] = c < valid ? s : 0.f;
}

// mean squared error gradient of the padded output: dY = 2 (Y - T) / (3 B) for the 3 real
// columns; writes dY packed [B x 32] (columns 16..31 stay zero) and transposed [16 x B],
// per-warp column sums for the bias and per-row losses
__global__ void k_mse_grad(const float* __restrict__ Y, const float* __restrict__ T, int B, uint8_t* dY, uint8_t* dYT,
                           float* wsum, float* loss_rows) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;   // blockDim = 128, B % 128 == 0
    float d[OUTP];
    float l = 0.f;
    const float scale = 2.f / (3.f * (float)B);
#pragma unroll
    for (int j = 0; j < OUTP; ++j) {
        if (j < OUT && r < B) {
            const float e = Y[(size_t)r * OUTP + j] - T[(size_t)r * OUT + j];
            d[j] = scale * e;
            l += e * e;
        } else {
            d[j] = 0.f;
        }
    }
    if (r < B) {
        store_bf16x8(dY, pk_off(r, 0, 32), d);
        store_bf16x8(dY, pk_off(r, 8, 32), d + 8);
#pragma unroll
        for (int j = 0; j < OUTP; ++j) *reinterpret_cast<__nv_bfloat16*>(dYT + pk_off(j, r, B)) = __float2bfloat16_rn(d[j]);
        loss_rows[r] = l;
    }
#pragma unroll
    for (int j = 0; j < OUTP; ++j) {
        float s = __bfloat162float(__float2bfloat16_rn(d[j]));
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) wsum[(size_t)(r >> 5) * OUTP + j] = s;
    }
}

// rows of a row-major FP32 feature matrix (selected by idx, or consecutive) -> packed bf16 X
// [B x 96] and, if XT, transposed [96 x B]; targets gathered alongside
__global__ void k_gather_batch(const float* __restrict__ feats, const float* __restrict__ targets,
                               const int* __restrict__ idx, int B, int n_valid, uint8_t* X, uint8_t* XT, float* T) {
    const long total = (long)B * IN;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int r = (int)(i / IN), c = (int)(i % IN);
        const bool ok = r < n_valid;
        const long src = ok ? (idx ? idx[r] : r) : 0;
        const float x = ok ? feats[src * IN + c] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        *reinterpret_cast<__nv_bfloat16*>(X + pk_off(r, c, IN)) = h;
        if (XT) *reinterpret_cast<__nv_bfloat16*>(XT + pk_off(c, r, B)) = h;
        if (T && c < OUT) T[(size_t)r * OUT + c] = ok ? targets[src * OUT + c] : 0.f;
    }
}

__global__ void k_sum(const float* a, int n, float* out) {
    __shared__ float sh[256];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += 256) s += a[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// ---- fused inference for the learned tet search --------------------------------------------------
// One persistent CTA of 16 warps per SM keeps the packed BF16 weights in shared memory (loaded
// once by bulk copies) and runs two tiles of 128 vertices at a time: the CTA is two groups of
// 8 warps, each with its own activation buffer, 128 TMEM columns and MMA barrier, so one
// group's ring gathers (global loads) overlap the other group's layer chain (MMAs and
// epilogues). Within a group the two threads of a row build its 96 inputs from the ring-vertex
// table, sixteen ring vertices each, straight into the packed A operand; the four layers then
// run back to back on the tensor cores, each layer's epilogue split over the group's warps by
// TMEM lane quadrant (rows) and 64-column half, overwriting the buffer its own MMAs have
// finished reading. Groups synchronise on their own named barrier.
constexpr int FI_THREADS = 512;
constexpr int FI_GROUPS = 2;
constexpr int FI_GTHREADS = FI_THREADS / FI_GROUPS;                 // threads of a group
constexpr uint32_t FI_W1 = 0, FI_W2 = FI_W1 + 3 * 8192, FI_W3 = FI_W2 + 4 * 8192, FI_W4 = FI_W3 + 4 * 8192;
constexpr uint32_t FI_WBYTES = FI_W4 + 4 * 1024;                    // weights: 94,208 bytes
constexpr uint32_t FI_BUF = FI_WBYTES;                              // + one 32 KB activation tile per group
constexpr uint32_t FI_SMEM = FI_BUF + FI_GROUPS * 4 * 8192;         // 159,744 bytes
constexpr int FI_PARTS = FI_GTHREADS / 128;                         // threads per row of the tile
constexpr int FI_NB_PART = MAX_NB / FI_PARTS;                       // ring vertices per thread

// packed offset of (row, col) inside one 128-row tile held in shared memory
__device__ __forceinline__ uint32_t tile_off(int r, int c) {
    return (uint32_t)(c >> 5) * 8192u + (uint32_t)(r >> 3) * 512u + (uint32_t)((c & 31) >> 3) * 128u +
           (uint32_t)(r & 7) * 16u + (uint32_t)(c & 7) * 2u;
}

__device__ __forceinline__ void fi_store8(uint8_t* base, uint32_t off, const float* v) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16_rn(v[i]);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(h);
}

// issue one layer: D[128 x N] = A (K columns, tile in smem) . B^T; b_chunk: bytes between the
// 32-column chunks of B (8192, or 1024 for the compact 16-row W4)
__device__ __forceinline__ void fi_layer_issue(uint32_t tmem, uint32_t a, uint32_t b, int K, uint32_t b_chunk,
                                               uint32_t idesc, uint32_t bar) {
    for (int j = 0; j < K / 16; ++j) {
        const uint32_t ao = a + (uint32_t)(j >> 1) * 8192u + (uint32_t)(j & 1) * 256u;
        const uint32_t bo = b + (uint32_t)(j >> 1) * b_chunk + (uint32_t)(j & 1) * 256u;
        tc::mma_bf16(tmem, tc::smem_desc(ao), tc::smem_desc(bo), idesc, j > 0 ? 1u : 0u);
    }
    tc::mma_commit(bar);
}

__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(FI_GTHREADS) : "memory");
}

__global__ void __launch_bounds__(FI_THREADS, 1)
k_mlp_tet_infer(const float4* __restrict__ pos, const int* __restrict__ nb, const int* __restrict__ nbn, int nb_base,
                int v0, int n, const uint8_t* __restrict__ W1p, const uint8_t* __restrict__ W2p,
                const uint8_t* __restrict__ W3p, const uint8_t* __restrict__ W4p, const float* __restrict__ params,
                float* __restrict__ Y, int ldy, int* err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t bars[1 + FI_GROUPS];
    __shared__ uint32_t tmem_slot;
    __shared__ int s_wfail;
    // expired MMA waits of a group, one slot per step parity: a slot written in step s is read
    // after the group barrier of step s and next written in step s + 2, after every thread of
    // the group has passed the barrier of step s + 1, so all threads of a group read the same value
    __shared__ int s_fail[FI_GROUPS][2];
    __shared__ float s_max[FI_GROUPS][FI_PARTS][128];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = warp >> 3, gt = threadIdx.x & (FI_GTHREADS - 1);  // group, thread in the group
    const int row = gt & 127, part = gt >> 7;
    const uint32_t sb = tc::smem_u32(sm);
    const uint32_t bar_w = tc::smem_u32(&bars[0]), bar_m = tc::smem_u32(&bars[1 + g]);
    if (threadIdx.x == 0) {
        for (int b = 0; b < 1 + FI_GROUPS; ++b) tc::mbar_init(tc::smem_u32(&bars[b]), 1);
        tc::mbar_init_fence();
        s_wfail = 0;
        for (int b = 0; b < FI_GROUPS; ++b) s_fail[b][0] = s_fail[b][1] = 0;
    }
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_slot), 128 * FI_GROUPS);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot + 128u * (uint32_t)g;             // this group's 128 columns
    if (threadIdx.x == 0) {
        tc::mbar_expect_tx(bar_w, FI_WBYTES);
        tc::bulk_g2s(sb + FI_W1, W1p, 3 * 8192, bar_w);
        tc::bulk_g2s(sb + FI_W2, W2p, 4 * 8192, bar_w);
        tc::bulk_g2s(sb + FI_W3, W3p, 4 * 8192, bar_w);
        for (int c = 0; c < 4; ++c) tc::bulk_g2s(sb + FI_W4 + 1024u * c, W4p + (size_t)c * 8192, 1024, bar_w);
    }
    bool weights = tc::mbar_wait_reported(bar_w, 0);
    if (!weights && lane == 0) {
        atomicExch(err, tc::TC_TIMEOUT_LOAD);
        s_wfail = 1;
    }
    __syncthreads();
    uint8_t* buf = sm + FI_BUF + (uint32_t)g * 4u * 8192u;
    const uint32_t sbuf = sb + FI_BUF + (uint32_t)g * 4u * 8192u;
    const uint32_t id128 = tc::idesc_bf16(HID), id16 = tc::idesc_bf16(OUTP);
    const int q = warp & 3, ch = (warp >> 2) & 1;                      // lane quadrant, 64-column half
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    const int erow = q * 32 + lane;                                     // this thread's row in the epilogue
    const bool issuer = gt == 0;
    uint32_t phase = 0;
    bool pending = false;                                               // an MMA commit not yet seen
    int step = 0;
    const int ntiles = (n + 127) / 128;
    const int stride = FI_GROUPS * gridDim.x;
    bool stop = s_wfail != 0;
    for (int tile = blockIdx.x + g * gridDim.x; tile < ntiles && !stop; tile += stride) {
        // ---- inputs: ring vertices FI_NB_PART * part .. + FI_NB_PART of this row's vertex
        {
            const int i = tile * 128 + row;
            float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f);
            int cnt = 0, self = 0;
            int idx[FI_NB_PART];
            if (i < n) {
                self = v0 + i;
                c0 = pos[self];
                cnt = nbn[self - nb_base];
                const int4* rw = reinterpret_cast<const int4*>(nb + (size_t)(self - nb_base) * MAX_NB) +
                                 part * (FI_NB_PART / 4);
#pragma unroll
                for (int k = 0; k < FI_NB_PART / 4; ++k) {
                    const int4 t = rw[k];
                    idx[4 * k] = t.x; idx[4 * k + 1] = t.y; idx[4 * k + 2] = t.z; idx[4 * k + 3] = t.w;
                }
            } else {
#pragma unroll
                for (int a = 0; a < FI_NB_PART; ++a) idx[a] = 0;
            }
            // unpredicated loads (slots past the ring load the vertex itself and contribute zeros)
            float f[3 * FI_NB_PART];
            float mm = 0.f;
#pragma unroll
            for (int a = 0; a < FI_NB_PART; ++a) {
                const bool ok = part * FI_NB_PART + a < cnt;
                const float4 p = pos[ok ? idx[a] : self];
                const float dx = ok ? p.x - c0.x : 0.f, dy = ok ? p.y - c0.y : 0.f, dz = ok ? p.z - c0.z : 0.f;
                mm = fmaxf(mm, fmaxf(fabsf(dx), fmaxf(fabsf(dy), fabsf(dz))));
                f[3 * a] = dx; f[3 * a + 1] = dy; f[3 * a + 2] = dz;
            }
            s_max[g][part][row] = mm;
            group_sync(g);
#pragma unroll
            for (int k = 0; k < FI_PARTS; ++k) mm = fmaxf(mm, s_max[g][k][row]);
            const float inv = mm > 0.f ? 1.f / mm : 0.f;
#pragma unroll
            for (int c = 0; c < 3 * FI_NB_PART; ++c) f[c] = f[c] * inv;
#pragma unroll
            for (int k = 0; k < 3 * FI_NB_PART / 8; ++k)
                fi_store8(buf, tile_off(row, 3 * FI_NB_PART * part + 8 * k), f + 8 * k);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc::tc_fence_before();
        group_sync(g);
        const uint32_t srcW[3] = { FI_W1, FI_W2, FI_W3 };
        const int Ks[3] = { IN, HID, HID };
        const int boff[3] = { OFF_B1, OFF_B2, OFF_B3 };
        for (int l = 0; l < 4; ++l, ++step) {
            if (issuer) {
                tc::tc_fence_after();
                if (l < 3) fi_layer_issue(tmem, sbuf, sb + srcW[l], Ks[l], 8192u, id128, bar_m);
                else fi_layer_issue(tmem, sbuf, sb + FI_W4, HID, 1024u, id16, bar_m);
            }
            pending = true;
            if (!tc::mbar_wait_reported(bar_m, phase)) {
                if (lane == 0) {
                    atomicExch(err, tc::TC_TIMEOUT_MMA);
                    s_fail[g][step & 1] = 1;
                }
            } else {
                pending = false;
                phase ^= 1u;
            }
            tc::tc_fence_after();
            const int i = tile * 128 + erow;
            if (!pending) {
                if (l < 3) {
                    // the MMAs are done with the buffer: this warp's 32 rows x 64 columns of the
                    // activations overwrite it
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = 64 * ch + 32 * h;
                        float v[32];
                        tc::tmem_ld32(lane_addr + (uint32_t)c, v);
                        const float4* b4 = reinterpret_cast<const float4*>(params + boff[l] + c);   // 16-byte aligned
#pragma unroll
                        for (int e = 0; e < 32; e += 4) {
                            const float4 bb = __ldg(b4 + e / 4);
                            v[e] = i < n ? fmaxf(v[e] + bb.x, 0.f) : 0.f;
                            v[e + 1] = i < n ? fmaxf(v[e + 1] + bb.y, 0.f) : 0.f;
                            v[e + 2] = i < n ? fmaxf(v[e + 2] + bb.z, 0.f) : 0.f;
                            v[e + 3] = i < n ? fmaxf(v[e + 3] + bb.w, 0.f) : 0.f;
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) fi_store8(buf, tile_off(erow, c + 8 * k), v + 8 * k);
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                } else if (ch == 0) {
                    float v[16];
                    tc::tmem_ld16(lane_addr, v);
                    if (i < n) {
                        const float* b4 = params + OFF_B4;
                        float* y = Y + (size_t)i * ldy;
                        y[0] = v[0] + b4[0];
                        y[1] = v[1] + b4[1];
                        y[2] = v[2] + b4[2];
                    }
                }
            }
            tc::tc_fence_before();
            group_sync(g);
            if (s_fail[g][step & 1]) { stop = true; ++step; break; }
        }
    }
    // after a timed-out wait, give the copies and MMAs in flight a bounded time to land before
    // the shared and tensor memory are released
    if (!weights) (void)tc::mbar_wait(bar_w, 0);
    if (pending) (void)tc::mbar_wait(bar_m, phase);
    __syncthreads();
    if (warp == 0) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem_slot, 128 * FI_GROUPS);
    }
}

}  // namespace

// ---- Model ------------------------------------------------------------------------------------------
void Model::init(uint64_t seed, cudaStream_t s) {
    stream = s;
    params.alloc(N_PARAMS, s);
    grads.alloc(N_PARAMS, s);
    adam_m.alloc(N_PARAMS, s);
    adam_v.alloc(N_PARAMS, s);
    adam_m.zero();
    adam_v.zero();
    err.alloc(1, s);
    err.zero();
    W1p.alloc(pk_bytes(HID, IN), s);
    W2p.alloc(pk_bytes(HID, HID), s);
    W3p.alloc(pk_bytes(HID, HID), s);
    W4p.alloc(pk_bytes(OUTP, HID), s);
    W2Tp.alloc(pk_bytes(HID, HID), s);
    W3Tp.alloc(pk_bytes(HID, HID), s);
    W4Tp.alloc(pk_bytes(HID, 32), s);
    W4Tp.zero();
    W4p.zero();
    // He-uniform initialisation of the weights, zero biases
    std::vector<float> h(N_PARAMS, 0.f);
    std::mt19937_64 g(seed);
    auto fill = [&](int off, int rows, int cols, int valid_rows) {
        const float a = std::sqrt(6.f / (float)cols);
        std::uniform_real_distribution<float> u(-a, a);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) h[(size_t)off + (size_t)r * cols + c] = r < valid_rows ? u(g) : 0.f;
    };
    fill(OFF_W1, HID, IN, HID);
    fill(OFF_W2, HID, HID, HID);
    fill(OFF_W3, HID, HID, HID);
    fill(OFF_W4, OUTP, HID, OUT);
    set_params(h.data());
    step = 0;
}

void Model::set_params(const float* host) {
    VSDMO_CUDA(cudaMemcpyAsync(params.p, host, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice, stream));
    k_mask_out<<<(OUTP * HID + 255) / 256, 256, 0, stream>>>(params.p);
    VSDMO_CHECK_LAUNCH();
    repack();
    VSDMO_CUDA(cudaStreamSynchronize(stream));
}

void Model::get_params(float* host) const {
    VSDMO_CUDA(cudaMemcpyAsync(host, params.p, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost, stream));
    VSDMO_CUDA(cudaStreamSynchronize(stream));
}

void Model::repack() {
    auto pack = [&](int off, int rows, int cols, uint8_t* out, int K, int tr) {
        k_pack_matrix<<<grid_for((long)rows * cols, 256), 256, 0, stream>>>(params.p + off, rows, cols, cols, out, K, tr);
        VSDMO_CHECK_LAUNCH();
    };
    pack(OFF_W1, HID, IN, W1p.p, IN, 0);
    pack(OFF_W2, HID, HID, W2p.p, HID, 0);
    pack(OFF_W3, HID, HID, W3p.p, HID, 0);
    pack(OFF_W4, OUTP, HID, W4p.p, HID, 0);
    pack(OFF_W2, HID, HID, W2Tp.p, HID, 1);
    pack(OFF_W3, HID, HID, W3Tp.p, HID, 1);
    pack(OFF_W4, OUTP, HID, W4Tp.p, 32, 1);
}

void Workspace::ensure(long rows, bool training, cudaStream_t s) {
    const long R = ((rows + 127) / 128) * 128;
    if (R <= cap_rows && (!training || has_train)) return;
    cap_rows = std::max(R, cap_rows);
    has_train = has_train || training;
    const long C = cap_rows;
    X.alloc(pk_bytes(C, IN), s);
    H1.alloc(pk_bytes(C, HID), s);
    H2.alloc(pk_bytes(C, HID), s);
    H3.alloc(pk_bytes(C, HID), s);
    Y.alloc((size_t)C * OUTP, s);
    if (has_train) {
        XT.alloc(pk_bytes(IN, (int)C), s);
        H1T.alloc(pk_bytes(HID, (int)C), s);
        H2T.alloc(pk_bytes(HID, (int)C), s);
        H3T.alloc(pk_bytes(HID, (int)C), s);
        T.alloc((size_t)C * OUT, s);
        dY.alloc(pk_bytes(C, 32), s);
        dY.zero();
        dYT.alloc(pk_bytes(OUTP, (int)C), s);
        dZ3.alloc(pk_bytes(C, HID), s);
        dZ3T.alloc(pk_bytes(HID, (int)C), s);
        dZ2.alloc(pk_bytes(C, HID), s);
        dZ2T.alloc(pk_bytes(HID, (int)C), s);
        dZ1.alloc(pk_bytes(C, HID), s);
        dZ1T.alloc(pk_bytes(HID, (int)C), s);
        wsum.alloc((size_t)(C / 32) * HID, s);
        loss_rows.alloc(C, s);
        loss.alloc(1, s);
        parts.alloc((size_t)MAX_PARTS * 128 * HID, s);
        idx.alloc(C, s);
    }
}

namespace {
// split-K parts for the weight-gradient GEMMs (batch as K)
int wgrad_parts(int B) {
    const int chunks = B / 32;
    int parts = std::min(MAX_PARTS, std::max(1, chunks / 4));
    while (chunks % parts) --parts;
    return parts;
}
}  // namespace

void Model::forward(Workspace& w, int n, bool training, cudaStream_t s) {
    const int tiles = (n + 127) / 128;
    const int Mtot = tiles * 128;
    GemmParams p{};
    p.err = err.p;
    p.M = n;
    p.Mtot = Mtot;
    p.chunks_per_part = 1 << 20;
    // layer 1
    p.A = w.X.p; p.B = W1p.p; p.K = IN; p.bias = params.p + OFF_B1; p.out = w.H1.p; p.outT = training ? w.H1T.p : nullptr;
    launch_gemm<HID, EPI_HIDDEN>(p, tiles, 1, s);
    p.A = w.H1.p; p.B = W2p.p; p.K = HID; p.bias = params.p + OFF_B2; p.out = w.H2.p; p.outT = training ? w.H2T.p : nullptr;
    launch_gemm<HID, EPI_HIDDEN>(p, tiles, 1, s);
    p.A = w.H2.p; p.B = W3p.p; p.K = HID; p.bias = params.p + OFF_B3; p.out = w.H3.p; p.outT = training ? w.H3T.p : nullptr;
    launch_gemm<HID, EPI_HIDDEN>(p, tiles, 1, s);
    p.A = w.H3.p; p.B = W4p.p; p.K = HID; p.bias = params.p + OFF_B4; p.out = nullptr; p.outT = nullptr;
    p.outf = w.Y.p; p.ldo = OUTP; p.nvalid = OUTP;
    launch_gemm<OUTP, EPI_OUT>(p, tiles, 1, s);
}

void Model::backward(Workspace& w, int B, cudaStream_t s) {
    const int tiles = B / 128;
    // loss gradient
    k_mse_grad<<<tiles, 128, 0, s>>>(w.Y.p, w.T.p, B, w.dY.p, w.dYT.p, w.wsum.p, w.loss_rows.p);
    VSDMO_CHECK_LAUNCH();
    k_reduce_bias<<<1, 32, 0, s>>>(w.wsum.p, B / 32, OUTP, OUT, grads.p + OFF_B4);
    VSDMO_CHECK_LAUNCH();
    k_sum<<<1, 256, 0, s>>>(w.loss_rows.p, B, w.loss.p);
    VSDMO_CHECK_LAUNCH();
    GemmParams p{};
    p.err = err.p;
    p.M = B;
    p.Mtot = B;
    p.chunks_per_part = 1 << 20;
    // dZ3 = (dY . W4) * [H3 > 0]
    p.A = w.dY.p; p.B = W4Tp.p; p.K = 32; p.H = w.H3.p; p.out = w.dZ3.p; p.outT = w.dZ3T.p; p.dbias = w.wsum.p;
    launch_gemm<HID, EPI_DRELU>(p, tiles, 1, s);
    k_reduce_bias<<<1, HID, 0, s>>>(w.wsum.p, B / 32, HID, HID, grads.p + OFF_B3);
    VSDMO_CHECK_LAUNCH();
    // dZ2 = (dZ3 . W3) * [H2 > 0]
    p.A = w.dZ3.p; p.B = W3Tp.p; p.K = HID; p.H = w.H2.p; p.out = w.dZ2.p; p.outT = w.dZ2T.p;
    launch_gemm<HID, EPI_DRELU>(p, tiles, 1, s);
    k_reduce_bias<<<1, HID, 0, s>>>(w.wsum.p, B / 32, HID, HID, grads.p + OFF_B2);
    VSDMO_CHECK_LAUNCH();
    // dZ1 = (dZ2 . W2) * [H1 > 0]
    p.A = w.dZ2.p; p.B = W2Tp.p; p.K = HID; p.H = w.H1.p; p.out = w.dZ1.p; p.outT = w.dZ1T.p;
    launch_gemm<HID, EPI_DRELU>(p, tiles, 1, s);
    k_reduce_bias<<<1, HID, 0, s>>>(w.wsum.p, B / 32, HID, HID, grads.p + OFF_B1);
    VSDMO_CHECK_LAUNCH();
    // weight gradients: batch is K, one 128-row tile, split over `parts` CTAs
    const int parts = wgrad_parts(B);
    const int cpp = (B / 32) / parts;
    GemmParams q{};
    q.err = err.p;
    q.K = B;
    q.chunks_per_part = cpp;
    q.M = 128;
    q.Mtot = 128;
    q.outf = w.parts.p;
    // dW4^T [128 x 16] = H3^T . dY^T^T
    q.A = w.H3T.p; q.B = w.dYT.p;
    launch_gemm<OUTP, EPI_RAW>(q, 1, parts, s);
    k_reduce_parts<<<grid_for(128 * OUTP, 256), 256, 0, s>>>(w.parts.p, parts, 128, OUTP, 128, grads.p + OFF_W4, 1, HID);
    VSDMO_CHECK_LAUNCH();
    // dW3 [128 x 128] = dZ3^T . H2
    q.A = w.dZ3T.p; q.B = w.H2T.p;
    launch_gemm<HID, EPI_RAW>(q, 1, parts, s);
    k_reduce_parts<<<grid_for(128 * HID, 256), 256, 0, s>>>(w.parts.p, parts, 128, HID, 128, grads.p + OFF_W3, 0, HID);
    VSDMO_CHECK_LAUNCH();
    q.A = w.dZ2T.p; q.B = w.H1T.p;
    launch_gemm<HID, EPI_RAW>(q, 1, parts, s);
    k_reduce_parts<<<grid_for(128 * HID, 256), 256, 0, s>>>(w.parts.p, parts, 128, HID, 128, grads.p + OFF_W2, 0, HID);
    VSDMO_CHECK_LAUNCH();
    // dW1 [128 x 96] = dZ1^T . X
    q.A = w.dZ1T.p; q.B = w.XT.p;
    launch_gemm<IN, EPI_RAW>(q, 1, parts, s);
    k_reduce_parts<<<grid_for(128 * IN, 256), 256, 0, s>>>(w.parts.p, parts, 128, IN, 128, grads.p + OFF_W1, 0, IN);
    VSDMO_CHECK_LAUNCH();
    // padded output rows of W4 carry no gradient
    k_mask_out<<<(OUTP * HID + 255) / 256, 256, 0, s>>>(grads.p);
    VSDMO_CHECK_LAUNCH();
}

void Model::adam(float lr, cudaStream_t s) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    k_adam<<<grid_for(N_PARAMS, 256), 256, 0, s>>>(params.p, grads.p, adam_m.p, adam_v.p, N_PARAMS, lr, b1, b2, eps, c1, c2);
    VSDMO_CHECK_LAUNCH();
    k_mask_out<<<(OUTP * HID + 255) / 256, 256, 0, s>>>(params.p);
    VSDMO_CHECK_LAUNCH();
    repack();
}

void Model::gather(Workspace& w, const float* feats, const float* targets, const int* idx, int B, int n_valid,
                   bool training, cudaStream_t s) {
    k_gather_batch<<<grid_for((long)B * IN, 256), 256, 0, s>>>(feats, targets, idx, B, n_valid, w.X.p,
                                                               training ? w.XT.p : nullptr, training ? w.T.p : nullptr);
    VSDMO_CHECK_LAUNCH();
}

void Model::infer_tet(const float4* pos, const int* nb, const int* nbn, int nb_base, int v0, int n, float* Y,
                      int ldy, cudaStream_t s) {
    if (n <= 0) return;
    const int tiles = (n + 127) / 128;
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_mlp_tet_infer<<<std::min(tiles, sms), FI_THREADS, FI_SMEM, s>>>(pos, nb, nbn, nb_base, v0, n, W1p.p, W2p.p, W3p.p,
                                                                     W4p.p, params.p, Y, ldy, err.p);
    VSDMO_CHECK_LAUNCH();
}

void Model::check(cudaStream_t s) {
    const int e = read_scalar(err.p, s);
    if (e) {
        // the report is consumed: the next launch on this model starts from a clear flag
        VSDMO_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
        VSDMO_CUDA(cudaStreamSynchronize(s));
        throw Error(VSDMO_E_TIMEOUT, "tensor-core wait expired (code " + std::to_string(e) + ")");
    }
}

void set_wait_limit(unsigned long long ns) {
    VSDMO_CUDA(cudaDeviceSynchronize());
    VSDMO_CUDA(cudaMemcpyToSymbol(tc::g_wait_limit_ns, &ns, sizeof(ns)));
    VSDMO_CUDA(cudaDeviceSynchronize());
}

// Prepares every GEMM instantiation (dynamic shared-memory limits) outside stream capture.
void prepare(cudaStream_t s) {
    (void)s;
    auto cfg = [](const void* f, size_t bytes) {
        VSDMO_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    };
    cfg((const void*)k_gemm<HID, EPI_HIDDEN>, tc::gemm_smem_bytes<HID>());
    cfg((const void*)k_gemm<OUTP, EPI_OUT>, tc::gemm_smem_bytes<OUTP>());
    cfg((const void*)k_gemm<HID, EPI_DRELU>, tc::gemm_smem_bytes<HID>());
    cfg((const void*)k_gemm<OUTP, EPI_RAW>, tc::gemm_smem_bytes<OUTP>());
    cfg((const void*)k_gemm<HID, EPI_RAW>, tc::gemm_smem_bytes<HID>());
    cfg((const void*)k_gemm<IN, EPI_RAW>, tc::gemm_smem_bytes<IN>());
    cfg((const void*)k_gemm<32, EPI_RAW>, tc::gemm_smem_bytes<32>());
    cfg((const void*)k_gemm<64, EPI_RAW>, tc::gemm_smem_bytes<64>());
    cfg((const void*)k_mlp_tet_infer, FI_SMEM);
}

// D [M x N] = A [M x K] . B [N x K]^T for the GEMM test entry point (FP32 in, BF16 operands)
void debug_gemm(const float* hA, const float* hB, int M, int N, int K, float* hD, cudaStream_t s) {
    const int tiles = (M + 127) / 128, Mtot = tiles * 128;
    std::vector<uint16_t> pa(pk_bytes(Mtot, K) / 2, 0), pb(pk_bytes(128, K) / 2, 0);
    auto bf = [](float x) {
        uint32_t u;
        std::memcpy(&u, &x, 4);
        u += 0x7FFFu + ((u >> 16) & 1u);
        return (uint16_t)(u >> 16);
    };
    for (int r = 0; r < M; ++r)
        for (int k = 0; k < K; ++k) pa[pk_off(r, k, K) / 2] = bf(hA[(size_t)r * K + k]);
    for (int r = 0; r < N; ++r)
        for (int k = 0; k < K; ++k) pb[pk_off(r, k, K) / 2] = bf(hB[(size_t)r * K + k]);
    DBuf<uint8_t> dA(pa.size() * 2, s), dB(pb.size() * 2, s);
    DBuf<float> dD((size_t)Mtot * N, s);
    DBuf<int> e(1, s);
    e.zero();
    VSDMO_CUDA(cudaMemcpyAsync(dA.p, pa.data(), pa.size() * 2, cudaMemcpyHostToDevice, s));
    VSDMO_CUDA(cudaMemcpyAsync(dB.p, pb.data(), pb.size() * 2, cudaMemcpyHostToDevice, s));
    GemmParams p{};
    p.A = dA.p; p.B = dB.p; p.K = K; p.chunks_per_part = K / 32; p.M = M; p.Mtot = Mtot; p.err = e.p; p.outf = dD.p;
    switch (N) {
    case 16: launch_gemm<16, EPI_RAW>(p, tiles, 1, s); break;
    case 32: launch_gemm<32, EPI_RAW>(p, tiles, 1, s); break;
    case 64: launch_gemm<64, EPI_RAW>(p, tiles, 1, s); break;
    case 96: launch_gemm<96, EPI_RAW>(p, tiles, 1, s); break;
    case 128: launch_gemm<128, EPI_RAW>(p, tiles, 1, s); break;
    default: throw Error(VSDMO_E_ARG, "debug GEMM: N must be 16, 32, 64, 96 or 128");
    }
    const int code = read_scalar(e.p, s);
    if (code) throw Error(VSDMO_E_TIMEOUT, "tensor-core GEMM wait expired (code " + std::to_string(code) + ")");
    std::vector<float> d = dD.to_host();
    for (int r = 0; r < M; ++r)
        for (int c = 0; c < N; ++c) hD[(size_t)r * N + c] = d[(size_t)r * N + c];
}

}  // namespace mlp
}  // namespace vsdmo
