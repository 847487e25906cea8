// tc_gemm.cuh -- BF16 tensor-core GEMM on sm_100a (tcgen05 + TMEM + bulk async copies).
//
// D[128 x N] (fp32, in tensor memory) = A[128 rows x K] . B[N rows x K]^T for one 128-row tile
// of A per CTA, N in {16, 32, ..., 128}, K streamed in chunks of 32 columns. Operands live in
// global memory pre-packed in the "K-major, no swizzle" canonical layout of the tensor cores,
// cut into chunks of 128 rows x 32 columns (8 KB) so that one chunk is one contiguous bulk
// copy (cp.async.bulk, no tensor map):
//
//   chunk (row tile rt, column chunk kc) at byte ((rt * K/32) + kc) * 8192, inside it
//   element (r, k) at (r % 128 / 8) * 512 + (k % 32 / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
//
// i.e. 8 x 8 "core matrices" of 128 contiguous bytes, leading-dimension byte offset (next core
// matrix along K) 128 and stride byte offset (next 8-row group) 512. One elected thread
// streams chunks through a 4-stage ring of shared memory (mbarrier complete_tx), issues two
// K=16 tcgen05.mma per chunk and commits each stage back to the ring; the four warps then
// read their 32 accumulator lanes with tcgen05.ld and run the epilogue functor.
//
// Every wait on an mbarrier is bounded (about one second of %globaltimer); on expiry the
// kernel records an error code, lets its copies and MMAs drain (bounded as well), frees its
// tensor memory and returns without writing results.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace vsdmo {
namespace tc {

constexpr int CHUNK_K = 32;            // columns per chunk
constexpr int CHUNK_BYTES = 8192;      // 128 rows x 32 bf16
constexpr int STAGES = 4;
constexpr int GEMM_THREADS = 128;
constexpr unsigned long long WAIT_NS = 1000000000ull;  // bound on any single wait

enum TcErr { TC_OK = 0, TC_TIMEOUT_LOAD = 1, TC_TIMEOUT_MMA = 2, TC_TIMEOUT_DONE = 3 };

// byte offset of element (r, k) in a packed operand with K columns (K % 32 == 0)
__host__ __device__ __forceinline__ size_t pk_off(long r, int k, int K) {
    return ((size_t)(r >> 7) * (size_t)(K >> 5) + (size_t)(k >> 5)) * CHUNK_BYTES + (size_t)((r & 127) >> 3) * 512 +
           (size_t)((k & 31) >> 3) * 128 + (size_t)(r & 7) * 16 + (size_t)(k & 7) * 2;
}
// bytes of a packed operand with R rows (padded to 128) and K columns
__host__ __device__ __forceinline__ size_t pk_bytes(long R, int K) {
    return (size_t)((R + 127) >> 7) * (size_t)(K >> 5) * CHUNK_BYTES;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// non-blocking test of the phase with the given parity
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// wait of at most limit_ns for the phase with the given parity; false on timeout. The first
// check does not block, so a zero limit expires unless the phase has already completed.
__device__ __forceinline__ bool mbar_wait_for(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (now_ns() - t0 < limit_ns)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// the limit of the waits whose expiry a kernel reports (the GEMM's stage waits, the inference
// kernel's weight and MMA waits): WAIT_NS unless the test-only vsdmo_debug_set_wait_limit_ns
// lowered it to make them expire; 0 makes them expire at once, whatever the barrier's state,
// so that a test does not depend on how fast a copy or an MMA lands. The waits that drain
// copies and MMAs in flight after an expiry, before shared and tensor memory are released,
// always use WAIT_NS.
static __device__ unsigned long long g_wait_limit_ns = WAIT_NS;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) { return mbar_wait_for(bar, parity, WAIT_NS); }
__device__ __forceinline__ bool mbar_wait_reported(uint32_t bar, uint32_t parity) {
    const unsigned long long lim = *(volatile unsigned long long*)&g_wait_limit_ns;
    return lim != 0 && mbar_wait_for(bar, parity, lim);
}

// global -> shared bulk copy, completion counted on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 512 B, version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(128u >> 4) << 16;
    d |= (uint64_t)(512u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t idesc_bf16(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 consecutive fp32 accumulator columns of this thread's lane (load and wait in one asm
// statement, so no use of the registers can be scheduled before the wait)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (one load, one wait)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 64 consecutive FP32 columns of this warp's 32 TMEM lanes (one load, one wait)
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
        "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

template <int N>
struct TmemCols {
    static constexpr uint32_t value = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
};

// One 128-row tile of D = A . B^T over column chunks [c0, c1) of K; epi(row_in_tile, col0,
// v[16]) is called by every thread for its lane, 16 columns at a time. A and B point at the
// packed operands (A already offset to the row tile); kA = K / 32 chunks per A row tile.
// Returns false (after recording *err) when a wait expired.
template <int N, class Epi>
__device__ bool gemm_tile(const uint8_t* __restrict__ A, const uint8_t* __restrict__ B, int kA, int c0, int c1,
                          uint8_t* smem, int* err, Epi& epi) {
    static_assert(N % 16 == 0 && N >= 16 && N <= 128, "N must be a multiple of 16 in [16, 128]");
    constexpr uint32_t B_BYTES = (uint32_t)N * 64;   // N rows x 32 columns
    constexpr uint32_t STAGE_BYTES = CHUNK_BYTES + ((B_BYTES + 1023) / 1024) * 1024;
    constexpr uint32_t NCOLS = TmemCols<N>::value;
    __shared__ __align__(8) uint64_t bars[2 * STAGES + 1];
    __shared__ uint32_t tmem_slot;
    __shared__ int fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[STAGES]), done = smem_u32(&bars[2 * STAGES]);
    const uint32_t sbase = smem_u32(smem);
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2 * STAGES + 1; ++s) mbar_init(smem_u32(&bars[s]), 1);
        mbar_init_fence();
        fail = 0;
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), NCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const int nk = c1 - c0;
    if (threadIdx.x == 0) {
        int code = TC_OK;
        int issued = 0;   // chunks whose copies were issued
        auto load = [&](int i) {
            const int s = i % STAGES;
            const uint32_t dst = sbase + (uint32_t)s * STAGE_BYTES;
            const uint32_t bar = full0 + 8u * s;
            mbar_expect_tx(bar, CHUNK_BYTES + B_BYTES);
            bulk_g2s(dst, A + (size_t)(c0 + i) * CHUNK_BYTES, CHUNK_BYTES, bar);
            bulk_g2s(dst + CHUNK_BYTES, B + (size_t)(c0 + i) * CHUNK_BYTES, B_BYTES, bar);
            ++issued;
        };
        const uint32_t idesc = idesc_bf16(N);
        for (int i = 0; i < nk && i < STAGES; ++i) load(i);
        int consumed = 0;
        for (int i = 0; i < nk; ++i) {
            const int s = i % STAGES;
            const uint32_t ph = (uint32_t)(i / STAGES) & 1u;
            if (!mbar_wait_reported(full0 + 8u * s, ph)) { code = TC_TIMEOUT_LOAD; break; }
            ++consumed;
            tc_fence_after();
            const uint32_t a = sbase + (uint32_t)s * STAGE_BYTES, b = a + CHUNK_BYTES;
#pragma unroll
            for (int j = 0; j < 2; ++j)
                mma_bf16(tmem, smem_desc(a + 256u * j), smem_desc(b + 256u * j), idesc, (i > 0 || j > 0) ? 1u : 0u);
            mma_commit(empty0 + 8u * s);
            if (i + STAGES < nk) {
                if (!mbar_wait_reported(empty0 + 8u * s, ph)) { code = TC_TIMEOUT_MMA; break; }
                load(i + STAGES);
            }
        }
        mma_commit(done);
        if (code != TC_OK) {
            // let the copies already issued land before the shared memory goes away
            for (int i = consumed; i < issued; ++i) (void)mbar_wait(full0 + 8u * (i % STAGES), (uint32_t)(i / STAGES) & 1u);
            atomicExch(err, code);
            fail = 1;
        }
    }
    __syncwarp();
    // every thread waits for the accumulator (all MMAs committed above)
    bool ok = mbar_wait(done, 0);
    if (!ok && lane == 0) { atomicExch(err, TC_TIMEOUT_DONE); fail = 1; }
    tc_fence_after();
    __syncthreads();
    const bool good = fail == 0;
    if (good) {
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        const int row = warp * 32 + lane;
#pragma unroll 1
        for (int c = 0; c < N; c += 16) {
            float v[16];
            tmem_ld16(lane_addr + (uint32_t)c, v);
            epi(row, c, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, NCOLS);
    }
    return good;
}

template <int N>
constexpr size_t gemm_smem_bytes() {
    return (size_t)STAGES * (CHUNK_BYTES + (((size_t)N * 64 + 1023) / 1024) * 1024) + 1024;
}

}  // namespace tc
}  // namespace vsdmo
