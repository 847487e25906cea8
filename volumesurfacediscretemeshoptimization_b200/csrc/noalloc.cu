// noalloc.cu -- a quality reduction that allocates no device memory.
//
// Callers that own their device memory up front (an engine that hands the optimiser a fixed
// arena and forbids further cudaMalloc), that run where cudaMalloc / cudaFree are not allowed
// or would synchronise the device at a bad moment, can still ask for the minimum, the sum and
// the count below a threshold of the element qualities of a mesh they hold on the device.
// The reduction's per-block partial results, which the stream-ordered version in
// dmo_kernels.cu keeps in buffers owned by an optimiser handle, live here in one file-scope
// __device__ array of fixed size, so the call needs no allocation at all.
#include "vsdmo_internal.cuh"
#include <cfloat>
#include <mutex>

namespace vsdmo {
namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_BLOCKS = 1024;
constexpr int NA_ELEMS_PER_THREAD = 32;
constexpr long NA_MAX_ELEMS = (long)NA_MAX_BLOCKS * NA_THREADS * NA_ELEMS_PER_THREAD;  // 8,388,608
constexpr int NA_MAX_DEVICES = 64;

// Layout of the scratch array: one done-counter, then per block a float minimum, an int
// count, a double sum and an int count of elements skipped for an index outside the mesh.
constexpr size_t NA_OFF_COUNTER = 0;
constexpr size_t NA_OFF_MIN = 256;
constexpr size_t NA_OFF_BELOW = NA_OFF_MIN + sizeof(float) * NA_MAX_BLOCKS;
constexpr size_t NA_OFF_SUM = NA_OFF_BELOW + sizeof(int) * NA_MAX_BLOCKS;
constexpr size_t NA_OFF_BAD = NA_OFF_SUM + sizeof(double) * NA_MAX_BLOCKS;
constexpr size_t NA_SCRATCH_BYTES = NA_OFF_BAD + sizeof(int) * NA_MAX_BLOCKS;  // 20,736 bytes

// Shared by every call on a device and kept for the life of the process. In host code this
// name is only a host-side stand-in; kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

std::mutex g_setup_mutex;
void* g_scratch_ptr[NA_MAX_DEVICES] = {};

__device__ __forceinline__ float na_q_tet(const float* X, const int* t) {
    const float* p0 = X + 3 * (long)t[0];
    const float* p1 = X + 3 * (long)t[1];
    const float* p2 = X + 3 * (long)t[2];
    const float* p3 = X + 3 * (long)t[3];
    const float e0x = p1[0] - p0[0], e0y = p1[1] - p0[1], e0z = p1[2] - p0[2];
    const float e1x = p2[0] - p0[0], e1y = p2[1] - p0[1], e1z = p2[2] - p0[2];
    const float e2x = p3[0] - p0[0], e2y = p3[1] - p0[1], e2z = p3[2] - p0[2];
    const float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
    const float volume = (1.f / 6.f) * ((e0x * cx + e0y * cy) + e0z * cz);
    if (volume < 0.f) return volume;
    const float mu = cbrtf(volume * volume);
    const float e3x = p2[0] - p1[0], e3y = p2[1] - p1[1], e3z = p2[2] - p1[2];
    const float e4x = p3[0] - p1[0], e4y = p3[1] - p1[1], e4z = p3[2] - p1[2];
    const float e5x = p3[0] - p2[0], e5y = p3[1] - p2[1], e5z = p3[2] - p2[2];
    float l = 0.f;
    l += (e0x * e0x + e0y * e0y) + e0z * e0z;
    l += (e1x * e1x + e1y * e1y) + e1z * e1z;
    l += (e2x * e2x + e2y * e2y) + e2z * e2z;
    l += (e3x * e3x + e3y * e3y) + e3z * e3z;
    l += (e4x * e4x + e4y * e4y) + e4z * e4z;
    l += (e5x * e5x + e5y * e5y) + e5z * e5z;
    const float cbrtf9 = 2.0800838230519f;
    return ((12.f * cbrtf9) * mu) / l;
}

__device__ __forceinline__ float na_q_tri2d(const float* X, const int* t) {
    const float* p0 = X + 3 * (long)t[0];
    const float* p1 = X + 3 * (long)t[1];
    const float* p2 = X + 3 * (long)t[2];
    const float e0x = p1[0] - p0[0], e0y = p1[1] - p0[1];
    const float e1x = p2[0] - p1[0], e1y = p2[1] - p1[1];
    const float e2x = p0[0] - p2[0], e2y = p0[1] - p2[1];
    const float l = ((e0x * e0x + e0y * e0y) + (e1x * e1x + e1y * e1y)) + (e2x * e2x + e2y * e2y);
    const float area = e0x * e1y - e0y * e1x;
    if (area < 0.f) return area;
    return ((2.f * sqrtf(3.f)) * area) / l;
}

// Elements with an index outside [0, nV) are skipped before any of their corners is loaded
// and counted; when there is one, the results are *out_below = -1 and NaN minimum and sum.
__global__ void __launch_bounds__(NA_THREADS)
k_quality_reduce_noalloc(const float* __restrict__ X, int nV, const int* __restrict__ el, int k, long nE,
                         float threshold, unsigned char* scratch, float* out_min, double* out_sum, int* out_below) {
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + NA_OFF_COUNTER);
    float* pmin = reinterpret_cast<float*>(scratch + NA_OFF_MIN);
    int* pbelow = reinterpret_cast<int*>(scratch + NA_OFF_BELOW);
    double* psum = reinterpret_cast<double*>(scratch + NA_OFF_SUM);
    int* pbad = reinterpret_cast<int*>(scratch + NA_OFF_BAD);
    __shared__ float smin[NA_THREADS / 32];
    __shared__ int sbelow[NA_THREADS / 32];
    __shared__ double ssum[NA_THREADS / 32];
    __shared__ int sbad[NA_THREADS / 32];
    __shared__ bool last;
    float mn = FLT_MAX;
    double sm = 0.0;
    int below = 0, bad = 0;
    for (long e = (long)blockIdx.x * NA_THREADS + threadIdx.x; e < nE; e += (long)gridDim.x * NA_THREADS) {
        const int* t = el + (long)k * e;
        bool inside = true;
        for (int c = 0; c < k; ++c) inside &= (unsigned)t[c] < (unsigned)nV;
        if (!inside) { ++bad; continue; }
        const float q = k == 4 ? na_q_tet(X, t) : na_q_tri2d(X, t);
        mn = fminf(mn, q);
        sm += (double)q;
        below += q < threshold ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        sm += __shfl_xor_sync(0xffffffffu, sm, o);
        below += __shfl_xor_sync(0xffffffffu, below, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { smin[w] = mn; ssum[w] = sm; sbelow[w] = below; sbad[w] = bad; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = smin[0]; double s = ssum[0]; int b = sbelow[0], x = sbad[0];
        for (int i = 1; i < NA_THREADS / 32; ++i) { a = fminf(a, smin[i]); s += ssum[i]; b += sbelow[i]; x += sbad[i]; }
        pmin[blockIdx.x] = a; psum[blockIdx.x] = s; pbelow[blockIdx.x] = b; pbad[blockIdx.x] = x;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        float a = FLT_MAX; double s = 0.0; int b = 0, x = 0;
        for (unsigned i = 0; i < gridDim.x; ++i) {
            a = fminf(a, ((volatile float*)pmin)[i]);
            s += ((volatile double*)psum)[i];
            b += ((volatile int*)pbelow)[i];
            x += ((volatile int*)pbad)[i];
        }
        *out_min = x ? __int_as_float(0x7fc00000) : a;
        *out_sum = x ? __longlong_as_double(0x7ff8000000000000LL) : s;
        *out_below = x ? -1 : b;
        *counter = 0u;
    }
}

// device (or managed) memory of the current device: the kernel and the scratch lookup run there
bool is_device_memory(const void* p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

long noalloc_max_elements() { return NA_MAX_ELEMS; }

// Device address of the scratch array on the current device, looked up once per device.
void* noalloc_scratch_for_current_device() {
    int dev = 0;
    VSDMO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) throw Error(VSDMO_E_ARG, "device ordinal beyond the no-alloc table");
    std::lock_guard<std::mutex> g(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw Error(VSDMO_E_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

void quality_reduce_noalloc(int k, const float* d_xyz, int n_vertices, const int* d_elems, long n_elems,
                            float threshold, float* d_min, double* d_sum, int* d_below, cudaStream_t s) {
    int dev = 0;
    VSDMO_CUDA(cudaGetDevice(&dev));
    if (!is_device_memory(d_xyz, dev) || !is_device_memory(d_elems, dev) || !is_device_memory(d_min, dev) ||
        !is_device_memory(d_sum, dev) || !is_device_memory(d_below, dev))
        throw Error(VSDMO_E_ARG, "the no-alloc reduction takes device pointers of the current device only");
    unsigned char* scratch = static_cast<unsigned char*>(noalloc_scratch_for_current_device());
    // the counter must start at zero even if an earlier call on this device was cut short
    VSDMO_CUDA(cudaMemsetAsync(scratch + NA_OFF_COUNTER, 0, sizeof(unsigned), s));
    long blocks = (n_elems + (long)NA_THREADS * NA_ELEMS_PER_THREAD - 1) / ((long)NA_THREADS * NA_ELEMS_PER_THREAD);
    if (blocks < 1) blocks = 1;
    if (blocks > NA_MAX_BLOCKS) blocks = NA_MAX_BLOCKS;
    k_quality_reduce_noalloc<<<(unsigned)blocks, NA_THREADS, 0, s>>>(d_xyz, n_vertices, d_elems, k, n_elems,
                                                                     threshold, scratch, d_min, d_sum, d_below);
    VSDMO_CHECK_LAUNCH();
}

}  // namespace vsdmo
