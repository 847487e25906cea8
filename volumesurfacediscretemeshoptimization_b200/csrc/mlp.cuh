// mlp.cuh -- host-side view of the learned proposal network (mlp.cu).
#pragma once
#include "vsdmo_internal.cuh"

namespace vsdmo {
namespace mlp {

constexpr int IN = 96;      // 32 neighbours x 3
constexpr int HID = 128;
constexpr int OUT = 3;
constexpr int OUTP = 16;    // output padded to the smallest tensor-core N
constexpr int MAX_NB = 32;
constexpr int MAX_PARTS = 64;

constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + HID * IN;
constexpr int OFF_W2 = OFF_B1 + HID;
constexpr int OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_W3 = OFF_B2 + HID;
constexpr int OFF_B3 = OFF_W3 + HID * HID;
constexpr int OFF_W4 = OFF_B3 + HID;
constexpr int OFF_B4 = OFF_W4 + OUTP * HID;
constexpr int N_PARAMS = OFF_B4 + OUTP;

// activations and gradients of one batch (rows padded to 128); grows on demand
struct Workspace {
    long cap_rows = 0;
    bool has_train = false;
    DBuf<uint8_t> X, H1, H2, H3;              // packed bf16 [rows x K]
    DBuf<float> Y;                            // [rows x 16]
    DBuf<uint8_t> XT, H1T, H2T, H3T;          // packed bf16 [features x rows]
    DBuf<float> T;                            // targets [rows x 3]
    DBuf<uint8_t> dY, dYT, dZ3, dZ3T, dZ2, dZ2T, dZ1, dZ1T;
    DBuf<float> wsum, loss_rows, loss, parts;
    DBuf<int> idx;
    void ensure(long rows, bool training, cudaStream_t s);
};

struct Model {
    cudaStream_t stream = nullptr;
    DBuf<float> params, grads, adam_m, adam_v;     // flat FP32 [N_PARAMS]
    DBuf<uint8_t> W1p, W2p, W3p, W4p;              // packed bf16 W (forward B operands)
    DBuf<uint8_t> W2Tp, W3Tp, W4Tp;                // packed bf16 W^T (backward B operands)
    DBuf<int> err;
    int step = 0;

    void init(uint64_t seed, cudaStream_t s);
    void set_params(const float* host);
    void get_params(float* host) const;
    void repack();
    // X of w (packed) -> Y of w; training also writes the transposed activations
    void forward(Workspace& w, int n, bool training, cudaStream_t s);
    // gradients of the mean squared error against w.T into grads (B multiple of 128)
    void backward(Workspace& w, int B, cudaStream_t s);
    void adam(float lr, cudaStream_t s);
    // rows idx (or 0..n_valid-1) of feats [*, 96] / targets [*, 3] -> w.X (+ w.XT, w.T)
    void gather(Workspace& w, const float* feats, const float* targets, const int* idx, int B, int n_valid,
                bool training, cudaStream_t s);
    void check(cudaStream_t s);
    // fused inference for tet vertices [v0, v0 + n): ring features from the neighbour table
    // (nb / nbn index vertices from nb_base) -> network -> Y [n x ldy] (first 3 columns)
    void infer_tet(const float4* pos, const int* nb, const int* nbn, int nb_base, int v0, int n, float* Y, int ldy,
                   cudaStream_t s);
};

void prepare(cudaStream_t s);
void debug_gemm(const float* hA, const float* hB, int M, int N, int K, float* hD, cudaStream_t s);
// limit of the reported tensor-core waits on the current device (test-only lowering)
void set_wait_limit(unsigned long long ns);

}  // namespace mlp
}  // namespace vsdmo
