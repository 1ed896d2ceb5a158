// The surrogate network of the control-variate estimator (see mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace scp3 {
namespace mlp {

struct Net {
    int n_in = 0, hid = 0, kin = 0, max_batch = 0;
    int in[4] = {0, 0, 0, 0}, out[4] = {0, 0, 0, 0}, inpad[4] = {0, 0, 0, 0};
    // FP32 masters, gradients, Adam moments (first n, then second n), BF16 copies
    float *w[4] = {}, *b[4] = {}, *gw[4] = {}, *gb[4] = {}, *mw[4] = {}, *mb[4] = {};
    __nv_bfloat16* wb[4] = {};
    // activations of one batch
    __nv_bfloat16* X = nullptr;
    float* Z[3] = {};
    __nv_bfloat16* H[3] = {};
    float *dA = nullptr, *dB = nullptr, *ybuf = nullptr, *dy = nullptr, *loss = nullptr;
    float out_scale = 1.0f, out_shift = 0.0f;   // y = raw * scale + shift
    int64_t step = 0;

    int alloc(int n_in, int hidden, int max_batch);
    void free_all();
    int sync_bf16(cudaStream_t s);
    int forward(const float* q, int M, float* y, cudaStream_t s);
    // Inference on a caller's workspace (X: Mp x kin, Ha/Hb: Mp x hid, BF16, Mp = M rounded
    // up to 64): reads only the weights, so several builds may run it at once on their streams.
    int infer(const float* q, int M, float* y, cudaStream_t s, __nv_bfloat16* X, __nv_bfloat16* Ha,
              __nv_bfloat16* Hb) const;
    size_t infer_workspace(int M) const;   // BF16 elements for X + Ha + Hb
    int apply_output(float* y, int M, cudaStream_t s);
    int backward(const float* q, const float* t, int M, cudaStream_t s, float* loss_out);
    int adam(float lr, cudaStream_t s);
};

// raw-unit outputs and targets for the loss
__global__ void normalise_kernel(const float* y, const float* t, int M, float scale, float shift, float* yr, float* tr);

}  // namespace mlp
}  // namespace scp3
