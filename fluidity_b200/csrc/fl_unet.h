// Learned block preconditioner: parameter layout, training cache layout and launchers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fl_internal.cuh"

namespace fl {

constexpr int kUNetLayers = 10;  // e1a e1b e2a e2b bt u2 d2 u1 d1 out

struct UNetLayout {
  int cin[kUNetLayers];
  int cout[kUNetLayers];
  int taps[kUNetLayers];          // 27 (3x3x3) or 1 (1x1)
  long long offset[kUNetLayers];  // weight offset (floats)
  long long bias[kUNetLayers];    // bias offset (floats)
  long long total;
};

// Offsets (floats) of each activation / scratch tensor in a training cache of `batch` items.
struct UNetCache {
  long long x, e1a, s1, p1, e2a, s2, p2, bt, c2, u2, d2, c1, u1, d1, y;
  long long activations;
  long long g8a, g8b, g8c, g4a, g4b, g4c, g2a, g2b;
  long long total;
};

UNetLayout unet_layout();
// Opts the convolution kernels into large dynamic shared memory (call before any stream capture).
void configure_unet_kernels();
UNetCache unet_cache_layout(int batch);

// Scratch of the tensor-core training convolutions (fl_unet_train_tc.cu): the
// cuBLAS handle, the BF16 im2col, packed-weight and gradient-row operands and
// the FP32 GEMM result, sized for a batch of up to max_batch items.
struct UNetTcTrain {
  void* handle = nullptr;  // cublasHandle_t
  __nv_bfloat16* col = nullptr;
  __nv_bfloat16* w = nullptr;
  __nv_bfloat16* g = nullptr;
  float* out = nullptr;
  float* part = nullptr;  // bias-gradient partial sums, 64 x 32
};
// Largest batch of the tensor-core path: its operands (at most 512 x 432 BF16
// per item) stay below 2^31 elements, so every index is 32-bit.
constexpr int kUNetTcMaxBatch = 8192;
cudaError_t unet_tc_train_create(int max_batch, UNetTcTrain* t);
void unet_tc_train_destroy(UNetTcTrain* t);
template <int S, bool VALID>
cudaError_t conv3_fwd_tc(UNetTcTrain& t, const float* in, int cin, const float* w, const float* bias, int cout,
                         float* out, int batch, int relu, cudaStream_t s);
template <int S>
cudaError_t conv3_bwd_data_tc(UNetTcTrain& t, const float* g, int cout, const float* w, int cin, const float* act,
                              float* din, int batch, cudaStream_t s);
template <int S, bool VALID>
cudaError_t conv3_bwd_weight_tc(UNetTcTrain& t, const float* in, int cin, const float* g, int cout, int batch,
                                float* dw, float* db, cudaStream_t s);

// tc == nullptr: the FP32 SIMT convolutions; otherwise the 3x3x3 convolutions
// run as BF16 tensor-core GEMMs with FP32 accumulation.
cudaError_t unet_forward(const float* params, const float* x, int batch, float* cache, float* y, cudaStream_t s,
                         UNetTcTrain* tc = nullptr);
cudaError_t unet_backward(const float* params, float* cache, const float* grad_y, int batch, float* grad_params,
                          cudaStream_t s, UNetTcTrain* tc = nullptr);
cudaError_t unet_masked_mse(const float* y, const float* target, const float* mask, int batch, int relative,
                            float* loss, float* grad, cudaStream_t s);
cudaError_t unet_block_residual_loss(const float* y, const float* x, int batch, float* loss, float* grad,
                                     cudaStream_t s);
cudaError_t adam_step(float* p, const float* g, float* m, float* v, long long n, int step, float lr, float b1,
                      float b2, float eps, cudaStream_t s);
cudaError_t unet_init_params(float* p, unsigned long long seed, cudaStream_t s);

// Solver-side data movement (level-0 vectors in the red-black block layout, cell types natural).
cudaError_t unet_gather(const GridView& g, const float* r_rb, const unsigned char* type, const int* blocks, int count,
                        float* inputs, float* scale, cudaStream_t s);
cudaError_t unet_targets(const GridView& g, const double* p_star, const double* p_k, const unsigned char* type,
                         const int* blocks, int count, const float* scale, float* targets, float* masks,
                         cudaStream_t s);
template <typename T>
cudaError_t unet_scatter(int nb, const float* y, const float* scale, const unsigned char* type, T* z, bool rb,
                         cudaStream_t s);
cudaError_t unet_block_has_fluid(int nb, const unsigned char* type, int* flags, cudaStream_t s);

// Tensor-core inference: per-block offsets (in 16-byte rows) of the BF16
// activation columns, stored tensor-major ([tensor][block][rows]); the packed
// BF16 conv weights (e1a e1b e2a e2b bt d2 d1) and their element offsets.
struct UNetTcLayout {
  long long x, t8, s1, p1, e2a, s2, p2, u2, d2;
  long long rows_per_block;
  long long bt_floats_per_block;
  long long w_off[7];
  long long w_total;
};
UNetTcLayout unet_tc_layout();
cudaError_t unet_tc_pack(const float* params, __nv_bfloat16* packed, cudaStream_t s);
// z = s * U(r / s) on fluid cells of every active block (r, z: level-0 layout).
// `act` holds rows_per_block * cap 16-byte rows (cap >= active blocks) and must
// be zeroed once when allocated: the pads of every column are read as zeros and
// never written.
template <typename T>
cudaError_t unet_tc_apply(const GridView& g, const float* params, const __nv_bfloat16* packed, uint4* act,
                          long long cap, float* bt, float* scale, const unsigned char* type, const float* r_rb, T* z,
                          int* error, int sms, cudaStream_t s, bool accumulate = false);

}  // namespace fl
