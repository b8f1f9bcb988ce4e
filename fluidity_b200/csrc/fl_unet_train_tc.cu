// Training convolutions of the learned preconditioner on tensor cores.
//
// Each 3x3x3 convolution of training (forward, data gradient, weight gradient)
// is one BF16 GEMM with FP32 accumulation, issued through cuBLAS (a plain
// library GEMM: on sm_100 it runs on the tcgen05 tensor cores), between
// memory-bound kernels of this file that form and consume its operands:
//
//   forward     Y[m][co]   = sum_k A[m][k] W[co][k]          (A = im2col of the input)
//   data grad   D[m][k]    = sum_co G[m][co] W[co][k]        (then col2im, ReLU mask)
//   weight grad dW[co][k]  = sum_m  G[m][co] A[m][k]         (bias gradient summed apart)
//
// with m = item * S^3 + output cell, k = ci * 27 + tap (dz, dy, dx) padded
// with zeros to Kp (a multiple of 16), G the output gradient. Operands A, W
// and G are BF16 (rounded from the FP32 master values); sums and every result
// are FP32, as are the parameters and Adam's state. The SIMT FP32 kernels of
// fl_unet.cu remain the exact reference path.
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fl_internal.cuh"
#include "fl_kernels.h"
#include "fl_unet.h"

#include <algorithm>

namespace fl {
namespace {

constexpr int kT = 256;

unsigned grid_of(long long n) { return (unsigned)std::min<long long>((n + kT - 1) / kT, 1 << 20); }

int padded_k(int cin) { return (cin * 27 + 15) / 16 * 16; }

// A[m][k] = in[b][ci][cell(o) + tap - pad] (0 outside, 0 for k >= 27 cin).
template <int S, bool VALID>
__global__ void k_im2col(const float* __restrict__ in, int cin, int kp, long long total,
                         __nv_bfloat16* __restrict__ a) {
  constexpr int S3 = S * S * S;
  constexpr int E = VALID ? S + 2 : S, E3 = E * E * E;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int k = (int)(i % kp);
    const long long m = i / kp;
    float v = 0.0f;
    if (k < cin * 27) {
      const int ci = k / 27, tap = k % 27;
      const int b = (int)(m / S3), o = (int)(m % S3);
      int z = o / (S * S) + tap / 9, y = (o / S) % S + (tap / 3) % 3, x = o % S + tap % 3;
      if (!VALID) {
        z -= 1;
        y -= 1;
        x -= 1;
      }
      if (VALID || (z >= 0 && z < S && y >= 0 && y < S && x >= 0 && x < S))
        v = in[((size_t)b * cin + ci) * E3 + (z * E + y) * E + x];
    }
    a[i] = __float2bfloat16_rn(v);
  }
}

// W[co][k] in BF16 from the FP32 weights [co][ci][27], zero padded to Kp.
__global__ void k_pack_weights(const float* __restrict__ w, int cout, int k27, int kp, __nv_bfloat16* __restrict__ out) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= cout * kp) return;
  const int co = i / kp, k = i % kp;
  out[i] = __float2bfloat16_rn(k < k27 ? w[(size_t)co * k27 + k] : 0.0f);
}

// out[b][co][o] = act(Y[m][co] + bias[co]).
__global__ void k_fwd_epilogue(const float* __restrict__ y, const float* __restrict__ bias, int cout, int s3,
                               long long total, int relu, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int o = (int)(i % s3);
    const int co = (int)((i / s3) % cout);
    const long long b = i / ((long long)s3 * cout);
    const float v = y[(b * s3 + o) * cout + co] + bias[co];
    out[i] = relu ? fmaxf(v, 0.0f) : v;
  }
}

// G[m][co] in BF16 from the FP32 gradient [b][co][o].
__global__ void k_grad_rows(const float* __restrict__ g, int cout, int s3, long long total,
                            __nv_bfloat16* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int co = (int)(i % cout);
    const long long m = i / cout;
    const long long b = m / s3;
    const int o = (int)(m % s3);
    out[i] = __float2bfloat16_rn(g[(b * cout + co) * s3 + o]);
  }
}

// din[b][ci][cell] = sum over taps (fixed order) of D[(b, cell - tap + pad)][ci * 27 + tap],
// times (act > 0) when act is given.
template <int S>
__global__ void k_col2im(const float* __restrict__ d, int cin, int kp, const float* __restrict__ act, long long total,
                         float* __restrict__ din) {
  constexpr int S3 = S * S * S;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    if (act != nullptr && !(act[i] > 0.0f)) {
      din[i] = 0.0f;
      continue;
    }
    const int cell = (int)(i % S3);
    const int ci = (int)((i / S3) % cin);
    const long long b = i / ((long long)S3 * cin);
    const int z = cell / (S * S), y = (cell / S) % S, x = cell % S;
    float acc = 0.0f;
    for (int tap = 0; tap < 27; ++tap) {
      const int oz = z - tap / 9 + 1, oy = y - (tap / 3) % 3 + 1, ox = x - tap % 3 + 1;
      if (oz < 0 || oz >= S || oy < 0 || oy >= S || ox < 0 || ox >= S) continue;
      acc += d[(b * S3 + (oz * S + oy) * S + ox) * kp + ci * 27 + tap];
    }
    din[i] = acc;
  }
}

// dw[co][k] (k < 27 cin) from the GEMM's [co][Kp] rows.
__global__ void k_unpack_dw(const float* __restrict__ c, int cout, int k27, int kp, float* __restrict__ dw) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= cout * k27) return;
  dw[i] = c[(size_t)(i / k27) * kp + i % k27];
}

// db[co] = sum_b sum_o g[b][co][o], one CTA per co, fixed order.
__global__ void __launch_bounds__(kT) k_bias_grad(const float* __restrict__ g, int cout, int s3, int batch,
                                                  float* __restrict__ db) {
  __shared__ float red[kT / 32];
  const int co = blockIdx.x;
  float acc = 0.0f;
  for (int i = threadIdx.x; i < batch * s3; i += kT) acc += g[((size_t)(i / s3) * cout + co) * s3 + i % s3];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (int k = 0; k < kT / 32; ++k) s += red[k];
    db[co] = s;
  }
}

cudaError_t gemm(UNetTcTrain& t, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                 const __nv_bfloat16* a, int lda, const __nv_bfloat16* b, int ldb, float* c, int ldc, cudaStream_t s) {
  const float one = 1.0f, zero = 0.0f;
  cublasHandle_t h = static_cast<cublasHandle_t>(t.handle);
  if (cublasSetStream(h, s) != CUBLAS_STATUS_SUCCESS) return cudaErrorUnknown;
  ++g_library_launches;
  const cublasStatus_t st = cublasGemmEx(h, ta, tb, m, n, k, &one, a, CUDA_R_16BF, lda, b, CUDA_R_16BF, ldb,
                                         &zero, c, CUDA_R_32F, ldc, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
  return st == CUBLAS_STATUS_SUCCESS ? cudaSuccess : cudaErrorUnknown;
}

}  // namespace

cudaError_t unet_tc_train_create(int max_batch, UNetTcTrain* t) {
  *t = UNetTcTrain{};
  const long long b = max_batch;
  // largest operands: the 8^3 layers with 16 input channels (Kp = 432)
  const long long col = b * 512 * padded_k(16);
  const long long rows = b * 512 * 64;
  const long long out = col;  // the data-gradient GEMM's [M][Kp] is the largest result
  cublasHandle_t h = nullptr;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return cudaErrorUnknown;
  t->handle = h;
  if (cudaMalloc(&t->col, sizeof(__nv_bfloat16) * col) != cudaSuccess ||
      cudaMalloc(&t->w, sizeof(__nv_bfloat16) * 64 * padded_k(64)) != cudaSuccess ||
      cudaMalloc(&t->g, sizeof(__nv_bfloat16) * rows) != cudaSuccess ||
      cudaMalloc(&t->out, sizeof(float) * out) != cudaSuccess) {
    cudaGetLastError();
    unet_tc_train_destroy(t);
    return cudaErrorMemoryAllocation;
  }
  return cudaSuccess;
}

void unet_tc_train_destroy(UNetTcTrain* t) {
  if (t->handle) cublasDestroy(static_cast<cublasHandle_t>(t->handle));
  cudaFree(t->col);
  cudaFree(t->w);
  cudaFree(t->g);
  cudaFree(t->out);
  *t = UNetTcTrain{};
}

template <int S, bool VALID>
cudaError_t conv3_fwd_tc(UNetTcTrain& t, const float* in, int cin, const float* w, const float* bias, int cout,
                         float* out, int batch, int relu, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cin), m = batch * S3;
  g_kernel_launches += 3;
  k_im2col<S, VALID><<<grid_of((long long)m * kp), kT, 0, s>>>(in, cin, kp, (long long)m * kp, t.col);
  k_pack_weights<<<(cout * kp + kT - 1) / kT, kT, 0, s>>>(w, cout, cin * 27, kp, t.w);
  cudaError_t e = gemm(t, CUBLAS_OP_T, CUBLAS_OP_N, cout, m, kp, t.w, kp, t.col, kp, t.out, cout, s);
  if (e != cudaSuccess) return e;
  k_fwd_epilogue<<<grid_of((long long)m * cout), kT, 0, s>>>(t.out, bias, cout, S3, (long long)m * cout, relu, out);
  return cudaGetLastError();
}

template <int S>
cudaError_t conv3_bwd_data_tc(UNetTcTrain& t, const float* g, int cout, const float* w, int cin, const float* act,
                              float* din, int batch, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cin), m = batch * S3;
  g_kernel_launches += 3;
  k_grad_rows<<<grid_of((long long)m * cout), kT, 0, s>>>(g, cout, S3, (long long)m * cout, t.g);
  k_pack_weights<<<(cout * kp + kT - 1) / kT, kT, 0, s>>>(w, cout, cin * 27, kp, t.w);
  cudaError_t e = gemm(t, CUBLAS_OP_N, CUBLAS_OP_N, kp, m, cout, t.w, kp, t.g, cout, t.out, kp, s);
  if (e != cudaSuccess) return e;
  k_col2im<S><<<grid_of((long long)batch * cin * S3), kT, 0, s>>>(t.out, cin, kp, act, (long long)batch * cin * S3,
                                                                    din);
  return cudaGetLastError();
}

template <int S, bool VALID>
cudaError_t conv3_bwd_weight_tc(UNetTcTrain& t, const float* in, int cin, const float* g, int cout, int batch,
                                float* dw, float* db, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cin), m = batch * S3;
  g_kernel_launches += 4;
  k_im2col<S, VALID><<<grid_of((long long)m * kp), kT, 0, s>>>(in, cin, kp, (long long)m * kp, t.col);
  k_grad_rows<<<grid_of((long long)m * cout), kT, 0, s>>>(g, cout, S3, (long long)m * cout, t.g);
  cudaError_t e = gemm(t, CUBLAS_OP_N, CUBLAS_OP_T, kp, cout, m, t.col, kp, t.g, cout, t.out, kp, s);
  if (e != cudaSuccess) return e;
  k_unpack_dw<<<(cout * cin * 27 + kT - 1) / kT, kT, 0, s>>>(t.out, cout, cin * 27, kp, dw);
  k_bias_grad<<<cout, kT, 0, s>>>(g, cout, S3, batch, db);
  return cudaGetLastError();
}

template cudaError_t conv3_fwd_tc<8, true>(UNetTcTrain&, const float*, int, const float*, const float*, int, float*,
                                           int, int, cudaStream_t);
template cudaError_t conv3_fwd_tc<8, false>(UNetTcTrain&, const float*, int, const float*, const float*, int, float*,
                                            int, int, cudaStream_t);
template cudaError_t conv3_fwd_tc<4, false>(UNetTcTrain&, const float*, int, const float*, const float*, int, float*,
                                            int, int, cudaStream_t);
template cudaError_t conv3_fwd_tc<2, false>(UNetTcTrain&, const float*, int, const float*, const float*, int, float*,
                                            int, int, cudaStream_t);
template cudaError_t conv3_bwd_data_tc<8>(UNetTcTrain&, const float*, int, const float*, int, const float*, float*,
                                          int, cudaStream_t);
template cudaError_t conv3_bwd_data_tc<4>(UNetTcTrain&, const float*, int, const float*, int, const float*, float*,
                                          int, cudaStream_t);
template cudaError_t conv3_bwd_data_tc<2>(UNetTcTrain&, const float*, int, const float*, int, const float*, float*,
                                          int, cudaStream_t);
template cudaError_t conv3_bwd_weight_tc<8, true>(UNetTcTrain&, const float*, int, const float*, int, int, float*,
                                                  float*, cudaStream_t);
template cudaError_t conv3_bwd_weight_tc<8, false>(UNetTcTrain&, const float*, int, const float*, int, int, float*,
                                                   float*, cudaStream_t);
template cudaError_t conv3_bwd_weight_tc<4, false>(UNetTcTrain&, const float*, int, const float*, int, int, float*,
                                                   float*, cudaStream_t);
template cudaError_t conv3_bwd_weight_tc<2, false>(UNetTcTrain&, const float*, int, const float*, int, int, float*,
                                                   float*, cudaStream_t);

}  // namespace fl
