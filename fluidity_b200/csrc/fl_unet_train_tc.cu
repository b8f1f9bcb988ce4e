// Training convolutions of the learned preconditioner on tensor cores.
//
// Each 3x3x3 convolution of training (forward, data gradient, weight gradient)
// is one BF16 GEMM with FP32 accumulation, issued through cuBLAS (a plain
// library GEMM: on sm_100 it runs on the tcgen05 tensor cores), between
// memory-bound kernels of this file that form and consume its operands:
//
//   forward     Y[b][co][o]  = sum_k A[b, o][k] W[co][k]            (A = im2col of the input)
//   data grad   D[b][ci][o]  = sum_k' Ag[b, o][k'] Wf[ci][k']        (Ag = im2col of the output
//                                                                     gradient, Wf the weights
//                                                                     with ci/co swapped and the
//                                                                     taps reversed)
//   weight grad dW[co][k]    = sum_m  Gt[co][m] A[m][k]              (bias gradient summed apart)
//
// with m = item * S^3 + output cell o, k = tap (dz, dy, dx) * C + channel, padded
// with zeros to Kp (a multiple of 16). The stride-1 zero-padded convolution's
// input gradient is itself such a convolution of the output gradient with
// W'[ci][co][tap] = W[co][ci][26 - tap], so it needs no scatter (col2im). The
// forward and data-gradient GEMMs are batched over items and write straight
// into the [item][channel][cell] activations; an in-place pass adds the bias
// and applies the ReLU, or the ReLU mask of the input. Operands are BF16
// (rounded from the FP32 master values); sums and every result are FP32, as
// are the parameters and Adam's state. The SIMT FP32 kernels of fl_unet.cu
// remain the exact path.
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

// A[m][k] = in[b][ci][cell(o) + tap - pad] with k = tap * C + ci (0 outside
// the input, 0 for k >= 27 C). CTA (item, z chunk) stages the ZC + 2 input
// planes its ZC output planes read, zero-padded and channels-last in BF16
// pairs (rows of C/2 + 1 words: odd, so the transposing stores do not
// conflict), then writes its rows of A as contiguous BF16 pairs: a warp's 32
// pairs are whole taps' channel runs, read from shared memory without
// conflicts within a tap.
template <int S, bool VALID, int C>
__global__ void __launch_bounds__(kT) k_im2col(const float* __restrict__ in, __nv_bfloat162* __restrict__ a) {
  constexpr int ZC = 2, E = S + 2, ZL = ZC + 2, PLANE = ZL * E * E;
  constexpr int KP = (C * 27 + 15) / 16 * 16, HALFK = KP / 2, S3 = S * S * S, HC = C / 2, ROW = HC + 1;
  constexpr int EIN = VALID ? S + 2 : S, EIN3 = EIN * EIN * EIN, OFF = VALID ? 0 : 1;
  __shared__ __nv_bfloat162 tile[PLANE * ROW];
  const int b = blockIdx.x / (S / ZC), z0 = (blockIdx.x % (S / ZC)) * ZC;
  const float* src = in + (size_t)b * C * EIN3;
  for (int i = threadIdx.x; i < PLANE * HC; i += kT) {
    const int cell = i % PLANE, cp = i / PLANE;
    const int zp = cell / (E * E), yp = (cell / E) % E, xp = cell % E;
    const int z = z0 + zp - OFF, y = yp - OFF, x = xp - OFF;
    float v0 = 0.0f, v1 = 0.0f;
    if (VALID || (z >= 0 && z < S && y >= 0 && y < S && x >= 0 && x < S)) {
      const float* p = src + (size_t)(2 * cp) * EIN3 + (z * EIN + y) * EIN + x;
      v0 = p[0];
      v1 = p[EIN3];
    }
    tile[cell * ROW + cp] = __floats2bfloat162_rn(v0, v1);
  }
  __syncthreads();
  __nv_bfloat162* out = a + ((size_t)b * S3 + z0 * S * S) * HALFK;
  if constexpr (HC % 4 == 0) {
    // four pairs (one 16-byte store) per thread, all in one tap (KP = 27 C here)
    constexpr int QK = HALFK / 4;
    uint4* out4 = reinterpret_cast<uint4*>(out);
    const unsigned* t32 = reinterpret_cast<const unsigned*>(tile);
    for (int i = threadIdx.x; i < ZC * S * S * QK; i += kT) {
      const int pos = i / QK, kq = i % QK;
      const int tap = (8 * kq) / C, cp = (4 * kq) % HC;
      const int zl = pos / (S * S), y = (pos / S) % S, x = pos % S;
      const unsigned* src4 = t32 + (((zl + tap / 9) * E + y + (tap / 3) % 3) * E + x + tap % 3) * ROW + cp;
      out4[i] = make_uint4(src4[0], src4[1], src4[2], src4[3]);
    }
  } else {
    const __nv_bfloat162 zero = __floats2bfloat162_rn(0.0f, 0.0f);
    for (int i = threadIdx.x; i < ZC * S * S * HALFK; i += kT) {
      const int pos = i / HALFK, kk = i % HALFK;
      const int tap = (2 * kk) / C, cp = kk % HC;
      __nv_bfloat162 v = zero;
      if (tap < 27) {
        const int zl = pos / (S * S), y = (pos / S) % S, x = pos % S;
        v = tile[(((zl + tap / 9) * E + y + (tap / 3) % 3) * E + x + tap % 3) * ROW + cp];
      }
      out[i] = v;
    }
  }
}

template <int S, bool VALID>
cudaError_t im2col(const float* in, int c, int batch, __nv_bfloat16* a, cudaStream_t s) {
  static_assert(S % 2 == 0, "two output planes per CTA");
  auto* a2 = reinterpret_cast<__nv_bfloat162*>(a);
  const unsigned grid = (unsigned)batch * (S / 2);
  // the network's layers: 2 channels (valid, first layer) or 16 at 8^3, 16 or 32 at 4^3, 32 or 64 at 2^3
  if constexpr (S == 8) {
    if (c == 2 && VALID) return k_im2col<S, VALID, 2><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
    if (c == 16) return k_im2col<S, VALID, 16><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
  } else if constexpr (S == 4) {
    if (c == 16) return k_im2col<S, VALID, 16><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
    if (c == 32) return k_im2col<S, VALID, 32><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
  } else {
    if (c == 32) return k_im2col<S, VALID, 32><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
    if (c == 64) return k_im2col<S, VALID, 64><<<grid, kT, 0, s>>>(in, a2), cudaSuccess;
  }
  return cudaErrorInvalidValue;
}

// W[co][tap * cin + ci] = w[co][ci][tap] in BF16, zero padded to Kp.
__global__ void k_pack_weights(const float* __restrict__ w, int cout, int cin, int kp, __nv_bfloat16* __restrict__ out) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= cout * kp) return;
  const int co = i / kp, k = i % kp;
  out[i] = __float2bfloat16_rn(k < 27 * cin ? w[((size_t)co * cin + k % cin) * 27 + k / cin] : 0.0f);
}

// Wf[ci][tap * cout + co] = W[co][ci][26 - tap] in BF16, zero padded to Kp(cout).
__global__ void k_pack_weights_flipped(const float* __restrict__ w, int cout, int cin, int kp,
                                       __nv_bfloat16* __restrict__ out) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= cin * kp) return;
  const int ci = i / kp, k = i % kp;
  float v = 0.0f;
  if (k < cout * 27) v = w[((size_t)(k % cout) * cin + ci) * 27 + 26 - k / cout];
  out[i] = __float2bfloat16_rn(v);
}

// In place: y[b][co][o] = act(y + bias[co]).
__global__ void k_bias_act(float* __restrict__ y, const float* __restrict__ bias, int cout, int s3, unsigned total,
                           int relu) {
  for (unsigned i = blockIdx.x * kT + threadIdx.x; i < total; i += gridDim.x * kT) {
    const float v = y[i] + bias[(i / s3) % cout];
    y[i] = relu ? fmaxf(v, 0.0f) : v;
  }
}

// In place: d = 0 where the layer's input activation is not positive.
__global__ void k_relu_mask(float* __restrict__ d, const float* __restrict__ act, unsigned total) {
  for (unsigned i = blockIdx.x * kT + threadIdx.x; i < total; i += gridDim.x * kT)
    if (!(act[i] > 0.0f)) d[i] = 0.0f;
}

// Gt[co][m] in BF16 from the FP32 gradient [b][co][o] (m = b * s3 + o).
__global__ void k_grad_cols(const float* __restrict__ g, int cout, int s3, unsigned m_total, unsigned total,
                            __nv_bfloat16* __restrict__ out) {
  for (unsigned i = blockIdx.x * kT + threadIdx.x; i < total; i += gridDim.x * kT) {
    const unsigned co = i / m_total, m = i % m_total;
    out[i] = __float2bfloat16_rn(g[((m / s3) * cout + co) * s3 + m % s3]);
  }
}

// dw[co][ci][tap] from the GEMM's [co][Kp] rows (k = tap * cin + ci).
__global__ void k_unpack_dw(const float* __restrict__ c, int cout, int cin, int kp, float* __restrict__ dw) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= cout * cin * 27) return;
  const int co = i / (cin * 27), r = i % (cin * 27);
  dw[i] = c[(size_t)co * kp + (r % 27) * cin + r / 27];
}

// db[co] = sum_b sum_o g[b][co][o] in a fixed order: CTA (co, c) sums chunk c
// of the items into part[co][c], then one thread per co adds the chunks.
constexpr int kBiasChunks = 32;

__global__ void __launch_bounds__(kT) k_bias_partial(const float* __restrict__ g, int cout, int s3_log2, int batch,
                                                     float* __restrict__ part) {
  __shared__ float red[kT / 32];
  const int co = blockIdx.x, c = blockIdx.y;
  const int lo = (int)((long long)batch * c / kBiasChunks), hi = (int)((long long)batch * (c + 1) / kBiasChunks);
  const int s3 = 1 << s3_log2;
  float acc = 0.0f;
  for (int i = threadIdx.x; i < (hi - lo) * s3; i += kT)
    acc += g[((size_t)(lo + (i >> s3_log2)) * cout + co) * s3 + (i & (s3 - 1))];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float sum = 0.0f;
    for (int k = 0; k < kT / 32; ++k) sum += red[k];
    part[co * kBiasChunks + c] = sum;
  }
}

__global__ void k_bias_final(const float* __restrict__ part, int cout, float* __restrict__ db) {
  const int co = threadIdx.x;
  if (co >= cout) return;
  float sum = 0.0f;
  for (int c = 0; c < kBiasChunks; ++c) sum += part[co * kBiasChunks + c];
  db[co] = sum;
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

// Per item b: C_b[o + n * s3] = sum_k A[(b * s3 + o) * kp + k] B[n * kp + k], C_b = c + b * n_count * s3,
// i.e. the [item][channel][cell] layout of the activations; B (the packed weights) is shared.
cudaError_t gemm_items(UNetTcTrain& t, int s3, int n_count, int kp, const __nv_bfloat16* a, const __nv_bfloat16* b,
                       float* c, int items, cudaStream_t s) {
  const float one = 1.0f, zero = 0.0f;
  cublasHandle_t h = static_cast<cublasHandle_t>(t.handle);
  if (cublasSetStream(h, s) != CUBLAS_STATUS_SUCCESS) return cudaErrorUnknown;
  ++g_library_launches;
  const cublasStatus_t st = cublasGemmStridedBatchedEx(
      h, CUBLAS_OP_T, CUBLAS_OP_N, s3, n_count, kp, &one, a, CUDA_R_16BF, kp, (long long)s3 * kp, b, CUDA_R_16BF, kp,
      0, &zero, c, CUDA_R_32F, s3, (long long)n_count * s3, items, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
  return st == CUBLAS_STATUS_SUCCESS ? cudaSuccess : cudaErrorUnknown;
}

}  // namespace

cudaError_t unet_tc_train_create(int max_batch, UNetTcTrain* t) {
  *t = UNetTcTrain{};
  if (max_batch <= 0 || max_batch > kUNetTcMaxBatch) return cudaErrorInvalidValue;
  const long long b = max_batch;
  // Largest im2col operand: the 8^3 layers with 16 channels on the gathered
  // side (Kp = 432); the 4^3 and 2^3 layers need at most a quarter of that.
  const long long col = b * 512 * padded_k(16);
  const long long cols = b * 512 * 16;  // Gt: cout x M, largest at 8^3
  // packed weights and the weight-gradient GEMM's [co][Kp] result: at most 64 x Kp(64)
  const long long wmax = 64LL * padded_k(64);
  cublasHandle_t h = nullptr;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return cudaErrorUnknown;
  t->handle = h;
  if (cudaMalloc(&t->col, sizeof(__nv_bfloat16) * col) != cudaSuccess ||
      cudaMalloc(&t->w, sizeof(__nv_bfloat16) * wmax) != cudaSuccess ||
      cudaMalloc(&t->g, sizeof(__nv_bfloat16) * cols) != cudaSuccess ||
      cudaMalloc(&t->out, sizeof(float) * wmax) != cudaSuccess ||
      cudaMalloc(&t->part, sizeof(float) * 64 * kBiasChunks) != cudaSuccess) {
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
  cudaFree(t->part);
  *t = UNetTcTrain{};
}

template <int S, bool VALID>
cudaError_t conv3_fwd_tc(UNetTcTrain& t, const float* in, int cin, const float* w, const float* bias, int cout,
                         float* out, int batch, int relu, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cin), m = batch * S3;
  g_kernel_launches += 3;
  cudaError_t e = im2col<S, VALID>(in, cin, batch, t.col, s);
  if (e != cudaSuccess) return e;
  k_pack_weights<<<(cout * kp + kT - 1) / kT, kT, 0, s>>>(w, cout, cin, kp, t.w);
  e = gemm_items(t, S3, cout, kp, t.col, t.w, out, batch, s);
  if (e != cudaSuccess) return e;
  k_bias_act<<<grid_of((long long)m * cout), kT, 0, s>>>(out, bias, cout, S3, (unsigned)m * cout, relu);
  return cudaGetLastError();
}

// The input gradient of a zero-padded stride-1 layer: the output gradient convolved with the
// flipped, transposed weights, then the ReLU mask of the input activation (when given).
template <int S>
cudaError_t conv3_bwd_data_tc(UNetTcTrain& t, const float* g, int cout, const float* w, int cin, const float* act,
                              float* din, int batch, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cout), m = batch * S3;
  g_kernel_launches += act != nullptr ? 3 : 2;
  cudaError_t e = im2col<S, false>(g, cout, batch, t.col, s);
  if (e != cudaSuccess) return e;
  k_pack_weights_flipped<<<(cin * kp + kT - 1) / kT, kT, 0, s>>>(w, cout, cin, kp, t.w);
  e = gemm_items(t, S3, cin, kp, t.col, t.w, din, batch, s);
  if (e != cudaSuccess) return e;
  if (act != nullptr) k_relu_mask<<<grid_of((long long)m * cin), kT, 0, s>>>(din, act, (unsigned)m * cin);
  return cudaGetLastError();
}

template <int S, bool VALID>
cudaError_t conv3_bwd_weight_tc(UNetTcTrain& t, const float* in, int cin, const float* g, int cout, int batch,
                                float* dw, float* db, cudaStream_t s) {
  constexpr int S3 = S * S * S;
  const int kp = padded_k(cin), m = batch * S3;
  constexpr int S3_LOG2 = S == 8 ? 9 : S == 4 ? 6 : 3;
  static_assert(1 << S3_LOG2 == S3, "S is 2, 4 or 8");
  g_kernel_launches += 5;
  cudaError_t e = im2col<S, VALID>(in, cin, batch, t.col, s);
  if (e != cudaSuccess) return e;
  k_grad_cols<<<grid_of((long long)m * cout), kT, 0, s>>>(g, cout, S3, m, (unsigned)m * cout, t.g);
  e = gemm(t, CUBLAS_OP_N, CUBLAS_OP_N, kp, cout, m, t.col, kp, t.g, m, t.out, kp, s);
  if (e != cudaSuccess) return e;
  k_unpack_dw<<<(cout * cin * 27 + kT - 1) / kT, kT, 0, s>>>(t.out, cout, cin, kp, dw);
  k_bias_partial<<<dim3(cout, kBiasChunks), kT, 0, s>>>(g, cout, S3_LOG2, batch, t.part);
  k_bias_final<<<1, 64, 0, s>>>(t.part, cout, db);
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
