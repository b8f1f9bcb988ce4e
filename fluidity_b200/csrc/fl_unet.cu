// Learned block preconditioner: a small 3D U-Net over one 8^3 pressure block
// plus a one-cell halo, trained on the GPU with these kernels.
//
// The reference has no learned solver; this is a build-only component. The
// network (channels 16/32/64, 3x3x3 convolutions, ReLU, 2x average pooling,
// nearest upsampling with 1x1 reductions and additive skips, 141,937
// parameters) is:
//   e1a = relu(conv3(x, 2->16, valid))        10^3 -> 8^3
//   s1  = relu(conv3(e1a, 16->16))            8^3
//   e2a = relu(conv3(pool(s1), 16->32))       4^3
//   s2  = relu(conv3(e2a, 32->32))            4^3
//   bt  = relu(conv3(pool(s2), 32->64))       2^3
//   u2  = relu(up(conv1(bt, 64->32)) + s2)    4^3
//   d2  = relu(conv3(u2, 32->32))
//   u1  = relu(up(conv1(d2, 32->16)) + s1)    8^3
//   d1  = relu(conv3(u1, 16->16))
//   y   = conv1(d1, 16->1)                    8^3
// conv1(up(x)) is evaluated as up(conv1(x)) (identical for a pointwise linear
// map and nearest upsampling). Parameters are FP32, flattened layer by layer as
// weight [Cout][Cin][27 taps (dz,dy,dx)] then bias [Cout]. Training activations
// are FP32 [batch][channel][z][y][x]. Every reduction (weight gradients, loss)
// runs in a fixed order, so a training step is bitwise reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"
#include "fl_unet.h"

namespace fl {
namespace {

constexpr int kT = 256;

// ---------------------------------------------------------------- forward

// out[b][co][cell] = act(bias[co] + sum_ci sum_tap w[co][ci][tap] in[b][ci][cell + tap]).
// VALID: the input is already (S+2)^3; otherwise it is S^3, zero padded here.
// One CTA per (batch item, chunk of output channels); the input item sits in
// shared memory as [ci][(S+2)^3].
template <int S, bool VALID>
__global__ void __launch_bounds__(kT) k_conv3_fwd(const float* __restrict__ in, int cin, const float* __restrict__ w,
                                                  const float* __restrict__ bias, int cout, int co_chunk,
                                                  float* __restrict__ out, int relu) {
  constexpr int P = S + 2, P3 = P * P * P, S3 = S * S * S;
  extern __shared__ float tile[];
  const int b = blockIdx.x;
  const int co0 = blockIdx.y * co_chunk;
  if (VALID) {
    const float* src = in + (size_t)b * cin * P3;
    for (int i = threadIdx.x; i < cin * P3; i += kT) tile[i] = src[i];
  } else {
    const float* src = in + (size_t)b * cin * S3;
    for (int i = threadIdx.x; i < cin * P3; i += kT) {
      const int ci = i / P3, r = i - ci * P3;
      const int pz = r / (P * P), py = (r / P) % P, px = r % P;
      const bool inside = pz >= 1 && pz <= S && py >= 1 && py <= S && px >= 1 && px <= S;
      tile[i] = inside ? src[ci * S3 + ((pz - 1) * S + (py - 1)) * S + (px - 1)] : 0.0f;
    }
  }
  __syncthreads();
  const int n_out = min(co_chunk, cout - co0) * S3;
  for (int idx = threadIdx.x; idx < n_out; idx += kT) {
    const int co = co0 + idx / S3, cell = idx % S3;
    const int z = cell / (S * S), y = (cell / S) % S, x = cell % S;
    float acc = bias[co];
    const float* wc = w + (size_t)co * cin * 27;
    for (int ci = 0; ci < cin; ++ci) {
      const float* t = tile + ci * P3 + (z * P + y) * P + x;
      const float* wk = wc + ci * 27;
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) acc = fmaf(__ldg(&wk[(dz * 3 + dy) * 3 + dx]), t[(dz * P + dy) * P + dx], acc);
    }
    out[((size_t)b * cout + co) * S3 + cell] = relu ? fmaxf(acc, 0.0f) : acc;
  }
}

// out[b][co][cell] = bias[co] + sum_ci w[co][ci] in[b][ci][cell].
__global__ void k_conv1_fwd(const float* __restrict__ in, int cin, const float* __restrict__ w,
                            const float* __restrict__ bias, int cout, int s3, long long total,
                            float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int cell = (int)(i % s3);
    const int co = (int)((i / s3) % cout);
    const long long b = i / ((long long)s3 * cout);
    float acc = bias[co];
    const float* src = in + (size_t)b * cin * s3 + cell;
    for (int ci = 0; ci < cin; ++ci) acc = fmaf(__ldg(&w[co * cin + ci]), src[(size_t)ci * s3], acc);
    out[i] = acc;
  }
}

// 2x average pooling: out [B][C][(S/2)^3] from in [B][C][S^3].
__global__ void k_pool(const float* __restrict__ in, int S, long long total, float* __restrict__ out) {
  const int H = S / 2, H3 = H * H * H, S3 = S * S * S;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int c = (int)(i % H3);
    const long long bc = i / H3;
    const int z = c / (H * H), y = (c / H) % H, x = c % H;
    const float* src = in + bc * S3 + ((2 * z) * S + 2 * y) * S + 2 * x;
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += src[((k >> 2) * S + ((k >> 1) & 1)) * S + (k & 1)];
    out[i] = s * 0.125f;
  }
}

// out = relu(coarse[parent] + skip) at resolution S.
__global__ void k_up_add_relu(const float* __restrict__ coarse, const float* __restrict__ skip, int S, long long total,
                              float* __restrict__ out) {
  const int H = S / 2, S3 = S * S * S, H3 = H * H * H;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int c = (int)(i % S3);
    const long long bc = i / S3;
    const int z = c / (S * S), y = (c / S) % S, x = c % S;
    out[i] = fmaxf(coarse[bc * H3 + ((z >> 1) * H + (y >> 1)) * H + (x >> 1)] + skip[i], 0.0f);
  }
}

// ---------------------------------------------------------------- backward

// din[b][ci][i] = (sum_co sum_tap w[co][ci][tap] g[b][co][i - tap + 1]) * (act[b][ci][i] > 0 if act).
// The gradient item sits in shared memory zero padded as [co][(S+2)^3].
template <int S>
__global__ void __launch_bounds__(kT) k_conv3_bwd_data(const float* __restrict__ g, int cout,
                                                       const float* __restrict__ w, int cin, int ci_chunk,
                                                       const float* __restrict__ act, float* __restrict__ din) {
  constexpr int P = S + 2, P3 = P * P * P, S3 = S * S * S;
  extern __shared__ float tile[];
  const int b = blockIdx.x;
  const int ci0 = blockIdx.y * ci_chunk;
  const float* src = g + (size_t)b * cout * S3;
  for (int i = threadIdx.x; i < cout * P3; i += kT) {
    const int co = i / P3, r = i - co * P3;
    const int pz = r / (P * P), py = (r / P) % P, px = r % P;
    const bool inside = pz >= 1 && pz <= S && py >= 1 && py <= S && px >= 1 && px <= S;
    tile[i] = inside ? src[co * S3 + ((pz - 1) * S + (py - 1)) * S + (px - 1)] : 0.0f;
  }
  __syncthreads();
  const int n_out = min(ci_chunk, cin - ci0) * S3;
  for (int idx = threadIdx.x; idx < n_out; idx += kT) {
    const int ci = ci0 + idx / S3, cell = idx % S3;
    const size_t o = ((size_t)b * cin + ci) * S3 + cell;
    if (act != nullptr && !(act[o] > 0.0f)) {
      din[o] = 0.0f;
      continue;
    }
    const int z = cell / (S * S), y = (cell / S) % S, x = cell % S;
    float acc = 0.0f;
    for (int co = 0; co < cout; ++co) {
      const float* t = tile + co * P3 + ((z + 2) * P + (y + 2)) * P + (x + 2);
      const float* wk = w + ((size_t)co * cin + ci) * 27;
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
          for (int dx = 0; dx < 3; ++dx)
            acc = fmaf(__ldg(&wk[(dz * 3 + dy) * 3 + dx]), t[-((dz * P + dy) * P + dx)], acc);
    }
    din[o] = acc;
  }
}

// 27 partial sums -> shared result in fixed order (warp shuffles, then warps in order).
__device__ __forceinline__ void block_sum27(float (&acc)[27], float* red /* 27 * (kT/32) */, float* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 27; ++t) {
    float v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[t * (kT / 32) + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 27) {
    float s = 0.0f;
    for (int k = 0; k < kT / 32; ++k) s += red[threadIdx.x * (kT / 32) + k];
    out[threadIdx.x] = s;
  }
}

// dw[co][ci][tap] = sum_b sum_o g[b][co][o] in[b][ci][o + tap - pad]; db[co] = sum_b sum_o g[b][co][o]
// (written by the ci == 0 CTA). One CTA per (ci, co). VALID: input extent S+2, pad 0.
template <int S, bool VALID>
__global__ void __launch_bounds__(kT) k_conv3_bwd_weight(const float* __restrict__ in, int cin,
                                                         const float* __restrict__ g, int cout, int batch,
                                                         float* __restrict__ dw, float* __restrict__ db) {
  constexpr int S3 = S * S * S;
  constexpr int E = VALID ? S + 2 : S;  // input extent
  constexpr int E3 = E * E * E;
  __shared__ float red[27 * (kT / 32)];
  __shared__ float res[27];
  __shared__ float bred[kT / 32];
  const int ci = blockIdx.x, co = blockIdx.y;
  float acc[27];
#pragma unroll
  for (int t = 0; t < 27; ++t) acc[t] = 0.0f;
  float bsum = 0.0f;
  const int total = batch * S3;
  for (int idx = threadIdx.x; idx < total; idx += kT) {
    const int b = idx / S3, o = idx % S3;
    const float gv = g[((size_t)b * cout + co) * S3 + o];
    bsum += gv;
    const int z = o / (S * S), y = (o / S) % S, x = o % S;
    const float* src = in + ((size_t)b * cin + ci) * E3;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          int zz = z + dz, yy = y + dy, xx = x + dx;
          if (!VALID) {
            zz -= 1;
            yy -= 1;
            xx -= 1;
          }
          float v = 0.0f;
          if (VALID || (zz >= 0 && zz < S && yy >= 0 && yy < S && xx >= 0 && xx < S)) v = src[(zz * E + yy) * E + xx];
          acc[(dz * 3 + dy) * 3 + dx] = fmaf(gv, v, acc[(dz * 3 + dy) * 3 + dx]);
        }
  }
  block_sum27(acc, red, res);
  __syncthreads();
  if (threadIdx.x < 27) dw[((size_t)co * cin + ci) * 27 + threadIdx.x] = res[threadIdx.x];
  if (ci == 0) {
    float v = bsum;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) bred[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      float s = 0.0f;
      for (int k = 0; k < kT / 32; ++k) s += bred[k];
      db[co] = s;
    }
  }
}

// dw[co][ci] = sum g[b][co][o] in[b][ci][o]; db[co] likewise (ci == 0 CTA). One CTA of NT
// threads per (ci, co): 1024 for the output layer, whose 16 CTAs each reduce a whole plane.
template <int NT>
__global__ void __launch_bounds__(NT) k_conv1_bwd_weight(const float* __restrict__ in, int cin,
                                                         const float* __restrict__ g, int cout, int s3, int batch,
                                                         float* __restrict__ dw, float* __restrict__ db) {
  __shared__ float red[2 * (NT / 32)];
  const int ci = blockIdx.x, co = blockIdx.y;
  float a = 0.0f, bs = 0.0f;
  for (int idx = threadIdx.x; idx < batch * s3; idx += NT) {
    const int b = idx / s3, o = idx % s3;
    const float gv = g[((size_t)b * cout + co) * s3 + o];
    a = fmaf(gv, in[((size_t)b * cin + ci) * s3 + o], a);
    bs += gv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    bs += __shfl_xor_sync(0xffffffffu, bs, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = a;
    red[NT / 32 + (threadIdx.x >> 5)] = bs;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.0f, t = 0.0f;
    for (int k = 0; k < NT / 32; ++k) {
      s += red[k];
      t += red[NT / 32 + k];
    }
    dw[co * cin + ci] = s;
    if (ci == 0) db[co] = t;
  }
}

// din[b][ci][o] = (sum_co w[co][ci] g[b][co][o]) * (act > 0).
__global__ void k_conv1_bwd_data(const float* __restrict__ g, int cout, const float* __restrict__ w, int cin, int s3,
                                 long long total, const float* __restrict__ act, float* __restrict__ din) {
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int o = (int)(i % s3);
    const int ci = (int)((i / s3) % cin);
    const long long b = i / ((long long)s3 * cin);
    float acc = 0.0f;
    if (act == nullptr || act[i] > 0.0f) {
      const float* src = g + (size_t)b * cout * s3 + o;
      for (int co = 0; co < cout; ++co) acc = fmaf(__ldg(&w[co * cin + ci]), src[(size_t)co * s3], acc);
    }
    din[i] = acc;
  }
}

// out[b][c][coarse] = sum of the 8 children of g at resolution S.
__global__ void k_up_back(const float* __restrict__ g, int S, long long total, float* __restrict__ out) {
  const int H = S / 2, H3 = H * H * H, S3 = S * S * S;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int c = (int)(i % H3);
    const long long bc = i / H3;
    const int z = c / (H * H), y = (c / H) % H, x = c % H;
    const float* src = g + bc * S3 + ((2 * z) * S + 2 * y) * S + 2 * x;
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += src[((k >> 2) * S + ((k >> 1) & 1)) * S + (k & 1)];
    out[i] = s;
  }
}

// out = (ga + gp[parent] / 8) * (act > 0) at resolution S.
__global__ void k_pool_back_add_mask(const float* __restrict__ ga, const float* __restrict__ gp,
                                     const float* __restrict__ act, int S, long long total, float* __restrict__ out) {
  const int H = S / 2, S3 = S * S * S, H3 = H * H * H;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < total; i += (long long)gridDim.x * kT) {
    const int c = (int)(i % S3);
    const long long bc = i / S3;
    const int z = c / (S * S), y = (c / S) % S, x = c % S;
    const float v = ga[i] + 0.125f * gp[bc * H3 + ((z >> 1) * H + (y >> 1)) * H + (x >> 1)];
    out[i] = act[i] > 0.0f ? v : 0.0f;
  }
}

// Masked squared error in one CTA (fixed order). relative == 0:
//   loss = sum m (y - t)^2 / max(1, sum m), grad = 2 m (y - t) / max(1, sum m);
// relative == 1 (every item weighs the same whatever its scale):
//   loss = (1/V) sum_items [sum m (y - t)^2 / sum m t^2] over the V items with
//   sum m t^2 > 0 (items without target energy add nothing), grad likewise.
__global__ void __launch_bounds__(1024) k_masked_mse(const float* __restrict__ y, const float* __restrict__ t,
                                                     const float* __restrict__ m, int batch, int relative,
                                                     float* __restrict__ loss, float* __restrict__ grad) {
  __shared__ double red[2 * 32];
  __shared__ double item_den[1024];
  const int n = batch * 512;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // per-item denominators (one warp per item, items in order)
  for (int b = warp; b < batch; b += nwarps) {
    double s = 0.0, c = 0.0;
    for (int k = lane; k < 512; k += 32) {
      const double tv = t[b * 512 + k];
      s += m[b * 512 + k] * tv * tv;
      c += m[b * 512 + k];
    }
    s = warp_sum(s);
    c = warp_sum(c);
    if (lane == 0) item_den[b] = relative ? s : c;
  }
  __syncthreads();
  double global_den = 0.0;
  int valid = 0;
  for (int b = 0; b < batch; ++b) {
    global_den += item_den[b];
    valid += item_den[b] > 0.0;
  }
  global_den = global_den > 1.0 ? global_den : 1.0;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int b = i >> 9;
    const double den = relative ? item_den[b] * valid : global_den;
    const double d = (double)y[i] - (double)t[i];
    const double w = relative && !(item_den[b] > 0.0) ? 0.0 : m[i] / den;
    acc += w * d * d;
    if (grad) grad[i] = (float)(2.0 * w * d);
  }
  acc = warp_sum(acc);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0 && loss) {
    double total = 0.0;
    for (int k = 0; k < nwarps; ++k) total += red[k];
    *loss = (float)total;
  }
}

// Block-residual loss in one CTA of 512 threads (a thread per block cell),
// items in order. For item b the input window holds r / s (channel 0) and the
// cell mask (channel 1: fluid 1, air 0, solid -1) on the block plus a one-cell
// halo; y is the network's correction on the block's 8^3 cells. With A_b the
// level-0 pressure operator restricted to the block's fluid cells (unit
// conductance to fluid and air neighbours, none to solid ones, the block's
// neighbours held at zero):
//   rho = r_b - A_b y,  loss = (1/V) sum_items |rho|^2 / D_b,
//   d loss / d y = -(2 / (V D_b)) A_b rho   (A_b is symmetric),
// with D_b = max(|r_b|^2, 1) (the window is scaled to max |r| = 1, so a block
// whose residual is mostly in its halo does not weigh more than the rest),
// over the V items whose block holds residual. The zero correction scores at
// most 1; a network that inverts A_b on its block scores 0.
__global__ void __launch_bounds__(512) k_block_residual_loss(const float* __restrict__ y,
                                                             const float* __restrict__ x, int batch,
                                                             float* __restrict__ loss, float* __restrict__ grad) {
  __shared__ float mask[1000];
  __shared__ float vec[512];
  __shared__ double item_den[1024];
  __shared__ double red[16];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int cx = t & 7, cy = (t >> 3) & 7, cz = t >> 6;
  const int w = ((cz + 1) * 10 + (cy + 1)) * 10 + (cx + 1);
  const int nb_w[6] = {w - 1, w + 1, w - 10, w + 10, w - 100, w + 100};
  const bool nb_in[6] = {cx > 0, cx < 7, cy > 0, cy < 7, cz > 0, cz < 7};
  const int nb_l[6] = {t - 1, t + 1, t - 8, t + 8, t - 64, t + 64};
  // pass 1: |r_b|^2 per item and the number of items with residual
  for (int b = 0; b < batch; ++b) {
    const float* xb = x + (size_t)b * 2000;
    const double rv = xb[1000 + w] == 1.0f ? (double)xb[w] : 0.0;
    double v = warp_sum(rv * rv);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int k = 0; k < 16; ++k) sum += red[k];
      item_den[b] = sum;
    }
  }
  __syncthreads();
  int valid = 0;
  for (int b = 0; b < batch; ++b) valid += item_den[b] > 0.0;
  double acc = 0.0;
  // pass 2: residual after the correction, the loss and its gradient
  for (int b = 0; b < batch; ++b) {
    const float* xb = x + (size_t)b * 2000;
    for (int i = t; i < 1000; i += 512) mask[i] = xb[1000 + i];
    __syncthreads();
    const bool fluid = mask[w] == 1.0f;
    const float yc = fluid ? y[(size_t)b * 512 + t] : 0.0f;
    vec[t] = yc;
    __syncthreads();
    float diag = 0.0f, off = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float mk = mask[nb_w[k]];
      diag += mk >= 0.0f ? 1.0f : 0.0f;
      if (nb_in[k] && mk == 1.0f) off += vec[nb_l[k]];
    }
    const float rho = fluid ? xb[w] - (diag * yc - off) : 0.0f;
    __syncthreads();
    vec[t] = rho;
    __syncthreads();
    float arho = 0.0f;
    if (fluid) {
      float o = 0.0f;
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (nb_in[k] && mask[nb_w[k]] == 1.0f) o += vec[nb_l[k]];
      arho = diag * rho - o;
    }
    const double den = item_den[b];
    const double scale = den > 0.0 ? 1.0 / (valid * fmax(den, 1.0)) : 0.0;
    acc += scale * (double)rho * (double)rho;
    if (grad) grad[(size_t)b * 512 + t] = (float)(-2.0 * scale * (double)arho);
    __syncthreads();
  }
  acc = warp_sum(acc);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (t == 0 && loss) {
    double total = 0.0;
    for (int k = 0; k < 16; ++k) total += red[k];
    *loss = (float)total;
  }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < n; i += (long long)gridDim.x * kT) {
    const float gi = g[i];
    const float mi = fmaf(b1, m[i], (1.0f - b1) * gi);
    const float vi = fmaf(b2, v[i], (1.0f - b2) * gi * gi);
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// He-uniform weights from a counter-based SplitMix64 stream, zero biases.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_init_params(float* p, UNetLayout L, unsigned long long seed) {
  const long long n = L.total;
  for (long long i = blockIdx.x * (long long)kT + threadIdx.x; i < n; i += (long long)gridDim.x * kT) {
    int l = 0;
    while (l + 1 < kUNetLayers && i >= L.offset[l + 1]) ++l;
    const long long local = i - L.offset[l];
    const long long nw = (long long)L.cout[l] * L.cin[l] * L.taps[l];
    if (local >= nw) {
      p[i] = 0.0f;
      continue;
    }
    const float bound = sqrtf(6.0f / (float)(L.cin[l] * L.taps[l]));
    const unsigned long long r = splitmix64(seed * 0x100000001B3ull + (unsigned long long)i);
    const float u = (float)((r >> 40) * (1.0 / 16777216.0));  // [0, 1)
    p[i] = (2.0f * u - 1.0f) * bound;
  }
}

unsigned grid_for(long long n) {
  long long b = (n + kT - 1) / kT;
  return (unsigned)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

template <int S, bool VALID>
void conv3_fwd(const float* in, int cin, const float* w, const float* bias, int cout, float* out, int batch, int relu,
               cudaStream_t s) {
  constexpr int P3 = (S + 2) * (S + 2) * (S + 2);
  const int chunk = S == 8 ? 8 : cout;
  const size_t smem = sizeof(float) * cin * P3;
  ++g_kernel_launches;
  k_conv3_fwd<S, VALID><<<dim3(batch, (cout + chunk - 1) / chunk), kT, smem, s>>>(in, cin, w, bias, cout, chunk, out,
                                                                                  relu);
}

template <int S>
void conv3_bwd_data(const float* g, int cout, const float* w, int cin, const float* act, float* din, int batch,
                    cudaStream_t s) {
  constexpr int P3 = (S + 2) * (S + 2) * (S + 2);
  const int chunk = S == 8 ? 8 : cin;
  const size_t smem = sizeof(float) * cout * P3;
  ++g_kernel_launches;
  k_conv3_bwd_data<S><<<dim3(batch, (cin + chunk - 1) / chunk), kT, smem, s>>>(g, cout, w, cin, chunk, act, din);
}

template <int S, bool VALID>
void conv3_bwd_weight(const float* in, int cin, const float* g, int cout, int batch, float* dw, float* db,
                      cudaStream_t s) {
  ++g_kernel_launches;
  k_conv3_bwd_weight<S, VALID><<<dim3(cin, cout), kT, 0, s>>>(in, cin, g, cout, batch, dw, db);
}

// A 3x3x3 layer on the SIMT kernels (tc == nullptr) or as a tensor-core GEMM;
// the first tensor-core failure is kept in `e` and the remaining layers skip.
template <int S, bool VALID>
void fwd3(UNetTcTrain* tc, cudaError_t& e, const float* in, int cin, const float* w, const float* bias, int cout,
          float* out, int batch, int relu, cudaStream_t s) {
  if (tc == nullptr) return conv3_fwd<S, VALID>(in, cin, w, bias, cout, out, batch, relu, s);
  if (e == cudaSuccess) e = conv3_fwd_tc<S, VALID>(*tc, in, cin, w, bias, cout, out, batch, relu, s);
}
template <int S>
void bwd3_data(UNetTcTrain* tc, cudaError_t& e, const float* g, int cout, const float* w, int cin, const float* act,
               float* din, int batch, cudaStream_t s) {
  if (tc == nullptr) return conv3_bwd_data<S>(g, cout, w, cin, act, din, batch, s);
  if (e == cudaSuccess) e = conv3_bwd_data_tc<S>(*tc, g, cout, w, cin, act, din, batch, s);
}
template <int S, bool VALID>
void bwd3_weight(UNetTcTrain* tc, cudaError_t& e, const float* in, int cin, const float* g, int cout, int batch,
                 float* dw, float* db, cudaStream_t s) {
  if (tc == nullptr) return conv3_bwd_weight<S, VALID>(in, cin, g, cout, batch, dw, db, s);
  if (e == cudaSuccess) e = conv3_bwd_weight_tc<S, VALID>(*tc, in, cin, g, cout, batch, dw, db, s);
}

}  // namespace

UNetLayout unet_layout() {
  static const int kCin[kUNetLayers] = {2, 16, 16, 32, 32, 64, 32, 32, 16, 16};
  static const int kCout[kUNetLayers] = {16, 16, 32, 32, 64, 32, 32, 16, 16, 1};
  static const int kTaps[kUNetLayers] = {27, 27, 27, 27, 27, 1, 27, 1, 27, 1};
  UNetLayout L{};
  long long off = 0;
  for (int l = 0; l < kUNetLayers; ++l) {
    L.cin[l] = kCin[l];
    L.cout[l] = kCout[l];
    L.taps[l] = kTaps[l];
    L.offset[l] = off;
    L.bias[l] = off + (long long)kCout[l] * kCin[l] * kTaps[l];
    off = L.bias[l] + kCout[l];
  }
  L.total = off;
  return L;
}

UNetCache unet_cache_layout(int batch) {
  UNetCache C{};
  long long off = 0;
  auto take = [&](long long per_item) {
    const long long o = off;
    off += per_item * batch;
    return o;
  };
  C.x = take(2 * 1000);
  C.e1a = take(16 * 512);
  C.s1 = take(16 * 512);
  C.p1 = take(16 * 64);
  C.e2a = take(32 * 64);
  C.s2 = take(32 * 64);
  C.p2 = take(32 * 8);
  C.bt = take(64 * 8);
  C.c2 = take(32 * 8);
  C.u2 = take(32 * 64);
  C.d2 = take(32 * 64);
  C.c1 = take(16 * 64);
  C.u1 = take(16 * 512);
  C.d1 = take(16 * 512);
  C.y = take(512);
  C.activations = off;
  // backward scratch
  C.g8a = take(16 * 512);
  C.g8b = take(16 * 512);
  C.g8c = take(16 * 512);
  C.g4a = take(32 * 64);
  C.g4b = take(32 * 64);
  C.g4c = take(32 * 64);
  C.g2a = take(64 * 8);
  C.g2b = take(64 * 8);
  C.total = off;
  return C;
}

void configure_unet_kernels() {
  static bool done = false;
  if (done) return;
  const int big = sizeof(float) * 32 * 1000;  // largest padded tile: 32 channels of 10^3
  cudaFuncSetAttribute(k_conv3_fwd<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(k_conv3_fwd<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(k_conv3_bwd_data<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  done = true;
}

// Forward pass of `batch` items; every activation is kept in `cache` (layout unet_cache_layout).
cudaError_t unet_forward(const float* P, const float* x, int batch, float* cache, float* y, cudaStream_t s,
                         UNetTcTrain* tc) {
  configure_unet_kernels();
  const UNetLayout L = unet_layout();
  const UNetCache C = unet_cache_layout(batch);
  float* A = cache;
  const long long B = batch;
  if (x != A + C.x) cudaMemcpyAsync(A + C.x, x, sizeof(float) * 2000 * B, cudaMemcpyDeviceToDevice, s);
  auto W = [&](int l) { return P + L.offset[l]; };
  auto Bi = [&](int l) { return P + L.bias[l]; };
  cudaError_t tce = cudaSuccess;
  fwd3<8, true>(tc, tce, A + C.x, 2, W(0), Bi(0), 16, A + C.e1a, batch, 1, s);
  fwd3<8, false>(tc, tce, A + C.e1a, 16, W(1), Bi(1), 16, A + C.s1, batch, 1, s);
  g_kernel_launches += 1;
  k_pool<<<grid_for(B * 16 * 64), kT, 0, s>>>(A + C.s1, 8, B * 16 * 64, A + C.p1);
  fwd3<4, false>(tc, tce, A + C.p1, 16, W(2), Bi(2), 32, A + C.e2a, batch, 1, s);
  fwd3<4, false>(tc, tce, A + C.e2a, 32, W(3), Bi(3), 32, A + C.s2, batch, 1, s);
  g_kernel_launches += 1;
  k_pool<<<grid_for(B * 32 * 8), kT, 0, s>>>(A + C.s2, 4, B * 32 * 8, A + C.p2);
  fwd3<2, false>(tc, tce, A + C.p2, 32, W(4), Bi(4), 64, A + C.bt, batch, 1, s);
  g_kernel_launches += 6;
  k_conv1_fwd<<<grid_for(B * 32 * 8), kT, 0, s>>>(A + C.bt, 64, W(5), Bi(5), 32, 8, B * 32 * 8, A + C.c2);
  k_up_add_relu<<<grid_for(B * 32 * 64), kT, 0, s>>>(A + C.c2, A + C.s2, 4, B * 32 * 64, A + C.u2);
  fwd3<4, false>(tc, tce, A + C.u2, 32, W(6), Bi(6), 32, A + C.d2, batch, 1, s);
  k_conv1_fwd<<<grid_for(B * 16 * 64), kT, 0, s>>>(A + C.d2, 32, W(7), Bi(7), 16, 64, B * 16 * 64, A + C.c1);
  k_up_add_relu<<<grid_for(B * 16 * 512), kT, 0, s>>>(A + C.c1, A + C.s1, 8, B * 16 * 512, A + C.u1);
  fwd3<8, false>(tc, tce, A + C.u1, 16, W(8), Bi(8), 16, A + C.d1, batch, 1, s);
  k_conv1_fwd<<<grid_for(B * 512), kT, 0, s>>>(A + C.d1, 16, W(9), Bi(9), 1, 512, B * 512, A + C.y);
  if (y != nullptr && y != A + C.y)
    cudaMemcpyAsync(y, A + C.y, sizeof(float) * 512 * B, cudaMemcpyDeviceToDevice, s);
  if (tce != cudaSuccess) return tce;
  return cudaGetLastError();
}

// Gradient of sum(gy * y) with respect to the parameters, from the cache of the last forward.
cudaError_t unet_backward(const float* P, float* cache, const float* gy, int batch, float* G, cudaStream_t s,
                          UNetTcTrain* tc) {
  configure_unet_kernels();
  cudaError_t tce = cudaSuccess;
  const UNetLayout L = unet_layout();
  const UNetCache C = unet_cache_layout(batch);
  float* A = cache;
  const long long B = batch;
  auto W = [&](int l) { return P + L.offset[l]; };
  auto GW = [&](int l) { return G + L.offset[l]; };
  auto GB = [&](int l) { return G + L.bias[l]; };
  // out layer (16 -> 1)
  g_kernel_launches += 2;
  k_conv1_bwd_weight<1024><<<dim3(16, 1), 1024, 0, s>>>(A + C.d1, 16, gy, 1, 512, batch, GW(9), GB(9));
  k_conv1_bwd_data<<<grid_for(B * 16 * 512), kT, 0, s>>>(gy, 1, W(9), 16, 512, B * 16 * 512, A + C.d1, A + C.g8a);
  // d1 (conv3 16->16 on u1); gu1 pre-activation -> g8b
  bwd3_weight<8, false>(tc, tce, A + C.u1, 16, A + C.g8a, 16, batch, GW(8), GB(8), s);
  bwd3_data<8>(tc, tce, A + C.g8a, 16, W(8), 16, A + C.u1, A + C.g8b, batch, s);
  // u1 = relu(up(c1) + s1): c1 = conv1(d2, 32->16)
  g_kernel_launches += 3;
  k_up_back<<<grid_for(B * 16 * 64), kT, 0, s>>>(A + C.g8b, 8, B * 16 * 64, A + C.g4c);
  k_conv1_bwd_weight<kT><<<dim3(32, 16), kT, 0, s>>>(A + C.d2, 32, A + C.g4c, 16, 64, batch, GW(7), GB(7));
  k_conv1_bwd_data<<<grid_for(B * 32 * 64), kT, 0, s>>>(A + C.g4c, 16, W(7), 32, 64, B * 32 * 64, A + C.d2,
                                                        A + C.g4a);
  // d2 (conv3 32->32 on u2); gu2 pre-activation -> g4b
  bwd3_weight<4, false>(tc, tce, A + C.u2, 32, A + C.g4a, 32, batch, GW(6), GB(6), s);
  bwd3_data<4>(tc, tce, A + C.g4a, 32, W(6), 32, A + C.u2, A + C.g4b, batch, s);
  // u2 = relu(up(c2) + s2): c2 = conv1(bt, 64->32)
  g_kernel_launches += 3;
  k_up_back<<<grid_for(B * 32 * 8), kT, 0, s>>>(A + C.g4b, 4, B * 32 * 8, A + C.g2b);
  k_conv1_bwd_weight<kT><<<dim3(64, 32), kT, 0, s>>>(A + C.bt, 64, A + C.g2b, 32, 8, batch, GW(5), GB(5));
  k_conv1_bwd_data<<<grid_for(B * 64 * 8), kT, 0, s>>>(A + C.g2b, 32, W(5), 64, 8, B * 64 * 8, A + C.bt, A + C.g2a);
  // bt (conv3 32->64 on p2) -> gp2 (g2b, 32 channels)
  bwd3_weight<2, false>(tc, tce, A + C.p2, 32, A + C.g2a, 64, batch, GW(4), GB(4), s);
  bwd3_data<2>(tc, tce, A + C.g2a, 64, W(4), 32, nullptr, A + C.g2b, batch, s);
  // s2 gradient: (gu2 + pool_back(gp2)) * (s2 > 0) -> g4a
  g_kernel_launches += 1;
  k_pool_back_add_mask<<<grid_for(B * 32 * 64), kT, 0, s>>>(A + C.g4b, A + C.g2b, A + C.s2, 4, B * 32 * 64,
                                                            A + C.g4a);
  // e2b (conv3 32->32 on e2a) -> ge2a (g4c)
  bwd3_weight<4, false>(tc, tce, A + C.e2a, 32, A + C.g4a, 32, batch, GW(3), GB(3), s);
  bwd3_data<4>(tc, tce, A + C.g4a, 32, W(3), 32, A + C.e2a, A + C.g4c, batch, s);
  // e2a (conv3 16->32 on p1) -> gp1 (g4b, 16 channels)
  bwd3_weight<4, false>(tc, tce, A + C.p1, 16, A + C.g4c, 32, batch, GW(2), GB(2), s);
  bwd3_data<4>(tc, tce, A + C.g4c, 32, W(2), 16, nullptr, A + C.g4b, batch, s);
  // s1 gradient: (gu1 + pool_back(gp1)) * (s1 > 0) -> g8a
  g_kernel_launches += 1;
  k_pool_back_add_mask<<<grid_for(B * 16 * 512), kT, 0, s>>>(A + C.g8b, A + C.g4b, A + C.s1, 8, B * 16 * 512,
                                                             A + C.g8a);
  // e1b (conv3 16->16 on e1a) -> ge1a (g8c)
  bwd3_weight<8, false>(tc, tce, A + C.e1a, 16, A + C.g8a, 16, batch, GW(1), GB(1), s);
  bwd3_data<8>(tc, tce, A + C.g8a, 16, W(1), 16, A + C.e1a, A + C.g8c, batch, s);
  // e1a (valid conv3 2->16 on x)
  bwd3_weight<8, true>(tc, tce, A + C.x, 2, A + C.g8c, 16, batch, GW(0), GB(0), s);
  if (tce != cudaSuccess) return tce;
  return cudaGetLastError();
}

cudaError_t unet_masked_mse(const float* y, const float* t, const float* m, int batch, int relative, float* loss,
                            float* grad, cudaStream_t s) {
  ++g_kernel_launches;
  k_masked_mse<<<1, 1024, 0, s>>>(y, t, m, batch, relative, loss, grad);
  return cudaGetLastError();
}

cudaError_t unet_block_residual_loss(const float* y, const float* x, int batch, float* loss, float* grad,
                                     cudaStream_t s) {
  ++g_kernel_launches;
  k_block_residual_loss<<<1, 512, 0, s>>>(y, x, batch, loss, grad);
  return cudaGetLastError();
}

cudaError_t adam_step(float* p, const float* g, float* m, float* v, long long n, int step, float lr, float b1,
                      float b2, float eps, cudaStream_t s) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  ++g_kernel_launches;
  k_adam<<<grid_for(n), kT, 0, s>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t unet_init_params(float* p, unsigned long long seed, cudaStream_t s) {
  const UNetLayout L = unet_layout();
  ++g_kernel_launches;
  k_init_params<<<grid_for(L.total), kT, 0, s>>>(p, L, seed);
  return cudaGetLastError();
}


// ---------------------------------------------------------------- solver <-> network

namespace {

// Input item of block b: its 8^3 cells plus a one-cell halo (10^3, z-major),
// channel 0 = residual / s, channel 1 = cell mask (fluid 1, air 0, solid -1),
// s = max |residual| over the window (0 -> all-zero input). Missing blocks
// read as air (inactive, inside the lattice) or solid (outside it).
__global__ void __launch_bounds__(512) k_unet_gather(GridView g, const float* __restrict__ r_rb,
                                                     const unsigned char* __restrict__ type,
                                                     const int* __restrict__ blocks, float* __restrict__ inputs,
                                                     float* __restrict__ scale) {
  __shared__ float red[16];
  const int item = blockIdx.x;
  const int b = blocks ? blocks[item] : item;
  float rv[2], mv[2], mx = 0.0f;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int i = threadIdx.x + 512 * k;
    rv[k] = 0.0f;
    mv[k] = 0.0f;
    if (i < 1000) {
      const int hz = i / 100 - 1, hy = (i / 10) % 10 - 1, hx = i % 10 - 1;
      const int ox = hx < 0 ? -1 : (hx > 7 ? 1 : 0), oy = hy < 0 ? -1 : (hy > 7 ? 1 : 0),
                oz = hz < 0 ? -1 : (hz > 7 ? 1 : 0);
      const int nb = (ox | oy | oz) ? g.nbr27[b * 27 + nbr_index(ox, oy, oz)] : b;
      if (nb >= 0) {
        const int l = ((hz - 8 * oz) * 8 + (hy - 8 * oy)) * 8 + (hx - 8 * ox);
        rv[k] = r_rb[nb * 512 + rb_of(l)];
        const int t = type[nb * 512 + l];
        mv[k] = t == 1 ? 1.0f : (t == 0 ? -1.0f : 0.0f);
      } else {
        mv[k] = nb == -1 ? 0.0f : -1.0f;
      }
      mx = fmaxf(mx, fabsf(rv[k]));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  float sc = 0.0f;
#pragma unroll
  for (int k = 0; k < 16; ++k) sc = fmaxf(sc, red[k]);
  float* out = inputs + (size_t)item * 2000;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int i = threadIdx.x + 512 * k;
    if (i < 1000) {
      out[i] = sc > 0.0f ? rv[k] / sc : 0.0f;
      out[1000 + i] = mv[k];
    }
  }
  if (threadIdx.x == 0) scale[item] = sc;
}

// Target item: (p_star - p_k) / s on fluid cells (natural order), mask = fluid.
__global__ void __launch_bounds__(512) k_unet_targets(GridView g, const double* __restrict__ p_star,
                                                      const double* __restrict__ p_k,
                                                      const unsigned char* __restrict__ type,
                                                      const int* __restrict__ blocks, const float* __restrict__ scale,
                                                      float* __restrict__ targets, float* __restrict__ masks) {
  const int item = blockIdx.x, l = threadIdx.x;
  const int b = blocks ? blocks[item] : item;
  const bool fluid = type[b * 512 + l] == 1;
  const float sc = scale[item];
  const int i = b * 512 + rb_of(l);
  targets[(size_t)item * 512 + l] = fluid && sc > 0.0f ? (float)((p_star[i] - p_k[i]) / (double)sc) : 0.0f;
  masks[(size_t)item * 512 + l] = fluid ? 1.0f : 0.0f;
}

// z = s * y on fluid cells, 0 elsewhere; RB: level-0 solver layout, else natural.
template <typename T, bool RB>
__global__ void __launch_bounds__(512) k_unet_scatter(int nb, const float* __restrict__ y,
                                                      const float* __restrict__ scale,
                                                      const unsigned char* __restrict__ type, T* __restrict__ z) {
  const int b = blockIdx.x, l = threadIdx.x;
  const float v = type[b * 512 + l] == 1 ? scale[b] * y[(size_t)b * 512 + l] : 0.0f;
  st_T(&z[b * 512 + (RB ? rb_of(l) : l)], v);
}

__global__ void __launch_bounds__(512) k_block_has_fluid(const unsigned char* __restrict__ type, int* flags) {
  const int b = blockIdx.x;
  const int any = __syncthreads_or(type[b * 512 + threadIdx.x] == 1);
  if (threadIdx.x == 0) flags[b] = any;
}

}  // namespace

cudaError_t unet_gather(const GridView& g, const float* r_rb, const unsigned char* type, const int* blocks, int count,
                        float* inputs, float* scale, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  ++g_kernel_launches;
  k_unet_gather<<<count, 512, 0, s>>>(g, r_rb, type, blocks, inputs, scale);
  return cudaGetLastError();
}

cudaError_t unet_targets(const GridView& g, const double* p_star, const double* p_k, const unsigned char* type,
                         const int* blocks, int count, const float* scale, float* targets, float* masks,
                         cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  ++g_kernel_launches;
  k_unet_targets<<<count, 512, 0, s>>>(g, p_star, p_k, type, blocks, scale, targets, masks);
  return cudaGetLastError();
}

template <typename T>
cudaError_t unet_scatter(int nb, const float* y, const float* scale, const unsigned char* type, T* z, bool rb,
                         cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  ++g_kernel_launches;
  if (rb)
    k_unet_scatter<T, true><<<nb, 512, 0, s>>>(nb, y, scale, type, z);
  else
    k_unet_scatter<T, false><<<nb, 512, 0, s>>>(nb, y, scale, type, z);
  return cudaGetLastError();
}
template cudaError_t unet_scatter<float>(int, const float*, const float*, const unsigned char*, float*, bool,
                                         cudaStream_t);
template cudaError_t unet_scatter<__nv_bfloat16>(int, const float*, const float*, const unsigned char*,
                                                 __nv_bfloat16*, bool, cudaStream_t);

cudaError_t unet_block_has_fluid(int nb, const unsigned char* type, int* flags, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  ++g_kernel_launches;
  k_block_has_fluid<<<nb, 512, 0, s>>>(type, flags);
  return cudaGetLastError();
}

}  // namespace fl

// ---------------------------------------------------------------- C-ABI

struct fl_unet {
  int device = 0;
  int max_batch = 0;
  float* cache = nullptr;
  fl::UNetTcTrain* tc = nullptr;  // set: the 3x3x3 training convolutions run on the tensor cores
};

namespace {
int unet_code(cudaError_t e) {
  if (e == cudaSuccess) return FL_OK;
  cudaGetLastError();
  return FL_INTERNAL;
}

int unet_device_ready() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FL_FAILED_PRECONDITION;
  }
  return FL_OK;
}
}  // namespace

extern "C" {

int64_t fl_unet_param_count(void) { return fl::unet_layout().total; }

int fl_unet_create(int max_batch, fl_unet** out) {
  if (out == nullptr || max_batch <= 0 || max_batch > (1 << 16)) return FL_INVALID_ARGUMENT;
  *out = nullptr;
  int st = unet_device_ready();
  if (st != FL_OK) return st;
  fl_unet* u = new fl_unet();
  cudaGetDevice(&u->device);
  u->max_batch = max_batch;
  const size_t bytes = sizeof(float) * (size_t)fl::unet_cache_layout(max_batch).total;
  if (cudaMalloc(&u->cache, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete u;
    return FL_RESOURCE_EXHAUSTED;
  }
  cudaMemset(u->cache, 0, bytes);
  *out = u;
  return FL_OK;
}

int fl_unet_destroy(fl_unet* u) {
  if (u == nullptr) return FL_OK;
  if (u->tc != nullptr) {
    fl::unet_tc_train_destroy(u->tc);
    delete u->tc;
  }
  cudaFree(u->cache);
  delete u;
  return FL_OK;
}

int fl_unet_set_tensor_cores(fl_unet* u, int enable) {
  if (u == nullptr || (enable != 0 && enable != 1)) return FL_INVALID_ARGUMENT;
  if (!enable) {
    if (u->tc != nullptr) {
      fl::unet_tc_train_destroy(u->tc);
      delete u->tc;
      u->tc = nullptr;
    }
    return FL_OK;
  }
  if (u->tc != nullptr) return FL_OK;
  if (u->max_batch > fl::kUNetTcMaxBatch) return FL_OUT_OF_RANGE;  // 32-bit operand indexing
  int st = fl::check_device();
  if (st != FL_OK) return st;
  auto* t = new fl::UNetTcTrain();
  if (fl::unet_tc_train_create(u->max_batch, t) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return FL_RESOURCE_EXHAUSTED;
  }
  u->tc = t;
  return FL_OK;
}

int fl_unet_init_params(float* params, uint64_t seed, void* stream) {
  if (params == nullptr) return FL_INVALID_ARGUMENT;
  int st = unet_device_ready();
  if (st != FL_OK) return st;
  return unet_code(fl::unet_init_params(params, seed, static_cast<cudaStream_t>(stream)));
}

int fl_unet_forward(fl_unet* u, const float* params, const float* input, int batch, float* output, void* stream) {
  if (u == nullptr || params == nullptr || input == nullptr || batch < 0) return FL_INVALID_ARGUMENT;
  if (batch > u->max_batch) return FL_RESOURCE_EXHAUSTED;
  if (batch == 0) return FL_OK;
  return unet_code(
      fl::unet_forward(params, input, batch, u->cache, output, static_cast<cudaStream_t>(stream), u->tc));
}

int fl_unet_backward(fl_unet* u, const float* params, const float* grad_output, int batch, float* grad_params,
                     void* stream) {
  if (u == nullptr || params == nullptr || grad_output == nullptr || grad_params == nullptr || batch <= 0)
    return FL_INVALID_ARGUMENT;
  if (batch > u->max_batch) return FL_RESOURCE_EXHAUSTED;
  return unet_code(fl::unet_backward(params, u->cache, grad_output, batch, grad_params,
                                     static_cast<cudaStream_t>(stream), u->tc));
}

int fl_unet_masked_mse(const float* output, const float* target, const float* mask, int batch, int relative,
                       float* loss, float* grad_output, void* stream) {
  if (output == nullptr || target == nullptr || mask == nullptr || batch <= 0 || batch > 1024 ||
      (relative != 0 && relative != 1))
    return FL_INVALID_ARGUMENT;
  return unet_code(fl::unet_masked_mse(output, target, mask, batch, relative, loss, grad_output,
                                       static_cast<cudaStream_t>(stream)));
}

int fl_unet_block_residual_loss(const float* output, const float* input, int batch, float* loss, float* grad_output,
                                void* stream) {
  if (output == nullptr || input == nullptr || batch <= 0 || batch > 1024) return FL_INVALID_ARGUMENT;
  return unet_code(fl::unet_block_residual_loss(output, input, batch, loss, grad_output,
                                                static_cast<cudaStream_t>(stream)));
}

int fl_adam_step(float* params, const float* grads, float* m, float* v, uint64_t count, int step, float lr,
                 float beta1, float beta2, float eps, void* stream) {
  if (params == nullptr || grads == nullptr || m == nullptr || v == nullptr || step < 1 || !(lr > 0.0f) ||
      !(beta1 >= 0.0f && beta1 < 1.0f) || !(beta2 >= 0.0f && beta2 < 1.0f) || !(eps > 0.0f))
    return FL_INVALID_ARGUMENT;
  if (count == 0) return FL_OK;
  return unet_code(fl::adam_step(params, grads, m, v, (long long)count, step, lr, beta1, beta2, eps,
                                 static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
