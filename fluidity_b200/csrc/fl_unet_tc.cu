// Tensor-core inference of the learned block preconditioner: the 3x3x3
// convolutions as implicit GEMM on tcgen05 (BF16 operands from shared memory,
// FP32 accumulators in tensor memory), one CTA-local MMA stream per block.
//
// Activation layout (BF16, one copy per active block, zero pads kept zero):
// a D^3 tensor with C channels is C/8 channel groups, each a column of rows of
// 8 channels (16 bytes). Rows follow a padded box whose x and y pads are shared
// between neighbouring lines and planes: Px = Py = D+1, Pz = D+2, and cell
// (x,y,z) sits at row ((z+1) Py + (y+1)) Px + (x+1). A tap (dz,dy,dx) is then a
// constant row shift dz Py Px + dy Px + dx, so the A operand of one tap for 128
// consecutive output rows is the activation column itself, shifted: the shared
// memory descriptor (K-major, no swizzle) starts at that row, its 8-row groups
// 128 bytes apart (SBO) and its two 8-channel K halves one channel group apart
// (LBO). Rows that are pads produce garbage outputs, which the epilogue drops.
// The block's input window (8^3 + one-cell halo) uses Px = Py = Pz = 10.
//
// Per conv layer one persistent kernel: each CTA keeps the layer's packed
// weights in shared memory ([tap][K chunk][K half][Cout][8]), and per block it
// copies the input rows in, one thread issues tiles x 27 x K-chunks MMAs
// (M = 128, N = Cout, K = 16), a commit arrives on an mbarrier, and four warps
// read the accumulators back (tcgen05.ld 32x32b) for bias, ReLU and the store
// to the next layout. The 1x1 layers, pooling and upsampling run as small
// SIMT kernels on the same layouts; the last layer's epilogue also applies the
// 16->1 output layer and writes the correction into the solver's vector.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"
#include "fl_unet.h"

namespace fl {

namespace {

constexpr int kTcThreads = 160;  // warps 0-3 read TMEM lanes 32w..32w+31; warp 4 copies and issues MMAs
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at 1.9 GHz: mbarrier wait bound

struct PadGeom {
  int D, Px, Py, rows, r_lo, tiles;
};
// rows >= 128 * tiles + 2 * r_lo, so every shifted tile stays inside the column
__host__ __device__ constexpr PadGeom geom8() { return {8, 9, 9, 824, 91, 5}; }
__host__ __device__ constexpr PadGeom geom4() { return {4, 5, 5, 192, 31, 1}; }
__host__ __device__ constexpr PadGeom geom2() { return {2, 3, 3, 160, 13, 1}; }
__host__ __device__ constexpr PadGeom geom10() { return {8, 10, 10, 1120, 111, 7}; }

__device__ __forceinline__ int pad_row(const PadGeom& g, int x, int y, int z) {
  return ((z + 1) * g.Py + (y + 1)) * g.Px + (x + 1);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared memory matrix descriptor (sm_100 version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
}

// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One contiguous global -> shared copy through the bulk-copy engine (no
// multicast; this GPU's own memory), completing on `mbar` as transaction bytes.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// TMEM columns of one accumulator stage (a power of two, at least 32).
__host__ __device__ constexpr int tc_cols(int used) { return used <= 32 ? 32 : (used <= 64 ? 64 : (used <= 128 ? 128 : 256)); }

__device__ __forceinline__ void mbar_init_count(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait on an mbarrier phase: false after ~1 s without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 o;
  __nv_bfloat162 h;
  h = __floats2bfloat162_rn(v[0], v[1]);
  o.x = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[2], v[3]);
  o.y = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[4], v[5]);
  o.z = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[6], v[7]);
  o.w = *reinterpret_cast<uint32_t*>(&h);
  return o;
}

__device__ __forceinline__ void unpack8(uint4 u, float* v) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 f = __bfloat1622float2(h[k]);
    v[2 * k] = f.x;
    v[2 * k + 1] = f.y;
  }
}

enum ConvMode : int { kToPadded = 0, kToPlain = 1, kToCorrection = 2 };

struct ConvArgs {
  const uint4* in;        // [nb][in_groups][rows_in] rows of 8 BF16 channels
  const uint4* weights;   // packed [27][kc][2][N] rows of 8 BF16
  const float* bias;      // N
  uint4* out;             // kToPadded: [nb][N/8][rows_out]
  float* out_plain;       // kToPlain: [nb][D^3][N]
  int nb;
  // final layer (kToCorrection)
  const float* w_out;     // 16
  const float* b_out;     // 1
  const float* scale;     // per block
  const unsigned char* type;
  void* z;                // level-0 vector (RB layout), T
  int z_bf16;
  int z_add;              // 1: z += s y (the correction added to the V-cycle's), 0: z = s y
  int* error;             // set to 1 when an mbarrier wait gives up
};

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// One conv layer over all blocks. IN/OUT: geometry of the input columns and of
// the output layout (same D except for the valid first layer, whose input is
// the 10^3 window). KG: input channel groups (1 = the 2-channel window, whose
// second K half re-reads the first with zero weights). N: output channels.
//
// A CTA handles blocks blockIdx.x, blockIdx.x + gridDim.x, ... through a
// two-stage pipeline. Warp 4's first thread copies block k + 1's operand
// columns into one shared-memory stage (a bulk copy) while it issues block
// k's MMAs from the other stage into one of two TMEM accumulator stages;
// warps 0-3 (TMEM lanes 32w..32w+31) drain the other accumulator stage,
// block k - 1's, for bias, ReLU and the store. Barriers per stage: operands
// arrived (full), operands consumed by the MMAs (empty), accumulators written
// (accf), accumulators read (acce, one arrival per epilogue warp). Every wait
// is bounded (~1 s); a wait that gives up sets the error flag and its role
// stops, and the TMEM is released only after a final commit shows every
// issued MMA complete.
template <int KG, int N, int MODE, int IN_KIND, int OUT_KIND>
__global__ void __launch_bounds__(kTcThreads) k_conv_tc(ConvArgs a) {
  constexpr PadGeom IN = IN_KIND == 10 ? geom10() : (IN_KIND == 8 ? geom8() : (IN_KIND == 4 ? geom4() : geom2()));
  constexpr PadGeom OUT = OUT_KIND == 8 ? geom8() : (OUT_KIND == 4 ? geom4() : geom2());
  constexpr int KC = KG >= 2 ? KG / 2 : 1;
  constexpr int TILES = IN.tiles;
  constexpr int NCOLS = tc_cols(TILES * N);
  constexpr uint32_t W_BYTES = 27u * KC * 2u * N * 16u;
  constexpr uint32_t A_BYTES = (uint32_t)KG * IN.rows * 16u;
  constexpr uint32_t GROUP_BYTES = (uint32_t)IN.rows * 16u;
  constexpr uint32_t IDESC = instr_desc(128, N);
  static_assert(IN.rows >= 128 * TILES + 2 * IN.r_lo, "shifted tiles must stay inside the column");
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "M = 128 needs N in 16..256, multiple of 16");
  static_assert(W_BYTES % 16 == 0 && A_BYTES % 16 == 0, "bulk copies need 16-byte alignment and sizes");
  static_assert(2 * NCOLS <= 512, "two accumulator stages within the SM's TMEM");

  extern __shared__ __align__(128) unsigned char smem[];
  uint4* w_s = reinterpret_cast<uint4*>(smem);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + W_BYTES + 2 * A_BYTES);  // 9 barriers
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 9);
  enum { kFull = 0, kEmpty = 2, kAccF = 4, kAccE = 6, kDrain = 8 };

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (uint32_t i = tid; i < W_BYTES / 16; i += kTcThreads) w_s[i] = a.weights[i];
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 9; ++k) mbar_init_count(smem_u32(bars + k), (k == kAccE || k == kAccE + 1) ? 4u : 1u);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)(2 * NCOLS)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();  // the weights, stored by every thread, before the MMAs read them
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  const uint32_t w_addr = smem_u32(w_s), a_addr = smem_u32(smem + W_BYTES);
  auto bar = [&](int k) { return smem_u32(bars + k); };
  // This CTA's blocks: blockIdx.x, blockIdx.x + gridDim.x, ..., skipping blocks whose
  // window holds no residual (scale 0: their correction is zero whatever the network
  // computes). Both roles walk the same sequence with their own cursor.
  auto next_block = [&](int& j) -> int {
    for (;;) {
      const int b = (int)blockIdx.x + j * (int)gridDim.x;
      if (b >= a.nb) return -1;
      ++j;
      if (a.scale == nullptr || __ldg(&a.scale[b]) != 0.0f) return b;
    }
  };

  if (warp == 4) {
    if (lane == 0) {
      bool ok = true;
      int issued = -1, arrived = -1;  // last block (in this CTA's sequence) copied / waited for
      auto copy = [&](int k, int blk) {
        const int st = k & 1;
        bulk_copy_g2s(a_addr + (uint32_t)st * A_BYTES, a.in + (size_t)blk * (KG * IN.rows), A_BYTES,
                      bar(kFull + st));
        issued = k;
      };
      int cursor = 0;
      int bk = next_block(cursor);                 // block k of the sequence
      int bn = bk >= 0 ? next_block(cursor) : -1;  // block k + 1
      if (bk >= 0) copy(0, bk);
      for (int k = 0; bk >= 0 && ok; ++k) {
        const int st = k & 1;
        const uint32_t u = (uint32_t)(k >> 1);
        if (bn >= 0) {  // the other stage is free once block k - 1's MMAs are done
          if (k >= 1 && !(ok = mbar_wait(bar(kEmpty + (st ^ 1)), (uint32_t)((k - 1) >> 1) & 1u))) break;
          copy(k + 1, bn);
        }
        if (!(ok = mbar_wait(bar(kFull + st), u & 1u))) break;
        arrived = k;
        if (k >= 2 && !(ok = mbar_wait(bar(kAccE + st), (u - 1u) & 1u))) break;
        fence_after_sync();
        // The descriptors' start-address field (bits 0-13) counts 16-byte rows,
        // so each tap's operands are the tile's base descriptors plus constant
        // row offsets (every address stays below 256 KB: no carry out of the
        // field; the static_assert above keeps shifted rows inside the column).
        const uint64_t a0 =
            smem_desc(a_addr + (uint32_t)st * A_BYTES + (uint32_t)IN.r_lo * 16u, KG >= 2 ? GROUP_BYTES : 0u, 128u);
        const uint64_t b0 = smem_desc(w_addr, N * 16u, 128u);
#pragma unroll 1
        for (int t = 0; t < TILES; ++t) {
          const uint64_t at = a0 + (uint64_t)(128 * t);
          const uint32_t dt = tmem + (uint32_t)(st * NCOLS + t * N);
#pragma unroll
          for (int tap = 0; tap < 27; ++tap) {
            const int shift = ((tap / 9 - 1) * IN.Py + ((tap / 3) % 3 - 1)) * IN.Px + (tap % 3 - 1);
#pragma unroll
            for (int kc = 0; kc < KC; ++kc) {
              const uint64_t ad = at + (uint64_t)(int64_t)(shift + 2 * kc * IN.rows);
              const uint64_t bd = b0 + (uint64_t)((tap * KC + kc) * 2 * N);
              mma_bf16(dt, ad, bd, IDESC, (tap | kc) != 0 ? 1u : 0u);
            }
          }
        }
        mma_commit(bar(kEmpty + st));
        mma_commit(bar(kAccF + st));
        bk = bn;
        bn = bk >= 0 ? next_block(cursor) : -1;
      }
      if (!ok) atomicExch(a.error, 1);
      // after a wait gave up: one more bounded wait for each copy still in flight
      for (int j = arrived + 1; j <= issued; ++j) mbar_wait(bar(kFull + (j & 1)), (uint32_t)(j >> 1) & 1u);
      mma_commit(bar(kDrain));  // arrives once every MMA this thread issued has completed
      if (!mbar_wait(bar(kDrain), 0u)) atomicExch(a.error, 1);
    }
  } else {
    int cursor = 0;
    for (int k = 0;; ++k) {
      const int b = next_block(cursor);
      if (b < 0) break;
      const int st = k & 1;
      const uint32_t u = (uint32_t)(k >> 1);
      if (!mbar_wait(bar(kAccF + st), u & 1u)) {
        if (lane == 0) atomicExch(a.error, 1);
        break;
      }
      fence_after_sync();
      // warp w owns tile rows 32w..32w+31
#pragma unroll 1
      for (int t = 0; t < TILES; ++t) {
        const int r = IN.r_lo + 128 * t + 32 * warp + lane;
        const int px = r % IN.Px, py = (r / IN.Px) % IN.Py, pz = r / (IN.Px * IN.Py);
        const bool interior = px >= 1 && px <= IN.D && py >= 1 && py <= IN.D && pz >= 1 && pz <= IN.D;
        const int x = px - 1, y = py - 1, z = pz - 1;
        float acc[N];
#pragma unroll
        for (int c = 0; c < N; c += 16) {
          float v[16];
          tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(st * NCOLS + t * N + c), v);
#pragma unroll
          for (int q = 0; q < 16; ++q) acc[c + q] = fmaxf(v[q] + __ldg(&a.bias[c + q]), 0.0f);
        }
        if (!interior) continue;
        if (MODE == kToPadded) {
          const int ro = pad_row(OUT, x, y, z);
          uint4* dst = a.out + (size_t)b * (N / 8) * OUT.rows;
#pragma unroll
          for (int g = 0; g < N / 8; ++g) dst[g * OUT.rows + ro] = pack8(acc + 8 * g);
        } else if (MODE == kToPlain) {
          float* dst = a.out_plain + ((size_t)b * IN.D * IN.D * IN.D + (z * IN.D + y) * IN.D + x) * N;
#pragma unroll
          for (int c = 0; c < N; c += 4)
            *reinterpret_cast<float4*>(dst + c) = make_float4(acc[c], acc[c + 1], acc[c + 2], acc[c + 3]);
        } else {
          float yv = __ldg(a.b_out);
#pragma unroll
          for (int c = 0; c < N; ++c) yv = fmaf(__ldg(&a.w_out[c]), acc[c], yv);
          const int l = (z * 8 + y) * 8 + x;
          const float v = a.type[b * 512 + l] == 1 ? a.scale[b] * yv : 0.0f;
          const int zi = b * 512 + rb_of(l);
          if (a.z_bf16) {
            __nv_bfloat16* zp = reinterpret_cast<__nv_bfloat16*>(a.z) + zi;
            *zp = __float2bfloat16_rn(a.z_add ? __bfloat162float(*zp) + v : v);
          } else {
            float* zp = reinterpret_cast<float*>(a.z) + zi;
            *zp = a.z_add ? *zp + v : v;
          }
        }
      }
      // this warp's accumulator reads are done (tmem_ld16 waits for them)
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(kAccE + st));
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)(2 * NCOLS)));
}

// Input window of block b in the 10^3 layout (one channel group: residual / s,
// cell mask, six zero channels) and the block scale s (max |residual| over the window).
// z_zero (not null when the network's output replaces z): a block whose window
// holds no residual is skipped by every layer, so its correction, zero, is
// written here.
template <typename T>
__global__ void __launch_bounds__(512) k_tc_gather(GridView g, const float* __restrict__ r_rb,
                                                   const unsigned char* __restrict__ type, uint4* __restrict__ x,
                                                   float* __restrict__ scale, T* __restrict__ z_zero) {
  constexpr PadGeom W = geom10();
  __shared__ float red[16];
  const int b = blockIdx.x;
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
  if (sc == 0.0f && z_zero != nullptr) z_zero[(size_t)b * 512 + threadIdx.x] = static_cast<T>(0.0f);
  uint4* dst = x + (size_t)b * W.rows;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int i = threadIdx.x + 512 * k;
    if (i < 1000) {  // window row (hz+1, hy+1, hx+1) == i in the 10^3 layout
      float v[8] = {sc > 0.0f ? rv[k] / sc : 0.0f, mv[k], 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      dst[i] = pack8(v);
    }
  }
  if (threadIdx.x == 0) scale[b] = sc;
}

// 2x average pooling between padded layouts (G channel groups). One thread per (block, coarse cell, group).
template <int DIN, int G>
__global__ void k_tc_pool(const uint4* __restrict__ in, uint4* __restrict__ out, int nb) {
  constexpr PadGeom I = DIN == 8 ? geom8() : geom4();
  constexpr PadGeom O = DIN == 8 ? geom4() : geom2();
  constexpr int H = DIN / 2, H3 = H * H * H;
  const long long total = (long long)nb * H3 * G;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int gi = (int)(i % G);
    const int c = (int)((i / G) % H3);
    const long long b = i / ((long long)G * H3);
    const int x = c % H, y = (c / H) % H, z = c / (H * H);
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const uint4* src = in + (size_t)b * G * I.rows + (size_t)gi * I.rows;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      float v[8];
      unpack8(src[pad_row(I, 2 * x + (k & 1), 2 * y + ((k >> 1) & 1), 2 * z + (k >> 2))], v);
#pragma unroll
      for (int j = 0; j < 8; ++j) s[j] += v[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) s[j] *= 0.125f;
    out[(size_t)b * G * O.rows + (size_t)gi * O.rows + pad_row(O, x, y, z)] = pack8(s);
  }
}

// u2 = relu(up(W_u2 bt + b_u2) + s2) at 4^3 (32 channels): one CTA per block,
// bt is [8 cells][64] FP32, s2 and u2 are 4-group padded 4^3 columns.
__global__ void __launch_bounds__(256) k_tc_upadd2(const float* __restrict__ bt, const uint4* __restrict__ s2,
                                                   const float* __restrict__ w, const float* __restrict__ bias,
                                                   uint4* __restrict__ u2) {
  constexpr PadGeom L = geom4();
  __shared__ float c2[8][32];
  __shared__ float wt[64][32];  // the 1x1 weights transposed: a warp's 32 output channels read one row
  __shared__ float in[8][64];
  const int b = blockIdx.x;
  for (int i = threadIdx.x; i < 64 * 32; i += 256) wt[i & 63][i >> 6] = __ldg(&w[i]);  // w[co][ci], coalesced
  for (int i = threadIdx.x; i < 8 * 64; i += 256) in[i >> 6][i & 63] = bt[(size_t)b * 8 * 64 + i];
  __syncthreads();
  {
    const int cell = threadIdx.x >> 5, co = threadIdx.x & 31;
    float acc = bias[co];
#pragma unroll 8
    for (int ci = 0; ci < 64; ++ci) acc = fmaf(wt[ci][co], in[cell][ci], acc);
    c2[cell][co] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 64 * 4; i += 256) {  // (fine cell, group)
    const int gi = i & 3, c = i >> 2;
    const int x = c & 3, y = (c >> 2) & 3, z = c >> 4;
    const int parent = ((z >> 1) * 2 + (y >> 1)) * 2 + (x >> 1);
    const size_t idx = (size_t)b * 4 * L.rows + (size_t)gi * L.rows + pad_row(L, x, y, z);
    float v[8];
    unpack8(s2[idx], v);
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = fmaxf(v[j] + c2[parent][8 * gi + j], 0.0f);
    u2[idx] = pack8(v);
  }
}

// u1 = relu(up(W_u1 d2 + b_u1) + s1) at 8^3 (16 channels): one CTA per block.
__global__ void __launch_bounds__(256) k_tc_upadd1(const uint4* __restrict__ d2, const uint4* __restrict__ s1,
                                                   const float* __restrict__ w, const float* __restrict__ bias,
                                                   uint4* __restrict__ u1) {
  constexpr PadGeom L4 = geom4();
  constexpr PadGeom L8 = geom8();
  __shared__ float din[64][33];
  __shared__ float c1[64][16];
  __shared__ float wt[32][16];  // the 1x1 weights transposed (w[co][ci] -> wt[ci][co])
  const int b = blockIdx.x;
  for (int i = threadIdx.x; i < 16 * 32; i += 256) wt[i & 31][i >> 5] = __ldg(&w[i]);
  for (int i = threadIdx.x; i < 64 * 4; i += 256) {
    const int gi = i & 3, c = i >> 2;
    const int x = c & 3, y = (c >> 2) & 3, z = c >> 4;
    float v[8];
    unpack8(d2[(size_t)b * 4 * L4.rows + (size_t)gi * L4.rows + pad_row(L4, x, y, z)], v);
#pragma unroll
    for (int j = 0; j < 8; ++j) din[c][8 * gi + j] = v[j];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 64 * 16; i += 256) {
    const int co = i & 15, c = i >> 4;
    float acc = bias[co];
#pragma unroll 8
    for (int ci = 0; ci < 32; ++ci) acc = fmaf(wt[ci][co], din[c][ci], acc);
    c1[c][co] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 512 * 2; i += 256) {
    const int gi = i & 1, c = i >> 1;
    const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
    const int parent = ((z >> 1) * 4 + (y >> 1)) * 4 + (x >> 1);
    const size_t idx = (size_t)b * 2 * L8.rows + (size_t)gi * L8.rows + pad_row(L8, x, y, z);
    float v[8];
    unpack8(s1[idx], v);
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = fmaxf(v[j] + c1[parent][8 * gi + j], 0.0f);
    u1[idx] = pack8(v);
  }
}

// Packs one FP32 conv layer (w[co][ci][27]) into [27][kc][2][cout][8] BF16 with
// input channels padded to 16 * kc (zeros).
__global__ void k_pack_conv(const float* __restrict__ w, int cin, int cout, int kc, __nv_bfloat16* __restrict__ out) {
  const int total = 27 * kc * 2 * cout * 8;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int j = i & 7;
    const int n = (i >> 3) % cout;
    const int kh = (i / (8 * cout)) & 1;
    const int k = (i / (16 * cout)) % kc;
    const int tap = i / (16 * cout * kc);
    const int ci = k * 16 + kh * 8 + j;
    out[i] = __float2bfloat16_rn(ci < cin ? w[((size_t)n * cin + ci) * 27 + tap] : 0.0f);
  }
}

// CTAs of one layer per SM: two TMEM accumulator stages each, within the
// SM's 512 columns.
template <int KG, int N, int MODE, int IN_KIND, int OUT_KIND>
constexpr int conv_ctas_per_sm() {
  constexpr PadGeom IN = IN_KIND == 10 ? geom10() : (IN_KIND == 8 ? geom8() : (IN_KIND == 4 ? geom4() : geom2()));
  return 512 / (2 * tc_cols(IN.tiles * N));
}

template <int KG, int N, int MODE, int IN_KIND, int OUT_KIND>
constexpr size_t conv_smem() {
  constexpr PadGeom IN = IN_KIND == 10 ? geom10() : (IN_KIND == 8 ? geom8() : (IN_KIND == 4 ? geom4() : geom2()));
  constexpr int KC = KG >= 2 ? KG / 2 : 1;
  constexpr size_t bytes = 27u * KC * 2u * N * 16u + 2u * (size_t)KG * IN.rows * 16u + 9 * 8 + 8;
  // Ask for enough shared memory that one more CTA than the TMEM allows does
  // not fit the SM (228 KB, 1 KB reserved per CTA), so no TMEM allocation
  // waits for another CTA's release.
  constexpr int cap = conv_ctas_per_sm<KG, N, MODE, IN_KIND, OUT_KIND>();
  constexpr size_t floor_bytes = (size_t)(233472 / (cap + 1)) - 1024 + 16;
  return bytes < floor_bytes ? floor_bytes : bytes;
}

template <int KG, int N, int MODE, int IN_KIND, int OUT_KIND>
cudaError_t launch_conv(const ConvArgs& a, int sms, cudaStream_t s) {
  constexpr size_t smem = conv_smem<KG, N, MODE, IN_KIND, OUT_KIND>();
  auto kern = k_conv_tc<KG, N, MODE, IN_KIND, OUT_KIND>;
  static unsigned long long configured = 0;
  if (first_on_device(configured))
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int by_smem = (int)(233472 / (smem + 1024));
  const int cap = conv_ctas_per_sm<KG, N, MODE, IN_KIND, OUT_KIND>();
  const int per_sm = by_smem < cap ? by_smem : cap;
  const int grid = a.nb < sms * per_sm ? a.nb : sms * per_sm;
  ++g_kernel_launches;
  kern<<<grid, kTcThreads, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

// Per-block element counts (16-byte rows) of the inference activations.
UNetTcLayout unet_tc_layout() {
  UNetTcLayout L{};
  long long off = 0;
  auto take = [&](long long rows16) {
    const long long o = off;
    off += rows16;
    return o;
  };
  L.x = take(geom10().rows);
  L.t8 = take(2 * geom8().rows);
  L.s1 = take(2 * geom8().rows);
  L.p1 = take(2 * geom4().rows);
  L.e2a = take(4 * geom4().rows);
  L.s2 = take(4 * geom4().rows);
  L.p2 = take(4 * geom2().rows);
  L.u2 = take(4 * geom4().rows);
  L.d2 = take(4 * geom4().rows);
  L.rows_per_block = off;
  L.bt_floats_per_block = 8 * 64;
  // packed weights (BF16 elements), conv layers e1a e1b e2a e2b bt d2 d1
  const int cin[7] = {2, 16, 16, 32, 32, 32, 16}, cout[7] = {16, 16, 32, 32, 64, 32, 16};
  long long w = 0;
  for (int k = 0; k < 7; ++k) {
    const int kc = cin[k] >= 32 ? 2 : 1;
    L.w_off[k] = w;
    w += 27ll * kc * 2 * cout[k] * 8;
  }
  L.w_total = w;
  return L;
}

cudaError_t unet_tc_pack(const float* params, __nv_bfloat16* packed, cudaStream_t s) {
  const UNetLayout P = unet_layout();
  const UNetTcLayout T = unet_tc_layout();
  const int layer[7] = {0, 1, 2, 3, 4, 6, 8};
  for (int k = 0; k < 7; ++k) {
    const int l = layer[k];
    const int kc = P.cin[l] >= 32 ? 2 : 1;
    ++g_kernel_launches;
    k_pack_conv<<<64, 256, 0, s>>>(params + P.offset[l], P.cin[l], P.cout[l], kc, packed + T.w_off[k]);
  }
  return cudaGetLastError();
}

// z = s * U(r / s) per active block through the tensor-core kernels
// (accumulate: z += s * U(r / s)).
template <typename T>
cudaError_t unet_tc_apply(const GridView& g, const float* params, const __nv_bfloat16* packed, uint4* act,
                          long long cap, float* bt, float* scale, const unsigned char* type, const float* r_rb, T* z,
                          int* error, int sms, cudaStream_t s, bool accumulate) {
  const int nb = g.nb;
  if (nb <= 0) return cudaSuccess;
  if (nb > cap) return cudaErrorInvalidValue;
  const UNetLayout P = unet_layout();
  const UNetTcLayout L = unet_tc_layout();
  // per-tensor bases: tensors are stored tensor-major ([tensor][block][rows]) with
  // the allocated capacity as stride, so every column keeps its place (and its
  // zero pads) whatever the active block count of a call
  auto base = [&](long long off) { return act + off * cap; };
  auto wp = [&](int k) { return reinterpret_cast<const uint4*>(packed + L.w_off[k]); };
  ++g_kernel_launches;
  k_tc_gather<T><<<nb, 512, 0, s>>>(g, r_rb, type, base(L.x), scale, accumulate ? nullptr : z);
  ConvArgs a{};
  a.nb = nb;
  a.error = error;
  a.scale = scale;  // every layer skips the blocks without residual
  cudaError_t e;
  // e1a: window (1 group) -> t8
  a.in = base(L.x); a.weights = wp(0); a.bias = params + P.bias[0]; a.out = base(L.t8);
  if ((e = launch_conv<1, 16, kToPadded, 10, 8>(a, sms, s)) != cudaSuccess) return e;
  // e1b: t8 -> s1
  a.in = base(L.t8); a.weights = wp(1); a.bias = params + P.bias[1]; a.out = base(L.s1);
  if ((e = launch_conv<2, 16, kToPadded, 8, 8>(a, sms, s)) != cudaSuccess) return e;
  g_kernel_launches += 1;
  k_tc_pool<8, 2><<<(nb * 64 * 2 + 255) / 256, 256, 0, s>>>(base(L.s1), base(L.p1), nb);
  // e2a: p1 -> e2a
  a.in = base(L.p1); a.weights = wp(2); a.bias = params + P.bias[2]; a.out = base(L.e2a);
  if ((e = launch_conv<2, 32, kToPadded, 4, 4>(a, sms, s)) != cudaSuccess) return e;
  // e2b: e2a -> s2
  a.in = base(L.e2a); a.weights = wp(3); a.bias = params + P.bias[3]; a.out = base(L.s2);
  if ((e = launch_conv<4, 32, kToPadded, 4, 4>(a, sms, s)) != cudaSuccess) return e;
  g_kernel_launches += 1;
  k_tc_pool<4, 4><<<(nb * 8 * 4 + 255) / 256, 256, 0, s>>>(base(L.s2), base(L.p2), nb);
  // bt: p2 -> bt (plain FP32)
  a.in = base(L.p2); a.weights = wp(4); a.bias = params + P.bias[4]; a.out = nullptr; a.out_plain = bt;
  if ((e = launch_conv<4, 64, kToPlain, 2, 2>(a, sms, s)) != cudaSuccess) return e;
  g_kernel_launches += 1;
  k_tc_upadd2<<<nb, 256, 0, s>>>(bt, base(L.s2), params + P.offset[5], params + P.bias[5], base(L.u2));
  // d2: u2 -> d2
  a.in = base(L.u2); a.weights = wp(5); a.bias = params + P.bias[6]; a.out = base(L.d2); a.out_plain = nullptr;
  if ((e = launch_conv<4, 32, kToPadded, 4, 4>(a, sms, s)) != cudaSuccess) return e;
  g_kernel_launches += 1;
  k_tc_upadd1<<<nb, 256, 0, s>>>(base(L.d2), base(L.s1), params + P.offset[7], params + P.bias[7], base(L.t8));
  // d1 + output layer: u1 (in t8) -> z
  a.in = base(L.t8); a.weights = wp(6); a.bias = params + P.bias[8]; a.out = nullptr;
  a.w_out = params + P.offset[9]; a.b_out = params + P.bias[9]; a.type = type; a.z = z;
  a.z_bf16 = sizeof(T) == 2;
  a.z_add = accumulate ? 1 : 0;
  return launch_conv<2, 16, kToCorrection, 8, 8>(a, sms, s);
}

template cudaError_t unet_tc_apply<float>(const GridView&, const float*, const __nv_bfloat16*, uint4*, long long,
                                          float*, float*, const unsigned char*, const float*, float*, int*, int,
                                          cudaStream_t, bool);
template cudaError_t unet_tc_apply<__nv_bfloat16>(const GridView&, const float*, const __nv_bfloat16*, uint4*,
                                                  long long, float*, float*, const unsigned char*, const float*,
                                                  __nv_bfloat16*, int*, int, cudaStream_t, bool);

}  // namespace fl
