// Internal device-side layout and helpers for the B200 liquid-step kernels.
//
// HBM layout (one GPU, everything resident):
//   * Sparse MAC grid in 8^3-cell blocks. Active blocks are the blocks that hold
//     particles plus a one-block ring; their ordinals follow (z,y,x) block order.
//     A dense table over the domain's block lattice maps block coordinates to
//     ordinals (-1 = inactive). nbr27[b*27 + (dz+1)*9 + (dy+1)*3 + (dx+1)] is the
//     ordinal of the neighbouring block, -1 if inactive, -2 outside the lattice.
//   * Face fields are three FP32 arrays (one per normal axis) of nb*512 entries;
//     the face at lattice index (i,j,k) is the low face of cell (i,j,k) and is
//     stored in that cell's block at local (z*64 + y*8 + x). This mirrors the
//     reference's owned low-face convention (sparse_mac_grid_3d.cc:388-409) with
//     8^3 instead of 4^3 blocks.
//   * Particles are FP32 SoA (x,y,z, vx,vy,vz, 9 affine entries: 60 B/particle),
//     sorted by (block ordinal, local cell) each step; cell_start[nb*512+1]
//     gives each cell's particle range.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fl {

// Host-side once-per-device flag: true the first time it is asked for the
// current device (bit d of `mask` records device d). Set-up such as a
// function's shared-memory attribute applies to the current device only, so
// a process that drives several GPUs repeats it on each.
inline bool first_on_device(unsigned long long& mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return true;
  }
  const unsigned long long bit = 1ull << dev;
  if (mask & bit) return false;
  mask |= bit;
  return true;
}

constexpr int kBlockAxis = 8;
constexpr int kBlockCells = 512;
constexpr int kTileFaces = 1100;  // 11 x 10 x 10 faces per normal component

// Status codes mirror absl::StatusCode numbering used by the reference.
enum Status : int {
  kOk = 0,
  kInvalidArgument = 3,
  kResourceExhausted = 8,
  kFailedPrecondition = 9,
  kAborted = 10,
  kOutOfRange = 11,
  kInternal = 13,
};

// Device error report: written with atomics by failing lanes, read after sync.
struct DeviceReport {
  int compiled_architecture;
  int error;
  unsigned long long first_bad_index;
};

struct GridView {
  float origin[3];
  float h;
  float inv_h;
  int nb;               // active blocks
  int blo[3];           // lattice origin (block coordinates)
  int bdim[3];          // lattice extent (blocks)
  const int* table;     // bdim product entries
  const int* coord;     // nb * 3 absolute block coordinates
  const int* nbr27;     // nb * 27
  int solid_lo[3];      // cells with index < solid_lo or > solid_hi are solid
  int solid_hi[3];
};

struct ParticlesView {
  float* x[3];
  float* v[3];
  float* c[9];
  float* mass;  // nullptr: uniform mass
  unsigned long long count;
};

__device__ __forceinline__ int nbr_index(int dx, int dy, int dz) { return (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1); }

__device__ __forceinline__ int floor_div8(int v) { return v >= 0 ? (v >> 3) : -((-v + 7) >> 3); }

// Lattice coordinate of a world position in FP32 cell units.
__device__ __forceinline__ float lattice_coord(const GridView& g, float x, int d) {
  return (x - g.origin[d]) * g.inv_h;
}

__device__ __forceinline__ void report_error(DeviceReport* r, int code, unsigned long long index) {
  if (r == nullptr) return;
  if (atomicCAS(&r->error, 0, code) == 0) {
    atomicExch(&r->first_bad_index, index);
  }
}

__device__ __forceinline__ int compiled_arch() {
#ifdef __CUDA_ARCH__
  return __CUDA_ARCH__;
#else
  return 0;
#endif
}

// Level-0 solver layout (red-black): inside each block the 256 cells of colour
// c = (x+y+z)&1 occupy [c*256, c*256+256) in (z, y, x/2) order, so a colour
// sweep reads and writes contiguous memory. Face and particle arrays keep the
// natural (z*64 + y*8 + x) order.
__device__ __forceinline__ int rb_of(int l) {
  const int x = l & 7, y = (l >> 3) & 7, z = l >> 6;
  return (((x + y + z) & 1) << 8) | (z << 5) | (y << 2) | (x >> 1);
}
__device__ __forceinline__ int nat_of(int r) {
  const int c = r >> 8, j = r & 255;
  const int z = j >> 5, y = (j >> 2) & 7, xh = j & 3;
  return (z << 6) | (y << 3) | (2 * xh + ((y + z + c) & 1));
}
__device__ __forceinline__ int rb_id(int natural_id) {
  return natural_id < 0 ? natural_id : ((natural_id & ~511) | rb_of(natural_id & 511));
}

// Storage helpers for FP32 or BF16 V-cycle vectors.
template <typename T>
__device__ __forceinline__ float ld(const T* p) {
  return static_cast<float>(*p);
}
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}
// Programmatic dependent launch: blocks until the grid this kernel depends on
// has completed and its writes are visible. A kernel launched with
// programmatic stream serialization calls it first, before any early return;
// launched without that attribute, it returns at once.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Four consecutive values from a 4-element-aligned position (16 B for FP32, 8 B for BF16).
template <typename T>
__device__ __forceinline__ void ld4(const T* p, float v[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
}
template <>
__device__ __forceinline__ void ld4<__nv_bfloat16>(const __nv_bfloat16* p, float v[4]) {
  const uint2 u = *reinterpret_cast<const uint2*>(p);
  const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  v[0] = lo.x;
  v[1] = lo.y;
  v[2] = hi.x;
  v[3] = hi.y;
}
template <typename T>
__device__ __forceinline__ void st_T(T* p, float v) {
  *p = static_cast<T>(v);
}
template <>
__device__ __forceinline__ void st_T<__nv_bfloat16>(__nv_bfloat16* p, float v) {
  *p = __float2bfloat16_rn(v);
}

// v as stored in T and read back (the value a sweep that stores v leaves for the next one).
template <typename T>
__device__ __forceinline__ float round_T(float v) {
  return static_cast<float>(static_cast<T>(v));
}
template <>
__device__ __forceinline__ float round_T<__nv_bfloat16>(float v) {
  return __bfloat162float(__float2bfloat16_rn(v));
}

// Warp + block reduction of doubles (deterministic order for a fixed launch shape).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int kThreads>
__device__ __forceinline__ double block_sum(double v, double* smem) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < kThreads / 32 ? smem[lane] : 0.0;
    t = warp_sum(t);
  }
  return t;  // valid in warp 0
}

}  // namespace fl
