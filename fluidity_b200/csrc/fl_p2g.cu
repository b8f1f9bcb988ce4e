// APIC particle-to-grid transfer on the 8^3-block MAC grid.
//
// Semantics follow DepositMac3D (native/src/transfers_3d.cc:139-145) and
// AccumulateMacParticleComponent (native/src/mac_deposit_3d_internal.h:39-75):
// for each normal component a and each of the 27 quadratic B-spline nodes,
//   mass_f     += w * m
//   momentum_f += w * m * (v_a + C_a . (x_f - x_p))
// with the stencil of BuildCheckedAxisStencil (sparse_mac_grid_3d.cc:266-310).
// The fused epilogue applies NormalizeCore (liquid_boundary_transfer_3d.cc:
// 462-515), ApplyForces (liquid_substep_3d_cpu.cc:156-178) and the stationary
// wall condition.
//
// B200 design. One CTA per active 8^3 block, one thread per cell. Particles
// are sorted by cell, so a thread walks its own cell's particles and
// accumulates into registers: along the normal axis a particle of the cell
// touches nodes cell-1..cell+1 or cell..cell+2, so 4 x 3 x 3 = 36 slots per
// channel cover every particle of the cell with static register indexing.
// Register partials go to shared memory ([slot][cell] mass/momentum pairs); each tile node
// then sums its (at most 36) contributing (cell, slot) entries in a fixed
// order. The 11x10x10 tile (normal extent 11, transverse 10) is written to a
// per-block scratch tile and a second kernel sums, for every owned face, the
// tiles of the (at most 8) blocks whose halo covers it, again in a fixed order.
// No floating-point atomics are used anywhere, so the result is bitwise
// reproducible run to run for a given particle order (the stable sort fixes it).
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kP2GThreads = 512;
constexpr int kSlots = 36;

template <int A>
__device__ __forceinline__ int slot_index(int sx, int sy, int sz) {
  constexpr int ex = A == 0 ? 4 : 3, ey = A == 1 ? 4 : 3;
  return (sz * ey + sy) * ex + sx;
}

// Axis factors for one particle coordinate. For the normal axis, 4 slots with
// node = cell - 1 + s (one slot is zero); for transverse axes, 3 slots with
// anchor cell - 1 + s + 1/2. affine[s] = C_a,d * (anchor_s - X) * h.
template <bool kNormal>
__device__ __forceinline__ void axis_factors(float X, int cell, float h, float cad, float w[4], float affine[4]) {
  if (kNormal) {
    const float first = floorf(X - 0.5f);
    const bool shifted = first > (float)(cell - 1);  // first node is the cell itself
    const float dl = X - (first + 0.5f);
    const float dr = fabsf(X - (first + 1.5f));
    const float c = X - (first + 1.0f);
    const float w0 = 0.5f * dr * dr, w1 = 0.75f - c * c, w2 = 0.5f * dl * dl;
    w[0] = shifted ? 0.0f : w0;
    w[1] = shifted ? w0 : w1;
    w[2] = shifted ? w1 : w2;
    w[3] = shifted ? w2 : 0.0f;
#pragma unroll
    for (int s = 0; s < 4; ++s) affine[s] = cad * (((float)(cell - 1 + s) - X) * h);
  } else {
    const float f = X - (float)cell;
    const float dr = fabsf(1.0f - f);
    const float c = f - 0.5f;
    w[0] = 0.5f * dr * dr;
    w[1] = 0.75f - c * c;
    w[2] = 0.5f * f * f;
    w[3] = 0.0f;
#pragma unroll
    for (int s = 0; s < 3; ++s) affine[s] = cad * (((float)(cell - 1 + s) + 0.5f - X) * h);
    affine[3] = 0.0f;
  }
}

template <int A>
__device__ __forceinline__ void p2g_component(const GridView& g, const ParticlesView& p, const unsigned int* order,
                                              int pbeg, int pend, const int cell[3], float2* part, int t,
                                              DeviceReport* rep) {
  constexpr int D1 = A == 0 ? 1 : 0;
  constexpr int D2 = A == 2 ? 1 : 2;
  // Accumulators in normal-axis slot pairs: entry (k * 3 + j) * 2 + hp holds
  // normal slots 2hp (x) and 2hp + 1 (y) of transverse node (j, k). Each pair
  // is updated by one packed FP32 FMA (fma.rn.f32x2), which rounds every lane
  // exactly as fmaf does, so the sums are bitwise those of the scalar form.
  float2 accW[kSlots / 2], accQ[kSlots / 2];
#pragma unroll
  for (int s = 0; s < kSlots / 2; ++s) {
    accW[s] = make_float2(0.0f, 0.0f);
    accQ[s] = make_float2(0.0f, 0.0f);
  }
  const float h = g.h;
  // The particle of cell-order slot q, with the next slot's entry loaded one
  // iteration ahead so the order lookup overlaps the particle loads.
  int next = order != nullptr && pbeg < pend ? (int)__ldg(&order[pbeg]) : pbeg;
  for (int q = pbeg; q < pend; ++q) {
    const int i = next;
    next = order != nullptr ? (q + 1 < pend ? (int)__ldg(&order[q + 1]) : 0) : q + 1;
    float X[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) X[d] = lattice_coord(g, __ldg(&p.x[d][i]), d);
    const float m = p.mass ? __ldg(&p.mass[i]) : 1.0f;
    const float va = __ldg(&p.v[A][i]);
    float wa[4], ta[4], w1[4], t1[4], w2[4], t2[4];
    axis_factors<true>(X[A], cell[A], h, __ldg(&p.c[3 * A + A][i]), wa, ta);
    axis_factors<false>(X[D1], cell[D1], h, __ldg(&p.c[3 * A + D1][i]), w1, t1);
    axis_factors<false>(X[D2], cell[D2], h, __ldg(&p.c[3 * A + D2][i]), w2, t2);
    if (!(isfinite(m) && isfinite(va))) report_error(rep, kInvalidArgument, (unsigned long long)i);
    // Per node: W += wa*P and Q += wa*(P*q12) + (wa*ta)*P, with wa the
    // mass-scaled normal weight, P the transverse weight product and q12 = v_a
    // plus the transverse affine terms (v_a + t1[j] formed once per j).
    const float2 m2 = make_float2(m, m);
    const float2 wa2[2] = {__fmul2_rn(m2, make_float2(wa[0], wa[1])), __fmul2_rn(m2, make_float2(wa[2], wa[3]))};
    const float2 wta2[2] = {__fmul2_rn(wa2[0], make_float2(ta[0], ta[1])),
                            __fmul2_rn(wa2[1], make_float2(ta[2], ta[3]))};
    float q1[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) q1[j] = va + t1[j];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float P = w1[j] * w2[k];
        const float PQ = P * (q1[j] + t2[k]);
        const float2 P2 = make_float2(P, P), PQ2 = make_float2(PQ, PQ);
#pragma unroll
        for (int hp = 0; hp < 2; ++hp) {
          const int e = (k * 3 + j) * 2 + hp;
          accW[e] = __ffma2_rn(wa2[hp], P2, accW[e]);
          accQ[e] = __ffma2_rn(wa2[hp], PQ2, __ffma2_rn(wta2[hp], P2, accQ[e]));
        }
      }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int slot = A == 0 ? slot_index<A>(s, j, k) : A == 1 ? slot_index<A>(j, s, k) : slot_index<A>(j, k, s);
        const int e = (k * 3 + j) * 2 + (s >> 1);
        part[slot * kP2GThreads + t] =
            (s & 1) ? make_float2(accW[e].y, accQ[e].y) : make_float2(accW[e].x, accQ[e].x);
      }
}

template <int A>
__device__ __forceinline__ void reduce_tile(const float2* part, float2* tile, int t) {
  constexpr int e0 = A == 0 ? 11 : 10, e1 = A == 1 ? 11 : 10;
  constexpr int ex = A == 0 ? 4 : 3, ey = A == 1 ? 4 : 3, ez = A == 2 ? 4 : 3;
  for (int n = t; n < kTileFaces; n += kP2GThreads) {
    const int nx = n % e0 - 1, ny = (n / e0) % e1 - 1, nz = n / (e0 * e1) - 1;
    float2 WQ = make_float2(0.0f, 0.0f);  // (mass, momentum), each lane summed in the same order
#pragma unroll
    for (int sz = 0; sz < ez; ++sz) {
      const int cz = nz + 1 - sz;
      if (cz < 0 || cz > 7) continue;
#pragma unroll
      for (int sy = 0; sy < ey; ++sy) {
        const int cy = ny + 1 - sy;
        if (cy < 0 || cy > 7) continue;
#pragma unroll
        for (int sx = 0; sx < ex; ++sx) {
          const int cx = nx + 1 - sx;
          if (cx < 0 || cx > 7) continue;
          const int c = cz * 64 + cy * 8 + cx;
          const int s = (sz * ey + sy) * ex + sx;
          WQ = __fadd2_rn(WQ, part[s * kP2GThreads + c]);
        }
      }
    }
    tile[n] = WQ;
  }
}

__global__ void __launch_bounds__(kP2GThreads, 1)
    k_p2g_tile(GridView g, ParticlesView p, const unsigned int* order, const int* cell_start, float2* tiles,
               DeviceReport* rep) {
  extern __shared__ float2 part[];  // [slot][cell] (mass, momentum) partials
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const int base = b * kBlockCells;
  float2* tile0 = tiles + (size_t)b * 3 * kTileFaces;
  if (cell_start[base] == cell_start[base + kBlockCells]) {  // no particles: a zero tile for the merge
    for (int n = t; n < 3 * kTileFaces; n += kP2GThreads) tile0[n] = make_float2(0.0f, 0.0f);
    return;
  }
  const int pbeg = cell_start[base + t], pend = cell_start[base + t + 1];
  const int cell[3] = {g.coord[3 * b] * 8 + (t & 7), g.coord[3 * b + 1] * 8 + ((t >> 3) & 7),
                       g.coord[3 * b + 2] * 8 + (t >> 6)};
  float2* tile = tiles + (size_t)b * 3 * kTileFaces;
  p2g_component<0>(g, p, order, pbeg, pend, cell, part, t, rep);
  __syncthreads();
  reduce_tile<0>(part, tile, t);
  __syncthreads();
  p2g_component<1>(g, p, order, pbeg, pend, cell, part, t, rep);
  __syncthreads();
  reduce_tile<1>(part, tile + kTileFaces, t);
  __syncthreads();
  p2g_component<2>(g, p, order, pbeg, pend, cell, part, t, rep);
  __syncthreads();
  reduce_tile<2>(part, tile + 2 * kTileFaces, t);
}

__device__ __forceinline__ bool is_solid(const GridView& g, int x, int y, int z) {
  return x < g.solid_lo[0] || y < g.solid_lo[1] || z < g.solid_lo[2] || x > g.solid_hi[0] || y > g.solid_hi[1] ||
         z > g.solid_hi[2];
}

// Sum, in a fixed order, of the tile entries of the (at most 8) blocks whose
// halo tile covers face `loc` of normal axis A in block b. Along each axis the
// covering blocks are the face's own block and at most one neighbour: the lower
// one when loc is within the neighbour tile's upper halo (loc <= 1 along the
// normal axis, loc == 0 across it), the upper one when loc == 7. All candidate
// loads are issued before the sum.
template <int A>
__device__ __forceinline__ float2 merge_face(const GridView& g, const float2* __restrict__ tiles, int b,
                                             const int loc[3]) {
  int alt[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) alt[d] = loc[d] <= (d == A ? 1 : 0) ? -1 : (loc[d] == 7 ? 1 : 0);
  constexpr int e0 = A == 0 ? 11 : 10, e1 = A == 1 ? 11 : 10;
  float2 v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int sx = k & 1, sy = (k >> 1) & 1, sz = k >> 2;
    const bool use = (!sx || alt[0] != 0) && (!sy || alt[1] != 0) && (!sz || alt[2] != 0);
    const int dx = sx ? alt[0] : 0, dy = sy ? alt[1] : 0, dz = sz ? alt[2] : 0;
    int nb = -1;
    if (k == 0)
      nb = b;
    else if (use)
      nb = g.nbr27[b * 27 + nbr_index(dx, dy, dz)];
    v[k] = make_float2(0.0f, 0.0f);
    if (nb >= 0) {
      const int n = ((loc[2] - 8 * dz + 1) * e1 + (loc[1] - 8 * dy + 1)) * e0 + (loc[0] - 8 * dx + 1);
      v[k] = tiles[((size_t)nb * 3 + A) * kTileFaces + n];
    }
  }
  float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    r.x += v[k].x;
    r.y += v[k].y;
  }
  return r;
}

// One thread per owned face (CTA = one block and normal axis, thread = cell):
// fixed-order sum of the covering tiles, then either raw mass/momentum or
// normalize + gravity + stationary walls.
__global__ void __launch_bounds__(kBlockCells)
    k_p2g_merge(GridView g, const int* cell_start, const float2* tiles, P2GMergeParams prm, float* out0_x,
                float* out0_y, float* out0_z, float* out1_x, float* out1_y, float* out1_z, DeviceReport* rep) {
  const int b = blockIdx.x, a = blockIdx.y, l = threadIdx.x;
  if (b == 0 && a == 0 && l == 0 && rep != nullptr) rep->compiled_architecture = compiled_arch();
  const int loc[3] = {l & 7, (l >> 3) & 7, l >> 6};
  const float2 wq = a == 0 ? merge_face<0>(g, tiles, b, loc) : (a == 1 ? merge_face<1>(g, tiles, b, loc)
                                                                       : merge_face<2>(g, tiles, b, loc));
  const float W = wq.x, Q = wq.y;
  float* out0 = a == 0 ? out0_x : (a == 1 ? out0_y : out0_z);
  float* out1 = a == 0 ? out1_x : (a == 1 ? out1_y : out1_z);
  const size_t slot = (size_t)b * kBlockCells + l;
  const float mass = W * prm.mass_scale;
  if (prm.mode == 0) {
    out0[slot] = mass;
    out1[slot] = Q * prm.mass_scale;
    return;
  }
  float u = 0.0f;
  if (mass != 0.0f && mass > prm.min_face_mass) u = Q / W;
  u += prm.dt * prm.gravity[a];
  const int head[3] = {g.coord[3 * b] * 8 + loc[0], g.coord[3 * b + 1] * 8 + loc[1], g.coord[3 * b + 2] * 8 + loc[2]};
  int tail[3] = {head[0], head[1], head[2]};
  tail[a] -= 1;
  if (prm.walls && (is_solid(g, head[0], head[1], head[2]) || is_solid(g, tail[0], tail[1], tail[2]))) u = 0.0f;
  if (!isfinite(u)) report_error(rep, kOutOfRange, (unsigned long long)slot);
  out0[slot] = u;
  if (out1 != nullptr) out1[slot] = mass;
}

cudaError_t launch_p2g(const GridView& g, const ParticlesView& p, const int* cell_start, float2* tiles,
                       const P2GMergeParams& prm, float* const out0[3], float* const out1[3], DeviceReport* rep,
                       cudaStream_t s, const unsigned int* order) {
  if (g.nb == 0) return cudaSuccess;
  const size_t smem = sizeof(float2) * kSlots * kP2GThreads;
  static unsigned long long configured = 0;
  if (first_on_device(configured))
    cudaFuncSetAttribute(k_p2g_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  ++g_kernel_launches;
  k_p2g_tile<<<g.nb, kP2GThreads, smem, s>>>(g, p, order, cell_start, tiles, rep);
  ++g_kernel_launches;
  k_p2g_merge<<<dim3(g.nb, 3), kBlockCells, 0, s>>>(g, cell_start, tiles, prm, out0[0], out0[1], out0[2], out1[0],
                                                    out1[1], out1[2], rep);
  return cudaGetLastError();
}

}  // namespace fl
