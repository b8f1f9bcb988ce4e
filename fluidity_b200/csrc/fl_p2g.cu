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
// B200 design. One CTA of 256 threads per active 8^3 block, each thread
// taking two cells in turn. Particles are sorted by cell, so a thread walks
// one cell's particles at a time and
// accumulates into registers: along the normal axis a particle of the cell
// touches nodes cell-1..cell+1 or cell..cell+2, so 4 x 3 x 3 = 36 slots per
// channel cover every particle of the cell with static register indexing.
// The register partials are then summed across the warp with shuffles: a
// warp holds one z-plane of four 8-cell rows, so the x-neighbours' slots that
// land on the same node are combined along each row and then across the rows,
// giving every warp a small tile of its nodes in shared memory (at most
// 4 x 6 x 10 entries). Each node of the block's 11x10x10 tile (normal extent 11,
// transverse 10) sums the (at most 8) warp tiles that cover it in a fixed
// order. The block tile is written to a per-block scratch tile and a second
// kernel sums, for every owned face, the tiles of the (at most 8) blocks whose
// halo covers it, again in a fixed order.
// No floating-point atomics are used anywhere, so the result is bitwise
// reproducible run to run for a given particle order (the stable sort fixes it).
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

// 256 threads per CTA, each thread taking two cells of the block (cells t and
// t + 256: the same warp shapes and warp tiles as one thread per cell). Two
// CTAs fit one SM (123 registers), so one CTA's barriers and tile sums overlap
// the other's particle loop, and with one 30 KB warp-tile set per CTA the SM
// keeps ~190 KB of L1: a warp's particle loads touch 8 lines per instruction
// (lanes walk different cells), and those lines are reused by the next ~8
// particles of each cell only while they stay in L1.
constexpr int kP2GThreads = 256;
constexpr int kP2GPasses = kBlockCells / kP2GThreads;
constexpr int kSlots = 36;

template <int A>
__device__ __forceinline__ void p2g_component(const GridView& g, const ParticlesView& p, const unsigned int* order,
                                              int pbeg, int pend, const int cell[3], float2 accW[kSlots / 2],
                                              float2 accQ[kSlots / 2], DeviceReport* rep) {
  constexpr int D1 = A == 0 ? 1 : 0;
  constexpr int D2 = A == 2 ? 1 : 2;
  // Accumulators in normal-axis slot pairs: entry (k * 3 + j) * 2 + hp holds
  // normal slots 2hp (x) and 2hp + 1 (y) of transverse node (j, k). Each pair
  // is updated by one packed FP32 FMA (fma.rn.f32x2), which rounds every lane
  // exactly as fmaf does, so the sums are bitwise those of the scalar form.
#pragma unroll
  for (int s = 0; s < kSlots / 2; ++s) {
    accW[s] = make_float2(0.0f, 0.0f);
    accQ[s] = make_float2(0.0f, 0.0f);
  }
  const float h = g.h;
  const float cellf[3] = {(float)cell[0], (float)cell[1], (float)cell[2]};
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
    const float cA = __ldg(&p.c[3 * A + A][i]), c1 = __ldg(&p.c[3 * A + D1][i]), c2 = __ldg(&p.c[3 * A + D2][i]);
    // Normal axis (face-centred nodes cell-1 .. cell+2): with f = X - cell
    // (exact) the particle's first node is cell - 1 for f < 1/2, else cell, and
    // g = X - (first + 1) gives the three weights 0.5 (1/2 - g)^2, 3/4 - g^2,
    // 0.5 (1/2 + g)^2; the unused slot is zero. Affine terms
    // ta[s] = C_aa h (s - 1 - f), formed by adding C_aa h slot by slot.
    float wa[4], ta[4];
    {
      const float f = X[A] - cellf[A];
      const bool shifted = f >= 0.5f;
      const float gg = shifted ? f - 1.0f : f;
      const float dm = 0.5f - gg, dp = 0.5f + gg;
      const float n0 = 0.5f * dm * dm, n1 = fmaf(-gg, gg, 0.75f), n2 = 0.5f * dp * dp;
      wa[0] = shifted ? 0.0f : n0;
      wa[1] = shifted ? n0 : n1;
      wa[2] = shifted ? n1 : n2;
      wa[3] = shifted ? n2 : 0.0f;
      const float ch = cA * h;
      ta[0] = fmaf(-ch, f, -ch);
      ta[1] = ta[0] + ch;
      ta[2] = ta[1] + ch;
      ta[3] = ta[2] + ch;
    }
    // Transverse axes D1, D2 as one packed pair (cell-centred nodes
    // cell-1 .. cell+1): weights 0.5 (1-f)^2, 3/4 - (f - 1/2)^2, 0.5 f^2 and
    // affine terms C h (s - 1/2 - f).
    float w1[3], w2[3], t1[3], t2[3];
    {
      const float2 f = __fadd2_rn(make_float2(X[D1], X[D2]), make_float2(-cellf[D1], -cellf[D2]));
      const float2 half = make_float2(0.5f, 0.5f);
      const float2 d = __fadd2_rn(make_float2(1.0f, 1.0f), make_float2(-f.x, -f.y));
      const float2 c = __fadd2_rn(f, make_float2(-0.5f, -0.5f));
      const float2 w0 = __fmul2_rn(__fmul2_rn(half, d), d);
      const float2 wm = __ffma2_rn(make_float2(-c.x, -c.y), c, make_float2(0.75f, 0.75f));
      const float2 wp = __fmul2_rn(__fmul2_rn(half, f), f);
      const float2 ch = __fmul2_rn(make_float2(c1, c2), make_float2(h, h));
      const float2 a0 = __fmul2_rn(ch, __fadd2_rn(make_float2(-0.5f, -0.5f), make_float2(-f.x, -f.y)));
      const float2 a1 = __fadd2_rn(a0, ch), a2 = __fadd2_rn(a1, ch);
      w1[0] = w0.x, w1[1] = wm.x, w1[2] = wp.x;
      w2[0] = w0.y, w2[1] = wm.y, w2[2] = wp.y;
      t1[0] = a0.x, t1[1] = a1.x, t1[2] = a2.x;
      t2[0] = a0.y, t2[1] = a1.y, t2[2] = a2.y;
    }
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
}

// Slot (sx, sy, sz) of the accumulators (offsets along x, y, z from the cell's
// first node), as a (mass, momentum) pair.
template <int A>
__device__ __forceinline__ float2 slot_val(const float2 accW[kSlots / 2], const float2 accQ[kSlots / 2], int sx, int sy,
                                           int sz) {
  const int s = A == 0 ? sx : (A == 1 ? sy : sz);
  const int j = A == 0 ? sy : sx;
  const int k = A == 2 ? sy : sz;
  const int e = (k * 3 + j) * 2 + (s >> 1);
  return (s & 1) ? make_float2(accW[e].y, accQ[e].y) : make_float2(accW[e].x, accQ[e].x);
}

__device__ __forceinline__ float2 shfl_up2(float2 v, int d) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ float2 shfl_down2(float2 v, int d) {
  return make_float2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// Extents of the warp tile of component A: a warp holds the cells of one
// z-plane and four y-rows of 8, so its slots cover ex + 7 nodes along x,
// ey + 3 along y and ez along z (node coordinates from the warp's first
// cell - 1).
template <int A>
struct WarpTile {
  static constexpr int ex = A == 0 ? 4 : 3, ey = A == 1 ? 4 : 3, ez = A == 2 ? 4 : 3;
  static constexpr int tx = ex + 7, ty = ey + 3, tz = ez;
  static constexpr int size = tx * ty * tz;
};
constexpr int kWarpTileMax = 240;  // max over the three components (10 x 6 x 4)
constexpr int kP2GWarps = kBlockCells / 32;  // warp tiles per component

// The warp's partials summed per node, in a fixed order, into its tile:
// along x within each 8-lane row (a lane keeps node x - 1 and, for x <= ex - 2,
// node x + 7), then along y across the four rows (node y - 1 and, for
// y <= ey - 2, node y + 3); every tile entry is written by exactly one lane.
template <int A>
__device__ __forceinline__ void warp_tile(const float2 accW[kSlots / 2], const float2 accQ[kSlots / 2], float2* wt,
                                          int lane) {
  using W = WarpTile<A>;
  const int x = lane & 7, y = lane >> 3;
#pragma unroll
  for (int sz = 0; sz < W::ez; ++sz) {
    float2 xf[W::ey], xb[W::ey];
#pragma unroll
    for (int sy = 0; sy < W::ey; ++sy) {
      float2 f = slot_val<A>(accW, accQ, 0, sy, sz), bk = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int sx = 1; sx < W::ex; ++sx) {
        const float2 v = slot_val<A>(accW, accQ, sx, sy, sz);
        const float2 up = shfl_up2(v, sx), dn = shfl_down2(v, 8 - sx);
        if (x >= sx) f = __fadd2_rn(f, up);
        if (sx >= x + 1) bk = __fadd2_rn(bk, dn);
      }
      xf[sy] = f;
      xb[sy] = bk;
    }
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      float2 f = part ? xb[0] : xf[0], bk = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int sy = 1; sy < W::ey; ++sy) {
        const float2 v = part ? xb[sy] : xf[sy];
        const float2 up = shfl_up2(v, 8 * sy), dn = shfl_down2(v, 8 * (4 - sy));
        if (y >= sy) f = __fadd2_rn(f, up);
        if (sy >= y + 1) bk = __fadd2_rn(bk, dn);
      }
      const int lx = x + 8 * part;
      if (part == 0 || x <= W::ex - 2) {
        wt[(sz * W::ty + y) * W::tx + lx] = f;
        if (y <= W::ey - 2) wt[(sz * W::ty + y + 4) * W::tx + lx] = bk;
      }
    }
  }
}

// Node n of the block's tile of component A: the sum of the warp tiles that
// cover it, warps in ascending (z, y-half) order.
template <int A>
__device__ __forceinline__ void block_tile(const float2* wtiles, float2* tile, int t) {
  using W = WarpTile<A>;
  constexpr int e0 = A == 0 ? 11 : 10, e1 = A == 1 ? 11 : 10;
  for (int n = t; n < kTileFaces; n += kP2GThreads) {
    const int lx = n % e0, ny = (n / e0) % e1 - 1, nz = n / (e0 * e1) - 1;
    float2 WQ = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int dz = 0; dz < W::ez; ++dz) {
      const int wz = nz + 1 - dz;  // warp plane whose local z index is dz
      if (wz < 0 || wz > 7) continue;
#pragma unroll
      for (int wy = 0; wy < 2; ++wy) {
        const int ly = ny + 1 - 4 * wy;
        if (ly < 0 || ly >= W::ty) continue;
        WQ = __fadd2_rn(WQ, wtiles[(wz * 2 + wy) * kWarpTileMax + (dz * W::ty + ly) * W::tx + lx]);
      }
    }
    tile[n] = WQ;
  }
}

template <int A>
__device__ __forceinline__ void p2g_pass(const GridView& g, const ParticlesView& p, const unsigned int* order,
                                         const int* cell_start, int b, int t, float2* wt, float2* tile,
                                         DeviceReport* rep) {
  const int base = b * kBlockCells;
#pragma unroll 1
  for (int pass = 0; pass < kP2GPasses; ++pass) {
    const int l = t + pass * kP2GThreads;  // the cell: x = l & 7, y = (l >> 3) & 7, z = l >> 6
    const int cell[3] = {g.coord[3 * b] * 8 + (l & 7), g.coord[3 * b + 1] * 8 + ((l >> 3) & 7),
                         g.coord[3 * b + 2] * 8 + (l >> 6)};
    float2 accW[kSlots / 2], accQ[kSlots / 2];
    p2g_component<A>(g, p, order, cell_start[base + l], cell_start[base + l + 1], cell, accW, accQ, rep);
    warp_tile<A>(accW, accQ, wt + (l >> 5) * kWarpTileMax, t & 31);
  }
  __syncthreads();
  block_tile<A>(wt, tile + A * kTileFaces, t);
  if (A < 2) __syncthreads();  // the next component overwrites the warp tiles
}

__global__ void __launch_bounds__(kP2GThreads, 2)
    k_p2g_tile(GridView g, ParticlesView p, const unsigned int* order, const int* cell_start, float2* tiles,
               DeviceReport* rep) {
  // The components in turn through one warp-tile set: particle loops and warp
  // tiles, a barrier, the block tile summed from the warp tiles, a barrier.
  extern __shared__ float2 wt_smem[];
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const int base = b * kBlockCells;
  float2* tile = tiles + (size_t)b * 3 * kTileFaces;
  if (cell_start[base] == cell_start[base + kBlockCells]) {  // no particles: a zero tile for the merge
    for (int n = t; n < 3 * kTileFaces; n += kP2GThreads) tile[n] = make_float2(0.0f, 0.0f);
    return;
  }
  p2g_pass<0>(g, p, order, cell_start, b, t, wt_smem, tile, rep);
  p2g_pass<1>(g, p, order, cell_start, b, t, wt_smem, tile, rep);
  p2g_pass<2>(g, p, order, cell_start, b, t, wt_smem, tile, rep);
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
  // NormalizeCore's validity (liquid_boundary_transfer_3d.cc:486-510): no
  // mass -> missing, positive mass at or below the minimum -> low mass
  // (selected, not indexed: a dynamic index into the parameter arrays would copy them to local memory)
  unsigned char* val = a == 0 ? prm.validity[0] : (a == 1 ? prm.validity[1] : prm.validity[2]);
  if (val != nullptr) val[slot] = mass == 0.0f ? kFaceMissing : (mass <= prm.min_face_mass ? kFaceLowMass : kFaceValid);
  u += prm.dt * (a == 0 ? prm.gravity[0] : (a == 1 ? prm.gravity[1] : prm.gravity[2]));
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
  const size_t smem = sizeof(float2) * kP2GWarps * kWarpTileMax;
  static unsigned long long configured = 0;
  if (first_on_device(configured)) {
    cudaFuncSetAttribute(k_p2g_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // two CTAs per SM: 2 x 30 KB of warp tiles in the 64 KB shared-memory
    // carveout (28% of 228 KB); the rest of the SM's 256 KB stays L1
    cudaFuncSetAttribute(k_p2g_tile, cudaFuncAttributePreferredSharedMemoryCarveout, 28);
  }
  ++g_kernel_launches;
  k_p2g_tile<<<g.nb, kP2GThreads, smem, s>>>(g, p, order, cell_start, tiles, rep);
  ++g_kernel_launches;
  k_p2g_merge<<<dim3(g.nb, 3), kBlockCells, 0, s>>>(g, cell_start, tiles, prm, out0[0], out0[1], out0[2], out1[0],
                                                    out1[1], out1[2], rep);
  return cudaGetLastError();
}

}  // namespace fl
