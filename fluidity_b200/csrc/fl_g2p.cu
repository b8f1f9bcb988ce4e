// APIC grid-to-particle transfer with fused advection.
//
// Semantics follow GatherMac3D / GatherMacVelocityComponentFromSlots
// (native/src/transfers_3d.cc:199-261; native/src/mac_gather_3d_internal.h:15-69):
//   v_a          = sum_n w_n u_n
//   increment_a  = v_a - sum_n w_n u_old_n
//   C_a (fitted) = 4 * sum_n w_n u_n (x_n - x_p)/h  /  h
//   grad_a       = sum_n grad(w_n) u_n
// The step mode keeps (v, C) and advects x += dt v with a clamp to the
// non-solid box (the reference's contact-constrained update,
// liquid_boundary_transfer_3d.cu:544, is out of scope; a plain clamp stands in).
//
// B200 design: one CTA per non-empty 8^3 block. The CTA stages the block's
// 11x10x10 halo tile of each face component in shared memory (coalesced from
// the owned-face arrays of the 27 neighbouring blocks), then its threads stride
// over the block's contiguous particle range, gather all 81 samples from
// shared memory and keep C in registers.
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kG2PThreads = 256;

__device__ __forceinline__ int tile_ext0(int a) { return a == 0 ? 11 : 10; }
__device__ __forceinline__ int tile_ext1(int a) { return a == 1 ? 11 : 10; }

__device__ void load_tile(const GridView& g, int b, const float* const u[3], float* tile, int t) {
  for (int n = t; n < 3 * kTileFaces; n += kG2PThreads) {
    const int a = n / kTileFaces, idx = n % kTileFaces;
    const int e0 = tile_ext0(a), e1 = tile_ext1(a);
    const int nx = idx % e0 - 1, ny = (idx / e0) % e1 - 1, nz = idx / (e0 * e1) - 1;
    const int dx = nx < 0 ? -1 : (nx > 7 ? 1 : 0), dy = ny < 0 ? -1 : (ny > 7 ? 1 : 0),
              dz = nz < 0 ? -1 : (nz > 7 ? 1 : 0);
    const int nb = g.nbr27[b * 27 + nbr_index(dx, dy, dz)];
    float v = 0.0f;
    if (nb >= 0) {
      const int l = ((nz - 8 * dz) * 8 + (ny - 8 * dy)) * 8 + (nx - 8 * dx);
      v = u[a][(size_t)nb * kBlockCells + l];
    }
    tile[n] = v;
  }
}

// Four CTAs per SM (at most 64 registers): with the packed sums below and no
// cap the step kernel runs at less than half the speed (2.29 vs 0.95 ms at the
// 256^3 splash).
constexpr int kG2PMinBlocks = 4;

template <bool kFull>
__global__ void __launch_bounds__(kG2PThreads, kG2PMinBlocks)
    k_g2p(GridView g, ParticlesView p, const int* cell_start, const float* u0, const float* u1, const float* u2,
          const float* o0, const float* o1, const float* o2, G2PParams prm, float* full_out, DeviceReport* rep) {
  __shared__ float tile[3 * kTileFaces];
  __shared__ float tile_old[kFull ? 3 * kTileFaces : 1];
  __shared__ unsigned int next_blocks;  // step mode: neighbouring blocks the advected particles land in
  const int b = blockIdx.x, t = threadIdx.x;
  if (b == 0 && t == 0 && rep != nullptr) rep->compiled_architecture = compiled_arch();
  const int pbeg = cell_start[b * kBlockCells], pend = cell_start[(b + 1) * kBlockCells];
  if (pbeg == pend) return;
  if (t == 0) next_blocks = 0u;
  const float* un[3] = {u0, u1, u2};
  load_tile(g, b, un, tile, t);
  if (kFull) {
    const float* uo[3] = {o0, o1, o2};
    if (o0 != nullptr)
      load_tile(g, b, uo, tile_old, t);
    else
      for (int n = t; n < 3 * kTileFaces; n += kG2PThreads) tile_old[n] = 0.0f;
  }
  __syncthreads();
  const int bc[3] = {g.coord[3 * b] * 8, g.coord[3 * b + 1] * 8, g.coord[3 * b + 2] * 8};
  const float four_inv_h = 4.0f * g.inv_h;  // fitted slopes 4 sum w u r / h (one multiply instead of a division)
  // Position of particle q (read through the cell order in step mode); the
  // next particle's is loaded one iteration ahead, so its two dependent loads
  // overlap the current particle's work.
  auto load_x = [&](int q, float out[3]) {
    const int src = (!kFull && prm.order != nullptr) ? (int)prm.order[q] : -1;
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = src >= 0 ? prm.x_in[d][src] : p.x[d][q];
  };
  float xnext[3] = {0.0f, 0.0f, 0.0f};
  if (pbeg + t < pend) load_x(pbeg + t, xnext);
  for (int q = pbeg + t; q < pend; q += kG2PThreads) {
    float xw[3] = {xnext[0], xnext[1], xnext[2]}, X[3];
    if (q + kG2PThreads < pend) load_x(q + kG2PThreads, xnext);
    int cell[3];
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      X[d] = lattice_coord(g, xw[d], d);
      cell[d] = __float2int_rd(X[d]);
      inside = inside && cell[d] >= bc[d] && cell[d] < bc[d] + 8;
    }
    if (!inside) {  // the sort binned this particle elsewhere: never index the tile
      report_error(rep, kInternal, (unsigned long long)q);
      continue;
    }
    float vel[3], fit[9], inc[3], grad[9];
    // Step mode: the cell-centred factors of each axis (shift 1/2) serve the
    // two components transverse to it, so they are formed once per particle;
    // only the normal axis's face-centred factors are formed per component.
    int firstC[3];
    float wC[3][3], wrC[3][3];
    if (!kFull) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float fst = floorf(X[d] - 1.0f);
        firstC[d] = (int)fst;
        const float a0 = fst + 0.5f;
        const float dl = X[d] - (a0 + 0.5f);
        const float dr = fabsf(X[d] - (a0 + 1.5f));
        const float c = X[d] - (a0 + 1.0f);
        wC[d][0] = 0.5f * dr * dr;
        wC[d][1] = 0.75f - c * c;
        wC[d][2] = 0.5f * dl * dl;
#pragma unroll
        for (int s = 0; s < 3; ++s) wrC[d][s] = wC[d][s] * ((a0 + (float)s) - X[d]);
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // Axis factors: first node, weights, normalized derivative and offset/h.
      int first[3];
      float w[3][3], dw[3][3], r[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (!kFull && d != a) {
          first[d] = firstC[d];
#pragma unroll
          for (int s = 0; s < 3; ++s) w[d][s] = wC[d][s], r[d][s] = 0.0f, dw[d][s] = 0.0f;
          continue;
        }
        const float shift = d == a ? 0.0f : 0.5f;
        const float fst = floorf(X[d] - shift - 0.5f);
        first[d] = (int)fst;
        const float a0 = fst + shift;
        const float dl = X[d] - (a0 + 0.5f);
        const float dr = fabsf(X[d] - (a0 + 1.5f));
        const float c = X[d] - (a0 + 1.0f);
        w[d][0] = 0.5f * dr * dr;
        w[d][1] = 0.75f - c * c;
        w[d][2] = 0.5f * dl * dl;
        dw[d][0] = -dr;
        dw[d][1] = -2.0f * c;
        dw[d][2] = dl;
#pragma unroll
        for (int s = 0; s < 3; ++s) r[d][s] = (a0 + (float)s) - X[d];
      }
      const int e0 = tile_ext0(a), e1 = tile_ext1(a);
      const int n0 = ((first[2] - bc[2] + 1) * e1 + (first[1] - bc[1] + 1)) * e0 + (first[0] - bc[0] + 1);
      const float* ta = tile + a * kTileFaces + n0;
      const float* to = tile_old + (kFull ? a * kTileFaces + n0 : 0);
      // The 27-node sums factor by axis: contract x (weights w0 and w0*r0, and
      // for the full gather dw0 and the old field), then y, then z. Every
      // output is the same sum of w-products times node values as the direct
      // 27-term form, with about half the FP32 operations.
      float wr[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int s = 0; s < 3; ++s) wr[d][s] = (!kFull && d != a) ? wrC[d][s] : w[d][s] * r[d][s];
      float pic = 0.0f, old = 0.0f, m0 = 0.0f, m1 = 0.0f, m2 = 0.0f, g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
      if (!kFull) {
        // Step mode, with the pairs (U0, U1), (V0, V1), (pic, m0) and (m1, m2)
        // each updated by one packed FP32 FMA: every lane performs the scalar
        // form's operations in the same order, so the results are bitwise equal.
        const float2 wA[3] = {make_float2(w[0][0], wr[0][0]), make_float2(w[0][1], wr[0][1]),
                              make_float2(w[0][2], wr[0][2])};
        float2 pm0 = make_float2(0.0f, 0.0f), m12 = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int kz = 0; kz < 3; ++kz) {
          float2 V01 = make_float2(0.0f, 0.0f);
          float V2 = 0.0f;
#pragma unroll
          for (int ky = 0; ky < 3; ++ky) {
            const int row = (kz * e1 + ky) * e0;
            const float u0 = ta[row], u1 = ta[row + 1], u2 = ta[row + 2];
            float2 U01 = __fmul2_rn(wA[0], make_float2(u0, u0));
            U01 = __ffma2_rn(wA[1], make_float2(u1, u1), U01);
            U01 = __ffma2_rn(wA[2], make_float2(u2, u2), U01);
            V01 = __ffma2_rn(make_float2(w[1][ky], w[1][ky]), U01, V01);
            V2 = fmaf(wr[1][ky], U01.x, V2);
          }
          pm0 = __ffma2_rn(make_float2(w[2][kz], w[2][kz]), V01, pm0);
          m12 = __ffma2_rn(make_float2(w[2][kz], wr[2][kz]), make_float2(V2, V01.x), m12);
        }
        pic = pm0.x;
        m0 = pm0.y;
        m1 = m12.x;
        m2 = m12.y;
      } else {
#pragma unroll
      for (int kz = 0; kz < 3; ++kz) {
        float V0 = 0.0f, V1 = 0.0f, V2 = 0.0f, V3 = 0.0f, V4 = 0.0f, V5 = 0.0f;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
          const int row = (kz * e1 + ky) * e0;
          const float u0 = ta[row], u1 = ta[row + 1], u2 = ta[row + 2];
          const float U0 = fmaf(w[0][2], u2, fmaf(w[0][1], u1, w[0][0] * u0));
          const float U1 = fmaf(wr[0][2], u2, fmaf(wr[0][1], u1, wr[0][0] * u0));
          V0 = fmaf(w[1][ky], U0, V0);
          V1 = fmaf(w[1][ky], U1, V1);
          V2 = fmaf(wr[1][ky], U0, V2);
          if (kFull) {
            const float Ud = fmaf(dw[0][2], u2, fmaf(dw[0][1], u1, dw[0][0] * u0));
            const float O = fmaf(w[0][2], to[row + 2], fmaf(w[0][1], to[row + 1], w[0][0] * to[row]));
            V3 = fmaf(w[1][ky], Ud, V3);
            V4 = fmaf(dw[1][ky], U0, V4);
            V5 = fmaf(w[1][ky], O, V5);
          }
        }
        pic = fmaf(w[2][kz], V0, pic);
        m0 = fmaf(w[2][kz], V1, m0);
        m1 = fmaf(w[2][kz], V2, m1);
        m2 = fmaf(wr[2][kz], V0, m2);
        if (kFull) {
          g0 = fmaf(w[2][kz], V3, g0);
          g1 = fmaf(w[2][kz], V4, g1);
          g2 = fmaf(dw[2][kz], V0, g2);
          old = fmaf(w[2][kz], V5, old);
        }
      }
      }
      vel[a] = pic;
      fit[3 * a] = four_inv_h * m0;
      fit[3 * a + 1] = four_inv_h * m1;
      fit[3 * a + 2] = four_inv_h * m2;
      inc[a] = pic - old;
      grad[3 * a] = g0 * g.inv_h;
      grad[3 * a + 1] = g1 * g.inv_h;
      grad[3 * a + 2] = g2 * g.inv_h;
    }
    bool finite = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) finite = finite && isfinite(vel[a]);
    if (!finite) report_error(rep, kOutOfRange, (unsigned long long)q);
    if (kFull) {
      float* o = full_out + 24 * (size_t)q;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        o[a] = vel[a];
        o[3 + a] = inc[a];
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        o[6 + k] = fit[k];
        o[15 + k] = grad[k];
      }
    } else {
      int off[3];
      bool near = true, valid = true;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        p.v[d][q] = vel[d];
        float nx = xw[d] + prm.dt * vel[d];
        nx = fminf(fmaxf(nx, prm.clamp_lo[d]), prm.clamp_hi[d]);
        p.x[d][q] = nx;
        // the next step's block of this particle (the cell rule of the sort)
        const float Xn = lattice_coord(g, nx, d);
        valid = valid && isfinite(Xn) && fabsf(Xn) < 1.0e9f;
        const int nb_d = floor_div8(valid ? __float2int_rd(Xn) : 0);
        off[d] = nb_d - bc[d] / 8;
        near = near && off[d] >= -1 && off[d] <= 1;
        valid = valid && nb_d - g.blo[d] >= 0 && nb_d - g.blo[d] < g.bdim[d];
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) p.c[k][q] = fit[k];
      // Particles that leave the lattice are reported by the next sort; here they mark nothing.
      if (prm.occ_next != nullptr) {
        // one shared-memory OR per warp for the neighbouring blocks
        const unsigned bit = valid && near ? 1u << nbr_index(off[0], off[1], off[2]) : 0u;
        const unsigned active = __activemask();
        const unsigned bits = __reduce_or_sync(active, bit);
        if (bits != 0u && (threadIdx.x & 31) == __ffs(active) - 1) atomicOr(&next_blocks, bits);
        if (valid && !near) {
          const int bx = bc[0] / 8 + off[0] - g.blo[0], by = bc[1] / 8 + off[1] - g.blo[1],
                    bz = bc[2] / 8 + off[2] - g.blo[2];
          prm.occ_next[((size_t)bz * g.bdim[1] + by) * g.bdim[0] + bx] = 1;
        }
      }
    }
  }
  if (!kFull && prm.occ_next != nullptr) {
    __syncthreads();
    if (t < 27 && ((next_blocks >> t) & 1u)) {
      const int bx = bc[0] / 8 + t % 3 - 1 - g.blo[0], by = bc[1] / 8 + (t / 3) % 3 - 1 - g.blo[1],
                bz = bc[2] / 8 + t / 9 - 1 - g.blo[2];
      prm.occ_next[((size_t)bz * g.bdim[1] + by) * g.bdim[0] + bx] = 1;
    }
  }
}

cudaError_t launch_g2p(const GridView& g, const ParticlesView& p, const int* cell_start, const float* const u[3],
                       const float* const u_old[3], const G2PParams& prm, float* full_out, DeviceReport* rep,
                       cudaStream_t s) {
  if (g.nb == 0 || p.count == 0) return cudaSuccess;
  if (full_out != nullptr) {
    ++g_kernel_launches;
    k_g2p<true><<<g.nb, kG2PThreads, 0, s>>>(g, p, cell_start, u[0], u[1], u[2], u_old ? u_old[0] : nullptr,
                                              u_old ? u_old[1] : nullptr, u_old ? u_old[2] : nullptr, prm, full_out,
                                              rep);
  } else {
    ++g_kernel_launches;
    k_g2p<false><<<g.nb, kG2PThreads, 0, s>>>(g, p, cell_start, u[0], u[1], u[2], nullptr, nullptr, nullptr, prm,
                                               nullptr, rep);
  }
  return cudaGetLastError();
}

}  // namespace fl
