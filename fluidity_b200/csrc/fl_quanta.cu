// Reference-compatible quantized P2G (DepositMacQuanta3D / CudaDepositMacQuanta3D).
//
// Restates native/src/transfers_3d.cc:44-54 (RoundNearestEven), :147-197 (the
// quantized accumulator) and the stencil of native/src/sparse_mac_grid_3d.cc:
// 266-310,451-548 in FP64 on the device, one thread per particle, with every
// product and sum explicitly rounded (no FMA contraction) so each contribution
// is bit-identical to the CPU operator's for power-of-two cell widths and
// exactly representable origins. Quanta are summed with 64-bit integer atomics,
// which makes the result independent of particle order -- the reference's own
// mechanism for reproducible deposits (native/cuda/transfers_3d.cu:44-97).
// This is the compatibility path; the FP32 hot path is fl_p2g.cu.
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

__device__ __forceinline__ long long round_nearest_even(double s) {
  const double mag = fabs(s);
  const double integral = floor(mag);
  const double frac = __dsub_rn(mag, integral);
  long long q = (long long)integral;
  if (frac > 0.5 || (frac == 0.5 && (q & 1))) ++q;
  return s < 0.0 ? -q : q;
}

struct QuantaParams {
  double origin[3];
  double h;
  double mass_per_quantum;
  double momentum_per_quantum;
  double limit;
};

__global__ void k_deposit_quanta(GridView g, const double* parts, unsigned long long n, QuantaParams prm,
                                 unsigned long long* mq0, unsigned long long* mq1, unsigned long long* mq2,
                                 unsigned long long* pq0, unsigned long long* pq1, unsigned long long* pq2,
                                 DeviceReport* rep) {
  const unsigned long long p = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if (p == 0) rep->compiled_architecture = compiled_arch();
  if (p >= n) return;
  const double* q = parts + 19 * p;
  const double mass = q[6];
  unsigned long long* mq[3] = {mq0, mq1, mq2};
  unsigned long long* pq[3] = {pq0, pq1, pq2};
  for (int a = 0; a < 3; ++a) {
    long long first[3];
    double w[3][3], off[3][3];
    for (int d = 0; d < 3; ++d) {
      const double shift = d == a ? 0.0 : 0.5;
      const double X = __ddiv_rn(__dsub_rn(q[3 + d], prm.origin[d]), prm.h);
      const double fst = floor(__dsub_rn(X, shift + 0.5));
      first[d] = (long long)fst;
      const double a0 = __dadd_rn(fst, shift);
      const double dl = __dsub_rn(X, __dadd_rn(a0, 0.5));
      const double dr = fabs(__dsub_rn(X, __dadd_rn(a0, 1.5)));
      const double c = __dsub_rn(X, __dadd_rn(a0, 1.0));
      w[d][0] = __dmul_rn(__dmul_rn(0.5, dr), dr);
      w[d][1] = __dsub_rn(0.75, __dmul_rn(c, c));
      w[d][2] = __dmul_rn(__dmul_rn(0.5, dl), dl);
      for (int s = 0; s < 3; ++s) off[d][s] = __dmul_rn(__dsub_rn(__dadd_rn(a0, (double)s), X), prm.h);
    }
    const double va = q[7 + a];
    const double* row = q + 10 + 3 * a;
    for (int kz = 0; kz < 3; ++kz)
      for (int ky = 0; ky < 3; ++ky)
        for (int kx = 0; kx < 3; ++kx) {
          const long long fi = first[0] + kx, fj = first[1] + ky, fk = first[2] + kz;
          const int bx = floor_div8((int)fi), by = floor_div8((int)fj), bz = floor_div8((int)fk);
          const int lx = bx - g.blo[0], ly = by - g.blo[1], lz = bz - g.blo[2];
          int o = -1;
          if (lx >= 0 && ly >= 0 && lz >= 0 && lx < g.bdim[0] && ly < g.bdim[1] && lz < g.bdim[2])
            o = g.table[((long long)lz * g.bdim[1] + ly) * g.bdim[0] + lx];
          if (o < 0) {
            report_error(rep, kFailedPrecondition, p);
            return;
          }
          const size_t slot = (size_t)o * kBlockCells + ((fk - 8 * bz) * 64 + (fj - 8 * by) * 8 + (fi - 8 * bx));
          const double weight = __dmul_rn(__dmul_rn(w[0][kx], w[1][ky]), w[2][kz]);
          const double mc = __dmul_rn(weight, mass);
          const double affine =
              __dadd_rn(__dadd_rn(__dmul_rn(row[0], off[0][kx]), __dmul_rn(row[1], off[1][ky])),
                        __dmul_rn(row[2], off[2][kz]));
          const double mom = __dmul_rn(mc, __dadd_rn(va, affine));
          const double sm = __ddiv_rn(mc, prm.mass_per_quantum);
          const double sp = __ddiv_rn(mom, prm.momentum_per_quantum);
          if (!isfinite(sm) || fabs(sm) > prm.limit || !isfinite(sp) || fabs(sp) > prm.limit) {
            report_error(rep, kOutOfRange, p);
            return;
          }
          atomicAdd(&mq[a][slot], (unsigned long long)round_nearest_even(sm));
          atomicAdd(&pq[a][slot], (unsigned long long)round_nearest_even(sp));
        }
  }
}

cudaError_t launch_deposit_quanta(const GridView& g, const double* parts, unsigned long long n,
                                  const double origin[3], double h, double mass_per_quantum,
                                  double momentum_per_quantum, double limit, unsigned long long* const mq[3],
                                  unsigned long long* const pq[3], DeviceReport* rep, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  QuantaParams prm;
  for (int d = 0; d < 3; ++d) prm.origin[d] = origin[d];
  prm.h = h;
  prm.mass_per_quantum = mass_per_quantum;
  prm.momentum_per_quantum = momentum_per_quantum;
  prm.limit = limit;
  ++g_kernel_launches;
  k_deposit_quanta<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(g, parts, n, prm, mq[0], mq[1], mq[2], pq[0], pq[1],
                                                                pq[2], rep);
  return cudaGetLastError();
}

}  // namespace fl
