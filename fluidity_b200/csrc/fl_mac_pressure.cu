// Reference-shaped integrated MAC pressure projection on the GPU.
//
// Replaces ProjectMacPressure3D / CudaProjectMacPressure3D
// (native/include/fluidity/host/mac_pressure_3d.h:14-102,
// native/include/fluidity/host/cuda_mac_pressure_3d.h:19-20) for the bounded
// owned-face systems those operators take (1-4096 pressure cells, at most
// 24576 faces): general fluid volumes, target divergences, compliance (bulk
// modulus), wall fluxes, apertures, mobilities, pressure-gradient distances,
// internal pressure jumps, Dirichlet exterior pressures and sealed faces. The
// arithmetic follows the integrated system of native/src/
// mac_pressure_3d_arithmetic.h (FreezeCell :110-146, FreezeLinkFromIncidence
// :174-245, AssembleIntegratedRhsInto :263-313 with compensated sums,
// SelectGaugesInto :328-399, ApplyOriginalPressureOperatorInto :404-436,
// CorrectFacesAndAccumulatePhysicalDefectInto :440-503), the warm start of
// InitializeMacPressure3D (mac_pressure_3d_multigrid.cc:401-419) and the
// evaluation and identity check of mac_pressure_workspace_3d.cc:399-461.
//
// B200 layout. Such a system is a few hundred KB, so one CTA of 1024 threads
// on one SM does all of it in a single launch, in FP64: per-face
// coefficients, then per cell the right-hand side and the diagonal summed over
// its incident faces in increasing face order (the order of the reference's
// face loop, so the compensated sums are the reference's sums), the gauge
// balance of every unanchored component, Jacobi-preconditioned CG from the
// warm start with its six vectors in shared memory (each face entry resolved
// once to its other cell and conductance), and the evaluation (corrected face
// velocities, residuals, physical defects, the residual/defect identity). The
// host does only index
// work: face endpoints by binary search, per-cell face lists, connected
// components and gauges. This file is compiled with -fmad=false so that no
// product is fused into a sum, as in the reference's FP64 arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {
namespace {

constexpr int kMpThreads = 1024;
constexpr uint64_t kMpMaxCells = 4096;   // mac_pressure_3d_arithmetic.h:19
constexpr uint64_t kMpMaxFaces = 24576;  // mac_pressure_3d_arithmetic.h:20
constexpr int kMpMaxIterations = 65536;

enum { kLinkSealed = 0, kLinkInternal = 1, kLinkDirichlet = 2 };

struct MpStatus {
  int status;
  int iterations;
  int arch;
  double true_residual_l2, max_volume_scaled_residual, max_defect, rhs_l2;
};

// Device view of one system. Per-cell face lists hold (face << 1) | side,
// side 1 when the cell is the face's head; unanchored components list their
// cells and their faces that do not join two cells of the same component,
// with the sign of the face's wall flux in the component's balance.
struct MpSystem {
  int nc, nf, ncomp;
  double h, dt, rel_tol;
  int max_iterations;
  const double* cell_values;  // nc x 5
  const double* face_values;  // nf x 6
  const int* face_kind;
  const int* tail;
  const int* head;
  const int* cell_off;  // nc + 1
  const int* cell_ent;
  const int* root;       // component root (smallest ordinal) per cell
  const unsigned char* pinned;
  const int* comp_cell_off;  // ncomp + 1 (unanchored components only)
  const int* comp_cells;
  const int* comp_face_off;
  const int* comp_faces;  // (face << 1) | (1 when the component holds the head)
  // work and results
  int* ent_other;                                         // per face entry: (other cell << 1) | side
  double* ent_cond;                                       // per face entry: the face's conductance
  double *scale, *cond, *wall_face;                       // nf
  double *compliance, *rhs, *rhs_abs;                    // nc
  double *p, *residual, *defect;                          // nc (the solver's vectors are in shared memory)
  double* corrected_u;                                    // nf
  MpStatus* out;
};

// Neumaier-compensated sum (CompensatedSum, mac_pressure_3d_arithmetic.h:57-74).
struct NSum {
  double sum = 0.0, corr = 0.0;
  __device__ void add(double t) {
    const double next = sum + t;
    if (fabs(sum) >= fabs(t))
      corr += (sum - next) + t;
    else
      corr += (t - next) + sum;
    sum = next;
  }
  __device__ double total() const { return sum + corr; }
};
struct Row {
  NSum flux, absolute;
  __device__ void add(double t) {
    flux.add(t);
    absolute.add(fabs(t));
  }
};

// Sum of v over the CTA, returned to every thread (fixed order for a fixed launch).
__device__ double cta_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();  // red may still be read from the previous call
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < kMpThreads / 32; ++k) s += red[k];
  return s;
}
// Two sums over the CTA in one pair of barriers, each exactly as cta_sum forms it.
__device__ double2 cta_sum2(double a, double b, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    red[w] = a;
    red[kMpThreads / 32 + w] = b;
  }
  __syncthreads();
  double sa = 0.0, sb = 0.0;
  for (int k = 0; k < kMpThreads / 32; ++k) {
    sa += red[k];
    sb += red[kMpThreads / 32 + k];
  }
  return make_double2(sa, sb);
}
__device__ double cta_max(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < kMpThreads / 32; ++k) s = fmax(s, red[k]);
  return s;
}

// out_i = (A x)_i: compliance, then each incident face's flux in face order.
// Entries are resolved once (other endpoint, conductance), so a row needs no
// face lookup; the flux is c (x_tail - x_head) as in the face loop, with a
// missing endpoint at zero.
// Every cell lists exactly its six incident faces (the host checks the face
// set), so row i's entries are 6i .. 6i+5: all twelve loads are issued
// before the sum, which keeps the face order.
__device__ double apply_row(const MpSystem& S, const double* x, int i) {
  const double xi = x[i];
  double out = S.compliance[i] * xi;
  double c[6];
  int o[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    c[k] = S.ent_cond[6 * i + k];
    o[k] = S.ent_other[6 * i + k];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    if (c[k] == 0.0) continue;
    const int other = o[k] >> 1;  // -1: no cell at the other end
    const double xo = other >= 0 ? x[other] : 0.0;
    if (o[k] & 1)
      out -= c[k] * (xo - xi);  // this cell is the head
    else
      out += c[k] * (xi - xo);
  }
  return out;
}

__device__ double corrected_velocity(const MpSystem& S, const double* p, int f) {
  const double* v = S.face_values + 6 * f;
  double u = v[3];
  if (v[0] > 0.0) {
    const int kind = S.face_kind[f];
    const double ext = kind == kLinkDirichlet ? v[5] : 0.0;
    const double jump = kind == kLinkInternal ? v[5] : 0.0;
    const int t = S.tail[f], hd = S.head[f];
    const double pt = t >= 0 ? p[t] : ext, ph = hd >= 0 ? p[hd] : ext;
    u += S.scale[f] * (pt - ph + jump);
  }
  return u;
}

__global__ void __launch_bounds__(kMpThreads, 1) k_mac_pressure(MpSystem S) {
  __shared__ double red[kMpThreads / 32];
  __shared__ int status;
  const int t = threadIdx.x;
  const int nc = S.nc, nf = S.nf;
  // The solver's vectors (at most 6 x 4096 doubles) live in shared memory;
  // the pressure goes to global memory at the end for the host.
  extern __shared__ double vec[];
  double* P = vec;
  double* D = P + nc;
  double* R = D + nc;
  double* Q = R + nc;
  double* Z = Q + nc;
  double* DG = Z + nc;
  if (t == 0) {
    status = FL_OK;
    S.out->arch = compiled_arch();
  }
  const double full_area = S.h * S.h;
  // Face coefficients (FreezeLinkFromIncidence).
  for (int f = t; f < nf; f += kMpThreads) {
    const double* v = S.face_values + 6 * f;
    double sc = 0.0, c = 0.0;
    if (v[0] > 0.0) {
      sc = (S.dt * v[1]) / v[2];
      c = v[0] * sc;
    }
    S.scale[f] = sc;
    S.cond[f] = c;
    S.wall_face[f] = (full_area - v[0]) * v[4];
  }
  for (int i = t; i < nc; i += kMpThreads) {
    const double* v = S.cell_values + 5 * i;
    S.compliance[i] = v[2] == 0.0 ? 0.0 : v[0] / (v[2] * S.dt);
  }
  __syncthreads();
  // Right-hand side and diagonal (AssembleIntegratedRhsInto): the cell's own
  // terms, then its faces in increasing face order; each face entry resolved
  // for the operator rows.
  for (int i = t; i < nc; i += kMpThreads) {
    for (int e = S.cell_off[i]; e < S.cell_off[i + 1]; ++e) {
      const int f = S.cell_ent[e] >> 1, side = S.cell_ent[e] & 1;
      const int other = side ? S.tail[f] : S.head[f];
      S.ent_other[e] = other * 2 + side;  // other = -1 gives -2 + side: >> 1 is -1, & 1 the side
      S.ent_cond[e] = S.cond[f];
    }
    const double* v = S.cell_values + 5 * i;
    Row row;
    row.add(v[0] * v[1]);
    row.add(v[4]);
    row.add(S.compliance[i] * v[3]);
    double dg = S.compliance[i];
    for (int e = S.cell_off[i]; e < S.cell_off[i + 1]; ++e) {
      const int f = S.cell_ent[e] >> 1;
      const bool is_head = S.cell_ent[e] & 1;
      const double* fv = S.face_values + 6 * f;
      const double fluid_flux = fv[0] * fv[3];
      const double sgn = is_head ? 1.0 : -1.0;
      row.add(sgn * fluid_flux);
      row.add(sgn * S.wall_face[f]);
      const int kind = S.face_kind[f];
      if (kind == kLinkInternal)
        row.add(sgn * (S.cond[f] * fv[5]));
      else if (kind == kLinkDirichlet)
        row.add(S.cond[f] * fv[5]);
      dg += S.cond[f];
    }
    S.rhs[i] = row.flux.total();
    S.rhs_abs[i] = row.absolute.total();
    DG[i] = dg;
  }
  // Gauge balance of each unanchored component (SelectGaugesInto): its cells'
  // source and wall terms, then the wall flux of its faces, in order.
  for (int k = t; k < S.ncomp; k += kMpThreads) {
    Row bal;
    for (int e = S.comp_cell_off[k]; e < S.comp_cell_off[k + 1]; ++e) {
      const double* v = S.cell_values + 5 * S.comp_cells[e];
      bal.add(v[0] * v[1]);
      bal.add(v[4]);
    }
    for (int e = S.comp_face_off[k]; e < S.comp_face_off[k + 1]; ++e) {
      const int f = S.comp_faces[e] >> 1;
      bal.add((S.comp_faces[e] & 1) ? S.wall_face[f] : -1.0 * S.wall_face[f]);
    }
    if (fabs(bal.flux.total()) > 32.0 * DBL_EPSILON * bal.absolute.total()) atomicExch(&status, FL_FAILED_PRECONDITION);
  }
  __syncthreads();
  if (status != FL_OK) {
    if (t == 0) {
      S.out->status = status;
      S.out->iterations = 0;
      S.out->true_residual_l2 = S.out->max_volume_scaled_residual = S.out->max_defect = S.out->rhs_l2 = 0.0;
    }
    return;  // (uniform: every thread read the same status after the barrier)
  }
  // Warm start: the previous pressure, less the pin's on unanchored components.
  for (int i = t; i < nc; i += kMpThreads) {
    const int rt = S.root[i];
    const double shift = S.pinned[rt] ? S.cell_values[5 * rt + 3] : 0.0;
    P[i] = S.cell_values[5 * i + 3] - shift;
  }
  __syncthreads();
  double bb = 0.0;
  for (int i = t; i < nc; i += kMpThreads) {
    const double q = apply_row(S, P, i);
    R[i] = S.pinned[i] ? 0.0 : S.rhs[i] - q;
    bb += S.rhs[i] * S.rhs[i];
  }
  const double bnorm = sqrt(cta_sum(bb, red));
  // ||b - Ap||_2 <= rel_tol ||b||_2, or the reference's gate 2e-6 + 2e-6 ||b||_2
  const double limit = S.rel_tol > 0.0 ? S.rel_tol * bnorm : 2e-6 + 2e-6 * bnorm;
  // Jacobi-preconditioned CG; the pinned rows stay at their warm start. The
  // residual norm, the preconditioned residual z = r / diag and r.z of each
  // iterate are formed in the pass that updates r (every thread visits its
  // rows in the same order as a separate pass would, so the sums are the same
  // bits), and both sums share one reduction.
  __shared__ double red2[2 * (kMpThreads / 32)];
  double rr = 0.0, rz = 0.0;
  for (int i = t; i < nc; i += kMpThreads) rr += R[i] * R[i];
  for (int i = t; i < nc; i += kMpThreads) {
    const double zi = (S.pinned[i] || DG[i] == 0.0) ? 0.0 : R[i] / DG[i];
    Z[i] = zi;
    rz += R[i] * zi;
  }
  {
    const double2 sums = cta_sum2(rr, rz, red2);
    rr = sums.x;
    rz = sums.y;
  }
  double rz_prev = 0.0;
  int it = 0;
  for (; it < S.max_iterations; ++it) {
    if (sqrt(rr) <= limit) break;
    const double beta = it == 0 ? 0.0 : rz / rz_prev;
    for (int i = t; i < nc; i += kMpThreads) D[i] = it == 0 ? Z[i] : Z[i] + beta * D[i];
    __syncthreads();
    double dq = 0.0;
    for (int i = t; i < nc; i += kMpThreads) {
      const double qi = S.pinned[i] ? 0.0 : apply_row(S, D, i);
      Q[i] = qi;
      dq += D[i] * qi;
    }
    dq = cta_sum(dq, red);
    if (!(dq > 0.0)) {
      if (t == 0) status = FL_ABORTED;
      break;
    }
    const double alpha = rz / dq;
    double rr_next = 0.0, rz_next = 0.0;
    for (int i = t; i < nc; i += kMpThreads) {
      P[i] += alpha * D[i];
      const double ri = R[i] - alpha * Q[i];
      R[i] = ri;
      rr_next += ri * ri;
      const double zi = (S.pinned[i] || DG[i] == 0.0) ? 0.0 : ri / DG[i];
      Z[i] = zi;
      rz_next += ri * zi;
    }
    const double2 sums = cta_sum2(rr_next, rz_next, red2);
    rz_prev = rz;
    rr = sums.x;
    rz = sums.y;
  }
  __syncthreads();
  // Evaluation: corrected faces, residuals b - Ap, physical defects and the
  // identity V d + r = 0 within 64 ulp of the terms' magnitudes.
  for (int f = t; f < nf; f += kMpThreads) {
    const double u = corrected_velocity(S, P, f);
    if (!isfinite(u)) atomicExch(&status, FL_OUT_OF_RANGE);
    S.corrected_u[f] = u;
  }
  __syncthreads();
  double l2 = 0.0, bl2 = 0.0, maxr = 0.0, maxd = 0.0;
  for (int i = t; i < nc; i += kMpThreads) {
    const double* v = S.cell_values + 5 * i;
    Row op, ph;
    op.add(S.compliance[i] * P[i]);
    ph.add(-v[0] * v[1]);
    ph.add(-v[4]);
    if (S.compliance[i] > 0.0) ph.add(S.compliance[i] * (P[i] - v[3]));
    for (int e = S.cell_off[i]; e < S.cell_off[i + 1]; ++e) {
      const int f = S.cell_ent[e] >> 1;
      const bool is_head = S.cell_ent[e] & 1;
      const double c = S.cond[f];
      if (c != 0.0) {
        const int tl = S.tail[f], hd = S.head[f];
        const double pt = tl >= 0 ? P[tl] : 0.0, phd = hd >= 0 ? P[hd] : 0.0;
        const double flux = c * (pt - phd);
        op.add(is_head ? -flux : flux);
      }
      const double flux = S.face_values[6 * f] * S.corrected_u[f];
      if (is_head) {
        ph.add(-flux);
        ph.add(-S.wall_face[f]);
      } else {
        ph.add(flux);
        ph.add(S.wall_face[f]);
      }
    }
    const double r = S.rhs[i] - op.flux.total();
    const double dd = ph.flux.total() / v[0];
    const double ident = v[0] * dd + r;
    const double absterms = S.rhs_abs[i] + op.absolute.total() + ph.absolute.total();
    if (fabs(ident) > 64.0 * DBL_EPSILON * absterms) atomicExch(&status, FL_INTERNAL);
    S.residual[i] = r;
    S.defect[i] = dd;
    S.p[i] = P[i];
    l2 += r * r;
    bl2 += S.rhs[i] * S.rhs[i];
    maxr = fmax(maxr, fabs(r) / v[0]);
    maxd = fmax(maxd, fabs(dd));
  }
  l2 = sqrt(cta_sum(l2, red));
  bl2 = sqrt(cta_sum(bl2, red));
  maxr = cta_max(maxr, red);
  maxd = cta_max(maxd, red);
  __syncthreads();
  if (t == 0) {
    int st = status;
    if (st == FL_OK && l2 > limit * 1.000001 + 1e-300) st = FL_ABORTED;
    S.out->status = st;
    S.out->iterations = it;
    S.out->true_residual_l2 = l2;
    S.out->max_volume_scaled_residual = maxr;
    S.out->max_defect = maxd;
    S.out->rhs_l2 = bl2;
  }
}

bool cell_less(const int32_t* a, const int32_t* b) {
  if (a[2] != b[2]) return a[2] < b[2];
  if (a[1] != b[1]) return a[1] < b[1];
  return a[0] < b[0];
}

int find_cell(const int32_t* cells, int nc, int32_t x, int32_t y, int32_t z) {
  const int32_t key[3] = {x, y, z};
  int lo = 0, hi = nc;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (cell_less(cells + 3 * mid, key))
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < nc && !cell_less(key, cells + 3 * lo)) return lo;
  return -1;
}

// Owned-slot order of a face in the reference's sparse grid of 4^3 blocks
// (SparseMacGrid3D::FaceSlot, sparse_mac_grid_3d.cc:388-409): blocks in
// (z,y,x) order, then the normal axis, then the local (z,y,x) position; the
// face at lattice index (i,j,k) is owned by the block of cell (i,j,k).
using FaceKey = OwnedFaceKey;

FaceKey face_key(int axis, int64_t x, int64_t y, int64_t z) {
  auto fdiv = [](int64_t a) { return (int32_t)(a >= 0 ? a / 4 : -((-a + 3) / 4)); };
  auto fmod = [](int64_t a) { return (int32_t)(((a % 4) + 4) % 4); };
  return FaceKey{{fdiv(z), fdiv(y), fdiv(x), axis, fmod(z), fmod(y), fmod(x)}};
}

// Largest cell bounding box (in lattice positions) given a dense ordinal lookup.
constexpr size_t kMpLutCap = 1 << 20;

// The owned-slot order of faces as two words: (block z, block y) and
// (block x, axis, local z, y, x); int32 order kept by flipping sign bits.
struct PackedFaceKey {
  uint64_t hi, lo;
  bool operator<(const PackedFaceKey& o) const { return hi != o.hi ? hi < o.hi : lo < o.lo; }
};

PackedFaceKey packed_face_key(int axis, int64_t x, int64_t y, int64_t z) {
  const FaceKey k = face_key(axis, x, y, z);  // block z, y, x, axis, local z, y, x
  auto u = [](int32_t v) { return (uint64_t)((uint32_t)v ^ 0x80000000u); };
  const uint64_t local = (uint64_t)((k.v[3] << 6) | (k.v[4] << 4) | (k.v[5] << 2) | k.v[6]);
  return PackedFaceKey{(u(k.v[0]) << 32) | u(k.v[1]), (u(k.v[2]) << 8) | local};
}

int find_root(std::vector<int>& parent, int c) {
  while (parent[c] != c) c = parent[c];
  return c;
}

}  // namespace

// Device arena bytes for nc cells, nf faces, ent cell-face entries, ncomp
// unanchored components, comp_faces component face entries.
size_t mp_arena_bytes(size_t nc, size_t nf, size_t ent, size_t ncomp, size_t comp_faces) {
  const size_t nd_in = 5 * nc + 6 * nf;
  const size_t nd_work = 3 * nf + 6 * nc + nf + ent;
  const size_t ni = 3 * nf + (nc + 1) + ent + nc + (ncomp + 1) + nc + (ncomp + 1) + comp_faces;
  return sizeof(double) * (nd_in + nd_work) + sizeof(MpStatus) + sizeof(int) * (ni + ent) + nc + 64;
}

bool MpScratch::reserve_caps() {
  const size_t nc = kMpMaxCells, nf = kMpMaxFaces;
  try {
    lut.reserve(kMpLutCap);
    tail.reserve(nf);
    head.reserve(nf);
    cell_off.reserve(nc + 1);
    cell_ent.reserve(2 * nf);
    fill.reserve(nc);
    parent.reserve(nc);
    root.reserve(nc);
    comp_of.reserve(nc);
    gauges.reserve(nc);
    comp_cell_off.reserve(nc + 1);
    comp_cells.reserve(nc);
    comp_face_off.reserve(nc + 1);
    comp_faces.reserve(2 * nf);
    host_ints.reserve(4 * nf + 5 * nc + 3);
    anchored.reserve(nc);
    pinned.reserve(nc);
    for (auto* v : {&hp, &hr, &hd, &hb}) v->reserve(nc);
    hu.reserve(nf);
  } catch (...) {
    return false;
  }
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  arena_bytes = mp_arena_bytes(nc, nf, 2 * nf, nc, 2 * nf);
  if (cudaMalloc(&arena, arena_bytes) != cudaSuccess) {
    cudaGetLastError();
    arena = nullptr;
    arena_bytes = 0;
    return false;
  }
  return true;
}

void MpScratch::release() {
  if (arena) cudaFree(arena);
  arena = nullptr;
  arena_bytes = 0;
}

void MpScratch::destroy() {
  release();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  e0 = e1 = nullptr;
}

}  // namespace fl

using namespace fl;

extern "C" int fl_project_mac_pressure_3d(double h, double dt, const int32_t* cell_index, const double* cell_values,
                                          uint64_t cell_count, const int32_t* face_index, const int32_t* face_kind,
                                          const double* face_values, uint64_t face_count, int max_iterations,
                                          double rel_tol, double* pressure, double* corrected_u, double* rhs,
                                          double* residual, double* defect, uint64_t* gauge_ordinals,
                                          fl_mac_pressure_diagnostics* diagnostics, fl_measurement* measurement) {
  MpScratch scratch;  // grows for this call and is released after it
  const int st = fl::mp_project(scratch, nullptr, h, dt, cell_index, cell_values, cell_count, face_index, face_kind,
                                face_values, face_count, max_iterations, rel_tol, pressure, corrected_u, rhs,
                                residual, defect, gauge_ordinals, diagnostics, measurement);
  scratch.destroy();
  return st;
}

namespace fl {

int mp_project(MpScratch& X, cudaStream_t stream, double h, double dt, const int32_t* cell_index,
               const double* cell_values, uint64_t cell_count, const int32_t* face_index, const int32_t* face_kind,
               const double* face_values, uint64_t face_count, int max_iterations, double rel_tol, double* pressure,
               double* corrected_u, double* rhs, double* residual, double* defect, uint64_t* gauge_ordinals,
               fl_mac_pressure_diagnostics* diagnostics, fl_measurement* measurement) {
  if (!(h > 0.0) || !std::isfinite(h) || !(dt > 0.0) || !std::isfinite(dt) || !(rel_tol >= 0.0) ||
      !std::isfinite(rel_tol))
    return FL_INVALID_ARGUMENT;
  if (cell_count == 0 || !cell_index || !cell_values || (face_count && (!face_index || !face_kind || !face_values)))
    return FL_INVALID_ARGUMENT;
  if (!pressure || !rhs || !residual || !defect || (face_count && !corrected_u)) return FL_INVALID_ARGUMENT;
  if (max_iterations < 1 || max_iterations > kMpMaxIterations) return FL_INVALID_ARGUMENT;
  if (cell_count > kMpMaxCells || face_count > kMpMaxFaces) return FL_RESOURCE_EXHAUSTED;
  const int nc = (int)cell_count, nf = (int)face_count;
  for (int i = 0; i < nc; ++i) {
    if (i > 0 && !cell_less(cell_index + 3 * (i - 1), cell_index + 3 * i)) return FL_INVALID_ARGUMENT;
    for (int k = 0; k < 5; ++k)
      if (!std::isfinite(cell_values[5 * i + k])) return FL_INVALID_ARGUMENT;
    if (!(cell_values[5 * i] > 0.0) || cell_values[5 * i + 2] < 0.0) return FL_INVALID_ARGUMENT;
  }
  // The faces must be exactly the cells' incident faces (six per cell, shared
  // faces once), unique and in the reference's owned-slot order, as
  // PrepareMacPressureSystem3D requires (mac_pressure_3d_system.cc:223-239).
  // Checked in the face loop below without building the incident set: the
  // owned-slot keys strictly increase, every face touches a listed cell, and
  // the faces' cell incidences number six per cell.
  for (int i = 0; i < nc; ++i)
    for (int a = 0; a < 3; ++a)
      if (cell_index[3 * i + a] == INT32_MAX) return FL_OUT_OF_RANGE;  // its high face is off the lattice
  // Cell lookups: a dense table over the cells' bounding box when it is small
  // enough, else a binary search of the sorted cells.
  int64_t lo[3], ext[3];
  for (int a = 0; a < 3; ++a) {
    int64_t mn = cell_index[a], mx = cell_index[a];
    for (int i = 1; i < nc; ++i) {
      mn = std::min<int64_t>(mn, cell_index[3 * i + a]);
      mx = std::max<int64_t>(mx, cell_index[3 * i + a]);
    }
    lo[a] = mn;
    ext[a] = mx - mn + 1;
  }
  const int64_t cap = (int64_t)kMpLutCap;
  const bool dense = ext[0] <= cap && ext[1] <= cap && ext[2] <= cap && ext[0] * ext[1] <= cap &&
                     ext[0] * ext[1] * ext[2] <= cap;
  auto& lut = X.lut;
  if (dense) {
    lut.assign((size_t)(ext[0] * ext[1] * ext[2]), -1);
    for (int i = 0; i < nc; ++i) {
      const int32_t* c = cell_index + 3 * i;
      lut[(size_t)(((c[2] - lo[2]) * ext[1] + (c[1] - lo[1])) * ext[0] + (c[0] - lo[0]))] = i;
    }
  }
  auto lookup = [&](int64_t x, int64_t y, int64_t z) {
    if (!dense) return find_cell(cell_index, nc, (int32_t)x, (int32_t)y, (int32_t)z);
    x -= lo[0];
    y -= lo[1];
    z -= lo[2];
    if (x < 0 || y < 0 || z < 0 || x >= ext[0] || y >= ext[1] || z >= ext[2]) return -1;
    return lut[(size_t)((z * ext[1] + y) * ext[0] + x)];
  };
  // Face endpoints and the link rules (internal: two cells; Dirichlet: one
  // cell and an open aperture; sealed: closed; the aperture within the full
  // face, mac_pressure_3d_arithmetic.h:182).
  auto& tail = X.tail;
  auto& head = X.head;
  tail.assign(nf, -1);
  head.assign(nf, -1);
  PackedFaceKey prev{0, 0};
  long long incidences = 0;
  for (int f = 0; f < nf; ++f) {
    const int32_t* fi = face_index + 4 * f;
    const double* v = face_values + 6 * f;
    if (fi[0] < 0 || fi[0] > 2 || face_kind[f] < kLinkSealed || face_kind[f] > kLinkDirichlet) return FL_INVALID_ARGUMENT;
    const PackedFaceKey key = packed_face_key(fi[0], fi[1], fi[2], fi[3]);
    if (f > 0 && !(prev < key)) return FL_INVALID_ARGUMENT;
    prev = key;
    for (int k = 0; k < 6; ++k)
      if (!std::isfinite(v[k])) return FL_INVALID_ARGUMENT;
    if (v[0] < 0.0 || v[0] > h * h) return FL_INVALID_ARGUMENT;
    int64_t tc[3] = {fi[1], fi[2], fi[3]};
    tc[fi[0]] -= 1;
    tail[f] = tc[fi[0]] < INT32_MIN ? -1 : lookup(tc[0], tc[1], tc[2]);
    head[f] = lookup(fi[1], fi[2], fi[3]);
    if (tail[f] < 0 && head[f] < 0) return FL_INVALID_ARGUMENT;
    incidences += (tail[f] >= 0) + (head[f] >= 0);
    const bool both = tail[f] >= 0 && head[f] >= 0, one = (tail[f] >= 0) != (head[f] >= 0);
    const int kind = face_kind[f];
    if (kind == kLinkInternal && !both) return FL_INVALID_ARGUMENT;
    if (kind == kLinkDirichlet && (!one || v[0] == 0.0)) return FL_INVALID_ARGUMENT;
    if (kind == kLinkSealed && v[0] != 0.0) return FL_INVALID_ARGUMENT;
    if (v[0] > 0.0 && !(v[2] > 0.0)) return FL_INVALID_ARGUMENT;
  }
  if (incidences != 6LL * nc) return FL_INVALID_ARGUMENT;
  int st = check_device();
  if (st != FL_OK) return st;
  // Per-cell face lists in increasing face order.
  auto& cell_off = X.cell_off;
  auto& cell_ent = X.cell_ent;
  cell_off.assign(nc + 1, 0);
  for (int f = 0; f < nf; ++f) {
    if (tail[f] >= 0) ++cell_off[tail[f] + 1];
    if (head[f] >= 0) ++cell_off[head[f] + 1];
  }
  for (int i = 0; i < nc; ++i) cell_off[i + 1] += cell_off[i];
  cell_ent.assign(std::max(cell_off[nc], 1), 0);
  {
    auto& fill = X.fill;
    fill.assign(cell_off.begin(), cell_off.end() - 1);
    for (int f = 0; f < nf; ++f) {
      if (tail[f] >= 0) cell_ent[fill[tail[f]]++] = f << 1;
      if (head[f] >= 0) cell_ent[fill[head[f]]++] = (f << 1) | 1;
    }
  }
  // Components over conducting two-cell faces (union towards the smaller
  // ordinal, so a component's root is its first cell); anchors are compliant
  // cells and Dirichlet faces; every unanchored component pins its root.
  auto& parent = X.parent;
  parent.resize(nc);
  for (int i = 0; i < nc; ++i) parent[i] = i;
  for (int f = 0; f < nf; ++f) {
    const double* v = face_values + 6 * f;
    const double cond = v[0] > 0.0 ? v[0] * ((dt * v[1]) / v[2]) : 0.0;
    if (cond > 0.0 && tail[f] >= 0 && head[f] >= 0) {
      const int a = find_root(parent, tail[f]), b = find_root(parent, head[f]);
      parent[std::max(a, b)] = std::min(a, b);
    }
  }
  auto& root = X.root;
  auto& anchored = X.anchored;
  auto& pinned = X.pinned;
  root.resize(nc);
  anchored.assign(nc, 0);
  pinned.assign(nc, 0);
  for (int i = 0; i < nc; ++i) {
    root[i] = find_root(parent, i);
    const double* v = cell_values + 5 * i;
    if (v[2] != 0.0 && v[0] / (v[2] * dt) > 0.0) anchored[root[i]] = 1;
  }
  for (int f = 0; f < nf; ++f)
    if (face_kind[f] == kLinkDirichlet) anchored[root[tail[f] >= 0 ? tail[f] : head[f]]] = 1;
  auto& comp_of = X.comp_of;
  auto& gauges = X.gauges;
  comp_of.assign(nc, -1);
  gauges.clear();
  for (int i = 0; i < nc; ++i)
    if (root[i] == i && !anchored[i]) {
      pinned[i] = 1;
      comp_of[i] = (int)gauges.size();
      gauges.push_back(i);
    }
  const int ncomp = (int)gauges.size();
  // Each unanchored component's cells (ascending) and its faces that do not
  // join two cells of the component (ascending), by counting then filling.
  auto& comp_cell_off = X.comp_cell_off;
  auto& comp_cells = X.comp_cells;
  auto& comp_face_off = X.comp_face_off;
  auto& comp_faces = X.comp_faces;
  comp_cell_off.assign(ncomp + 1, 0);
  comp_face_off.assign(ncomp + 1, 0);
  for (int i = 0; i < nc; ++i)
    if (comp_of[root[i]] >= 0) ++comp_cell_off[comp_of[root[i]] + 1];
  for (int f = 0; f < nf; ++f) {
    const int tl = tail[f], hd = head[f];
    if (tl >= 0 && hd >= 0 && root[tl] == root[hd]) continue;
    if (tl >= 0 && comp_of[root[tl]] >= 0) ++comp_face_off[comp_of[root[tl]] + 1];
    if (hd >= 0 && comp_of[root[hd]] >= 0) ++comp_face_off[comp_of[root[hd]] + 1];
  }
  for (int k = 0; k < ncomp; ++k) {
    comp_cell_off[k + 1] += comp_cell_off[k];
    comp_face_off[k + 1] += comp_face_off[k];
  }
  comp_cells.assign(comp_cell_off[ncomp], 0);
  comp_faces.assign(comp_face_off[ncomp], 0);
  {
    auto& fill = X.fill;
    fill.assign(comp_cell_off.begin(), comp_cell_off.end() - 1);
    for (int i = 0; i < nc; ++i)
      if (comp_of[root[i]] >= 0) comp_cells[fill[comp_of[root[i]]]++] = i;
    fill.assign(comp_face_off.begin(), comp_face_off.end() - 1);
    for (int f = 0; f < nf; ++f) {
      const int tl = tail[f], hd = head[f];
      if (tl >= 0 && hd >= 0 && root[tl] == root[hd]) continue;
      if (tl >= 0 && comp_of[root[tl]] >= 0) comp_faces[fill[comp_of[root[tl]]]++] = f << 1;
      if (hd >= 0 && comp_of[root[hd]] >= 0) comp_faces[fill[comp_of[root[hd]]]++] = (f << 1) | 1;
    }
  }
  // One device arena: inputs, index lists, work arrays and the status.
  const size_t bytes = mp_arena_bytes(nc, nf, cell_ent.size(), ncomp, comp_faces.size());
  if (X.arena_bytes < bytes) {
    X.release();
    if (cudaMalloc(&X.arena, bytes) != cudaSuccess) {
      cudaGetLastError();
      X.arena = nullptr;
      return FL_RESOURCE_EXHAUSTED;
    }
    X.arena_bytes = bytes;
  }
  if (!X.e0 && (cudaEventCreate(&X.e0) != cudaSuccess || cudaEventCreate(&X.e1) != cudaSuccess)) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  MpSystem S{};
  S.nc = nc;
  S.nf = nf;
  S.ncomp = ncomp;
  S.h = h;
  S.dt = dt;
  S.rel_tol = rel_tol;
  S.max_iterations = max_iterations;
  double* dp = reinterpret_cast<double*>(X.arena);
  auto take_d = [&](size_t n) {
    double* r = dp;
    dp += n;
    return r;
  };
  double* d_cells = take_d((size_t)5 * nc);
  double* d_faces = take_d((size_t)6 * nf);
  S.scale = take_d(nf);
  S.cond = take_d(nf);
  S.wall_face = take_d(nf);
  S.compliance = take_d(nc);
  S.rhs = take_d(nc);
  S.rhs_abs = take_d(nc);
  S.p = take_d(nc);
  S.residual = take_d(nc);
  S.defect = take_d(nc);
  S.corrected_u = take_d(nf);
  S.ent_cond = take_d(cell_ent.size());
  S.out = reinterpret_cast<MpStatus*>(dp);
  int* ip = reinterpret_cast<int*>(S.out + 1);
  auto& host_ints = X.host_ints;
  host_ints.clear();
  auto put = [&](const int* src, size_t n) {
    int* r = ip + host_ints.size();
    host_ints.insert(host_ints.end(), src, src + n);
    return r;
  };
  S.face_kind = put(face_kind, nf);
  S.tail = put(tail.data(), nf);
  S.head = put(head.data(), nf);
  S.cell_off = put(cell_off.data(), nc + 1);
  S.cell_ent = put(cell_ent.data(), cell_ent.size());
  S.root = put(root.data(), nc);
  S.comp_cell_off = put(comp_cell_off.data(), ncomp + 1);
  S.comp_cells = put(comp_cells.data(), comp_cells.size());
  S.comp_face_off = put(comp_face_off.data(), ncomp + 1);
  S.comp_faces = put(comp_faces.data(), comp_faces.size());
  S.ent_other = ip + host_ints.size();  // written by the kernel
  unsigned char* d_pinned = reinterpret_cast<unsigned char*>(S.ent_other + cell_ent.size());
  S.pinned = d_pinned;
  S.cell_values = d_cells;
  S.face_values = d_faces;
  cudaStream_t s = stream;
  MpStatus res{};
  float ms = 0.0f;
  bool ok = cudaMemcpyAsync(d_cells, cell_values, sizeof(double) * 5 * nc, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            (nf == 0 || cudaMemcpyAsync(d_faces, face_values, sizeof(double) * 6 * nf, cudaMemcpyHostToDevice, s) ==
                            cudaSuccess) &&
            cudaMemcpyAsync(ip, host_ints.data(), sizeof(int) * host_ints.size(), cudaMemcpyHostToDevice, s) ==
                cudaSuccess &&
            cudaMemcpyAsync(d_pinned, pinned.data(), nc, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaEventRecord(X.e0, s) == cudaSuccess;
  if (ok) {
    const size_t vec_bytes = sizeof(double) * 6 * (size_t)nc;
    static unsigned long long configured = 0;
    if (first_on_device(configured))
      cudaFuncSetAttribute(k_mac_pressure, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(sizeof(double) * 6 * kMpMaxCells));
    ++g_kernel_launches;
    k_mac_pressure<<<1, kMpThreads, vec_bytes, s>>>(S);
    ok = cudaGetLastError() == cudaSuccess && cudaEventRecord(X.e1, s) == cudaSuccess &&
         cudaMemcpyAsync(&res, S.out, sizeof(MpStatus), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess && cudaEventElapsedTime(&ms, X.e0, X.e1) == cudaSuccess;
  }
  auto &hp = X.hp, &hr = X.hr, &hd = X.hd, &hb = X.hb, &hu = X.hu;
  if (ok && res.status == FL_OK) {
    hp.resize(nc);
    hr.resize(nc);
    hd.resize(nc);
    hb.resize(nc);
    hu.resize(std::max(nf, 1));
    ok = cudaMemcpyAsync(hp.data(), S.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(hr.data(), S.residual, sizeof(double) * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(hd.data(), S.defect, sizeof(double) * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaMemcpyAsync(hb.data(), S.rhs, sizeof(double) * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         (nf == 0 || cudaMemcpyAsync(hu.data(), S.corrected_u, sizeof(double) * nf, cudaMemcpyDeviceToHost, s) ==
                         cudaSuccess) &&
         cudaStreamSynchronize(s) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  if (diagnostics) {
    diagnostics->iterations = (uint64_t)res.iterations;
    diagnostics->true_residual_l2 = res.true_residual_l2;
    diagnostics->max_volume_scaled_residual = res.max_volume_scaled_residual;
    diagnostics->max_cell_constraint_defect = res.max_defect;
    diagnostics->rhs_l2 = res.rhs_l2;
    diagnostics->gauge_count = (uint64_t)ncomp;
  }
  if (measurement) {
    measurement->compiled_architecture = res.arch;
    measurement->kernel_ms = ms;
  }
  if (res.status != FL_OK) return res.status;  // no projection is published
  std::memcpy(pressure, hp.data(), sizeof(double) * nc);
  std::memcpy(residual, hr.data(), sizeof(double) * nc);
  std::memcpy(defect, hd.data(), sizeof(double) * nc);
  std::memcpy(rhs, hb.data(), sizeof(double) * nc);
  if (nf) std::memcpy(corrected_u, hu.data(), sizeof(double) * nf);
  if (gauge_ordinals)
    for (int k = 0; k < ncomp; ++k) gauge_ordinals[k] = (uint64_t)gauges[k];
  return FL_OK;
}

}  // namespace fl
