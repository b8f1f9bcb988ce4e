// Bounded boundary-aware transfers on the reference's owned sparse grid: the
// operations behind the liquid scheduler's backend table (.deposit, .normalize,
// .predict_missing_face, .forces, .gather, .freeze, .wetted_piston, .links,
// and the bounded projection's staging; liquid_substep_backend_3d.h:121-194).
//
// Restated from the reference's CPU operations, which its CPU table binds
// (liquid_substep_3d_cpu.cc:775-803, 847-849):
//   owned stencil      sparse_mac_grid_3d.cc:42-58 (floor division, lattice
//                      shifts), 79-254 (coordinate normalisation, lattice
//                      edges, sort bin, half-cell motion), 266-336 (axis
//                      stencil, physical weight gradient), 388-409 (owned
//                      slot), 451-548 and 627-656 (the 27 samples)
//   compatible deposit liquid_boundary_transfer_3d.cc:327-460
//   normalize          liquid_boundary_transfer_3d.cc:463-517
//   ghost continuation liquid_boundary_transfer_3d.cc:97-306 (history checks,
//                      anchors, donors, wall projection) and the pivoted
//                      Householder fit of base/liquid_boundary_transfer_math_3d.h:
//                      35-144
//   gather             liquid_boundary_transfer_3d.cc:519-653 with
//                      mac_gather_3d_internal.h:15-67
//   forces / predict   liquid_substep_3d_cpu.cc:156-179, 782-800
//   geometry freeze    liquid_boundary_geometry_3d.cc:765-1075 (FreezeCore) with
//                      the queries of base/liquid_boundary_geometry_math_3d.h:
//                      160-415 (clipping, measures), 657-847 (modes)
//   pressure links     liquid_boundary_geometry_3d.cc:1077-1380
//   wetted piston      wetted_piston_3d.cc:60-575 with base/wetted_piston_math_3d.h
// The whole file is compiled without FMA contraction (-fmad=false), so every
// expression rounds as the CPU's does; fma() appears only where the reference
// calls std::fma.
//
// Layout: one thread per (particle, component) for the deposit and the
// stencils, one per (particle, component, sample) for the ghost fills, one per
// particle for the gather's sums, one per face slot for normalize and forces.
// Errors are ordered: a failing lane writes atomicMin((order << 8) | code) into
// the report, where order follows the CPU loop (particle, component, sample,
// old then new history), so the call returns the CPU's first error.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "fl_internal.cuh"
#include "fl_kernels.h"
#include "../../include/fluidity_b200.h"

namespace fl {
namespace {

constexpr int kMaxParticles = 1024;
constexpr int kMaxFaces = 24576;
constexpr int kMaxBlocks = kMaxFaces / 192;
constexpr int kGhostRows = 36;  // same-component anchors within 2h of a lattice target (33, or 36 shifted)
constexpr int kFitRowCap = 125;
constexpr int kMaxDonors = 268;
constexpr long long kMaxQuantaSum = 1LL << 62;
constexpr unsigned long long kNoError = ~0ULL;

constexpr int kValidityMissing = 0, kValidityValid = 1, kValidityPredicted = 2, kValidityLowMass = 3;

struct Grid {
  double origin[3];
  double h;
  const int* blocks;  // nb x 3
  int nb;
};

struct Report {
  unsigned long long key;  // (order << 8) | code, kNoError when clean
  int arch;
  int pad;
  double predicted;  // predict_face result
};

__device__ __forceinline__ void fail(Report* r, unsigned long long order, int code) {
  atomicMin(&r->key, (order << 8) | (unsigned long long)code);
}

__device__ __forceinline__ bool finite3(const double* v) { return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]); }

__device__ __forceinline__ bool is_normal(double v) { return isfinite(v) && fabs(v) >= DBL_MIN; }

// ---- owned-grid stencil (sparse_mac_grid_3d.cc) ----

__device__ __forceinline__ long long floor_div4(long long i) { return i >= 0 ? i / 4 : -1 - (-(i + 1)) / 4; }

// FastTwoSum residual of a finite subtraction.
__device__ __forceinline__ double subtraction_roundoff(double a, double b, double diff) {
  if (fabs(a) >= fabs(b)) return (a - diff) - b;
  return a - (diff + b);
}

// A world coordinate in cell units with the subtraction's residual kept, so
// lattice decisions near an edge use the unrounded position.
struct Coord {
  double cells;       // rounded (x - origin) / h
  double diff;        // scaled x - origin
  double diff_error;  // its rounding residual
  double width;       // scaled h
  int scale_exp;
  __device__ double scaled_offset(double edge) const { return fma(-edge, width, diff) + diff_error; }
  __device__ bool below(double edge) const {
    const double off = cells - edge;
    const double bound = fabs(cells) * (2.0 * DBL_EPSILON);
    if (fabs(off) > bound) return off < 0.0;
    return scaled_offset(edge) < 0.0;
  }
  __device__ double offset_from(double edge) const {
    const double off = cells - edge;
    if (fabs(off) >= fabs(cells) && off != 0.0) return off;
    const double s = scaled_offset(edge);
    return isfinite(s) ? s / width : off;
  }
  __device__ double displacement(double anchor, double h) const {
    const double nd = -offset_from(anchor);
    const double d = nd * h;
    if (is_normal(nd) && isfinite(d)) return d;
    const double s = scaled_offset(anchor);
    return s == 0.0 ? 0.0 : -scalbn(s, -scale_exp);
  }
};

__device__ Coord make_coord(double x, double origin, double h) {
  double diff = x - origin;
  int e = 0;
  if (!isfinite(diff)) {
    x *= 0.5;
    origin *= 0.5;
    diff = x - origin;
    e = -1;
  }
  double width = scalbn(h, e);
  const double cells = diff / width;
  double err = subtraction_roundoff(x, origin, diff);
  if (isfinite(cells) && width < 0x1p-960) {
    e += 64;
    diff = scalbn(diff, 64);
    err = scalbn(err, 64);
    width = scalbn(width, 64);
  }
  return Coord{cells, diff, err, width, e};
}

__device__ long long floor_shifted(const Coord& c, double shift) {
  const long long cand = (long long)floor(c.cells - shift);
  const double edge = (double)cand + shift;
  if (c.below(edge)) return cand - 1;
  if (c.below(edge + 1.0)) return cand;
  return cand + 1;
}

__device__ bool within_half_cell(double a, double b, double h) {
  const double hi = fmax(a, b), lo = fmin(a, b);
  const double d = hi - lo;
  const double dd = 2.0 * d;
  if (dd != h) return dd < h;
  return subtraction_roundoff(hi, lo, d) <= 0.0;
}

// Quadratic B-spline factor; an outer factor keeps its edge distance so an
// underflowed weight still has an exponent.
struct Factor {
  double value;
  double edge = 0.0;
  __device__ bool zero() const { return value == 0.0 && edge == 0.0; }
  __device__ double mantissa(int* e) const {
    if (is_normal(value) || edge == 0.0) return frexp(value, e);
    int de;
    const double dm = frexp(edge, &de);
    *e = 2 * de;
    return 0.5 * dm * dm;
  }
};

__device__ double weight_gradient(Factor x, Factor y, Factor z, double h) {
  const double g = x.value * y.value * z.value;
  if (is_normal(g) || x.zero() || y.zero() || z.zero()) return g / h;
  int ex, ey, ez, eh;
  const double mx = x.mantissa(&ex), my = y.mantissa(&ey), mz = z.mantissa(&ez);
  const double mh = frexp(h, &eh);
  return scalbn((mx * my * mz) / mh, ex + ey + ez - eh);
}

struct AxisSamples {
  int lattice[3];
  Factor w[3];
  double disp[3];
  double deriv[3];
};

__device__ int axis_samples(const Coord& c, double shift, int bin, double h, AxisSamples* a) {
  const double start = shift + 0.5;
  const double lo_edge = (double)INT32_MIN + start;
  const double hi_edge = (double)(INT32_MAX - 1) + start;
  if (c.below(lo_edge) || !c.below(hi_edge)) return kOutOfRange;
  const long long first = floor_shifted(c, start);
  const long long tile = (long long)bin * 4;
  if (first < tile || first + 2 >= tile + 8) return kFailedPrecondition;
  const double a0 = (double)first + shift;
  const double dl = c.offset_from(a0 + 0.5);
  const double dr = fabs(c.offset_from(a0 + 1.5));
  const double mid = c.offset_from(a0 + 1.0);
  a->w[0] = Factor{0.5 * dr * dr, dr};
  a->w[1] = Factor{0.75 - mid * mid, 0.0};
  a->w[2] = Factor{0.5 * dl * dl, dl};
  a->deriv[0] = -dr;
  a->deriv[1] = -2.0 * mid;
  a->deriv[2] = dl;
  for (int s = 0; s < 3; ++s) {
    const long long li = first + s;
    a->lattice[s] = (int)li;
    a->disp[s] = c.displacement((double)li + shift, h);
  }
  return kOk;
}

// Ordinal of block (x,y,z) among the sorted active blocks, -1 if inactive.
__device__ int block_ordinal(const Grid& g, long long bx, long long by, long long bz) {
  int lo = 0, hi = g.nb;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const int* b = g.blocks + 3 * mid;
    const bool less = b[2] != bz ? b[2] < bz : (b[1] != by ? b[1] < by : b[0] < bx);
    if (less)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < g.nb) {
    const int* b = g.blocks + 3 * lo;
    if (b[0] == bx && b[1] == by && b[2] == bz) return lo;
  }
  return -1;
}

struct Sample {
  long long slot;
  double w;
  double off[3];
  double grad[3];
};

// The particle's 27 owned samples of one face component, (z,y,x) order.
__device__ int owned_stencil(const Grid& g, int axis, const double* sorted, const double* trial, Sample* out) {
  Coord cs[3], ct[3];
  if (!finite3(sorted)) return kInvalidArgument;
  for (int d = 0; d < 3; ++d) {
    cs[d] = make_coord(sorted[d], g.origin[d], g.h);
    if (!isfinite(cs[d].cells)) return kOutOfRange;
  }
  if (!finite3(trial)) return kInvalidArgument;
  for (int d = 0; d < 3; ++d) {
    ct[d] = make_coord(trial[d], g.origin[d], g.h);
    if (!isfinite(ct[d].cells)) return kOutOfRange;
  }
  int bin[3];
  const double bin_lo = (double)((long long)INT32_MIN * 4) + 1.5;
  const double bin_hi = (double)(((long long)INT32_MAX + 1) * 4) + 1.5;
  for (int d = 0; d < 3; ++d) {
    if (cs[d].below(bin_lo) || !cs[d].below(bin_hi)) return kOutOfRange;
    bin[d] = (int)floor_div4(floor_shifted(cs[d], 1.5));
  }
  for (int d = 0; d < 3; ++d)
    if (!within_half_cell(sorted[d], trial[d], g.h)) return kFailedPrecondition;
  AxisSamples ax[3];
  for (int d = 0; d < 3; ++d) {
    const int st = axis_samples(ct[d], d == axis ? 0.0 : 0.5, bin[d], g.h, &ax[d]);
    if (st != kOk) return st;
  }
  int k = 0;
  for (int sz = 0; sz < 3; ++sz)
    for (int sy = 0; sy < 3; ++sy)
      for (int sx = 0; sx < 3; ++sx, ++k) {
        Sample& s = out[k];
        s.off[0] = ax[0].disp[sx];
        s.off[1] = ax[1].disp[sy];
        s.off[2] = ax[2].disp[sz];
        s.grad[0] = weight_gradient(Factor{ax[0].deriv[sx]}, ax[1].w[sy], ax[2].w[sz], g.h);
        s.grad[1] = weight_gradient(ax[0].w[sx], Factor{ax[1].deriv[sy]}, ax[2].w[sz], g.h);
        s.grad[2] = weight_gradient(ax[0].w[sx], ax[1].w[sy], Factor{ax[2].deriv[sz]}, g.h);
        if (!finite3(s.off) || !finite3(s.grad)) return kOutOfRange;
        s.w = ax[0].w[sx].value * ax[1].w[sy].value * ax[2].w[sz].value;
      }
  k = 0;
  for (int sz = 0; sz < 3; ++sz)
    for (int sy = 0; sy < 3; ++sy)
      for (int sx = 0; sx < 3; ++sx, ++k) {
        const long long li[3] = {ax[0].lattice[sx], ax[1].lattice[sy], ax[2].lattice[sz]};
        const long long b[3] = {floor_div4(li[0]), floor_div4(li[1]), floor_div4(li[2])};
        const int o = block_ordinal(g, b[0], b[1], b[2]);
        if (o < 0) return kFailedPrecondition;
        const long long local = ((li[2] - 4 * b[2]) * 4 + (li[1] - 4 * b[1])) * 4 + (li[0] - 4 * b[0]);
        out[k].slot = (long long)o * 192 + axis * 64 + local;
      }
  return kOk;
}

__device__ __forceinline__ long long round_nearest_even(double s) {
  const double mag = fabs(s);
  const double integral = floor(mag);
  const double frac = mag - integral;
  long long q = (long long)integral;
  if (frac > 0.5 || (frac == 0.5 && (q & 1))) ++q;
  return s < 0.0 ? -q : q;
}

__device__ __forceinline__ bool compatible(const fl_face_tag& t, long long side) {
  return t.structurally_eligible && t.side_tag == side;
}

__device__ __forceinline__ bool usable(uint8_t v) { return v == kValidityValid || v == kValidityPredicted; }

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

// ---- compatible deposit ----

struct DepositArgs {
  Grid g;
  const fl_boundary_particle* parts;
  int n;
  const fl_face_tag* tags;
  double mass_q, mom_q, limit;
  unsigned long long* quanta;  // 3 x int64 per slot (mass, momentum, stress)
  fl_compatible_sample* stencils;
  Report* rep;
};

__global__ void k_compatible_deposit(DepositArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) a.rep->arch = compiled_arch();
  if (t >= 3 * a.n) return;
  const int p = t / 3, comp = t % 3;
  const fl_boundary_particle& q = a.parts[p];
  if (comp == 0 && (!isfinite(q.mass) || q.mass < 0.0 || !finite3(q.velocity))) {
    fail(a.rep, 4ull * p, kInvalidArgument);
    return;
  }
  const unsigned long long order = 4ull * p + 1 + comp;
  Sample st[27];
  int code = owned_stencil(a.g, comp, q.sorted_position, q.trial_position, st);
  if (code != kOk) {
    fail(a.rep, order, code);
    return;
  }
  double row[3] = {0.0, 0.0, 0.0};
  if (q.affine_enabled)
    for (int d = 0; d < 3; ++d) row[d] = q.slopes[3 * comp + d];
  if (!finite3(row)) {
    fail(a.rep, order, kInvalidArgument);
    return;
  }
  double wsum = 0.0, gsum[3] = {0.0, 0.0, 0.0};
  bool ok[27];
  for (int s = 0; s < 27; ++s) {
    ok[s] = compatible(a.tags[st[s].slot], q.side_tag);
    if (ok[s]) {
      wsum += st[s].w;
      for (int d = 0; d < 3; ++d) gsum[d] += st[s].grad[d] * 1.0;
    }
  }
  if (!isfinite(wsum) || !finite3(gsum)) {
    fail(a.rep, order, kOutOfRange);
    return;
  }
  if (wsum <= 0.0) {
    fail(a.rep, order, kFailedPrecondition);
    return;
  }
  fl_compatible_sample* out = a.stencils + (size_t)t * 27;
  double nw[27], mean[3] = {0.0, 0.0, 0.0};
  for (int s = 0; s < 27; ++s) {
    fl_compatible_sample& o = out[s];
    std::memset(&o, 0, sizeof(o));
    o.face_slot = (uint64_t)st[s].slot;
    o.compatible = ok[s];
    if (!ok[s]) continue;
    nw[s] = st[s].w / wsum;
    o.normalized_weight = nw[s];
    for (int d = 0; d < 3; ++d) o.normalized_weight_gradient[d] = (st[s].grad[d] - nw[s] * gsum[d]) / wsum;
    if (!isfinite(nw[s]) || !finite3(o.normalized_weight_gradient)) {
      fail(a.rep, order, kOutOfRange);
      return;
    }
    for (int d = 0; d < 3; ++d) mean[d] += st[s].off[d] * nw[s];
  }
  if (!finite3(mean)) {
    fail(a.rep, order, kOutOfRange);
    return;
  }
  for (int s = 0; s < 27; ++s) {
    if (!ok[s]) continue;
    fl_compatible_sample& o = out[s];
    for (int d = 0; d < 3; ++d) o.centered_face_offset[d] = st[s].off[d] - mean[d];
    if (!finite3(o.centered_face_offset)) {
      fail(a.rep, order, kOutOfRange);
      return;
    }
    const double mc = q.mass * nw[s];
    const double vn = q.velocity[comp] + dot3(row, o.centered_face_offset);
    const double pm = mc * vn;
    const double sm = mc / a.mass_q, sp = pm / a.mom_q;
    if (!isfinite(sm) || fabs(sm) > a.limit || !isfinite(sp) || fabs(sp) > a.limit) {
      fail(a.rep, order, kOutOfRange);
      return;
    }
    unsigned long long* qs = a.quanta + 3 * (size_t)st[s].slot;
    atomicAdd(qs + 0, (unsigned long long)round_nearest_even(sm));
    atomicAdd(qs + 1, (unsigned long long)round_nearest_even(sp));
  }
}

// ---- normalize and forces ----

__global__ void k_normalize(const long long* quanta, int count, double mass_q, double mom_q, double min_mass,
                            double* masses, double* velocities, uint8_t* validity, Report* rep) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f == 0) rep->arch = compiled_arch();
  if (f >= count) return;
  const long long m = quanta[3 * f], p = quanta[3 * f + 1], s = quanta[3 * f + 2];
  if (m < 0 || m > kMaxQuantaSum || p < -kMaxQuantaSum || p > kMaxQuantaSum || s != 0) {
    fail(rep, f, kInvalidArgument);
    return;
  }
  const double dm = (double)m * mass_q, dp = (double)p * mom_q;
  if (!isfinite(dm) || !isfinite(dp)) {
    fail(rep, f, kOutOfRange);
    return;
  }
  masses[f] = dm;
  velocities[f] = 0.0;
  validity[f] = kValidityMissing;
  if (dm == 0.0) return;
  if (dm <= min_mass) {
    validity[f] = kValidityLowMass;
    return;
  }
  const double v = dp / dm;
  if (!isfinite(v)) {
    fail(rep, f, kOutOfRange);
    return;
  }
  velocities[f] = v;
  validity[f] = kValidityValid;
}

__global__ void k_forces(const double* old_v, int count, double ax, double ay, double az, double dt,
                         double* predicted, Report* rep) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f == 0) rep->arch = compiled_arch();
  if (f >= count) return;
  const int axis = (f % 192) / 64;
  const double acc = axis == 0 ? ax : (axis == 1 ? ay : az);
  const double v = old_v[f] + dt * acc;
  if (!isfinite(v)) {
    fail(rep, f, kOutOfRange);
    return;
  }
  predicted[f] = v;
}

// ---- ghost continuation ----

struct History {
  const double* vel;
  const uint8_t* validity;
  const fl_face_tag* tags;
  const fl_wall_sample* walls;
};

__device__ __forceinline__ void slot_anchor(const Grid& g, long long slot, double* a) {
  const int* b = g.blocks + 3 * (slot / 192);
  const int within = (int)(slot % 192);
  const int axis = within / 64, local = within % 64;
  const int l[3] = {local % 4, (local / 4) % 4, local / 16};
  for (int d = 0; d < 3; ++d) a[d] = 4.0 * b[d] + l[d] + (axis == d ? 0.0 : 0.5);
}

struct Continued {
  double v;
  bool fallback;
};

// Least-squares affine fit [1, x, y, z] of the donors by Householder QR with
// column pivoting on recomputed norms, in donor order; rank loss (a pivot
// below 1e-10 of the largest) is a successful non-full-rank result.
__device__ int ghost_fit(const double (*off)[3], const double* vel, int n, bool* full, double* v0) {
  *full = false;
  if (n > kFitRowCap) return kInvalidArgument;
  double A[kGhostRows][4], b[kGhostRows], refl[kGhostRows];
  double scale = 0.0;
  for (int r = 0; r < n; ++r) {
    if (!finite3(off[r]) || !isfinite(vel[r])) return kInvalidArgument;
    A[r][0] = 1.0;
    A[r][1] = off[r][0];
    A[r][2] = off[r][1];
    A[r][3] = off[r][2];
    scale = fmax(scale, fabs(vel[r]));
  }
  if (n < 4) return kOk;
  if (scale == 0.0) scale = 1.0;
  for (int r = 0; r < n; ++r) b[r] = vel[r] / scale;
  int order[4] = {0, 1, 2, 3};
  double largest = 0.0;
  for (int piv = 0; piv < 4; ++piv) {
    int sel = piv;
    double sel_norm = 0.0;
    for (int col = piv; col < 4; ++col) {
      double norm = 0.0;
      for (int r = piv; r < n; ++r) norm = hypot(norm, A[r][col]);
      if (norm > sel_norm) {
        sel_norm = norm;
        sel = col;
      }
    }
    if (!isfinite(sel_norm)) return kOutOfRange;
    largest = fmax(largest, sel_norm);
    if (sel_norm == 0.0 || sel_norm < 1e-10 * largest) return kOk;
    {
      const int t = order[piv];
      order[piv] = order[sel];
      order[sel] = t;
    }
    for (int r = 0; r < n; ++r) {
      const double t = A[r][piv];
      A[r][piv] = A[r][sel];
      A[r][sel] = t;
    }
    const double diag = -copysign(sel_norm, A[piv][piv]);
    double rn = 0.0;
    for (int r = piv; r < n; ++r) {
      refl[r] = A[r][piv] / sel_norm;
      if (r == piv) refl[r] -= diag / sel_norm;
      rn = hypot(rn, refl[r]);
    }
    for (int r = piv; r < n; ++r) refl[r] /= rn;
    for (int col = piv + 1; col < 4; ++col) {
      double proj = 0.0;
      for (int r = piv; r < n; ++r) proj += refl[r] * A[r][col];
      for (int r = piv; r < n; ++r) {
        A[r][col] -= 2.0 * refl[r] * proj;
        if (!isfinite(A[r][col])) return kOutOfRange;
      }
    }
    double bp = 0.0;
    for (int r = piv; r < n; ++r) bp += refl[r] * b[r];
    for (int r = piv; r < n; ++r) b[r] -= 2.0 * refl[r] * bp;
    A[piv][piv] = diag;
  }
  double pc[4] = {0.0, 0.0, 0.0, 0.0}, coef[4] = {0.0, 0.0, 0.0, 0.0};
  for (int piv = 3; piv >= 0; --piv) {
    double res = b[piv];
    for (int col = piv + 1; col < 4; ++col) res -= A[piv][col] * pc[col];
    pc[piv] = res / A[piv][piv];
    coef[order[piv]] = pc[piv] * scale;
    if (!isfinite(coef[order[piv]])) return kOutOfRange;
  }
  *full = true;
  *v0 = coef[0];
  return kOk;
}

// Same-side, same-component donors within sqrt(r2) cell widths of `target`,
// in owned-slot order: the candidate blocks are visited in ordinal order,
// which is the order of a scan over every slot.
__device__ int continue_component(const Grid& g, const History& h, const double* target, int comp, long long side,
                                  const fl_wall_sample& wall, double r2, Continued* out) {
  double off[kGhostRows][3], vel[kGhostRows];
  int n = 0;
  long long nearest = -1;
  double nearest_d2 = INFINITY;
  const double radius = sqrt(r2);
  long long blo[3], bhi[3];
  for (int d = 0; d < 3; ++d) {
    blo[d] = (long long)floor((target[d] - radius - 4.0) / 4.0);
    bhi[d] = (long long)floor((target[d] + radius) / 4.0);
  }
  int cand[64];
  int nc = 0;
  for (long long bz = blo[2]; bz <= bhi[2]; ++bz)
    for (long long by = blo[1]; by <= bhi[1]; ++by)
      for (long long bx = blo[0]; bx <= bhi[0]; ++bx) {
        const int o = block_ordinal(g, bx, by, bz);
        if (o >= 0 && nc < 64) cand[nc++] = o;
      }
  for (int i = 1; i < nc; ++i) {
    const int v = cand[i];
    int j = i - 1;
    while (j >= 0 && cand[j] > v) {
      cand[j + 1] = cand[j];
      --j;
    }
    cand[j + 1] = v;
  }
  for (int ci = 0; ci < nc; ++ci) {
    for (int local = 0; local < 64; ++local) {
      const long long slot = (long long)cand[ci] * 192 + comp * 64 + local;
      if (!compatible(h.tags[slot], side) || !usable(h.validity[slot])) continue;
      double a[3], o[3];
      slot_anchor(g, slot, a);
      for (int d = 0; d < 3; ++d) o[d] = a[d] - target[d];
      const double d2 = dot3(o, o);
      if (d2 > r2) continue;
      if (n == kMaxDonors) return kResourceExhausted;
      if (n == kGhostRows) return kInternal;  // beyond the lattice bound: not reachable at r2 <= 4
      for (int d = 0; d < 3; ++d) off[n][d] = o[d];
      vel[n] = h.vel[slot];
      ++n;
      if (d2 < nearest_d2) {
        nearest = slot;
        nearest_d2 = d2;
      }
    }
  }
  bool full = false;
  double v0 = 0.0;
  const int st = ghost_fit(off, vel, n, &full, &v0);
  if (st != kOk) return st;
  if (full) {
    *out = Continued{v0, false};
    return kOk;
  }
  if (nearest >= 0) {
    *out = Continued{h.vel[nearest], true};
    return kOk;
  }
  if (wall.available && wall.side_tag == side) {
    *out = Continued{wall.wall_velocity[comp], true};
    return kOk;
  }
  return kFailedPrecondition;
}

__device__ int fill_velocity(const Grid& g, const History& h, long long slot, int comp, long long side, double r2,
                             Continued* out) {
  if (compatible(h.tags[slot], side) && usable(h.validity[slot])) {
    *out = Continued{h.vel[slot], false};
    return kOk;
  }
  const fl_wall_sample& wall = h.walls[slot];
  double target[3];
  slot_anchor(g, slot, target);
  int st = continue_component(g, h, target, comp, side, wall, r2, out);
  if (st != kOk) return st;
  const bool wall_ok = wall.available && wall.side_tag == side;
  const double nc = wall.unit_normal[comp];
  if (wall_ok && nc != 0.0) {
    double fitted[3] = {wall.wall_velocity[0], wall.wall_velocity[1], wall.wall_velocity[2]};
    fitted[comp] = out->v;
    for (int o = 0; o < 3; ++o) {
      if (o == comp || wall.unit_normal[o] == 0.0) continue;
      Continued other;
      st = continue_component(g, h, target, o, side, wall, 4.0, &other);
      if (st != kOk) return st;
      fitted[o] = other.v;
      out->fallback = out->fallback || other.fallback;
    }
    double rel[3];
    for (int d = 0; d < 3; ++d) rel[d] = fitted[d] - wall.wall_velocity[d];
    const double rn = dot3(rel, wall.unit_normal);
    out->v -= rn * nc;
    if (!isfinite(out->v)) return kOutOfRange;
  }
  return kOk;
}

// ---- gather ----

// Per (particle, component, sample): the stencil sample and both continued velocities.
struct FillRecord {
  double w;
  double off[3];
  double grad[3];
  double v_old;
  double v_new;
  unsigned flags;  // 1 old fallback, 2 new fallback, 4 low mass in either history, 8 stencil failed
  unsigned slot;   // owned face slot (< 24576)
};

// Per-particle order of the CPU loop: 0 velocity check; component c at
// 1 + 55c (stencil) and 2 + 55c + 2s + history (fills); 166 + c the component
// gathers; 169 the retained residual.
constexpr unsigned long long kGatherOrders = 170;

struct GatherArgs {
  Grid g;
  const fl_boundary_particle* parts;
  int n;
  History old_h, new_h;
  FillRecord* rec;  // n x 3 x 27
  fl_gathered_particle* out;
  Report* rep;
};

__global__ void k_gather_stencils(GatherArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) a.rep->arch = compiled_arch();
  if (t >= 3 * a.n) return;
  const int p = t / 3, comp = t % 3;
  const fl_boundary_particle& q = a.parts[p];
  if (comp == 0 && !finite3(q.velocity)) fail(a.rep, kGatherOrders * p, kInvalidArgument);
  Sample st[27];
  const int code = owned_stencil(a.g, comp, q.sorted_position, q.trial_position, st);
  FillRecord* r = a.rec + (size_t)t * 27;
  if (code != kOk) {
    fail(a.rep, kGatherOrders * p + 1 + 55 * comp, code);
    for (int s = 0; s < 27; ++s) r[s].flags = 8;
    return;
  }
  for (int s = 0; s < 27; ++s) {
    r[s].w = st[s].w;
    for (int d = 0; d < 3; ++d) {
      r[s].off[d] = st[s].off[d];
      r[s].grad[d] = st[s].grad[d];
    }
    r[s].v_old = 0.0;
    r[s].v_new = 0.0;
    r[s].flags = 0;
    r[s].slot = (unsigned)st[s].slot;
  }
}

__global__ void k_gather_fill(GatherArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 81 * a.n) return;
  const int p = t / 81, comp = (t / 27) % 3, s = t % 27;
  FillRecord& r = a.rec[t];
  if (r.flags & 8) return;
  const long long slot = r.slot;
  const long long side = a.parts[p].side_tag;
  const unsigned long long base = kGatherOrders * p + 2 + 55 * comp + 2 * s;
  Continued o, nw;
  int st = fill_velocity(a.g, a.old_h, slot, comp, side, 4.0, &o);
  if (st != kOk) {
    fail(a.rep, base, st);
    return;
  }
  st = fill_velocity(a.g, a.new_h, slot, comp, side, 4.0, &nw);
  if (st != kOk) {
    fail(a.rep, base + 1, st);
    return;
  }
  r.v_old = o.v;
  r.v_new = nw.v;
  r.flags = (o.fallback ? 1u : 0u) | (nw.fallback ? 2u : 0u) |
            ((a.old_h.validity[slot] == kValidityLowMass || a.new_h.validity[slot] == kValidityLowMass) ? 4u : 0u);
}

__global__ void k_gather_finish(GatherArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  const fl_boundary_particle& q = a.parts[p];
  const FillRecord* r = a.rec + (size_t)p * 81;
  for (int i = 0; i < 81; ++i)
    if (r[i].flags & 8) return;  // a stencil failed: reported in order already
  fl_gathered_particle g;
  std::memset(&g, 0, sizeof(g));
  double old_pic[3] = {0.0, 0.0, 0.0};
  unsigned flags = 0;
  for (int c = 0; c < 3; ++c)
    for (int s = 0; s < 27; ++s) {
      const FillRecord& f = r[27 * c + s];
      old_pic[c] += f.w * f.v_old;
      flags |= f.flags;
    }
  g.old_pic_fallback = (flags & 1) != 0;
  g.new_pic_fallback = (flags & 2) != 0;
  g.low_mass_fallback = (flags & 4) != 0;
  const double h = a.g.h;
  for (int c = 0; c < 3; ++c) {
    double op = 0.0, np = 0.0, m[3] = {0.0, 0.0, 0.0}, gr[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < 27; ++s) {
      const FillRecord& f = r[27 * c + s];
      const double wn = f.w * f.v_new;
      op += f.w * f.v_old;
      np += wn;
      const double nd[3] = {f.off[0] / h, f.off[1] / h, f.off[2] / h};
      for (int d = 0; d < 3; ++d) m[d] += nd[d] * wn;
      for (int d = 0; d < 3; ++d) gr[d] += f.grad[d] * f.v_new;
    }
    double slope[3];
    for (int d = 0; d < 3; ++d) slope[d] = (4.0 * m[d]) / h;
    const double inc = np - op;
    if (!isfinite(np) || !isfinite(inc) || !finite3(slope) || !finite3(gr)) {
      fail(a.rep, kGatherOrders * p + 166 + c, kOutOfRange);
      return;
    }
    g.new_pic_velocity[c] = np;
    g.grid_velocity_increment[c] = inc;
    for (int d = 0; d < 3; ++d) {
      g.fitted_velocity_slopes[3 * c + d] = slope[d];
      g.velocity_gradient[3 * c + d] = gr[d];
    }
  }
  const bool pic_fallback = g.old_pic_fallback || g.new_pic_fallback || g.low_mass_fallback;
  g.affine_enabled = q.affine_enabled && !pic_fallback;
  if (!pic_fallback)
    for (int d = 0; d < 3; ++d) g.particle_minus_old_pic_velocity[d] = q.velocity[d] - old_pic[d];
  if (!finite3(g.particle_minus_old_pic_velocity)) {
    fail(a.rep, kGatherOrders * p + 169, kOutOfRange);
    return;
  }
  a.out[p] = g;
}

__global__ void k_predict_face(Grid g, History h, long long slot, long long side, double acc, double dt,
                               Report* rep) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  rep->arch = compiled_arch();
  const int comp = (int)((slot % 192) / 64);
  Continued c;
  const int st = fill_velocity(g, h, slot, comp, side, 4.0, &c);
  if (st != kOk) {
    fail(rep, 0, st);
    return;
  }
  const double v = c.v + dt * acc;
  if (!isfinite(v)) {
    fail(rep, 0, kOutOfRange);
    return;
  }
  rep->predicted = v;
}


// ---- pressure-link assembly (.links) ----

__device__ __forceinline__ bool cell_less(const int32_t* a, const int32_t* b) {
  return a[2] != b[2] ? a[2] < b[2] : (a[1] != b[1] ? a[1] < b[1] : a[0] < b[0]);
}
__device__ __forceinline__ bool cell_equal(const int32_t* a, const int32_t* b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

// Index of the record with cell key `key` in a (z,y,x)-sorted array of records
// `stride` bytes apart whose cell index sits at their start, else -1.
__device__ int find_cell_record(const void* base, int count, size_t stride, const int32_t* key) {
  const char* p = static_cast<const char*>(base);
  int lo = 0, hi = count;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cell_less(reinterpret_cast<const int32_t*>(p + mid * stride), key))
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < count && cell_equal(reinterpret_cast<const int32_t*>(p + lo * stride), key)) return lo;
  return -1;
}

__device__ __forceinline__ bool positive_finite(double v) { return isfinite(v) && v > 0.0; }
__device__ __forceinline__ bool normal_or_zero(double v) { return v == 0.0 || is_normal(v); }

// C++20 std::lerp for a, b > 0 (the monotone, exact-at-the-ends formula of P0811).
__device__ double lerp_positive(double a, double b, double t) {
  if (t == 1.0) return b;
  const double x = a + t * (b - a);
  return (t > 1.0) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}

// C++20 std::midpoint for doubles (P0811).
__device__ double midpoint_double(double a, double b) {
  const double lo = DBL_MIN * 2, hi = DBL_MAX / 2;
  const double aa = a < 0 ? -a : a, ab = b < 0 ? -b : b;
  if (aa <= hi && ab <= hi) return (a + b) / 2;
  if (aa < lo) return a + b / 2;
  if (ab < lo) return a / 2 + b;
  return a / 2 + b / 2;
}

// sqrt((rho_t + rho_h) h^3 / (4 pi sigma)) with the operands scaled to their
// mantissas first, as InternalLiquidCapillaryStepBound3D forms it
// (liquid_boundary_geometry_3d.cc:1669-1698).
__device__ int capillary_step_bound(double tail_density, double head_density, double h, double sigma, double* out) {
  if (!positive_finite(tail_density) || !positive_finite(head_density) || !positive_finite(h) || !isfinite(sigma) ||
      sigma < 0.0)
    return kInvalidArgument;
  if (sigma == 0.0) {
    *out = INFINITY;
    return kOk;
  }
  const double larger = tail_density < head_density ? head_density : tail_density;
  const double smaller = head_density < tail_density ? head_density : tail_density;
  const double ratio = smaller / larger;
  int de, we, te;
  const double sd = frexp(larger, &de) * (1.0 + ratio);
  const double sw = frexp(h, &we);
  const double st = frexp(sigma, &te);
  const double square = sd * sw * sw * sw / (4.0 * 3.141592653589793 * st);
  const int e = de + 3 * we - te;
  const double bound = scalbn(sqrt(scalbn(square, e % 2)), e / 2);
  if (!positive_finite(bound)) return kOutOfRange;
  *out = bound;
  return kOk;
}

struct LinksArgs {
  double h, density, step_duration, sigma, ambient;
  const fl_frozen_cell* cells;
  int nc;
  const fl_frozen_face* faces;
  int nf;
  const fl_pressure_cell_fields* fields;
  const double* predicted;
  const double* wetted;  // nullptr: no wetted piston fluxes
  const uint8_t* has_wetted;
  const fl_air_cell_pressure* air;
  int nair;
  const fl_internal_interface* interfaces;
  int ninterfaces;
  const fl_center_sample* centers;
  int ncenters;
  fl_pressure_link* out;
  uint8_t* regularized;
  Report* rep;
};

// One thread per frozen face: the face's stage, geometry and consume steps
// of LinksCore (liquid_boundary_geometry_3d.cc:1139-1273), errors ordered by face.
__global__ void k_links(LinksArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f == 0) a.rep->arch = compiled_arch();
  if (f >= a.nf) return;
  const fl_frozen_face& face = a.faces[f];
  a.regularized[f] = 0;
  if (!isfinite(a.predicted[f])) {
    fail(a.rep, f, kInvalidArgument);
    return;
  }
  fl_pressure_link link;
  memset(&link, 0, sizeof(link));
  link.axis = face.axis;
  for (int d = 0; d < 3; ++d) link.lattice[d] = face.lattice[d];
  link.open_area = face.open_area;
  link.inverse_density = 1 / a.density;
  link.pressure_gradient_distance = a.h;
  link.predicted_normal_velocity = a.predicted[f];
  link.wall_normal_velocity = face.wall_normal_velocity;
  link.link_kind = 0;
  link.has_prescribed_wall_flux = face.has_prescribed_wall_flux;
  link.prescribed_wall_flux = face.has_prescribed_wall_flux ? face.prescribed_wall_flux : 0.0;
  const int32_t head[3] = {face.lattice[0], face.lattice[1], face.lattice[2]};
  int32_t tail[3] = {head[0], head[1], head[2]};
  const bool tail_ok = head[face.axis] != INT32_MIN;
  if (tail_ok) tail[face.axis] -= 1;
  const int hf = find_cell_record(a.cells, a.nc, sizeof(fl_frozen_cell), head);
  const int tf = tail_ok ? find_cell_record(a.cells, a.nc, sizeof(fl_frozen_cell), tail) : -1;
  const bool has_head = hf >= 0, has_tail = tf >= 0;
  if (a.wetted != nullptr) {
    const bool receiver = face.is_low_x_piston_face && face.axis == 0 && face.open_area == 0 && has_head &&
                          !has_tail && face.has_prescribed_wall_flux;
    const bool has = a.has_wetted[f] != 0;
    if (receiver != has) {
      fail(a.rep, f, kInvalidArgument);
      return;
    }
    if (has) {
      const double flux = a.wetted[f], w = face.wall_normal_velocity;
      const bool wrong = (flux > 0 && w <= 0) || (flux < 0 && w >= 0);
      if (!isfinite(flux) || wrong) {
        fail(a.rep, f, kInvalidArgument);
        return;
      }
      link.has_prescribed_wall_flux = 1;
      link.prescribed_wall_flux = flux;
    }
  }
  // the certified internal interface on this face, if any
  int lo = 0, hi = a.ninterfaces;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a.interfaces[mid].face_ordinal < (uint64_t)f)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < a.ninterfaces && a.interfaces[lo].face_ordinal == (uint64_t)f) {
    const fl_internal_interface& c = a.interfaces[lo];
    if (!has_head || !has_tail || face.open_area <= 0.0 || !a.fields[hf].has_density || !a.fields[tf].has_density) {
      fail(a.rep, f, kInvalidArgument);
      return;
    }
    const double tail_density = a.fields[tf].density, head_density = a.fields[hf].density;
    double bound = 0.0;
    const int st = capillary_step_bound(tail_density, head_density, a.h, c.surface_tension, &bound);
    if (st != kOk) {
      fail(a.rep, f, st);
      return;
    }
    if (a.step_duration > bound) {
      fail(a.rep, f, kAborted);
      return;
    }
    const double face_density = lerp_positive(head_density, tail_density, c.tail_fraction);
    const double inverse_density = 1.0 / face_density;
    const double jump = fma(-c.surface_tension, c.curvature_tail_to_head, c.normal_viscous_jump_tail_to_head);
    if (!is_normal(inverse_density) || !isfinite(jump)) {
      fail(a.rep, f, kOutOfRange);
      return;
    }
    link.inverse_density = inverse_density;
    link.link_kind = 1;
    link.link_value = jump;
    a.out[f] = link;
    return;
  }
  if (!tail_ok) {
    if (face.open_area > 0) {
      fail(a.rep, f, kOutOfRange);
      return;
    }
    a.out[f] = link;
    return;
  }
  if (!has_head && !has_tail) {
    fail(a.rep, f, kFailedPrecondition);
    return;
  }
  if (face.open_area > 0) {
    const bool hd = has_head && a.fields[hf].has_density, td = has_tail && a.fields[tf].has_density;
    if (hd || td) {
      const double head_density = hd ? a.fields[hf].density : a.density;
      const double tail_density = td ? a.fields[tf].density : a.density;
      const double face_density = has_head && has_tail ? midpoint_double(head_density, tail_density)
                                                       : (has_head ? head_density : tail_density);
      link.inverse_density = 1.0 / face_density;
      if (!is_normal(link.inverse_density)) {
        fail(a.rep, f, kOutOfRange);
        return;
      }
    }
  }
  if (has_head && has_tail) {
    link.link_kind = 1;
    link.link_value = 0.0;
  } else if (face.open_area > 0) {
    const int32_t* air_cell = has_head ? tail : head;
    const int ci = find_cell_record(a.centers, a.ncenters, sizeof(fl_center_sample), air_cell);
    if (ci < 0 || a.centers[ci].signed_distance < 0) {
      fail(a.rep, f, kFailedPrecondition);
      return;
    }
    const double air_distance = a.centers[ci].signed_distance;
    const fl_frozen_cell& liquid = a.cells[has_head ? hf : tf];
    const int pi = find_cell_record(a.air, a.nair, sizeof(fl_air_cell_pressure), air_cell);
    const double ambient = pi >= 0 ? a.air[pi].gas_gauge_pressure : a.ambient;
    // the link arithmetic (liquid_boundary_geometry_math_3d.h:676-689)
    const double mag = -liquid.center_distance < air_distance ? air_distance : -liquid.center_distance;
    const double ls = -liquid.center_distance / mag;
    const double theta = ls / (ls + air_distance / mag);
    const double clamped = theta < 0.05 ? 0.05 : (1.0 < theta ? 1.0 : theta);
    const double distance = clamped * a.h;
    const double lift = a.sigma * liquid.curvature;
    const double exterior = ambient + lift;
    if ((a.sigma > 0 && liquid.curvature != 0 && lift == 0) || !normal_or_zero(lift) || !isfinite(exterior) ||
        !is_normal(distance)) {
      fail(a.rep, f, kOutOfRange);
      return;
    }
    a.regularized[f] = theta < 0.05 ? 1 : 0;
    link.pressure_gradient_distance = distance;
    link.link_kind = 2;
    link.link_value = exterior;
  }
  a.out[f] = link;
}

}  // namespace
}  // namespace fl

// ---- host side ----

using namespace fl;

namespace {

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// Offsets of every region; the pinned host buffer mirrors the device arena up
// to `staged` (inputs and outputs); the gather's fill records are device-only.
struct Regions {
  size_t blocks, particles, tags_a, vel_a, valid_a, walls_a, tags_b, vel_b, valid_b, walls_b;
  size_t quanta, stencils, masses, velocities, validity, gathered, report, staged, records, total;
  Regions() {
    size_t o = 0;
    auto take = [&](size_t bytes) {
      const size_t r = o;
      o = align_up(o + bytes);
      return r;
    };
    blocks = take(sizeof(int32_t) * 3 * kMaxBlocks);
    particles = take(sizeof(fl_boundary_particle) * kMaxParticles);
    tags_a = take(sizeof(fl_face_tag) * kMaxFaces);
    vel_a = take(sizeof(double) * kMaxFaces);
    valid_a = take(kMaxFaces);
    walls_a = take(sizeof(fl_wall_sample) * kMaxFaces);
    tags_b = take(sizeof(fl_face_tag) * kMaxFaces);
    vel_b = take(sizeof(double) * kMaxFaces);
    valid_b = take(kMaxFaces);
    walls_b = take(sizeof(fl_wall_sample) * kMaxFaces);
    quanta = take(sizeof(fl_face_quanta) * kMaxFaces);
    stencils = take(sizeof(fl_compatible_sample) * 81 * kMaxParticles);
    masses = take(sizeof(double) * kMaxFaces);
    velocities = take(sizeof(double) * kMaxFaces);
    validity = take(kMaxFaces);
    gathered = take(sizeof(fl_gathered_particle) * kMaxParticles);
    report = take(sizeof(Report));
    staged = o;
    records = take(sizeof(FillRecord) * 81 * kMaxParticles);
    total = o;
  }
};

const Regions kRegions;

}  // namespace

struct fl_boundary {
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  char* dev = nullptr;
  char* pin = nullptr;
  int device = -1;
  fl::MpScratch pressure;  // the bounded projection's scratch, reserved for its caps
  char* ldev = nullptr;    // pressure-link assembly: device arena
  char* lpin = nullptr;    // and its pinned mirror
  char* fdev = nullptr;    // geometry freeze: device arena
  char* fpin = nullptr;    // and its pinned mirror
  char* pdev = nullptr;    // wetted piston: device arena
  char* ppin = nullptr;    // and its pinned mirror (all but the interval banks)
  // Host working storage of the freeze and the wetted piston, reserved at
  // create so that an attempt allocates nothing; results reach the caller's
  // buffers only on success.
  std::vector<double> frz_centre;
  std::vector<uint8_t> frz_needs;
  std::vector<uint64_t> frz_ordinal;
  std::vector<fl_frozen_cell> frz_cells;
  std::vector<fl_frozen_face> frz_faces;
  std::vector<int32_t> pst_idx;
  std::vector<fl_piston_patch> pst_patches;
  std::vector<double> pst_flux;
  std::vector<uint8_t> pst_has;
};

namespace {

static_assert(sizeof(fl_boundary_particle) == 168, "particle record");
static_assert(sizeof(fl_face_tag) == 16, "face tag record");
static_assert(sizeof(fl_face_quanta) == 24, "quanta record");
static_assert(sizeof(fl_compatible_sample) == 72, "compatible sample record");
static_assert(sizeof(fl_wall_sample) == 64, "wall record");
static_assert(sizeof(fl_gathered_particle) == 224, "gather record");

template <typename T>
T* dptr(fl_boundary* b, size_t off) {
  return reinterpret_cast<T*>(b->dev + off);
}
template <typename T>
T* hptr(fl_boundary* b, size_t off) {
  return reinterpret_cast<T*>(b->pin + off);
}

bool pow2_scale(double v) {
  int e = 0;
  return std::isnormal(v) && v > 0.0 && std::frexp(v, &e) == 0.5;
}

// ValidateQuantization (liquid_boundary_transfer_3d.cc:56-73).
int check_quantization(const fl_quantization* q, uint64_t particles) {
  if (!pow2_scale(q->mass_per_quantum) || !pow2_scale(q->momentum_per_quantum)) return FL_INVALID_ARGUMENT;
  if (q->declared_capacity > (uint64_t)kMaxParticles || particles > q->declared_capacity) return FL_RESOURCE_EXHAUSTED;
  return FL_OK;
}

// Blocks as SparseMacGrid3D::Create leaves them: strictly increasing (z,y,x).
int check_grid(const fl_owned_grid* g) {
  if (!g || (g->block_count && !g->blocks)) return FL_INVALID_ARGUMENT;
  if (g->block_count > (uint64_t)kMaxBlocks) return FL_RESOURCE_EXHAUSTED;
  for (uint64_t i = 1; i < g->block_count; ++i) {
    const int32_t* a = g->blocks + 3 * (i - 1);
    const int32_t* b = g->blocks + 3 * i;
    const bool less = a[2] != b[2] ? a[2] < b[2] : (a[1] != b[1] ? a[1] < b[1] : a[0] < b[0]);
    if (!less) return FL_INVALID_ARGUMENT;
  }
  return FL_OK;
}

// ValidateGeometry (sparse_mac_grid_3d.cc:18-27): checked where the CPU
// operation builds its first stencil.
bool geometry_ok(const fl_owned_grid* g) {
  return std::isfinite(g->origin[0]) && std::isfinite(g->origin[1]) && std::isfinite(g->origin[2]) && g->h > 0.0 &&
         std::isnormal(g->h);
}

Grid device_grid(fl_boundary* b, const fl_owned_grid* g) {
  Grid d;
  for (int k = 0; k < 3; ++k) d.origin[k] = g->origin[k];
  d.h = g->h;
  d.blocks = dptr<int>(b, kRegions.blocks);
  d.nb = (int)g->block_count;
  return d;
}

// Stage [off, off + bytes) of the pinned buffer to the device.
bool upload(fl_boundary* b, size_t off, const void* src, size_t bytes) {
  if (bytes == 0) return true;
  std::memcpy(b->pin + off, src, bytes);
  return cudaMemcpyAsync(b->dev + off, b->pin + off, bytes, cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
}

bool download(fl_boundary* b, size_t off, size_t bytes) {
  if (bytes == 0) return true;
  return cudaMemcpyAsync(b->pin + off, b->dev + off, bytes, cudaMemcpyDeviceToHost, b->stream) == cudaSuccess;
}

bool begin(fl_boundary* b) {
  if (cudaSetDevice(b->device) != cudaSuccess) return false;
  const Report clean{kNoError, 0, 0, 0.0};
  return upload(b, kRegions.report, &clean, sizeof(clean)) && cudaEventRecord(b->e0, b->stream) == cudaSuccess;
}

// Waits for the stream; returns the first ordered error, or FL_OK.
int finish(fl_boundary* b, fl_measurement* m) {
  if (cudaGetLastError() != cudaSuccess || cudaEventRecord(b->e1, b->stream) != cudaSuccess ||
      !download(b, kRegions.report, sizeof(Report)) || cudaStreamSynchronize(b->stream) != cudaSuccess) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  const Report* r = hptr<Report>(b, kRegions.report);
  if (m) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    m->compiled_architecture = r->arch;
    m->kernel_ms = ms;
  }
  if (r->key != kNoError) return (int)(r->key & 0xff);
  return FL_OK;
}

int check_history(const fl_velocity_history* h, uint64_t faces, double stage_time) {
  if (!h) return FL_INVALID_ARGUMENT;
  if (h->velocity_sample_time != stage_time || h->wall_sample_time != stage_time) return FL_INVALID_ARGUMENT;
  if (faces && (!h->face_velocities || !h->validity || !h->face_tags || !h->walls)) return FL_INVALID_ARGUMENT;
  for (uint64_t s = 0; s < faces; ++s) {
    const uint8_t v = h->validity[s];
    if (v > kValidityLowMass) return FL_INVALID_ARGUMENT;
    if ((v == kValidityValid || v == kValidityPredicted) && !std::isfinite(h->face_velocities[s]))
      return FL_INVALID_ARGUMENT;
    const fl_wall_sample& w = h->walls[s];
    if (w.available) {
      for (int d = 0; d < 3; ++d)
        if (!std::isfinite(w.wall_velocity[d]) || !std::isfinite(w.unit_normal[d])) return FL_INVALID_ARGUMENT;
      const double* n = w.unit_normal;
      if (std::abs((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2] - 1.0) > 1e-12) return FL_INVALID_ARGUMENT;
    }
  }
  return FL_OK;
}

bool upload_history(fl_boundary* b, const fl_velocity_history* h, uint64_t faces, bool second) {
  const Regions& R = kRegions;
  return upload(b, second ? R.vel_b : R.vel_a, h->face_velocities, sizeof(double) * faces) &&
         upload(b, second ? R.valid_b : R.valid_a, h->validity, faces) &&
         upload(b, second ? R.tags_b : R.tags_a, h->face_tags, sizeof(fl_face_tag) * faces) &&
         upload(b, second ? R.walls_b : R.walls_a, h->walls, sizeof(fl_wall_sample) * faces);
}

History device_history(fl_boundary* b, bool second) {
  const Regions& R = kRegions;
  return History{dptr<double>(b, second ? R.vel_b : R.vel_a), dptr<uint8_t>(b, second ? R.valid_b : R.valid_a),
                 dptr<fl_face_tag>(b, second ? R.tags_b : R.tags_a),
                 dptr<fl_wall_sample>(b, second ? R.walls_b : R.walls_a)};
}

unsigned grid_of(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

namespace {
size_t link_arena_bytes();  // the pressure-link assembly's staging, defined with its regions below
}  // namespace
size_t freeze_arena_bytes();  // the geometry freeze's staging, likewise
size_t piston_arena_bytes();  // the wetted piston's device arena
size_t piston_pinned_bytes();  // and its staged part

extern "C" int fl_boundary_create(fl_boundary** out) {
  if (!out) return FL_INVALID_ARGUMENT;
  *out = nullptr;
  const int st = check_device();
  if (st != FL_OK) return st;
  auto* b = new fl_boundary();
  bool ok = cudaGetDevice(&b->device) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&b->e0) == cudaSuccess && cudaEventCreate(&b->e1) == cudaSuccess &&
            cudaMalloc(&b->dev, kRegions.total) == cudaSuccess &&
            cudaMallocHost(&b->pin, kRegions.staged) == cudaSuccess && b->pressure.reserve_caps() &&
            cudaMalloc(&b->ldev, link_arena_bytes()) == cudaSuccess &&
            cudaMallocHost(&b->lpin, link_arena_bytes()) == cudaSuccess &&
            cudaMalloc(&b->fdev, freeze_arena_bytes()) == cudaSuccess &&
            cudaMallocHost(&b->fpin, freeze_arena_bytes()) == cudaSuccess &&
            cudaMalloc(&b->pdev, piston_arena_bytes()) == cudaSuccess &&
            cudaMallocHost(&b->ppin, piston_pinned_bytes()) == cudaSuccess;
  try {
    b->frz_centre.reserve(4096);
    b->frz_needs.reserve(4096);
    b->frz_ordinal.reserve(4096);
    b->frz_cells.reserve(4096);
    b->frz_faces.reserve(6 * 4096);
    b->pst_idx.reserve(2 * (size_t)kMaxFaces);
    b->pst_patches.reserve(kMaxFaces);
    b->pst_flux.reserve(kMaxFaces);
    b->pst_has.reserve(kMaxFaces);
  } catch (...) {
    ok = false;
  }
  if (!ok) {
    cudaGetLastError();
    fl_boundary_destroy(b);
    return FL_RESOURCE_EXHAUSTED;
  }
  *out = b;
  return FL_OK;
}

extern "C" int fl_boundary_destroy(fl_boundary* b) {
  if (!b) return FL_INVALID_ARGUMENT;
  if (b->device >= 0) cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  b->pressure.destroy();
  if (b->ppin) cudaFreeHost(b->ppin);
  if (b->pdev) cudaFree(b->pdev);
  if (b->fpin) cudaFreeHost(b->fpin);
  if (b->fdev) cudaFree(b->fdev);
  if (b->lpin) cudaFreeHost(b->lpin);
  if (b->ldev) cudaFree(b->ldev);
  if (b->pin) cudaFreeHost(b->pin);
  if (b->dev) cudaFree(b->dev);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FL_OK;
}

extern "C" int fl_boundary_deposit(fl_boundary* b, const fl_owned_grid* grid, const fl_boundary_particle* parts,
                                   uint64_t n, const fl_face_tag* tags, const fl_quantization* q,
                                   fl_face_quanta* quanta, fl_compatible_sample* stencils, fl_measurement* m) {
  if (!b || !q) return FL_INVALID_ARGUMENT;
  int st = check_grid(grid);
  if (st != FL_OK) return st;
  const uint64_t faces = 192 * grid->block_count;
  if (faces > (uint64_t)kMaxFaces || n > (uint64_t)kMaxParticles) return FL_RESOURCE_EXHAUSTED;
  st = check_quantization(q, n);
  if (st != FL_OK) return st;
  if ((faces && (!tags || !quanta)) || (n && (!parts || !stencils))) return FL_INVALID_ARGUMENT;
  if (n && !geometry_ok(grid)) return FL_INVALID_ARGUMENT;
  const Regions& R = kRegions;
  const uint64_t cap = std::max<uint64_t>(1, q->declared_capacity);
  int width = 0;
  while (width < 64 && (1ULL << width) < cap) ++width;  // bit_width(cap - 1)
  DepositArgs a;
  a.g = device_grid(b, grid);
  a.parts = dptr<fl_boundary_particle>(b, R.particles);
  a.n = (int)n;
  a.tags = dptr<fl_face_tag>(b, R.tags_a);
  a.mass_q = q->mass_per_quantum;
  a.mom_q = q->momentum_per_quantum;
  a.limit = std::ldexp(1.0, 62 - width);
  a.quanta = dptr<unsigned long long>(b, R.quanta);
  a.stencils = dptr<fl_compatible_sample>(b, R.stencils);
  a.rep = dptr<Report>(b, R.report);
  bool ok = begin(b) && upload(b, R.blocks, grid->blocks, sizeof(int32_t) * 3 * grid->block_count) &&
            upload(b, R.particles, parts, sizeof(fl_boundary_particle) * n) &&
            upload(b, R.tags_a, tags, sizeof(fl_face_tag) * faces) &&
            cudaMemsetAsync(b->dev + R.quanta, 0, sizeof(fl_face_quanta) * faces, b->stream) == cudaSuccess;
  if (ok && n) {
    ++g_kernel_launches;
    k_compatible_deposit<<<grid_of(3 * n, 128), 128, 0, b->stream>>>(a);
  }
  ok = ok && download(b, R.quanta, sizeof(fl_face_quanta) * faces) &&
       download(b, R.stencils, sizeof(fl_compatible_sample) * 81 * n);
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  st = finish(b, m);
  if (st != FL_OK) return st;
  std::memcpy(quanta, hptr<char>(b, R.quanta), sizeof(fl_face_quanta) * faces);
  std::memcpy(stencils, hptr<char>(b, R.stencils), sizeof(fl_compatible_sample) * 81 * n);
  return FL_OK;
}

extern "C" int fl_boundary_normalize(fl_boundary* b, const fl_face_quanta* quanta, uint64_t count,
                                     const fl_quantization* q, double min_mass, double* masses, double* velocities,
                                     uint8_t* validity, fl_measurement* m) {
  if (!b || !q) return FL_INVALID_ARGUMENT;
  if (count > (uint64_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  int st = check_quantization(q, 0);
  if (st != FL_OK) return st;
  if (!std::isfinite(min_mass) || min_mass < 0.0) return FL_INVALID_ARGUMENT;
  if (count && (!quanta || !masses || !velocities || !validity)) return FL_INVALID_ARGUMENT;
  const Regions& R = kRegions;
  bool ok = begin(b) && upload(b, R.quanta, quanta, sizeof(fl_face_quanta) * count);
  if (ok && count) {
    ++g_kernel_launches;
    k_normalize<<<grid_of(count, 256), 256, 0, b->stream>>>(
        dptr<long long>(b, R.quanta), (int)count, q->mass_per_quantum, q->momentum_per_quantum, min_mass,
        dptr<double>(b, R.masses), dptr<double>(b, R.velocities), dptr<uint8_t>(b, R.validity),
        dptr<Report>(b, R.report));
  }
  ok = ok && download(b, R.masses, sizeof(double) * count) && download(b, R.velocities, sizeof(double) * count) &&
       download(b, R.validity, count);
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  st = finish(b, m);
  if (st != FL_OK) return st;
  std::memcpy(masses, hptr<char>(b, R.masses), sizeof(double) * count);
  std::memcpy(velocities, hptr<char>(b, R.velocities), sizeof(double) * count);
  std::memcpy(validity, hptr<char>(b, R.validity), count);
  return FL_OK;
}

extern "C" int fl_boundary_forces(fl_boundary* b, const fl_owned_grid* grid, const double* old_v,
                                  const double acc[3], double dt, double* predicted, fl_measurement* m) {
  if (!b || !acc) return FL_INVALID_ARGUMENT;
  int st = check_grid(grid);
  if (st != FL_OK) return st;
  const uint64_t faces = 192 * grid->block_count;
  if (faces > (uint64_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  if (faces && (!old_v || !predicted)) return FL_INVALID_ARGUMENT;
  const Regions& R = kRegions;
  bool ok = begin(b) && upload(b, R.vel_a, old_v, sizeof(double) * faces);
  if (ok && faces) {
    ++g_kernel_launches;
    k_forces<<<grid_of(faces, 256), 256, 0, b->stream>>>(dptr<double>(b, R.vel_a), (int)faces, acc[0], acc[1],
                                                           acc[2], dt, dptr<double>(b, R.velocities),
                                                           dptr<Report>(b, R.report));
  }
  ok = ok && download(b, R.velocities, sizeof(double) * faces);
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  st = finish(b, m);
  if (st != FL_OK) return st;
  std::memcpy(predicted, hptr<char>(b, R.velocities), sizeof(double) * faces);
  return FL_OK;
}

extern "C" int fl_boundary_predict_face(fl_boundary* b, const fl_owned_grid* grid, const fl_velocity_history* old_h,
                                        uint64_t slot, int64_t side, const double acc[3], double dt,
                                        double* predicted, fl_measurement* m) {
  if (!b || !acc || !predicted || !old_h) return FL_INVALID_ARGUMENT;
  int st = check_grid(grid);
  if (st != FL_OK) return st;
  const uint64_t faces = 192 * grid->block_count;
  if (faces > (uint64_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  if (slot >= faces) return FL_OUT_OF_RANGE;
  st = check_history(old_h, faces, old_h->velocity_sample_time);
  if (st != FL_OK) return st;
  const int axis = (int)((slot % 192) / 64);
  const Regions& R = kRegions;
  bool ok = begin(b) && upload(b, R.blocks, grid->blocks, sizeof(int32_t) * 3 * grid->block_count) &&
            upload_history(b, old_h, faces, false);
  if (ok) {
    ++g_kernel_launches;
    k_predict_face<<<1, 32, 0, b->stream>>>(device_grid(b, grid), device_history(b, false), (long long)slot, side,
                                            acc[axis], dt, dptr<Report>(b, R.report));
  }
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  st = finish(b, m);
  if (st != FL_OK) return st;
  *predicted = hptr<Report>(b, R.report)->predicted;
  return FL_OK;
}

extern "C" int fl_boundary_gather(fl_boundary* b, const fl_owned_grid* grid, const fl_boundary_particle* parts,
                                  uint64_t n, double old_time, double new_time, const fl_velocity_history* old_h,
                                  const fl_velocity_history* new_h, fl_gathered_particle* out, uint64_t counts[3],
                                  fl_measurement* m) {
  if (!b) return FL_INVALID_ARGUMENT;
  int st = check_grid(grid);
  if (st != FL_OK) return st;
  const uint64_t faces = 192 * grid->block_count;
  if (faces > (uint64_t)kMaxFaces || n > (uint64_t)kMaxParticles) return FL_RESOURCE_EXHAUSTED;
  if (!std::isfinite(old_time) || !std::isfinite(new_time) || new_time <= old_time) return FL_INVALID_ARGUMENT;
  st = check_history(old_h, faces, old_time);
  if (st != FL_OK) return st;
  st = check_history(new_h, faces, new_time);
  if (st != FL_OK) return st;
  if (n && (!parts || !out)) return FL_INVALID_ARGUMENT;
  if (n && !geometry_ok(grid)) return FL_INVALID_ARGUMENT;
  const Regions& R = kRegions;
  GatherArgs a;
  a.g = device_grid(b, grid);
  a.parts = dptr<fl_boundary_particle>(b, R.particles);
  a.n = (int)n;
  a.old_h = device_history(b, false);
  a.new_h = device_history(b, true);
  a.rec = dptr<FillRecord>(b, R.records);
  a.out = dptr<fl_gathered_particle>(b, R.gathered);
  a.rep = dptr<Report>(b, R.report);
  bool ok = begin(b) && upload(b, R.blocks, grid->blocks, sizeof(int32_t) * 3 * grid->block_count) &&
            upload(b, R.particles, parts, sizeof(fl_boundary_particle) * n) &&
            upload_history(b, old_h, faces, false) && upload_history(b, new_h, faces, true);
  if (ok && n) {
    g_kernel_launches += 3;
    k_gather_stencils<<<grid_of(3 * n, 128), 128, 0, b->stream>>>(a);
    k_gather_fill<<<grid_of(81 * n, 128), 128, 0, b->stream>>>(a);
    k_gather_finish<<<grid_of(n, 128), 128, 0, b->stream>>>(a);
  }
  ok = ok && download(b, R.gathered, sizeof(fl_gathered_particle) * n);
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  st = finish(b, m);
  if (st != FL_OK) return st;
  const fl_gathered_particle* g = hptr<fl_gathered_particle>(b, R.gathered);
  uint64_t c[3] = {0, 0, 0};
  for (uint64_t p = 0; p < n; ++p) {
    out[p] = g[p];
    c[0] += g[p].old_pic_fallback;
    c[1] += g[p].new_pic_fallback;
    c[2] += g[p].low_mass_fallback;
  }
  if (counts)
    for (int k = 0; k < 3; ++k) counts[k] = c[k];
  return FL_OK;
}

extern "C" int fl_boundary_project(fl_boundary* b, double h, double dt, const int32_t* cell_index,
                                   const double* cell_values, uint64_t cell_count, const int32_t* face_index,
                                   const int32_t* face_kind, const double* face_values, uint64_t face_count,
                                   int max_iterations, double rel_tol, double* pressure, double* corrected_u,
                                   double* rhs, double* residual, double* defect, uint64_t* gauge_ordinals,
                                   fl_mac_pressure_diagnostics* diagnostics, fl_measurement* measurement) {
  if (!b) return FL_INVALID_ARGUMENT;
  if (cudaSetDevice(b->device) != cudaSuccess) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  return fl::mp_project(b->pressure, b->stream, h, dt, cell_index, cell_values, cell_count, face_index, face_kind,
                        face_values, face_count, max_iterations, rel_tol, pressure, corrected_u, rhs, residual,
                        defect, gauge_ordinals, diagnostics, measurement);
}

// ---- pressure-link assembly: host checks and launch ----

namespace {

constexpr int kMaxLinkCells = 4096;
constexpr size_t kMaxCenters = 27 * (size_t)kMaxLinkCells;

bool host_cell_less(const int32_t* a, const int32_t* b) {
  return a[2] != b[2] ? a[2] < b[2] : (a[1] != b[1] ? a[1] < b[1] : a[0] < b[0]);
}

template <typename R>
long long host_find_cell(const R* recs, uint64_t n, const int32_t* key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) / 2;
    if (host_cell_less(recs[mid].cell_index, key))
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < n && !host_cell_less(key, recs[lo].cell_index)) return (long long)lo;
  return -1;
}

// SparseMacGridView3D::FaceSlot (sparse_mac_grid_3d.cc:388-409): the owned slot
// of face (axis, lattice) or the reference's status.
int host_face_slot(const fl_owned_grid* g, int axis, const int64_t lat[3], uint64_t* slot) {
  if (axis < 0 || axis > 2) return FL_INVALID_ARGUMENT;
  auto fdiv = [](int64_t i) { return i >= 0 ? i / 4 : -1 - (-(i + 1)) / 4; };
  const int64_t b[3] = {fdiv(lat[0]), fdiv(lat[1]), fdiv(lat[2])};
  uint64_t lo = 0, hi = g->block_count;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) / 2;
    const int32_t* m = g->blocks + 3 * mid;
    const bool less = m[2] != b[2] ? m[2] < b[2] : (m[1] != b[1] ? m[1] < b[1] : m[0] < b[0]);
    if (less)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo >= g->block_count) return FL_FAILED_PRECONDITION;
  const int32_t* m = g->blocks + 3 * lo;
  if (m[0] != b[0] || m[1] != b[1] || m[2] != b[2]) return FL_FAILED_PRECONDITION;
  const int64_t local = ((lat[2] - 4 * b[2]) * 4 + (lat[1] - 4 * b[1])) * 4 + (lat[0] - 4 * b[0]);
  *slot = lo * 192 + (uint64_t)axis * 64 + (uint64_t)local;
  return FL_OK;
}

bool positive_finite_h(double v) { return std::isfinite(v) && v > 0.0; }

// ValidateFrozenView (liquid_boundary_geometry_3d.cc:1289-1380) and the field
// checks at the head of LinksCore (:1084-1135), in their order.
// The capacity check of the bounded workspace comes first
// (LiquidBoundaryWorkspace3D::BuildLinksWithBackend, :2151-2159).
int check_links(const fl_frozen_geometry* G, const fl_pressure_fields* F) {
  if (G->cell_count > (uint64_t)kMaxLinkCells || G->face_count > (uint64_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  if (!positive_finite_h(G->step_duration) || !positive_finite_h(G->liquid_density) ||
      !std::isfinite(G->surface_tension) || G->surface_tension < 0)
    return FL_INVALID_ARGUMENT;
  const double h = G->grid->h, area = h * h, volume = area * h, inv = 1 / G->liquid_density;
  if (!std::isnormal(area) || !std::isnormal(volume) || !std::isnormal(inv)) return FL_OUT_OF_RANGE;
  for (uint64_t i = 0; i < G->center_count; ++i)
    if (!std::isfinite(G->centers[i].signed_distance) ||
        (i > 0 && !host_cell_less(G->centers[i - 1].cell_index, G->centers[i].cell_index)))
      return FL_INVALID_ARGUMENT;
  for (uint64_t i = 0; i < G->cell_count; ++i) {
    const fl_frozen_cell& c = G->cells[i];
    if (!positive_finite_h(c.fluid_volume) || c.fluid_volume > volume || !std::isfinite(c.center_distance) ||
        c.center_distance >= 0 || !std::isfinite(c.curvature))
      return FL_INVALID_ARGUMENT;
    if (i > 0 && !host_cell_less(G->cells[i - 1].cell_index, c.cell_index)) return FL_INVALID_ARGUMENT;
  }
  for (uint64_t i = 0; i < G->face_count; ++i) {
    const fl_frozen_face& f = G->faces[i];
    const int64_t lat[3] = {f.lattice[0], f.lattice[1], f.lattice[2]};
    uint64_t slot = 0;
    const int st = host_face_slot(G->grid, f.axis, lat, &slot);
    if (st != FL_OK) return st;
    if (slot != f.face_slot || (i > 0 && f.face_slot <= G->faces[i - 1].face_slot)) return FL_INVALID_ARGUMENT;
    if (!std::isfinite(f.open_area) || f.open_area < 0 || f.open_area > area || f.blocked_area != area - f.open_area ||
        !std::isfinite(f.wall_normal_velocity))
      return FL_INVALID_ARGUMENT;
    if (f.has_prescribed_wall_flux &&
        (!std::isfinite(f.prescribed_wall_flux) || (f.blocked_area == 0 && f.prescribed_wall_flux != 0)))
      return FL_INVALID_ARGUMENT;
    const int32_t head[3] = {f.lattice[0], f.lattice[1], f.lattice[2]};
    const bool tail_ok = head[f.axis] != INT32_MIN;
    int32_t tail[3] = {head[0], head[1], head[2]};
    if (tail_ok) tail[f.axis] -= 1;
    const bool has_head = host_find_cell(G->cells, G->cell_count, head) >= 0;
    const bool has_tail = tail_ok && host_find_cell(G->cells, G->cell_count, tail) >= 0;
    if (!has_head && !has_tail) return FL_FAILED_PRECONDITION;
    if (!tail_ok && f.open_area > 0) return FL_OUT_OF_RANGE;
  }
  // every incident owner present in the face union
  for (uint64_t i = 0; i < G->cell_count; ++i)
    for (int a = 0; a < 3; ++a)
      for (int side = 0; side < 2; ++side) {
        int64_t lat[3] = {G->cells[i].cell_index[0], G->cells[i].cell_index[1], G->cells[i].cell_index[2]};
        lat[a] += side;
        if (lat[a] > INT32_MAX) return FL_OUT_OF_RANGE;
        uint64_t slot = 0;
        const int st = host_face_slot(G->grid, a, lat, &slot);
        if (st != FL_OK) return st;
        uint64_t lo = 0, hi = G->face_count;
        while (lo < hi) {
          const uint64_t mid = (lo + hi) / 2;
          if (G->faces[mid].face_slot < slot)
            lo = mid + 1;
          else
            hi = mid;
        }
        if (lo >= G->face_count || G->faces[lo].face_slot != slot) return FL_FAILED_PRECONDITION;
      }
  if (F->air_count > G->center_count || F->interface_count > G->face_count || !std::isfinite(F->ambient_pressure))
    return FL_INVALID_ARGUMENT;
  for (uint64_t k = 0; k < F->interface_count; ++k) {
    const fl_internal_interface& c = F->interfaces[k];
    if (c.face_ordinal >= G->face_count || (k > 0 && F->interfaces[k - 1].face_ordinal >= c.face_ordinal) ||
        !std::isfinite(c.tail_fraction) || c.tail_fraction < 0.0 || c.tail_fraction > 1.0 ||
        !std::isfinite(c.surface_tension) || c.surface_tension < 0.0 || !std::isfinite(c.curvature_tail_to_head) ||
        !std::isfinite(c.normal_viscous_jump_tail_to_head))
      return FL_INVALID_ARGUMENT;
  }
  for (uint64_t k = 0; k < F->air_count; ++k) {
    const fl_air_cell_pressure& p = F->air[k];
    if (!std::isfinite(p.gas_gauge_pressure) ||
        (k > 0 && !host_cell_less(F->air[k - 1].cell_index, p.cell_index)))
      return FL_INVALID_ARGUMENT;
    const long long c = host_find_cell(G->centers, G->center_count, p.cell_index);
    if (c < 0) return FL_FAILED_PRECONDITION;
    if (G->centers[c].signed_distance < 0.0 || host_find_cell(G->cells, G->cell_count, p.cell_index) >= 0)
      return FL_INVALID_ARGUMENT;
  }
  for (uint64_t i = 0; i < G->cell_count; ++i) {
    const fl_pressure_cell_fields& f = F->cells[i];
    if (!std::isfinite(f.target_divergence) || !std::isfinite(f.previous_pressure) || std::isnan(f.bulk_modulus) ||
        f.bulk_modulus <= 0 || (f.has_density && !positive_finite_h(f.density)))
      return FL_INVALID_ARGUMENT;
  }
  return FL_OK;
}

}  // namespace

namespace {

struct LinkRegions {
  size_t cells, faces, fields, pred, wet, has_wet, air, itf, cent, out, reg, report, total;
  LinkRegions() {
    size_t o = 0;
    auto take = [&](size_t bytes) {
      const size_t r = o;
      o = align_up(o + bytes);
      return r;
    };
    cells = take(sizeof(fl_frozen_cell) * kMaxLinkCells);
    faces = take(sizeof(fl_frozen_face) * kMaxFaces);
    fields = take(sizeof(fl_pressure_cell_fields) * kMaxLinkCells);
    pred = take(sizeof(double) * kMaxFaces);
    wet = take(sizeof(double) * kMaxFaces);
    has_wet = take(kMaxFaces);
    air = take(sizeof(fl_air_cell_pressure) * kMaxCenters);
    itf = take(sizeof(fl_internal_interface) * kMaxFaces);
    cent = take(sizeof(fl_center_sample) * kMaxCenters);
    out = take(sizeof(fl_pressure_link) * kMaxFaces);
    reg = take(kMaxFaces);
    report = take(sizeof(Report));
    total = o;
  }
};

const LinkRegions kLinkRegions;

size_t link_arena_bytes() { return kLinkRegions.total; }

bool lupload(fl_boundary* b, size_t off, const void* src, size_t bytes) {
  if (bytes == 0) return true;
  std::memcpy(b->lpin + off, src, bytes);
  return cudaMemcpyAsync(b->ldev + off, b->lpin + off, bytes, cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
}

bool ldownload(fl_boundary* b, size_t off, size_t bytes) {
  if (bytes == 0) return true;
  return cudaMemcpyAsync(b->lpin + off, b->ldev + off, bytes, cudaMemcpyDeviceToHost, b->stream) == cudaSuccess;
}

}  // namespace

extern "C" int fl_boundary_links(fl_boundary* b, const fl_frozen_geometry* G, const fl_pressure_fields* F,
                                 fl_pressure_cell* cells_out, fl_pressure_link* faces_out, uint64_t* lower_theta,
                                 fl_measurement* m) {
  if (!b || !G || !F) return FL_INVALID_ARGUMENT;
  int st = check_grid(G->grid);
  if (st != FL_OK) return st;
  if ((G->center_count && !G->centers) || (G->cell_count && (!G->cells || !F->cells || !cells_out)) ||
      (G->face_count && (!G->faces || !F->predicted_face_velocities || !faces_out)) || (F->air_count && !F->air) ||
      (F->interface_count && !F->interfaces) || (F->wetted_piston_face_fluxes && !F->has_wetted_piston_face_flux))
    return FL_INVALID_ARGUMENT;
  if (G->center_count > kMaxCenters) return FL_RESOURCE_EXHAUSTED;
  st = check_links(G, F);
  if (st != FL_OK) return st;
  const LinkRegions& R = kLinkRegions;
  const uint64_t nf = G->face_count, nc = G->cell_count;
  const Report clean{kNoError, 0, 0, 0.0};
  bool ok = cudaSetDevice(b->device) == cudaSuccess && lupload(b, R.report, &clean, sizeof(clean)) &&
            cudaEventRecord(b->e0, b->stream) == cudaSuccess &&
            lupload(b, R.cells, G->cells, sizeof(fl_frozen_cell) * nc) &&
            lupload(b, R.faces, G->faces, sizeof(fl_frozen_face) * nf) &&
            lupload(b, R.fields, F->cells, sizeof(fl_pressure_cell_fields) * nc) &&
            lupload(b, R.pred, F->predicted_face_velocities, sizeof(double) * nf) &&
            (!F->wetted_piston_face_fluxes || (lupload(b, R.wet, F->wetted_piston_face_fluxes, sizeof(double) * nf) &&
                                               lupload(b, R.has_wet, F->has_wetted_piston_face_flux, nf))) &&
            lupload(b, R.air, F->air, sizeof(fl_air_cell_pressure) * F->air_count) &&
            lupload(b, R.itf, F->interfaces, sizeof(fl_internal_interface) * F->interface_count) &&
            lupload(b, R.cent, G->centers, sizeof(fl_center_sample) * G->center_count);
  if (ok && nf) {
    LinksArgs a;
    a.h = G->grid->h;
    a.density = G->liquid_density;
    a.step_duration = G->step_duration;
    a.sigma = G->surface_tension;
    a.ambient = F->ambient_pressure;
    a.cells = reinterpret_cast<const fl_frozen_cell*>(b->ldev + R.cells);
    a.nc = (int)nc;
    a.faces = reinterpret_cast<const fl_frozen_face*>(b->ldev + R.faces);
    a.nf = (int)nf;
    a.fields = reinterpret_cast<const fl_pressure_cell_fields*>(b->ldev + R.fields);
    a.predicted = reinterpret_cast<const double*>(b->ldev + R.pred);
    a.wetted = F->wetted_piston_face_fluxes ? reinterpret_cast<const double*>(b->ldev + R.wet) : nullptr;
    a.has_wetted = reinterpret_cast<const uint8_t*>(b->ldev + R.has_wet);
    a.air = reinterpret_cast<const fl_air_cell_pressure*>(b->ldev + R.air);
    a.nair = (int)F->air_count;
    a.interfaces = reinterpret_cast<const fl_internal_interface*>(b->ldev + R.itf);
    a.ninterfaces = (int)F->interface_count;
    a.centers = reinterpret_cast<const fl_center_sample*>(b->ldev + R.cent);
    a.ncenters = (int)G->center_count;
    a.out = reinterpret_cast<fl_pressure_link*>(b->ldev + R.out);
    a.regularized = reinterpret_cast<uint8_t*>(b->ldev + R.reg);
    a.rep = reinterpret_cast<Report*>(b->ldev + R.report);
    ++g_kernel_launches;
    k_links<<<grid_of(nf, 128), 128, 0, b->stream>>>(a);
  }
  ok = ok && cudaGetLastError() == cudaSuccess && cudaEventRecord(b->e1, b->stream) == cudaSuccess &&
       ldownload(b, R.out, sizeof(fl_pressure_link) * nf) && ldownload(b, R.reg, nf) &&
       ldownload(b, R.report, sizeof(Report)) && cudaStreamSynchronize(b->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return FL_INTERNAL;
  }
  const Report* r = reinterpret_cast<const Report*>(b->lpin + R.report);
  if (m) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    m->compiled_architecture = r->arch;
    m->kernel_ms = ms;
  }
  if (nf && r->key != kNoError) return (int)(r->key & 0xff);
  for (uint64_t i = 0; i < nc; ++i) {
    fl_pressure_cell& c = cells_out[i];
    std::memset(&c, 0, sizeof(c));
    for (int d = 0; d < 3; ++d) c.cell_index[d] = G->cells[i].cell_index[d];
    c.fluid_volume = G->cells[i].fluid_volume;
    c.target_divergence = F->cells[i].target_divergence;
    c.bulk_modulus = F->cells[i].bulk_modulus;
    c.previous_pressure = F->cells[i].previous_pressure;
    c.integrated_inward_wall_flux = 0.0;
  }
  std::memcpy(faces_out, b->lpin + R.out, sizeof(fl_pressure_link) * nf);
  uint64_t count = 0;
  const uint8_t* reg = reinterpret_cast<const uint8_t*>(b->lpin + R.reg);
  for (uint64_t f = 0; f < nf; ++f) count += reg[f];
  if (lower_theta) *lower_theta = count;
  return FL_OK;
}

// ---- geometry freeze (.freeze) ----
//
// The geometry queries of base/liquid_boundary_geometry_math_3d.h restated for
// the obstacle kinds offered here (none, halfspace, slab): cell volumes
// (:739-780), face areas (:782-847), curvature (:686-725) and the capillary
// bound (:667-675). Positions are in cell widths; a clipping vertex carries
// the liquid distance interpolated along the clipped edges. The host stages
// the sample lookups in the reference's order (liquid_boundary_geometry_3d.cc:
// 765-1075), one thread computes one query, and each query keeps its own
// status so the host can report the first failure in ordinal order.
namespace fl {
namespace {

// Clipping-list capacities. With at most two planes after the liquid plane
// (halfspace, slab) a tetrahedron face stays within 5 vertices and a cap
// within 2 per cut edge; with the five planes of an open tank a face takes up
// to 9 vertices and the polyhedron up to 10 faces.
constexpr int kPolyCap = 10, kPolyhCap = 7;
constexpr int kTankPolyCap = 20, kTankPolyhCap = 10;
constexpr double kNaN = __builtin_nan("");
constexpr double kInf = __builtin_inf();

struct ClipVertex {
  double p[3];  // position in cell widths
  double d;     // interpolated liquid distance (m)
};

template <int N>
struct VertexList {
  static constexpr int kCap = N;
  ClipVertex v[N];
  int n = 0;
  bool overflow = false;
  __device__ void push(const ClipVertex& x) {
    if (n == N) {
      overflow = true;
      return;
    }
    v[n++] = x;
  }
};
using Polygon = VertexList<kPolyCap>;

template <int V, int F>
struct PolyhedronT {
  static constexpr int kVerts = V, kFaces = F;
  VertexList<V> f[F];
  int n = 0;
  bool overflow = false;
};
using Polyhedron = PolyhedronT<kPolyCap, kPolyhCap>;
using TankPolyhedron = PolyhedronT<kTankPolyCap, kTankPolyhCap>;

// A plane's clip distance: the liquid distance itself, or n . p - c. An
// axis-aligned plane (snap >= 0) pins its cut points' coordinate on that axis
// to the plane's own.
struct ClipPlane {
  double n[3];
  double c;
  bool liquid;
  int snap = -1;
};

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// Euclidean norm by scaling with the largest magnitude (the overflow-safe
// textbook form, as the host's three-argument hypot evaluates it).
__device__ __forceinline__ double norm3(double x, double y, double z) {
  x = fabs(x);
  y = fabs(y);
  z = fabs(z);
  const double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
  if (a == 0.0) return 0.0;
  const double sx = x / a, sy = y / a, sz = z / a;
  return a * sqrt(sx * sx + sy * sy + sz * sz);
}

__device__ __forceinline__ double clip_distance(const ClipVertex& v, const ClipPlane& pl) {
  return pl.liquid ? v.d : dot3(pl.n, v.p) - pl.c;
}

// Keeps the part with distance <= 0; each crossing gets an intersection whose
// weights are formed from the distances scaled by their larger magnitude.
template <int NO, int NI, int NC = 1>
__device__ void clip_polygon(const VertexList<NI>& in, const ClipPlane& pl, VertexList<NO>& out,
                             VertexList<NC>* cuts = nullptr) {
  out.n = 0;
  out.overflow = false;
  if (in.overflow) {
    out.overflow = true;
    return;
  }
  if (in.n == 0) return;
  ClipVertex prev = in.v[in.n - 1];
  double dprev = clip_distance(prev, pl);
  for (int k = 0; k < in.n; ++k) {
    const ClipVertex cur = in.v[k];
    const double dcur = clip_distance(cur, pl);
    if ((dprev <= 0.0) != (dcur <= 0.0)) {
      const double mag = fabs(dprev) < fabs(dcur) ? fabs(dcur) : fabs(dprev);
      const double sp = dprev / mag, sc = dcur / mag;
      const double diff = sp - sc;
      const double wp = -sc / diff, wc = sp / diff;
      ClipVertex x;
      for (int a = 0; a < 3; ++a) x.p[a] = prev.p[a] * wp + cur.p[a] * wc;
      x.d = wp * prev.d + wc * cur.d;
      if (pl.snap >= 0) x.p[pl.snap] = pl.c * pl.n[pl.snap];
      out.push(x);
      if (cuts) cuts->push(x);
    }
    if (dcur <= 0.0) out.push(cur);
    prev = cur;
    dprev = dcur;
  }
}

// Scales a direction by a power of two so its largest component is in
// [1/2, 1), then to unit length.
__device__ void unit_direction(const double* d, double* o) {
  const double big = fmax(fmax(fabs(d[0]), fabs(d[1])), fabs(d[2]));
  if (big == 0.0) {
    o[0] = o[1] = o[2] = 0.0;
    return;
  }
  int e = 0;
  (void)frexp(big, &e);
  double s[3];
  for (int a = 0; a < 3; ++a) s[a] = ldexp(d[a], -e);
  const double inv = 1 / norm3(s[0], s[1], s[2]);
  for (int a = 0; a < 3; ++a) o[a] = s[a] * inv;
}

__device__ bool same_position(const ClipVertex& a, const ClipVertex& b) {
  return a.p[0] == b.p[0] && a.p[1] == b.p[1] && a.p[2] == b.p[2];
}

// A tetrahedron as four triangles (the first polyhedron of a cell query).
struct Tetrahedron {
  VertexList<3> f[4];
  int n = 4;
  bool overflow = false;
};

// Clips every face of a convex polyhedron and closes it with the cap through
// the distinct cut points, ordered by angle about their centroid.
template <typename In, typename Out>
__device__ void clip_polyhedron(const In& in, const ClipPlane& pl, Out& out) {
  using Face = VertexList<Out::kVerts>;
  out.n = 0;
  out.overflow = false;
  if (in.overflow) {
    out.overflow = true;
    return;
  }
  VertexList<2 * Out::kFaces> cuts;
  for (int k = 0; k < in.n; ++k) {
    Face clipped;
    clip_polygon(in.f[k], pl, clipped, &cuts);
    if (clipped.overflow || cuts.overflow) {
      out.overflow = true;
      return;
    }
    if (clipped.n >= 3) {
      if (out.n == Out::kFaces) {
        out.overflow = true;
        return;
      }
      out.f[out.n++] = clipped;
    }
  }
  Face cap;
  for (int k = 0; k < cuts.n; ++k) {
    bool seen = false;
    for (int j = 0; j < cap.n; ++j) seen = seen || same_position(cap.v[j], cuts.v[k]);
    if (!seen) cap.push(cuts.v[k]);
  }
  if (cap.overflow) {
    out.overflow = true;
    return;
  }
  if (cap.n < 3) return;
  double center[3] = {0.0, 0.0, 0.0};
  const double w = 1.0 / cap.n;
  for (int k = 0; k < cap.n; ++k)
    for (int a = 0; a < 3; ++a) center[a] = center[a] + cap.v[k].p[a] * w;
  double t[3], nrm[3] = {0.0, 0.0, 0.0}, d[3];
  for (int a = 0; a < 3; ++a) d[a] = cap.v[0].p[a] - center[a];
  unit_direction(d, t);
  for (int k = 1; k < cap.n; ++k) {
    double u[3], c[3];
    for (int a = 0; a < 3; ++a) d[a] = cap.v[k].p[a] - center[a];
    unit_direction(d, u);
    cross3(t, u, c);
    unit_direction(c, nrm);
    if (norm3(nrm[0], nrm[1], nrm[2]) > 0.0) break;
  }
  double bt[3];
  cross3(nrm, t, bt);
  const double tl = norm3(t[0], t[1], t[2]), bl = norm3(bt[0], bt[1], bt[2]);
  if (!(tl > 0.0 && bl > 0.0)) return;
  double ut[3], ub[3];
  const double it = 1 / tl, ib = 1 / bl;
  for (int a = 0; a < 3; ++a) {
    ut[a] = t[a] * it;
    ub[a] = bt[a] * ib;
  }
  auto angle = [&](const ClipVertex& v) {
    double e[3];
    for (int a = 0; a < 3; ++a) e[a] = v.p[a] - center[a];
    return atan2(dot3(e, ub), dot3(e, ut));
  };
  for (int k = 1; k < cap.n; ++k) {  // insertion sort, stable
    const ClipVertex v = cap.v[k];
    int j = k;
    while (j > 0 && angle(v) < angle(cap.v[j - 1])) {
      cap.v[j] = cap.v[j - 1];
      --j;
    }
    cap.v[j] = v;
  }
  if (out.n == Out::kFaces) {
    out.overflow = true;
    return;
  }
  out.f[out.n++] = cap;
}

// Each coordinate row of a small set of vectors scaled by a power of two so
// its largest entry is in [1/2, 1); returns the exponent taken out.
template <int N>
__device__ int normalize_row(double (*e)[3], int axis) {
  double big = 0.0;
  for (int k = 0; k < N; ++k) big = fmax(big, fabs(e[k][axis]));
  if (big == 0.0) return 0;
  int x = 0;
  (void)frexp(big, &x);
  for (int k = 0; k < N; ++k) e[k][axis] = ldexp(e[k][axis], -x);
  return x;
}

// A scaled determinant times h^dim, with the exponents combined before the
// rounding; NaN when a nonzero measure is not representable.
__device__ double physical_measure(double det, int exp, double h, int dim) {
  if (det == 0.0) return 0.0;
  int he = 0;
  const double hm = frexp(h, &he);
  double m = det;
  for (int a = 0; a < dim; ++a) m *= hm;
  const double r = ldexp(m, exp + dim * he);
  if (!isfinite(r) || r == 0.0) return kNaN;
  return r;
}

// Volume as tetrahedra from the mean of all polygon vertices.
template <typename Ph>
__device__ double clipped_volume(const Ph& ph, double h) {
  if (ph.overflow) return kNaN;
  double apex[3] = {0.0, 0.0, 0.0};
  int count = 0;
  for (int k = 0; k < ph.n; ++k) {
    if (ph.f[k].overflow) return kNaN;
    for (int j = 0; j < ph.f[k].n; ++j) {
      for (int a = 0; a < 3; ++a) apex[a] = apex[a] + ph.f[k].v[j].p[a];
      ++count;
    }
  }
  if (count == 0) return 0.0;
  const double inv = 1.0 / count;
  for (int a = 0; a < 3; ++a) apex[a] = apex[a] * inv;
  double vol = 0.0;
  for (int k = 0; k < ph.n; ++k) {
    const auto& pg = ph.f[k];
    for (int j = 1; j + 1 < pg.n; ++j) {
      double e[3][3];
      for (int a = 0; a < 3; ++a) {
        e[0][a] = pg.v[0].p[a] - apex[a];
        e[1][a] = pg.v[j].p[a] - apex[a];
        e[2][a] = pg.v[j + 1].p[a] - apex[a];
      }
      int x = 0;
      for (int a = 0; a < 3; ++a) x += normalize_row<3>(e, a);
      double c[3];
      cross3(e[1], e[2], c);
      vol += physical_measure(fabs(dot3(e[0], c)) / 6, x, h, 3);
    }
  }
  return vol;
}

// Area of a planar polygon's triangle fan, each component of a triangle's
// area vector with its own two coordinate rows scaled.
template <int N>
__device__ double clipped_area(const VertexList<N>& pg, double h) {
  if (pg.overflow) return kNaN;
  double area = 0.0;
  for (int j = 1; j + 1 < pg.n; ++j) {
    double e[2][3];
    for (int a = 0; a < 3; ++a) {
      e[0][a] = pg.v[j].p[a] - pg.v[0].p[a];
      e[1][a] = pg.v[j + 1].p[a] - pg.v[0].p[a];
    }
    double w[3];
    for (int a = 0; a < 3; ++a) {
      double s[2][3] = {{e[0][0], e[0][1], e[0][2]}, {e[1][0], e[1][1], e[1][2]}};
      const int f = (a + 1) % 3, g = (a + 2) % 3;
      const int x = normalize_row<2>(s, f) + normalize_row<2>(s, g);
      w[a] = physical_measure((s[0][f] * s[1][g] - s[0][g] * s[1][f]) / 2, x, h, 2);
    }
    area += norm3(w[0], w[1], w[2]);
  }
  return area;
}

// A polygon lying wholly on the kept side's boundary or beyond is closed.
template <int N>
__device__ double open_face_area(const VertexList<N>& pg, const ClipPlane& pl, double h) {
  if (pg.overflow) return kNaN;
  bool any = false;
  for (int k = 0; k < pg.n; ++k) any = any || clip_distance(pg.v[k], pl) < 0.0;
  if (!any) return 0.0;
  Polygon c;
  clip_polygon(pg, pl, c);
  return clipped_area(c, h);
}

struct FreezeObstacle {
  int kind;  // FL_OBSTACLE_*
  double n[3];
  double coordinate, half_width;
  double tank[6];  // open tank: start low x, high x, floor y, low z, high z, piston velocity x
};

// ---- open tank (base/liquid_boundary_math.h:94-296 for the certified plane
// offsets, base/liquid_boundary_geometry_math_3d.h:440-624 for the clipping) ----

struct SumResidual {
  double value, residual;
};

// FastTwoSum with the larger magnitude first.
__host__ __device__ SumResidual add_with_residual(double a, double b) {
  if (fabs(a) < fabs(b)) {
    const double t = a;
    a = b;
    b = t;
  }
  const double s = a + b;
  if (!isfinite(s)) return {s, 0.0};
  return {s, b - (s - a)};
}

__host__ __device__ double add_down(double a, double b) {
  const SumResidual s = add_with_residual(a, b);
  return s.residual < 0 ? nextafter(s.value, -kInf) : s.value;
}

__host__ __device__ double add_up(double a, double b) {
  const SumResidual s = add_with_residual(a, b);
  return s.residual > 0 ? nextafter(s.value, kInf) : s.value;
}

// Midpoint without overflow, correctly rounded (the P0811 formulation).
__host__ __device__ double midpoint(double a, double b) {
  const double lo = DBL_MIN * 2, hi = DBL_MAX / 2;
  const double aa = a < 0 ? -a : a, ab = b < 0 ? -b : b;
  if (aa <= hi && ab <= hi) return (a + b) / 2;
  if (aa < lo) return a + b / 2;
  if (ab < lo) return a / 2 + b;
  return a / 2 + b / 2;
}

struct OffsetBounds {
  double estimate, lower, upper;
};

// A rounded sum with outward-rounded bounds on its accumulated residuals, so
// the sign of a tank plane's offset from a lattice plane can be certified.
struct CertifiedSum {
  double sum = 0.0, lower = 0.0, upper = 0.0;
  __host__ __device__ void correct(double c) {
    if (!isfinite(lower) || !isfinite(upper)) {
      sum = kInf;
      return;
    }
    lower = add_down(lower, c);
    upper = add_up(upper, c);
  }
  __host__ __device__ void add(double term) {
    if (!isfinite(sum) || !isfinite(term)) {
      sum = kInf;
      return;
    }
    const SumResidual s = add_with_residual(sum, term);
    sum = s.value;
    correct(s.residual);
  }
  __host__ __device__ void add_product(double l, double r) {
    const double product = l * r;
    add(product);
    if (isfinite(product) && l != 0 && r != 0 && fabs(l) != 1 && fabs(r) != 1) {
      correct(fma(l, r, -product));
      if (fabs(product) <= 0x1p-969) {
        const double tiny = 4.9406564584124654e-324;  // the smallest subnormal
        lower = add_down(lower, -tiny);
        upper = add_up(upper, tiny);
      }
    }
  }
  __host__ __device__ OffsetBounds bounds() const {
    if (!isfinite(sum) || !isfinite(lower) || !isfinite(upper)) return {kInf, kInf, kInf};
    return {sum + midpoint(lower, upper), add_down(sum, lower), add_up(sum, upper)};
  }
};

constexpr int kSignUnresolved = 2;

__host__ __device__ int certified_sign(const OffsetBounds& b) {
  if (!isfinite(b.estimate) || !isfinite(b.lower) || !isfinite(b.upper)) return kSignUnresolved;
  if (b.lower > 0) return 1;
  if (b.upper < 0) return -1;
  if (b.lower == 0 && b.upper == 0) return 0;
  return kSignUnresolved;
}

// world - (origin + h * index), exactly enough to certify its sign.
__host__ __device__ CertifiedSum tank_plane_offset(double world, double origin, double index, double h) {
  CertifiedSum o;
  o.add(world);
  o.add(-origin);
  o.add_product(-h, index);
  return o;
}

__host__ __device__ int tank_plane_sign(double world, double origin, double index, double h, int* sign) {
  const double translated = world - origin;
  if (isinf(translated)) {
    *sign = translated > 0 ? 1 : -1;
    return FL_OK;
  }
  *sign = certified_sign(tank_plane_offset(world, origin, index, h).bounds());
  return *sign == kSignUnresolved ? FL_OUT_OF_RANGE : FL_OK;
}

// The plane's coordinate in the cell's unit frame: 0 at or below the low
// face, 1 at or beyond the high face, else the interior cut.
__host__ __device__ int tank_clip_coordinate(double world, double origin, double index, double h, double* out) {
  const double translated = world - origin;
  if (isinf(translated)) {
    *out = translated > 0 ? 1.0 : 0.0;
    return FL_OK;
  }
  CertifiedSum o = tank_plane_offset(world, origin, index, h);
  const OffsetBounds low = o.bounds();
  const int low_side = certified_sign(low);
  if (low_side == kSignUnresolved) return FL_OUT_OF_RANGE;
  if (low_side <= 0) {
    *out = 0.0;
    return FL_OK;
  }
  o.add(-h);
  const int high_side = certified_sign(o.bounds());
  if (high_side == kSignUnresolved) return FL_OUT_OF_RANGE;
  if (high_side >= 0) {
    *out = 1.0;
    return FL_OK;
  }
  const double c = low.estimate / h;
  if (c <= 0 || c >= 1) return FL_OUT_OF_RANGE;
  *out = c;
  return FL_OK;
}

struct TankBounds {
  double low[3] = {0.0, 0.0, 0.0};
  double high[3] = {1.0, 1.0, 1.0};
};

// The tank's clip box in the unit frame of the queried cell or face (a face
// skips its normal axis).
__device__ int local_tank_bounds(const FreezeObstacle& ob, const double origin[3], double h, const int32_t idx[3],
                                 int skip_axis, TankBounds& tb) {
  const double lw[3] = {ob.tank[0], ob.tank[2], ob.tank[3]};
  const double hw[3] = {ob.tank[1], kInf, ob.tank[4]};
  for (int a = 0; a < 3; ++a) {
    if (a == skip_axis) continue;
    double lo = 0.0, hi = 0.0;
    if (tank_clip_coordinate(lw[a], origin[a], (double)idx[a], h, &lo) != FL_OK ||
        tank_clip_coordinate(hw[a], origin[a], (double)idx[a], h, &hi) != FL_OK)
      return FL_OUT_OF_RANGE;
    tb.low[a] = lo;
    tb.high[a] = hi;
    if (lo == hi && lo > 0 && hi < 1) return FL_OUT_OF_RANGE;
  }
  return FL_OK;
}

// Product of the box's extents (one axis excluded for a face), scaled by
// powers of two before the multiply.
__device__ double tank_box_measure(const TankBounds& tb, double h, int excluded) {
  double mantissa = 1.0;
  int exponent = 0, dim = 0;
  for (int a = 0; a < 3; ++a) {
    if (a == excluded) continue;
    const double extent = tb.high[a] - tb.low[a];
    if (extent <= 0) return 0.0;
    int e = 0;
    mantissa *= frexp(extent, &e);
    exponent += e;
    ++dim;
  }
  return physical_measure(mantissa, exponent, h, dim);
}

// Both ends of each cell edge resolvable in world coordinates.
__device__ bool tank_cell_resolved(const double origin[3], double h, const int32_t idx[3]) {
  for (int a = 0; a < 3; ++a) {
    const double low = origin[a] + h * (double)idx[a];
    const double high = origin[a] + h * ((double)idx[a] + 1);
    if (!isfinite(low) || !isfinite(high) || low >= high) return false;
    if (nextafter(low, high) - low > h || high - nextafter(high, low) > h) return false;
  }
  return true;
}

// The obstacle's planes in the query's cell-width frame (anchor: the lattice
// corner of the queried cell or face); present = false without an obstacle.
struct LocalPlanes {
  bool present, slab;
  double n[3];
  double low, high;
};

__device__ int local_planes(const FreezeObstacle& ob, const double origin[3], double h, const int32_t idx[3],
                            LocalPlanes& lp) {
  lp.present = ob.kind == FL_OBSTACLE_HALFSPACE || ob.kind == FL_OBSTACLE_SLAB;
  lp.slab = ob.kind == FL_OBSTACLE_SLAB;
  for (int a = 0; a < 3; ++a) lp.n[a] = ob.n[a];
  const double hw = lp.slab ? ob.half_width : 0.0;
  lp.low = ob.coordinate - hw;
  lp.high = ob.coordinate + hw;
  if (!lp.present) return FL_OK;
  double anchor[3];
  for (int a = 0; a < 3; ++a) anchor[a] = origin[a] + h * (double)idx[a];
  const double proj = dot3(lp.n, anchor);
  lp.low = (lp.low - proj) / h;
  lp.high = (lp.high - proj) / h;
  if (!finite3(anchor) || !isfinite(lp.low) || !isfinite(lp.high) || (lp.slab && lp.low >= lp.high))
    return FL_OUT_OF_RANGE;
  return FL_OK;
}

// The six tetrahedra of the cube around its 0-7 diagonal (corner bit a = offset along axis a).
__constant__ int kCubeTets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

struct CellQuery {
  double corner[8];
  int32_t index[3];
  int32_t pad;
};
struct CellResult {
  double low, high;  // liquid volume on each side of a slab (high: all of it otherwise), m^3
  int32_t status;
  int32_t pad;
};
struct FaceQuery {
  int32_t axis;
  int32_t lattice[3];
};
struct FaceResult {
  double open, blocked;
  double piston_velocity, wall_flux;  // open tank: the piston's share of a closed low-x face
  int32_t status;
  int32_t is_piston;
};
struct CurvatureQuery {
  double d[27];  // centre distances, x fastest, the eight outer corners unused
};
struct CurvatureResult {
  double curvature;
  int32_t status;
  int32_t pad;
};

struct FreezeArgs {
  double origin[3];
  double h;
  FreezeObstacle obstacle;
  const CellQuery* cq;
  CellResult* cr;
  int ncell;
  const FaceQuery* fq;
  FaceResult* fr;
  int nface;
  const CurvatureQuery* kq;
  CurvatureResult* kr;
  int ncurv;
  double density, sigma;
  double* capillary;  // [0] bound, [1] status
  int* arch;
};

// One thread per (cell, tetrahedron), 32 cells per CTA: each thread clips its
// tetrahedron; the cell's first thread sums the six contributions in
// tetrahedron order (a tetrahedron without liquid adds +0, which leaves the
// sum's bits unchanged) and writes the cell's result.
constexpr int kFreezeCellsPerCta = 32;
constexpr int kFreezeCellThreads = 6 * kFreezeCellsPerCta;

__device__ void tet_corners(const CellQuery& q, int t, ClipVertex v[4]) {
  for (int k = 0; k < 4; ++k) {
    const int c = kCubeTets[t][k];
    for (int d = 0; d < 3; ++d) v[k].p[d] = (double)((c >> d) & 1);
    v[k].d = q.corner[c];
  }
}

__device__ void tet_faces(const ClipVertex v[4], Tetrahedron& tet) {
  const int f[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 3; ++j) tet.f[k].push(v[f[k][j]]);
}

__device__ void sum_cell(FreezeArgs& a, int cell, int tet, int status, double lo, double hi) {
  __shared__ double s_lo[kFreezeCellThreads], s_hi[kFreezeCellThreads];
  const int slot = threadIdx.x;
  s_lo[slot] = lo;
  s_hi[slot] = hi;
  __syncthreads();
  if (cell < a.ncell && tet == 0) {
    CellResult r{0.0, 0.0, status, 0};
    if (status == FL_OK)
      for (int k = 0; k < 6; ++k) {
        r.low += s_lo[slot + k];
        r.high += s_hi[slot + k];
      }
    a.cr[cell] = r;
  }
}

__global__ void __launch_bounds__(kFreezeCellThreads) k_freeze_cells(FreezeArgs a) {
  const int cell = blockIdx.x * kFreezeCellsPerCta + threadIdx.x / 6, t = threadIdx.x % 6;
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.arch = compiled_arch();
  double lo = 0.0, hi = 0.0;
  int status = FL_OK;
  if (cell < a.ncell) {
    const CellQuery& q = a.cq[cell];
    LocalPlanes lp;
    status = local_planes(a.obstacle, a.origin, a.h, q.index, lp);
    ClipVertex v[4];
    tet_corners(q, t, v);
    if (status == FL_OK && (v[0].d < 0.0 || v[1].d < 0.0 || v[2].d < 0.0 || v[3].d < 0.0)) {
      Tetrahedron tet;
      tet_faces(v, tet);
      const ClipPlane liquid{{0.0, 0.0, 0.0}, 0.0, true};
      Polyhedron wet;
      clip_polyhedron(tet, liquid, wet);
      if (!lp.present) {
        hi = clipped_volume(wet, a.h);
      } else {
        const ClipPlane above{{-lp.n[0], -lp.n[1], -lp.n[2]}, -lp.high, false};
        Polyhedron side;
        clip_polyhedron(wet, above, side);
        hi = clipped_volume(side, a.h);
        if (lp.slab) {
          const ClipPlane below{{lp.n[0], lp.n[1], lp.n[2]}, lp.low, false};
          clip_polyhedron(wet, below, side);
          lo = clipped_volume(side, a.h);
        }
      }
    }
  }
  sum_cell(a, cell, t, status, lo, hi);
}

// Cell volumes inside an open tank: the liquid part of each tetrahedron
// clipped to the tank's box in the cell's unit frame (low then high plane of
// each axis strictly inside the cell).
__global__ void __launch_bounds__(kFreezeCellThreads) k_freeze_cells_tank(FreezeArgs a) {
  const int cell = blockIdx.x * kFreezeCellsPerCta + threadIdx.x / 6, t = threadIdx.x % 6;
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.arch = compiled_arch();
  double hi = 0.0;
  int status = FL_OK;
  if (cell < a.ncell) {
    const CellQuery& q = a.cq[cell];
    TankBounds tb;
    if (!tank_cell_resolved(a.origin, a.h, q.index) ||
        local_tank_bounds(a.obstacle, a.origin, a.h, q.index, -1, tb) != FL_OK)
      status = FL_OUT_OF_RANGE;
    const double box = status == FL_OK ? tank_box_measure(tb, a.h, -1) : 0.0;
    bool all_liquid = true;
    for (int c = 0; c < 8; ++c) all_liquid = all_liquid && q.corner[c] < 0;
    if (status == FL_OK && !normal_or_zero(box)) status = FL_OUT_OF_RANGE;
    ClipVertex v[4];
    tet_corners(q, t, v);
    if (status == FL_OK && box != 0.0 && all_liquid) {
      hi = t == 0 ? box : 0.0;  // the whole box, once
    } else if (status == FL_OK && box != 0.0 && (v[0].d < 0.0 || v[1].d < 0.0 || v[2].d < 0.0 || v[3].d < 0.0)) {
      Tetrahedron tet;
      tet_faces(v, tet);
      const ClipPlane liquid{{0.0, 0.0, 0.0}, 0.0, true};
      TankPolyhedron buf[2];
      int cur = 0;
      clip_polyhedron(tet, liquid, buf[cur]);
      for (int ax = 0; ax < 3; ++ax) {
        ClipPlane pl{{0.0, 0.0, 0.0}, 0.0, false, ax};
        if (tb.low[ax] > 0) {
          pl.n[ax] = -1;
          pl.c = -tb.low[ax];
          clip_polyhedron(buf[cur], pl, buf[1 - cur]);
          cur = 1 - cur;
        }
        if (tb.high[ax] < 1) {
          pl.n[ax] = 1;
          pl.c = tb.high[ax];
          clip_polyhedron(buf[cur], pl, buf[1 - cur]);
          cur = 1 - cur;
        }
      }
      hi = clipped_volume(buf[cur], a.h);
    }
  }
  sum_cell(a, cell, t, status, 0.0, hi);
}

__global__ void k_freeze_faces(FreezeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nface) return;
  const FaceQuery& q = a.fq[i];
  FaceResult r{0.0, 0.0, 0.0, 0.0, FL_OK, 0};
  const double h = a.h, full = h * h;
  if (q.axis < 0 || q.axis >= 3) {
    r.status = FL_INVALID_ARGUMENT;
    a.fr[i] = r;
    return;
  }
  if (a.obstacle.kind == FL_OBSTACLE_OPEN_TANK) {
    // The tank's walls close a face outside its planes; the piston owns the
    // part of a closed low-x face inside the floor and z bounds.
    TankBounds tb;
    r.status = local_tank_bounds(a.obstacle, a.origin, h, q.lattice, q.axis, tb);
    const double lw[3] = {a.obstacle.tank[0], a.obstacle.tank[2], a.obstacle.tank[3]};
    const double hw[3] = {a.obstacle.tank[1], kInf, a.obstacle.tank[4]};
    int low_sign = 0, high_sign = 0;
    if (r.status == FL_OK &&
        (tank_plane_sign(lw[q.axis], a.origin[q.axis], (double)q.lattice[q.axis], h, &low_sign) != FL_OK ||
         tank_plane_sign(hw[q.axis], a.origin[q.axis], (double)q.lattice[q.axis], h, &high_sign) != FL_OK))
      r.status = FL_OUT_OF_RANGE;
    if (r.status == FL_OK) {
      const bool piston_side = q.axis == 0 && low_sign >= 0;
      const bool open = low_sign < 0 && high_sign > 0;
      if (open || piston_side) {
        const double transverse = tank_box_measure(tb, h, q.axis);
        if (!normal_or_zero(transverse) || transverse > full) {
          r.status = FL_OUT_OF_RANGE;
        } else if (open) {
          r.open = transverse;
          for (int ax = 0; ax < 3; ++ax)
            if (ax != q.axis && transverse == full && (tb.low[ax] > 0 || tb.high[ax] < 1)) r.status = FL_OUT_OF_RANGE;
        } else if (transverse > 0) {
          r.is_piston = 1;
          r.piston_velocity = a.obstacle.tank[5];
          r.wall_flux = transverse * r.piston_velocity;
          if (!normal_or_zero(r.wall_flux) || (r.piston_velocity != 0 && r.wall_flux == 0)) r.status = FL_OUT_OF_RANGE;
        }
      }
      if (r.status == FL_OK) {
        r.blocked = full - r.open;
        if (!normal_or_zero(r.blocked)) r.status = FL_OUT_OF_RANGE;
      }
    }
    a.fr[i] = r;
    return;
  }
  LocalPlanes lp;
  r.status = local_planes(a.obstacle, a.origin, h, q.lattice, lp);
  if (r.status != FL_OK) {
    a.fr[i] = r;
    return;
  }
  const int t0 = q.axis == 0 ? 1 : 0, t1 = q.axis == 2 ? 1 : 2;
  ClipVertex v[4] = {};
  v[1].p[t0] = 1.0;
  v[2].p[t0] = 1.0;
  v[2].p[t1] = 1.0;
  v[3].p[t1] = 1.0;
  const ClipPlane inside{{lp.n[0], lp.n[1], lp.n[2]}, lp.high, false};
  const ClipPlane beyond{{-lp.n[0], -lp.n[1], -lp.n[2]}, -lp.low, false};
  const ClipPlane above{{-lp.n[0], -lp.n[1], -lp.n[2]}, -lp.high, false};
  const ClipPlane below{{lp.n[0], lp.n[1], lp.n[2]}, lp.low, false};
  double geometric_open = 0.0, geometric_blocked = 0.0;
  for (int tri = 0; tri < 2; ++tri) {
    VertexList<3> pg;
    pg.push(v[0]);
    pg.push(v[tri + 1]);
    pg.push(v[tri + 2]);
    if (!lp.present) {
      geometric_open += clipped_area(pg, h);
      continue;
    }
    Polygon blocked;
    clip_polygon(pg, inside, blocked);
    if (lp.slab) {
      Polygon b2;
      clip_polygon(blocked, beyond, b2);
      blocked = b2;
    }
    geometric_blocked += clipped_area(blocked, h);
    geometric_open += open_face_area(pg, above, h);
    if (lp.slab) geometric_open += open_face_area(pg, below, h);
  }
  r.open = full < geometric_open ? full : geometric_open;
  r.blocked = full - r.open;
  if (!isfinite(geometric_open) || !isfinite(geometric_blocked) ||
      geometric_open / full > 1 + 64 * DBL_EPSILON || !(r.open == 0.0 || is_normal(r.open)) ||
      !(r.blocked == 0.0 || is_normal(r.blocked)) || (geometric_blocked > 0 && r.blocked == 0.0))
    r.status = FL_OUT_OF_RANGE;
  a.fr[i] = r;
}

// Outward curvature from centred differences: div(grad d / |grad d|) with the
// Hessian's mixed entries from the four edge neighbours of each plane.
__global__ void k_freeze_curvature(FreezeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.ncurv) return;
  const double* d = a.kq[i].d;
  const double h = a.h;
  const int stride[3] = {1, 3, 9};
  double g[3], H[3][3];
  for (int ax = 0; ax < 3; ++ax) {
    const double lo = d[13 - stride[ax]], hi = d[13 + stride[ax]];
    g[ax] = (hi - lo) / (2 * h);
    H[ax][ax] = ((hi - d[13]) + (lo - d[13])) / h / h;
    for (int o = 0; o < ax; ++o) {
      double mixed = 0.0;
      for (int s = -1; s <= 1; s += 2)
        for (int u = -1; u <= 1; u += 2) mixed += (double)(s * u) * (d[13 + s * stride[ax] + u * stride[o]] / 4);
      H[ax][o] = mixed / h / h;
      H[o][ax] = H[ax][o];
    }
  }
  CurvatureResult r{0.0, FL_OK, 0};
  const double norm = norm3(g[0], g[1], g[2]);
  if (!finite3(g) || !isfinite(norm)) {
    r.status = FL_OUT_OF_RANGE;
  } else if (norm < 1e-8) {
    r.status = FL_FAILED_PRECONDITION;
  } else {
    const double inv = 1 / norm;
    const double nv[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
    double k = 0.0;
    for (int ax = 0; ax < 3 && r.status == FL_OK; ++ax) {
      if (!finite3(H[ax])) {
        r.status = FL_OUT_OF_RANGE;
        break;
      }
      k += (H[ax][ax] - nv[ax] * dot3(H[ax], nv)) / norm;
    }
    if (r.status == FL_OK && !isfinite(k)) r.status = FL_OUT_OF_RANGE;
    r.curvature = k;
  }
  a.kr[i] = r;
}

// sqrt(rho h^3 / (4 pi sigma)): the step below which a capillary wave of the
// cell's size stays resolved.
__global__ void k_freeze_capillary(FreezeArgs a) {
  const double pi = 3.141592653589793238462643383279502884;
  const double h = a.h, volume = h * h * h;
  const double square = a.density * volume / (4 * pi * a.sigma);
  a.capillary[0] = is_normal(square) ? sqrt(square) : 0.0;
  a.capillary[1] = is_normal(square) ? (double)FL_OK : (double)FL_OUT_OF_RANGE;
}

}  // namespace
}  // namespace fl

namespace {

struct FreezeRegions {
  size_t cq, cr, fq, fr, kq, kr, cap, arch, total;
  FreezeRegions() {
    size_t o = 0;
    auto take = [&](size_t bytes) {
      const size_t r = o;
      o = align_up(o + bytes);
      return r;
    };
    cq = take(sizeof(CellQuery) * kMaxLinkCells);
    cr = take(sizeof(CellResult) * kMaxLinkCells);
    fq = take(sizeof(FaceQuery) * kMaxFaces);
    fr = take(sizeof(FaceResult) * kMaxFaces);
    kq = take(sizeof(CurvatureQuery) * kMaxLinkCells);
    kr = take(sizeof(CurvatureResult) * kMaxLinkCells);
    cap = take(2 * sizeof(double));
    arch = take(sizeof(int));
    total = o;
  }
};

const FreezeRegions kFreezeRegions;

}  // namespace

size_t freeze_arena_bytes() { return kFreezeRegions.total; }

namespace {

// OffsetCellIndex (liquid_boundary_geometry_3d.cc:47-60): one lattice step,
// out of range past the int32 lattice.
int offset_cell(const int32_t* in, int axis, int amount, int32_t* out) {
  int64_t v = (int64_t)in[axis] + amount;
  if (v < INT32_MIN || v > INT32_MAX) return FL_OUT_OF_RANGE;
  out[0] = in[0];
  out[1] = in[1];
  out[2] = in[2];
  out[axis] = (int32_t)v;
  return FL_OK;
}

// LookupSignedDistance (:82-92) over either sample kind; FailedPrecondition when absent.
template <typename R>
int lookup_distance(const R* recs, uint64_t n, const int32_t* key, const int32_t* (*keyof)(const R&), double* out) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) / 2;
    if (host_cell_less(keyof(recs[mid]), key))
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo >= n || host_cell_less(key, keyof(recs[lo]))) return FL_FAILED_PRECONDITION;
  *out = recs[lo].signed_distance;
  return FL_OK;
}

const int32_t* center_key(const fl_center_sample& s) { return s.cell_index; }
const int32_t* corner_key(const fl_corner_sample& s) { return s.corner_index; }

template <typename R>
bool samples_valid(const R* recs, uint64_t n, const int32_t* (*keyof)(const R&)) {
  for (uint64_t i = 0; i < n; ++i)
    if (!std::isfinite(recs[i].signed_distance) || (i > 0 && !host_cell_less(keyof(recs[i - 1]), keyof(recs[i]))))
      return false;
  return true;
}

bool fupload(fl_boundary* b, size_t off, size_t bytes);
bool fdownload(fl_boundary* b, size_t off, size_t bytes);

}  // namespace

namespace {

bool fupload(fl_boundary* b, size_t off, size_t bytes) {
  if (bytes == 0) return true;
  return cudaMemcpyAsync(b->fdev + off, b->fpin + off, bytes, cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
}

bool fdownload(fl_boundary* b, size_t off, size_t bytes) {
  if (bytes == 0) return true;
  return cudaMemcpyAsync(b->fpin + off, b->fdev + off, bytes, cudaMemcpyDeviceToHost, b->stream) == cudaSuccess;
}

template <typename T>
T* fhost(fl_boundary* b, size_t off) {
  return reinterpret_cast<T*>(b->fpin + off);
}
template <typename T>
T* fdevp(fl_boundary* b, size_t off) {
  return reinterpret_cast<T*>(b->fdev + off);
}

// One device phase: uploads of the staged queries, the kernel, the results
// back; adds its event time to *ms. False on a CUDA failure.
template <typename Launch>
bool freeze_phase(fl_boundary* b, size_t qoff, size_t qbytes, size_t roff, size_t rbytes, Launch launch, float* ms) {
  bool ok = cudaEventRecord(b->e0, b->stream) == cudaSuccess && fupload(b, qoff, qbytes);
  if (ok) launch();
  ok = ok && cudaGetLastError() == cudaSuccess && fdownload(b, roff, rbytes) &&
       fdownload(b, kFreezeRegions.arch, sizeof(int)) && cudaEventRecord(b->e1, b->stream) == cudaSuccess &&
       cudaStreamSynchronize(b->stream) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cudaStreamSynchronize(b->stream);
    return false;
  }
  float t = 0.0f;
  cudaEventElapsedTime(&t, b->e0, b->e1);
  *ms += t;
  return true;
}

// ValidateObstacle (liquid_boundary_geometry_3d.cc:132-175) for the kinds offered here.
int check_obstacle(const fl_obstacle& o, double step, FreezeObstacle* out) {
  out->kind = o.kind;
  out->coordinate = o.coordinate;
  out->half_width = o.kind == FL_OBSTACLE_SLAB ? o.half_width : 0.0;
  for (int a = 0; a < 3; ++a) out->n[a] = o.unit_normal[a];
  for (int k = 0; k < 6; ++k) out->tank[k] = o.tank[k];
  if (o.kind == FL_OBSTACLE_NONE) return FL_OK;
  if (o.kind == FL_OBSTACLE_OPEN_TANK) {
    // CheckTankStep (base/liquid_boundary_math.h:252-276)
    const double* t = o.tank;
    for (int k = 0; k < 6; ++k)
      if (!std::isfinite(t[k])) return FL_INVALID_ARGUMENT;
    if (t[0] >= t[1] || t[3] >= t[4]) return FL_INVALID_ARGUMENT;
    const double displacement = t[5] * step;
    const double end_x = std::fma(t[5], step, t[0]);
    const double start_width = t[1] - t[0], end_width = t[1] - end_x, width_z = t[4] - t[3];
    if (!std::isfinite(displacement) || !std::isfinite(end_x) || !std::isfinite(start_width) ||
        !std::isfinite(end_width) || !std::isfinite(width_z))
      return FL_OUT_OF_RANGE;
    if (end_x >= t[1]) return FL_FAILED_PRECONDITION;
    return FL_OK;
  }
  if (o.kind != FL_OBSTACLE_HALFSPACE && o.kind != FL_OBSTACLE_SLAB) return FL_INVALID_ARGUMENT;
  double low = o.coordinate, high = o.coordinate;
  if (o.kind == FL_OBSTACLE_SLAB) {
    if (!(std::isfinite(o.half_width) && o.half_width > 0)) return FL_INVALID_ARGUMENT;
    low = o.coordinate - o.half_width;
    high = o.coordinate + o.half_width;
    if (!std::isfinite(o.coordinate)) return FL_INVALID_ARGUMENT;
    if (!std::isfinite(low) || !std::isfinite(high) || low >= high) return FL_OUT_OF_RANGE;
  }
  const double* n = o.unit_normal;
  const double* v = o.wall_velocity;
  const bool finite_n = std::isfinite(n[0]) && std::isfinite(n[1]) && std::isfinite(n[2]);
  const bool finite_v = std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
  if (!finite_n || !finite_v || !std::isfinite(low) || std::fabs((n[0] * n[0] + n[1] * n[1] + n[2] * n[2]) - 1.0) > 1e-12)
    return FL_INVALID_ARGUMENT;
  return FL_OK;
}

}  // namespace

extern "C" int fl_boundary_freeze(fl_boundary* b, const fl_freeze_inputs* in, fl_frozen_cell* cells_out,
                                  uint64_t* cell_count, fl_frozen_face* faces_out, uint64_t* face_count,
                                  double* capillary_step_bound, fl_measurement* m) {
  if (!b || !in || !cell_count || !face_count || !capillary_step_bound) return FL_INVALID_ARGUMENT;
  int st = check_grid(in->grid);
  if (st != FL_OK) return st;
  const uint64_t n = in->cell_count;
  if ((n && (!in->cell_indices || !cells_out || !faces_out)) || (in->center_count && !in->centers) ||
      (in->corner_count && !in->corners))
    return FL_INVALID_ARGUMENT;
  // the bounded workspace's capacity (FreezeWithBackend, :2109-2113), then FreezeCore (:772-797)
  if (n > (uint64_t)kMaxLinkCells || in->center_count > kMaxCenters) return FL_RESOURCE_EXHAUSTED;
  if (!positive_finite_h(in->step_duration) || !positive_finite_h(in->liquid_density) ||
      !std::isfinite(in->surface_tension) || in->surface_tension < 0)
    return FL_INVALID_ARGUMENT;
  if (in->has_exact_curvature && !std::isfinite(in->exact_curvature)) return FL_INVALID_ARGUMENT;
  FreezeObstacle ob;
  st = check_obstacle(in->obstacle, in->step_duration, &ob);
  if (st != FL_OK) return st;
  const fl_owned_grid* g = in->grid;
  const double h = g->h, full_area = h * h, full_volume = full_area * h;
  if (!std::isnormal(full_area) || !std::isnormal(full_volume) || !std::isnormal(1 / in->liquid_density))
    return FL_OUT_OF_RANGE;
  if (!samples_valid(in->centers, in->center_count, center_key) ||
      !samples_valid(in->corners, in->corner_count, corner_key))
    return FL_INVALID_ARGUMENT;
  if (cudaSetDevice(b->device) != cudaSuccess) return FL_INTERNAL;
  const FreezeRegions& R = kFreezeRegions;
  FreezeArgs a{};
  for (int k = 0; k < 3; ++k) a.origin[k] = g->origin[k];
  a.h = h;
  a.obstacle = ob;
  a.cq = fdevp<CellQuery>(b, R.cq);
  a.cr = fdevp<CellResult>(b, R.cr);
  a.fq = fdevp<FaceQuery>(b, R.fq);
  a.fr = fdevp<FaceResult>(b, R.fr);
  a.kq = fdevp<CurvatureQuery>(b, R.kq);
  a.kr = fdevp<CurvatureResult>(b, R.kr);
  a.density = in->liquid_density;
  a.sigma = in->surface_tension;
  a.capillary = fdevp<double>(b, R.cap);
  a.arch = fdevp<int>(b, R.arch);
  float ms = 0.0f;
  auto finish_measure = [&]() {
    if (m) {
      m->compiled_architecture = *fhost<int>(b, R.arch);
      m->kernel_ms = ms;
    }
  };

  // Cells: stage until the first staging failure, compute the staged prefix,
  // then consume it in order (stage, compute and consume errors of one
  // ordinal come before those of the next).
  CellQuery* cq = fhost<CellQuery>(b, R.cq);
  b->frz_centre.assign(n ? n : 1, 0.0);
  double* centre = b->frz_centre.data();
  // working records, published to cells_out / faces_out on success
  b->frz_cells.resize(n ? n : 1);
  b->frz_faces.resize(6 * (n ? n : 1));
  fl_frozen_cell* const kept_cells = b->frz_cells.data();
  fl_frozen_face* const kept_faces = b->frz_faces.data();
  uint64_t staged = 0;
  int stage_error = FL_OK;
  for (; staged < n; ++staged) {
    const int32_t* idx = in->cell_indices + 3 * staged;
    if (staged > 0 && !host_cell_less(in->cell_indices + 3 * (staged - 1), idx)) {
      stage_error = FL_INVALID_ARGUMENT;
      break;
    }
    stage_error = lookup_distance(in->centers, in->center_count, idx, center_key, &centre[staged]);
    if (stage_error != FL_OK) break;
    CellQuery& q = cq[staged];
    for (int d = 0; d < 3; ++d) q.index[d] = idx[d];
    q.pad = 0;
    for (int c = 0; c < 8 && stage_error == FL_OK; ++c) {
      int32_t ci[3] = {idx[0], idx[1], idx[2]};
      for (int axis = 0; axis < 3 && stage_error == FL_OK; ++axis)
        stage_error = offset_cell(ci, axis, (c >> axis) & 1, ci);
      if (stage_error == FL_OK)
        stage_error = lookup_distance(in->corners, in->corner_count, ci, corner_key, &q.corner[c]);
    }
    if (stage_error != FL_OK) break;
  }
  uint64_t kept = 0, nfaces = 0;
  if (staged > 0) {
    a.ncell = (int)staged;
    if (!freeze_phase(
            b, R.cq, sizeof(CellQuery) * staged, R.cr, sizeof(CellResult) * staged,
            [&]() {
              ++g_kernel_launches;
              const unsigned ctas = (unsigned)((staged + kFreezeCellsPerCta - 1) / kFreezeCellsPerCta);
              if (ob.kind == FL_OBSTACLE_OPEN_TANK)
                k_freeze_cells_tank<<<ctas, kFreezeCellThreads, 0, b->stream>>>(a);
              else
                k_freeze_cells<<<ctas, kFreezeCellThreads, 0, b->stream>>>(a);
            },
            &ms))
      return FL_INTERNAL;
  }
  const CellResult* cr = fhost<CellResult>(b, R.cr);
  for (uint64_t i = 0; i < staged; ++i) {
    if (cr[i].status != FL_OK) return cr[i].status;
    const double low = cr[i].low, high = cr[i].high, dc = centre[i];
    if (low > 0 && high > 0 && dc < 0) return FL_FAILED_PRECONDITION;
    const double unclamped = low + high;
    if (!std::isfinite(unclamped) || unclamped < 0 || unclamped / full_volume > 1 + 64 * DBL_EPSILON)
      return FL_OUT_OF_RANGE;
    const double volume = std::min(full_volume, unclamped);
    if (!(volume == 0.0 || std::isnormal(volume))) return FL_OUT_OF_RANGE;
    if (dc >= 0 || volume == 0) continue;
    fl_frozen_cell& c = kept_cells[kept++];
    std::memset(&c, 0, sizeof(c));
    for (int d = 0; d < 3; ++d) c.cell_index[d] = in->cell_indices[3 * i + d];
    c.fluid_volume = volume;
    c.center_distance = dc;
    c.curvature = 0.0;
    for (int axis = 0; axis < 3; ++axis)
      for (int side = 0; side < 2; ++side) {
        int32_t lat[3];
        st = offset_cell(c.cell_index, axis, side, lat);
        if (st != FL_OK) return st;
        const int64_t lat64[3] = {lat[0], lat[1], lat[2]};
        uint64_t slot = 0;
        st = host_face_slot(g, axis, lat64, &slot);
        if (st != FL_OK) return st;
        fl_frozen_face& f = kept_faces[nfaces++];
        std::memset(&f, 0, sizeof(f));
        f.axis = axis;
        for (int d = 0; d < 3; ++d) f.lattice[d] = lat[d];
        f.face_slot = slot;
      }
  }
  if (stage_error != FL_OK) return stage_error;
  // faces by owned slot, one record per slot
  std::stable_sort(kept_faces, kept_faces + nfaces,
                   [](const fl_frozen_face& x, const fl_frozen_face& y) { return x.face_slot < y.face_slot; });
  nfaces = (uint64_t)(std::unique(kept_faces, kept_faces + nfaces,
                                  [](const fl_frozen_face& x, const fl_frozen_face& y) {
                                    return x.face_slot == y.face_slot;
                                  }) -
                      kept_faces);
  if (nfaces > (uint64_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  if (nfaces > 0) {
    FaceQuery* fq = fhost<FaceQuery>(b, R.fq);
    for (uint64_t f = 0; f < nfaces; ++f) {
      fq[f].axis = kept_faces[f].axis;
      for (int d = 0; d < 3; ++d) fq[f].lattice[d] = kept_faces[f].lattice[d];
    }
    a.nface = (int)nfaces;
    if (!freeze_phase(
            b, R.fq, sizeof(FaceQuery) * nfaces, R.fr, sizeof(FaceResult) * nfaces,
            [&]() {
              ++g_kernel_launches;
              k_freeze_faces<<<grid_of(nfaces, 128), 128, 0, b->stream>>>(a);
            },
            &ms))
      return FL_INTERNAL;
    const FaceResult* fr = fhost<FaceResult>(b, R.fr);
    for (uint64_t f = 0; f < nfaces; ++f) {
      if (fr[f].status != FL_OK) return fr[f].status;
      kept_faces[f].open_area = fr[f].open;
      kept_faces[f].blocked_area = fr[f].blocked;
      if (ob.kind == FL_OBSTACLE_OPEN_TANK) {
        kept_faces[f].wall_normal_velocity = fr[f].piston_velocity;
        kept_faces[f].prescribed_wall_flux = fr[f].wall_flux;
        kept_faces[f].has_prescribed_wall_flux = 1;
        kept_faces[f].is_low_x_piston_face = (uint8_t)fr[f].is_piston;
      } else {
        kept_faces[f].wall_normal_velocity =
            ob.kind == FL_OBSTACLE_NONE ? 0.0 : in->obstacle.wall_velocity[kept_faces[f].axis];
      }
    }
  }
  // Interface cells (:983-1009): a kept cell with an open face toward an air centre.
  b->frz_needs.assign(kept ? kept : 1, 0);
  uint8_t* needs = b->frz_needs.data();
  for (uint64_t f = 0; f < nfaces; ++f) {
    const fl_frozen_face& face = kept_faces[f];
    if (face.open_area == 0 || in->surface_tension == 0) continue;
    const int32_t head[3] = {face.lattice[0], face.lattice[1], face.lattice[2]};
    int32_t tail[3];
    st = offset_cell(head, face.axis, -1, tail);
    if (st != FL_OK) return st;
    const long long hc = host_find_cell(kept_cells, kept, head), tc = host_find_cell(kept_cells, kept, tail);
    if (hc >= 0 && tc >= 0) continue;
    double air = 0.0;
    st = lookup_distance(in->centers, in->center_count, hc >= 0 ? tail : head, center_key, &air);
    if (st != FL_OK) return st;
    if (air >= 0) needs[hc >= 0 ? hc : tc] = 1;
  }
  bool capillary = false;
  for (uint64_t i = 0; i < kept; ++i) capillary = capillary || needs[i];
  if (in->has_exact_curvature) {
    if (capillary && in->exact_curvature != 0) {
      const double lift = in->surface_tension * in->exact_curvature;
      if (!std::isnormal(lift)) return FL_OUT_OF_RANGE;
    }
    for (uint64_t i = 0; i < kept; ++i)
      if (needs[i]) kept_cells[i].curvature = in->exact_curvature;
  } else if (capillary) {
    // StageCenteredCurvature (:177-215): the 19 centre samples of the
    // derivative stencil, in z, y, x order; staging stops at its first failure.
    CurvatureQuery* kq = fhost<CurvatureQuery>(b, R.kq);
    b->frz_ordinal.resize(kept);
    uint64_t* ordinal = b->frz_ordinal.data();
    uint64_t nk = 0;
    int kstage = FL_OK;
    for (uint64_t i = 0; i < kept && kstage == FL_OK; ++i) {
      if (!needs[i]) continue;
      CurvatureQuery& q = kq[nk];
      for (int k = 0; k < 27; ++k) q.d[k] = 0.0;
      for (int z = -1; z <= 1 && kstage == FL_OK; ++z)
        for (int y = -1; y <= 1 && kstage == FL_OK; ++y)
          for (int x = -1; x <= 1 && kstage == FL_OK; ++x) {
            if (x != 0 && y != 0 && z != 0) continue;
            int32_t idx[3] = {kept_cells[i].cell_index[0], kept_cells[i].cell_index[1], kept_cells[i].cell_index[2]};
            const int off[3] = {x, y, z};
            for (int axis = 0; axis < 3 && kstage == FL_OK; ++axis) kstage = offset_cell(idx, axis, off[axis], idx);
            if (kstage == FL_OK)
              kstage = lookup_distance(in->centers, in->center_count, idx, center_key,
                                       &q.d[(z + 1) * 9 + (y + 1) * 3 + x + 1]);
          }
      if (kstage == FL_OK) ordinal[nk++] = i;
    }
    if (nk > 0) {
      a.ncurv = (int)nk;
      if (!freeze_phase(
              b, R.kq, sizeof(CurvatureQuery) * nk, R.kr, sizeof(CurvatureResult) * nk,
              [&]() {
                ++g_kernel_launches;
                k_freeze_curvature<<<grid_of(nk, 64), 64, 0, b->stream>>>(a);
              },
              &ms))
        return FL_INTERNAL;
      const CurvatureResult* kr = fhost<CurvatureResult>(b, R.kr);
      for (uint64_t k = 0; k < nk; ++k) {
        if (kr[k].status != FL_OK) return kr[k].status;
        kept_cells[ordinal[k]].curvature = kr[k].curvature;
      }
    }
    if (kstage != FL_OK) return kstage;
  }
  double bound = std::numeric_limits<double>::infinity();
  if (capillary) {
    if (!freeze_phase(
            b, R.cap, 0, R.cap, 2 * sizeof(double),
            [&]() {
              ++g_kernel_launches;
              k_freeze_capillary<<<1, 1, 0, b->stream>>>(a);
            },
            &ms))
      return FL_INTERNAL;
    const double* cap = fhost<double>(b, R.cap);
    if ((int)cap[1] != FL_OK) return (int)cap[1];
    bound = cap[0];
    if (in->step_duration > bound) return FL_FAILED_PRECONDITION;
  }
  if (kept) std::memcpy(cells_out, kept_cells, sizeof(fl_frozen_cell) * kept);
  if (nfaces) std::memcpy(faces_out, kept_faces, sizeof(fl_frozen_face) * nfaces);
  *cell_count = kept;
  *face_count = nfaces;
  *capillary_step_bound = bound;
  finish_measure();
  return FL_OK;
}

// ---- wetted piston (.wetted_piston) ----
//
// ComputeWettedPiston3D (wetted_piston_3d.cc:342-566) with the enclosure
// arithmetic of base/wetted_piston_math_3d.h: the wet area of the open tank's
// low-x piston, patch by lattice patch, under the liquid field (a horizontal
// plane, an analytic sphere or a union of particle spheres), as outward-rounded
// [lower, upper] bounds, and the signed fluxes handed to the piston's receiver
// faces. The device computes the spheres' sections on the piston plane (one
// thread per source) and each patch's banded area integral (one thread per
// patch); the host enumerates the patches, finds the receivers and assigns the
// patches in the reference's order.
namespace fl {
namespace {

struct WBounds {
  double lower = 0.0, upper = 0.0;
};

__host__ __device__ inline double smax(double a, double b) { return a < b ? b : a; }
__host__ __device__ inline double smin(double a, double b) { return b < a ? b : a; }
__host__ __device__ inline bool wfinite(WBounds b) { return isfinite(b.lower) && isfinite(b.upper) && b.lower <= b.upper; }
__host__ __device__ inline WBounds wpoint(double v) { return {v, v}; }
__host__ __device__ inline WBounds wadd(WBounds a, WBounds b) {
  return {add_down(a.lower, b.lower), add_up(a.upper, b.upper)};
}
__host__ __device__ inline WBounds wneg(WBounds a) { return {-a.upper, -a.lower}; }
__host__ __device__ inline WBounds wsub(WBounds a, WBounds b) { return wadd(a, wneg(b)); }

// A rounded result moved one double outward when its exact residual lies
// outward (or could have underflowed to zero).
__host__ __device__ inline double directed(double rounded, double residual, double scale, bool up) {
  if (!isfinite(rounded)) return rounded;
  const bool uncertain = residual == 0 && fabs(scale) <= 0x1p-969;
  if (uncertain || (up ? residual > 0 : residual < 0)) return nextafter(rounded, up ? kInf : -kInf);
  return rounded;
}

__host__ __device__ inline double directed_product(double a, double b, bool up) {
  const double p = a * b;
  if (a == 0 || b == 0 || fabs(a) == 1 || fabs(b) == 1 || !isfinite(p)) return p;
  return directed(p, fma(a, b, -p), p, up);
}

__host__ __device__ inline WBounds wmul_nonneg(WBounds a, WBounds b) {
  return {smax(0.0, directed_product(a.lower, b.lower, false)), directed_product(a.upper, b.upper, true)};
}

__host__ __device__ inline WBounds area_to_flux(WBounds area, double v) {
  const WBounds m = wmul_nonneg(area, wpoint(fabs(v)));
  return v < 0 ? wneg(m) : m;
}

__host__ __device__ inline double directed_quotient(double value, double divisor, bool up) {
  const double q = value / divisor;
  if (value == 0 || divisor == 1 || !isfinite(q)) return q;
  return directed(q, fma(-q, divisor, value), value, up);
}

__host__ __device__ inline WBounds wdiv(WBounds a, double d) {
  return {directed_quotient(a.lower, d, false), directed_quotient(a.upper, d, true)};
}

__host__ __device__ inline double directed_root(double v, bool up) {
  if (v <= 0) return 0.0;
  const double r = sqrt(v);
  return smax(0.0, directed(r, fma(-r, r, v), v, up));
}

__host__ __device__ inline WBounds wroot(WBounds a) { return {directed_root(a.lower, false), directed_root(a.upper, true)}; }
__host__ __device__ inline WBounds wmax(WBounds a, WBounds b) { return {smax(a.lower, b.lower), smax(a.upper, b.upper)}; }
__host__ __device__ inline WBounds wmin(WBounds a, WBounds b) { return {smin(a.lower, b.lower), smin(a.upper, b.upper)}; }
__host__ __device__ inline WBounds wmag(WBounds a) {
  return {smax(0.0, smax(a.lower, -a.upper)), smax(a.upper, -a.lower)};
}
__host__ __device__ inline WBounds wsquare(WBounds a) {
  const WBounds m = wmag(a);
  return wmul_nonneg(m, m);
}

// (world - origin) / h - index as an enclosure, in cell widths.
__host__ __device__ inline WBounds lattice_offset(double world, double origin, double index, double h) {
  const OffsetBounds b = tank_plane_offset(world, origin, index, h).bounds();
  if (!isfinite(b.estimate) || !isfinite(b.lower) || !isfinite(b.upper)) return {kInf, kInf};
  return wdiv({b.lower, b.upper}, h);
}

struct PistonField {
  double origin[3], h;
  double tank[6];  // start low x, high x, floor y, low z, high z, piston velocity x
  double radius;   // sphere radius (m)
  double plane_y;  // plane height (m)
  int is_plane;
};

// A sphere's section by the piston plane, in cell widths (radius squared
// zero: the sphere misses the plane).
struct PistonDisk {
  WBounds y, z, r2;
  int status;
};

__host__ __device__ inline PistonDisk piston_section(const PistonField& f, const double c[3]) {
  PistonDisk d{};
  d.status = FL_OK;
  const double h = f.h;
  const WBounds dist = wmag(wsub(wpoint(c[0]), wpoint(f.tank[0])));
  if (!wfinite(dist)) {
    d.status = FL_OUT_OF_RANGE;
    return d;
  }
  if (dist.lower >= f.radius) return d;
  const WBounds R = wpoint(f.radius);
  const WBounds less = wmax(wpoint(0.0), wsub(R, dist));
  const WBounds more = wadd(wdiv(R, h), wdiv(dist, h));
  const WBounds r2 = wmul_nonneg(wdiv(less, h), more);
  const WBounds cy = lattice_offset(c[1], f.origin[1], 0.0, h), cz = lattice_offset(c[2], f.origin[2], 0.0, h);
  if (!wfinite(r2) || !wfinite(cy) || !wfinite(cz) || r2.upper <= 0) {
    d.status = FL_OUT_OF_RANGE;
    return d;
  }
  d.y = cy;
  d.z = cz;
  d.r2 = r2;
  return d;
}

struct PistonInterval {
  double low, high;
};

__host__ __device__ inline bool interval_less(PistonInterval a, PistonInterval b) {
  return a.low < b.low || (a.low == b.low && a.high < b.high);
}

__host__ __device__ inline void sift(PistonInterval* v, size_t count, size_t root) {
  while (root < count / 2) {
    size_t child = root * 2 + 1;
    if (child + 1 < count && interval_less(v[child], v[child + 1])) ++child;
    if (!interval_less(v[root], v[child])) break;
    const PistonInterval t = v[root];
    v[root] = v[child];
    v[child] = t;
    root = child;
  }
}

// Length of a union of intervals (heap sort, then a sweep), lower or upper bound.
__host__ __device__ inline double union_length(PistonInterval* v, size_t count, bool upper) {
  if (count == 0) return 0.0;
  for (size_t start = count / 2; start > 0; --start) sift(v, count, start - 1);
  for (size_t end = count - 1; end > 0; --end) {
    const PistonInterval t = v[0];
    v[0] = v[end];
    v[end] = t;
    sift(v, end, 0);
  }
  WBounds length;
  PistonInterval cur = v[0];
  for (size_t k = 1; k < count; ++k) {
    const PistonInterval nx = v[k];
    if (nx.low <= cur.high) {
      cur.high = smax(cur.high, nx.high);
      continue;
    }
    length = wadd(length, wsub(wpoint(cur.high), wpoint(cur.low)));
    cur = nx;
  }
  length = wadd(length, wsub(wpoint(cur.high), wpoint(cur.low)));
  return upper ? length.upper : length.lower;
}

__host__ __device__ inline WBounds world_area(WBounds lattice_area, double h) {
  return wmul_nonneg(wmul_nonneg(lattice_area, wpoint(h)), wpoint(h));
}

__host__ __device__ inline WBounds width_of(WBounds lo, WBounds hi) { return wmax(wpoint(0.0), wsub(hi, lo)); }
__host__ __device__ inline WBounds nearest_of(WBounds c, WBounds lo, WBounds hi) {
  return wmax(wpoint(0.0), wmax(wsub(lo, c), wsub(c, hi)));
}
__host__ __device__ inline WBounds farthest_of(WBounds c, WBounds lo, WBounds hi) {
  return wmax(wmag(wsub(c, lo)), wmag(wsub(c, hi)));
}
__host__ __device__ inline WBounds gap_of(WBounds r2, WBounds dy, WBounds dz) {
  return wsub(wsub(r2, wsquare(dy)), wsquare(dz));
}

struct PatchResult {
  WBounds area;
  double midpoint_flux;
  int cross_lower;  // every wet source crosses the patch's lower edge
  int status;
};

constexpr int kPistonBands = 64;

// IntegratePatch + MeasurePatch (wetted_piston_math_3d.h:280-424), split so
// that a patch's 64 z-bands run on 64 threads: the patch's frame (its
// rectangle inside the tank's floor and z walls and under a plane surface),
// the wet test over all sources, and one band's interval-union lengths times
// its width; the band products are summed in band order.
struct PatchFrame {
  WBounds rlo_y, rhi_y, rlo_z, rhi_z, rect, floor_, surface, zw;
  int status;
  bool empty;  // a zero-width rectangle
};

__device__ PatchFrame patch_frame(const PistonField& f, int32_t py, int32_t pz) {
  PatchFrame fr{};
  fr.status = FL_OK;
  const double h = f.h;
  fr.floor_ = lattice_offset(f.tank[2], f.origin[1], (double)py, h);
  const WBounds low_z = lattice_offset(f.tank[3], f.origin[2], (double)pz, h);
  const WBounds high_z = lattice_offset(f.tank[4], f.origin[2], (double)pz, h);
  fr.surface = f.is_plane ? lattice_offset(f.plane_y, f.origin[1], (double)py, h) : wpoint(1.0);
  if (!wfinite(fr.floor_) || !wfinite(low_z) || !wfinite(high_z) || !wfinite(fr.surface)) {
    fr.status = FL_OUT_OF_RANGE;
    return fr;
  }
  fr.rlo_y = wmax(wpoint(0.0), fr.floor_);
  fr.rhi_y = wmin(wpoint(1.0), fr.surface);
  fr.rlo_z = wmax(wpoint(0.0), low_z);
  fr.rhi_z = wmin(wpoint(1.0), high_z);
  const WBounds yw = width_of(fr.rlo_y, fr.rhi_y);
  fr.zw = width_of(fr.rlo_z, fr.rhi_z);
  fr.empty = yw.upper == 0 || fr.zw.upper == 0;
  if (!fr.empty) fr.rect = wmul_nonneg(yw, fr.zw);
  return fr;
}

// Whether any source's section reaches the patch rectangle, and whether every
// such source crosses the patch's lower edge.
__device__ bool patch_wet(const PatchFrame& fr, int32_t py, int32_t pz, const PistonDisk* disks, int nd, int* status,
                          bool* cross) {
  *cross = fr.floor_.upper <= 0 && fr.zw.lower > 0;
  bool wet = false;
  for (int k = 0; k < nd; ++k) {
    const PistonDisk& d = disks[k];
    if (d.r2.upper == 0) continue;
    const WBounds y = wsub(d.y, wpoint((double)py)), z = wsub(d.z, wpoint((double)pz));
    const WBounds ny = nearest_of(y, fr.rlo_y, fr.rhi_y), nz = nearest_of(z, fr.rlo_z, fr.rhi_z);
    const WBounds pg = gap_of(d.r2, ny, nz);
    if (!wfinite(pg)) {
      *status = FL_OUT_OF_RANGE;
      return false;
    }
    if (pg.upper <= 0) continue;
    wet = true;
    const WBounds eg = gap_of(d.r2, wmag(y), nz);
    if (!wfinite(eg)) {
      *status = FL_OUT_OF_RANGE;
      return false;
    }
    *cross = *cross && eg.lower > 0;
  }
  *status = FL_OK;
  return wet;
}

// Band `band` of the patch: [inner, outer] union length of the sections'
// chords times the band's width; used = false for a band outside the rectangle.
__device__ int band_product(const PatchFrame& fr, int32_t py, int32_t pz, const PistonDisk* disks, int nd, int band,
                            PistonInterval* inner, PistonInterval* outer, WBounds* prod, bool* used) {
  const WBounds blo = wmax(fr.rlo_z, wpoint((double)band / kPistonBands));
  const WBounds bhi = wmin(fr.rhi_z, wpoint((double)(band + 1) / kPistonBands));
  const WBounds bw = width_of(blo, bhi);
  *used = bw.upper != 0;
  if (!*used) return FL_OK;
  size_t ni = 0, no = 0;
  for (int k = 0; k < nd; ++k) {
    const PistonDisk& d = disks[k];
    if (d.r2.upper == 0) continue;
    const WBounds z = wsub(d.z, wpoint((double)pz));
    const WBounds near2 = wsquare(nearest_of(z, blo, bhi)), far2 = wsquare(farthest_of(z, blo, bhi));
    const WBounds outer2 = wsub(d.r2, near2), inner2 = wsub(d.r2, far2);
    if (!wfinite(outer2) || !wfinite(inner2)) return FL_OUT_OF_RANGE;
    if (outer2.upper <= 0) continue;
    const WBounds y = wsub(d.y, wpoint((double)py));
    const double ro = directed_root(outer2.upper, true);
    const double olo = wmax(fr.rlo_y, wsub(y, wpoint(ro))).lower;
    const double ohi = wmin(fr.rhi_y, wadd(y, wpoint(ro))).upper;
    if (olo < ohi) outer[no++] = {olo, ohi};
    if (inner2.lower > 0) {
      const double ri = directed_root(inner2.lower, false);
      const double ilo = wmax(fr.rlo_y, wsub(y, wpoint(ri))).upper;
      const double ihi = wmin(fr.rhi_y, wadd(y, wpoint(ri))).lower;
      if (ilo < ihi) inner[ni++] = {ilo, ihi};
    }
  }
  const WBounds len{union_length(inner, ni, false), union_length(outer, no, true)};
  *prod = wmul_nonneg(len, bw);
  return FL_OK;
}

__global__ void k_piston_sections(PistonField f, const double* centers, int n, PistonDisk* disks, int* arch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *arch = compiled_arch();
  if (i < n) disks[i] = piston_section(f, centers + 3 * i);
}

// One CTA of 64 threads (one per band) per patch in flight, patches strided
// over the CTAs; each thread sorts its band's intervals in its own two banks
// of nd records.
__global__ void __launch_bounds__(kPistonBands) k_piston_patches(PistonField f, const PistonDisk* disks, int nd,
                                                                 const int32_t* patches, int np,
                                                                 PistonInterval* banks, PatchResult* out) {
  __shared__ WBounds prod[kPistonBands];
  __shared__ int used[kPistonBands], bad[kPistonBands];
  const int band = threadIdx.x;
  const size_t ndc = nd > 0 ? (size_t)nd : 1;
  PistonInterval* inner = banks + ((size_t)blockIdx.x * kPistonBands + band) * 2 * ndc;
  PistonInterval* outer = inner + ndc;
  for (int p = blockIdx.x; p < np; p += gridDim.x) {
    const int32_t py = patches[2 * p], pz = patches[2 * p + 1];
    const PatchFrame fr = patch_frame(f, py, pz);
    PatchResult m{};
    m.cross_lower = 1;
    m.status = fr.status;
    bool bands = false;
    if (m.status == FL_OK && !fr.empty) {
      if (f.is_plane) {
        m.area = world_area(fr.rect, f.h);
        m.cross_lower = fr.floor_.upper <= 0 && fr.surface.lower > 0 && fr.zw.lower > 0;
        if (!wfinite(m.area)) m.status = FL_OUT_OF_RANGE;
      } else {
        bool cross = true;
        int st = FL_OK;
        const bool wet = patch_wet(fr, py, pz, disks, nd, &st, &cross);
        m.status = st;
        if (st == FL_OK && wet) {
          bands = true;  // the same on every thread: all compute the frame and wet test alike
          m.cross_lower = cross;
        }
      }
    }
    if (bands) {
      WBounds pr;
      bool u = false;
      bad[band] = band_product(fr, py, pz, disks, nd, band, inner, outer, &pr, &u);
      prod[band] = pr;
      used[band] = u;
      __syncthreads();
      if (band == 0) {
        WBounds area;
        for (int k = 0; k < kPistonBands && m.status == FL_OK; ++k) {
          if (bad[k] != FL_OK)
            m.status = bad[k];
          else if (used[k])
            area = wadd(area, prod[k]);
        }
        if (m.status == FL_OK) {
          m.area = world_area(wmin(area, fr.rect), f.h);
          if (!wfinite(m.area)) m.status = FL_OUT_OF_RANGE;
        }
      }
      __syncthreads();  // the shared band results are reused by the next patch
    }
    if (band == 0) {
      if (m.status == FL_OK) {
        m.midpoint_flux = midpoint(m.area.lower, m.area.upper) * f.tank[5];
        if (!isfinite(m.midpoint_flux)) m.status = FL_OUT_OF_RANGE;
      }
      out[p] = m;
    }
  }
}

}  // namespace
}  // namespace fl

namespace {

constexpr int kPistonCtas = 32;  // patches measured at once (64 band threads each, two interval banks per thread)

struct PistonRegions {
  size_t centers, disks, patches, results, arch, staged, banks, total;
  PistonRegions() {
    size_t o = 0;
    auto take = [&](size_t bytes) {
      const size_t r = o;
      o = align_up(o + bytes);
      return r;
    };
    centers = take(sizeof(double) * 3 * kMaxParticles);
    disks = take(sizeof(PistonDisk) * kMaxParticles);
    patches = take(sizeof(int32_t) * 2 * kMaxFaces);
    results = take(sizeof(PatchResult) * kMaxFaces);
    arch = take(sizeof(int));
    staged = o;
    banks = take(sizeof(PistonInterval) * 2 * kPistonCtas * kPistonBands * kMaxParticles);
    total = o;
  }
};

const PistonRegions kPistonRegions;

}  // namespace

size_t piston_arena_bytes() { return kPistonRegions.total; }
size_t piston_pinned_bytes() { return kPistonRegions.staged; }

namespace {

constexpr int64_t kFirstLattice = INT32_MIN;
constexpr int64_t kPastLastLattice = (int64_t)INT32_MAX + 1;

// CheckTankStep (base/liquid_boundary_math.h:252-276).
int check_tank(const double* t, double step) {
  for (int k = 0; k < 6; ++k)
    if (!std::isfinite(t[k])) return FL_INVALID_ARGUMENT;
  if (t[0] >= t[1] || t[3] >= t[4]) return FL_INVALID_ARGUMENT;
  const double displacement = t[5] * step;
  const double end_x = std::fma(t[5], step, t[0]);
  const double start_width = t[1] - t[0], end_width = t[1] - end_x, width_z = t[4] - t[3];
  if (!std::isfinite(displacement) || !std::isfinite(end_x) || !std::isfinite(start_width) ||
      !std::isfinite(end_width) || !std::isfinite(width_z))
    return FL_OUT_OF_RANGE;
  if (end_x >= t[1]) return FL_FAILED_PRECONDITION;
  return FL_OK;
}

bool patch_less(const int32_t* a, const int32_t* b) { return a[1] != b[1] ? a[1] < b[1] : a[0] < b[0]; }

// AddIndex (wetted_piston_3d.cc:131-149): a sorted, deduplicated (z, y) insert.
int add_patch(std::vector<int32_t>& idx, int32_t y, int32_t z) {
  const int32_t key[2] = {y, z};
  size_t lo = 0, hi = idx.size() / 2;
  while (lo < hi) {
    const size_t mid = (lo + hi) / 2;
    if (patch_less(&idx[2 * mid], key))
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < idx.size() / 2 && idx[2 * lo] == y && idx[2 * lo + 1] == z) return FL_OK;
  if (idx.size() / 2 == (size_t)kMaxFaces) return FL_RESOURCE_EXHAUSTED;
  idx.insert(idx.begin() + 2 * lo, key, key + 2);
  return FL_OK;
}

// AddRectangle (:158-186): every patch the rectangle (in cell widths) touches.
int add_rectangle(std::vector<int32_t>& idx, double low_y, double high_y, double low_z, double high_z) {
  if (!(low_y < high_y && low_z < high_z)) return FL_OK;
  if (low_y < kFirstLattice || low_z < kFirstLattice || high_y > kPastLastLattice || high_z > kPastLastLattice)
    return FL_OUT_OF_RANGE;
  const int64_t fy = (int64_t)std::floor(low_y), fz = (int64_t)std::floor(low_z);
  const int64_t ey = (int64_t)std::ceil(high_y), ez = (int64_t)std::ceil(high_z);
  const uint64_t rows = (uint64_t)(ey - fy), cols = (uint64_t)(ez - fz);
  if (rows > (uint64_t)kMaxFaces || cols > (uint64_t)kMaxFaces / rows) return FL_RESOURCE_EXHAUSTED;
  for (int64_t z = fz; z < ez; ++z)
    for (int64_t y = fy; y < ey; ++y) {
      const int st = add_patch(idx, (int32_t)y, (int32_t)z);
      if (st != FL_OK) return st;
    }
  return FL_OK;
}

}  // namespace

extern "C" int fl_boundary_wetted_piston(fl_boundary* b, const fl_owned_grid* grid, const fl_frozen_cell* cells,
                                         uint64_t nc, const fl_frozen_face* faces, uint64_t nf,
                                         const fl_piston_field* field, const double* particles, uint64_t np,
                                         const double tank[6], fl_piston_patch* patches, uint64_t patch_capacity,
                                         uint64_t* patch_count, double* face_fluxes, uint8_t* has_face_flux,
                                         double whole_area[2], double whole_flux[2], uint64_t* attached,
                                         fl_measurement* m) {
  if (!b || !field || !tank || !patch_count || !whole_area || !whole_flux || !attached ||
      (nc && !cells) || (nf && (!faces || !face_fluxes || !has_face_flux)) || (np && !particles) ||
      (patch_capacity && !patches))
    return FL_INVALID_ARGUMENT;
  int st = check_grid(grid);
  if (st != FL_OK) return st;
  // the workspace's capacities, then Run (wetted_piston_3d.cc:351-383)
  if (nf > (uint64_t)kMaxFaces || nc > (uint64_t)kMaxLinkCells || np > (uint64_t)kMaxParticles)
    return FL_RESOURCE_EXHAUSTED;
  st = check_tank(tank, 0.0);
  if (st != FL_OK) return st;
  const double h = grid->h;
  const WBounds nominal = world_area(wpoint(1.0), h);
  if (!wfinite(nominal) || nominal.lower <= 0) return FL_OUT_OF_RANGE;
  for (uint64_t f = 0; f < nf; ++f) {
    const int64_t lat[3] = {faces[f].lattice[0], faces[f].lattice[1], faces[f].lattice[2]};
    uint64_t slot = 0;
    if (host_face_slot(grid, faces[f].axis, lat, &slot) != FL_OK || slot != faces[f].face_slot ||
        (f > 0 && faces[f - 1].face_slot >= slot))
      return FL_INVALID_ARGUMENT;
  }
  for (uint64_t i = 0; i < nc; ++i)
    if (!std::isfinite(cells[i].fluid_volume) || cells[i].fluid_volume <= 0 ||
        (i > 0 && !host_cell_less(cells[i - 1].cell_index, cells[i].cell_index)))
      return FL_INVALID_ARGUMENT;
  PistonField pf{};
  for (int a = 0; a < 3; ++a) pf.origin[a] = grid->origin[a];
  pf.h = h;
  for (int k = 0; k < 6; ++k) pf.tank[k] = tank[k];
  if (field->kind == FL_PISTON_FIELD_PLANE) {
    pf.is_plane = 1;
    pf.plane_y = field->plane_height_y;
    if (!std::isfinite(pf.plane_y)) return FL_INVALID_ARGUMENT;
  } else {
    if (field->kind != FL_PISTON_FIELD_SPHERE && field->kind != FL_PISTON_FIELD_PARTICLE_UNION)
      return FL_INVALID_ARGUMENT;
    pf.radius = field->radius;
    const double* c = field->sphere_center;
    if (!std::isfinite(pf.radius) || pf.radius <= 0 ||
        (field->kind == FL_PISTON_FIELD_SPHERE &&
         !(std::isfinite(c[0]) && std::isfinite(c[1]) && std::isfinite(c[2]))))
      return FL_INVALID_ARGUMENT;
  }
  for (uint64_t i = 0; i < np; ++i)
    if (!std::isfinite(particles[3 * i]) || !std::isfinite(particles[3 * i + 1]) || !std::isfinite(particles[3 * i + 2]))
      return FL_INVALID_ARGUMENT;
  // FindPistonOwnerLatticeX (:102-129): the cell whose half-open x span holds the piston plane.
  auto side = [&](int64_t index, int* sg) { return tank_plane_sign(tank[0], grid->origin[0], (double)index, h, sg); };
  int64_t lo = kFirstLattice, hi = kPastLastLattice;
  int lo_side = 0, hi_side = 0;
  if (side(lo, &lo_side) != FL_OK || side(hi, &hi_side) != FL_OK || lo_side < 0 || hi_side >= 0)
    return FL_OUT_OF_RANGE;
  while (hi - lo > 1) {
    const int64_t mid = lo + (hi - lo) / 2;
    int sg = 0;
    if (side(mid, &sg) != FL_OK) return FL_OUT_OF_RANGE;
    if (sg < 0)
      hi = mid;
    else
      lo = mid;
  }
  const int32_t px = (int32_t)lo;
  const double velocity = tank[5];
  std::vector<int32_t>& idx = b->pst_idx;  // reserved for every patch the workspace admits
  idx.clear();
  for (uint64_t i = 0; i < nc; ++i)
    if (cells[i].cell_index[0] == px) {
      st = add_patch(idx, cells[i].cell_index[1], cells[i].cell_index[2]);
      if (st != FL_OK) return st;
    }
  // sections of the field's spheres by the piston plane
  const PistonRegions& R = kPistonRegions;
  const int sources = field->kind == FL_PISTON_FIELD_SPHERE ? 1 : (field->kind == FL_PISTON_FIELD_PARTICLE_UNION ? (int)np : 0);
  if (cudaSetDevice(b->device) != cudaSuccess) return FL_INTERNAL;
  double* centers = reinterpret_cast<double*>(b->ppin + R.centers);
  if (field->kind == FL_PISTON_FIELD_SPHERE)
    for (int a = 0; a < 3; ++a) centers[a] = field->sphere_center[a];
  else if (sources > 0)
    std::memcpy(centers, particles, sizeof(double) * 3 * sources);
  float ms = 0.0f;
  auto phase = [&](size_t qoff, size_t qbytes, size_t roff, size_t rbytes, auto launch) {
    bool ok = cudaEventRecord(b->e0, b->stream) == cudaSuccess &&
              (qbytes == 0 || cudaMemcpyAsync(b->pdev + qoff, b->ppin + qoff, qbytes, cudaMemcpyHostToDevice,
                                              b->stream) == cudaSuccess);
    if (ok) launch();
    ok = ok && cudaGetLastError() == cudaSuccess &&
         (rbytes == 0 || cudaMemcpyAsync(b->ppin + roff, b->pdev + roff, rbytes, cudaMemcpyDeviceToHost, b->stream) ==
                             cudaSuccess) &&
         cudaMemcpyAsync(b->ppin + R.arch, b->pdev + R.arch, sizeof(int), cudaMemcpyDeviceToHost, b->stream) ==
             cudaSuccess &&
         cudaEventRecord(b->e1, b->stream) == cudaSuccess && cudaStreamSynchronize(b->stream) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      cudaStreamSynchronize(b->stream);
      return false;
    }
    float t = 0.0f;
    cudaEventElapsedTime(&t, b->e0, b->e1);
    ms += t;
    return true;
  };
  PistonDisk* disks_d = reinterpret_cast<PistonDisk*>(b->pdev + R.disks);
  int* arch_d = reinterpret_cast<int*>(b->pdev + R.arch);
  if (sources > 0 &&
      !phase(R.centers, sizeof(double) * 3 * sources, R.disks, sizeof(PistonDisk) * sources, [&]() {
        ++g_kernel_launches;
        k_piston_sections<<<grid_of(sources, 128), 128, 0, b->stream>>>(
            pf, reinterpret_cast<const double*>(b->pdev + R.centers), sources, disks_d, arch_d);
      }))
    return FL_INTERNAL;
  const PistonDisk* disks = reinterpret_cast<const PistonDisk*>(b->ppin + R.disks);
  for (int k = 0; k < sources; ++k) {
    if (disks[k].status != FL_OK) return disks[k].status;
    if (!wfinite(disks[k].r2) || disks[k].r2.lower < 0 || !wfinite(disks[k].y) || !wfinite(disks[k].z))
      return FL_OUT_OF_RANGE;
  }
  // AddSupport (:188-232): the patches each section's circumscribed square touches
  {
    const WBounds fl_ = lattice_offset(tank[2], grid->origin[1], 0.0, h);
    const WBounds lz = lattice_offset(tank[3], grid->origin[2], 0.0, h);
    const WBounds hz = lattice_offset(tank[4], grid->origin[2], 0.0, h);
    if (!wfinite(fl_) || !wfinite(lz) || !wfinite(hz)) return FL_OUT_OF_RANGE;
    if (pf.is_plane) {
      if (pf.plane_y > tank[2]) {
        const WBounds sf = lattice_offset(pf.plane_y, grid->origin[1], 0.0, h);
        if (!wfinite(sf)) return FL_OUT_OF_RANGE;
        st = add_rectangle(idx, fl_.lower, sf.upper, lz.lower, hz.upper);
        if (st != FL_OK) return st;
      }
    } else {
      for (int k = 0; k < sources; ++k) {
        const PistonDisk& d = disks[k];
        if (d.r2.upper == 0) continue;
        const WBounds r = wroot(d.r2);
        const WBounds ys = wadd(d.y, {-r.upper, r.upper}), zs = wadd(d.z, {-r.upper, r.upper});
        if (!wfinite(ys) || !wfinite(zs)) return FL_OUT_OF_RANGE;
        st = add_rectangle(idx, std::max(ys.lower, fl_.lower), ys.upper, std::max(zs.lower, lz.lower),
                           std::min(zs.upper, hz.upper));
        if (st != FL_OK) return st;
      }
    }
  }
  const size_t npatch = idx.size() / 2;
  if (npatch > patch_capacity) return FL_RESOURCE_EXHAUSTED;
  // working outputs, published to the caller's buffers on success
  b->pst_patches.resize(npatch);
  b->pst_flux.assign(nf, 0.0);
  b->pst_has.assign(nf, 0);
  fl_piston_patch* const work = b->pst_patches.data();
  double* const fluxes = b->pst_flux.data();
  uint8_t* const has_flux = b->pst_has.data();
  for (size_t k = 0; k < npatch; ++k) {
    fl_piston_patch& rec = work[k];
    std::memset(&rec, 0, sizeof(rec));
    rec.lattice_y = idx[2 * k];
    rec.lattice_z = idx[2 * k + 1];
    const int32_t key[3] = {px, rec.lattice_y, rec.lattice_z};
    if (host_find_cell(cells, nc, key) < 0) continue;
    // FindReceiverFaceOrdinal (:234-256): the piston face of the selected cell
    const int64_t lat[3] = {px, rec.lattice_y, rec.lattice_z};
    uint64_t slot = 0;
    if (host_face_slot(grid, 0, lat, &slot) != FL_OK) return FL_FAILED_PRECONDITION;
    uint64_t a = 0, e = nf;
    while (a < e) {
      const uint64_t mid = (a + e) / 2;
      if (faces[mid].face_slot < slot)
        a = mid + 1;
      else
        e = mid;
    }
    const int32_t tail_key[3] = {px - 1, rec.lattice_y, rec.lattice_z};
    const bool has_tail = (int64_t)px > kFirstLattice && host_find_cell(cells, nc, tail_key) >= 0;
    if (a == nf || faces[a].face_slot != slot || has_tail) return FL_FAILED_PRECONDITION;
    const fl_frozen_face& face = faces[a];
    const double flux = face.prescribed_wall_flux;
    if (face.open_area != 0 || face.blocked_area != h * h || face.wall_normal_velocity != velocity ||
        !face.has_prescribed_wall_flux || !std::isfinite(flux) || (velocity == 0 && flux != 0) ||
        (velocity > 0 && flux <= 0) || (velocity < 0 && flux >= 0))
      return FL_FAILED_PRECONDITION;
    rec.has_receiver = 1;
    rec.receiver_face_ordinal = a;
    has_flux[a] = 1;
    fluxes[a] = 0.0;
  }
  for (uint64_t f = 0; f < nf; ++f)
    if (faces[f].has_prescribed_wall_flux && faces[f].prescribed_wall_flux != 0 && !has_flux[f])
      return FL_FAILED_PRECONDITION;
  // every patch's wet area on the device
  PatchResult* res = reinterpret_cast<PatchResult*>(b->ppin + R.results);
  if (npatch > 0) {
    std::memcpy(b->ppin + R.patches, idx.data(), sizeof(int32_t) * idx.size());
    const int nd = sources;
    if (!phase(R.patches, sizeof(int32_t) * idx.size(), R.results, sizeof(PatchResult) * npatch, [&]() {
          ++g_kernel_launches;
          const int blocks = (int)std::min<size_t>(npatch, kPistonCtas);
          k_piston_patches<<<blocks, kPistonBands, 0, b->stream>>>(
              pf, disks_d, nd, reinterpret_cast<const int32_t*>(b->pdev + R.patches), (int)npatch,
              reinterpret_cast<PistonInterval*>(b->pdev + R.banks), reinterpret_cast<PatchResult*>(b->pdev + R.results));
        }))
      return FL_INTERNAL;
  }
  WBounds whole;
  for (size_t k = 0; k < npatch; ++k) {
    if (res[k].status != FL_OK) return res[k].status;
    if (!wfinite(res[k].area) || res[k].area.lower < 0 || res[k].area.upper > nominal.upper ||
        !std::isfinite(res[k].midpoint_flux))
      return FL_OUT_OF_RANGE;
    work[k].area[0] = res[k].area.lower;
    work[k].area[1] = res[k].area.upper;
    whole = wadd(whole, res[k].area);
  }
  const WBounds wflux = area_to_flux(whole, velocity);
  if (!wfinite(whole) || !wfinite(wflux)) return FL_OUT_OF_RANGE;
  if (whole.upper > 0) {
    const double width = add_up(whole.upper, -whole.lower);
    const double limit = directed_quotient(whole.lower, 1000, false);
    if (whole.lower <= 0 || width > limit) return FL_FAILED_PRECONDITION;
  }
  // AssignPatches (:285-328): per z column, a wet patch without a receiver
  // joins the column's highest receiver when that lies directly below it.
  uint64_t joined = 0;
  for (size_t begin = 0; begin < npatch;) {
    size_t end = begin;
    long long highest = -1;
    while (end < npatch && work[end].lattice_z == work[begin].lattice_z) {
      if (work[end].has_receiver) highest = (long long)end;
      ++end;
    }
    for (size_t k = begin; k < end; ++k) {
      fl_piston_patch& p = work[k];
      if (p.area[1] == 0) continue;
      fl_piston_patch* recv = &p;
      if (!p.has_receiver) {
        if (highest < 0 || (int64_t)p.lattice_y - work[highest].lattice_y != 1 || !res[k].cross_lower)
          return FL_FAILED_PRECONDITION;
        recv = &work[highest];
        p.has_receiver = 1;
        p.receiver_face_ordinal = recv->receiver_face_ordinal;
        ++joined;
      }
      const WBounds ra = wadd({recv->receiver_area[0], recv->receiver_area[1]}, {p.area[0], p.area[1]});
      const WBounds rf = wadd({recv->receiver_flux[0], recv->receiver_flux[1]},
                              area_to_flux({p.area[0], p.area[1]}, velocity));
      recv->receiver_area[0] = ra.lower;
      recv->receiver_area[1] = ra.upper;
      recv->receiver_flux[0] = rf.lower;
      recv->receiver_flux[1] = rf.upper;
      double& acc = fluxes[recv->receiver_face_ordinal];
      acc += res[k].midpoint_flux;
      if (!wfinite(ra) || !wfinite(rf) || !std::isfinite(acc)) return FL_OUT_OF_RANGE;
    }
    begin = end;
  }
  WBounds assigned_area, assigned_flux;
  for (size_t k = 0; k < npatch; ++k) {
    const fl_piston_patch& p = work[k];
    if (p.receiver_area[1] == 0) continue;
    const WBounds enc{p.receiver_flux[0], p.receiver_flux[1]};
    const double given = fluxes[p.receiver_face_ordinal];
    if (!wfinite(enc) || given < enc.lower || given > enc.upper) return FL_OUT_OF_RANGE;
    assigned_area = wadd(assigned_area, {p.receiver_area[0], p.receiver_area[1]});
    assigned_flux = wadd(assigned_flux, enc);
  }
  const bool area_ok =
      wfinite(assigned_area) && assigned_area.upper >= whole.lower && assigned_area.lower <= whole.upper;
  const bool flux_ok =
      wfinite(assigned_flux) && assigned_flux.upper >= wflux.lower && assigned_flux.lower <= wflux.upper;
  if (!area_ok || !flux_ok) return FL_OUT_OF_RANGE;
  if (npatch) std::memcpy(patches, work, sizeof(fl_piston_patch) * npatch);
  if (nf) {
    std::memcpy(face_fluxes, fluxes, sizeof(double) * nf);
    std::memcpy(has_face_flux, has_flux, nf);
  }
  *patch_count = npatch;
  whole_area[0] = whole.lower;
  whole_area[1] = whole.upper;
  whole_flux[0] = wflux.lower;
  whole_flux[1] = wflux.upper;
  *attached = joined;
  if (m) {
    m->compiled_architecture = *reinterpret_cast<int*>(b->ppin + R.arch);
    m->kernel_ms = ms;
  }
  return FL_OK;
}
