// Bounded boundary-aware transfers on the reference's owned sparse grid: the
// operations behind the liquid scheduler's backend table (.deposit, .normalize,
// .predict_missing_face, .forces, .gather; liquid_substep_backend_3d.h:121-194).
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
#include <cfloat>
#include <cmath>
#include <cstring>

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
            cudaMallocHost(&b->lpin, link_arena_bytes()) == cudaSuccess;
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
