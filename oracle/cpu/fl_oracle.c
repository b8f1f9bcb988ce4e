/* FP64 CPU restatement of FluidiTy's liquid-step hot path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Each function names the reference code it restates (paths inside FluidiTy).
 * The restatement drops the reference's error-free edge handling
 * (NormalizeCoordinate / IsBelow / FaceDisplacement, sparse_mac_grid_3d.cc:95-165),
 * which only changes results for coordinates within a few ulps of a lattice edge
 * or for extreme magnitudes; the parity tests pin the two against each other on
 * ordinary inputs through oracle/_ref/libfluidity_ref.so.
 */
#include "fl_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Box helpers                                                                */

static inline int64_t face_dim(const fo_box* b, int axis, int d) { return b->n[d] + (axis == d ? 1 : 0); }

size_t fo_face_count(const fo_box* b, int axis) {
  return (size_t)(face_dim(b, axis, 0) * face_dim(b, axis, 1) * face_dim(b, axis, 2));
}

/* Face (axis, i, j, k) in global lattice indices -> dense index, or -1 outside the box. */
static inline int64_t face_at(const fo_box* b, int axis, int64_t i, int64_t j, int64_t k) {
  const int64_t li = i - b->lo[0], lj = j - b->lo[1], lk = k - b->lo[2];
  const int64_t nx = face_dim(b, axis, 0), ny = face_dim(b, axis, 1), nz = face_dim(b, axis, 2);
  if (li < 0 || lj < 0 || lk < 0 || li >= nx || lj >= ny || lk >= nz) return -1;
  return (lk * ny + lj) * nx + li;
}

static inline int64_t cell_at(const fo_box* b, int64_t i, int64_t j, int64_t k) {
  const int64_t li = i - b->lo[0], lj = j - b->lo[1], lk = k - b->lo[2];
  if (li < 0 || lj < 0 || lk < 0 || li >= b->n[0] || lj >= b->n[1] || lk >= b->n[2]) return -1;
  return (lk * b->n[1] + lj) * b->n[0] + li;
}

/* ------------------------------------------------------------------------- */
/* Quadratic B-spline axis stencil.
 * Restates BuildCheckedAxisStencil (native/src/sparse_mac_grid_3d.cc:266-310):
 * first node floor(X - shift - 1/2); outer weights from the distances to the
 * support edges, 0.5*d^2, centre weight 3/4 - c^2; normalized derivatives
 * {-d_right, -2c, d_left}; face offset (anchor - X)*h.                       */

typedef struct {
  int64_t first;
  double w[3];
  double dw[3];
  double off[3];
} axis_stencil;

static inline void build_axis(double X, double shift, double h, axis_stencil* s) {
  const double start_shift = shift + 0.5;
  s->first = (int64_t)floor(X - start_shift);
  const double a0 = (double)s->first + shift;
  const double dl = X - (a0 + 0.5);
  const double dr = fabs(X - (a0 + 1.5));
  const double c = X - (a0 + 1.0);
  s->w[0] = 0.5 * dr * dr;
  s->w[1] = 0.75 - c * c;
  s->w[2] = 0.5 * dl * dl;
  s->dw[0] = -dr;
  s->dw[1] = -2.0 * c;
  s->dw[2] = dl;
  for (int i = 0; i < 3; ++i) s->off[i] = ((double)(s->first + i) + shift - X) * h;
}

static inline void build_component(const double origin[3], double h, int axis, const double pos[3],
                                   axis_stencil st[3]) {
  for (int d = 0; d < 3; ++d) {
    const double X = (pos[d] - origin[d]) / h;
    build_axis(X, d == axis ? 0.0 : 0.5, h, &st[d]);
  }
}

/* Restates BuildMacFaceGeometryStencil3D (sparse_mac_grid_3d.cc:451-548): tensor
 * products in (z,y,x) order; gradient = derivative factor times the two other
 * weights, divided by h (PhysicalWeightGradient :312-336, normal range).      */
int fo_stencil(const double origin[3], double h, int axis, const double pos[3], int32_t* faces, double* values) {
  if (axis < 0 || axis > 2 || !(h > 0.0) || !isfinite(h)) return FO_INVALID;
  for (int d = 0; d < 3; ++d)
    if (!isfinite(pos[d])) return FO_INVALID;
  axis_stencil st[3];
  build_component(origin, h, axis, pos, st);
  int s = 0;
  for (int kz = 0; kz < 3; ++kz)
    for (int ky = 0; ky < 3; ++ky)
      for (int kx = 0; kx < 3; ++kx, ++s) {
        faces[4 * s] = axis;
        faces[4 * s + 1] = (int32_t)(st[0].first + kx);
        faces[4 * s + 2] = (int32_t)(st[1].first + ky);
        faces[4 * s + 3] = (int32_t)(st[2].first + kz);
        double* v = values + 7 * s;
        v[0] = st[0].w[kx] * st[1].w[ky] * st[2].w[kz];
        v[1] = st[0].off[kx];
        v[2] = st[1].off[ky];
        v[3] = st[2].off[kz];
        v[4] = st[0].dw[kx] * st[1].w[ky] * st[2].w[kz] / h;
        v[5] = st[0].w[kx] * st[1].dw[ky] * st[2].w[kz] / h;
        v[6] = st[0].w[kx] * st[1].w[ky] * st[2].dw[kz] / h;
      }
  return FO_OK;
}

/* ------------------------------------------------------------------------- */
/* P2G. Restates DepositMac3D / AccumulateMacParticleComponent
 * (native/src/transfers_3d.cc:56-104,139-145; mac_deposit_3d_internal.h:39-75):
 * mass = w*m; pure momentum = mass * (v_a + (C_a.x*r.x + C_a.y*r.y) + C_a.z*r.z). */

typedef void (*deposit_fn)(void* ctx, int axis, int64_t face, double mass, double momentum, int* status);

static int deposit_loop(const fo_box* b, const double* x, const double* v, const double* c, const double* mass,
                        int mass_stride, size_t np, deposit_fn fn, void* ctx) {
  for (size_t p = 0; p < np; ++p) {
    const double m = mass[mass_stride ? p : 0];
    if (!isfinite(m) || m < 0.0) return FO_INVALID;
    for (int q = 0; q < 3; ++q)
      if (!isfinite(v[3 * p + q])) return FO_INVALID;
    for (int q = 0; q < 9; ++q)
      if (!isfinite(c[9 * p + q])) return FO_INVALID;
  }
  for (size_t p = 0; p < np; ++p) {
    const double* pos = x + 3 * p;
    const double m = mass[mass_stride ? p : 0];
    for (int axis = 0; axis < 3; ++axis) {
      axis_stencil st[3];
      build_component(b->origin, b->h, axis, pos, st);
      const double va = v[3 * p + axis];
      const double* row = c + 9 * p + 3 * axis;
      for (int kz = 0; kz < 3; ++kz)
        for (int ky = 0; ky < 3; ++ky)
          for (int kx = 0; kx < 3; ++kx) {
            const int64_t f = face_at(b, axis, st[0].first + kx, st[1].first + ky, st[2].first + kz);
            if (f < 0) return FO_PRECONDITION;
            const double w = st[0].w[kx] * st[1].w[ky] * st[2].w[kz];
            const double mc = w * m;
            const double affine = (row[0] * st[0].off[kx] + row[1] * st[1].off[ky]) + row[2] * st[2].off[kz];
            const double mom = mc * (va + affine);
            int status = FO_OK;
            fn(ctx, axis, f, mc, mom, &status);
            if (status != FO_OK) return status;
          }
    }
  }
  return FO_OK;
}

typedef struct {
  double** mass;
  double** mom;
} dep_ctx;

static void dep_f64(void* vctx, int axis, int64_t f, double mc, double mom, int* status) {
  dep_ctx* ctx = (dep_ctx*)vctx;
  ctx->mass[axis][f] += mc;
  ctx->mom[axis][f] += mom;
  if (!isfinite(ctx->mass[axis][f]) || !isfinite(ctx->mom[axis][f])) *status = FO_RANGE;
}

int fo_p2g(const fo_box* b, const double* x, const double* v, const double* c, const double* mass, int mass_stride,
           size_t np, double* face_mass[3], double* face_momentum[3]) {
  for (int a = 0; a < 3; ++a) {
    memset(face_mass[a], 0, sizeof(double) * fo_face_count(b, a));
    memset(face_momentum[a], 0, sizeof(double) * fo_face_count(b, a));
  }
  dep_ctx ctx = {face_mass, face_momentum};
  return deposit_loop(b, x, v, c, mass, mass_stride, np, dep_f64, &ctx);
}

/* RoundNearestEven (transfers_3d.cc:44-54): truncate the magnitude, then resolve
 * the fraction and the parity of the integral part. */
static int64_t round_nearest_even(double s) {
  const double mag = fabs(s);
  const double integral = floor(mag);
  const double frac = mag - integral;
  int64_t q = (int64_t)integral;
  if (frac > 0.5 || (frac == 0.5 && (q % 2) != 0)) ++q;
  return s < 0.0 ? -q : q;
}

typedef struct {
  int64_t** mq;
  int64_t** pq;
  double ms, ps, limit;
} quanta_ctx;

static void dep_quanta(void* vctx, int axis, int64_t f, double mc, double mom, int* status) {
  quanta_ctx* ctx = (quanta_ctx*)vctx;
  const double sm = mc / ctx->ms, sp = mom / ctx->ps;
  if (!isfinite(sm) || fabs(sm) > ctx->limit || !isfinite(sp) || fabs(sp) > ctx->limit) {
    *status = FO_RANGE;
    return;
  }
  ctx->mq[axis][f] += round_nearest_even(sm);
  ctx->pq[axis][f] += round_nearest_even(sp);
}

/* DepositMacQuanta3D (transfers_3d.cc:147-197); the capacity bound uses np. */
int fo_p2g_quanta(const fo_box* b, const double* x, const double* v, const double* c, const double* mass,
                  int mass_stride, size_t np, double mass_per_quantum, double momentum_per_quantum,
                  int64_t* mass_q[3], int64_t* momentum_q[3]) {
  for (int a = 0; a < 3; ++a) {
    memset(mass_q[a], 0, sizeof(int64_t) * fo_face_count(b, a));
    memset(momentum_q[a], 0, sizeof(int64_t) * fo_face_count(b, a));
  }
  size_t cap = np < 1 ? 1 : np;
  int e = 0;
  while (((size_t)1 << e) < cap) ++e;
  quanta_ctx ctx = {mass_q, momentum_q, mass_per_quantum, momentum_per_quantum, ldexp(1.0, 62 - e)};
  return deposit_loop(b, x, v, c, mass, mass_stride, np, dep_quanta, &ctx);
}

/* NormalizeCore (native/src/liquid_boundary_transfer_3d.cc:462-515) followed by
 * ApplyForces (native/src/liquid_substep_3d_cpu.cc:156-178). */
void fo_normalize_forces(const fo_box* b, double* face_mass[3], double* face_momentum[3], double m_min, double dt,
                         const double g[3], double* u_pred[3], uint8_t* validity[3]) {
  for (int a = 0; a < 3; ++a) {
    const size_t nf = fo_face_count(b, a);
    for (size_t f = 0; f < nf; ++f) {
      const double m = face_mass[a][f];
      double u = 0.0;
      uint8_t valid = 0; /* LiquidFaceValidity3D: 0 missing, 1 valid, 3 low mass */
      if (m != 0.0) {
        if (m <= m_min) {
          valid = 3;
        } else {
          u = face_momentum[a][f] / m;
          valid = 1;
        }
      }
      if (validity) validity[a][f] = valid;
      u_pred[a][f] = u + dt * g[a];
    }
  }
}

/* ------------------------------------------------------------------------- */
/* G2P. Restates GatherMac3D / GatherMacVelocityComponentFromSlots
 * (transfers_3d.cc:199-261; mac_gather_3d_internal.h:15-69):
 * pic = sum w u_new; increment = pic - sum w u_old; fitted row = 4*sum(w u_new r/h)/h;
 * gradient row = sum grad(w) u_new.                                          */
int fo_g2p(const fo_box* b, const double* x, size_t np, double* u_old[3], double* u_new[3], double* out) {
  const double h = b->h;
  for (size_t p = 0; p < np; ++p) {
    const double* pos = x + 3 * p;
    double* o = out + 24 * p;
    for (int axis = 0; axis < 3; ++axis) {
      axis_stencil st[3];
      build_component(b->origin, h, axis, pos, st);
      double old_pic = 0.0, new_pic = 0.0, mom[3] = {0, 0, 0}, grad[3] = {0, 0, 0};
      for (int kz = 0; kz < 3; ++kz)
        for (int ky = 0; ky < 3; ++ky)
          for (int kx = 0; kx < 3; ++kx) {
            const int64_t f = face_at(b, axis, st[0].first + kx, st[1].first + ky, st[2].first + kz);
            if (f < 0) return FO_PRECONDITION;
            const double w = st[0].w[kx] * st[1].w[ky] * st[2].w[kz];
            const double uo = u_old ? u_old[axis][f] : 0.0;
            const double un = u_new[axis][f];
            const double wn = w * un;
            old_pic += w * uo;
            new_pic += wn;
            mom[0] += (st[0].off[kx] / h) * wn;
            mom[1] += (st[1].off[ky] / h) * wn;
            mom[2] += (st[2].off[kz] / h) * wn;
            grad[0] += (st[0].dw[kx] * st[1].w[ky] * st[2].w[kz] / h) * un;
            grad[1] += (st[0].w[kx] * st[1].dw[ky] * st[2].w[kz] / h) * un;
            grad[2] += (st[0].w[kx] * st[1].w[ky] * st[2].dw[kz] / h) * un;
          }
      o[axis] = new_pic;
      o[3 + axis] = new_pic - old_pic;
      for (int d = 0; d < 3; ++d) {
        o[6 + 3 * axis + d] = (4.0 * mom[d]) / h;
        o[15 + 3 * axis + d] = grad[d];
      }
      if (!isfinite(new_pic)) return FO_RANGE;
    }
  }
  return FO_OK;
}

/* ------------------------------------------------------------------------- */
/* Pressure. Restates the FP64 integrated system and evaluation of
 * native/src/mac_pressure_3d_arithmetic.h (CompensatedSum :57-74, FreezeCell
 * :110-146, FreezeLinkFromIncidence :174-245, AssembleIntegratedRhsInto :263-313,
 * SelectGaugesInto :328-399, ApplyOriginalPressureOperatorInto :404-436,
 * CorrectFacesAndAccumulatePhysicalDefectInto :440-503) and the evaluation and
 * gates of native/src/mac_pressure_workspace_3d.cc:399-461 and
 * native/src/mac_pressure_3d_multigrid.cc:431-465. The linear solve itself is an
 * FP64 Jacobi-preconditioned CG (the reference's aggregation-AMG PCG,
 * mac_pressure_workspace_3d.cc:462-659, is pinned separately through the
 * compiled reference at its own size caps).                                  */

typedef struct {
  double sum, corr;
} nsum;

static inline void nadd(nsum* s, double t) {
  const double next = s->sum + t;
  if (fabs(s->sum) >= fabs(t))
    s->corr += (s->sum - next) + t;
  else
    s->corr += (t - next) + s->sum;
  s->sum = next;
}
static inline double ntotal(const nsum* s) { return s->sum + s->corr; }

typedef struct {
  nsum flux, absolute;
} frow;
static inline void radd(frow* r, double t) {
  nadd(&r->flux, t);
  nadd(&r->absolute, fabs(t));
}

typedef struct {
  int64_t tail, head; /* -1 when exterior */
  int kind;
  double open_area, scale, conductance, predicted_u, wall_flux, lift;
} plink;

typedef struct {
  size_t nc, nf;
  double* volume;
  double* target_flux;
  double* wall_flux;
  double* compliance;
  double* previous;
  plink* links;
  double* rhs;
  double* rhs_abs;
  int64_t* component;
  uint8_t* pinned;
  size_t gauge_count;
} psystem;

static int cmp_cell(const int32_t* a, const int32_t* b) {
  if (a[2] != b[2]) return a[2] < b[2] ? -1 : 1;
  if (a[1] != b[1]) return a[1] < b[1] ? -1 : 1;
  if (a[0] != b[0]) return a[0] < b[0] ? -1 : 1;
  return 0;
}

static int64_t find_cell(const fo_pressure_inputs* in, int32_t x, int32_t y, int32_t z) {
  const int32_t key[3] = {x, y, z};
  size_t lo = 0, hi = in->nc;
  while (lo < hi) {
    const size_t mid = (lo + hi) / 2;
    const int c = cmp_cell(in->cell_index + 3 * mid, key);
    if (c == 0) return (int64_t)mid;
    if (c < 0)
      lo = mid + 1;
    else
      hi = mid;
  }
  return -1;
}

static int64_t find_root(int64_t* parent, int64_t c) {
  while (parent[c] != c) c = parent[c];
  return c;
}

static void psystem_free(psystem* s) {
  free(s->volume);
  free(s->target_flux);
  free(s->wall_flux);
  free(s->compliance);
  free(s->previous);
  free(s->links);
  free(s->rhs);
  free(s->rhs_abs);
  free(s->component);
  free(s->pinned);
}

static int psystem_build(const fo_pressure_inputs* in, psystem* s) {
  memset(s, 0, sizeof(*s));
  const size_t nc = in->nc, nf = in->nf;
  if (nc == 0) return FO_INVALID;
  s->nc = nc;
  s->nf = nf;
  s->volume = (double*)malloc(sizeof(double) * nc);
  s->target_flux = (double*)malloc(sizeof(double) * nc);
  s->wall_flux = (double*)malloc(sizeof(double) * nc);
  s->compliance = (double*)malloc(sizeof(double) * nc);
  s->previous = (double*)malloc(sizeof(double) * nc);
  s->links = (plink*)malloc(sizeof(plink) * (nf ? nf : 1));
  s->rhs = (double*)malloc(sizeof(double) * nc);
  s->rhs_abs = (double*)malloc(sizeof(double) * nc);
  s->component = (int64_t*)malloc(sizeof(int64_t) * nc);
  s->pinned = (uint8_t*)calloc(nc, 1);
  const double full_area = in->h * in->h;
  for (size_t i = 0; i < nc; ++i) {
    if (i > 0 && cmp_cell(in->cell_index + 3 * (i - 1), in->cell_index + 3 * i) >= 0) return FO_INVALID;
    const double* v = in->cell_values + 5 * i;
    s->volume[i] = v[0];
    s->target_flux[i] = v[0] * v[1];
    s->wall_flux[i] = v[4];
    s->compliance[i] = v[2] == 0.0 ? 0.0 : v[0] / (v[2] * in->dt);
    s->previous[i] = v[3];
  }
  for (size_t f = 0; f < nf; ++f) {
    const int32_t* fi = in->face_index + 4 * f;
    const double* v = in->face_values + 6 * f;
    plink* l = &s->links[f];
    int32_t t[3] = {fi[1], fi[2], fi[3]};
    t[fi[0]] -= 1;
    l->tail = find_cell(in, t[0], t[1], t[2]);
    l->head = find_cell(in, fi[1], fi[2], fi[3]);
    l->kind = in->face_kind[f];
    l->open_area = v[0];
    l->scale = 0.0;
    l->conductance = 0.0;
    if (v[0] > 0.0) {
      l->scale = (in->dt * v[1]) / v[2];
      l->conductance = v[0] * l->scale;
    }
    l->predicted_u = v[3];
    l->wall_flux = (full_area - v[0]) * v[4];
    l->lift = v[5];
    const int both = l->tail >= 0 && l->head >= 0;
    const int one = (l->tail >= 0) != (l->head >= 0);
    if (l->kind == 1 && !both) return FO_INVALID;
    if (l->kind == 2 && (!one || v[0] == 0.0)) return FO_INVALID;
    if (l->kind == 0 && v[0] != 0.0) return FO_INVALID;
  }
  /* AssembleIntegratedRhsInto */
  frow* rows = (frow*)calloc(nc, sizeof(frow));
  for (size_t i = 0; i < nc; ++i) {
    radd(&rows[i], s->target_flux[i]);
    radd(&rows[i], s->wall_flux[i]);
    radd(&rows[i], s->compliance[i] * s->previous[i]);
  }
  for (size_t f = 0; f < nf; ++f) {
    const plink* l = &s->links[f];
    const double fluid_flux = l->open_area * l->predicted_u;
    if (l->tail >= 0) {
      radd(&rows[l->tail], -1.0 * fluid_flux);
      radd(&rows[l->tail], -1.0 * l->wall_flux);
    }
    if (l->head >= 0) {
      radd(&rows[l->head], 1.0 * fluid_flux);
      radd(&rows[l->head], 1.0 * l->wall_flux);
    }
    if (l->kind == 1) {
      const double jf = l->conductance * l->lift;
      if (l->tail >= 0) radd(&rows[l->tail], -1.0 * jf);
      if (l->head >= 0) radd(&rows[l->head], 1.0 * jf);
    } else if (l->kind == 2) {
      const double ef = l->conductance * l->lift;
      if (l->tail >= 0) radd(&rows[l->tail], ef);
      if (l->head >= 0) radd(&rows[l->head], ef);
    }
  }
  for (size_t i = 0; i < nc; ++i) {
    s->rhs[i] = ntotal(&rows[i].flux);
    s->rhs_abs[i] = ntotal(&rows[i].absolute);
  }
  free(rows);
  /* SelectGaugesInto */
  for (size_t i = 0; i < nc; ++i) s->component[i] = (int64_t)i;
  for (size_t f = 0; f < nf; ++f) {
    const plink* l = &s->links[f];
    if (l->conductance > 0.0 && l->tail >= 0 && l->head >= 0) {
      const int64_t a = find_root(s->component, l->tail), b = find_root(s->component, l->head);
      s->component[a > b ? a : b] = a < b ? a : b;
    }
  }
  uint8_t* anchored = (uint8_t*)calloc(nc, 1);
  frow* bal = (frow*)calloc(nc, sizeof(frow));
  for (size_t i = 0; i < nc; ++i) {
    s->component[i] = find_root(s->component, (int64_t)i);
    if (s->compliance[i] > 0.0) anchored[s->component[i]] = 1;
  }
  for (size_t f = 0; f < nf; ++f) {
    const plink* l = &s->links[f];
    if (l->kind == 2) {
      if (l->tail >= 0) anchored[s->component[l->tail]] = 1;
      if (l->head >= 0) anchored[s->component[l->head]] = 1;
    }
  }
  for (size_t i = 0; i < nc; ++i) {
    if (!anchored[s->component[i]]) {
      radd(&bal[s->component[i]], s->target_flux[i]);
      radd(&bal[s->component[i]], s->wall_flux[i]);
    }
  }
  for (size_t f = 0; f < nf; ++f) {
    const plink* l = &s->links[f];
    if (l->tail >= 0 && l->head >= 0 && s->component[l->tail] == s->component[l->head]) continue;
    if (l->tail >= 0 && !anchored[s->component[l->tail]]) radd(&bal[s->component[l->tail]], -1.0 * l->wall_flux);
    if (l->head >= 0 && !anchored[s->component[l->head]]) radd(&bal[s->component[l->head]], 1.0 * l->wall_flux);
  }
  int status = FO_OK;
  for (size_t i = 0; i < nc; ++i) {
    if (s->component[i] != (int64_t)i || anchored[i]) continue;
    const double pb = ntotal(&bal[i].flux), ab = ntotal(&bal[i].absolute);
    if (fabs(pb) > 32.0 * DBL_EPSILON * ab) status = FO_PRECONDITION;
    s->pinned[i] = 1;
    s->gauge_count++;
  }
  free(anchored);
  free(bal);
  return status;
}

/* ApplyOriginalPressureOperatorInto, plain FP64 (used inside the solver). */
static void papply(const psystem* s, const double* p, double* out) {
  for (size_t i = 0; i < s->nc; ++i) out[i] = s->compliance[i] * p[i];
  for (size_t f = 0; f < s->nf; ++f) {
    const plink* l = &s->links[f];
    if (l->conductance == 0.0) continue;
    const double pt = l->tail >= 0 ? p[l->tail] : 0.0, ph = l->head >= 0 ? p[l->head] : 0.0;
    const double flux = l->conductance * (pt - ph);
    if (l->tail >= 0) out[l->tail] += flux;
    if (l->head >= 0) out[l->head] -= flux;
  }
}

static int pevaluate(const psystem* s, const double* p, double* residual, double* defect, double* corrected_u,
                     fo_pressure_diag* diag) {
  const size_t nc = s->nc;
  frow* op = (frow*)calloc(nc, sizeof(frow));
  frow* ph = (frow*)calloc(nc, sizeof(frow));
  for (size_t i = 0; i < nc; ++i) radd(&op[i], s->compliance[i] * p[i]);
  for (size_t f = 0; f < s->nf; ++f) {
    const plink* l = &s->links[f];
    if (l->conductance == 0.0) continue;
    const double pt = l->tail >= 0 ? p[l->tail] : 0.0, phd = l->head >= 0 ? p[l->head] : 0.0;
    const double flux = l->conductance * (pt - phd);
    if (l->tail >= 0) radd(&op[l->tail], flux);
    if (l->head >= 0) radd(&op[l->head], -flux);
  }
  for (size_t i = 0; i < nc; ++i) {
    radd(&ph[i], -s->target_flux[i]);
    radd(&ph[i], -s->wall_flux[i]);
    if (s->compliance[i] > 0.0) radd(&ph[i], s->compliance[i] * (p[i] - s->previous[i]));
  }
  for (size_t f = 0; f < s->nf; ++f) {
    const plink* l = &s->links[f];
    double u = l->predicted_u;
    if (l->open_area > 0.0) {
      const double ext = l->kind == 2 ? l->lift : 0.0;
      const double jump = l->kind == 1 ? l->lift : 0.0;
      const double pt = l->tail >= 0 ? p[l->tail] : ext, phd = l->head >= 0 ? p[l->head] : ext;
      u += l->scale * (pt - phd + jump);
    }
    if (!isfinite(u)) {
      free(op);
      free(ph);
      return FO_RANGE;
    }
    if (corrected_u) corrected_u[f] = u;
    const double flux = l->open_area * u;
    if (l->tail >= 0) {
      radd(&ph[l->tail], flux);
      radd(&ph[l->tail], l->wall_flux);
    }
    if (l->head >= 0) {
      radd(&ph[l->head], -flux);
      radd(&ph[l->head], -l->wall_flux);
    }
  }
  double l2 = 0.0, maxr = 0.0, maxd = 0.0, bl2 = 0.0;
  int status = FO_OK;
  for (size_t i = 0; i < nc; ++i) {
    const double r = s->rhs[i] - ntotal(&op[i].flux);
    const double d = ntotal(&ph[i].flux) / s->volume[i];
    const double ident = s->volume[i] * d + r;
    const double absterms = s->rhs_abs[i] + ntotal(&op[i].absolute) + ntotal(&ph[i].absolute);
    if (fabs(ident) > 64.0 * DBL_EPSILON * absterms) status = FO_INTERNAL;
    if (residual) residual[i] = r;
    if (defect) defect[i] = d;
    l2 = hypot(l2, r);
    bl2 = hypot(bl2, s->rhs[i]);
    if (fabs(r) / s->volume[i] > maxr) maxr = fabs(r) / s->volume[i];
    if (fabs(d) > maxd) maxd = fabs(d);
  }
  free(op);
  free(ph);
  if (diag) {
    diag->true_residual_l2 = l2;
    diag->max_volume_scaled_residual = maxr;
    diag->max_defect = maxd;
    diag->rhs_l2 = bl2;
    diag->gauge_count = (double)s->gauge_count;
  }
  return status;
}

int fo_pressure_evaluate(const fo_pressure_inputs* in, const double* pressure, double* residual, double* defect,
                         double* rhs, double* corrected_u, fo_pressure_diag* diag) {
  psystem s;
  int st = psystem_build(in, &s);
  if (st != FO_OK) {
    psystem_free(&s);
    return st;
  }
  if (rhs) memcpy(rhs, s.rhs, sizeof(double) * s.nc);
  st = pevaluate(&s, pressure, residual, defect, corrected_u, diag);
  psystem_free(&s);
  return st;
}

int fo_pressure_solve(const fo_pressure_inputs* in, double rel_tol, size_t max_iterations, double* pressure,
                      double* residual, double* defect, double* rhs, double* corrected_u, fo_pressure_diag* diag) {
  psystem s;
  int st = psystem_build(in, &s);
  if (st != FO_OK) {
    psystem_free(&s);
    return st;
  }
  const size_t nc = s.nc;
  if (rhs) memcpy(rhs, s.rhs, sizeof(double) * nc);
  /* Warm start: previous pressure, shifted by the pin's previous pressure on
   * unanchored components (InitializeMacPressure3D, mac_pressure_3d_multigrid.cc:401-419). */
  double* pin_prev = (double*)calloc(nc, sizeof(double));
  for (size_t i = 0; i < nc; ++i)
    if (s.pinned[i]) pin_prev[s.component[i]] = s.previous[i];
  for (size_t i = 0; i < nc; ++i) pressure[i] = s.previous[i] - pin_prev[s.component[i]];
  free(pin_prev);
  double* diagA = (double*)calloc(nc, sizeof(double));
  for (size_t i = 0; i < nc; ++i) diagA[i] = s.compliance[i];
  for (size_t f = 0; f < s.nf; ++f) {
    const plink* l = &s.links[f];
    if (l->tail >= 0) diagA[l->tail] += l->conductance;
    if (l->head >= 0) diagA[l->head] += l->conductance;
  }
  double* r = (double*)malloc(sizeof(double) * nc);
  double* z = (double*)malloc(sizeof(double) * nc);
  double* d = (double*)malloc(sizeof(double) * nc);
  double* q = (double*)malloc(sizeof(double) * nc);
  papply(&s, pressure, q);
  double bnorm = 0.0;
  for (size_t i = 0; i < nc; ++i) {
    r[i] = s.pinned[i] ? 0.0 : s.rhs[i] - q[i];
    bnorm = hypot(bnorm, s.rhs[i]);
  }
  const double limit = rel_tol > 0.0 ? rel_tol * bnorm : 2e-6 + 2e-6 * bnorm;
  double rz_prev = 0.0;
  size_t it = 0;
  for (; it < max_iterations; ++it) {
    double rn = 0.0;
    for (size_t i = 0; i < nc; ++i) rn = hypot(rn, r[i]);
    if (rn <= limit) break;
    double rz = 0.0;
    for (size_t i = 0; i < nc; ++i) {
      z[i] = (s.pinned[i] || diagA[i] == 0.0) ? 0.0 : r[i] / diagA[i];
      rz += r[i] * z[i];
    }
    if (it == 0) {
      memcpy(d, z, sizeof(double) * nc);
    } else {
      const double beta = rz / rz_prev;
      for (size_t i = 0; i < nc; ++i) d[i] = z[i] + beta * d[i];
    }
    papply(&s, d, q);
    double dq = 0.0;
    for (size_t i = 0; i < nc; ++i) {
      if (s.pinned[i]) q[i] = 0.0;
      dq += d[i] * q[i];
    }
    if (!(dq > 0.0)) {
      st = FO_ABORTED;
      break;
    }
    const double alpha = rz / dq;
    for (size_t i = 0; i < nc; ++i) {
      pressure[i] += alpha * d[i];
      r[i] -= alpha * q[i];
    }
    rz_prev = rz;
  }
  free(diagA);
  free(r);
  free(z);
  free(d);
  free(q);
  fo_pressure_diag local;
  int est = pevaluate(&s, pressure, residual, defect, corrected_u, &local);
  local.iterations = (double)it;
  if (diag) *diag = local;
  if (st == FO_OK) st = est;
  if (st == FO_OK && local.true_residual_l2 > limit * 1.000001 + 1e-300) st = FO_ABORTED;
  psystem_free(&s);
  return st;
}

/* ------------------------------------------------------------------------- */
/* Box scene: one-cell solid walls on the box boundary; fluid = occupied cell. */

void fo_classify_cells(const fo_box* b, const double* x, size_t np, uint8_t* type) {
  const size_t ncell = (size_t)b->n[0] * b->n[1] * b->n[2];
  for (int64_t k = 0; k < b->n[2]; ++k)
    for (int64_t j = 0; j < b->n[1]; ++j)
      for (int64_t i = 0; i < b->n[0]; ++i) {
        const int wall = i == 0 || j == 0 || k == 0 || i == b->n[0] - 1 || j == b->n[1] - 1 || k == b->n[2] - 1;
        type[(k * b->n[1] + j) * b->n[0] + i] = wall ? 0 : 2;
      }
  (void)ncell;
  for (size_t p = 0; p < np; ++p) {
    int64_t c[3];
    for (int d = 0; d < 3; ++d) c[d] = (int64_t)floor((x[3 * p + d] - b->origin[d]) / b->h);
    const int64_t id = cell_at(b, c[0], c[1], c[2]);
    if (id >= 0 && type[id] == 2) type[id] = 1;
  }
}

/* Pressure inputs for the box scene: fluid cells (z,y,x order) and every face
 * incident to one, sealed against solid cells, Dirichlet p=0 at distance h
 * against air, internal between fluid cells. */
typedef struct {
  size_t nc, nf;
  int32_t* cell_index;
  double* cell_values;
  int32_t* face_index;
  int32_t* face_kind;
  double* face_values;
  int64_t* face_dense; /* dense face index per pressure face */
  int64_t* cell_dense;
} box_pressure;

static void box_pressure_free(box_pressure* bp) {
  free(bp->cell_index);
  free(bp->cell_values);
  free(bp->face_index);
  free(bp->face_kind);
  free(bp->face_values);
  free(bp->face_dense);
  free(bp->cell_dense);
}

static void box_pressure_build(const fo_box* b, const uint8_t* type, double* u_pred[3], double density,
                               box_pressure* bp) {
  const int64_t nx = b->n[0], ny = b->n[1], nz = b->n[2];
  const double h = b->h;
  size_t nc = 0;
  for (int64_t c = 0; c < nx * ny * nz; ++c) nc += type[c] == 1;
  bp->nc = nc;
  bp->cell_index = (int32_t*)malloc(sizeof(int32_t) * 3 * (nc + 1));
  bp->cell_values = (double*)malloc(sizeof(double) * 5 * (nc + 1));
  bp->cell_dense = (int64_t*)malloc(sizeof(int64_t) * (nc + 1));
  size_t w = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        const int64_t c = (k * ny + j) * nx + i;
        if (type[c] != 1) continue;
        bp->cell_index[3 * w] = (int32_t)(i + b->lo[0]);
        bp->cell_index[3 * w + 1] = (int32_t)(j + b->lo[1]);
        bp->cell_index[3 * w + 2] = (int32_t)(k + b->lo[2]);
        double* v = bp->cell_values + 5 * w;
        v[0] = h * h * h;
        v[1] = 0.0;
        v[2] = 0.0;
        v[3] = 0.0;
        v[4] = 0.0;
        bp->cell_dense[w] = c;
        ++w;
      }
  /* faces: walk axes; a face is incident when either side is fluid */
  size_t cap = 6 * nc + 1;
  bp->face_index = (int32_t*)malloc(sizeof(int32_t) * 4 * cap);
  bp->face_kind = (int32_t*)malloc(sizeof(int32_t) * cap);
  bp->face_values = (double*)malloc(sizeof(double) * 6 * cap);
  bp->face_dense = (int64_t*)malloc(sizeof(int64_t) * cap);
  size_t nf = 0;
  for (int axis = 0; axis < 3; ++axis) {
    const int64_t fx = face_dim(b, axis, 0), fy = face_dim(b, axis, 1), fz = face_dim(b, axis, 2);
    for (int64_t k = 0; k < fz; ++k)
      for (int64_t j = 0; j < fy; ++j)
        for (int64_t i = 0; i < fx; ++i) {
          int64_t t[3] = {i, j, k};
          t[axis] -= 1;
          const int64_t head = cell_at(b, i + b->lo[0], j + b->lo[1], k + b->lo[2]);
          const int64_t tail = cell_at(b, t[0] + b->lo[0], t[1] + b->lo[1], t[2] + b->lo[2]);
          const int ht = head >= 0 ? type[head] : 0, tt = tail >= 0 ? type[tail] : 0;
          if (ht != 1 && tt != 1) continue;
          const int64_t f = (k * fy + j) * fx + i;
          int32_t* fi = bp->face_index + 4 * nf;
          fi[0] = axis;
          fi[1] = (int32_t)(i + b->lo[0]);
          fi[2] = (int32_t)(j + b->lo[1]);
          fi[3] = (int32_t)(k + b->lo[2]);
          double* v = bp->face_values + 6 * nf;
          const int other = ht == 1 ? tt : ht;
          if (other == 0) {
            bp->face_kind[nf] = 0;
            v[0] = 0.0;
            v[1] = 0.0;
            v[2] = 0.0;
          } else {
            bp->face_kind[nf] = other == 1 ? 1 : 2;
            v[0] = h * h;
            v[1] = 1.0 / density;
            v[2] = h;
          }
          v[3] = u_pred[axis][f];
          v[4] = 0.0;
          v[5] = 0.0;
          bp->face_dense[nf] = f;
          ++nf;
        }
  }
  bp->nf = nf;
}

/* Zero the predicted velocity on faces touching a solid cell (stationary walls). */
static void apply_wall_bc(const fo_box* b, const uint8_t* type, double* u[3]) {
  for (int axis = 0; axis < 3; ++axis) {
    const int64_t fx = face_dim(b, axis, 0), fy = face_dim(b, axis, 1), fz = face_dim(b, axis, 2);
    for (int64_t k = 0; k < fz; ++k)
      for (int64_t j = 0; j < fy; ++j)
        for (int64_t i = 0; i < fx; ++i) {
          int64_t t[3] = {i, j, k};
          t[axis] -= 1;
          const int64_t head = cell_at(b, i + b->lo[0], j + b->lo[1], k + b->lo[2]);
          const int64_t tail = cell_at(b, t[0] + b->lo[0], t[1] + b->lo[1], t[2] + b->lo[2]);
          const int ht = head >= 0 ? type[head] : 0, tt = tail >= 0 ? type[tail] : 0;
          if (ht == 0 || tt == 0) u[axis][(k * fy + j) * fx + i] = 0.0;
        }
  }
}

int fo_step(const fo_box* b, const fo_step_params* prm, double* x, double* v, double* c, size_t np, double* u_pred[3],
            double* u_new[3], double* cell_pressure, uint8_t* type, fo_pressure_diag* diag) {
  const double h = b->h;
  const double pmass = prm->density * h * h * h / 8.0;
  double* fm[3];
  double* fq[3];
  for (int a = 0; a < 3; ++a) {
    const size_t nf = fo_face_count(b, a);
    fm[a] = (double*)malloc(sizeof(double) * nf);
    fq[a] = (double*)malloc(sizeof(double) * nf);
  }
  int st = fo_p2g(b, x, v, c, &pmass, 0, np, fm, fq);
  if (st == FO_OK) {
    fo_normalize_forces(b, fm, fq, prm->m_min, prm->dt, prm->gravity, u_pred, NULL);
    fo_classify_cells(b, x, np, type);
    apply_wall_bc(b, type, u_pred);
    for (int a = 0; a < 3; ++a) memcpy(u_new[a], u_pred[a], sizeof(double) * fo_face_count(b, a));
    box_pressure bp;
    box_pressure_build(b, type, u_pred, prm->density, &bp);
    const size_t ncell = (size_t)b->n[0] * b->n[1] * b->n[2];
    if (cell_pressure) memset(cell_pressure, 0, sizeof(double) * ncell);
    if (bp.nc > 0) {
      fo_pressure_inputs in = {bp.nc, bp.nf, bp.cell_index, bp.cell_values, bp.face_index, bp.face_kind,
                               bp.face_values, h, prm->dt};
      double* p = (double*)malloc(sizeof(double) * bp.nc);
      double* uc = (double*)malloc(sizeof(double) * bp.nf);
      st = fo_pressure_solve(&in, prm->rel_tol, prm->max_iterations, p, NULL, NULL, NULL, uc, diag);
      for (size_t f = 0; f < bp.nf; ++f) u_new[bp.face_index[4 * f]][bp.face_dense[f]] = uc[f];
      if (cell_pressure)
        for (size_t i = 0; i < bp.nc; ++i) cell_pressure[bp.cell_dense[i]] = p[i];
      free(p);
      free(uc);
    }
    box_pressure_free(&bp);
  }
  if (st == FO_OK) {
    double* g = (double*)malloc(sizeof(double) * 24 * (np ? np : 1));
    st = fo_g2p(b, x, np, NULL, u_new, g);
    if (st == FO_OK) {
      const double lo_clamp[3] = {b->origin[0] + (b->lo[0] + 1) * h + prm->clamp_margin * h,
                                  b->origin[1] + (b->lo[1] + 1) * h + prm->clamp_margin * h,
                                  b->origin[2] + (b->lo[2] + 1) * h + prm->clamp_margin * h};
      const double hi_clamp[3] = {b->origin[0] + (b->lo[0] + b->n[0] - 1) * h - prm->clamp_margin * h,
                                  b->origin[1] + (b->lo[1] + b->n[1] - 1) * h - prm->clamp_margin * h,
                                  b->origin[2] + (b->lo[2] + b->n[2] - 1) * h - prm->clamp_margin * h};
      for (size_t p = 0; p < np; ++p) {
        const double* o = g + 24 * p;
        for (int d = 0; d < 3; ++d) {
          v[3 * p + d] = o[d];
          double nx = x[3 * p + d] + prm->dt * o[d];
          if (nx < lo_clamp[d]) nx = lo_clamp[d];
          if (nx > hi_clamp[d]) nx = hi_clamp[d];
          x[3 * p + d] = nx;
        }
        for (int q = 0; q < 9; ++q) c[9 * p + q] = o[6 + q];
      }
    }
    free(g);
  }
  for (int a = 0; a < 3; ++a) {
    free(fm[a]);
    free(fq[a]);
  }
  return st;
}

/* ------------------------------------------------------------------------- */
/* Geometric V-cycle restatement (no reference counterpart: the reference uses
 * aggregation AMG with weighted Jacobi). Mirrors the CUDA preconditioner.
 * Level 0 (units of the full-face conductance): k = 1 on faces between two
 * fluid cells, anchor = number of air neighbours (Dirichlet p = 0), solid
 * neighbours contribute nothing. Level l+1 aggregates 2x2x2 cells: fluid if
 * any child is fluid, anchor = 0.8 * (sum of child anchors), the low-face
 * coefficient = (sum of the four crossing fine coefficients)/2; diag = anchor
 * + the six face coefficients. Red-black Gauss-Seidel (red = even global
 * parity), `pre` sweeps red->black, restriction sums fluid-child residuals,
 * piecewise-constant prolongation, `post` sweeps black->red; the coarsest level
 * runs `coarse_sweeps` forward and `coarse_sweeps` backward sweeps from zero. */

#define FO_COARSE_ANCHOR_SCALE 0.8

typedef struct {
  int64_t n[3];
  uint8_t* fluid;
  double* k[3];
  double* anchor;
  double* diag;
  double* x;
  double* b;
} mg_level;

static inline int64_t mg_id(const mg_level* L, int64_t i, int64_t j, int64_t k) {
  if (i < 0 || j < 0 || k < 0 || i >= L->n[0] || j >= L->n[1] || k >= L->n[2]) return -1;
  return (k * L->n[1] + j) * L->n[0] + i;
}

/* sum over the 6 faces of k_f * x_j for fluid neighbours */
static double mg_offdiag(const mg_level* L, int64_t i, int64_t j, int64_t k, const double* x) {
  const int64_t id = mg_id(L, i, j, k);
  double s = 0.0;
  const int64_t c[3] = {i, j, k};
  for (int a = 0; a < 3; ++a) {
    int64_t lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
    lo[a] -= 1;
    hi[a] += 1;
    const int64_t jl = mg_id(L, lo[0], lo[1], lo[2]), jh = mg_id(L, hi[0], hi[1], hi[2]);
    if (jl >= 0 && L->k[a][id] != 0.0) s += L->k[a][id] * x[jl];
    if (jh >= 0 && L->k[a][jh] != 0.0) s += L->k[a][jh] * x[jh];
  }
  return s;
}

static void mg_sweep(mg_level* L, int color, int first) {
  for (int64_t k = 0; k < L->n[2]; ++k)
    for (int64_t j = 0; j < L->n[1]; ++j)
      for (int64_t i = 0; i < L->n[0]; ++i) {
        if (((i + j + k) & 1) != color) continue;
        const int64_t id = mg_id(L, i, j, k);
        if (!L->fluid[id]) continue;
        const double s = L->b[id] + (first ? 0.0 : mg_offdiag(L, i, j, k, L->x));
        L->x[id] = s / L->diag[id];
      }
}

static void mg_vcycle(mg_level* Ls, int l, int levels, int pre, int post, int coarse_sweeps) {
  mg_level* L = &Ls[l];
  const size_t nc = (size_t)(L->n[0] * L->n[1] * L->n[2]);
  memset(L->x, 0, sizeof(double) * nc);
  if (l == levels - 1) {
    for (int s = 0; s < coarse_sweeps; ++s) {
      mg_sweep(L, 0, 0);
      mg_sweep(L, 1, 0);
    }
    for (int s = 0; s < coarse_sweeps; ++s) {
      mg_sweep(L, 1, 0);
      mg_sweep(L, 0, 0);
    }
    return;
  }
  for (int s = 0; s < pre; ++s) {
    mg_sweep(L, 0, s == 0);
    mg_sweep(L, 1, 0);
  }
  mg_level* C = &Ls[l + 1];
  memset(C->b, 0, sizeof(double) * (size_t)(C->n[0] * C->n[1] * C->n[2]));
  for (int64_t k = 0; k < L->n[2]; ++k)
    for (int64_t j = 0; j < L->n[1]; ++j)
      for (int64_t i = 0; i < L->n[0]; ++i) {
        const int64_t id = mg_id(L, i, j, k);
        if (!L->fluid[id]) continue;
        const double r = L->b[id] - (L->diag[id] * L->x[id] - mg_offdiag(L, i, j, k, L->x));
        C->b[mg_id(C, i / 2, j / 2, k / 2)] += r;
      }
  mg_vcycle(Ls, l + 1, levels, pre, post, coarse_sweeps);
  for (int64_t k = 0; k < L->n[2]; ++k)
    for (int64_t j = 0; j < L->n[1]; ++j)
      for (int64_t i = 0; i < L->n[0]; ++i) {
        const int64_t id = mg_id(L, i, j, k);
        if (L->fluid[id]) L->x[id] += C->x[mg_id(C, i / 2, j / 2, k / 2)];
      }
  for (int s = 0; s < post; ++s) {
    mg_sweep(L, 1, 0);
    mg_sweep(L, 0, 0);
  }
}

static void mg_finish_diag(mg_level* L) {
  for (int64_t k = 0; k < L->n[2]; ++k)
    for (int64_t j = 0; j < L->n[1]; ++j)
      for (int64_t i = 0; i < L->n[0]; ++i) {
        const int64_t id = mg_id(L, i, j, k);
        double d = L->anchor[id];
        const int64_t c[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) {
          int64_t hi[3] = {c[0], c[1], c[2]};
          hi[a] += 1;
          const int64_t jh = mg_id(L, hi[0], hi[1], hi[2]);
          d += L->k[a][id];
          if (jh >= 0) d += L->k[a][jh];
        }
        L->diag[id] = L->fluid[id] ? d : 1.0;
      }
}

int fo_vcycle(const fo_box* b, const uint8_t* cell_type, int levels, int pre, int post, int coarse_sweeps,
              const double* r, double* z) {
  if (levels < 1 || levels > 8 || pre < 1 || post < 1) return FO_INVALID;
  mg_level Ls[8];
  for (int l = 0; l < levels; ++l) {
    for (int d = 0; d < 3; ++d) Ls[l].n[d] = l == 0 ? b->n[d] : (Ls[l - 1].n[d] + 1) / 2;
    const size_t nc = (size_t)(Ls[l].n[0] * Ls[l].n[1] * Ls[l].n[2]);
    Ls[l].fluid = (uint8_t*)calloc(nc, 1);
    for (int a = 0; a < 3; ++a) Ls[l].k[a] = (double*)calloc(nc, sizeof(double));
    Ls[l].anchor = (double*)calloc(nc, sizeof(double));
    Ls[l].diag = (double*)calloc(nc, sizeof(double));
    Ls[l].x = (double*)calloc(nc, sizeof(double));
    Ls[l].b = (double*)calloc(nc, sizeof(double));
  }
  mg_level* L0 = &Ls[0];
  for (int64_t k = 0; k < L0->n[2]; ++k)
    for (int64_t j = 0; j < L0->n[1]; ++j)
      for (int64_t i = 0; i < L0->n[0]; ++i) {
        const int64_t id = mg_id(L0, i, j, k);
        const int fl = cell_type[id] == 1;
        L0->fluid[id] = (uint8_t)fl;
        if (!fl) continue;
        const int64_t c[3] = {i, j, k};
        double anchor = 0.0;
        for (int a = 0; a < 3; ++a) {
          int64_t lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
          lo[a] -= 1;
          hi[a] += 1;
          const int64_t jl = mg_id(L0, lo[0], lo[1], lo[2]), jh = mg_id(L0, hi[0], hi[1], hi[2]);
          const int tl = jl >= 0 ? cell_type[jl] : 0, th = jh >= 0 ? cell_type[jh] : 0;
          L0->k[a][id] = tl == 1 ? 1.0 : 0.0;
          anchor += (tl == 2) + (th == 2);
        }
        L0->anchor[id] = anchor;
      }
  mg_finish_diag(L0);
  for (int l = 1; l < levels; ++l) {
    mg_level* F = &Ls[l - 1];
    mg_level* C = &Ls[l];
    for (int64_t k = 0; k < F->n[2]; ++k)
      for (int64_t j = 0; j < F->n[1]; ++j)
        for (int64_t i = 0; i < F->n[0]; ++i) {
          const int64_t fid = mg_id(F, i, j, k), cid = mg_id(C, i / 2, j / 2, k / 2);
          if (F->fluid[fid]) C->fluid[cid] = 1;
          C->anchor[cid] += FO_COARSE_ANCHOR_SCALE * F->anchor[fid];
          const int64_t c[3] = {i, j, k};
          for (int a = 0; a < 3; ++a)
            if ((c[a] & 1) == 0) C->k[a][cid] += 0.5 * F->k[a][fid];
        }
    mg_finish_diag(C);
  }
  const size_t n0 = (size_t)(L0->n[0] * L0->n[1] * L0->n[2]);
  for (size_t i = 0; i < n0; ++i) L0->b[i] = L0->fluid[i] ? r[i] : 0.0;
  mg_vcycle(Ls, 0, levels, pre, post, coarse_sweeps);
  for (size_t i = 0; i < n0; ++i) z[i] = L0->fluid[i] ? L0->x[i] : 0.0;
  for (int l = 0; l < levels; ++l) {
    free(Ls[l].fluid);
    for (int a = 0; a < 3; ++a) free(Ls[l].k[a]);
    free(Ls[l].anchor);
    free(Ls[l].diag);
    free(Ls[l].x);
    free(Ls[l].b);
  }
  return FO_OK;
}

/* ------------------------------------------------------------------------- */
/* Replay of one device step at full size: fo_step with the pressure given
 * instead of solved. Reads the state as FP32 SoA (15 x np floats: x[3], v[3],
 * C rows[9]) and works in FP64: P2G over every particle (in chunks), normalize
 * + gravity, stationary walls, the box system of the resulting predicted
 * velocities, its FP64 evaluation at `cell_pressure` (dense over the box:
 * corrected faces into u_new, the true residual into diag), then G2P and
 * advection for the sampled particles p = first, first + stride, ...; each
 * sampled particle gets 15 doubles in `sample_out` (x, v, C rows after the
 * step). */
int fo_step_replay(const fo_box* b, const fo_step_params* prm, const float* soa, size_t np, const double* cell_pressure,
                   size_t first, size_t stride, double* u_pred[3], double* u_new[3], uint8_t* type,
                   fo_pressure_diag* diag, double* sample_out) {
  const double h = b->h;
  const double pmass = prm->density * h * h * h / 8.0;
  const size_t chunk = (size_t)1 << 20;
  double* fm[3];
  double* fq[3];
  for (int a = 0; a < 3; ++a) {
    const size_t nf = fo_face_count(b, a);
    fm[a] = (double*)calloc(nf, sizeof(double));
    fq[a] = (double*)calloc(nf, sizeof(double));
  }
  double* cx = (double*)malloc(sizeof(double) * 3 * chunk);
  double* cv = (double*)malloc(sizeof(double) * 3 * chunk);
  double* cc = (double*)malloc(sizeof(double) * 9 * chunk);
  double* g = (double*)malloc(sizeof(double) * 24 * chunk);
  dep_ctx dctx = {fm, fq};
  int st = FO_OK;
  for (size_t p0 = 0; p0 < np && st == FO_OK; p0 += chunk) {
    const size_t m = np - p0 < chunk ? np - p0 : chunk;
    for (size_t p = 0; p < m; ++p) {
      for (int d = 0; d < 3; ++d) {
        cx[3 * p + d] = soa[(size_t)d * np + p0 + p];
        cv[3 * p + d] = soa[(size_t)(3 + d) * np + p0 + p];
      }
      for (int q = 0; q < 9; ++q) cc[9 * p + q] = soa[(size_t)(6 + q) * np + p0 + p];
    }
    st = deposit_loop(b, cx, cv, cc, &pmass, 0, m, dep_f64, &dctx);
  }
  /* cell classification from FP64 positions, as fo_classify_cells does */
  if (st == FO_OK) {
    fo_classify_cells(b, NULL, 0, type);
    for (size_t p = 0; p < np; ++p) {
      int64_t c[3];
      for (int d = 0; d < 3; ++d) c[d] = (int64_t)floor(((double)soa[(size_t)d * np + p] - b->origin[d]) / b->h);
      const int64_t id = cell_at(b, c[0], c[1], c[2]);
      if (id >= 0 && type[id] == 2) type[id] = 1;
    }
    fo_normalize_forces(b, fm, fq, prm->m_min, prm->dt, prm->gravity, u_pred, NULL);
    apply_wall_bc(b, type, u_pred);
    for (int a = 0; a < 3; ++a) memcpy(u_new[a], u_pred[a], sizeof(double) * fo_face_count(b, a));
    box_pressure bp;
    box_pressure_build(b, type, u_pred, prm->density, &bp);
    if (bp.nc > 0) {
      fo_pressure_inputs in = {bp.nc, bp.nf, bp.cell_index, bp.cell_values, bp.face_index, bp.face_kind,
                               bp.face_values, h, prm->dt};
      double* p = (double*)malloc(sizeof(double) * bp.nc);
      double* uc = (double*)malloc(sizeof(double) * bp.nf);
      for (size_t i = 0; i < bp.nc; ++i) p[i] = cell_pressure[bp.cell_dense[i]];
      st = fo_pressure_evaluate(&in, p, NULL, NULL, NULL, uc, diag);
      for (size_t f = 0; f < bp.nf; ++f) u_new[bp.face_index[4 * f]][bp.face_dense[f]] = uc[f];
      free(p);
      free(uc);
    }
    box_pressure_free(&bp);
  }
  if (st == FO_OK && stride > 0) {
    const double lo_clamp[3] = {b->origin[0] + (b->lo[0] + 1) * h + prm->clamp_margin * h,
                                b->origin[1] + (b->lo[1] + 1) * h + prm->clamp_margin * h,
                                b->origin[2] + (b->lo[2] + 1) * h + prm->clamp_margin * h};
    const double hi_clamp[3] = {b->origin[0] + (b->lo[0] + b->n[0] - 1) * h - prm->clamp_margin * h,
                                b->origin[1] + (b->lo[1] + b->n[1] - 1) * h - prm->clamp_margin * h,
                                b->origin[2] + (b->lo[2] + b->n[2] - 1) * h - prm->clamp_margin * h};
    size_t done = 0;
    for (size_t p = first; p < np && st == FO_OK;) {
      size_t m = 0;
      for (; m < chunk && p < np; ++m, p += stride)
        for (int d = 0; d < 3; ++d) cx[3 * m + d] = soa[(size_t)d * np + p];
      st = fo_g2p(b, cx, m, NULL, u_new, g);
      for (size_t k = 0; k < m && st == FO_OK; ++k) {
        const double* o = g + 24 * k;
        double* s = sample_out + 15 * (done + k);
        for (int d = 0; d < 3; ++d) {
          double nx = cx[3 * k + d] + prm->dt * o[d];
          if (nx < lo_clamp[d]) nx = lo_clamp[d];
          if (nx > hi_clamp[d]) nx = hi_clamp[d];
          s[d] = nx;
          s[3 + d] = o[d];
        }
        for (int q = 0; q < 9; ++q) s[6 + q] = o[6 + q];
      }
      done += m;
    }
  }
  free(cx);
  free(cv);
  free(cc);
  free(g);
  for (int a = 0; a < 3; ++a) {
    free(fm[a]);
    free(fq[a]);
  }
  return st;
}
