// MAC pressure projection: mixed-precision multigrid-preconditioned flexible CG
// with FP64 iterative refinement.
//
// System. The integrated finite-volume operator of the reference
// (ApplyOriginalPressureOperatorInto, native/src/mac_pressure_3d_arithmetic.h:
// 404-436), A p = sum_faces k_f (p_tail - p_head) incidence, with the RHS of
// AssembleIntegratedRhsInto (:263-313). For the box scene every open face has
// the same conductance k = dt*h/rho (area h^2, distance h), so the device works
// in units of k: level-0 face coefficients are 1 between fluid cells, a fluid
// cell gains 1 on its diagonal per air (Dirichlet p = 0) neighbour, sealed
// faces against solid cells contribute nothing, and b' = b/k. Pressures stay
// in Pa. Corrected velocities follow CorrectFacesAndAccumulatePhysicalDefectInto
// (:440-503): u += dt/(rho h) (p_tail - p_head).
//
// Solver (structure mirrors the reference's FP32 inner iteration with FP64
// true-residual restarts, native/src/mac_pressure_workspace_3d.cc:584-657):
//   outer:  r64 = b' - A p64 in FP64; stop when ||r64|| <= rel_tol ||b'||
//   inner:  flexible (Polak-Ribiere) PCG in FP32 on A e = r64, FP64 dot
//           products, preconditioned by one geometric V-cycle
//   p64 += e.
// V-cycle: levels 0-2 live inside each 8^3 block (8^3, 4^3, 2^3 cells), levels
// >= 3 are dense over the block lattice; piecewise-constant prolongation, sum
// restriction, coarse coefficients = (sum of crossing fine coefficients)/2 and
// coarse anchors = (sum of child anchors)/2 (for uniform coefficients this is
// the rediscretized 2^l-scaled operator); red-black Gauss-Seidel, `pre` sweeps
// red->black before and `post` sweeps black->red after the coarse correction
// (symmetric); the coarsest level is solved by `coarse_sweeps` symmetric sweeps
// inside one CTA's shared memory. x and k are stored as T (FP32 or BF16),
// arithmetic is FP32.
#include <cuda_bf16.h>

#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kThreads = 256;

static inline unsigned blocks_for(long long n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

// ----------------------------------------------------------------- neighbours

// Sparse level with S cells per block axis: neighbour of cell (b, l) along
// axis a in direction dir (+1/-1). Returns the global cell id, or -1 (inactive
// block: no unknown there) / -2 (outside the lattice).
__device__ __forceinline__ long long sparse_nbr(const GridView& g, int S, int b, int lx, int ly, int lz, int a,
                                                int dir) {
  int l[3] = {lx, ly, lz};
  l[a] += dir;
  int d[3] = {0, 0, 0};
  if (l[a] < 0) {
    d[a] = -1;
    l[a] += S;
  } else if (l[a] >= S) {
    d[a] = 1;
    l[a] -= S;
  }
  int nb = b;
  if (d[a] != 0) {
    nb = g.nbr27[b * 27 + nbr_index(d[0], d[1], d[2])];
    if (nb < 0) return nb;
  }
  return (long long)nb * S * S * S + (l[2] * S + l[1]) * S + l[0];
}

__device__ __forceinline__ long long dense_nbr(const LevelDesc& L, int x, int y, int z, int a, int dir) {
  int c[3] = {x, y, z};
  c[a] += dir;
  if (c[a] < 0 || c[a] >= L.dim[a]) return -2;
  return ((long long)c[2] * L.dim[1] + c[1]) * L.dim[0] + c[0];
}

struct CellPos {
  int b, x, y, z;  // sparse: block + local coords; dense: b = -1 and lattice coords
};

__device__ __forceinline__ CellPos cell_pos(const LevelDesc& L, long long id) {
  CellPos p;
  if (L.sparse) {
    const int S = L.S, S3 = S * S * S;
    p.b = (int)(id / S3);
    const int l = (int)(id % S3);
    p.x = l % S;
    p.y = (l / S) % S;
    p.z = l / (S * S);
  } else {
    p.b = -1;
    p.x = (int)(id % L.dim[0]);
    p.y = (int)((id / L.dim[0]) % L.dim[1]);
    p.z = (int)(id / ((long long)L.dim[0] * L.dim[1]));
  }
  return p;
}

__device__ __forceinline__ long long level_nbr(const GridView& g, const LevelDesc& L, const CellPos& p, int a,
                                               int dir) {
  return L.sparse ? sparse_nbr(g, L.S, p.b, p.x, p.y, p.z, a, dir) : dense_nbr(L, p.x, p.y, p.z, a, dir);
}

// Global parity of a level cell (red = 0).
__device__ __forceinline__ int cell_parity(const GridView& g, const LevelDesc& L, const CellPos& p) {
  if (L.sparse) {
    const int S = L.S;
    return (g.coord[3 * p.b] * S + p.x + g.coord[3 * p.b + 1] * S + p.y + g.coord[3 * p.b + 2] * S + p.z) & 1;
  }
  return (p.x + p.y + p.z + L.parity) & 1;
}

// ----------------------------------------------------------------- level-0 setup (box scene)

__device__ __forceinline__ bool last_block(SolverState* st) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}


__device__ __forceinline__ bool solid_cell(const GridView& g, int x, int y, int z) {
  return x < g.solid_lo[0] || y < g.solid_lo[1] || z < g.solid_lo[2] || x > g.solid_hi[0] || y > g.solid_hi[1] ||
         z > g.solid_hi[2];
}

__global__ void k_classify(GridView g, const int* cell_start, unsigned char* type) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)g.nb * kBlockCells) return;
  const int b = (int)(i / kBlockCells), l = (int)(i % kBlockCells);
  const int x = g.coord[3 * b] * 8 + (l & 7), y = g.coord[3 * b + 1] * 8 + ((l >> 3) & 7),
            z = g.coord[3 * b + 2] * 8 + (l >> 6);
  unsigned char t;
  if (solid_cell(g, x, y, z))
    t = 0;
  else
    t = cell_start[i + 1] > cell_start[i] ? 1 : 2;
  type[i] = t;
}

// Type of a level-0 neighbour: inactive blocks inside the lattice hold no
// particles and no walls adjacent to fluid, i.e. air; outside the lattice is solid.
__device__ __forceinline__ int nbr_type(const unsigned char* type, long long id) {
  if (id == -1) return 2;
  if (id < 0) return 0;
  return type[id];
}

template <typename T>
__global__ void k_setup_level0(GridView g, const unsigned char* type, const float* u0, const float* u1,
                               const float* u2, double rhs_scale, LevelPtrs<T> L0, double* b64, double* p64,
                               double* partial, SolverState* st) {
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)g.nb * kBlockCells;
  double bb = 0.0;
  if (i < n) {
    const int b = (int)(i / kBlockCells), l = (int)(i % kBlockCells);
    const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
    const float* u[3] = {u0, u1, u2};
    const bool fluid = type[i] == 1;
    float anchor = 0.0f, diag = 0.0f;
    double div = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long long lo = sparse_nbr(g, 8, b, lx, ly, lz, a, -1);
      const long long hi = sparse_nbr(g, 8, b, lx, ly, lz, a, +1);
      const int tlo = nbr_type(type, lo), thi = nbr_type(type, hi);
      const float klo = (fluid && tlo == 1) ? 1.0f : 0.0f;
      st_T(&L0.k[a][i], klo);
      if (fluid) {
        anchor += (tlo == 2 ? 1.0f : 0.0f) + (thi == 2 ? 1.0f : 0.0f);
        diag += (tlo != 0 ? 1.0f : 0.0f) + (thi != 0 ? 1.0f : 0.0f);
        const double ulo = (double)u[a][i];
        const double uhi = hi >= 0 ? (double)u[a][hi] : 0.0;
        div += uhi - ulo;
      }
    }
    L0.fluid[i] = fluid ? 1 : 0;
    L0.anchor[i] = anchor;
    L0.diag[i] = diag;
    const double rhs = fluid ? -rhs_scale * div : 0.0;
    b64[i] = rhs;
    p64[i] = 0.0;
    bb = rhs * rhs;
  }
  const double s = block_sum<kThreads>(bb, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(st)) {
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += partial[k];
    t = block_sum<kThreads>(t, red);
    if (threadIdx.x == 0) {
      st->b_norm = sqrt(t);
      st->ticket = 0;
    }
  }
}

// ----------------------------------------------------------------- coarsening

// Child count per axis is 2; for sparse->sparse the block is shared, for
// sparse(S=2)->dense the block maps to one dense cell, dense->dense halves.
template <typename T>
__global__ void k_coarsen(GridView g, LevelDesc F, LevelPtrs<T> fp, LevelDesc C, LevelPtrs<T> cp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= C.count) return;
  const CellPos p = cell_pos(C, i);
  // Locate children.
  long long child[8];
  int nchild = 0;
  int cl[8][3];
  if (C.sparse) {
    const int S = F.S;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          cl[nchild][0] = dx;
          cl[nchild][1] = dy;
          cl[nchild][2] = dz;
          child[nchild++] = (long long)p.b * S * S * S + ((2 * p.z + dz) * S + 2 * p.y + dy) * S + 2 * p.x + dx;
        }
  } else if (F.sparse) {
    // dense cell = block lattice coordinate; find the block ordinal
    const int bx = p.x + g.blo[0], by = p.y + g.blo[1], bz = p.z + g.blo[2];
    (void)bx;
    (void)by;
    (void)bz;
    const int o = g.table[((long long)p.z * g.bdim[1] + p.y) * g.bdim[0] + p.x];
    if (o >= 0) {
      for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx) {
            cl[nchild][0] = dx;
            cl[nchild][1] = dy;
            cl[nchild][2] = dz;
            child[nchild++] = (long long)o * 8 + (dz * 2 + dy) * 2 + dx;
          }
    }
  } else {
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int x = 2 * p.x + dx, y = 2 * p.y + dy, z = 2 * p.z + dz;
          if (x >= F.dim[0] || y >= F.dim[1] || z >= F.dim[2]) continue;
          cl[nchild][0] = dx;
          cl[nchild][1] = dy;
          cl[nchild][2] = dz;
          child[nchild++] = ((long long)z * F.dim[1] + y) * F.dim[0] + x;
        }
  }
  bool fluid = false;
  float anchor = 0.0f, k[3] = {0.0f, 0.0f, 0.0f};
  for (int c = 0; c < nchild; ++c) {
    const long long id = child[c];
    if (fp.fluid[id]) fluid = true;
    anchor += fp.anchor[id];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (cl[c][a] == 0) k[a] += ld(&fp.k[a][id]);
  }
  cp.fluid[i] = fluid ? 1 : 0;
  cp.anchor[i] = 0.5f * anchor;
#pragma unroll
  for (int a = 0; a < 3; ++a) st_T(&cp.k[a][i], 0.5f * k[a]);
}

// diag = anchor + sum of the six face coefficients (after coarsening, since a
// cell's high faces belong to its neighbours).
template <typename T>
__global__ void k_level_diag(GridView g, LevelDesc L, LevelPtrs<T> lp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.count) return;
  const CellPos p = cell_pos(L, i);
  float d = lp.anchor[i];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    d += ld(&lp.k[a][i]);
    const long long hi = level_nbr(g, L, p, a, +1);
    if (hi >= 0) d += ld(&lp.k[a][hi]);
  }
  lp.diag[i] = lp.fluid[i] ? d : 1.0f;
}

// ----------------------------------------------------------------- smoothing

// Gauss-Seidel update of cells of one colour. mode 0: plain; mode 1: first
// sweep from x = 0 (neighbours read as zero); mode 2: neighbour values include
// the coarse correction xc[parent] (prolongation fused into the first post sweep).
template <typename T>
__global__ void k_smooth(GridView g, LevelDesc L, LevelPtrs<T> lp, const float* b, int color, int mode,
                         LevelDesc Cd, const T* xc, const int* done) {
  if (*done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.count) return;
  if (!lp.fluid[i]) return;
  const CellPos p = cell_pos(L, i);
  if (cell_parity(g, L, p) != color) return;
  float s = b[i];
  if (mode != 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int dir = -1; dir <= 1; dir += 2) {
        const long long j = level_nbr(g, L, p, a, dir);
        if (j < 0) continue;
        const float k = dir < 0 ? ld(&lp.k[a][i]) : ld(&lp.k[a][j]);
        if (k == 0.0f) continue;
        float xj = ld(&lp.x[j]);
        if (mode == 2) xj += ld(&xc[parent_of(g, L, Cd, j)]);
        s = fmaf(k, xj, s);
      }
    }
  }
  st_T(&lp.x[i], s / lp.diag[i]);
}

// Residual of the fine level restricted (summed) into the coarse RHS.
template <typename T>
__global__ void k_residual_restrict(GridView g, LevelDesc F, LevelPtrs<T> fp, const float* fb, LevelDesc C,
                                    LevelPtrs<T> cp, float* cb, const int* done) {
  if (*done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= C.count) return;
  float sum = 0.0f;
  if (cp.fluid[i]) {
    const CellPos p = cell_pos(C, i);
    long long child[8];
    int nchild = 0;
    if (C.sparse) {
      const int S = F.S;
      for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx)
            child[nchild++] = (long long)p.b * S * S * S + ((2 * p.z + dz) * S + 2 * p.y + dy) * S + 2 * p.x + dx;
    } else if (F.sparse) {
      const int o = g.table[((long long)p.z * g.bdim[1] + p.y) * g.bdim[0] + p.x];
      if (o >= 0)
        for (int c = 0; c < 8; ++c) child[nchild++] = (long long)o * 8 + c;
    } else {
      for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx) {
            const int x = 2 * p.x + dx, y = 2 * p.y + dy, z = 2 * p.z + dz;
            if (x >= F.dim[0] || y >= F.dim[1] || z >= F.dim[2]) continue;
            child[nchild++] = ((long long)z * F.dim[1] + y) * F.dim[0] + x;
          }
    }
    for (int c = 0; c < nchild; ++c) {
      const long long id = child[c];
      if (!fp.fluid[id]) continue;
      const CellPos q = cell_pos(F, id);
      const float xi = ld(&fp.x[id]);
      float ax = fp.diag[id] * xi;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int dir = -1; dir <= 1; dir += 2) {
          const long long j = level_nbr(g, F, q, a, dir);
          if (j < 0) continue;
          const float k = dir < 0 ? ld(&fp.k[a][id]) : ld(&fp.k[a][j]);
          if (k == 0.0f) continue;
          ax = fmaf(-k, ld(&fp.x[j]), ax);
        }
      }
      sum += fb[id] - ax;
    }
  }
  cb[i] = sum;
}

// Coarsest level: symmetric red-black sweeps in shared memory, one CTA.
template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_solve(LevelDesc L, LevelPtrs<T> lp, const float* b, int sweeps,
                                                       const int* done) {
  if (*done) return;
  extern __shared__ float sm[];
  const int n = (int)L.count;
  float* x = sm;
  float* bb = x + n;
  float* dg = bb + n;
  float* k0 = dg + n;
  float* k1 = k0 + n;
  float* k2 = k1 + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    x[i] = 0.0f;
    bb[i] = b[i];
    dg[i] = lp.fluid[i] ? lp.diag[i] : 0.0f;
    k0[i] = ld(&lp.k[0][i]);
    k1[i] = ld(&lp.k[1][i]);
    k2[i] = ld(&lp.k[2][i]);
  }
  __syncthreads();
  const int nx = L.dim[0], ny = L.dim[1], nz = L.dim[2];
  for (int pass = 0; pass < 4 * sweeps; ++pass) {
    // forward sweeps red,black; backward sweeps black,red
    const int half = pass % 2;
    const int color = pass < 2 * sweeps ? half : 1 - half;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      if (dg[i] == 0.0f) continue;
      const int cx = i % nx, cy = (i / nx) % ny, cz = i / (nx * ny);
      if (((cx + cy + cz + L.parity) & 1) != color) continue;
      float s = bb[i];
      if (cx > 0) s = fmaf(k0[i], x[i - 1], s);
      if (cx + 1 < nx) s = fmaf(k0[i + 1], x[i + 1], s);
      if (cy > 0) s = fmaf(k1[i], x[i - nx], s);
      if (cy + 1 < ny) s = fmaf(k1[i + nx], x[i + nx], s);
      if (cz > 0) s = fmaf(k2[i], x[i - nx * ny], s);
      if (cz + 1 < nz) s = fmaf(k2[i + nx * ny], x[i + nx * ny], s);
      x[i] = s / dg[i];
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) st_T(&lp.x[i], lp.fluid[i] ? x[i] : 0.0f);
}

// ----------------------------------------------------------------- CG kernels (level 0)

// r64 = b' - A p64 (FP64); r = (float)r64; e = 0; ||r64||^2. The last block
// decides whether to stop and arms the inner solve.
template <typename T>
__global__ void k_residual64(GridView g, LevelPtrs<T> L0, const double* b64, const double* p64, float* r, float* e,
                             double* partial, SolverState* st) {
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)g.nb * kBlockCells;
  double rr = 0.0;
  if (i < n) {
    double res = 0.0;
    if (L0.fluid[i]) {
      const int b = (int)(i / kBlockCells), l = (int)(i % kBlockCells);
      const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
      double ax = (double)L0.diag[i] * p64[i];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int dir = -1; dir <= 1; dir += 2) {
          const long long j = sparse_nbr(g, 8, b, lx, ly, lz, a, dir);
          if (j < 0) continue;
          const float k = dir < 0 ? ld(&L0.k[a][i]) : ld(&L0.k[a][j]);
          if (k != 0.0f) ax -= (double)k * p64[j];
        }
      }
      res = b64[i] - ax;
    }
    r[i] = (float)res;
    e[i] = 0.0f;
    rr = res * res;
  }
  const double s = block_sum<kThreads>(rr, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(st)) {
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += partial[k];
    t = block_sum<kThreads>(t, red);
    if (threadIdx.x == 0) {
      st->res64 = sqrt(t);
      const double target = st->target;
      st->converged = st->res64 <= target ? 1 : 0;
      const double stop = fmax(st->inner_rtol * st->res64, 0.5 * target);
      st->stop2 = stop * stop;
      st->inner_iter = 0;
      st->done = st->converged;
      st->ticket = 0;
    }
  }
}

// z.r and z.r_prev -> beta (flexible Polak-Ribiere), rz.
template <typename T>
__global__ void k_dots(long long n, const T* z, const float* r, const float* r_prev, double* partial,
                       SolverState* st) {
  if (st->done) return;
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double zr = 0.0, zp = 0.0;
  if (i < n) {
    const double zi = (double)ld(&z[i]);
    zr = zi * (double)r[i];
    zp = zi * (double)r_prev[i];
  }
  const double s0 = block_sum<kThreads>(zr, red);
  const double s1 = block_sum<kThreads>(zp, red);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
  if (last_block(st)) {
    double t0 = 0.0, t1 = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
      t0 += partial[2 * k];
      t1 += partial[2 * k + 1];
    }
    t0 = block_sum<kThreads>(t0, red);
    t1 = block_sum<kThreads>(t1, red);
    if (threadIdx.x == 0) {
      if (!(t0 > 0.0) || !isfinite(t0)) {
        st->status = kAborted;
        st->done = 1;
      }
      st->beta = st->inner_iter == 0 ? 0.0 : (t0 - t1) / st->rz_prev;
      st->rz = t0;
      st->ticket = 0;
    }
  }
}

// d = z + beta d_old; q = A d (neighbours' d formed on the fly); d.q -> alpha.
template <typename T>
__global__ void k_direction(GridView g, LevelPtrs<T> L0, const T* z, const float* d_old, float* d_new, float* q,
                            double* partial, SolverState* st) {
  if (st->done) return;
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)g.nb * kBlockCells;
  const float beta = (float)st->beta;
  const bool first = st->inner_iter == 0;
  double dq = 0.0;
  if (i < n) {
    float di = 0.0f, qi = 0.0f;
    if (L0.fluid[i]) {
      di = first ? ld(&z[i]) : fmaf(beta, d_old[i], ld(&z[i]));
      const int b = (int)(i / kBlockCells), l = (int)(i % kBlockCells);
      const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
      float ax = L0.diag[i] * di;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int dir = -1; dir <= 1; dir += 2) {
          const long long j = sparse_nbr(g, 8, b, lx, ly, lz, a, dir);
          if (j < 0) continue;
          const float k = dir < 0 ? ld(&L0.k[a][i]) : ld(&L0.k[a][j]);
          if (k == 0.0f) continue;
          const float dj = first ? ld(&z[j]) : fmaf(beta, d_old[j], ld(&z[j]));
          ax = fmaf(-k, dj, ax);
        }
      }
      qi = ax;
      dq = (double)di * (double)qi;
    }
    d_new[i] = di;
    q[i] = qi;
  }
  const double s = block_sum<kThreads>(dq, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(st)) {
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += partial[k];
    t = block_sum<kThreads>(t, red);
    if (threadIdx.x == 0) {
      if (!(t > 0.0) || !isfinite(t)) {
        st->status = kAborted;
        st->done = 1;
      }
      st->alpha = st->rz / t;
      st->rz_prev = st->rz;
      st->ticket = 0;
    }
  }
}

// e += alpha d; r_next = r - alpha q; ||r_next||^2 -> stop test.
__global__ void k_update(long long n, const float* d, const float* q, const float* r, float* r_next, float* e,
                         double* partial, SolverState* st) {
  if (st->done) return;
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const float alpha = (float)st->alpha;
  double rr = 0.0;
  if (i < n) {
    e[i] = fmaf(alpha, d[i], e[i]);
    const float rn = fmaf(-alpha, q[i], r[i]);
    r_next[i] = rn;
    rr = (double)rn * (double)rn;
  }
  const double s = block_sum<kThreads>(rr, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(st)) {
    double t = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += partial[k];
    t = block_sum<kThreads>(t, red);
    if (threadIdx.x == 0) {
      st->rr = t;
      st->inner_iter += 1;
      st->total_iter += 1;
      if (t <= st->stop2 || !isfinite(t) || st->inner_iter >= st->inner_max) st->done = 1;
      if (!isfinite(t)) st->status = kOutOfRange;
      st->ticket = 0;
    }
  }
}

__global__ void k_accumulate(long long n, const float* e, double* p64) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p64[i] += (double)e[i];
}

// Corrected face velocities and the post-projection divergence in FP64.
// u_new = u_pred + scale (p_tail - p_head) on faces with a fluid side and no
// solid side (air pressure 0); other faces keep u_pred.
__global__ void k_correct_faces(GridView g, const unsigned char* type, const double* p64, const float* up0,
                                const float* up1, const float* up2, float* un0, float* un1, float* un2,
                                double scale) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)g.nb * 3 * kBlockCells) return;
  const int b = (int)(i / (3 * kBlockCells));
  const int a = (int)((i / kBlockCells) % 3);
  const int l = (int)(i % kBlockCells);
  const long long head = (long long)b * kBlockCells + l;
  const long long tail = sparse_nbr(g, 8, b, l & 7, (l >> 3) & 7, l >> 6, a, -1);
  const int th = type[head], tt = nbr_type(type, tail);
  const float* up = a == 0 ? up0 : (a == 1 ? up1 : up2);
  float* un = a == 0 ? un0 : (a == 1 ? un1 : un2);
  double u = (double)up[head];
  if (th != 0 && tt != 0 && (th == 1 || tt == 1)) {
    const double ph = th == 1 ? p64[head] : 0.0;
    const double pt = tt == 1 ? p64[tail] : 0.0;
    u += scale * (pt - ph);
  }
  un[head] = (float)u;
}

// Diagnostics over fluid cells: max |r64| and max |divergence| of the corrected
// FP64 velocities (pred + scale * dp, per face), both in device units.
__global__ void k_diagnostics(GridView g, const unsigned char* type, const double* p64, const double* b64,
                              const float* L0diag, const float* up0, const float* up1, const float* up2,
                              double scale, double* partial, SolverState* st) {
  __shared__ double red[kThreads / 32];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)g.nb * kBlockCells;
  double maxdiv = 0.0, sumsq_div = 0.0;
  if (i < n && type[i] == 1) {
    const int b = (int)(i / kBlockCells), l = (int)(i % kBlockCells);
    const int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
    const float* up[3] = {up0, up1, up2};
    double div = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long long lo = sparse_nbr(g, 8, b, lx, ly, lz, a, -1);
      const long long hi = sparse_nbr(g, 8, b, lx, ly, lz, a, +1);
      const int tlo = nbr_type(type, lo), thi = nbr_type(type, hi);
      double ulo = (double)up[a][i], uhi = hi >= 0 ? (double)up[a][hi] : 0.0;
      if (tlo != 0) ulo += scale * ((tlo == 1 ? p64[lo] : 0.0) - p64[i]);
      if (thi != 0) uhi += scale * (p64[i] - (thi == 1 ? p64[hi] : 0.0));
      div += uhi - ulo;
    }
    maxdiv = fabs(div);
    sumsq_div = div * div;
  }
  (void)b64;
  (void)L0diag;
  // max via warp/block: use sum for L2 and a separate max reduction
  double m = maxdiv;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double mx[kThreads / 32];
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
  const double s = block_sum<kThreads>(sumsq_div, red);
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) mm = fmax(mm, mx[w]);
    partial[2 * blockIdx.x] = s;
    partial[2 * blockIdx.x + 1] = mm;
  }
  if (last_block(st)) {
    if (threadIdx.x == 0) {
      double t = 0.0, mm = 0.0;
      for (unsigned k = 0; k < gridDim.x; ++k) {
        t += partial[2 * k];
        mm = fmax(mm, partial[2 * k + 1]);
      }
      st->div_l2 = sqrt(t);
      st->div_max = mm;
      st->ticket = 0;
    }
  }
}

// ----------------------------------------------------------------- host orchestration

template <typename T>
static void vcycle(const GridView& g, const MgHierarchy<T>& H, const float* r0, const MgOptions& opt,
                   const int* done, cudaStream_t s) {
  const int L = H.levels;
  const float* b = r0;
  for (int l = 0; l < L - 1; ++l) {
    const LevelDesc& D = H.desc[l];
    const unsigned nblk = blocks_for(D.count);
    const float* bl = l == 0 ? r0 : H.b[l];
    k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 0, 1, D, nullptr, done);
    k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 1, 0, D, nullptr, done);
    for (int sw = 1; sw < opt.pre; ++sw) {
      k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 0, 0, D, nullptr, done);
      k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 1, 0, D, nullptr, done);
    }
    const LevelDesc& C = H.desc[l + 1];
    k_residual_restrict<T><<<blocks_for(C.count), kThreads, 0, s>>>(g, D, H.ptr[l], bl, C, H.ptr[l + 1],
                                                                     H.b[l + 1], done);
  }
  {
    const LevelDesc& C = H.desc[L - 1];
    const size_t smem = (size_t)C.count * 6 * sizeof(float);
    static bool configured = false;
    if (!configured) {
      cudaFuncSetAttribute(k_coarse_solve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 6 * (int)sizeof(float));
      configured = true;
    }
    k_coarse_solve<T><<<1, 1024, smem, s>>>(C, H.ptr[L - 1], H.b[L - 1], opt.coarse_sweeps, done);
  }
  for (int l = L - 2; l >= 0; --l) {
    const LevelDesc& D = H.desc[l];
    const unsigned nblk = blocks_for(D.count);
    const float* bl = l == 0 ? r0 : H.b[l];
    k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 1, 2, H.desc[l + 1], H.ptr[l + 1].x, done);
    k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 0, 0, D, nullptr, done);
    for (int sw = 1; sw < opt.post; ++sw) {
      k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 1, 0, D, nullptr, done);
      k_smooth<T><<<nblk, kThreads, 0, s>>>(g, D, H.ptr[l], bl, 0, 0, D, nullptr, done);
    }
  }
  (void)b;
}

template <typename T>
cudaError_t launch_pressure_setup(const GridView& g, const int* cell_start, unsigned char* type,
                                  const float* const u_pred[3], double rhs_scale, MgHierarchy<T>& H, double* b64,
                                  double* p64, double* partial, SolverState* st, cudaStream_t s) {
  const long long n = (long long)g.nb * kBlockCells;
  k_classify<<<blocks_for(n), kThreads, 0, s>>>(g, cell_start, type);
  k_setup_level0<T><<<blocks_for(n), kThreads, 0, s>>>(g, type, u_pred[0], u_pred[1], u_pred[2], rhs_scale,
                                                       H.ptr[0], b64, p64, partial, st);
  for (int l = 1; l < H.levels; ++l)
    k_coarsen<T><<<blocks_for(H.desc[l].count), kThreads, 0, s>>>(g, H.desc[l - 1], H.ptr[l - 1], H.desc[l],
                                                                   H.ptr[l]);
  for (int l = 0; l < H.levels; ++l)
    k_level_diag<T><<<blocks_for(H.desc[l].count), kThreads, 0, s>>>(g, H.desc[l], H.ptr[l]);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_apply_vcycle(const GridView& g, const MgHierarchy<T>& H, const float* r, const MgOptions& opt,
                                const int* done, cudaStream_t s) {
  vcycle<T>(g, H, r, opt, done, s);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual64(const GridView& g, const MgHierarchy<T>& H, const double* b64, const double* p64,
                              float* r, float* e, double* partial, SolverState* st, cudaStream_t s) {
  const long long n = (long long)g.nb * kBlockCells;
  k_residual64<T><<<blocks_for(n), kThreads, 0, s>>>(g, H.ptr[0], b64, p64, r, e, partial, st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fcg_iteration(const GridView& g, const MgHierarchy<T>& H, const MgOptions& opt, float* r_cur,
                                 float* r_prev, float* d_old, float* d_new, float* q, float* e, double* partial,
                                 SolverState* st, const int* done, cudaStream_t s) {
  const long long n = (long long)g.nb * kBlockCells;
  vcycle<T>(g, H, r_cur, opt, done, s);
  const T* z = H.ptr[0].x;
  k_dots<T><<<blocks_for(n), kThreads, 0, s>>>(n, z, r_cur, r_prev, partial, st);
  k_direction<T><<<blocks_for(n), kThreads, 0, s>>>(g, H.ptr[0], z, d_old, d_new, q, partial, st);
  k_update<<<blocks_for(n), kThreads, 0, s>>>(n, d_new, q, r_cur, r_prev, e, partial, st);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const GridView& g, const float* e, double* p64, cudaStream_t s) {
  const long long n = (long long)g.nb * kBlockCells;
  k_accumulate<<<blocks_for(n), kThreads, 0, s>>>(n, e, p64);
  return cudaGetLastError();
}

cudaError_t launch_correct_faces(const GridView& g, const unsigned char* type, const double* p64,
                                 const float* const u_pred[3], float* const u_new[3], double scale,
                                 double* partial, SolverState* st, cudaStream_t s) {
  const long long nf = (long long)g.nb * 3 * kBlockCells;
  k_correct_faces<<<blocks_for(nf), kThreads, 0, s>>>(g, type, p64, u_pred[0], u_pred[1], u_pred[2], u_new[0],
                                                      u_new[1], u_new[2], scale);
  const long long n = (long long)g.nb * kBlockCells;
  k_diagnostics<<<blocks_for(n), kThreads, 0, s>>>(g, type, p64, nullptr, nullptr, u_pred[0], u_pred[1], u_pred[2],
                                                   scale, partial, st);
  return cudaGetLastError();
}

#define FL_INSTANTIATE(T)                                                                                         \
  template cudaError_t launch_pressure_setup<T>(const GridView&, const int*, unsigned char*, const float* const[3], \
                                                double, MgHierarchy<T>&, double*, double*, double*, SolverState*,   \
                                                cudaStream_t);                                                      \
  template cudaError_t launch_apply_vcycle<T>(const GridView&, const MgHierarchy<T>&, const float*,                \
                                              const MgOptions&, const int*, cudaStream_t);                         \
  template cudaError_t launch_residual64<T>(const GridView&, const MgHierarchy<T>&, const double*, const double*,  \
                                            float*, float*, double*, SolverState*, cudaStream_t);                  \
  template cudaError_t launch_fcg_iteration<T>(const GridView&, const MgHierarchy<T>&, const MgOptions&, float*,   \
                                               float*, float*, float*, float*, float*, double*, SolverState*,      \
                                               const int*, cudaStream_t);

FL_INSTANTIATE(float)
FL_INSTANTIATE(__nv_bfloat16)

}  // namespace fl
