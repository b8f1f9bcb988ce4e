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
// restriction, coarse coefficients = (sum of crossing fine coefficients)/2 (for
// uniform coefficients the rediscretized 2^l-scaled operator) and coarse
// anchors = 0.8 x (sum of child anchors) (kCoarseAnchorScale); red-black
// Gauss-Seidel, `pre` sweeps red->black before and `post` sweeps black->red
// after the coarse correction (symmetric); the restriction into a level also
// performs that level's first sweep; the coarsest level is solved by
// `coarse_sweeps` symmetric sweeps inside one CTA's shared memory, together
// with the last dense level when both fit (k_coarse_tail). x and k are stored
// as T (FP32 or BF16), arithmetic is FP32.
#include <cuda_bf16.h>

#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kThreads = 256;
constexpr int kReduceCtas = 4 * 148;  // fixed grid of the reduction kernels (multiple of the SM count)

static inline unsigned blocks_for(long long n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }
static inline unsigned reduce_grid(long long n) {
  const unsigned b = blocks_for(n);
  return b < 1 ? 1u : (b > (unsigned)kReduceCtas ? (unsigned)kReduceCtas : b);
}

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

// ----------------------------------------------------------------- fast in-block neighbours

// Neighbour of local cell l of block b on a sparse level with 2^LS cells per
// axis (shifts and masks only). Returns the cell id, -1 for an inactive block
// inside the lattice (air, no unknown) or -2 outside the lattice (solid).
template <int LS>
__device__ __forceinline__ int nbr_s(const GridView& g, int b, int l, int a, int dir) {
  constexpr int S = 1 << LS, S3 = S * S * S;
  const int c = (l >> (LS * a)) & (S - 1);
  const int step = 1 << (LS * a);
  if (dir < 0 ? c > 0 : c < S - 1) return b * S3 + l + dir * step;
  const int n = g.nbr27[b * 27 + 13 + dir * (a == 0 ? 1 : (a == 1 ? 3 : 9))];
  if (n < 0) return n;
  return n * S3 + l - dir * (S - 1) * step;
}

// Coarse parent of fine cell j on sparse level LS: the next sparse level, or
// (LS == 1) the dense block-lattice cell of j's block.
template <int LS>
__device__ __forceinline__ int parent_s(const GridView& g, int j, int cdx, int cdy) {
  constexpr int S = 1 << LS, S3 = S * S * S;
  const int b = j / S3, l = j % S3;
  if (LS > 1) {
    constexpr int SC = S / 2;
    const int x = (l & (S - 1)) >> 1, y = ((l >> LS) & (S - 1)) >> 1, z = (l >> (2 * LS)) >> 1;
    return b * SC * SC * SC + (z * SC + y) * SC + x;
  }
  return ((g.coord[3 * b + 2] - g.blo[2]) * cdy + (g.coord[3 * b + 1] - g.blo[1])) * cdx + (g.coord[3 * b] - g.blo[0]);
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

// Sum of per-CTA partials by the last CTA, in a fixed order.
__device__ __forceinline__ double finish_sum(const double* partial, int stride, int offset, double* red) {
  double t = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) t += partial[stride * k + offset];
  return block_sum<kThreads>(t, red);
}

__device__ __forceinline__ bool solid_cell(const GridView& g, int x, int y, int z) {
  return x < g.solid_lo[0] || y < g.solid_lo[1] || z < g.solid_lo[2] || x > g.solid_hi[0] || y > g.solid_hi[1] ||
         z > g.solid_hi[2];
}

__global__ void k_classify(GridView g, const int* cell_start, unsigned char* type) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nb * kBlockCells) return;
  const int b = i >> 9, l = i & 511;
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
__device__ __forceinline__ int nbr_type(const unsigned char* type, int id) {
  if (id == -1) return 2;
  if (id < 0) return 0;
  return type[id];
}

// Lattice-indexed cell id (stable across steps, unlike block ordinals).
__device__ __forceinline__ long long lattice_cell(const GridView& g, int b, int l) {
  const long long lb = ((long long)(g.coord[3 * b + 2] - g.blo[2]) * g.bdim[1] + (g.coord[3 * b + 1] - g.blo[1])) *
                           g.bdim[0] +
                       (g.coord[3 * b] - g.blo[0]);
  return lb * 512 + l;
}

// ||b'|| over the per-block partials, in block order.
__global__ void __launch_bounds__(1024) k_setup_finish(int nb, const double* __restrict__ partial, SolverState* st) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += partial[k];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    st->b_norm = sqrt(t);
  }
}

// ----------------------------------------------------------------- coarsening (once per solve)

// Coarse operator: a face coefficient is half the sum of the four fine faces
// that cross it (a uniform grid then reproduces the operator rediscretised at
// twice the spacing); the Dirichlet anchor (coupling to the air at p = 0) is
// 0.8 times the sum of the children's anchors. The free surface does not move
// away from a coarse cell as the cell grows, so halving the anchors like the
// face coefficients under-weights it: on the splash, column-drop and dam-break
// scenes 0.8 needs 20-45% fewer flexible-CG iterations than 0.5 (0.7-0.9 are
// within a few percent of each other; 1.0 and above are slower again).
constexpr float kCoarseAnchorScale = 0.8f;

// Child count per axis is 2; for sparse->sparse the block is shared, for
// sparse(S=2)->dense the block maps to one dense cell, dense->dense halves.
// Level-0 coefficients come from the neighbour mask.
template <typename T>
__global__ void k_coarsen(GridView g, LevelDesc F, LevelPtrs<T> fp, LevelDesc C, LevelPtrs<T> cp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= C.count) return;
  const CellPos p = cell_pos(C, i);
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
    const long long id = fp.mask ? (long long)rb_id((int)child[c]) : child[c];
    if (fp.fluid[id]) fluid = true;
    anchor += fp.anchor[id];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (cl[c][a] == 0) k[a] += fp.mask ? (float)((fp.mask[id] >> (2 * a)) & 1u) : ld(&fp.k[a][id]);
  }
  cp.fluid[i] = fluid ? 1 : 0;
  cp.anchor[i] = kCoarseAnchorScale * anchor;
#pragma unroll
  for (int a = 0; a < 3; ++a) st_T(&cp.k[a][i], 0.5f * k[a]);
}

// diag = anchor + sum of the six face coefficients (after coarsening, since a
// cell's high faces belong to its neighbours). Levels >= 1.
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

// ----------------------------------------------------------------- smoothing (sparse levels)

// Gauss-Seidel update of one colour on a sparse level (2^LS cells per block
// axis). 256 threads per CTA, each owning one cell of the colour; a CTA covers
// 256/(S^3/2) blocks. MODE 0: plain; 1: first sweep from x = 0 (no neighbour
// reads); 2: neighbour values include the coarse correction (prolongation
// fused into the first post-smoothing sweep).
// Colour sweep on an in-block level (LS = 2: 4^3, LS = 1: 2^3 cells per block).
// Every load a cell needs is issued before any result is used -- the cell's
// flag, right-hand side and diagonal, the neighbour ordinals, then the
// coefficients and neighbour values -- and neighbours with k == 0 are masked
// rather than skipped, so a sweep costs one or two memory round trips instead of
// four. The arithmetic (order of the fused multiply-adds) is unchanged.
template <typename T, int LS, int MODE>
__global__ void __launch_bounds__(kThreads)
    k_smooth_sparse(GridView g, LevelPtrs<T> lp, const float* __restrict__ b, int color, const T* __restrict__ xc,
                    int cdx, int cdy, const int* done) {
  static_assert(LS == 1 || LS == 2, "level 0 has its own kernel");
  grid_dependency_wait();
  if (*done) return;
  constexpr int S = 1 << LS, S3 = S * S * S, HALF = S3 / 2, BPC = kThreads / HALF;
  const int t = threadIdx.x;
  const int blk = blockIdx.x * BPC + t / HALF;
  if (blk >= g.nb) return;
  const int j = t % HALF;
  const int z = j / (S * S / 2), rr = j % (S * S / 2), y = rr / (S / 2), xh = rr % (S / 2);
  const int x = 2 * xh + ((y + z + color) & 1);
  const int l = (z * S + y) * S + x;
  const int i = blk * S3 + l;
  const bool fluid = lp.fluid[i] != 0;
  const float bi = b[i];
  const float di = lp.diag[i];
  float s = bi;
  if (MODE != 1) {
    int jn[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) jn[q] = nbr_s<LS>(g, blk, l, q >> 1, (q & 1) ? 1 : -1);
    float kq[6], xq[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int a = q >> 1;
      const bool ok = jn[q] >= 0;
      kq[q] = ok ? ((q & 1) ? ld(&lp.k[a][jn[q]]) : ld(&lp.k[a][i])) : 0.0f;
      float xv = ok ? ld(&lp.x[jn[q]]) : 0.0f;
      if (MODE == 2 && ok) xv += ld(&xc[parent_s<LS>(g, jn[q], cdx, cdy)]);
      xq[q] = xv;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
      if (kq[q] != 0.0f) s = fmaf(kq[q], xq[q], s);
  }
  if (fluid) st_T(&lp.x[i], s / di);
}

// Residual of a sparse level summed into the next level's RHS. 512 threads per
// CTA, one per fine cell; 64 threads then sum 2x2x2 children in a fixed order.
template <typename T, int LS>
__global__ void __launch_bounds__(512)
    k_restrict_sparse(GridView g, LevelPtrs<T> fp, const float* __restrict__ fb, float* cb, int cdx, int cdy,
                      LevelPtrs<T> cp, int cparity, int seed, const int* done) {
  static_assert(LS == 1 || LS == 2, "level 0 has its own kernel");
  grid_dependency_wait();
  if (*done) return;
  constexpr int S = 1 << LS, S3 = S * S * S, BPC = 512 / S3;
  constexpr int SC = S / 2, SC3 = SC * SC * SC;
  __shared__ float r[512];
  const int t = threadIdx.x;
  const int blk = blockIdx.x * BPC + t / S3;
  const int l = t % S3;
  // Coarse cell of thread t < 64, and (seed) its colour-0 first sweep inputs,
  // loaded with the fine inputs below.
  const int cbl = t / SC3, ccl = t % SC3, cblk = blockIdx.x * BPC + cbl;
  const bool cown = t < 64 && cblk < g.nb;
  int out = 0;
  bool cseed = false;
  unsigned char cfl = 0;
  float cdg = 1.0f;
  if (cown) {
    const int cx = ccl % SC, cy = (ccl / SC) % SC, cz = ccl / (SC * SC);
    if (LS > 1) {
      out = cblk * SC3 + ccl;
      cseed = seed && ((cx + cy + cz) & 1) == 0;
    } else {
      const int X = g.coord[3 * cblk] - g.blo[0], Y = g.coord[3 * cblk + 1] - g.blo[1],
                Z = g.coord[3 * cblk + 2] - g.blo[2];
      out = (Z * cdy + Y) * cdx + X;
      cseed = seed && ((X + Y + Z + cparity) & 1) == 0;
    }
    if (cseed) {
      cfl = cp.fluid[out];
      cdg = cp.diag[out];
    }
  }
  float res = 0.0f;
  if (blk < g.nb) {
    const int i = blk * S3 + l;
    const bool fluid = fp.fluid[i] != 0;
    const float di = fp.diag[i];
    const float xi = ld(&fp.x[i]);
    const float bi = fb[i];
    int jn[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) jn[q] = nbr_s<LS>(g, blk, l, q >> 1, (q & 1) ? 1 : -1);
    float kq[6], xq[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int a = q >> 1;
      const bool ok = jn[q] >= 0;
      kq[q] = ok ? ((q & 1) ? ld(&fp.k[a][jn[q]]) : ld(&fp.k[a][i])) : 0.0f;
      xq[q] = ok ? ld(&fp.x[jn[q]]) : 0.0f;
    }
    if (fluid) {
      float ax = di * xi;
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (kq[q] != 0.0f) ax = fmaf(-kq[q], xq[q], ax);
      res = bi - ax;
    }
  }
  r[t] = res;
  __syncthreads();
  if (cown) {
    const int cx = ccl % SC, cy = (ccl / SC) % SC, cz = ccl / (SC * SC);
    float sum = 0.0f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) sum += r[cbl * S3 + ((2 * cz + dz) * S + 2 * cy + dy) * S + 2 * cx + dx];
    cb[out] = sum;
    if (cseed && cfl) st_T(&cp.x[out], sum / cdg);  // the coarse level's first sweep (from zero), colour 0
  }
}


// ----------------------------------------------------------------- tiled level-0 kernels

// Face halo of block blk on level 0: for face f = 2a + (dir > 0), the 8x8
// cells of the neighbouring block that touch it, stored at f * 64 + w * 8 + u
// with (u, w) the two transverse coordinates in increasing axis order. For
// halo entry e in [0, 384) this gives the entry's slot and the natural id of
// the neighbour cell it holds (where the neighbouring block is missing, its
// nbr27 code: -1 inactive, -2 outside the lattice).
__device__ __forceinline__ int halo_src0(const GridView& g, int blk, int e, int* slot) {
  const int f = e >> 6, q = e & 63, a = f >> 1, dir = (f & 1) ? 1 : -1;
  const int u = q & 7, w = q >> 3;
  *slot = e;
  const int nbb = g.nbr27[blk * 27 + 13 + dir * (a == 0 ? 1 : (a == 1 ? 3 : 9))];
  if (nbb < 0) return nbb;  // -1 inactive block (air), -2 outside the lattice (solid)
  const int c = dir < 0 ? 7 : 0;
  const int x = a == 0 ? c : u, y = a == 1 ? c : (a == 0 ? u : w), z = a == 2 ? c : w;
  return nbb * 512 + ((z << 6) | (y << 3) | x);
}

// One-colour face halo: entry e in [0, 192) is one of the 32 cells of colour
// oc on each face of the neighbouring blocks (the only ones a sweep of colour
// 1 - oc reads), stored at the same slot as in the full halo.
__device__ __forceinline__ int halo_src0_colour(const GridView& g, int blk, int oc, int e, int* slot) {
  const int f = e >> 5, k = e & 31, a = f >> 1, dir = (f & 1) ? 1 : -1;
  const int c = dir < 0 ? 7 : 0;  // plane of the neighbour block next to this face
  const int w = k >> 2;
  const int u = 2 * (k & 3) + ((oc + c + w) & 1);  // (c + u + w) & 1 == oc
  *slot = f * 64 + ((w << 3) | u);
  const int nbb = g.nbr27[blk * 27 + 13 + dir * (a == 0 ? 1 : (a == 1 ? 3 : 9))];
  if (nbb < 0) return -1;
  const int x = a == 0 ? c : u, y = a == 1 ? c : (a == 0 ? u : w), z = a == 2 ? c : w;
  return nbb * 512 + ((z << 6) | (y << 3) | x);
}

// Level-0 staging in shared memory: a 10^3 shell around the 8^3 block. Natural
// local cell (x,y,z) sits at (z+1)*100 + (y+1)*10 + x+1; the face cells of the
// six neighbouring blocks fill the outer layer (edges and corners stay unused),
// so every face neighbour is at a constant offset: +-1, +-10, +-100.
constexpr int kShell0 = 1000;
__device__ __forceinline__ int sidx(int l) { return ((l >> 6) + 1) * 100 + (((l >> 3) & 7) + 1) * 10 + (l & 7) + 1; }

// Shell position of halo slot f * 64 + w * 8 + u (face f = 2a + (dir > 0);
// (u, w) the two transverse coordinates in increasing axis order).
__device__ __forceinline__ int shell_of_slot(int slot) {
  const int f = slot >> 6, q = slot & 63, a = f >> 1, c = (f & 1) ? 9 : 0;
  const int u = (q & 7) + 1, w = (q >> 3) + 1;
  return a == 0 ? w * 100 + u * 10 + c : (a == 1 ? w * 100 + c * 10 + u : c * 100 + w * 10 + u);
}

// The halo entries e = t + k * NT (< COUNT) of thread t, loaded in two batches
// (every neighbour-block lookup, then every value) before any shared store, so
// a CTA waits for two memory round trips whatever its cells per thread; each
// value goes to its place in the shell. value(j) maps a neighbour's natural
// cell id to the staged value.
template <int NT, int COUNT, bool kColour, typename V, typename F>
__device__ __forceinline__ void load_halo0(const GridView& g, int blk, int oc, V* shell, F value) {
  constexpr int PER = (COUNT + NT - 1) / NT;
  const int t = threadIdx.x;
  int src[PER], slot[PER];
  V v[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = t + k * NT;
    src[k] = -1;
    slot[k] = -1;
    if (e < COUNT) src[k] = kColour ? halo_src0_colour(g, blk, oc, e, &slot[k]) : halo_src0(g, blk, e, &slot[k]);
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) v[k] = src[k] >= 0 ? value(src[k]) : V(0);
#pragma unroll
  for (int k = 0; k < PER; ++k)
    if (slot[k] >= 0) shell[shell_of_slot(slot[k])] = v[k];
}

// Offsets of the six face neighbours in the shell, in axis/direction order.
__device__ __forceinline__ int shell_off(int q) {
  return (q & 1 ? 1 : -1) * (q < 2 ? 1 : (q < 4 ? 10 : 100));
}

// A (natural local cell at shell position i) applied to the staged shell minus
// the diagonal term: the sum of the neighbour values across the open faces in
// m, in axis/direction order.
template <typename V>
__device__ __forceinline__ V nbr_sum0(const V* sh, int i, unsigned m) {
  V s = V(0);
#pragma unroll
  for (int q = 0; q < 6; ++q)
    if ((m >> q) & 1u) s += sh[i + shell_off(q)];
  return s;
}

__device__ __forceinline__ int parent1_of_nat(int j) {  // level-1 (4^3 per block) parent of a level-0 natural id
  const int b = j >> 9, l = j & 511;
  const int x = (l & 7) >> 1, y = ((l >> 3) & 7) >> 1, z = (l >> 6) >> 1;
  return b * 64 + (z << 4) + (y << 2) + x;
}

// Cells per thread of the tiled level-0 kernels. One CTA still covers one 8^3
// block, so with fewer threads per block more blocks are resident per SM and
// each thread keeps CPT independent loads in flight.
constexpr int kSmooth0Cpt = 4;    // k_smooth0_tiled: 64 threads for the 256 cells of a colour
constexpr int kRestrict0Cpt = 4;  // k_restrict0_tiled: 128 threads
constexpr int kDirectionCpt = 4;  // k_direction_tiled: 128 threads
constexpr int kResidualCpt = 4;   // k_residual64_tiled: 128 threads
constexpr int kCorrectCpt = 4;    // k_correct_tiled: 128 threads
constexpr int kSetupCpt = 4;      // k_setup_level0_tiled: 128 threads

// Red-black sweep of one colour on level 0 (MODE 0 plain, 2 prolongation
// fused); MODE 1 (first sweep from zero) needs no neighbour values. MODE 3 is
// colour 1 of the first pre-smoothing pair with colour 0's sweep from zero
// folded in: the colour-0 neighbour values are formed from b and diag and
// rounded to the storage type exactly as that sweep stores them, and the
// block's fluid colour-0 cells are written too, so the pair takes one launch
// and gives bitwise the two sweeps' result. The cells' masks, right-hand
// sides and diagonals are loaded with the other colour's values and the halo
// lookups, so their latencies overlap.
template <typename T, int MODE, int CPT>
__global__ void __launch_bounds__(256 / CPT)
    k_smooth0_tiled(GridView g, LevelPtrs<T> lp, const float* __restrict__ b, int color, const T* __restrict__ xc,
                    const int* done) {
  constexpr int NT = 256 / CPT;
  grid_dependency_wait();
  if (*done) return;
  __shared__ float sh[kShell0];
  const int blk = blockIdx.x, t = threadIdx.x;
  const T* __restrict__ x = lp.x;
  unsigned m[CPT];
  float bi[CPT], di[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + (color << 8) + t + k * NT;
    m[k] = lp.mask[i];
    bi[k] = b[i];
    di[k] = lp.diag[i];
  }
  if (MODE != 1) {
    const int oc = 1 - color;
    float v[CPT];
    if (MODE == 3) {
      unsigned mo[CPT];
      float bo[CPT], dgo[CPT];
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        const int i = blk * 512 + (oc << 8) + t + k * NT;
        mo[k] = lp.mask[i];
        bo[k] = b[i];
        dgo[k] = lp.diag[i];
      }
      // (a halo cell that is not fluid gets a value no open face ever reads)
      load_halo0<NT, 192, true>(g, blk, oc, sh, [&](int j) {
        const int r = rb_id(j);
        return round_T<T>(b[r] / lp.diag[r]);
      });
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        const float s0 = bo[k] / dgo[k];
        v[k] = round_T<T>(s0);
        if (mo[k] & 64u) st_T(&lp.x[blk * 512 + (oc << 8) + t + k * NT], s0);
      }
    } else {
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        const int c = (oc << 8) + t + k * NT;
        v[k] = ld(&x[blk * 512 + c]);
        if (MODE == 2) v[k] += ld(&xc[parent1_of_nat(blk * 512 + nat_of(c))]);
      }
      load_halo0<NT, 192, true>(g, blk, oc, sh, [&](int j) {
        float hv = ld(&x[rb_id(j)]);
        if (MODE == 2) hv += ld(&xc[parent1_of_nat(j)]);
        return hv;
      });
    }
#pragma unroll
    for (int k = 0; k < CPT; ++k) sh[sidx(nat_of((oc << 8) + t + k * NT))] = v[k];
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    if (!(m[k] & 64u)) continue;
    const int c = (color << 8) + t + k * NT;
    float s = bi[k];
    if (MODE != 1) s += nbr_sum0(sh, sidx(nat_of(c)), m[k]);
    st_T(&lp.x[blk * 512 + c], s / di[k]);
  }
}

// Level-0 residual restricted to level 1: all 512 cells of the block and its
// face halos staged in shared memory.
template <typename T, int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_restrict0_tiled(GridView g, LevelPtrs<T> fp, const float* __restrict__ fb, float* __restrict__ cb,
                      LevelPtrs<T> cp, int seed, const int* done) {
  constexpr int NT = 512 / CPT;
  static_assert(NT >= 64, "one thread per level-1 cell of the block");
  grid_dependency_wait();
  if (*done) return;
  __shared__ float sh[kShell0];
  __shared__ float r[512];
  const int blk = blockIdx.x, t = threadIdx.x;
  unsigned m[CPT];
  float di[CPT], bi[CPT], xv[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT;  // solver (red-black) index
    m[k] = fp.mask[i];
    di[k] = fp.diag[i];
    bi[k] = fb[i];
    xv[k] = ld(&fp.x[i]);
  }
  // (seed) level-1 cell t < 64: colour-0 first-sweep inputs, loaded with the rest
  const bool cseed = seed && t < 64 && (((t & 3) + ((t >> 2) & 3) + (t >> 4)) & 1) == 0;
  const unsigned char cfl = cseed ? cp.fluid[blk * 64 + t] : 0;
  const float cdg = cseed ? cp.diag[blk * 64 + t] : 1.0f;
  load_halo0<NT, 384, false>(g, blk, 0, sh, [&](int j) { return ld(&fp.x[rb_id(j)]); });
#pragma unroll
  for (int k = 0; k < CPT; ++k) sh[sidx(nat_of(t + k * NT))] = xv[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = nat_of(t + k * NT);
    float res = 0.0f;
    if (m[k] & 64u) res = bi[k] - (di[k] * xv[k] - nbr_sum0(sh, sidx(l), m[k]));
    r[l] = res;
  }
  __syncthreads();
  if (t < 64) {
    const int cx = t & 3, cy = (t >> 2) & 3, cz = t >> 4;
    float sum = 0.0f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) sum += r[((2 * cz + dz) << 6) | ((2 * cy + dy) << 3) | (2 * cx + dx)];
    cb[blk * 64 + t] = sum;
    if (cseed && cfl) st_T(&cp.x[blk * 64 + t], sum / cdg);  // level 1's first sweep (from zero), colour 0
  }
}

// Level-0 residual of the V-cycle's iterate, rho = r - A x, one block per CTA
// with x staged with its halo (the input of a learned correction that follows
// the V-cycle).
template <typename T, int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_residual0_tiled(GridView g, LevelPtrs<T> fp, const float* __restrict__ r, float* __restrict__ rho,
                      const int* done) {
  constexpr int NT = 512 / CPT;
  if (*done) return;
  __shared__ float sh[kShell0];
  const int blk = blockIdx.x, t = threadIdx.x;
  unsigned m[CPT];
  float di[CPT], ri[CPT], xv[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT;
    m[k] = fp.mask[i];
    di[k] = fp.diag[i];
    ri[k] = r[i];
    xv[k] = ld(&fp.x[i]);
  }
  load_halo0<NT, 384, false>(g, blk, 0, sh, [&](int j) { return ld(&fp.x[rb_id(j)]); });
#pragma unroll
  for (int k = 0; k < CPT; ++k) sh[sidx(nat_of(t + k * NT))] = xv[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = nat_of(t + k * NT);
    rho[blk * 512 + t + k * NT] = (m[k] & 64u) ? ri[k] - (di[k] * xv[k] - nbr_sum0(sh, sidx(l), m[k])) : 0.0f;
  }
}

// d = z + beta d_old and q = A d for one block, d staged with its halo; the
// block's d.q partial goes to partial[blk].
template <typename T, int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_direction_tiled(GridView g, LevelPtrs<T> L0, const T* __restrict__ z, const float* __restrict__ d_old,
                      float* __restrict__ d_new, float* __restrict__ q, double* partial, SolverState* st) {
  constexpr int NT = 512 / CPT;
  grid_dependency_wait();
  if (st->done) return;
  __shared__ float sh[kShell0];
  __shared__ double red[NT / 32];
  const int blk = blockIdx.x, t = threadIdx.x;
  const float beta = (float)st->beta;
  const bool first = st->inner_iter == 0;
  unsigned m[CPT];
  float dg[CPT], di[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT;
    m[k] = L0.mask[i];
    dg[k] = L0.diag[i];
    const float zi = ld(&z[i]), dold = d_old[i];
    di[k] = (m[k] & 64u) ? (first ? zi : fmaf(beta, dold, zi)) : 0.0f;
  }
  load_halo0<NT, 384, false>(g, blk, 0, sh, [&](int j) {
    const int r = rb_id(j);
    return first ? ld(&z[r]) : fmaf(beta, d_old[r], ld(&z[r]));
  });
#pragma unroll
  for (int k = 0; k < CPT; ++k) sh[sidx(nat_of(t + k * NT))] = di[k];
  __syncthreads();
  double dq = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT;
    float qi = 0.0f;
    if (m[k] & 64u) qi = dg[k] * di[k] - nbr_sum0(sh, sidx(nat_of(t + k * NT)), m[k]);
    d_new[i] = di[k];
    q[i] = qi;
    dq += (double)di[k] * (double)qi;
  }
  dq = warp_sum(dq);
  if ((t & 31) == 0) red[t >> 5] = dq;
  __syncthreads();
  if (t < 32) {
    double v = t < NT / 32 ? red[t] : 0.0;
    v = warp_sum(v);
    if (t == 0) partial[blk] = v;
  }
}

// d.q over the per-block partials of k_direction_tiled, in block order, -> alpha.
__global__ void __launch_bounds__(1024) k_direction_finish(int nb, const double* __restrict__ partial,
                                                           SolverState* st) {
  grid_dependency_wait();
  if (st->done) return;
  __shared__ double red[32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += partial[k];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
    if (!(tot > 0.0) || !isfinite(tot)) {
      st->status = kAborted;
      st->done = 1;
    }
    st->alpha = st->rz / tot;
    st->rz_prev = st->rz;
  }
}

// ----------------------------------------------------------------- dense levels (>= 3)

__device__ __forceinline__ int dense_id(const LevelDesc& L, int x, int y, int z) {
  return (z * L.dim[1] + y) * L.dim[0] + x;
}

// Colour sweep on a dense level (loads issued before use, as on the in-block levels).
template <typename T, int MODE>
__global__ void k_smooth_dense(LevelDesc L, LevelPtrs<T> lp, const float* __restrict__ b, int color, LevelDesc C,
                               const T* __restrict__ xc, const int* done) {
  grid_dependency_wait();
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.count) return;
  const int x = i % L.dim[0], y = (i / L.dim[0]) % L.dim[1], z = i / (L.dim[0] * L.dim[1]);
  if (((x + y + z + L.parity) & 1) != color) return;
  const bool fluid = lp.fluid[i] != 0;
  const float bi = b[i];
  const float di = lp.diag[i];
  float s = bi;
  if (MODE != 1) {
    const int c[3] = {x, y, z};
    float kq[6], xq[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int a = q >> 1, dir = (q & 1) ? 1 : -1;
      int n[3] = {c[0], c[1], c[2]};
      n[a] += dir;
      const bool ok = n[a] >= 0 && n[a] < L.dim[a];
      const int jn = ok ? dense_id(L, n[0], n[1], n[2]) : i;
      kq[q] = ok ? (dir < 0 ? ld(&lp.k[a][i]) : ld(&lp.k[a][jn])) : 0.0f;
      float xv = ok ? ld(&lp.x[jn]) : 0.0f;
      if (MODE == 2 && ok) xv += ld(&xc[dense_id(C, n[0] >> 1, n[1] >> 1, n[2] >> 1)]);
      xq[q] = xv;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
      if (kq[q] != 0.0f) s = fmaf(kq[q], xq[q], s);
  }
  if (fluid) st_T(&lp.x[i], s / di);
}

// Dense-level residual restricted to the next level: one thread per coarse
// cell sums its (up to 8) children's residuals in a fixed order; all child and
// neighbour loads are issued before the sum.
template <typename T>
__global__ void k_restrict_dense(LevelDesc F, LevelPtrs<T> fp, const float* __restrict__ fb, LevelDesc C, float* cb,
                                 LevelPtrs<T> cp, int seed, const int* done) {
  grid_dependency_wait();
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C.count) return;
  const int X = i % C.dim[0], Y = (i / C.dim[0]) % C.dim[1], Z = i / (C.dim[0] * C.dim[1]);
  // (seed) the coarse level's colour-0 first sweep inputs, loaded with the children's
  const bool cseed = seed && ((X + Y + Z + C.parity) & 1) == 0;
  const unsigned char cfl = cseed ? cp.fluid[i] : 0;
  const float cdg = cseed ? cp.diag[i] : 1.0f;
  float sum = 0.0f;
#pragma unroll
  for (int ch = 0; ch < 8; ++ch) {
    const int x = 2 * X + (ch & 1), y = 2 * Y + ((ch >> 1) & 1), z = 2 * Z + (ch >> 2);
    const bool inside = x < F.dim[0] && y < F.dim[1] && z < F.dim[2];
    const int id = inside ? dense_id(F, x, y, z) : 0;
    const bool fluid = inside && fp.fluid[id] != 0;
    const float di = inside ? fp.diag[id] : 0.0f;
    const float xi = inside ? ld(&fp.x[id]) : 0.0f;
    const float bi = inside ? fb[id] : 0.0f;
    const int c[3] = {x, y, z};
    float kq[6], xq[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int a = q >> 1, dir = (q & 1) ? 1 : -1;
      int n[3] = {c[0], c[1], c[2]};
      n[a] += dir;
      const bool ok = inside && n[a] >= 0 && n[a] < F.dim[a];
      const int jn = ok ? dense_id(F, n[0], n[1], n[2]) : 0;
      kq[q] = ok ? (dir < 0 ? ld(&fp.k[a][id]) : ld(&fp.k[a][jn])) : 0.0f;
      xq[q] = ok ? ld(&fp.x[jn]) : 0.0f;
    }
    if (fluid) {
      float ax = di * xi;
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (kq[q] != 0.0f) ax = fmaf(-kq[q], xq[q], ax);
      sum += bi - ax;
    }
  }
  cb[i] = sum;
  if (cseed && cfl) st_T(&cp.x[i], sum / cdg);  // the coarse level's first sweep (from zero), colour 0
}

// Coarsest level: symmetric red-black sweeps in shared memory, one CTA.
template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_solve(LevelDesc L, LevelPtrs<T> lp, const float* b, int sweeps,
                                                       const int* done) {
  grid_dependency_wait();
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
  if (n <= (int)blockDim.x) {
    // One cell per thread: coefficients and neighbour offsets stay in registers.
    const int i = threadIdx.x;
    bool active = false;
    int color = 0;
    float kk[6] = {0, 0, 0, 0, 0, 0}, inv = 0.0f, bi = 0.0f;
    int nb[6] = {0, 0, 0, 0, 0, 0};
    if (i < n && dg[i] != 0.0f) {
      active = true;
      const int cx = i % nx, cy = (i / nx) % ny, cz = i / (nx * ny);
      color = (cx + cy + cz + L.parity) & 1;
      inv = 1.0f / dg[i];
      bi = bb[i];
      if (cx > 0) { kk[0] = k0[i]; nb[0] = i - 1; }
      if (cx + 1 < nx) { kk[1] = k0[i + 1]; nb[1] = i + 1; }
      if (cy > 0) { kk[2] = k1[i]; nb[2] = i - nx; }
      if (cy + 1 < ny) { kk[3] = k1[i + nx]; nb[3] = i + nx; }
      if (cz > 0) { kk[4] = k2[i]; nb[4] = i - nx * ny; }
      if (cz + 1 < nz) { kk[5] = k2[i + nx * ny]; nb[5] = i + nx * ny; }
    }
    for (int pass = 0; pass < 4 * sweeps; ++pass) {
      const int half = pass % 2;
      const int c = pass < 2 * sweeps ? half : 1 - half;
      if (active && color == c) {
        float s = bi;
#pragma unroll
        for (int q = 0; q < 6; ++q) s = fmaf(kk[q], x[nb[q]], s);
        x[i] = s * inv;
      }
      __syncthreads();
    }
    if (i < n) st_T(&lp.x[i], lp.fluid[i] ? x[i] : 0.0f);
    return;
  }
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

// Coarse tail of the V-cycle in one CTA: the last dense level F (at most
// kTailMaxCells cells) pre-smoothed, its residual restricted to the coarsest
// level C, C solved by symmetric sweeps, then F corrected and post-smoothed,
// all in shared memory. The sweeps, restriction and coarsest solve are those
// of k_smooth_dense, k_restrict_dense and k_coarse_solve, in the same order;
// F's iterate stays in FP32 between them (one launch instead of ten).
constexpr int kTailMaxCells = 4096;
constexpr int kTailThreads = 1024;
constexpr int kTailCpt = kTailMaxCells / kTailThreads;

__host__ __device__ constexpr size_t tail_smem_bytes(int nf, int nc) {
  return sizeof(float) * (7 * (size_t)nf + 6 * (size_t)nc) + (size_t)nf;
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads)
    k_coarse_tail(LevelDesc F, LevelPtrs<T> fp, const float* __restrict__ fb, LevelDesc C, LevelPtrs<T> cp,
                  float* __restrict__ cb, int pre, int post, int sweeps, const int* done) {
  grid_dependency_wait();
  if (*done) return;
  extern __shared__ float sm[];
  const int nf = (int)F.count, nc = (int)C.count;
  float* x = sm;                 // F iterate
  float* bf = x + nf;            // F right-hand side
  float* df = bf + nf;           // F diagonal
  float* kf[3] = {df + nf, df + 2 * nf, df + 3 * nf};
  float* xc = df + 4 * nf;       // C iterate
  float* bc = xc + nc;           // C right-hand side
  float* dc = bc + nc;           // C diagonal of fluid cells, 0 elsewhere
  float* kc[3] = {dc + nc, dc + 2 * nc, dc + 3 * nc};
  float* rf = kc[2] + nc;        // F residual before the restriction
  unsigned char* ff = reinterpret_cast<unsigned char*>(rf + nf);  // F fluid flags
  const int t = threadIdx.x;
  for (int i = t; i < nf; i += kTailThreads) {
    x[i] = 0.0f;
    bf[i] = fb[i];
    df[i] = fp.diag[i];
    ff[i] = fp.fluid[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) kf[a][i] = ld(&fp.k[a][i]);
  }
  for (int i = t; i < nc; i += kTailThreads) {
    xc[i] = 0.0f;
    dc[i] = cp.fluid[i] ? cp.diag[i] : 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) kc[a][i] = ld(&cp.k[a][i]);
  }
  // This thread's F cells, worked out once (in `info`): the in-range face
  // neighbours (bits 0-5, axis/direction order), the colour (bit 6) and
  // whether the cell exists (bit 7).
  const int nx = F.dim[0], nxy = F.dim[0] * F.dim[1];
  unsigned info[kTailCpt];
#pragma unroll
  for (int j = 0; j < kTailCpt; ++j) {
    const int i = t + j * kTailThreads;
    const int c0 = i % nx, c1 = (i / nx) % F.dim[1], c2 = i / nxy;
    unsigned m = 0;
    m |= (c0 > 0 ? 1u : 0u) | (c0 + 1 < F.dim[0] ? 2u : 0u);
    m |= (c1 > 0 ? 4u : 0u) | (c1 + 1 < F.dim[1] ? 8u : 0u);
    m |= (c2 > 0 ? 16u : 0u) | (c2 + 1 < F.dim[2] ? 32u : 0u);
    info[j] = m | ((unsigned)((c0 + c1 + c2 + F.parity) & 1) << 6) | (i < nf ? 128u : 0u);
  }
  const int off[6] = {-1, 1, -nx, nx, -nxy, nxy};  // face neighbours in axis/direction order
  __syncthreads();
  // One colour sweep on F: mode 1 from zero, mode 2 with the coarse correction
  // added to the neighbour values read (as k_smooth_dense).
  auto sweep = [&](int color, int mode) {
#pragma unroll
    for (int j = 0; j < kTailCpt; ++j) {
      const unsigned inf = info[j];
      const int i = t + j * kTailThreads;
      if (!(inf & 128u) || (int)((inf >> 6) & 1u) != color || !ff[i]) continue;
      float s = bf[i];
      if (mode != 1) {
        const int c[3] = {i % nx, (i / nx) % F.dim[1], i / nxy};  // used by mode 2 only
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          if (!((inf >> q) & 1u)) continue;
          const int a = q >> 1, jn = i + off[q];
          const float kq = (q & 1) ? kf[a][jn] : kf[a][i];
          float xv = x[jn];
          if (mode == 2) {
            int n[3] = {c[0], c[1], c[2]};
            n[a] += (q & 1) ? 1 : -1;
            xv += xc[dense_id(C, n[0] >> 1, n[1] >> 1, n[2] >> 1)];
          }
          if (kq != 0.0f) s = fmaf(kq, xv, s);
        }
      }
      x[i] = s / df[i];
    }
    __syncthreads();
  };
  sweep(0, 1);
  sweep(1, 0);
  for (int sw = 1; sw < pre; ++sw) {
    sweep(0, 0);
    sweep(1, 0);
  }
  // Residual of F (every cell, all threads), then restricted to C in the
  // children order of k_restrict_dense, one thread per C cell.
#pragma unroll
  for (int j = 0; j < kTailCpt; ++j) {
    const unsigned inf = info[j];
    const int i = t + j * kTailThreads;
    if (!(inf & 128u) || !ff[i]) continue;
    float ax = df[i] * x[i];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if (!((inf >> q) & 1u)) continue;
      const int a = q >> 1, jn = i + off[q];
      const float kq = (q & 1) ? kf[a][jn] : kf[a][i];
      if (kq != 0.0f) ax = fmaf(-kq, x[jn], ax);
    }
    rf[i] = bf[i] - ax;
  }
  __syncthreads();
  for (int I = t; I < nc; I += kTailThreads) {
    const int X = I % C.dim[0], Y = (I / C.dim[0]) % C.dim[1], Z = I / (C.dim[0] * C.dim[1]);
    float sum = 0.0f;
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const int c[3] = {2 * X + (ch & 1), 2 * Y + ((ch >> 1) & 1), 2 * Z + (ch >> 2)};
      if (c[0] >= F.dim[0] || c[1] >= F.dim[1] || c[2] >= F.dim[2]) continue;
      const int id = dense_id(F, c[0], c[1], c[2]);
      if (ff[id]) sum += rf[id];
    }
    bc[I] = sum;
    cb[I] = sum;
  }
  __syncthreads();
  // Coarsest level: symmetric red-black sweeps, one cell per thread (as k_coarse_solve).
  {
    const int i = t;
    bool active = false;
    int color = 0;
    float kk[6] = {0, 0, 0, 0, 0, 0}, inv = 0.0f, bi = 0.0f;
    int nb[6] = {0, 0, 0, 0, 0, 0};
    const int nx = C.dim[0], ny = C.dim[1], nz = C.dim[2];
    if (i < nc && dc[i] != 0.0f) {
      active = true;
      const int X = i % nx, Y = (i / nx) % ny, Z = i / (nx * ny);
      color = (X + Y + Z + C.parity) & 1;
      inv = 1.0f / dc[i];
      bi = bc[i];
      if (X > 0) { kk[0] = kc[0][i]; nb[0] = i - 1; }
      if (X + 1 < nx) { kk[1] = kc[0][i + 1]; nb[1] = i + 1; }
      if (Y > 0) { kk[2] = kc[1][i]; nb[2] = i - nx; }
      if (Y + 1 < ny) { kk[3] = kc[1][i + nx]; nb[3] = i + nx; }
      if (Z > 0) { kk[4] = kc[2][i]; nb[4] = i - nx * ny; }
      if (Z + 1 < nz) { kk[5] = kc[2][i + nx * ny]; nb[5] = i + nx * ny; }
    }
    for (int pass = 0; pass < 4 * sweeps; ++pass) {
      const int half = pass % 2;
      const int c = pass < 2 * sweeps ? half : 1 - half;
      if (active && color == c) {
        float sacc = bi;
#pragma unroll
        for (int q = 0; q < 6; ++q) sacc = fmaf(kk[q], xc[nb[q]], sacc);
        xc[i] = sacc * inv;
      }
      __syncthreads();
    }
    if (i < nc) st_T(&cp.x[i], cp.fluid[i] ? xc[i] : 0.0f);
  }
  __syncthreads();
  sweep(1, 2);
  sweep(0, 0);
  for (int sw = 1; sw < post; ++sw) {
    sweep(1, 0);
    sweep(0, 0);
  }
  for (int i = t; i < nf; i += kTailThreads)
    if (ff[i]) st_T(&fp.x[i], x[i]);
}

// ----------------------------------------------------------------- CG kernels (level 0, grid-stride)


// r64 = b' - A p64 (FP64) for one 8^3 block; r = (float)r64; e = 0; the
// block's ||r64||^2 goes to partial[blk]. One CTA per block with CPT cells per
// thread, p64 staged with its face halo (every load issued before any store).
template <typename T, int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_residual64_tiled(GridView g, LevelPtrs<T> L0, const double* __restrict__ b64, const double* __restrict__ p64,
                       float* __restrict__ r, float* __restrict__ e, double* partial) {
  constexpr int NT = 512 / CPT;
  __shared__ double sh[kShell0];
  __shared__ double red[NT / 32];
  const int blk = blockIdx.x, t = threadIdx.x;
  unsigned m[CPT];
  double bi[CPT], pi[CPT], dg[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT;  // solver (red-black) index
    m[k] = L0.mask[i];
    bi[k] = b64[i];
    pi[k] = p64[i];
    dg[k] = (double)L0.diag[i];
  }
  load_halo0<NT, 384, false>(g, blk, 0, sh, [&](int j) { return p64[rb_id(j)]; });
#pragma unroll
  for (int k = 0; k < CPT; ++k) sh[sidx(nat_of(t + k * NT))] = pi[k];
  __syncthreads();
  double rr = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = blk * 512 + t + k * NT, si = sidx(nat_of(t + k * NT));
    double res = 0.0;
    if (m[k] & 64u) {  // (A p)_i = diag_i p_i - the fluid neighbours, in axis/direction order
      double ax = dg[k] * pi[k];
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if ((m[k] >> q) & 1u) ax -= sh[si + shell_off(q)];
      res = bi[k] - ax;
    }
    r[i] = (float)res;
    e[i] = 0.0f;
    rr += res * res;
  }
  rr = warp_sum(rr);
  if ((t & 31) == 0) red[t >> 5] = rr;
  __syncthreads();
  if (t < 32) {
    double v = t < NT / 32 ? red[t] : 0.0;
    v = warp_sum(v);
    if (t == 0) partial[blk] = v;
  }
}

// ||r64|| over the per-block partials, in block order; decides whether to stop
// and arms the inner solve.
__global__ void __launch_bounds__(1024) k_residual64_finish(int nb, const double* __restrict__ partial,
                                                            SolverState* st) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) acc += partial[k];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    st->res64 = sqrt(t);
    const double target = st->target;
    st->converged = st->res64 <= target ? 1 : 0;
    const double stop = fmax(st->inner_rtol * st->res64, 0.5 * target);
    st->stop2 = stop * stop;
    st->inner_iter = 0;
    st->done = st->converged;
    if (t < st->rr_best) st->rr_best = t;
  }
}

// z.r and z.r_prev -> beta (flexible Polak-Ribiere), rz.
template <typename T>
__global__ void k_dots(int n, const T* __restrict__ z, const float* __restrict__ r, const float* __restrict__ r_prev,
                       double* partial, SolverState* st) {
  grid_dependency_wait();
  if (st->done) return;
  __shared__ double red[kThreads / 32];
  double zr = 0.0, zp = 0.0;
  // Four cells per thread and iteration (n is a multiple of 512): 16-byte loads.
  const float4* r4 = reinterpret_cast<const float4*>(r);
  const float4* p4 = reinterpret_cast<const float4*>(r_prev);
#pragma unroll 2
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n >> 2); i += gridDim.x * blockDim.x) {
    float zv[4];
    ld4(z + 4 * i, zv);
    const float4 rv = r4[i], pv = p4[i];
    zr += (double)zv[0] * (double)rv.x + (double)zv[1] * (double)rv.y + (double)zv[2] * (double)rv.z +
          (double)zv[3] * (double)rv.w;
    zp += (double)zv[0] * (double)pv.x + (double)zv[1] * (double)pv.y + (double)zv[2] * (double)pv.z +
          (double)zv[3] * (double)pv.w;
  }
  const double s0 = block_sum<kThreads>(zr, red);
  const double s1 = block_sum<kThreads>(zp, red);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
  if (last_block(st)) {
    const double t0 = finish_sum(partial, 2, 0, red);
    const double t1 = finish_sum(partial, 2, 1, red);
    if (threadIdx.x == 0) {
      if (!(t0 > 0.0) || !isfinite(t0)) {
        // A learned correction that is not a descent direction ends this inner
        // solve and hands the rest of the projection to the V-cycle.
        if (st->learned && !st->fallback)
          st->fallback = 1;
        else
          st->status = kAborted;
        st->done = 1;
      }
      st->beta = st->inner_iter == 0 ? 0.0 : (t0 - t1) / st->rz_prev;
      st->rz = t0;
      st->ticket = 0;
    }
  }
}

// e += alpha d; r_next = r - alpha q; ||r_next||^2 -> stop test.
__global__ void k_update(int n, const float* __restrict__ d, const float* __restrict__ q, const float* __restrict__ r,
                         float* __restrict__ r_next, float* __restrict__ e, double* partial, SolverState* st) {
  grid_dependency_wait();
  if (st->done) return;
  __shared__ double red[kThreads / 32];
  const float alpha = (float)st->alpha;
  double rr = 0.0;
  // Four cells per thread and iteration (n is a multiple of 512): 16-byte accesses.
  const float4* d4 = reinterpret_cast<const float4*>(d);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  const float4* r4 = reinterpret_cast<const float4*>(r);
  float4* e4 = reinterpret_cast<float4*>(e);
  float4* n4 = reinterpret_cast<float4*>(r_next);
#pragma unroll 2
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n >> 2); i += gridDim.x * blockDim.x) {
    const float4 dv = d4[i], qv = q4[i], rv = r4[i];
    float4 ev = e4[i];
    ev.x = fmaf(alpha, dv.x, ev.x);
    ev.y = fmaf(alpha, dv.y, ev.y);
    ev.z = fmaf(alpha, dv.z, ev.z);
    ev.w = fmaf(alpha, dv.w, ev.w);
    const float4 rn = make_float4(fmaf(-alpha, qv.x, rv.x), fmaf(-alpha, qv.y, rv.y), fmaf(-alpha, qv.z, rv.z),
                                  fmaf(-alpha, qv.w, rv.w));
    e4[i] = ev;
    n4[i] = rn;
    rr += (double)rn.x * (double)rn.x + (double)rn.y * (double)rn.y + (double)rn.z * (double)rn.z +
          (double)rn.w * (double)rn.w;
  }
  const double s = block_sum<kThreads>(rr, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (last_block(st)) {
    const double t = finish_sum(partial, 1, 0, red);
    if (threadIdx.x == 0) {
      st->rr = t;
      st->inner_iter += 1;
      st->total_iter += 1;
      if (st->learned && !st->fallback) {
        st->learned_iter += 1;
        st->stalls = t < st->stall_ratio2 * st->rr_best ? 0 : st->stalls + 1;
        // A stalled learned solve ends here, like a breakdown in k_dots: the
        // rest of the replayed graph would still apply the network.
        if (st->stalls >= st->stall_limit) {
          st->fallback = 1;
          st->done = 1;
        }
      }
      if (t < st->rr_best) st->rr_best = t;
      if (t <= st->stop2 || !isfinite(t) || st->inner_iter >= st->inner_max) st->done = 1;
      if (!isfinite(t)) st->status = kOutOfRange;
      st->ticket = 0;
    }
  }
}

__global__ void k_accumulate(int n, const float* e, double* p64) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p64[i] += (double)e[i];
}

// Corrected face velocities and the post-projection divergence, one CTA per
// 8^3 block with CPT cells per thread. Each owned (low) face gets
// u_new = u_pred + scale (p_tail - p_head) where it has a fluid side and no
// solid side (air pressure 0); other faces keep u_pred. The divergence of each
// fluid cell is taken from the FP64 correction of its six FP32 predicted face
// velocities (l2 and max, m/s summed over the cell's faces); the block's sum of
// squares and maximum go to partial[2 blk] and partial[2 blk + 1]. Types,
// pressures and predicted velocities are staged with their face halos (the
// upper faces of the block's last planes are owned by the upper neighbours).
template <int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_correct_tiled(GridView g, const unsigned char* __restrict__ type, const double* __restrict__ p64,
                    const float* __restrict__ up0, const float* __restrict__ up1, const float* __restrict__ up2,
                    float* __restrict__ un0, float* __restrict__ un1, float* __restrict__ un2, double scale,
                    double* partial) {
  constexpr int NT = 512 / CPT;
  constexpr int PER = 384 / NT;
  static_assert(384 % NT == 0, "whole halo entries per thread");
  __shared__ double ptile[512];
  __shared__ double phalo[6][64];
  __shared__ unsigned char ttile[512];
  __shared__ unsigned char thalo[6][64];
  __shared__ float utile[3][512];
  __shared__ float uhalo[6][64];  // entries of the upper faces (odd f) only
  __shared__ double red[NT / 32], mx[NT / 32];
  const int blk = blockIdx.x, t = threadIdx.x;
  const float* up[3] = {up0, up1, up2};
  float* un[3] = {un0, un1, un2};
  // loads first: the block's cells, then the halo (lookups, then values)
  unsigned char tv[CPT];
  double pv[CPT];
  float uv[3][CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT, i = blk * 512 + l;  // natural order
    tv[k] = type[i];
    pv[k] = p64[blk * 512 + rb_of(l)];
#pragma unroll
    for (int a = 0; a < 3; ++a) uv[a][k] = up[a][i];
  }
  int src[PER], slot[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) src[k] = halo_src0(g, blk, t + k * NT, &slot[k]);
  unsigned char th[PER];
  double ph[PER];
  float uh[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int f = slot[k] >> 6, a = f >> 1;
    th[k] = (unsigned char)nbr_type(type, src[k]);
    ph[k] = src[k] >= 0 ? p64[rb_id(src[k])] : 0.0;
    uh[k] = ((f & 1) && src[k] >= 0) ? up[a][src[k]] : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT;
    ttile[l] = tv[k];
    ptile[l] = pv[k];
#pragma unroll
    for (int a = 0; a < 3; ++a) utile[a][l] = uv[a][k];
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    (&thalo[0][0])[slot[k]] = th[k];
    (&phalo[0][0])[slot[k]] = ph[k];
    (&uhalo[0][0])[slot[k]] = uh[k];
  }
  __syncthreads();
  double maxdiv = 0.0, sumsq = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT, i = blk * 512 + l;
    const int c[3] = {l & 7, (l >> 3) & 7, l >> 6};
    const int ti = tv[k];
    const double pi = pv[k];
    double div = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int step = 1 << (3 * a);
      const int q = a == 0 ? (c[2] << 3) | c[1] : (a == 1 ? (c[2] << 3) | c[0] : (c[1] << 3) | c[0]);
      // lower neighbour (tail of the owned face) and upper neighbour
      const bool lo_in = c[a] > 0, hi_in = c[a] < 7;
      const int tlo = lo_in ? ttile[l - step] : thalo[2 * a][q];
      const int thi = hi_in ? ttile[l + step] : thalo[2 * a + 1][q];
      const double plo = lo_in ? ptile[l - step] : phalo[2 * a][q];
      const double phi = hi_in ? ptile[l + step] : phalo[2 * a + 1][q];
      const double uhi_pred = hi_in ? (double)utile[a][l + step] : (double)uhalo[2 * a + 1][q];
      // owned face: head = this cell, tail = the lower neighbour
      double u = (double)uv[a][k];
      if (ti != 0 && tlo != 0 && (ti == 1 || tlo == 1)) u += scale * ((tlo == 1 ? plo : 0.0) - (ti == 1 ? pi : 0.0));
      un[a][i] = (float)u;
      if (ti == 1) {
        double ulo = (double)uv[a][k], uhi = uhi_pred;
        if (tlo != 0) ulo += scale * ((tlo == 1 ? plo : 0.0) - pi);
        if (thi != 0) uhi += scale * (pi - (thi == 1 ? phi : 0.0));
        div += uhi - ulo;
      }
    }
    if (ti == 1) {
      maxdiv = fmax(maxdiv, fabs(div));
      sumsq += div * div;
    }
  }
  sumsq = warp_sum(sumsq);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxdiv = fmax(maxdiv, __shfl_xor_sync(0xffffffffu, maxdiv, o));
  if ((t & 31) == 0) {
    red[t >> 5] = sumsq;
    mx[t >> 5] = maxdiv;
  }
  __syncthreads();
  if (t == 0) {
    double s2 = 0.0, m2 = 0.0;
    for (int w = 0; w < NT / 32; ++w) {
      s2 += red[w];
      m2 = fmax(m2, mx[w]);
    }
    partial[2 * blk] = s2;
    partial[2 * blk + 1] = m2;
  }
}

// Divergence l2 and max over the per-block partials, in block order.
__global__ void __launch_bounds__(1024) k_correct_finish(int nb, const double* __restrict__ partial,
                                                         SolverState* st) {
  __shared__ double red[32], mx[32];
  double acc = 0.0, mm = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    acc += partial[2 * k];
    mm = fmax(mm, partial[2 * k + 1]);
  }
  acc = warp_sum(acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, o));
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = acc;
    mx[threadIdx.x >> 5] = mm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0, all = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t += red[w];
      all = fmax(all, mx[w]);
    }
    st->div_l2 = sqrt(t);
    st->div_max = all;
  }
}

// Level-0 operator and right-hand side for one 8^3 block, one CTA per block
// with CPT cells per thread: for each fluid cell the fluid-neighbour mask, the
// air anchor (count of air neighbours), the diagonal, b' = -rhs_scale div u
// and the warm-start pressure (p_prev, or 2 p_prev - p_prev2 when both are
// given); the block's ||b'||^2 goes to partial[blk].
// Types and predicted velocities are staged with their face halos (the upper
// faces of the block's last planes are owned by the upper neighbours).
template <typename T, int CPT>
__global__ void __launch_bounds__(512 / CPT)
    k_setup_level0_tiled(GridView g, const unsigned char* __restrict__ type, const float* __restrict__ u0,
                         const float* __restrict__ u1, const float* __restrict__ u2, double rhs_scale,
                         LevelPtrs<T> L0, double* __restrict__ b64, double* __restrict__ p64,
                         const float* __restrict__ p_prev, const float* __restrict__ p_prev2, double* partial) {
  constexpr int NT = 512 / CPT;
  constexpr int PER = 384 / NT;
  static_assert(384 % NT == 0, "whole halo entries per thread");
  __shared__ unsigned char ttile[512];
  __shared__ unsigned char thalo[6][64];
  __shared__ float utile[3][512];
  __shared__ float uhalo[6][64];  // entries of the upper faces (odd f) only
  __shared__ double red[NT / 32];
  const int blk = blockIdx.x, t = threadIdx.x;
  const float* u[3] = {u0, u1, u2};
  // loads first (whatever the cell type): the block's cells, then the halo
  unsigned char tv[CPT];
  float pp[CPT], uv[3][CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT, i = blk * 512 + l;  // natural order
    tv[k] = type[i];
    // warm start: the previous pressure, or extrapolated from the last two
    const int lc = lattice_cell(g, blk, l);
    pp[k] = p_prev != nullptr ? (p_prev2 != nullptr ? 2.0f * p_prev[lc] - p_prev2[lc] : p_prev[lc]) : 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) uv[a][k] = u[a][i];
  }
  int src[PER], slot[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) src[k] = halo_src0(g, blk, t + k * NT, &slot[k]);
  unsigned char th[PER];
  float uh[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int f = slot[k] >> 6, a = f >> 1;
    th[k] = (unsigned char)nbr_type(type, src[k]);
    uh[k] = ((f & 1) && src[k] >= 0) ? u[a][src[k]] : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT;
    ttile[l] = tv[k];
#pragma unroll
    for (int a = 0; a < 3; ++a) utile[a][l] = uv[a][k];
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    (&thalo[0][0])[slot[k]] = th[k];
    (&uhalo[0][0])[slot[k]] = uh[k];
  }
  __syncthreads();
  double bb = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = t + k * NT;
    const int c[3] = {l & 7, (l >> 3) & 7, l >> 6};
    const bool fluid = tv[k] == 1;
    float anchor = 0.0f;
    unsigned mask = fluid ? 64u : 0u;
    double div = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int step = 1 << (3 * a);
      const int q = a == 0 ? (c[2] << 3) | c[1] : (a == 1 ? (c[2] << 3) | c[0] : (c[1] << 3) | c[0]);
      const bool lo_in = c[a] > 0, hi_in = c[a] < 7;
      const int tlo = lo_in ? ttile[l - step] : thalo[2 * a][q];
      const int thi = hi_in ? ttile[l + step] : thalo[2 * a + 1][q];
      const float uh_a = hi_in ? utile[a][l + step] : uhalo[2 * a + 1][q];
      if (fluid) {
        mask |= (tlo == 1 ? 1u : 0u) << (2 * a);
        mask |= (thi == 1 ? 1u : 0u) << (2 * a + 1);
        anchor += (tlo == 2 ? 1.0f : 0.0f) + (thi == 2 ? 1.0f : 0.0f);
        div += (double)uh_a - (double)uv[a][k];
      }
    }
    const int r = blk * 512 + rb_of(l);
    L0.mask[r] = (unsigned char)mask;
    L0.fluid[r] = fluid ? 1 : 0;
    L0.anchor[r] = anchor;
    L0.diag[r] = fluid ? anchor + (float)__popc(mask & 63u) : 1.0f;
    const double rhs = fluid ? -rhs_scale * div : 0.0;
    b64[r] = rhs;
    p64[r] = (fluid && p_prev != nullptr) ? (double)pp[k] : 0.0;
    bb += rhs * rhs;
  }
  bb = warp_sum(bb);
  if ((t & 31) == 0) red[t >> 5] = bb;
  __syncthreads();
  if (t < 32) {
    double v = t < NT / 32 ? red[t] : 0.0;
    v = warp_sum(v);
    if (t == 0) partial[blk] = v;
  }
}

// Solver (red-black) <-> natural level-0 layout conversions.
__global__ void k_export_pressure(GridView g, int n, const double* p64_rb, double* p_nat, float* p_keep) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double p = p64_rb[rb_id(i)];
    p_nat[i] = p;
    if (p_keep != nullptr) p_keep[lattice_cell(g, i >> 9, i & 511)] = (float)p;
  }
}
template <typename T>
__global__ void k_to_natural(int n, const T* x_rb, const unsigned char* fluid_rb, float* out_nat) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = rb_id(i);
    out_nat[i] = fluid_rb[r] ? ld(&x_rb[r]) : 0.0f;
  }
}
__global__ void k_to_rb(int n, const float* in_nat, float* out_rb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out_rb[rb_id(i)] = in_nat[i];
}
__global__ void k_from_rb(int n, const float* in_rb, float* out_nat) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out_nat[i] = in_rb[rb_id(i)];
}

// ----------------------------------------------------------------- host orchestration

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor on the stream drains, hiding the launch gap between
// the many short kernels of a V-cycle. Every kernel launched this way calls
// grid_dependency_wait() before anything else, so it reads no input before the
// predecessor grid has completed (and, the wait being unconditional, each
// grid completes only after its own predecessor: the ordering is transitive).
template <typename... P, typename... A>
static void launch_dep(void (*kernel)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                       A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);  // a failure is left for cudaGetLastError()
}

template <typename T, int LS>
static void smooth_sparse(const GridView& g, const MgHierarchy<T>& H, int l, const float* bl, int color, int mode,
                          const int* done, cudaStream_t s) {
  constexpr int HALF = (1 << (3 * LS)) / 2, BPC = kThreads / HALF;
  const unsigned grid = (unsigned)((g.nb + BPC - 1) / BPC);
  const LevelDesc& C = H.desc[l + 1];
  const T* xc = H.ptr[l + 1].x;
  ++g_kernel_launches;
  // (mode 1, the first sweep from zero, is done by the restriction into this level)
  if (mode == 2)
    launch_dep(k_smooth_sparse<T, LS, 2>, grid, kThreads, 0, s, g, H.ptr[l], bl, color, xc, C.dim[0], C.dim[1], done);
  else
    launch_dep(k_smooth_sparse<T, LS, 0>, grid, kThreads, 0, s, g, H.ptr[l], bl, color, xc, C.dim[0], C.dim[1], done);
}

template <typename T>
static void smooth(const GridView& g, const MgHierarchy<T>& H, int l, const float* bl, int color, int mode,
                   const int* done, cudaStream_t s) {
  if (l == 0) {
    ++g_kernel_launches;
    const T* xc = H.ptr[1].x;
    constexpr int C = kSmooth0Cpt, NT = 256 / C;
    if (mode == 3)
      launch_dep(k_smooth0_tiled<T, 3, C>, g.nb, NT, 0, s, g, H.ptr[0], bl, color, xc, done);
    else if (mode == 1)
      launch_dep(k_smooth0_tiled<T, 1, C>, g.nb, NT, 0, s, g, H.ptr[0], bl, color, xc, done);
    else if (mode == 2)
      launch_dep(k_smooth0_tiled<T, 2, C>, g.nb, NT, 0, s, g, H.ptr[0], bl, color, xc, done);
    else
      launch_dep(k_smooth0_tiled<T, 0, C>, g.nb, NT, 0, s, g, H.ptr[0], bl, color, xc, done);
    return;
  }
  if (l == 1) return smooth_sparse<T, 2>(g, H, l, bl, color, mode, done, s);
  if (l == 2) return smooth_sparse<T, 1>(g, H, l, bl, color, mode, done, s);
  const LevelDesc& D = H.desc[l];
  const LevelDesc& C = H.desc[l + 1 < H.levels ? l + 1 : l];
  const unsigned grid = blocks_for(D.count);
  ++g_kernel_launches;
  // (mode 1, the first sweep from zero, is done by the restriction into this level)
  if (mode == 2)
    launch_dep(k_smooth_dense<T, 2>, grid, kThreads, 0, s, D, H.ptr[l], bl, color, C, H.ptr[l + 1].x, done);
  else
    launch_dep(k_smooth_dense<T, 0>, grid, kThreads, 0, s, D, H.ptr[l], bl, color, C, nullptr, done);
}

// Residual of level l restricted to level l + 1; with `seed`, the restriction
// also performs level l + 1's first pre-smoothing sweep (colour 0 from zero:
// x = b / diag on fluid cells), which then needs no launch of its own.
template <typename T>
static void restrict_level(const GridView& g, const MgHierarchy<T>& H, int l, const float* bl, bool seed,
                           const int* done, cudaStream_t s) {
  const LevelDesc& C = H.desc[l + 1];
  ++g_kernel_launches;
  if (l < 3) {
    const int S3 = 1 << (3 * (3 - l));
    const int bpc = 512 / S3;
    const unsigned grid = (unsigned)((g.nb + bpc - 1) / bpc);
    if (l == 0)
      launch_dep(k_restrict0_tiled<T, kRestrict0Cpt>, g.nb, 512 / kRestrict0Cpt, 0, s, g, H.ptr[0], bl, H.b[1],
                 H.ptr[1], (int)seed, done);
    else if (l == 1)
      launch_dep(k_restrict_sparse<T, 2>, grid, 512, 0, s, g, H.ptr[1], bl, H.b[2], C.dim[0], C.dim[1], H.ptr[2],
                 C.parity, (int)seed, done);
    else
      launch_dep(k_restrict_sparse<T, 1>, grid, 512, 0, s, g, H.ptr[2], bl, H.b[3], C.dim[0], C.dim[1], H.ptr[3],
                 C.parity, (int)seed, done);
    return;
  }
  launch_dep(k_restrict_dense<T>, blocks_for(C.count), kThreads, 0, s, H.desc[l], H.ptr[l], bl, C, H.b[l + 1],
             H.ptr[l + 1], (int)seed, done);
}

template <typename T>
static void vcycle(const GridView& g, const MgHierarchy<T>& H, const float* r0, const MgOptions& opt,
                   const int* done, cudaStream_t s) {
  const int L = H.levels;
  // The last dense level and the coarsest in one CTA when both fit.
  const bool tail = L >= 2 && !H.desc[L - 2].sparse && H.desc[L - 2].count <= kTailMaxCells &&
                    H.desc[L - 1].count <= kTailThreads;
  const int top = tail ? L - 2 : L - 1;  // levels smoothed by the per-level kernels: [0, top)
  for (int l = 0; l < top; ++l) {
    const float* bl = l == 0 ? r0 : H.b[l];
    // colour 0's first sweep (from zero) is folded into colour 1's kernel on
    // level 0 and into the restriction that fills each coarser level
    smooth<T>(g, H, l, bl, 1, l == 0 ? 3 : 0, done, s);
    for (int sw = 1; sw < opt.pre; ++sw) {
      smooth<T>(g, H, l, bl, 0, 0, done, s);
      smooth<T>(g, H, l, bl, 1, 0, done, s);
    }
    restrict_level<T>(g, H, l, bl, l + 1 < top, done, s);
  }
  if (tail) {
    const LevelDesc& F = H.desc[L - 2];
    const LevelDesc& C = H.desc[L - 1];
    const size_t smem = tail_smem_bytes((int)F.count, (int)C.count);
    static unsigned long long configured = 0;
    if (first_on_device(configured))
      cudaFuncSetAttribute(k_coarse_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)tail_smem_bytes(kTailMaxCells, kTailThreads));
    ++g_kernel_launches;
    launch_dep(k_coarse_tail<T>, 1, kTailThreads, smem, s, F, H.ptr[L - 2], (const float*)H.b[L - 2], C,
               H.ptr[L - 1], H.b[L - 1], opt.pre, opt.post, opt.coarse_sweeps, done);
  } else {
    const LevelDesc& C = H.desc[L - 1];
    const size_t smem = (size_t)C.count * 6 * sizeof(float);
    const int threads = C.count <= 1024 ? (int)((C.count + 31) / 32 * 32) : 1024;
    ++g_kernel_launches;
    launch_dep(k_coarse_solve<T>, 1, threads, smem, s, C, H.ptr[L - 1], H.b[L - 1], opt.coarse_sweeps, done);
  }
  for (int l = top - 1; l >= 0; --l) {
    const float* bl = l == 0 ? r0 : H.b[l];
    smooth<T>(g, H, l, bl, 1, 2, done, s);
    smooth<T>(g, H, l, bl, 0, 0, done, s);
    for (int sw = 1; sw < opt.post; ++sw) {
      smooth<T>(g, H, l, bl, 1, 0, done, s);
      smooth<T>(g, H, l, bl, 0, 0, done, s);
    }
  }
}

cudaError_t launch_classify(const GridView& g, const int* cell_start, unsigned char* type, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_classify<<<blocks_for(n), kThreads, 0, s>>>(g, cell_start, type);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pressure_setup(const GridView& g, const int* cell_start, unsigned char* type,
                                  const float* const u_pred[3], double rhs_scale, MgHierarchy<T>& H, double* b64,
                                  double* p64, const float* p_prev, const float* p_prev2, double* partial,
                                  SolverState* st, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_classify<<<blocks_for(n), kThreads, 0, s>>>(g, cell_start, type);
  ++g_kernel_launches;
  k_setup_level0_tiled<T, kSetupCpt><<<g.nb, 512 / kSetupCpt, 0, s>>>(g, type, u_pred[0], u_pred[1], u_pred[2],
                                                                      rhs_scale, H.ptr[0], b64, p64, p_prev,
                                                                      p_prev2, partial);
  ++g_kernel_launches;
  k_setup_finish<<<1, 1024, 0, s>>>(g.nb, partial, st);
  for (int l = 1; l < H.levels; ++l) {
    ++g_kernel_launches;
    k_coarsen<T><<<blocks_for(H.desc[l].count), kThreads, 0, s>>>(g, H.desc[l - 1], H.ptr[l - 1], H.desc[l],
                                                                   H.ptr[l]);
  }
  for (int l = 1; l < H.levels; ++l) {
    ++g_kernel_launches;
    k_level_diag<T><<<blocks_for(H.desc[l].count), kThreads, 0, s>>>(g, H.desc[l], H.ptr[l]);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_apply_vcycle(const GridView& g, const MgHierarchy<T>& H, const float* r, const MgOptions& opt,
                                const int* done, cudaStream_t s) {
  vcycle<T>(g, H, r, opt, done, s);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual0(const GridView& g, const MgHierarchy<T>& H, const float* r, float* rho, const int* done,
                             cudaStream_t s) {
  ++g_kernel_launches;
  k_residual0_tiled<T, kResidualCpt><<<g.nb, 512 / kResidualCpt, 0, s>>>(g, H.ptr[0], r, rho, done);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual64(const GridView& g, const MgHierarchy<T>& H, const double* b64, const double* p64,
                              float* r, float* e, double* partial, SolverState* st, cudaStream_t s) {
  g_kernel_launches += 2;
  k_residual64_tiled<T, kResidualCpt><<<g.nb, 512 / kResidualCpt, 0, s>>>(g, H.ptr[0], b64, p64, r, e, partial);
  k_residual64_finish<<<1, 1024, 0, s>>>(g.nb, partial, st);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fcg_iteration(const GridView& g, const MgHierarchy<T>& H, const MgOptions& opt, float* r_cur,
                                 float* r_prev, float* d_old, float* d_new, float* q, float* e, double* partial,
                                 SolverState* st, const int* done, cudaStream_t s, const PrecondHook* hook) {
  const int n = g.nb * kBlockCells;
  if (hook != nullptr && !hook->compose) {
    const cudaError_t e = hook->apply(hook->ctx, r_cur, H.ptr[0].x, s);
    if (e != cudaSuccess) return e;
  } else {
    vcycle<T>(g, H, r_cur, opt, done, s);
    if (hook != nullptr) {  // the learned correction from the V-cycle's residual, added to z (q as scratch)
      ++g_kernel_launches;
      k_residual0_tiled<T, kResidualCpt><<<g.nb, 512 / kResidualCpt, 0, s>>>(g, H.ptr[0], r_cur, q, done);
      const cudaError_t e = hook->apply(hook->ctx, q, H.ptr[0].x, s);
      if (e != cudaSuccess) return e;
    }
  }
  const T* z = H.ptr[0].x;
  const unsigned grid = reduce_grid(n);
  g_kernel_launches += 4;
  launch_dep(k_dots<T>, grid, kThreads, 0, s, n, z, r_cur, r_prev, partial, st);
  launch_dep(k_direction_tiled<T, kDirectionCpt>, g.nb, 512 / kDirectionCpt, 0, s, g, H.ptr[0], z, d_old, d_new, q, partial, st);
  launch_dep(k_direction_finish, 1, 1024, 0, s, g.nb, partial, st);
  launch_dep(k_update, grid, kThreads, 0, s, n, d_new, q, r_cur, r_prev, e, partial, st);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const GridView& g, const float* e, double* p64, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_accumulate<<<reduce_grid(n), kThreads, 0, s>>>(n, e, p64);
  return cudaGetLastError();
}

cudaError_t launch_correct_faces(const GridView& g, const unsigned char* type, const double* p64,
                                 const float* const u_pred[3], float* const u_new[3], double scale,
                                 double* partial, SolverState* st, cudaStream_t s) {
  g_kernel_launches += 2;
  k_correct_tiled<kCorrectCpt><<<g.nb, 512 / kCorrectCpt, 0, s>>>(g, type, p64, u_pred[0], u_pred[1], u_pred[2],
                                                                  u_new[0], u_new[1], u_new[2], scale, partial);
  k_correct_finish<<<1, 1024, 0, s>>>(g.nb, partial, st);
  return cudaGetLastError();
}

cudaError_t launch_export_pressure(const GridView& g, const double* p64, double* p_nat, float* p_keep,
                                   cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_export_pressure<<<reduce_grid(n), kThreads, 0, s>>>(g, n, p64, p_nat, p_keep);
  return cudaGetLastError();
}

cudaError_t launch_to_rb(const GridView& g, const float* in_nat, float* out_rb, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_to_rb<<<reduce_grid(n), kThreads, 0, s>>>(n, in_nat, out_rb);
  return cudaGetLastError();
}

cudaError_t launch_to_natural_f32(const GridView& g, const float* in_rb, float* out_nat, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_from_rb<<<reduce_grid(n), kThreads, 0, s>>>(n, in_rb, out_nat);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_to_natural(const GridView& g, const MgHierarchy<T>& H, float* out_nat, cudaStream_t s) {
  const int n = g.nb * kBlockCells;
  ++g_kernel_launches;
  k_to_natural<T><<<reduce_grid(n), kThreads, 0, s>>>(n, H.ptr[0].x, H.ptr[0].fluid, out_nat);
  return cudaGetLastError();
}

void configure_pressure_kernels() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_coarse_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 6 * (int)sizeof(float));
  cudaFuncSetAttribute(k_coarse_solve<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       8192 * 6 * (int)sizeof(float));
  done = true;
}

#define FL_INSTANTIATE(T)                                                                                         \
  template cudaError_t launch_pressure_setup<T>(const GridView&, const int*, unsigned char*, const float* const[3], \
                                                double, MgHierarchy<T>&, double*, double*, const float*,            \
                                                const float*, double*, SolverState*, cudaStream_t);                 \
  template cudaError_t launch_apply_vcycle<T>(const GridView&, const MgHierarchy<T>&, const float*,                \
                                              const MgOptions&, const int*, cudaStream_t);                         \
  template cudaError_t launch_residual0<T>(const GridView&, const MgHierarchy<T>&, const float*, float*, const int*, \
                                           cudaStream_t);                                                          \
  template cudaError_t launch_residual64<T>(const GridView&, const MgHierarchy<T>&, const double*, const double*,  \
                                            float*, float*, double*, SolverState*, cudaStream_t);                  \
  template cudaError_t launch_fcg_iteration<T>(const GridView&, const MgHierarchy<T>&, const MgOptions&, float*,   \
                                               float*, float*, float*, float*, float*, double*, SolverState*,      \
                                               const int*, cudaStream_t, const PrecondHook*);                      \
  template cudaError_t launch_to_natural<T>(const GridView&, const MgHierarchy<T>&, float*, cudaStream_t);

FL_INSTANTIATE(float)
FL_INSTANTIATE(__nv_bfloat16)

}  // namespace fl
