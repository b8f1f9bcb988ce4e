// Sparse-grid topology and the per-step particle sort.
//
// Topology: blocks holding particles plus a one-block ring become active; the
// ring guarantees that every stencil node and every neighbour of a fluid cell
// is stored (the reference requires owner blocks to be allocated,
// sparse_mac_grid_3d.cc:388-398, and checks support in BuildOwnedMacFaceStencil3D
// :627-657).
//
// Sort: the particle's cell key is (block ordinal * 512 + local cell), local cell
// = z*64 + y*8 + x. A counting sort: an atomic histogram gives each particle an
// arrival rank in its cell, an exclusive scan gives cell_start, original
// indices are scattered to (cell_start + rank), each cell's indices are sorted
// ascending -- the result equals a stable sort, so it is reproducible run to
// run. The operator-level sort then gathers the SoA arrays once; the step does
// not move the particles (P2G and G2P read through the cell order). The reference sorts by
// the signed bin floor((X - 1.5)/4) with CUB (native/cuda/liquid_arena_3d.cu:29-52);
// with 8^3 blocks and per-step re-binning the bin is simply the containing cell.
#include <cub/device/device_scan.cuh>

#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

__device__ __forceinline__ bool particle_cell(const GridView& g, const ParticlesView& p, unsigned long long i,
                                              int cell[3]) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float X = lattice_coord(g, p.x[d][i], d);
    ok = ok && isfinite(X) && fabsf(X) < 1.0e9f;
    cell[d] = ok ? __float2int_rd(X) : 0;
  }
  return ok;
}

__global__ void k_mark_blocks(GridView g, ParticlesView p, unsigned char* occ, DeviceReport* rep) {
  const unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if (i >= p.count) return;
  int cell[3];
  if (!particle_cell(g, p, i, cell)) {
    report_error(rep, kOutOfRange, i);
    return;
  }
  int b[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    b[d] = floor_div8(cell[d]) - g.blo[d];
    if (b[d] < 0 || b[d] >= g.bdim[d]) {
      report_error(rep, kFailedPrecondition, i);
      return;
    }
  }
  // Most particles of a block mark the same byte: read first so only the
  // first visitors store (contended same-address stores serialize in L2).
  const unsigned int idx = (unsigned int)(((size_t)b[2] * g.bdim[1] + b[1]) * g.bdim[0] + b[0]);
  const unsigned int same = __match_any_sync(__activemask(), idx);
  if ((threadIdx.x & 31) == __ffs(same) - 1 && occ[idx] == 0) occ[idx] = 1;
}

__global__ void k_flag_active(GridView g, const unsigned char* occ, int* flag, int total) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int bx = idx % g.bdim[0], by = (idx / g.bdim[0]) % g.bdim[1], bz = idx / (g.bdim[0] * g.bdim[1]);
  int active = 0;
  for (int dz = -1; dz <= 1 && !active; ++dz)
    for (int dy = -1; dy <= 1 && !active; ++dy)
      for (int dx = -1; dx <= 1 && !active; ++dx) {
        const int x = bx + dx, y = by + dy, z = bz + dz;
        if (x < 0 || y < 0 || z < 0 || x >= g.bdim[0] || y >= g.bdim[1] || z >= g.bdim[2]) continue;
        active = occ[((size_t)z * g.bdim[1] + y) * g.bdim[0] + x];
      }
  flag[idx] = active;
}

__global__ void k_compact(GridView g, const int* flag, const int* ordinal, int* table, int* coord, int total,
                          int* nb_out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int bx = idx % g.bdim[0], by = (idx / g.bdim[0]) % g.bdim[1], bz = idx / (g.bdim[0] * g.bdim[1]);
  if (flag[idx]) {
    const int o = ordinal[idx];
    table[idx] = o;
    coord[3 * o] = bx + g.blo[0];
    coord[3 * o + 1] = by + g.blo[1];
    coord[3 * o + 2] = bz + g.blo[2];
  } else {
    table[idx] = -1;
  }
  if (idx == total - 1) *nb_out = ordinal[idx] + flag[idx];
}

__global__ void k_build_nbr27(GridView g, int* nbr27) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nb * 27) return;
  const int b = i / 27, n = i % 27;
  const int dx = n % 3 - 1, dy = (n / 3) % 3 - 1, dz = n / 9 - 1;
  const int x = g.coord[3 * b] + dx - g.blo[0], y = g.coord[3 * b + 1] + dy - g.blo[1],
            z = g.coord[3 * b + 2] + dz - g.blo[2];
  int v;
  if (x < 0 || y < 0 || z < 0 || x >= g.bdim[0] || y >= g.bdim[1] || z >= g.bdim[2])
    v = -2;
  else
    v = g.table[((size_t)z * g.bdim[1] + y) * g.bdim[0] + x];
  nbr27[i] = v;
}

// Particles per thread in k_cell_keys and k_scatter_index: a CTA of 256
// threads covers 1024 consecutive particles, particle k * 256 + t of the CTA's
// range on thread t, with every independent load of the four issued together.
constexpr int kSortIlp = 4;
constexpr int kSortThreads = 256;

__global__ void __launch_bounds__(kSortThreads)
    k_cell_keys(GridView g, ParticlesView p, unsigned int* keys, unsigned int* index, int* counts,
                DeviceReport* rep) {
  const unsigned long long i0 = (unsigned long long)blockIdx.x * (kSortIlp * kSortThreads) + threadIdx.x;
  float X[kSortIlp][3];
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k) {
    const unsigned long long i = i0 + (unsigned long long)k * kSortThreads;
#pragma unroll
    for (int d = 0; d < 3; ++d) X[k][d] = i < p.count ? lattice_coord(g, p.x[d][i], d) : 0.0f;
  }
  int o[kSortIlp], lcell[kSortIlp];
  bool fin_k[kSortIlp];
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k) {
    const unsigned long long i = i0 + (unsigned long long)k * kSortThreads;
    bool fin = true, inside = true;
    int bidx = 0, l = 0;
    if (i < p.count) {
      int b[3], c[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        fin = fin && isfinite(X[k][d]) && fabsf(X[k][d]) < 1.0e9f;
        c[d] = fin ? __float2int_rd(X[k][d]) : 0;
        b[d] = floor_div8(c[d]) - g.blo[d];
        inside = inside && b[d] >= 0 && b[d] < g.bdim[d];
      }
      l = (c[2] - 8 * (b[2] + g.blo[2])) * 64 + (c[1] - 8 * (b[1] + g.blo[1])) * 8 + (c[0] - 8 * (b[0] + g.blo[0]));
      bidx = (int)(((size_t)b[2] * g.bdim[1] + b[1]) * g.bdim[0] + b[0]);
    }
    fin_k[k] = fin;
    o[k] = (i < p.count && fin && inside) ? g.table[bidx] : -1;
    lcell[k] = l;
  }
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k) {
    const unsigned long long i = i0 + (unsigned long long)k * kSortThreads;
    unsigned int key = 0xffffffffu, rank = 0;
    if (o[k] >= 0)
      key = (unsigned int)o[k] * 512u + (unsigned int)lcell[k];
    else if (i < p.count)  // not finite: out of range; else outside the lattice or in an inactive block
      report_error(rep, fin_k[k] ? kFailedPrecondition : kOutOfRange, i);
    // One counter update per cell present in the warp: particles arrive nearly
    // in cell order (the previous step's), so most lanes share a few cells.
    // Each lane of a group takes the group's base plus its position among the
    // group's lanes; ranks within a cell are unique, and k_sort_cells_block
    // fixes their final order.
    const unsigned peers = __match_any_sync(__activemask(), key);
    if (key != 0xffffffffu) {
      const int lane = (int)(threadIdx.x & 31), leader = __ffs(peers) - 1;
      unsigned int base = 0;
      if (lane == leader) base = (unsigned int)atomicAdd(&counts[key], __popc(peers));
      base = __shfl_sync(peers, base, leader);
      rank = base + (unsigned int)__popc(peers & ((1u << lane) - 1u));
    }
    if (i < p.count) {
      keys[i] = key;
      index[i] = rank;  // arrival rank within the cell (order not yet deterministic)
    }
  }
}

// Places each particle's original index at its cell's range start + arrival rank.
__global__ void __launch_bounds__(kSortThreads)
    k_scatter_index(unsigned long long n, const unsigned int* keys, const unsigned int* rank, const int* cell_start,
                    unsigned int* slots) {
  const unsigned long long i0 = (unsigned long long)blockIdx.x * (kSortIlp * kSortThreads) + threadIdx.x;
  unsigned int key[kSortIlp], rk[kSortIlp];
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k) {
    const unsigned long long i = i0 + (unsigned long long)k * kSortThreads;
    key[k] = i < n ? keys[i] : 0xffffffffu;
    rk[k] = i < n ? rank[i] : 0u;
  }
  int start[kSortIlp];
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k) start[k] = key[k] != 0xffffffffu ? cell_start[key[k]] : 0;
#pragma unroll
  for (int k = 0; k < kSortIlp; ++k)
    if (key[k] != 0xffffffffu) slots[start[k] + rk[k]] = (unsigned int)(i0 + (unsigned long long)k * kSortThreads);
}

// Sorts each cell's original indices ascending, which makes the permutation
// equal to a stable sort by cell (deterministic whatever the atomic order).
// One CTA per 8^3 block: the block's slots are staged in shared memory
// (coalesced in and out) and each thread insertion-sorts its cell there; a
// block holding more than kSortBlockCap particles sorts its cells in place.
constexpr int kSortBlockCap = 12288;  // 48 KB of staged slots

__device__ __forceinline__ void insertion_sort(unsigned int* v, int n) {
  for (int k = 1; k < n; ++k) {
    const unsigned int key = v[k];
    int j = k - 1;
    while (j >= 0 && v[j] > key) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = key;
  }
}

__global__ void __launch_bounds__(512) k_sort_cells_block(const int* cell_start, unsigned int* slots) {
  __shared__ unsigned int buf[kSortBlockCap];
  const int b = blockIdx.x, t = threadIdx.x;
  const int beg = cell_start[b * 512], end = cell_start[b * 512 + 512];
  const int cb = cell_start[b * 512 + t], ce = cell_start[b * 512 + t + 1];
  const int n = end - beg;
  if (n > kSortBlockCap) {
    insertion_sort(slots + cb, ce - cb);
    return;
  }
  for (int i = t; i < n; i += 512) buf[i] = slots[beg + i];
  __syncthreads();
  insertion_sort(buf + (cb - beg), ce - cb);
  __syncthreads();
  for (int i = t; i < n; i += 512) slots[beg + i] = buf[i];
}


// Gathers every attribute of particle index[s] into slot s. All 15 (16) loads
// are issued before any store: the buffers may not be declared disjoint to the
// compiler, and interleaving each load with its store would serialize 15 memory
// round trips per particle.
__global__ void k_permute(ParticlesView in, ParticlesView out, const unsigned int* index) {
  const unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if (s >= in.count) return;
  const unsigned int j = index[s];
  float v[16];
#pragma unroll
  for (int d = 0; d < 3; ++d) v[d] = in.x[d][j];
#pragma unroll
  for (int d = 0; d < 3; ++d) v[3 + d] = in.v[d][j];
#pragma unroll
  for (int d = 0; d < 9; ++d) v[6 + d] = in.c[d][j];
  v[15] = in.mass != nullptr ? in.mass[j] : 0.0f;
#pragma unroll
  for (int d = 0; d < 3; ++d) out.x[d][s] = v[d];
#pragma unroll
  for (int d = 0; d < 3; ++d) out.v[d][s] = v[3 + d];
#pragma unroll
  for (int d = 0; d < 9; ++d) out.c[d][s] = v[6 + d];
  if (in.mass != nullptr) out.mass[s] = v[15];
}

__global__ void k_write_arch(DeviceReport* rep) {
  if (threadIdx.x == 0 && blockIdx.x == 0) rep->compiled_architecture = compiled_arch();
}

// ------------------------------------------------------------------ host side

static inline unsigned int grid_for(unsigned long long n, int threads) {
  return (unsigned int)((n + threads - 1) / threads);
}

// Scratch of the exclusive scans (the largest runs over every cell + 1).
size_t sort_temp_bytes(size_t particle_capacity, size_t cell_capacity) {
  (void)particle_capacity;
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, (int)(cell_capacity + 1));
  return b + 256;
}

cudaError_t launch_topology_from_particles(const GridView& g, const ParticlesView& p, unsigned char* occ,
                                           int* flag, int* ordinal, int* table, int* coord, int* nb_dev,
                                           void* temp, size_t temp_bytes, DeviceReport* rep, cudaStream_t s) {
  const int total = g.bdim[0] * g.bdim[1] * g.bdim[2];
  cudaMemsetAsync(occ, 0, (size_t)total, s);
  if (p.count > 0) {
    ++g_kernel_launches;
    k_mark_blocks<<<grid_for(p.count, 256), 256, 0, s>>>(g, p, occ, rep);
  }
  ++g_kernel_launches;
  k_flag_active<<<grid_for(total, 256), 256, 0, s>>>(g, occ, flag, total);
  size_t tb = temp_bytes;
  ++g_library_launches;
  cub::DeviceScan::ExclusiveSum(temp, tb, flag, ordinal, total, s);
  ++g_kernel_launches;
  k_compact<<<grid_for(total, 256), 256, 0, s>>>(g, flag, ordinal, table, coord, total, nb_dev);
  return cudaGetLastError();
}

cudaError_t launch_topology_from_occupancy(const GridView& g, const unsigned char* occ, int* flag, int* ordinal,
                                           int* table, int* coord, int* nb_dev, void* temp, size_t temp_bytes,
                                           cudaStream_t s) {
  const int total = g.bdim[0] * g.bdim[1] * g.bdim[2];
  ++g_kernel_launches;
  k_flag_active<<<grid_for(total, 256), 256, 0, s>>>(g, occ, flag, total);
  size_t tb = temp_bytes;
  ++g_library_launches;
  cub::DeviceScan::ExclusiveSum(temp, tb, flag, ordinal, total, s);
  ++g_kernel_launches;
  k_compact<<<grid_for(total, 256), 256, 0, s>>>(g, flag, ordinal, table, coord, total, nb_dev);
  return cudaGetLastError();
}

cudaError_t launch_build_neighbors(const GridView& g, int* nbr27, cudaStream_t s) {
  if (g.nb > 0) {
    ++g_kernel_launches;
    k_build_nbr27<<<grid_for((unsigned long long)g.nb * 27, 256), 256, 0, s>>>(g, nbr27);
  }
  return cudaGetLastError();
}

cudaError_t launch_sort(const GridView& g, const ParticlesView& in, const ParticlesView& out, unsigned int* keys,
                        unsigned int* index, unsigned int* index_alt, int* counts,
                        int* cell_start, void* temp, size_t temp_bytes, DeviceReport* rep, cudaStream_t s,
                        bool permute) {
  const size_t ncell = (size_t)g.nb * 512;
  cudaMemsetAsync(counts, 0, sizeof(int) * (ncell + 1), s);
  ++g_kernel_launches;
  k_write_arch<<<1, 32, 0, s>>>(rep);
  if (in.count > 0) {
    ++g_kernel_launches;
    k_cell_keys<<<grid_for(in.count, kSortIlp * kSortThreads), kSortThreads, 0, s>>>(g, in, keys, index, counts, rep);
  }
  size_t tb = temp_bytes;
  ++g_library_launches;
  cub::DeviceScan::ExclusiveSum(temp, tb, counts, cell_start, (int)(ncell + 1), s);
  if (in.count > 0) {
    g_kernel_launches += permute ? 3 : 2;
    k_scatter_index<<<grid_for(in.count, kSortIlp * kSortThreads), kSortThreads, 0, s>>>(in.count, keys, index,
                                                                                          cell_start, index_alt);
    k_sort_cells_block<<<(unsigned)(ncell / 512), 512, 0, s>>>(cell_start, index_alt);
    if (permute) k_permute<<<grid_for(in.count, 256), 256, 0, s>>>(in, out, index_alt);
  }
  return cudaGetLastError();
}

}  // namespace fl
