// P2G with library-owned static scratch: an entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they deposit: a host
// engine that owns every device allocation through its own pool and forbids
// driver allocations inside its frame loop, or a substep that must not
// allocate once it has started (the reference's own rule for persistent
// attempts, liquid_transfer_stages_3d.h:5-15). fl_p2g_static_scratch runs the
// same P2G kernels as fl_p2g, but without a context: the caller passes the
// block layout, the sorted particles and the output face arrays, and the
// per-block tile scratch lives in a file-scope static __device__ array that
// every GPU loading this library holds until process exit.
//
// The block layout comes from the caller, not from a context, so a first
// kernel checks it and copies it into static arrays with every entry forced
// into range (neighbour ordinals below the block count, particle ranges
// inside [0, count]); the P2G kernels read only those copies, so a malformed
// layout cannot make them access memory outside the caller's buffers or the
// scratch. With a report, the call waits for that check and returns
// FL_INVALID_ARGUMENT before any output is written.
#include <cuda_runtime.h>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kStaticMaxBlocks = 512;  // 512 * 3 * 1100 float2 = 13.5 MB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float2 g_static_tiles[(size_t)kStaticMaxBlocks * 3 * kTileFaces];
static __device__ __align__(256) DeviceReport g_static_report;
static __device__ __align__(256) int g_static_cell_start[kStaticMaxBlocks * kBlockCells + 1];
static __device__ __align__(256) int g_static_neighbors[kStaticMaxBlocks * 27];

// Device addresses of the static arrays, looked up once per device (with
// that device current) on the first call. Host code never passes the symbols
// themselves to a kernel: in host code they are only host-side stand-ins.
struct StaticScratch {
  float2* tiles;
  DeviceReport* report;
  int* cell_start;
  int* neighbors;
};
static StaticScratch g_scratch[kMaxDevices] = {};

template <typename T>
static int symbol(void** out, const T& sym) {
  if (cudaGetSymbolAddress(out, sym) != cudaSuccess) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  return FL_OK;
}

static int static_scratch(int device, StaticScratch* out) {
  if (device < 0 || device >= kMaxDevices) return FL_RESOURCE_EXHAUSTED;
  StaticScratch& s = g_scratch[device];
  if (s.tiles == nullptr) {
    void *t = nullptr, *r = nullptr, *c = nullptr, *n = nullptr;
    int st = symbol(&t, g_static_tiles);
    if (st == FL_OK) st = symbol(&r, g_static_report);
    if (st == FL_OK) st = symbol(&c, g_static_cell_start);
    if (st == FL_OK) st = symbol(&n, g_static_neighbors);
    if (st != FL_OK) return st;
    s = StaticScratch{static_cast<float2*>(t), static_cast<DeviceReport*>(r), static_cast<int*>(c),
                      static_cast<int*>(n)};
  }
  *out = s;
  return FL_OK;
}

// Clears the report, then copies the caller's layout into the static arrays
// with each entry forced into range: a neighbour ordinal at or above the
// block count becomes -1 (inactive), a cell-range bound outside [0, count]
// is clamped into it. Each out-of-range entry, and a decreasing pair of
// bounds, is reported as kInvalidArgument with its index.
__global__ void k_static_layout(const int* __restrict__ cell_start, const int* __restrict__ neighbors, int nb,
                                long long count, int* cs_out, int* nbr_out, DeviceReport* rep) {
  const int n_cs = nb * kBlockCells + 1, n_nb = nb * 27;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cs + n_nb; i += gridDim.x * blockDim.x) {
    if (i < n_cs) {
      const long long v = cell_start[i];
      const bool bad = v < 0 || v > count || (i > 0 && cell_start[i - 1] > v);
      if (bad) report_error(rep, kInvalidArgument, (unsigned long long)i);
      cs_out[i] = (int)(v < 0 ? 0 : (v > count ? count : v));
    } else {
      const int k = i - n_cs;
      const int v = neighbors[k];
      if (v >= nb || v < -2) report_error(rep, kInvalidArgument, (unsigned long long)i);
      nbr_out[k] = v >= nb ? -1 : v;
    }
  }
}

}  // namespace fl

using namespace fl;

extern "C" int fl_p2g_static_scratch(const fl_static_grid* grid, const fl_particles* sorted,
                                     const fl_transfer_params* params, int mode, float* const out0[3],
                                     float* const out1[3], void* stream, fl_report* report) {
  if (!grid || !sorted || !params || !out0 || (mode == 0 && !out1) || (mode != 0 && mode != 1))
    return FL_INVALID_ARGUMENT;
  for (int a = 0; a < 3; ++a)
    if (!out0[a] || (mode == 0 && !out1[a])) return FL_INVALID_ARGUMENT;
  if (grid->block_count > (uint64_t)kStaticMaxBlocks) return FL_RESOURCE_EXHAUSTED;
  if (grid->block_count > 0 && (!grid->block_coords || !grid->neighbors || !grid->cell_start))
    return FL_INVALID_ARGUMENT;
  if (!(grid->h > 0.0) || sorted->count > (uint64_t)INT32_MAX) return FL_INVALID_ARGUMENT;
  for (int d = 0; d < 3; ++d)
    if (sorted->count > 0 && (!sorted->x[d] || !sorted->v[d])) return FL_INVALID_ARGUMENT;
  for (int d = 0; d < 9; ++d)
    if (sorted->count > 0 && !sorted->c[d]) return FL_INVALID_ARGUMENT;
  const int ready = check_device();
  if (ready != FL_OK) return ready;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return FL_FAILED_PRECONDITION;
  }
  StaticScratch sc{};
  const int st = static_scratch(device, &sc);
  if (st != FL_OK) return st;
  DeviceReport* rep = sc.report;
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = (int)grid->block_count;
  // The report starts at zero for every call; the tiles need no clearing: the
  // tile kernel writes the tile of every block of this call (a zero tile for a
  // block without particles) before the merge reads any of them.
  if (cudaMemsetAsync(rep, 0, sizeof(DeviceReport), s) != cudaSuccess) return FL_INTERNAL;
  if (nb > 0) {
    ++g_kernel_launches;
    k_static_layout<<<64, 256, 0, s>>>(grid->cell_start, grid->neighbors, nb, (long long)sorted->count,
                                       sc.cell_start, sc.neighbors, rep);
    if (cudaGetLastError() != cudaSuccess) return FL_INTERNAL;
    if (report) {  // publish nothing for a malformed layout
      DeviceReport host{};
      if (cudaMemcpyAsync(&host, rep, sizeof(DeviceReport), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return FL_INTERNAL;
      if (host.error != 0) {
        report->compiled_architecture = 0;
        report->error = host.error;
        report->first_bad_index = host.first_bad_index;
        return host.error;
      }
    }
  }
  GridView g{};
  for (int d = 0; d < 3; ++d) {
    g.origin[d] = (float)grid->origin[d];
    g.solid_lo[d] = grid->solid_lo[d];
    g.solid_hi[d] = grid->solid_hi[d];
  }
  g.h = (float)grid->h;
  g.inv_h = (float)(1.0 / grid->h);
  g.nb = nb;
  g.coord = grid->block_coords;
  g.nbr27 = sc.neighbors;
  ParticlesView p{};
  for (int d = 0; d < 3; ++d) {
    p.x[d] = sorted->x[d];
    p.v[d] = sorted->v[d];
  }
  for (int d = 0; d < 9; ++d) p.c[d] = sorted->c[d];
  p.mass = sorted->mass;
  p.count = sorted->count;
  P2GMergeParams prm{};
  prm.mode = mode;
  prm.walls = mode == 1 ? 1 : 0;
  prm.mass_scale = sorted->mass ? 1.0f : (float)params->particle_mass;
  prm.min_face_mass = (float)params->min_face_mass;
  prm.dt = (float)params->dt;
  for (int d = 0; d < 3; ++d) prm.gravity[d] = (float)params->gravity[d];
  float* o1[3] = {out1 ? out1[0] : nullptr, out1 ? out1[1] : nullptr, out1 ? out1[2] : nullptr};
  if (launch_p2g(g, p, sc.cell_start, sc.tiles, prm, out0, o1, rep, s) != cudaSuccess) return FL_INTERNAL;
  if (report) {
    DeviceReport host{};
    if (cudaMemcpyAsync(&host, rep, sizeof(DeviceReport), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return FL_INTERNAL;
    report->compiled_architecture = host.compiled_architecture;
    report->error = host.error;
    report->first_bad_index = host.first_bad_index;
    return host.error;
  }
  return FL_OK;
}
