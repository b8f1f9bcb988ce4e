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
#include <cuda_runtime.h>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {

constexpr int kStaticMaxBlocks = 512;  // 512 * 3 * 1100 float2 = 13.5 MB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float2 g_static_tiles[(size_t)kStaticMaxBlocks * 3 * kTileFaces];
static __device__ __align__(256) DeviceReport g_static_report;

// Device addresses of the two static arrays, looked up once per device (with
// that device current) on the first call. Host code never passes the symbols
// themselves to a kernel: in host code they are only host-side stand-ins.
static float2* g_tiles_ptr[kMaxDevices] = {};
static DeviceReport* g_report_ptr[kMaxDevices] = {};

static int static_scratch(int device, float2** tiles, DeviceReport** report) {
  if (device < 0 || device >= kMaxDevices) return FL_RESOURCE_EXHAUSTED;
  if (g_tiles_ptr[device] == nullptr) {
    void* t = nullptr;
    void* r = nullptr;
    if (cudaGetSymbolAddress(&t, g_static_tiles) != cudaSuccess) {
      cudaGetLastError();
      return FL_INTERNAL;
    }
    if (cudaGetSymbolAddress(&r, g_static_report) != cudaSuccess) {
      cudaGetLastError();
      return FL_INTERNAL;
    }
    g_tiles_ptr[device] = static_cast<float2*>(t);
    g_report_ptr[device] = static_cast<DeviceReport*>(r);
  }
  *tiles = g_tiles_ptr[device];
  *report = g_report_ptr[device];
  return FL_OK;
}

}  // namespace fl

using namespace fl;

extern "C" int fl_p2g_static_scratch(const fl_static_grid* grid, const fl_particles* sorted,
                                     const fl_transfer_params* params, int mode, float* const out0[3],
                                     float* const out1[3], void* stream, fl_report* report) {
  if (!grid || !sorted || !params || !out0 || (mode == 0 && !out1) || (mode != 0 && mode != 1))
    return FL_INVALID_ARGUMENT;
  if (grid->block_count > (uint64_t)kStaticMaxBlocks) return FL_RESOURCE_EXHAUSTED;
  if (grid->block_count > 0 && (!grid->block_coords || !grid->neighbors || !grid->cell_start))
    return FL_INVALID_ARGUMENT;
  if (!(grid->h > 0.0)) return FL_INVALID_ARGUMENT;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return FL_FAILED_PRECONDITION;
  }
  float2* tiles = nullptr;
  DeviceReport* rep = nullptr;
  const int st = static_scratch(device, &tiles, &rep);
  if (st != FL_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  // The report starts at zero for every call; the tiles need no clearing: the
  // tile kernel writes the tile of every block of this call (a zero tile for a
  // block without particles) before the merge reads any of them.
  if (cudaMemsetAsync(rep, 0, sizeof(DeviceReport), s) != cudaSuccess) return FL_INTERNAL;
  GridView g{};
  for (int d = 0; d < 3; ++d) {
    g.origin[d] = (float)grid->origin[d];
    g.solid_lo[d] = grid->solid_lo[d];
    g.solid_hi[d] = grid->solid_hi[d];
  }
  g.h = (float)grid->h;
  g.inv_h = (float)(1.0 / grid->h);
  g.nb = (int)grid->block_count;
  g.coord = grid->block_coords;
  g.nbr27 = grid->neighbors;
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
  if (launch_p2g(g, p, grid->cell_start, tiles, prm, out0, o1, rep, s) != cudaSuccess) return FL_INTERNAL;
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
