// Launch-level declarations shared by the CUDA translation units and the host
// orchestration (fl_context.cu). Not part of the public C-ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include "fl_internal.cuh"

namespace fl {

struct P2GMergeParams {
  int mode;             // 0: raw mass + momentum; 1: normalize + gravity (+ walls)
  int walls;            // apply the stationary-wall condition on solid-adjacent faces
  float mass_scale;     // uniform particle mass (1 when masses are per particle)
  float min_face_mass;  // NormalizeCore threshold
  float dt;
  float gravity[3];
  unsigned char* validity[3];  // mode 1: NormalizeCore's per-face validity when not null
};

// LiquidFaceValidity3D (liquid_boundary_transfer_types_3d.h:37-42).
enum FaceValidity : unsigned char { kFaceMissing = 0, kFaceValid = 1, kFacePredicted = 2, kFaceLowMass = 3 };

struct G2PParams {
  float dt;
  float clamp_lo[3];
  float clamp_hi[3];
  // step mode: when set, the blocks of the advected positions are marked here
  // (zeroed beforehand) for the next step's topology
  unsigned char* occ_next = nullptr;
  // step mode: when set, particle q (in cell order) is read from x_in at
  // order[q] (the unpermuted state) and written to the output view at q, so the
  // step needs no separate permutation pass
  const unsigned int* order = nullptr;
  const float* x_in[3] = {nullptr, nullptr, nullptr};
};

// One multigrid level. Sparse levels keep S^3 cells per active block; dense
// levels cover the block lattice (coarsened by 2 per level above level 3).
struct LevelDesc {
  int sparse;
  int S;
  int dim[3];
  long long count;
  int parity;
};

template <typename T>
struct LevelPtrs {
  unsigned char* mask;  // level 0 only: bit 2a (2a+1) = low (high) face joins two fluid cells; bit 6 = fluid
  unsigned char* fluid;
  T* k[3];        // coefficient of the cell's low face (to the -e_a neighbour)
  float* anchor;  // Dirichlet/compliance part of the diagonal
  float* diag;
  T* x;
};

template <typename T>
struct MgHierarchy {
  int levels;
  LevelDesc desc[12];
  LevelPtrs<T> ptr[12];
  float* b[12];  // b[0] unused: level 0 reads the CG residual
};

struct MgOptions {
  int pre;
  int post;
  int coarse_sweeps;
};

struct SolverState {
  double b_norm;      // ||b'||
  double target;      // rel_tol * ||b'||
  double res64;       // ||b' - A p64|| (FP64)
  double inner_rtol;  // inner FCG stop, relative to res64
  double stop2;
  double rz, rz_prev, beta, alpha, rr;
  double div_l2, div_max;
  double rr_best;       // learned preconditioner: best ||r||^2 so far
  double stall_ratio2;  // an iteration stalls unless ||r||^2 < stall_ratio2 * rr_best
  int learned;          // 1: the learned preconditioner is active until `fallback`
  int stall_limit;
  int stalls;
  int fallback;
  int learned_iter;
  int nn_error;         // the learned preconditioner's kernels gave up waiting
  int converged;
  int done;
  int status;
  int inner_iter;
  int inner_max;
  int total_iter;
  unsigned int ticket;
  int pad;
};

__device__ __forceinline__ long long parent_of(const GridView& g, const LevelDesc& F, const LevelDesc& C,
                                               long long j);

// Number of this library's own kernels launched so far (host-side count).
extern unsigned long long g_kernel_launches;
// Library (CUB) device-wide algorithm invocations so far.
extern unsigned long long g_library_launches;

size_t sort_temp_bytes(size_t particle_capacity, size_t cell_capacity);
// Topology from an occupancy already marked (by the previous step's G2P): the
// active blocks (occupied + one-block ring), their ordinals and coordinates.
cudaError_t launch_topology_from_occupancy(const GridView& g, const unsigned char* occ, int* flag, int* ordinal,
                                           int* table, int* coord, int* nb_dev, void* temp, size_t temp_bytes,
                                           cudaStream_t s);
cudaError_t launch_topology_from_particles(const GridView& g, const ParticlesView& p, unsigned char* occ, int* flag,
                                           int* ordinal, int* table, int* coord, int* nb_dev, void* temp,
                                           size_t temp_bytes, DeviceReport* rep, cudaStream_t s);
cudaError_t launch_build_neighbors(const GridView& g, int* nbr27, cudaStream_t s);
cudaError_t launch_sort(const GridView& g, const ParticlesView& in, const ParticlesView& out, unsigned int* keys,
                        unsigned int* index, unsigned int* index_alt, int* counts,
                        int* cell_start, void* temp, size_t temp_bytes, DeviceReport* rep, cudaStream_t s,
                        bool permute = true);  // false: index_alt holds the cell order, `out` is not written
cudaError_t launch_p2g(const GridView& g, const ParticlesView& p, const int* cell_start, float2* tiles,
                       const P2GMergeParams& prm, float* const out0[3], float* const out1[3], DeviceReport* rep,
                       cudaStream_t s, const unsigned int* order = nullptr);  // order: particle of cell-order slot q
cudaError_t launch_g2p(const GridView& g, const ParticlesView& p, const int* cell_start, const float* const u[3],
                       const float* const u_old[3], const G2PParams& prm, float* full_out, DeviceReport* rep,
                       cudaStream_t s);

template <typename T>
cudaError_t launch_pressure_setup(const GridView& g, const int* cell_start, unsigned char* type,
                                  const float* const u_pred[3], double rhs_scale, MgHierarchy<T>& H, double* b64,
                                  double* p64, const float* p_prev,
                                  const float* p_prev2, double* partial, SolverState* st,
                                  cudaStream_t s);
template <typename T>
cudaError_t launch_apply_vcycle(const GridView& g, const MgHierarchy<T>& H, const float* r, const MgOptions& opt,
                                const int* done, cudaStream_t s);
template <typename T>
cudaError_t launch_residual0(const GridView& g, const MgHierarchy<T>& H, const float* r, float* rho, const int* done,
                             cudaStream_t s);
template <typename T>
cudaError_t launch_residual64(const GridView& g, const MgHierarchy<T>& H, const double* b64, const double* p64,
                              float* r, float* e, double* partial, SolverState* st, cudaStream_t s);
// Replacement preconditioner z = M(r) launched in place of the V-cycle (z is the
// level-0 vector H.ptr[0].x, of the hierarchy's storage type).
// A learned preconditioner inside the flexible-CG iteration. compose 0: z =
// apply(r) in place of the V-cycle; compose 1: z = V(r), then apply adds its
// correction computed from the V-cycle's residual r - A z into z.
struct PrecondHook {
  cudaError_t (*apply)(void* ctx, const float* r, void* z, cudaStream_t s);
  void* ctx;
  int compose;
};

template <typename T>
cudaError_t launch_fcg_iteration(const GridView& g, const MgHierarchy<T>& H, const MgOptions& opt, float* r_cur,
                                 float* r_prev, float* d_old, float* d_new, float* q, float* e, double* partial,
                                 SolverState* st, const int* done, cudaStream_t s, const PrecondHook* hook = nullptr);
cudaError_t launch_export_pressure(const GridView& g, const double* p64, double* p_nat, float* p_keep,
                                   cudaStream_t s);
cudaError_t launch_to_rb(const GridView& g, const float* in_nat, float* out_rb, cudaStream_t s);
// Level-0 float vector from the red-black block layout to natural cell order.
cudaError_t launch_to_natural_f32(const GridView& g, const float* in_rb, float* out_nat, cudaStream_t s);
// Cell types of the last sort: 0 solid, 1 fluid (holds particles), 2 air.
cudaError_t launch_classify(const GridView& g, const int* cell_start, unsigned char* type, cudaStream_t s);
template <typename T>
cudaError_t launch_to_natural(const GridView& g, const MgHierarchy<T>& H, float* out_nat, cudaStream_t s);
void configure_pressure_kernels();
cudaError_t launch_accumulate(const GridView& g, const float* e, double* p64, cudaStream_t s);
cudaError_t launch_correct_faces(const GridView& g, const unsigned char* type, const double* p64,
                                 const float* const u_pred[3], float* const u_new[3], double scale, double* partial,
                                 SolverState* st, cudaStream_t s);

// ------------------------------------------------------------- device helpers

__device__ __forceinline__ long long parent_of(const GridView& g, const LevelDesc& F, const LevelDesc& C,
                                               long long j) {
  if (F.sparse) {
    const int S = F.S, S3 = S * S * S;
    const int b = (int)(j / S3);
    const int l = (int)(j % S3);
    const int x = l % S, y = (l / S) % S, z = l / (S * S);
    if (C.sparse) {
      const int SC = C.S;
      return (long long)b * SC * SC * SC + ((z >> 1) * SC + (y >> 1)) * SC + (x >> 1);
    }
    const int bx = g.coord[3 * b] - g.blo[0], by = g.coord[3 * b + 1] - g.blo[1], bz = g.coord[3 * b + 2] - g.blo[2];
    return ((long long)bz * C.dim[1] + by) * C.dim[0] + bx;
  }
  const int x = (int)(j % F.dim[0]), y = (int)((j / F.dim[0]) % F.dim[1]),
            z = (int)(j / ((long long)F.dim[0] * F.dim[1]));
  return ((long long)(z >> 1) * C.dim[1] + (y >> 1)) * C.dim[0] + (x >> 1);
}

// ---- the context's particle state as seen by the snapshot queue (fl_snapshot.cu)
struct SnapshotSource {
  const float* base;  // 15 arrays of pcap floats: x[3], v[3], C rows [9]
  size_t pcap;
  unsigned long long count;
  int buffer;  // which of the context's two particle buffers holds the state
  int device;
  GridView g;  // lattice (origin, inv_h, blo, bdim) for the position check
};

}  // namespace fl

struct fl_context;
namespace fl {
void context_snapshot_source(::fl_context* c, SnapshotSource* out);
// Event recorded after every snapshot copy of particle buffer `buffer`; writes into it wait on it.
cudaEvent_t context_buffer_fence(::fl_context* c, int buffer);
void context_attach_snapshot_queue(::fl_context* c, int delta);
// FL_OK when an sm_100 device is current, else FL_FAILED_PRECONDITION.
int check_device();
}  // namespace fl

// ---- bounded MAC pressure projection (fl_mac_pressure.cu) ----
#include <vector>

#include "../../include/fluidity_b200.h"
namespace fl {
// A face of the reference's owned sparse grid as (4^3 block z, y, x, normal
// axis, local z, y, x): its owned-slot order.
struct OwnedFaceKey {
  int32_t v[7];
  bool operator<(const OwnedFaceKey& o) const {
    for (int k = 0; k < 7; ++k)
      if (v[k] != o.v[k]) return v[k] < o.v[k];
    return false;
  }
  bool operator==(const OwnedFaceKey& o) const {
    for (int k = 0; k < 7; ++k)
      if (v[k] != o.v[k]) return false;
    return true;
  }
};
// Host and device scratch of one projection. reserve_caps() sizes every part
// for the operator's caps (4096 cells, 24576 faces) once, after which
// projections through it allocate nothing; a scratch left empty grows for the
// call.
struct MpScratch {
  std::vector<int> tail, head, cell_off, cell_ent, fill, parent, root, comp_of, gauges, comp_cell_off, comp_cells,
      comp_face_off, comp_faces, host_ints;
  std::vector<int> lut;  // cell ordinal per lattice position of the cells' bounding box (-1: none), when it fits
  std::vector<unsigned char> anchored, pinned;
  std::vector<double> hp, hr, hd, hb, hu;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool reserve_caps();
  void release();  // the device arena
  void destroy();  // arena and events
};
// fl_project_mac_pressure_3d's work on a caller's scratch and stream (NULL:
// the default stream).
int mp_project(MpScratch& scratch, cudaStream_t stream, double h, double dt, const int32_t* cell_index,
               const double* cell_values, uint64_t cell_count, const int32_t* face_index, const int32_t* face_kind,
               const double* face_values, uint64_t face_count, int max_iterations, double rel_tol, double* pressure,
               double* corrected_u, double* rhs, double* residual, double* defect, uint64_t* gauge_ordinals,
               fl_mac_pressure_diagnostics* diagnostics, fl_measurement* measurement);
}  // namespace fl
