// Host orchestration and the extern "C" boundary of the liquid-step hot path.
//
// The context is the resident device arena (the role of the reference's
// CudaLiquidSubstepBackend3D arena, native/include/fluidity/host/
// cuda_liquid_substep_3d.h:28-81): every buffer is allocated once, at
// creation, for the full block lattice and the declared particle capacity
// (the two extra particle buffers of staged inputs at the first
// fl_stage_particles), so a step allocates nothing. Kernels report arithmetic failures through a
// device report (native/cuda/transfer_3d_bridge.h:49-57) that the host reads
// after synchronizing, and failing calls publish nothing the caller owns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"
#include "fl_unet.h"

namespace fl {
unsigned long long g_kernel_launches = 0;
unsigned long long g_library_launches = 0;
cudaError_t launch_deposit_quanta(const GridView& g, const double* parts, unsigned long long n,
                                  const double origin[3], double h, double mass_per_quantum,
                                  double momentum_per_quantum, double limit, unsigned long long* const mq[3],
                                  unsigned long long* const pq[3], DeviceReport* rep, cudaStream_t s);
}

using namespace fl;

constexpr int kStateBuffers = 4;

struct fl_context {
  int device = 0;
  fl_grid_desc desc{};
  size_t pcap = 0;
  int lattice = 0;  // blocks in the lattice
  int nb = 0;       // active blocks
  // topology
  unsigned char* occ = nullptr;
  int* flag = nullptr;
  int* ordinal = nullptr;
  int* table = nullptr;
  int* coord = nullptr;
  int* nbr27 = nullptr;
  int* nb_dev = nullptr;
  int* nb_host = nullptr;
  // sort
  unsigned int *keys = nullptr, *index = nullptr, *index_alt = nullptr;
  int* counts = nullptr;
  int* cell_start = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0;
  // particles (ping-pong, 16 arrays each incl. mass)
  // Particle buffers: two at creation, four once a next input is staged.
  float* pbuf[kStateBuffers] = {};
  int nbuf = 2;
  int cur = 0;
  // fence[b]: recorded by a snapshot queue after its copy of buffer b; every
  // write into buffer b waits on it (a never-recorded event is complete)
  cudaEvent_t fence[kStateBuffers] = {};
  int snapshot_queues = 0;  // live fl_snapshot_queue objects over this context
  // Staged next inputs (fl_stage_particles), oldest first: buffer, count, and
  // the event recorded on the staging stream after the buffer's copies.
  int stage_buf[2] = {-1, -1};
  uint64_t stage_count[2] = {0, 0};
  int nstage = 0;
  cudaEvent_t staged[kStateBuffers] = {};
  cudaStream_t stage_stream = nullptr;
  uint64_t count = 0;
  // faces
  float* u_pred[3] = {};
  float* u_new[3] = {};
  float* fmass[3] = {};
  float2* tiles = nullptr;
  // pressure
  unsigned char* type = nullptr;
  double* b64 = nullptr;
  double* p64 = nullptr;
  float* r[2] = {};
  float* d[2] = {};
  float* q = nullptr;
  float* e = nullptr;
  double* partial = nullptr;
  SolverState* st = nullptr;
  SolverState* st_host = nullptr;
  // multigrid storage (x and k sized for FP32; BF16 uses the first half)
  int max_levels = 0;
  unsigned char* lv_fluid[12] = {};
  unsigned char* lv_mask0 = nullptr;
  void* lv_k[12][3] = {};
  float* lv_anchor[12] = {};
  float* lv_diag[12] = {};
  void* lv_x[12] = {};
  float* lv_b[12] = {};
  long long lv_cap[12] = {};
  DeviceReport* rep = nullptr;
  DeviceReport* rep_host = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool in_step = false;  // fl_step keeps one device report across its stages
  cudaEvent_t phase[5] = {};  // topology+sort | P2G | pressure | G2P boundaries of the last fl_step
  bool phases_valid = false;
  // pressure solver: own stream (graph capture needs a non-legacy stream), the
  // replayed two-iteration FCG graph, handoff events and the natural-layout pressure
  cudaStream_t work = nullptr;
  cudaStream_t cap = nullptr;  // graph capture only (overlaps the solver's setup on `work`)
  long long fcg_key[8] = {};   // what the executable graphs were captured for
  long long fcg_nn_key[8] = {};
  cudaGraphExec_t fcg_exec = nullptr;
  unsigned long long fcg_graph_kernels = 0;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  double* p_nat = nullptr;
  float* p_keep = nullptr;  // last pressure per lattice cell (warm start across topology changes)
  bool p_keep_valid = false;
  float* p_keep_prev = nullptr;  // the one before it (warm start by linear extrapolation)
  bool p_keep_prev_valid = false;
  bool occ_ready = false;  // occ holds the blocks of the current state (marked by the last fl_step's G2P)
  // learned preconditioner: FP32 parameters, per-block scales, the inference
  // activations (grown on demand to the active block count) and its own
  // one-iteration FCG graph
  float* nn_params = nullptr;
  bool nn_ready = false;
  float* nn_scale = nullptr;
  float* nn_act = nullptr;  // FP32 training-forward activations (checking path)
  long long nn_act_items = 0;
  __nv_bfloat16* nn_packed = nullptr;  // BF16 conv weights for the tensor-core kernels
  uint4* nn_tc = nullptr;              // BF16 activation columns, zeroed at allocation
  float* nn_bt = nullptr;
  long long nn_tc_items = 0;
  int sms = 0;
  cudaGraphExec_t fcg_nn_exec = nullptr;
  unsigned long long fcg_nn_kernels = 0;
  PrecondHook nn_hook{};
};

namespace {

int Code(cudaError_t e) { return e == cudaSuccess ? FL_OK : FL_INTERNAL; }

#define FL_CUDA(expr)                    \
  do {                                   \
    cudaError_t fl_e_ = (expr);          \
    if (fl_e_ != cudaSuccess) return Code(fl_e_); \
  } while (0)

int device_ready() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FL_FAILED_PRECONDITION;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  // one attribute query (a full property query costs milliseconds per call)
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return FL_FAILED_PRECONDITION;
  }
  if (major != 10) return FL_FAILED_PRECONDITION;  // image is sm_100a only
  return FL_OK;
}

template <typename T>
int dalloc(T** p, size_t count) {
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count) == cudaSuccess ? FL_OK : FL_RESOURCE_EXHAUSTED;
}

GridView view(const fl_context* c) {
  GridView g{};
  for (int d = 0; d < 3; ++d) {
    g.origin[d] = (float)c->desc.origin[d];
    g.blo[d] = c->desc.block_lo[d];
    g.bdim[d] = c->desc.block_dim[d];
    g.solid_lo[d] = c->desc.solid_lo[d];
    g.solid_hi[d] = c->desc.solid_hi[d];
  }
  g.h = (float)c->desc.h;
  g.inv_h = (float)(1.0 / c->desc.h);
  g.nb = c->nb;
  g.table = c->table;
  g.coord = c->coord;
  g.nbr27 = c->nbr27;
  return g;
}

ParticlesView pview(const fl_particles* p) {
  ParticlesView v{};
  for (int d = 0; d < 3; ++d) {
    v.x[d] = p->x[d];
    v.v[d] = p->v[d];
  }
  for (int d = 0; d < 9; ++d) v.c[d] = p->c[d];
  v.mass = p->mass;
  v.count = p->count;
  return v;
}

fl_particles state_particles(fl_context* c, int which) {
  fl_particles p{};
  float* base = c->pbuf[which];
  for (int d = 0; d < 3; ++d) {
    p.x[d] = base + (size_t)d * c->pcap;
    p.v[d] = base + (size_t)(3 + d) * c->pcap;
  }
  for (int d = 0; d < 9; ++d) p.c[d] = base + (size_t)(6 + d) * c->pcap;
  p.mass = nullptr;
  p.count = c->count;
  return p;
}

// Orders `s` after every snapshot copy of any particle buffer.
void wait_state_fences(fl_context* c, cudaStream_t s) {
  for (int b = 0; b < c->nbuf; ++b) cudaStreamWaitEvent(s, c->fence[b], 0);
}

// A particle buffer to write next: not in `exclude` (bit per buffer),
// preferring one whose last snapshot copy has finished, so that the write
// need not wait; otherwise the lowest candidate (its fence orders the write).
int pick_buffer(fl_context* c, unsigned exclude) {
  int fallback = -1;
  for (int b = 0; b < c->nbuf; ++b) {
    if (exclude & (1u << b)) continue;
    const cudaError_t q = cudaEventQuery(c->fence[b]);
    if (q == cudaSuccess) return b;
    if (q == cudaErrorNotReady && cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    if (fallback < 0) fallback = b;
  }
  return fallback;
}

unsigned staged_mask(const fl_context* c) {
  unsigned m = 0;
  for (int k = 0; k < c->nstage; ++k) m |= 1u << c->stage_buf[k];
  return m;
}

int read_report(fl_context* c, cudaStream_t s, fl_report* out) {
  FL_CUDA(cudaMemcpyAsync(c->rep_host, c->rep, sizeof(DeviceReport), cudaMemcpyDeviceToHost, s));
  FL_CUDA(cudaStreamSynchronize(s));
  if (out) {
    out->compiled_architecture = c->rep_host->compiled_architecture;
    out->error = c->rep_host->error;
    out->first_bad_index = c->rep_host->first_bad_index;
  }
  return c->rep_host->error;
}

int reset_report(fl_context* c, cudaStream_t s) {
  if (c->in_step) return FL_OK;
  FL_CUDA(cudaMemsetAsync(c->rep, 0, sizeof(DeviceReport), s));
  return FL_OK;
}

int dense_dim(int bdim, int l) {  // level l >= 3 extent along one axis
  int v = bdim;
  for (int k = 3; k < l; ++k) v = (v + 1) / 2;
  return v;
}

int auto_levels(const fl_context* c) {
  for (int L = 4; L <= c->max_levels; ++L) {
    long long n = 1;
    for (int d = 0; d < 3; ++d) n *= dense_dim(c->desc.block_dim[d], L - 1);
    if (n <= 512) return L;
  }
  return c->max_levels;
}

template <typename T>
int make_hierarchy(fl_context* c, int levels, MgHierarchy<T>& H) {
  if (levels < 4 || levels > c->max_levels) return FL_INVALID_ARGUMENT;
  H.levels = levels;
  for (int l = 0; l < levels; ++l) {
    LevelDesc D{};
    if (l < 3) {
      D.sparse = 1;
      D.S = 8 >> l;
      D.count = (long long)c->nb * D.S * D.S * D.S;
      D.dim[0] = D.dim[1] = D.dim[2] = 0;
      D.parity = 0;
    } else {
      D.sparse = 0;
      D.S = 0;
      D.count = 1;
      int par = 0;
      for (int d = 0; d < 3; ++d) {
        D.dim[d] = dense_dim(c->desc.block_dim[d], l);
        D.count *= D.dim[d];
        par += c->desc.block_lo[d] >> (l - 3);
      }
      D.parity = par & 1;
    }
    H.desc[l] = D;
    LevelPtrs<T> P{};
    P.mask = l == 0 ? c->lv_mask0 : nullptr;
    P.fluid = c->lv_fluid[l];
    for (int a = 0; a < 3; ++a) P.k[a] = reinterpret_cast<T*>(c->lv_k[l][a]);
    P.anchor = c->lv_anchor[l];
    P.diag = c->lv_diag[l];
    P.x = reinterpret_cast<T*>(c->lv_x[l]);
    H.ptr[l] = P;
    H.b[l] = c->lv_b[l];
  }
  const LevelDesc& C = H.desc[levels - 1];
  if (C.count > 8192) return FL_RESOURCE_EXHAUSTED;  // coarsest must fit one CTA's shared memory
  return FL_OK;
}

__global__ void k_init_state(SolverState* st, double rel_tol, double inner_rtol, int inner_max, int learned,
                             int stall_limit, double stall_ratio) {
  st->rr_best = INFINITY;
  st->stall_ratio2 = stall_ratio * stall_ratio;
  st->learned = learned;
  st->stall_limit = stall_limit;
  st->stalls = 0;
  st->fallback = 0;
  st->learned_iter = 0;
  st->nn_error = 0;
  st->target = 0.0;
  st->inner_rtol = inner_rtol;
  st->inner_max = inner_max;
  st->total_iter = 0;
  st->status = 0;
  st->done = 0;
  st->converged = 0;
  st->ticket = 0;
  st->rz = st->rz_prev = st->beta = st->alpha = st->rr = 0.0;
  st->res64 = 0.0;
  st->stop2 = 0.0;
  st->div_l2 = st->div_max = 0.0;
  (void)rel_tol;
}

__global__ void k_set_target(SolverState* st, double rel_tol) { st->target = rel_tol * st->b_norm; }

__global__ void k_set_inner_budget(SolverState* st, int inner_max) {
  st->inner_max = inner_max;
  st->done = st->converged;
}

// Captures two flexible-CG iterations (V-cycle + 3 CG kernels each, r/d
// buffers swapping roles) into one graph and updates the executable graph in
// place when only launch parameters changed (the block count changes per step).
// The learned variant runs the network in place of the V-cycle. The host picks
// the graph per replay, so the V-cycle takes over at the first replay after the
// device flags the fallback (at most one further learned iteration).
template <typename T>
int capture_fcg(fl_context* c, const GridView& g, const MgHierarchy<T>& H, const MgOptions& mo, bool learned,
                cudaGraphExec_t* exec, unsigned long long* kernels) {
  cudaGraph_t graph = nullptr;
  const unsigned long long before = g_kernel_launches;
  const int a = 0, b = 1;
  FL_CUDA(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal));
  cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
  if (learned) {
    e1 = launch_fcg_iteration<T>(g, H, mo, c->r[a], c->r[b], c->d[a], c->d[b], c->q, c->e, c->partial, c->st,
                                 &c->st->done, c->cap, &c->nn_hook);
    e2 = launch_fcg_iteration<T>(g, H, mo, c->r[b], c->r[a], c->d[b], c->d[a], c->q, c->e, c->partial, c->st,
                                 &c->st->done, c->cap, &c->nn_hook);
  } else {
    e1 = launch_fcg_iteration<T>(g, H, mo, c->r[a], c->r[b], c->d[a], c->d[b], c->q, c->e, c->partial, c->st,
                                 &c->st->done, c->cap);
    e2 = launch_fcg_iteration<T>(g, H, mo, c->r[b], c->r[a], c->d[b], c->d[a], c->q, c->e, c->partial, c->st,
                                 &c->st->done, c->cap);
  }
  cudaError_t e3 = cudaStreamEndCapture(c->cap, &graph);
  *kernels = g_kernel_launches - before;
  g_kernel_launches = before;  // counted again at every replay
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return FL_INTERNAL;
  }
  bool updated = false;
  if (*exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(*exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(*exec);
      *exec = nullptr;
    }
  }
  if (!updated) {
    if (cudaGraphInstantiate(exec, graph, 0) != cudaSuccess) {
      cudaGraphDestroy(graph);
      *exec = nullptr;
      return FL_INTERNAL;
    }
  }
  cudaGraphDestroy(graph);
  return FL_OK;
}

// Learned preconditioner application z = s * U(r / s) per block: the
// tensor-core kernels (BF16 activations, FP32 accumulation) on the solver's
// vectors. Captured into the learned FCG graph.
template <typename T>
cudaError_t nn_apply(void* vc, const float* r, void* z, cudaStream_t s) {
  fl_context* c = static_cast<fl_context*>(vc);
  const GridView g = view(c);
  return unet_tc_apply<T>(g, c->nn_params, c->nn_packed, c->nn_tc, c->nn_tc_items, c->nn_bt, c->nn_scale, c->type,
                          r, static_cast<T*>(z), &c->st->nn_error, c->sms, s, c->nn_hook.compose != 0);
}

int nn_reserve_tc(fl_context* c, long long items) {
  if (items <= c->nn_tc_items) return FL_OK;
  cudaFree(c->nn_tc);
  cudaFree(c->nn_bt);
  c->nn_tc = nullptr;
  c->nn_bt = nullptr;
  c->nn_tc_items = 0;
  const long long want = std::min<long long>(items + items / 4 + 16, c->lattice);
  const UNetTcLayout L = unet_tc_layout();
  const size_t bytes = sizeof(uint4) * (size_t)(L.rows_per_block * want);
  if (cudaMalloc(&c->nn_tc, bytes) != cudaSuccess ||
      cudaMalloc(&c->nn_bt, sizeof(float) * (size_t)(L.bt_floats_per_block * want)) != cudaSuccess) {
    cudaGetLastError();
    return FL_RESOURCE_EXHAUSTED;
  }
  // pads are read as zeros and never written (tensors are based on the allocated
  // capacity, so their columns never move while this allocation lives)
  if (cudaMemset(c->nn_tc, 0, bytes) != cudaSuccess) return FL_INTERNAL;
  c->nn_tc_items = want;
  return FL_OK;
}

// FP32 training-forward path over the same gathered windows (for checking the
// tensor-core kernels).
int nn_reserve(fl_context* c, long long items) {
  if (items <= c->nn_act_items) return FL_OK;
  cudaFree(c->nn_act);
  c->nn_act = nullptr;
  c->nn_act_items = 0;
  const long long want = std::min<long long>(items + items / 4 + 16, c->lattice);
  if (cudaMalloc(&c->nn_act, sizeof(float) * (size_t)unet_cache_layout((int)want).activations) != cudaSuccess) {
    cudaGetLastError();
    return FL_RESOURCE_EXHAUSTED;
  }
  c->nn_act_items = want;
  return FL_OK;
}

template <typename T>
int pressure_solve(fl_context* c, const float* const u_pred[3], float* const u_new[3], const fl_transfer_params* tp,
                   const fl_pressure_options* opt, fl_pressure_diagnostics* diag, double* pressure_out,
                   cudaStream_t user) {
  GridView g = view(c);
  MgHierarchy<T> H{};
  const int levels = opt->levels > 0 ? opt->levels : auto_levels(c);
  int st = make_hierarchy<T>(c, levels, H);
  if (st != FL_OK) return st;
  const double h = c->desc.h, dt = tp->dt, rho = tp->density;
  const double k_ref = dt * h / rho;          // conductance of a full open face
  const double rhs_scale = (h * h) / k_ref;   // b' = -(h^2 sum_out u)/k_ref
  const double vel_scale = dt / (rho * h);    // u += vel_scale * (p_tail - p_head)
  const long long n = (long long)c->nb * kBlockCells;
  MgOptions mo{std::max(1, opt->pre_sweeps), std::max(1, opt->post_sweeps), std::max(1, opt->coarse_sweeps)};
  const bool use_nn = opt->preconditioner == 1 || opt->preconditioner == 2;
  if (opt->preconditioner != 0 && !use_nn) return FL_INVALID_ARGUMENT;
  if (use_nn) {
    if (!c->nn_ready) return FL_FAILED_PRECONDITION;
    st = nn_reserve_tc(c, c->nb);
    if (st != FL_OK) return st;
    c->nn_hook.apply = nn_apply<T>;
    c->nn_hook.ctx = c;
    c->nn_hook.compose = opt->preconditioner == 2 ? 1 : 0;
  }
  const int stall_limit = opt->stall_limit > 0 ? opt->stall_limit : 3;
  const double stall_ratio = opt->stall_ratio > 0.0 ? opt->stall_ratio : 0.9;
  cudaStream_t s = c->work;
  FL_CUDA(cudaEventRecord(c->ev_in, user));
  FL_CUDA(cudaStreamWaitEvent(s, c->ev_in, 0));
  FL_CUDA(cudaEventRecord(c->ev0, s));
  ++g_kernel_launches;
  k_init_state<<<1, 1, 0, s>>>(c->st, opt->rel_tol, opt->inner_rtol, opt->max_iterations, use_nn ? 1 : 0,
                               stall_limit, stall_ratio);
  const float* p_prev = (opt->warm_start && c->p_keep_valid) ? c->p_keep : nullptr;
  const float* p_prev2 = (opt->warm_start == 2 && p_prev && c->p_keep_prev_valid) ? c->p_keep_prev : nullptr;
  FL_CUDA(launch_pressure_setup<T>(g, c->cell_start, c->type, u_pred, rhs_scale, H, c->b64, c->p64, p_prev, p_prev2,
                                   c->partial, c->st, s));
  ++g_kernel_launches;
  k_set_target<<<1, 1, 0, s>>>(c->st, opt->rel_tol);
  FL_CUDA(cudaMemsetAsync(c->lv_x[0], 0, sizeof(T) * (size_t)n, s));
  FL_CUDA(cudaMemsetAsync(c->d[0], 0, sizeof(float) * (size_t)n, s));
  FL_CUDA(cudaMemsetAsync(c->d[1], 0, sizeof(float) * (size_t)n, s));
  FL_CUDA(cudaMemsetAsync(c->r[1], 0, sizeof(float) * (size_t)n, s));
  int total = 0, refinements = 0;
  bool converged = false;
  int status = FL_OK;
  const int max_ref = std::max(1, opt->max_refinements);
  // (Re)capture the FCG graphs on the capture stream while `work` runs the
  // setup; skipped when the block count and options match the last capture
  // (pointers are fixed for the context's lifetime, grid sizes follow nb).
  {
    const long long key[8] = {c->nb, levels, mo.pre, mo.post, mo.coarse_sweeps, (long long)sizeof(T), 1, 0};
    if (!c->fcg_exec || std::memcmp(key, c->fcg_key, sizeof(key)) != 0) {
      st = capture_fcg<T>(c, g, H, mo, false, &c->fcg_exec, &c->fcg_graph_kernels);
      if (st != FL_OK) return st;
      std::memcpy(c->fcg_key, key, sizeof(key));
    }
    if (use_nn) {
      const long long nkey[8] = {c->nb, levels, mo.pre, mo.post, mo.coarse_sweeps,
                                 (long long)sizeof(T) + 16 * c->nn_hook.compose, (long long)(uintptr_t)c->nn_tc,
                                 c->nn_tc_items};
      if (!c->fcg_nn_exec || std::memcmp(nkey, c->fcg_nn_key, sizeof(nkey)) != 0) {
        st = capture_fcg<T>(c, g, H, mo, true, &c->fcg_nn_exec, &c->fcg_nn_kernels);
        if (st != FL_OK) return st;
        std::memcpy(c->fcg_nn_key, nkey, sizeof(nkey));
      }
    }
  }
  for (int outer = 0; outer <= max_ref; ++outer) {
    FL_CUDA(launch_residual64<T>(g, H, c->b64, c->p64, c->r[0], c->e, c->partial, c->st, s));
    FL_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
    FL_CUDA(cudaStreamSynchronize(s));
    if (c->st_host->converged) {
      converged = true;
      break;
    }
    if (outer == max_ref || total >= opt->max_iterations) break;
    ++refinements;
    ++g_kernel_launches;
    k_set_inner_budget<<<1, 1, 0, s>>>(c->st, opt->max_iterations - total);
    for (;;) {
      const bool nn_now = use_nn && !c->st_host->fallback;
      FL_CUDA(cudaGraphLaunch(nn_now ? c->fcg_nn_exec : c->fcg_exec, s));
      g_kernel_launches += nn_now ? c->fcg_nn_kernels : c->fcg_graph_kernels;
      FL_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
      FL_CUDA(cudaStreamSynchronize(s));
      if (c->st_host->done) break;
    }
    total = c->st_host->total_iter;
    if (c->st_host->nn_error) {
      status = FL_INTERNAL;
      break;
    }
    if (c->st_host->status != 0) {
      status = c->st_host->status;
      break;
    }
    FL_CUDA(launch_accumulate(g, c->e, c->p64, s));
  }
  FL_CUDA(launch_correct_faces(g, c->type, c->p64, u_pred, u_new, vel_scale, c->partial, c->st, s));
  // The kept copy is rewritten in full: cells that are not fluid now read back as 0.
  std::swap(c->p_keep, c->p_keep_prev);  // the last pressure becomes the one before
  c->p_keep_prev_valid = c->p_keep_valid;
  FL_CUDA(cudaMemsetAsync(c->p_keep, 0, sizeof(float) * (size_t)c->lattice * kBlockCells, s));
  FL_CUDA(launch_export_pressure(g, c->p64, c->p_nat, c->p_keep, s));
  c->p_keep_valid = true;
  FL_CUDA(cudaEventRecord(c->ev1, s));
  if (pressure_out) FL_CUDA(cudaMemcpyAsync(pressure_out, c->p_nat, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  FL_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
  FL_CUDA(cudaEventRecord(c->ev_out, s));
  FL_CUDA(cudaStreamWaitEvent(user, c->ev_out, 0));
  FL_CUDA(cudaStreamSynchronize(s));
  const SolverState& S = *c->st_host;
  if (diag) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    diag->status = status;
    diag->iterations = S.total_iter;
    diag->refinements = refinements;
    diag->levels = levels;
    diag->active_blocks = c->nb;
    diag->fluid_cells = 0;
    diag->rhs_l2 = S.b_norm * k_ref;
    diag->true_residual_l2 = S.res64 * k_ref;
    diag->relative_residual = S.b_norm > 0 ? S.res64 / S.b_norm : 0.0;
    diag->reference_limit = 2e-6 + 2e-6 * diag->rhs_l2;
    diag->max_volume_residual = S.res64 * k_ref / (h * h * h);
    diag->max_divergence = S.div_max / h;
    diag->solve_ms = ms;
    diag->learned_iterations = S.learned_iter;
    diag->fell_back = S.fallback;
  }
  if (status != FL_OK) return status;
  return converged ? FL_OK : FL_ABORTED;
}

template <typename T>
int apply_vcycle(fl_context* c, const float* r, float* z, const fl_pressure_options* opt, cudaStream_t s) {
  GridView g = view(c);
  MgHierarchy<T> H{};
  const int levels = opt->levels > 0 ? opt->levels : auto_levels(c);
  int st = make_hierarchy<T>(c, levels, H);
  if (st != FL_OK) return st;
  MgOptions mo{std::max(1, opt->pre_sweeps), std::max(1, opt->post_sweeps), std::max(1, opt->coarse_sweeps)};
  const long long n = (long long)c->nb * kBlockCells;
  ++g_kernel_launches;
  k_init_state<<<1, 1, 0, s>>>(c->st, 1e-6, 1e-4, 1, 0, 3, 0.9);
  const float* up[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  for (int a = 0; a < 3; ++a) FL_CUDA(cudaMemsetAsync(c->u_pred[a], 0, sizeof(float) * n, s));
  FL_CUDA(launch_pressure_setup<T>(g, c->cell_start, c->type, up, 1.0, H, c->b64, c->p64, nullptr, nullptr, c->partial,
                                   c->st, s));
  FL_CUDA(cudaMemsetAsync(c->lv_x[0], 0, sizeof(T) * (size_t)n, s));
  FL_CUDA(launch_to_rb(g, r, c->r[0], s));
  FL_CUDA(launch_apply_vcycle<T>(g, H, c->r[0], mo, &c->st->done, s));
  FL_CUDA(launch_to_natural<T>(g, H, z, s));
  FL_CUDA(cudaStreamSynchronize(s));
  return FL_OK;
}

// Reference 4^3 layout helpers for the reference-shaped operators.
struct RefLayout {
  std::vector<std::array<int, 3>> blocks4;  // sorted (z,y,x)
  std::vector<std::array<int, 3>> blocks8;  // sorted (z,y,x)
  int blo[3], bdim[3];
  std::vector<int> table;  // lattice -> 8^3 ordinal
};

int floor_div(int v, int k) { return v >= 0 ? v / k : -((-v + k - 1) / k); }

void make_layout(const int32_t* blocks, uint64_t nb4, RefLayout& L) {
  L.blocks4.resize(nb4);
  for (uint64_t i = 0; i < nb4; ++i) L.blocks4[i] = {blocks[3 * i], blocks[3 * i + 1], blocks[3 * i + 2]};
  auto key = [](const std::array<int, 3>& b) { return std::make_tuple(b[2], b[1], b[0]); };
  std::sort(L.blocks4.begin(), L.blocks4.end(), [&](auto& a, auto& b) { return key(a) < key(b); });
  std::map<std::tuple<int, int, int>, std::array<int, 3>> b8;
  for (auto& b : L.blocks4) {
    std::array<int, 3> c = {floor_div(b[0], 2), floor_div(b[1], 2), floor_div(b[2], 2)};
    b8[key(c)] = c;
  }
  // include one ring of 8^3 blocks so every stencil node has storage
  std::map<std::tuple<int, int, int>, std::array<int, 3>> ring = b8;
  for (auto& kv : b8)
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          std::array<int, 3> c = {kv.second[0] + dx, kv.second[1] + dy, kv.second[2] + dz};
          ring[key(c)] = c;
        }
  L.blocks8.clear();
  for (auto& kv : ring) L.blocks8.push_back(kv.second);
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (auto& b : L.blocks8)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], b[d]);
      hi[d] = std::max(hi[d], b[d]);
    }
  for (int d = 0; d < 3; ++d) {
    L.blo[d] = L.blocks8.empty() ? 0 : lo[d];
    L.bdim[d] = L.blocks8.empty() ? 1 : hi[d] - lo[d] + 1;
  }
  L.table.assign((size_t)L.bdim[0] * L.bdim[1] * L.bdim[2], -1);
  for (size_t o = 0; o < L.blocks8.size(); ++o) {
    auto& b = L.blocks8[o];
    L.table[((size_t)(b[2] - L.blo[2]) * L.bdim[1] + (b[1] - L.blo[1])) * L.bdim[0] + (b[0] - L.blo[0])] = (int)o;
  }
}

// Reference slot s -> (axis, 8^3 face slot) in this library's layout.
void slot_map(const RefLayout& L, std::vector<int>& axis, std::vector<long long>& slot8) {
  const size_t fc = L.blocks4.size() * 192;
  axis.resize(fc);
  slot8.resize(fc);
  for (size_t s = 0; s < fc; ++s) {
    const auto& b = L.blocks4[s / 192];
    const int within = (int)(s % 192);
    const int a = within / 64, local = within % 64;
    const int x = 4 * b[0] + local % 4, y = 4 * b[1] + (local / 4) % 4, z = 4 * b[2] + local / 16;
    const int bx = floor_div(x, 8), by = floor_div(y, 8), bz = floor_div(z, 8);
    const int o = L.table[((size_t)(bz - L.blo[2]) * L.bdim[1] + (by - L.blo[1])) * L.bdim[0] + (bx - L.blo[0])];
    axis[s] = a;
    slot8[s] = (long long)o * 512 + ((z - 8 * bz) * 64 + (y - 8 * by) * 8 + (x - 8 * bx));
  }
}

int validate_particles(const double* parts, uint64_t np, double h, bool need_mass) {
  for (uint64_t i = 0; i < np; ++i) {
    const double* q = parts + 19 * i;
    for (int k = 0; k < 6; ++k)
      if (!std::isfinite(q[k])) return FL_INVALID_ARGUMENT;
    if (need_mass) {
      if (!std::isfinite(q[6]) || q[6] < 0.0) return FL_INVALID_ARGUMENT;
      for (int k = 7; k < 19; ++k)
        if (!std::isfinite(q[k])) return FL_INVALID_ARGUMENT;
    }
    for (int d = 0; d < 3; ++d)
      if (2.0 * std::fabs(q[d] - q[3 + d]) > h) return FL_FAILED_PRECONDITION;  // motion beyond h/2
  }
  return FL_OK;
}

struct TempContext {
  fl_context* ctx = nullptr;
  ~TempContext() {
    if (ctx) fl_context_destroy(ctx);
  }
};

int make_ref_context(const double origin[3], double h, const RefLayout& L, uint64_t np, TempContext& tc) {
  fl_grid_desc d{};
  for (int k = 0; k < 3; ++k) {
    d.origin[k] = origin[k];
    d.block_lo[k] = L.blo[k];
    d.block_dim[k] = L.bdim[k];
    d.solid_lo[k] = INT_MIN;
    d.solid_hi[k] = INT_MAX;
  }
  d.h = h;
  int st = fl_context_create(&d, std::max<uint64_t>(np, 1), &tc.ctx);
  if (st != FL_OK) return st;
  std::vector<int32_t> coords;
  for (auto& b : L.blocks8) {
    coords.push_back(b[0]);
    coords.push_back(b[1]);
    coords.push_back(b[2]);
  }
  return fl_topology_from_blocks(tc.ctx, coords.data(), L.blocks8.size());
}

// Uploads AoS FP64 particles (trial positions) into the context's spare buffer
// as FP32 SoA with per-particle mass, sorts them into the state buffer.
int upload_ref_particles(fl_context* c, const double* parts, uint64_t np, cudaStream_t s, std::vector<float>& soa) {
  const size_t cap = c->pcap;
  soa.assign(16 * cap, 0.0f);
  for (uint64_t i = 0; i < np; ++i) {
    const double* q = parts + 19 * i;
    for (int d = 0; d < 3; ++d) soa[d * cap + i] = (float)q[3 + d];
    for (int d = 0; d < 3; ++d) soa[(3 + d) * cap + i] = (float)q[7 + d];
    for (int k = 0; k < 9; ++k) soa[(6 + k) * cap + i] = (float)q[10 + k];
    soa[15 * cap + i] = (float)q[6];
  }
  FL_CUDA(cudaMemcpyAsync(c->pbuf[1], soa.data(), sizeof(float) * 16 * cap, cudaMemcpyHostToDevice, s));
  c->count = np;
  fl_particles in = state_particles(c, 1), out = state_particles(c, 0);
  in.mass = c->pbuf[1] + 15 * cap;
  out.mass = c->pbuf[0] + 15 * cap;
  c->cur = 0;
  fl_report rep{};
  int st = fl_sort_particles_by_block(c, &in, &out, s, &rep);
  if (st != FL_OK) return st;
  return rep.error;
}

}  // namespace

// ======================================================================= C-ABI

// G2P on sorted particles; occ_next (step mode only) receives the blocks of the
// advected positions for the next topology.
// With `order` (step mode), particle q of the cell order is read from `in` at
// order[q] and written to `sorted` at q.
int g2p_impl(fl_context* c, fl_particles* sorted, const float* const u_new[3], const float* const u_old[3], float dt,
             float* full_out, cudaStream_t s, fl_report* report, unsigned char* occ_next,
             const unsigned int* order = nullptr, const fl_particles* in = nullptr) {
  reset_report(c, s);
  GridView g = view(c);
  ParticlesView pv = pview(sorted);
  G2PParams prm{};
  prm.dt = dt;
  prm.occ_next = full_out ? nullptr : occ_next;
  if (order != nullptr && in != nullptr && full_out == nullptr) {
    prm.order = order;
    for (int d = 0; d < 3; ++d) prm.x_in[d] = in->x[d];
  }
  for (int d = 0; d < 3; ++d) {
    const double lo = c->desc.solid_lo[d] == INT_MIN ? -1e30 : c->desc.origin[d] + (c->desc.solid_lo[d] + 1e-3) * c->desc.h;
    const double hi =
        c->desc.solid_hi[d] == INT_MAX ? 1e30 : c->desc.origin[d] + (c->desc.solid_hi[d] + 1 - 1e-3) * c->desc.h;
    prm.clamp_lo[d] = (float)lo;
    prm.clamp_hi[d] = (float)hi;
  }
  FL_CUDA(launch_g2p(g, pv, c->cell_start, u_new, u_old, prm, full_out, c->rep, s));
  if (report) return read_report(c, s, report);
  return FL_OK;
}

// Active blocks of the state about to be stepped: from the occupancy the last
// step's G2P marked when it is current, else by marking the particles; then
// occ is cleared for this step's G2P to mark.
int step_topology(fl_context* c, const fl_particles* p, cudaStream_t s, fl_report* report) {
  if (!c->occ_ready) return fl_topology_from_particles(c, p, s, report);
  reset_report(c, s);
  GridView g = view(c);
  FL_CUDA(launch_topology_from_occupancy(g, c->occ, c->flag, c->ordinal, c->table, c->coord, c->nb_dev, c->temp,
                                         c->temp_bytes, s));
  FL_CUDA(cudaMemcpyAsync(c->nb_host, c->nb_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  const int err = read_report(c, s, report);
  if (err != FL_OK) return err;
  c->nb = *c->nb_host;
  g = view(c);
  FL_CUDA(launch_build_neighbors(g, c->nbr27, s));
  return FL_OK;
}

namespace fl {
// The residual the composite preconditioner's network sees: one V-cycle on the
// current hierarchy from r, then rho = r - A V(r) (rho may be c->q).
template <typename T>
int post_vcycle_residual(fl_context* c, const fl_pressure_options* opt, const float* r, float* rho, cudaStream_t s) {
  GridView g = view(c);
  MgHierarchy<T> H{};
  const int levels = opt->levels > 0 ? opt->levels : auto_levels(c);
  int st = make_hierarchy<T>(c, levels, H);
  if (st != FL_OK) return st;
  MgOptions mo{std::max(1, opt->pre_sweeps), std::max(1, opt->post_sweeps), std::max(1, opt->coarse_sweeps)};
  ++g_kernel_launches;
  k_init_state<<<1, 1, 0, s>>>(c->st, 1e-6, 1e-4, 1, 0, 3, 0.9);  // clears the done flag of the last solve
  FL_CUDA(launch_apply_vcycle<T>(g, H, r, mo, &c->st->done, s));
  FL_CUDA(launch_residual0<T>(g, H, r, rho, &c->st->done, s));
  return FL_OK;
}
}  // namespace fl

extern "C" {

int fl_runtime_info(int* compiled_architecture, int* device_count, int* device_major, int* device_minor) {
  if (compiled_architecture) *compiled_architecture = 1000;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  if (device_count) *device_count = n;
  int major = 0, minor = 0;
  if (n > 0) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, 0) == cudaSuccess) {
      major = p.major;
      minor = p.minor;
    }
  }
  if (device_major) *device_major = major;
  if (device_minor) *device_minor = minor;
  return FL_OK;
}

int fl_copy_to_host(void* host, const void* device, uint64_t bytes) {
  if ((!host || !device) && bytes) return FL_INVALID_ARGUMENT;
  FL_CUDA(cudaMemcpy(host, device, bytes, cudaMemcpyDeviceToHost));
  return FL_OK;
}

int fl_copy_to_device(void* device, const void* host, uint64_t bytes) {
  if ((!host || !device) && bytes) return FL_INVALID_ARGUMENT;
  FL_CUDA(cudaMemcpy(device, host, bytes, cudaMemcpyHostToDevice));
  return FL_OK;
}

int fl_context_create(const fl_grid_desc* grid, uint64_t particle_capacity, fl_context** out) {
  if (!grid || !out) return FL_INVALID_ARGUMENT;
  *out = nullptr;
  if (!(grid->h > 0.0) || !std::isfinite(grid->h)) return FL_INVALID_ARGUMENT;
  for (int d = 0; d < 3; ++d)
    if (grid->block_dim[d] <= 0 || !std::isfinite(grid->origin[d])) return FL_INVALID_ARGUMENT;
  const long long lattice = (long long)grid->block_dim[0] * grid->block_dim[1] * grid->block_dim[2];
  if (lattice > (1LL << 21)) return FL_RESOURCE_EXHAUSTED;
  if (particle_capacity >= (1ULL << 31)) return FL_RESOURCE_EXHAUSTED;
  int st = device_ready();
  if (st != FL_OK) return st;
  fl_context* c = new fl_context();
  cudaGetDevice(&c->device);
  c->desc = *grid;
  c->pcap = std::max<uint64_t>(particle_capacity, 1);
  c->lattice = (int)lattice;
  const size_t cells = (size_t)lattice * kBlockCells;
  int e = FL_OK;
  auto chk = [&](int v) {
    if (v != FL_OK && e == FL_OK) e = v;
  };
  chk(dalloc(&c->occ, lattice));
  chk(dalloc(&c->flag, lattice));
  chk(dalloc(&c->ordinal, lattice));
  chk(dalloc(&c->table, lattice));
  chk(dalloc(&c->coord, 3 * lattice));
  chk(dalloc(&c->nbr27, 27 * lattice));
  chk(dalloc(&c->nb_dev, 1));
  chk(cudaMallocHost(&c->nb_host, sizeof(int)) == cudaSuccess ? FL_OK : FL_RESOURCE_EXHAUSTED);
  chk(dalloc(&c->keys, c->pcap));
  chk(dalloc(&c->index, c->pcap));
  chk(dalloc(&c->index_alt, c->pcap));
  chk(dalloc(&c->counts, cells + 1));
  chk(dalloc(&c->cell_start, cells + 1));
  c->temp_bytes = std::max(sort_temp_bytes(c->pcap, cells), (size_t)lattice * 8 + 4096);
  chk(cudaMalloc(&c->temp, c->temp_bytes) == cudaSuccess ? FL_OK : FL_RESOURCE_EXHAUSTED);
  for (int b = 0; b < 2; ++b) chk(dalloc(&c->pbuf[b], 16 * c->pcap));
  for (int a = 0; a < 3; ++a) {
    chk(dalloc(&c->u_pred[a], cells));
    chk(dalloc(&c->u_new[a], cells));
    chk(dalloc(&c->fmass[a], cells));
  }
  chk(dalloc(&c->tiles, (size_t)lattice * 3 * kTileFaces));
  chk(dalloc(&c->type, cells));
  chk(dalloc(&c->b64, cells));
  chk(dalloc(&c->p64, cells));
  chk(dalloc(&c->p_nat, cells));
  chk(dalloc(&c->p_keep, cells));
  chk(dalloc(&c->p_keep_prev, cells));
  if (cudaStreamCreateWithFlags(&c->work, cudaStreamNonBlocking) != cudaSuccess) chk(FL_INTERNAL);
  if (cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking) != cudaSuccess) chk(FL_INTERNAL);
  if (cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming) != cudaSuccess) chk(FL_INTERNAL);
  if (cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming) != cudaSuccess) chk(FL_INTERNAL);
  for (int b = 0; b < 2; ++b)
    if (cudaEventCreateWithFlags(&c->fence[b], cudaEventDisableTiming) != cudaSuccess) chk(FL_INTERNAL);
  configure_pressure_kernels();
  for (int k = 0; k < 2; ++k) {
    chk(dalloc(&c->r[k], cells));
    chk(dalloc(&c->d[k], cells));
  }
  chk(dalloc(&c->q, cells));
  chk(dalloc(&c->e, cells));
  chk(dalloc(&c->partial, 2 * (cells / 256 + 1024)));
  chk(dalloc(&c->st, 1));
  chk(cudaMallocHost(&c->st_host, sizeof(SolverState)) == cudaSuccess ? FL_OK : FL_RESOURCE_EXHAUSTED);
  chk(dalloc(&c->rep, 1));
  chk(cudaMallocHost(&c->rep_host, sizeof(DeviceReport)) == cudaSuccess ? FL_OK : FL_RESOURCE_EXHAUSTED);
  // multigrid levels
  chk(dalloc(&c->lv_mask0, cells));
  int maxbd = std::max(grid->block_dim[0], std::max(grid->block_dim[1], grid->block_dim[2]));
  int L = 4;
  while (L < 12 && dense_dim(maxbd, L - 1) > 1) ++L;
  c->max_levels = L;
  for (int l = 0; l < L; ++l) {
    long long cnt;
    if (l < 3) {
      const int S = 8 >> l;
      cnt = lattice * S * S * S;
    } else {
      cnt = 1;
      for (int d = 0; d < 3; ++d) cnt *= dense_dim(grid->block_dim[d], l);
    }
    c->lv_cap[l] = cnt;
    chk(dalloc(&c->lv_fluid[l], cnt));
    for (int a = 0; a < 3; ++a) chk(dalloc(reinterpret_cast<float**>(&c->lv_k[l][a]), cnt));
    chk(dalloc(&c->lv_anchor[l], cnt));
    chk(dalloc(&c->lv_diag[l], cnt));
    chk(dalloc(reinterpret_cast<float**>(&c->lv_x[l]), cnt));
    chk(dalloc(&c->lv_b[l], cnt));
    if (l >= 3) {
      // dense levels: zero once so cells never written read as non-fluid
      cudaMemset(c->lv_fluid[l], 0, cnt);
    }
  }
  if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) chk(FL_INTERNAL);
  for (int k = 0; k < 5; ++k)
    if (cudaEventCreate(&c->phase[k]) != cudaSuccess) chk(FL_INTERNAL);
  if (e == FL_OK) {
    cudaMemset(c->st, 0, sizeof(SolverState));
    cudaMemset(c->rep, 0, sizeof(DeviceReport));
    cudaMemset(c->lv_x[0], 0, sizeof(float) * c->lv_cap[0]);
    if (cudaDeviceSynchronize() != cudaSuccess) e = FL_INTERNAL;
  }
  if (e != FL_OK) {
    fl_context_destroy(c);
    return e;
  }
  *out = c;
  return FL_OK;
}

int fl_context_destroy(fl_context* c) {
  if (!c) return FL_OK;
  if (c->snapshot_queues > 0) return FL_FAILED_PRECONDITION;  // destroy its snapshot queues first
  cudaFree(c->occ);
  cudaFree(c->flag);
  cudaFree(c->ordinal);
  cudaFree(c->table);
  cudaFree(c->coord);
  cudaFree(c->nbr27);
  cudaFree(c->nb_dev);
  if (c->nb_host) cudaFreeHost(c->nb_host);
  cudaFree(c->keys);
  cudaFree(c->index);
  cudaFree(c->index_alt);
  cudaFree(c->counts);
  cudaFree(c->cell_start);
  cudaFree(c->temp);
  if (c->stage_stream) cudaStreamSynchronize(c->stage_stream);
  for (int b = 0; b < kStateBuffers; ++b) cudaFree(c->pbuf[b]);
  for (int a = 0; a < 3; ++a) {
    cudaFree(c->u_pred[a]);
    cudaFree(c->u_new[a]);
    cudaFree(c->fmass[a]);
  }
  cudaFree(c->tiles);
  cudaFree(c->type);
  cudaFree(c->b64);
  cudaFree(c->p64);
  cudaFree(c->p_nat);
  cudaFree(c->p_keep);
  cudaFree(c->p_keep_prev);
  if (c->fcg_exec) cudaGraphExecDestroy(c->fcg_exec);
  if (c->fcg_nn_exec) cudaGraphExecDestroy(c->fcg_nn_exec);
  cudaFree(c->nn_params);
  cudaFree(c->nn_scale);
  cudaFree(c->nn_act);
  cudaFree(c->nn_packed);
  cudaFree(c->nn_tc);
  cudaFree(c->nn_bt);
  if (c->work) cudaStreamDestroy(c->work);
  if (c->cap) cudaStreamDestroy(c->cap);
  if (c->ev_in) cudaEventDestroy(c->ev_in);
  if (c->ev_out) cudaEventDestroy(c->ev_out);
  for (int b = 0; b < kStateBuffers; ++b) {
    if (c->fence[b]) cudaEventDestroy(c->fence[b]);
    if (c->staged[b]) cudaEventDestroy(c->staged[b]);
  }
  if (c->stage_stream) cudaStreamDestroy(c->stage_stream);
  for (int k = 0; k < 2; ++k) {
    cudaFree(c->r[k]);
    cudaFree(c->d[k]);
  }
  cudaFree(c->q);
  cudaFree(c->e);
  cudaFree(c->partial);
  cudaFree(c->st);
  if (c->st_host) cudaFreeHost(c->st_host);
  cudaFree(c->rep);
  if (c->rep_host) cudaFreeHost(c->rep_host);
  cudaFree(c->lv_mask0);
  for (int l = 0; l < 12; ++l) {
    cudaFree(c->lv_fluid[l]);
    for (int a = 0; a < 3; ++a) cudaFree(c->lv_k[l][a]);
    cudaFree(c->lv_anchor[l]);
    cudaFree(c->lv_diag[l]);
    cudaFree(c->lv_x[l]);
    cudaFree(c->lv_b[l]);
  }
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (int k = 0; k < 5; ++k)
    if (c->phase[k]) cudaEventDestroy(c->phase[k]);
  delete c;
  return FL_OK;
}

int fl_topology_from_particles(fl_context* c, const fl_particles* p, void* stream, fl_report* report) {
  if (!c || !p) return FL_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  c->occ_ready = false;
  reset_report(c, s);
  GridView g = view(c);
  ParticlesView pv = pview(p);
  FL_CUDA(launch_topology_from_particles(g, pv, c->occ, c->flag, c->ordinal, c->table, c->coord, c->nb_dev, c->temp,
                                         c->temp_bytes, c->rep, s));
  FL_CUDA(cudaMemcpyAsync(c->nb_host, c->nb_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  const int err = read_report(c, s, report);
  if (err != FL_OK) return err;
  c->nb = *c->nb_host;
  g = view(c);
  FL_CUDA(launch_build_neighbors(g, c->nbr27, s));
  return FL_OK;
}

int fl_topology_from_blocks(fl_context* c, const int32_t* coords, uint64_t count) {
  if (!c || (!coords && count)) return FL_INVALID_ARGUMENT;
  std::vector<int> table(c->lattice, -1);
  std::vector<std::tuple<int, int, int>> keys;
  for (uint64_t i = 0; i < count; ++i) {
    int l[3];
    for (int d = 0; d < 3; ++d) {
      l[d] = coords[3 * i + d] - c->desc.block_lo[d];
      if (l[d] < 0 || l[d] >= c->desc.block_dim[d]) return FL_OUT_OF_RANGE;
    }
    keys.emplace_back(l[2], l[1], l[0]);
  }
  std::sort(keys.begin(), keys.end());
  if (std::adjacent_find(keys.begin(), keys.end()) != keys.end()) return FL_INVALID_ARGUMENT;
  std::vector<int> cd;
  for (size_t o = 0; o < keys.size(); ++o) {
    auto [z, y, x] = keys[o];
    table[((size_t)z * c->desc.block_dim[1] + y) * c->desc.block_dim[0] + x] = (int)o;
    cd.insert(cd.end(), {x + c->desc.block_lo[0], y + c->desc.block_lo[1], z + c->desc.block_lo[2]});
  }
  FL_CUDA(cudaMemcpy(c->table, table.data(), sizeof(int) * table.size(), cudaMemcpyHostToDevice));
  if (!cd.empty()) FL_CUDA(cudaMemcpy(c->coord, cd.data(), sizeof(int) * cd.size(), cudaMemcpyHostToDevice));
  c->nb = (int)keys.size();
  GridView g = view(c);
  FL_CUDA(launch_build_neighbors(g, c->nbr27, 0));
  FL_CUDA(cudaDeviceSynchronize());
  return FL_OK;
}

int fl_active_blocks(fl_context* c, int32_t* coords, uint64_t capacity, uint64_t* count) {
  if (!c) return FL_INVALID_ARGUMENT;
  if (count) *count = (uint64_t)c->nb;
  if (coords && capacity) {
    const uint64_t n = std::min<uint64_t>(capacity, (uint64_t)c->nb);
    FL_CUDA(cudaMemcpy(coords, c->coord, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost));
  }
  return FL_OK;
}

// Sort by block and cell. permute = false (the step) leaves `out` unwritten:
// c->index_alt then holds, for every cell-order slot, the particle of `in`.
static int sort_impl(fl_context* c, const fl_particles* in, fl_particles* out, bool permute, cudaStream_t s,
                     fl_report* report) {
  reset_report(c, s);
  GridView g = view(c);
  ParticlesView iv = pview(in), ov = pview(out);
  ov.count = in->count;
  FL_CUDA(launch_sort(g, iv, ov, c->keys, c->index, c->index_alt, c->counts, c->cell_start, c->temp,
                      c->temp_bytes, c->rep, s, permute));
  out->count = in->count;
  if (report) return read_report(c, s, report);
  return FL_OK;
}

int fl_sort_particles_by_block(fl_context* c, const fl_particles* in, fl_particles* out, void* stream,
                               fl_report* report) {
  if (!c || !in || !out) return FL_INVALID_ARGUMENT;
  if (in->count > c->pcap) return FL_RESOURCE_EXHAUSTED;
  if ((in->mass == nullptr) != (out->mass == nullptr)) return FL_INVALID_ARGUMENT;
  wait_state_fences(c, (cudaStream_t)stream);  // `out` may be a context buffer under a snapshot copy
  return sort_impl(c, in, out, true, (cudaStream_t)stream, report);
}

// P2G of the particles in cell order: slot q is particle q of `parts`, or
// particle order[q] when an order is given (the step, which skips the permutation).
static int p2g_impl(fl_context* c, const fl_particles* parts, const unsigned int* order, const fl_transfer_params* tp,
                    int mode, float* const out0[3], float* const out1[3], cudaStream_t s, fl_report* report,
                    uint8_t* const validity[3] = nullptr) {
  reset_report(c, s);
  GridView g = view(c);
  ParticlesView pv = pview(parts);
  P2GMergeParams prm{};
  prm.mode = mode;
  prm.walls = mode == 1 ? 1 : 0;
  prm.mass_scale = parts->mass ? 1.0f : (float)tp->particle_mass;
  prm.min_face_mass = (float)tp->min_face_mass;
  prm.dt = (float)tp->dt;
  for (int d = 0; d < 3; ++d) prm.gravity[d] = (float)tp->gravity[d];
  for (int d = 0; d < 3; ++d) prm.validity[d] = validity ? validity[d] : nullptr;
  float* o1[3] = {out1 ? out1[0] : nullptr, out1 ? out1[1] : nullptr, out1 ? out1[2] : nullptr};
  FL_CUDA(launch_p2g(g, pv, c->cell_start, c->tiles, prm, out0, o1, c->rep, s, order));
  if (report) return read_report(c, s, report);
  return FL_OK;
}

int fl_p2g(fl_context* c, const fl_particles* sorted, const fl_transfer_params* tp, int mode, float* const out0[3],
           float* const out1[3], void* stream, fl_report* report) {
  if (!c || !sorted || !tp || !out0 || (mode == 0 && !out1)) return FL_INVALID_ARGUMENT;
  return p2g_impl(c, sorted, nullptr, tp, mode, out0, out1, (cudaStream_t)stream, report);
}

int fl_p2g_normalized(fl_context* c, const fl_particles* sorted, const fl_transfer_params* tp, float* const u_pred[3],
                      float* const face_mass[3], uint8_t* const validity[3], void* stream, fl_report* report) {
  if (!c || !sorted || !tp || !u_pred || !validity) return FL_INVALID_ARGUMENT;
  for (int a = 0; a < 3; ++a)
    if (!u_pred[a] || !validity[a] || (face_mass && !face_mass[a])) return FL_INVALID_ARGUMENT;
  return p2g_impl(c, sorted, nullptr, tp, 1, u_pred, face_mass, (cudaStream_t)stream, report, validity);
}

int fl_pressure_project(fl_context* c, const float* const u_pred[3], float* const u_new[3],
                        const fl_transfer_params* tp, const fl_pressure_options* opt, fl_pressure_diagnostics* diag,
                        double* pressure_out, void* stream) {
  if (!c || !u_pred || !u_new || !tp || !opt) return FL_INVALID_ARGUMENT;
  if (!(opt->rel_tol > 0.0)) return FL_INVALID_ARGUMENT;
  if (c->nb == 0) return FL_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (opt->precision == 1)
    return pressure_solve<__nv_bfloat16>(c, u_pred, u_new, tp, opt, diag, pressure_out, s);
  return pressure_solve<float>(c, u_pred, u_new, tp, opt, diag, pressure_out, s);
}

int fl_apply_vcycle(fl_context* c, const float* r, float* z, const fl_pressure_options* opt, void* stream) {
  if (!c || !r || !z || !opt) return FL_INVALID_ARGUMENT;
  if (c->nb == 0) return FL_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (opt->precision == 1) return apply_vcycle<__nv_bfloat16>(c, r, z, opt, s);
  return apply_vcycle<float>(c, r, z, opt, s);
}

int fl_g2p(fl_context* c, fl_particles* sorted, const float* const u_new[3], const float* const u_old[3], float dt,
           float* full_out, void* stream, fl_report* report) {
  if (!c || !sorted || !u_new) return FL_INVALID_ARGUMENT;
  if (!full_out) {
    c->occ_ready = false;                       // positions may move: the next topology marks again
    wait_state_fences(c, (cudaStream_t)stream);  // step mode writes `sorted`, possibly a context buffer
  }
  return g2p_impl(c, sorted, u_new, u_old, dt, full_out, (cudaStream_t)stream, report, nullptr);
}

int fl_upload_particles(fl_context* c, const float* host, uint64_t count, void* stream) {
  if (!c || (!host && count)) return FL_INVALID_ARGUMENT;
  if (count > c->pcap) return FL_RESOURCE_EXHAUSTED;
  cudaStream_t s = (cudaStream_t)stream;
  c->nstage = 0;  // the uploaded state replaces any staged input
  const int b = pick_buffer(c, 0);
  c->cur = b;
  c->count = count;
  c->p_keep_valid = false;
  c->p_keep_prev_valid = false;
  c->occ_ready = false;
  FL_CUDA(cudaStreamWaitEvent(s, c->fence[b], 0));  // a snapshot copy of the buffer still in flight
  if (c->staged[b]) FL_CUDA(cudaStreamWaitEvent(s, c->staged[b], 0));  // a dropped staging copy into it
  for (int k = 0; k < 15; ++k)
    FL_CUDA(cudaMemcpyAsync(c->pbuf[b] + (size_t)k * c->pcap, host + (size_t)k * count, sizeof(float) * count,
                            cudaMemcpyHostToDevice, s));
  return FL_OK;
}

int fl_stage_particles(fl_context* c, const float* host, uint64_t count) {
  if (!c || (!host && count)) return FL_INVALID_ARGUMENT;
  if (count > c->pcap) return FL_RESOURCE_EXHAUSTED;
  if (c->nstage == 2) return FL_UNAVAILABLE;
  if (c->nbuf < kStateBuffers) {  // first staging: two more buffers and the staging stream
    for (int b = c->nbuf; b < kStateBuffers; ++b) {
      if (dalloc(&c->pbuf[b], 16 * c->pcap) != FL_OK) return FL_RESOURCE_EXHAUSTED;
      FL_CUDA(cudaEventCreateWithFlags(&c->fence[b], cudaEventDisableTiming));
    }
    for (int b = 0; b < kStateBuffers; ++b) FL_CUDA(cudaEventCreateWithFlags(&c->staged[b], cudaEventDisableTiming));
    FL_CUDA(cudaStreamCreateWithFlags(&c->stage_stream, cudaStreamNonBlocking));
    c->nbuf = kStateBuffers;
  }
  const int b = pick_buffer(c, (1u << c->cur) | staged_mask(c));
  cudaStream_t s = c->stage_stream;
  FL_CUDA(cudaStreamWaitEvent(s, c->fence[b], 0));
  for (int k = 0; k < 15; ++k)
    FL_CUDA(cudaMemcpyAsync(c->pbuf[b] + (size_t)k * c->pcap, host + (size_t)k * count, sizeof(float) * count,
                            cudaMemcpyHostToDevice, s));
  FL_CUDA(cudaEventRecord(c->staged[b], s));
  c->stage_buf[c->nstage] = b;
  c->stage_count[c->nstage] = count;
  ++c->nstage;
  return FL_OK;
}

int fl_download_particles(fl_context* c, float* host, void* stream) {
  if (!c || !host) return FL_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < 15; ++k)
    FL_CUDA(cudaMemcpyAsync(host + (size_t)k * c->count, c->pbuf[c->cur] + (size_t)k * c->pcap,
                            sizeof(float) * c->count, cudaMemcpyDeviceToHost, s));
  FL_CUDA(cudaStreamSynchronize(s));
  return FL_OK;
}

int fl_state_particles(fl_context* c, fl_particles* out) {
  if (!c || !out) return FL_INVALID_ARGUMENT;
  *out = state_particles(c, c->cur);
  return FL_OK;
}

int fl_state_fields(fl_context* c, float* u_pred[3], float* u_new[3], double** pressure, uint8_t** cell_type,
                    int32_t** cell_start) {
  if (!c) return FL_INVALID_ARGUMENT;
  for (int a = 0; a < 3; ++a) {
    if (u_pred) u_pred[a] = c->u_pred[a];
    if (u_new) u_new[a] = c->u_new[a];
  }
  if (pressure) *pressure = c->p_nat;
  if (cell_type) *cell_type = c->type;
  if (cell_start) *cell_start = c->cell_start;
  return FL_OK;
}

int fl_step(fl_context* c, const fl_transfer_params* tp, const fl_pressure_options* opt,
            fl_pressure_diagnostics* diag, void* stream, fl_report* report) {
  if (!c || !tp || !opt) return FL_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  if (c->nstage > 0) {  // the oldest staged input becomes the state this step advances
    const int b = c->stage_buf[0];
    FL_CUDA(cudaStreamWaitEvent(s, c->staged[b], 0));
    c->cur = b;
    c->count = c->stage_count[0];
    c->stage_buf[0] = c->stage_buf[1];
    c->stage_count[0] = c->stage_count[1];
    --c->nstage;
    c->p_keep_valid = false;
    c->p_keep_prev_valid = false;
    c->occ_ready = false;
  }
  const int out_buf = pick_buffer(c, (1u << c->cur) | staged_mask(c));
  fl_particles A = state_particles(c, c->cur), B = state_particles(c, out_buf);
  fl_report rep{};
  c->phases_valid = false;
  cudaEventRecord(c->phase[0], s);
  int st = step_topology(c, &A, s, &rep);
  if (st != FL_OK) {
    if (report) *report = rep;
    return st;
  }
  c->occ_ready = false;
  FL_CUDA(cudaMemsetAsync(c->occ, 0, (size_t)c->lattice, s));  // this step's G2P marks the next topology
  struct StepScope {
    fl_context* c;
    ~StepScope() { c->in_step = false; }
  } scope{c};
  c->in_step = true;
  // The particles are not permuted: P2G reads state A through the cell order
  // and G2P writes the advected state into B in that order.
  st = sort_impl(c, &A, &B, false, s, nullptr);
  if (st != FL_OK) return st;
  cudaEventRecord(c->phase[1], s);
  float* o0[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  float* o1[3] = {c->fmass[0], c->fmass[1], c->fmass[2]};
  st = p2g_impl(c, &A, c->index_alt, tp, 1, o0, o1, s, nullptr);
  if (st != FL_OK) return st;
  cudaEventRecord(c->phase[2], s);
  const float* up[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  float* un[3] = {c->u_new[0], c->u_new[1], c->u_new[2]};
  st = fl_pressure_project(c, up, un, tp, opt, diag, nullptr, stream);
  if (st != FL_OK && st != FL_ABORTED) return st;
  const int pressure_status = st;
  cudaEventRecord(c->phase[3], s);
  const float* unc[3] = {c->u_new[0], c->u_new[1], c->u_new[2]};
  // B may still be read by a snapshot of the previous state: only the write into it waits
  FL_CUDA(cudaStreamWaitEvent(s, c->fence[out_buf], 0));
  if (c->staged[out_buf]) FL_CUDA(cudaStreamWaitEvent(s, c->staged[out_buf], 0));  // a dropped staging copy
  st = g2p_impl(c, &B, unc, nullptr, (float)tp->dt, nullptr, s, nullptr, c->occ, c->index_alt, &A);
  if (st != FL_OK) return st;
  cudaEventRecord(c->phase[4], s);
  c->phases_valid = true;
  c->cur = out_buf;
  const int err = read_report(c, s, report);
  if (err != FL_OK) return err;
  c->occ_ready = true;
  return pressure_status;
}

int fl_step_timings(fl_context* c, float* ms) {
  if (!c || !ms) return FL_INVALID_ARGUMENT;
  if (!c->phases_valid) return FL_FAILED_PRECONDITION;
  FL_CUDA(cudaEventSynchronize(c->phase[4]));
  for (int k = 0; k < 4; ++k) FL_CUDA(cudaEventElapsedTime(&ms[k], c->phase[k], c->phase[k + 1]));
  return FL_OK;
}

int fl_kernel_launches(unsigned long long* own, unsigned long long* library) {
  if (own) *own = g_kernel_launches;
  if (library) *library = g_library_launches;
  return FL_OK;
}

int fl_step_host(fl_context* c, const float* host_in, float* host_out, uint64_t count, const fl_transfer_params* tp,
                 const fl_pressure_options* opt, fl_pressure_diagnostics* diag, void* stream) {
  int st = fl_upload_particles(c, host_in, count, stream);
  if (st != FL_OK) return st;
  st = fl_step(c, tp, opt, diag, stream, nullptr);
  if (st != FL_OK && st != FL_ABORTED) return st;
  const int r = fl_download_particles(c, host_out, stream);
  return r != FL_OK ? r : st;
}

int fl_deposit_mac_3d(const double origin[3], double h, const int32_t* blocks, uint64_t nb4, const double* parts,
                      uint64_t np, double* face_mass, double* face_momentum, fl_measurement* meas) {
  if (!origin || !(h > 0.0) || (!blocks && nb4) || (!parts && np) || (!face_mass && nb4) || (!face_momentum && nb4))
    return FL_INVALID_ARGUMENT;
  int st = device_ready();
  if (st != FL_OK) return st;
  st = validate_particles(parts, np, h, true);
  if (st != FL_OK) return st;
  RefLayout L;
  make_layout(blocks, nb4, L);
  TempContext tc;
  st = make_ref_context(origin, h, L, np, tc);
  if (st != FL_OK) return st;
  fl_context* c = tc.ctx;
  cudaStream_t s = 0;
  std::vector<float> soa;
  cudaEventRecord(c->ev0, s);
  st = upload_ref_particles(c, parts, np, s, soa);
  if (st != FL_OK) return st;
  fl_particles P = state_particles(c, 0);
  P.mass = c->pbuf[0] + 15 * c->pcap;
  fl_transfer_params tp{};
  tp.particle_mass = 1.0f;
  float* o0[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  float* o1[3] = {c->fmass[0], c->fmass[1], c->fmass[2]};
  fl_report rep{};
  st = fl_p2g(c, &P, &tp, 0, o0, o1, s, &rep);
  cudaEventRecord(c->ev1, s);
  if (st != FL_OK) return st;
  const size_t n8 = (size_t)c->nb * 512;
  std::vector<float> m[3], q[3];
  for (int a = 0; a < 3; ++a) {
    m[a].resize(n8);
    q[a].resize(n8);
    FL_CUDA(cudaMemcpy(m[a].data(), c->u_pred[a], sizeof(float) * n8, cudaMemcpyDeviceToHost));
    FL_CUDA(cudaMemcpy(q[a].data(), c->fmass[a], sizeof(float) * n8, cudaMemcpyDeviceToHost));
  }
  std::vector<int> axis;
  std::vector<long long> slot8;
  slot_map(L, axis, slot8);
  // Support outside the reference's active 4^3 blocks is a failed precondition.
  std::vector<char> owned(n8 * 3, 0);
  for (size_t sidx = 0; sidx < axis.size(); ++sidx) owned[(size_t)axis[sidx] * n8 + slot8[sidx]] = 1;
  for (int a = 0; a < 3; ++a)
    for (size_t i = 0; i < n8; ++i)
      if (!owned[(size_t)a * n8 + i] && m[a][i] != 0.0f) return FL_FAILED_PRECONDITION;
  for (size_t sidx = 0; sidx < axis.size(); ++sidx) {
    face_mass[sidx] = m[axis[sidx]][slot8[sidx]];
    face_momentum[sidx] = q[axis[sidx]][slot8[sidx]];
  }
  if (meas) {
    meas->compiled_architecture = rep.compiled_architecture;
    cudaEventElapsedTime(&meas->kernel_ms, c->ev0, c->ev1);
  }
  return FL_OK;
}

int fl_deposit_mac_quanta_3d(const double origin[3], double h, const int32_t* blocks, uint64_t nb4,
                             const double* parts, uint64_t np, double mq, double pq, uint64_t cap,
                             int64_t* mass_quanta, int64_t* momentum_quanta, fl_measurement* meas) {
  if (!origin || !(h > 0.0) || (!blocks && nb4) || (!parts && np)) return FL_INVALID_ARGUMENT;
  auto pow2 = [](double v) {
    int e;
    return std::isnormal(v) && v > 0 && std::frexp(v, &e) == 0.5;
  };
  if (!pow2(mq) || !pow2(pq)) return FL_INVALID_ARGUMENT;
  if (cap > (1ULL << 20) || np > cap) return FL_RESOURCE_EXHAUSTED;
  int st = device_ready();
  if (st != FL_OK) return st;
  st = validate_particles(parts, np, h, true);
  if (st != FL_OK) return st;
  RefLayout L;
  make_layout(blocks, nb4, L);
  TempContext tc;
  st = make_ref_context(origin, h, L, np, tc);
  if (st != FL_OK) return st;
  fl_context* c = tc.ctx;
  const size_t n8 = (size_t)c->nb * 512;
  unsigned long long* acc = nullptr;
  double* dparts = nullptr;
  if (cudaMalloc(&acc, sizeof(unsigned long long) * 6 * std::max<size_t>(n8, 1)) != cudaSuccess)
    return FL_RESOURCE_EXHAUSTED;
  if (cudaMalloc(&dparts, sizeof(double) * 19 * std::max<uint64_t>(np, 1)) != cudaSuccess) {
    cudaFree(acc);
    return FL_RESOURCE_EXHAUSTED;
  }
  int result = FL_OK;
  do {
    cudaMemset(acc, 0, sizeof(unsigned long long) * 6 * n8);
    if (np) cudaMemcpy(dparts, parts, sizeof(double) * 19 * np, cudaMemcpyHostToDevice);
    cudaMemset(c->rep, 0, sizeof(DeviceReport));
    const uint64_t nz = std::max<uint64_t>(cap, 1);
    int e = 0;
    while ((1ULL << e) < nz) ++e;
    const double limit = std::ldexp(1.0, 62 - e);
    unsigned long long* mqp[3] = {acc, acc + n8, acc + 2 * n8};
    unsigned long long* pqp[3] = {acc + 3 * n8, acc + 4 * n8, acc + 5 * n8};
    GridView g = view(c);
    cudaEventRecord(c->ev0, 0);
    if (launch_deposit_quanta(g, dparts, np, origin, h, mq, pq, limit, mqp, pqp, c->rep, 0) != cudaSuccess) {
      result = FL_INTERNAL;
      break;
    }
    cudaEventRecord(c->ev1, 0);
    fl_report rep{};
    const int err = read_report(c, 0, &rep);
    if (err != FL_OK) {
      result = err;
      break;
    }
    std::vector<unsigned long long> host(6 * n8);
    cudaMemcpy(host.data(), acc, sizeof(unsigned long long) * 6 * n8, cudaMemcpyDeviceToHost);
    std::vector<int> axis;
    std::vector<long long> slot8;
    slot_map(L, axis, slot8);
    std::vector<char> owned(n8 * 3, 0);
    for (size_t sidx = 0; sidx < axis.size(); ++sidx) owned[(size_t)axis[sidx] * n8 + slot8[sidx]] = 1;
    for (int a = 0; a < 3; ++a)
      for (size_t i = 0; i < n8; ++i)
        if (!owned[(size_t)a * n8 + i] && host[(size_t)a * n8 + i] != 0ULL) result = FL_FAILED_PRECONDITION;
    if (result != FL_OK) break;
    for (size_t sidx = 0; sidx < axis.size(); ++sidx) {
      mass_quanta[sidx] = (int64_t)host[(size_t)axis[sidx] * n8 + slot8[sidx]];
      momentum_quanta[sidx] = (int64_t)host[(size_t)(3 + axis[sidx]) * n8 + slot8[sidx]];
    }
    if (meas) {
      meas->compiled_architecture = rep.compiled_architecture;
      cudaEventElapsedTime(&meas->kernel_ms, c->ev0, c->ev1);
    }
  } while (false);
  cudaFree(acc);
  cudaFree(dparts);
  return result;
}

int fl_gather_mac_3d(const double origin[3], double h, const int32_t* blocks, uint64_t nb4, const double* parts,
                     uint64_t np, const double* old_u, const double* new_u, double* results, fl_measurement* meas) {
  if (!origin || !(h > 0.0) || (!blocks && nb4) || (!parts && np) || !new_u || !old_u) return FL_INVALID_ARGUMENT;
  int st = device_ready();
  if (st != FL_OK) return st;
  st = validate_particles(parts, np, h, false);
  if (st != FL_OK) return st;
  const size_t fc = (size_t)nb4 * 192;
  for (size_t i = 0; i < fc; ++i)
    if (!std::isfinite(old_u[i]) || !std::isfinite(new_u[i])) return FL_INVALID_ARGUMENT;
  RefLayout L;
  make_layout(blocks, nb4, L);
  TempContext tc;
  st = make_ref_context(origin, h, L, np, tc);
  if (st != FL_OK) return st;
  fl_context* c = tc.ctx;
  cudaStream_t s = 0;
  // Gather ignores deposit-only data: replace mass/velocity/slopes by zeros.
  std::vector<double> clean(parts, parts + 19 * np);
  for (uint64_t i = 0; i < np; ++i)
    for (int k = 6; k < 19; ++k) clean[19 * i + k] = 0.0;
  std::vector<float> soa;
  st = upload_ref_particles(c, clean.data(), np, s, soa);
  if (st != FL_OK) return st;
  const size_t n8 = (size_t)c->nb * 512;
  std::vector<int> axis;
  std::vector<long long> slot8;
  slot_map(L, axis, slot8);
  std::vector<float> un(3 * n8, 0.0f), uo(3 * n8, 0.0f);
  for (size_t sidx = 0; sidx < fc; ++sidx) {
    un[(size_t)axis[sidx] * n8 + slot8[sidx]] = (float)new_u[sidx];
    uo[(size_t)axis[sidx] * n8 + slot8[sidx]] = (float)old_u[sidx];
  }
  for (int a = 0; a < 3; ++a) {
    FL_CUDA(cudaMemcpy(c->u_new[a], un.data() + a * n8, sizeof(float) * n8, cudaMemcpyHostToDevice));
    FL_CUDA(cudaMemcpy(c->u_pred[a], uo.data() + a * n8, sizeof(float) * n8, cudaMemcpyHostToDevice));
  }
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * 24 * std::max<uint64_t>(np, 1)) != cudaSuccess) return FL_RESOURCE_EXHAUSTED;
  fl_particles P = state_particles(c, 0);
  const float* unp[3] = {c->u_new[0], c->u_new[1], c->u_new[2]};
  const float* uop[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  fl_report rep{};
  cudaEventRecord(c->ev0, s);
  st = fl_g2p(c, &P, unp, uop, 0.0f, out, s, &rep);
  cudaEventRecord(c->ev1, s);
  if (st == FL_OK) {
    std::vector<float> host(24 * np);
    std::vector<unsigned int> perm(np);
    cudaMemcpy(host.data(), out, sizeof(float) * 24 * np, cudaMemcpyDeviceToHost);
    cudaMemcpy(perm.data(), c->index_alt, sizeof(unsigned int) * np, cudaMemcpyDeviceToHost);
    for (uint64_t sidx = 0; sidx < np; ++sidx)
      for (int k = 0; k < 24; ++k) results[24 * (size_t)perm[sidx] + k] = host[24 * sidx + k];
    if (meas) {
      meas->compiled_architecture = rep.compiled_architecture;
      cudaEventElapsedTime(&meas->kernel_ms, c->ev0, c->ev1);
    }
  }
  cudaFree(out);
  return st;
}

int fl_set_learned_preconditioner(fl_context* c, const float* params, void* stream) {
  if (!c || !params) return FL_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const long long np = unet_layout().total;
  if (!c->nn_params && cudaMalloc(&c->nn_params, sizeof(float) * np) != cudaSuccess) {
    cudaGetLastError();
    return FL_RESOURCE_EXHAUSTED;
  }
  if (!c->nn_scale && cudaMalloc(&c->nn_scale, sizeof(float) * (size_t)c->lattice) != cudaSuccess) {
    cudaGetLastError();
    return FL_RESOURCE_EXHAUSTED;
  }
  if (!c->nn_packed &&
      cudaMalloc(&c->nn_packed, sizeof(__nv_bfloat16) * (size_t)unet_tc_layout().w_total) != cudaSuccess) {
    cudaGetLastError();
    return FL_RESOURCE_EXHAUSTED;
  }
  if (c->sms == 0) cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  configure_unet_kernels();
  FL_CUDA(cudaMemcpyAsync(c->nn_params, params, sizeof(float) * np, cudaMemcpyDeviceToDevice, s));
  FL_CUDA(unet_tc_pack(c->nn_params, c->nn_packed, s));
  FL_CUDA(cudaStreamSynchronize(s));
  c->nn_ready = true;
  return FL_OK;
}

int fl_apply_learned(fl_context* c, const float* r, float* z, int kernels, void* stream) {
  if (!c || !r || !z || (kernels != 0 && kernels != 1)) return FL_INVALID_ARGUMENT;
  if (!c->nn_ready) return FL_FAILED_PRECONDITION;
  if (c->nb == 0) return FL_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int st = kernels == 0 ? nn_reserve_tc(c, c->nb) : nn_reserve(c, c->nb);
  if (st != FL_OK) return st;
  GridView g = view(c);
  FL_CUDA(launch_classify(g, c->cell_start, c->type, s));
  FL_CUDA(launch_to_rb(g, r, c->r[0], s));
  if (kernels == 0) {
    FL_CUDA(cudaMemsetAsync(&c->st->nn_error, 0, sizeof(int), s));
    FL_CUDA(unet_tc_apply<float>(g, c->nn_params, c->nn_packed, c->nn_tc, c->nn_tc_items, c->nn_bt, c->nn_scale,
                                 c->type, c->r[0], c->q, &c->st->nn_error, c->sms, s));
    FL_CUDA(launch_to_natural_f32(g, c->q, z, s));
    FL_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s));
    FL_CUDA(cudaStreamSynchronize(s));
    if (c->st_host->nn_error) return FL_INTERNAL;
    return FL_OK;
  }
  const UNetCache C = unet_cache_layout(g.nb);
  FL_CUDA(unet_gather(g, c->r[0], c->type, nullptr, g.nb, c->nn_act + C.x, c->nn_scale, s));
  FL_CUDA(unet_forward(c->nn_params, c->nn_act + C.x, g.nb, c->nn_act, nullptr, s));
  FL_CUDA(unet_scatter<float>(g.nb, c->nn_act + C.y, c->nn_scale, c->type, z, false, s));
  FL_CUDA(cudaStreamSynchronize(s));
  return FL_OK;
}

int fl_collect_training_pairs(fl_context* c, const fl_transfer_params* tp, const fl_pressure_options* opt,
                              const int32_t* iterations, int iteration_count, float* inputs, float* targets,
                              float* target_mask, uint64_t capacity, uint64_t* written) {
  if (!c || !tp || !opt || !iterations || iteration_count <= 0 || !inputs || !targets || !target_mask || !written)
    return FL_INVALID_ARGUMENT;
  *written = 0;
  if (c->nb == 0 || capacity == 0) return FL_OK;
  fl_pressure_options o = *opt;
  o.warm_start = 0;
  o.preconditioner = 0;
  const float* up[3] = {c->u_pred[0], c->u_pred[1], c->u_pred[2]};
  float* un[3] = {c->u_new[0], c->u_new[1], c->u_new[2]};
  int st = fl_pressure_project(c, up, un, tp, &o, nullptr, nullptr, nullptr);
  if (st != FL_OK) return st;
  const int nb = c->nb;
  const size_t n = (size_t)nb * kBlockCells;
  double* p_star = nullptr;
  int* dlist = nullptr;
  float* scale = nullptr;
  if (cudaMalloc(&p_star, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dlist, sizeof(int) * nb) != cudaSuccess ||
      cudaMalloc(&scale, sizeof(float) * nb) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(p_star);
    cudaFree(dlist);
    return FL_RESOURCE_EXHAUSTED;
  }
  cudaStream_t s = c->work;
  GridView g = view(c);
  std::vector<int> flags(nb), list;
  cudaError_t e = cudaMemcpyAsync(p_star, c->p64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = unet_block_has_fluid(nb, c->type, dlist, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(flags.data(), dlist, sizeof(int) * nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  for (int b = 0; b < nb; ++b)
    if (flags[b]) list.push_back(b);
  if (e == cudaSuccess && !list.empty())
    e = cudaMemcpy(dlist, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice);
  uint64_t w = 0;
  for (int k = 0; k < iteration_count && e == cudaSuccess && st == FL_OK && w < capacity && !list.empty(); ++k) {
    fl_pressure_options ok = o;
    ok.max_iterations = std::max(0, (int)iterations[k]);
    const int rc = fl_pressure_project(c, up, un, tp, &ok, nullptr, nullptr, nullptr);
    if (rc != FL_OK && rc != FL_ABORTED) {
      st = rc;
      break;
    }
    // r[0] holds b - A p_k of the capped solve (its last residual evaluation);
    // for the composite preconditioner the input is what follows a V-cycle on it
    const float* src = c->r[0];
    if (opt->preconditioner == 2) {
      const int rc2 = o.precision == 1 ? post_vcycle_residual<__nv_bfloat16>(c, &o, c->r[0], c->q, s)
                                       : post_vcycle_residual<float>(c, &o, c->r[0], c->q, s);
      if (rc2 != FL_OK) {
        st = rc2;
        break;
      }
      src = c->q;
    }
    const int take = (int)std::min<uint64_t>(list.size(), capacity - w);
    e = unet_gather(g, src, c->type, dlist, take, inputs + w * 2000, scale, s);
    if (e == cudaSuccess)
      e = unet_targets(g, p_star, c->p64, c->type, dlist, take, scale, targets + w * 512, target_mask + w * 512, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    w += take;
  }
  cudaFree(p_star);
  cudaFree(dlist);
  cudaFree(scale);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  if (st != FL_OK) return st;
  *written = w;
  return FL_OK;
}

}  // extern "C"

// Accessors for the snapshot queue (fl_snapshot.cu).
namespace fl {
void context_snapshot_source(fl_context* c, SnapshotSource* out) {
  out->base = c->pbuf[c->cur];
  out->pcap = c->pcap;
  out->count = c->count;
  out->buffer = c->cur;
  out->device = c->device;
  out->g = view(c);
}
cudaEvent_t context_buffer_fence(fl_context* c, int buffer) { return c->fence[buffer]; }
void context_attach_snapshot_queue(fl_context* c, int delta) { c->snapshot_queues += delta; }
int check_device() { return device_ready(); }
}  // namespace fl
