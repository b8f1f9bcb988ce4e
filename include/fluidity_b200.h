/* fluidity_b200 -- C-ABI of the B200-native liquid-step hot path.
 *
 * One CUDA library (fluidity_b200/_lib/libfluidity_b200.so) exports these
 * entry points. Signatures use plain pointers, sizes and a cudaStream_t passed
 * as void*; no C++ or torch types cross the boundary. Every function returns
 * a status with the reference's absl numbering (FL_OK = 0). There is no CPU
 * fallback: without a usable sm_100 device the calls return
 * FL_FAILED_PRECONDITION, as the reference's CUDA operators do
 * (native/include/fluidity/host/cuda_mac_pressure_3d.h:154-158).
 *
 * The path replaces, in the FluidiTy reference (paths inside that project):
 *   - DepositMac3D / DepositMacQuanta3D / GatherMac3D
 *       native/include/fluidity/host/transfers_3d.h:23-61
 *   - CudaDepositMacQuanta3D / CudaGatherMac3D
 *       native/include/fluidity/host/cuda_transfers_3d.h:18-39
 *   - ProjectMacPressure3D / CudaProjectMacPressure3D
 *       native/include/fluidity/host/mac_pressure_3d.h:101-102,
 *       native/include/fluidity/host/cuda_mac_pressure_3d.h:19-20
 *   - the thin bridges LaunchDeposit3D / LaunchGather3D
 *       (native/cuda/transfer_3d_bridge.h:62-83) and LaunchMacPressure3D /
 *       LaunchMacPressureBatch3D (native/cuda/mac_pressure_3d_bridge.h:115-120)
 *   - the scheduler backend ops .topology/.deposit/.normalize/.forces/.project/
 *     .gather of LiquidSubstepBackend3D
 *       (native/include/fluidity/host/liquid_substep_backend_3d.h:121-194)
 *
 * Threading: a context is single-threaded and non-reentrant, like the
 * reference's backend (liquid_substep_backend_3d.h:37-46). Calls are ordered
 * on the stream they are given; functions that must read a device value
 * (block counts, convergence) synchronize that stream.
 *
 * Device-side errors: a call that takes an fl_report* and is given one
 * synchronizes its stream, copies the kernels' report into it and returns its
 * error code (the reference's checked report, transfer_3d_host.cc:69-92).
 * Given report == NULL, the call returns after queueing its kernels: it
 * reports argument and launch errors only, and no device-side error check is
 * made.
 */
#ifndef FLUIDITY_B200_H_
#define FLUIDITY_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (absl::StatusCode numbering, as in the reference's transfers_3d.h:13-22,
 * mac_pressure_3d.h:88-100, operator_runtime.h:18-40). */
#define FL_OK 0
#define FL_INVALID_ARGUMENT 3
#define FL_ALREADY_EXISTS 6
#define FL_RESOURCE_EXHAUSTED 8
#define FL_FAILED_PRECONDITION 9
#define FL_ABORTED 10
#define FL_OUT_OF_RANGE 11
#define FL_INTERNAL 13
#define FL_UNAVAILABLE 14
#define FL_DATA_LOSS 15

typedef struct fl_context fl_context;

/* Device kernel report (MacTransferKernelReport3D, native/cuda/transfer_3d_bridge.h:54-57,
 * plus the first failing index). */
typedef struct {
  int compiled_architecture; /* __CUDA_ARCH__ of the image that ran, e.g. 1000 */
  int error;                 /* FL_* code written by the first failing lane, 0 if none */
  unsigned long long first_bad_index;
} fl_report;

/* CudaOperatorMeasurement (native/include/fluidity/host/cuda_measurement.h:4-10). */
typedef struct {
  int compiled_architecture;
  float kernel_ms;
} fl_measurement;

/* Uniform MAC geometry on a lattice of 8^3-cell blocks. Cells whose index lies
 * outside [solid_lo, solid_hi] on any axis are solid (stationary walls); use
 * INT32_MIN / INT32_MAX for a domain without walls. */
typedef struct {
  double origin[3]; /* world position of the lower corner of cell (0,0,0), m */
  double h;         /* cell width, m */
  int32_t block_lo[3];
  int32_t block_dim[3];
  int32_t solid_lo[3];
  int32_t solid_hi[3];
} fl_grid_desc;

/* Device particle SoA in FP32 (60 B/particle without per-particle mass). */
typedef struct {
  float* x[3]; /* world position, m */
  float* v[3]; /* velocity, m/s */
  float* c[9]; /* APIC affine rows C[a][d], 1/s */
  float* mass; /* kg per particle, or NULL for the uniform mass of the call */
  uint64_t count;
} fl_particles;

typedef struct {
  double dt;            /* s */
  double particle_mass; /* kg, used when fl_particles.mass is NULL */
  double gravity[3];    /* m/s^2 */
  double min_face_mass; /* kg; faces at or below it are low-mass (velocity 0) */
  double density;       /* kg/m^3 for the pressure conductance */
} fl_transfer_params;

typedef struct {
  int levels;         /* multigrid levels (>= 4), 0 = automatic */
  int pre_sweeps;     /* red-black Gauss-Seidel sweeps before the coarse correction */
  int post_sweeps;    /* ... and after it */
  int coarse_sweeps;  /* symmetric sweeps on the coarsest level */
  int precision;      /* 0: FP32 V-cycle storage; 1: BF16 V-cycle storage */
  int max_iterations; /* total inner flexible-CG iterations */
  int max_refinements;
  int warm_start;     /* 1: start from the previous projection's pressure (InitializeMacPressure3D);
                         2: from 2 p(n) - p(n-1), the last two projections' pressures (falls back to 1) */
  double rel_tol;    /* ||b - A p||_2 <= rel_tol * ||b||_2, checked in FP64 */
  double inner_rtol; /* inner FP32 solve reduction per refinement */
  int preconditioner; /* 0: V-cycle; 1: learned block U-Net (fl_set_learned_preconditioner) in place of the
                         V-cycle, V-cycle fallback; 2: V-cycle, then the U-Net's correction from the V-cycle's
                         residual r - A V(r) added to it, V-cycle-only fallback */
  int stall_limit;    /* learned: consecutive stalled iterations before the V-cycle takes over (0 -> 3) */
  double stall_ratio; /* learned: an iteration stalls unless ||r||_2 < stall_ratio * best so far (0 -> 0.9) */
} fl_pressure_options;

typedef struct {
  int status;
  int iterations;
  int refinements;
  int levels;
  int fluid_cells;
  int active_blocks;
  double rhs_l2;                 /* ||b||_2 in reference units, m^3/s */
  double true_residual_l2;       /* ||b - A p||_2 in FP64, m^3/s */
  double relative_residual;      /* true_residual_l2 / rhs_l2 */
  double reference_limit;        /* 2e-6 + 2e-6 ||b||_2 (MacPressureStoppingCriteria) */
  double max_volume_residual;    /* max |r|/V, 1/s (estimated from the FP64 l2 bound) */
  double max_divergence;         /* max |div u_new| over fluid cells, 1/s */
  double solve_ms;
  int learned_iterations; /* iterations preconditioned by the learned network */
  int fell_back;          /* 1: the V-cycle took over after stalled learned iterations */
} fl_pressure_diagnostics;

/* ---- context (the resident device arena) -------------------------------- */

int fl_context_create(const fl_grid_desc* grid, uint64_t particle_capacity, fl_context** out);
int fl_context_destroy(fl_context* ctx);

/* Active blocks: blocks holding particles plus a one-block ring
 * (replaces the .topology backend op, liquid_substep_backend_3d.h:121-127). */
int fl_topology_from_particles(fl_context* ctx, const fl_particles* particles, void* stream, fl_report* report);
/* Explicit active blocks (8^3-block coordinates). */
int fl_topology_from_blocks(fl_context* ctx, const int32_t* block_coords, uint64_t block_count);
/* Copies up to `capacity` active block coordinates (x,y,z per block, ordinal order). */
int fl_active_blocks(fl_context* ctx, int32_t* coords, uint64_t capacity, uint64_t* block_count);

/* ---- the hot path ---------------------------------------------------- */

/* Stable sort of the particles by (8^3 block, cell) into `out` (a separate
 * buffer of the same capacity) and per-cell ranges kept in the context. */
int fl_sort_particles_by_block(fl_context* ctx, const fl_particles* in, fl_particles* out, void* stream,
                               fl_report* report);

/* APIC P2G over sorted particles (DepositMac3D semantics). mode 0 writes face
 * mass (out0) and pure momentum (out1); mode 1 writes the normalized velocity
 * plus dt*gravity with stationary walls (out0, the predicted velocity) and the
 * face mass (out1, may be NULL). Face arrays hold active_blocks*512 floats per axis. */
int fl_p2g(fl_context* ctx, const fl_particles* sorted, const fl_transfer_params* params, int mode,
           float* const out0[3], float* const out1[3], void* stream, fl_report* report);

/* fl_p2g mode 1 (NormalizeLiquidMacFaces3D + ApplyForces + stationary walls)
 * that also writes NormalizeCore's per-face validity, one byte per face
 * (LiquidFaceValidity3D numbering: 0 missing = no mass, 1 valid, 3 low mass =
 * positive mass at or below min_face_mass; liquid_boundary_transfer_3d.cc:
 * 785-805, validity 486-510), so a consumer can tell a face without liquid
 * from one whose normalized velocity is zero. face_mass may be NULL. */
int fl_p2g_normalized(fl_context* ctx, const fl_particles* sorted, const fl_transfer_params* params,
                      float* const u_pred[3], float* const face_mass[3], uint8_t* const validity[3], void* stream,
                      fl_report* report);

/* Pressure projection of the predicted face velocities of the box scene:
 * fluid = non-solid cells holding particles (from the last sort), Dirichlet
 * p = 0 against air, sealed against solid cells. Writes corrected velocities
 * and, optionally, the FP64 cell pressure (active_blocks*512 doubles, Pa). */
int fl_pressure_project(fl_context* ctx, const float* const u_pred[3], float* const u_new[3],
                        const fl_transfer_params* params, const fl_pressure_options* options,
                        fl_pressure_diagnostics* diagnostics, double* pressure_out, void* stream);

/* One application of the V-cycle preconditioner z = M^-1 r on the cells of the
 * last sort (fluid = non-solid cells holding particles), for checking the
 * multigrid against its FP64 restatement. r and z hold active_blocks*512 floats
 * in units of the full-face conductance. */
int fl_apply_vcycle(fl_context* ctx, const float* r, float* z, const fl_pressure_options* options, void* stream);

/* APIC G2P over sorted particles. With full_out == NULL: v <- PIC velocity,
 * C <- fitted slopes, x <- clamp(x + dt v) in place. Otherwise writes 24 floats
 * per sorted particle (MacParticleGatherResult3D layout) and leaves the state. */
int fl_g2p(fl_context* ctx, fl_particles* sorted, const float* const u_new[3], const float* const u_old[3],
           float dt, float* full_out, void* stream, fl_report* report);

/* One full liquid substep on the context-resident particle state:
 * topology -> sort -> P2G (+normalize, gravity, walls) -> pressure -> G2P (+advect).
 * The sort computes the cell order without moving the particles; P2G reads the
 * state through it and G2P writes the advected state, in cell order, into the
 * context's other particle buffer, which is the state after the call (take
 * fresh pointers from fl_state_particles after each step). */
int fl_step(fl_context* ctx, const fl_transfer_params* params, const fl_pressure_options* options,
            fl_pressure_diagnostics* diagnostics, void* stream, fl_report* report);

/* CUDA-event durations of the last fl_step's phases, ms:
 * [0] topology + sort, [1] P2G (tile + merge kernels), [2] pressure, [3] G2P. */
int fl_step_timings(fl_context* ctx, float* ms);

/* Host-side counts of kernels launched by this library since load: its own
 * kernels, and device-wide CUB algorithm invocations (exclusive scans). */
int fl_kernel_launches(unsigned long long* own, unsigned long long* library);

/* Context-resident particle state and buffers (device pointers). fl_step
 * records, in its G2P, which blocks the advected particles occupy and the next
 * fl_step builds its topology from that record; a caller that writes positions
 * through fl_state_particles' pointers between steps calls
 * fl_topology_from_particles afterwards so the record is rebuilt. */
int fl_upload_particles(fl_context* ctx, const float* host_soa, uint64_t count, void* stream);
/* Stages a next input: copies 15 x count FP32 SoA from host memory (pinned,
 * for the copy to run asynchronously) on the context's own non-blocking stream
 * into a free particle buffer and returns. The next fl_step starts from the
 * oldest staged input instead of the current state (as if it had been
 * uploaded), so the input of step k + 1 can be copied while step k runs. At
 * most two inputs wait (FL_UNAVAILABLE otherwise); fl_upload_particles drops
 * them. The first call allocates two more particle buffers. */
int fl_stage_particles(fl_context* ctx, const float* host_soa, uint64_t count);
int fl_download_particles(fl_context* ctx, float* host_soa, void* stream);
int fl_state_particles(fl_context* ctx, fl_particles* out);
/* Face buffers of the last step: u_pred[3], u_new[3] (floats), pressure (doubles), cell type (bytes). */
int fl_state_fields(fl_context* ctx, float* u_pred[3], float* u_new[3], double** pressure, uint8_t** cell_type,
                    int32_t** cell_start);

/* End-to-end substep with host buffers: uploads 15 x count FP32 SoA from
 * host_in (pinned or pageable), runs fl_step and downloads the state to host_out. */
int fl_step_host(fl_context* ctx, const float* host_in, float* host_out, uint64_t count,
                 const fl_transfer_params* params, const fl_pressure_options* options,
                 fl_pressure_diagnostics* diagnostics, void* stream);

/* ---- reference-shaped operators (host FP64 data, reference 4^3 slot order) ---- */

/* DepositMac3D on the GPU: particles are MacTransferParticle3D records of 19
 * doubles (sorted xyz, trial xyz, mass, velocity xyz, slope rows); blocks are
 * the reference's 4^3 active blocks; outputs follow the reference's owned-slot
 * order (192 slots per 4^3 block, blocks sorted by (z,y,x)). FP32 arithmetic. */
int fl_deposit_mac_3d(const double origin[3], double h, const int32_t* blocks, uint64_t block_count,
                      const double* particles, uint64_t particle_count, double* face_mass, double* face_momentum,
                      fl_measurement* measurement);

/* DepositMacQuanta3D / CudaDepositMacQuanta3D: FP64 contributions rounded to
 * nearest-even quanta and summed with 64-bit integer atomics (order-independent). */
int fl_deposit_mac_quanta_3d(const double origin[3], double h, const int32_t* blocks, uint64_t block_count,
                             const double* particles, uint64_t particle_count, double mass_per_quantum,
                             double momentum_per_quantum, uint64_t declared_capacity, int64_t* mass_quanta,
                             int64_t* momentum_quanta, fl_measurement* measurement);

/* GatherMac3D / CudaGatherMac3D: 24 doubles per particle in input order. */
int fl_gather_mac_3d(const double origin[3], double h, const int32_t* blocks, uint64_t block_count,
                     const double* particles, uint64_t particle_count, const double* old_face_velocities,
                     const double* new_face_velocities, double* results, fl_measurement* measurement);

/* Block layout passed to fl_p2g_static_scratch: device arrays of 8^3-block
 * coordinates (block_count x 3, ordinal order), 26-neighbourhood ordinals
 * (block_count x 27, index (dz+1)*9+(dy+1)*3+(dx+1), -1 inactive, -2 outside
 * the lattice) and per-cell particle ranges (block_count*512 + 1). */
typedef struct {
  double origin[3];
  double h;
  int32_t solid_lo[3];
  int32_t solid_hi[3];
  const int32_t* block_coords;
  const int32_t* neighbors;
  const int32_t* cell_start;
  uint64_t block_count;
} fl_static_grid;

/* P2G that allocates nothing (no counterpart in the reference). For callers
 * that cannot call cudaMalloc where they deposit -- a host engine whose
 * device memory all comes from its own pool, or a substep that must not
 * allocate once started -- this runs the fl_p2g kernels without a context.
 * The caller passes layout, sorted particles and output face arrays (same
 * meaning and modes as fl_p2g); the per-block tile scratch is a file-scope
 * static device array of at most 512 active blocks (13.5 MB, plus 1.1 MB for
 * a checked copy of the layout, held on every GPU that loads the library
 * until exit). More blocks return FL_RESOURCE_EXHAUSTED. The layout is
 * checked on the device first (neighbour ordinals below block_count, cell
 * ranges non-decreasing inside [0, count]) and the P2G kernels read a copy
 * forced into range, so a malformed layout cannot make them read or write
 * out of bounds; with a report the call waits for the check and returns
 * FL_INVALID_ARGUMENT (first bad entry in first_bad_index: cell_start
 * index, or block_count*512+1 + neighbour index) without writing any output.
 * Without an sm_100 device it returns FL_FAILED_PRECONDITION. The first call
 * on a device looks up the arrays' device addresses, so make it before any
 * stream capture. All calls on a GPU share that GPU's arrays, which keep the
 * last call's contents: calls that overlap on the same GPU (for example on
 * concurrent streams) race and must be serialized by the caller. */
int fl_p2g_static_scratch(const fl_static_grid* grid, const fl_particles* sorted, const fl_transfer_params* params,
                          int mode, float* const out0[3], float* const out1[3], void* stream, fl_report* report);

/* ---- learned block preconditioner (no counterpart in the reference) -------
 * A 3D U-Net over one 8^3 pressure block plus a one-cell halo (channels
 * 16/32/64, 3x3x3 convolutions, 141,937 FP32 parameters flattened layer by
 * layer as weight [Cout][Cin][taps] then bias). Input item: 2 x 10^3 floats
 * (residual / block scale, cell mask 1 fluid, 0 air, -1 solid), output item: 512
 * floats (correction / block scale), both [channel][z][y][x]. All pointers are
 * device pointers; calls are stream-ordered and allocate nothing. */
typedef struct fl_unet fl_unet;
int64_t fl_unet_param_count(void);
/* Training workspace for up to max_batch items (all activations of one forward). */
int fl_unet_create(int max_batch, fl_unet** out);
int fl_unet_destroy(fl_unet* net);
/* Training precision of fl_unet_forward / fl_unet_backward: 0 (default) the
 * FP32 convolution kernels; 1 each 3x3x3 convolution (forward, data and weight
 * gradients) as a GEMM of BF16 operands with FP32 accumulation on the tensor
 * cores (im2col operands formed by this library's kernels, the GEMM by
 * cuBLAS), parameters, activations, gradients and Adam in FP32. Enabling
 * reserves the operand buffers: FL_OUT_OF_RANGE for a workspace of more than
 * 8192 items, FL_RESOURCE_EXHAUSTED if they cannot be allocated. */
int fl_unet_set_tensor_cores(fl_unet* net, int enable);
/* He-uniform weights from a counter-based stream (SplitMix64 of seed and index), zero biases. */
int fl_unet_init_params(float* params, uint64_t seed, void* stream);
/* FP32 forward pass; keeps the activations for fl_unet_backward. */
int fl_unet_forward(fl_unet* net, const float* params, const float* input, int batch, float* output, void* stream);
/* Gradient of sum(grad_output * output) of the last forward with respect to the parameters. */
int fl_unet_backward(fl_unet* net, const float* params, const float* grad_output, int batch, float* grad_params,
                     void* stream);
/* Masked squared error of batch (<= 1024) items of 512 cells and d loss / d output.
 * relative 0: loss = sum mask (output - target)^2 / max(1, sum mask);
 * relative 1: loss = mean over the items with sum mask target^2 > 0 of
 *             sum mask (output - target)^2 / sum mask target^2. */
int fl_unet_masked_mse(const float* output, const float* target, const float* mask, int batch, int relative,
                       float* loss, float* grad_output, void* stream);
/* Block-residual loss of batch (<= 1024) items and d loss / d output: with
 * r_b the input's residual on the block's fluid cells (channel 0 of the 10^3
 * window, channel 1 the cell mask) and A_b the level-0 pressure operator on
 * those cells (unit conductance to fluid and air neighbours, the block's
 * neighbours held at zero), loss = mean over the items with r_b != 0 of
 * |r_b - A_b output|^2 / max(|r_b|^2, 1) (windows scaled to max |r| = 1). The
 * zero output scores at most 1; an exact inverse of A_b on the block scores 0. */
int fl_unet_block_residual_loss(const float* output, const float* input, int batch, float* loss, float* grad_output,
                                void* stream);
/* Adam with bias correction at step >= 1: m, v updated in place, params -= lr mhat / (sqrt(vhat) + eps). */
int fl_adam_step(float* params, const float* grads, float* m, float* v, uint64_t count, int step, float lr,
                 float beta1, float beta2, float eps, void* stream);

/* Training pairs from the context's current projection (the last step's
 * predicted velocities and cells): a converged solve gives p*, then for each
 * iteration cap k in `iterations` the solve from p = 0 is stopped after k
 * flexible-CG iterations and every block holding fluid yields one item:
 * input = (r_k / s, mask) on the block plus halo, target = (p* - p_k) / s,
 * target_mask = fluid cells, with r_k = b - A p_k and s = max |r_k| over the
 * input window. With options->preconditioner == 2 the input residual is the
 * one the composite preconditioner's network sees, r_k - A V(r_k) after one
 * V-cycle V (the target stays p* - p_k). Writes at most `capacity` items;
 * `written` gets the count. */
int fl_collect_training_pairs(fl_context* ctx, const fl_transfer_params* params, const fl_pressure_options* options,
                              const int32_t* iterations, int iteration_count, float* inputs, float* targets,
                              float* target_mask, uint64_t capacity, uint64_t* written);
/* Loads trained FP32 parameters (device pointer) into the context's BF16
 * inference weights used when fl_pressure_options.preconditioner == 1. */
int fl_set_learned_preconditioner(fl_context* ctx, const float* params, void* stream);
/* One application z = U(r) of the learned preconditioner on the cells of the
 * last sort (r, z: active_blocks*512 floats, natural layout). kernels 0: the
 * tensor-core inference used inside the solver (BF16 activations, FP32
 * accumulation); 1: the FP32 training forward pass, for checking the former. */
int fl_apply_learned(fl_context* ctx, const float* r, float* z, int kernels, void* stream);

/* ProjectMacPressure3D / CudaProjectMacPressure3D on the GPU
 * (native/include/fluidity/host/mac_pressure_3d.h:14-102,
 * native/include/fluidity/host/cuda_mac_pressure_3d.h:19-20) for the bounded
 * owned-face systems they take: 1-4096 cells in strictly increasing (z,y,x)
 * order, at most 24576 faces. Host FP64 arrays, one record per cell / face:
 *   cell_index  3 x int32 (x, y, z)
 *   cell_values 5 doubles: fluid volume m^3, target divergence 1/s, bulk
 *               modulus Pa (0 = infinite: no compliance), previous pressure Pa,
 *               integrated inward wall flux m^3/s
 *   face_index  4 x int32 (normal axis, x, y, z of the head cell)
 *   face_kind   0 sealed, 1 internal, 2 Dirichlet (MacPressureFace3D::pressure_link)
 *   face_values 6 doubles: open area m^2, inverse density m^3/kg, pressure-gradient
 *               distance m, predicted normal velocity m/s, wall normal velocity m/s,
 *               pressure lift Pa (the internal jump, or the Dirichlet exterior pressure)
 * Solves in FP64 to ||b - Ap||_2 <= rel_tol ||b||_2, or the reference's gate
 * 2e-6 + 2e-6 ||b||_2 when rel_tol == 0, within max_iterations (1-65536), and
 * evaluates the corrected face velocities, residuals b - Ap and physical defects.
 * Outputs (pressure, rhs, residual, defect: cell_count; corrected_u: face_count;
 * gauge_ordinals: up to cell_count, may be NULL) are written only on FL_OK.
 * FL_INVALID_ARGUMENT for bad data or face topology, FL_RESOURCE_EXHAUSTED above
 * the caps, FL_FAILED_PRECONDITION for an incompatible unanchored component (or
 * no device), FL_OUT_OF_RANGE for an unrepresentable velocity, FL_INTERNAL for a
 * residual/defect identity mismatch, FL_ABORTED when the gate is not met. */
typedef struct {
  uint64_t iterations;
  double true_residual_l2;           /* m^3/s */
  double max_volume_scaled_residual; /* max |b - Ap| / V, 1/s */
  double max_cell_constraint_defect; /* 1/s */
  double rhs_l2;                     /* ||b||_2, m^3/s */
  uint64_t gauge_count;              /* cells pinned to zero pressure */
} fl_mac_pressure_diagnostics;
int fl_project_mac_pressure_3d(double h, double dt, const int32_t* cell_index, const double* cell_values,
                               uint64_t cell_count, const int32_t* face_index, const int32_t* face_kind,
                               const double* face_values, uint64_t face_count, int max_iterations, double rel_tol,
                               double* pressure, double* corrected_u, double* rhs, double* residual, double* defect,
                               uint64_t* gauge_ordinals, fl_mac_pressure_diagnostics* diagnostics,
                               fl_measurement* measurement);

/* ---- asynchronous device-to-host snapshots of the particle state ----
 *
 * Replaces CudaLiquidSnapshotQueue3D (native/include/fluidity/host/
 * cuda_liquid_snapshot_3d.h:56-110, native/cuda/liquid_snapshot_3d_host.cc:
 * 228-380): two reservations, each with its own non-blocking stream and a pair
 * of timing events; tickets carry a never-reused reservation number and the
 * source epoch; a slot goes Pending -> Ready (copy complete) -> Writer
 * (finished, held by the caller) -> Free. The copy reads the context's current
 * particle buffer in place: every later write into that buffer (the G2P of the
 * step after next, an upload, a permuting sort) waits for the copy, so the
 * steps in between run beside it. A device kernel on the slot's stream checks
 * the copied state (all 15 values finite, positions inside the block lattice)
 * and stamps count and epoch into a control record copied behind it; finish
 * verifies that record (FL_DATA_LOSS, after which the queue only returns
 * FL_INTERNAL, as the reference's poisoned job). Host memory: three pinned
 * buffers of 15 x capacity floats, reference-counted between the slots and the
 * last valid snapshot, so finish copies nothing on the host. A queue and its
 * context are used from one thread with the context's device current; destroy
 * the queue before the context (fl_context_destroy returns
 * FL_FAILED_PRECONDITION while a queue is live). */
typedef struct fl_snapshot_queue fl_snapshot_queue;
typedef struct {
  uint64_t generation;    /* > 0, increasing between finished snapshots */
  uint64_t frame_ordinal; /* completed frame */
  double time;            /* s */
} fl_epoch;
typedef struct {
  uint32_t slot;
  uint64_t reservation;
  fl_epoch epoch;
} fl_snapshot_ticket;
typedef struct {
  const float* soa; /* host: 15 arrays of `count` floats (x[3], v[3], C rows[9]), in cell order */
  uint64_t count;
  fl_epoch epoch;
  float copy_ms; /* CUDA-event interval around the check and the copy on the slot's stream */
} fl_snapshot_view;
#define FL_SNAPSHOT_PENDING 0
#define FL_SNAPSHOT_READY 1
#define FL_SNAPSHOT_CANCELED 2

/* Create (CudaLiquidSnapshotQueue3D::Create): pinned buffers for the context's capacity. */
int fl_snapshot_queue_create(fl_context* ctx, fl_snapshot_queue** out);
/* Drains the slot streams and frees everything; views from it end. */
int fl_snapshot_queue_destroy(fl_snapshot_queue* queue);
/* BeginCopy: snapshot of the context's state after the work queued on `stream`.
 * FL_INVALID_ARGUMENT: generation 0; FL_FAILED_PRECONDITION: generation not
 * above the last finished one, or another device current; FL_ALREADY_EXISTS:
 * the epoch's generation is live in a slot; FL_UNAVAILABLE: both slots held
 * (poll/finish/release/cancel, then retry); FL_OUT_OF_RANGE: reservations exhausted. */
int fl_snapshot_begin(fl_snapshot_queue* queue, const fl_epoch* epoch, void* stream, fl_snapshot_ticket* ticket);
/* Poll: nonblocking; *progress = FL_SNAPSHOT_PENDING, _READY, or _CANCELED (once,
 * for a canceled copy that has completed; the ticket is stale afterwards).
 * FL_FAILED_PRECONDITION for a stale ticket or one already finished. */
int fl_snapshot_poll(fl_snapshot_queue* queue, const fl_snapshot_ticket* ticket, int* progress);
/* Poll that blocks until the copy has completed. */
int fl_snapshot_wait(fl_snapshot_queue* queue, const fl_snapshot_ticket* ticket, int* progress);
/* Finish: requires READY and an epoch not older than the last finished one
 * (generation above, frame and time not below); validates the control record
 * and publishes the view (held until fl_snapshot_release) as the last valid
 * snapshot. FL_FAILED_PRECONDITION for pending/stale/out-of-order/canceled
 * tickets, FL_DATA_LOSS for a failed check. Failures keep the last valid snapshot. */
int fl_snapshot_finish(fl_snapshot_queue* queue, const fl_snapshot_ticket* ticket, fl_snapshot_view* out);
/* Ends a finished snapshot's lease (LiquidSnapshotLease3D destruction); the slot becomes free. */
int fl_snapshot_release(fl_snapshot_queue* queue, const fl_snapshot_ticket* ticket);
/* Cancel: a READY slot is freed at once; a PENDING one is freed when poll reports
 * FL_SNAPSHOT_CANCELED. FL_FAILED_PRECONDITION for stale or finished tickets. */
int fl_snapshot_cancel(fl_snapshot_queue* queue, const fl_snapshot_ticket* ticket);
/* LastValidHostSnapshot: the last finished snapshot (kept after its release, until
 * the next finish); FL_FAILED_PRECONDITION before the first finish. */
int fl_snapshot_last_valid(fl_snapshot_queue* queue, fl_snapshot_view* out);

/* Plain device<->host copies for callers without their own CUDA runtime binding. */
int fl_copy_to_host(void* host, const void* device, uint64_t bytes);
int fl_copy_to_device(void* device, const void* host, uint64_t bytes);

/* Library information: compiled architecture (e.g. 1000) and whether a usable device exists. */
int fl_runtime_info(int* compiled_architecture, int* device_count, int* device_major, int* device_minor);

/* ---- bounded boundary-aware transfers: the liquid scheduler's backend operations ----
 *
 * The operations behind LiquidSubstepBackend3D's .deposit, .normalize,
 * .predict_missing_face, .forces and .gather
 * (native/include/fluidity/host/liquid_substep_backend_3d.h:121-194), as the
 * reference's CPU table binds them (native/src/liquid_substep_3d_cpu.cc:
 * 775-803, 847-849; numerics native/src/liquid_boundary_transfer_3d.cc:
 * 56-308, 327-668, 785-805, 953-984) and its CUDA table replaces them
 * (native/cuda/liquid_transfer_stages_3d_host.cc:375-620). They run on the
 * reference's owned sparse grid: 4^3-cell blocks in strictly increasing (z,y,x)
 * order, 192 face slots per block (normal axis, then local (z,y,x)), at most
 * 1024 particles and 24576 face slots (liquid_boundary_transfer_3d.h:16-17).
 *
 * An fl_boundary reserves its device and pinned host storage for those caps
 * when it is created; the operations allocate nothing. Each call copies its
 * inputs to the device, runs its kernels in FP64 on one non-blocking stream and
 * synchronizes it, and writes its outputs only on FL_OK (the reference's
 * "errors publish nothing"). Codes follow the CPU operations: for several
 * failing items the code is that of the first in the CPU loop order
 * (particle, then component, then stencil sample). Deposit quanta, normalized
 * faces and forces are bit-identical to the CPU operations; the gather's ghost
 * fits use the device's hypot, so a filled ghost velocity can differ from the
 * CPU's in its last bits.
 *
 * The record layouts below are byte-compatible with the reference's
 * (LiquidBoundaryParticle3D, LiquidBoundaryFaceTag3D, MacFaceDepositQuanta3D,
 * CompatibleMacFaceSample3D, LiquidPrescribedWallSample3D,
 * LiquidBoundaryParticleGather3D: native/include/fluidity/base/
 * liquid_boundary_transfer_types_3d.h:4-45, mac_transfer_types_3d.h:7-30), so a
 * backend passes the scheduler's spans through unchanged. */
typedef struct fl_boundary fl_boundary;

typedef struct {
  double origin[3];      /* world position of lattice point (0,0,0), m */
  double h;              /* cell width, m (positive normal) */
  const int32_t* blocks; /* block_count x (x, y, z), 4^3-cell blocks, strictly increasing (z,y,x) */
  uint64_t block_count;  /* face slots = 192 x block_count */
} fl_owned_grid;

typedef struct {
  double sorted_position[3]; /* m, position at the last sort */
  double trial_position[3];  /* m, position used for this transfer */
  double mass;               /* kg */
  double velocity[3];        /* m/s */
  double slopes[9];          /* APIC slope rows (x, y, z), 1/s */
  int64_t side_tag;
  uint8_t affine_enabled;
  uint8_t pad[7];
} fl_boundary_particle;

typedef struct {
  int64_t side_tag;
  uint8_t structurally_eligible;
  uint8_t pad[7];
} fl_face_tag;

typedef struct {
  int64_t mass;     /* quanta */
  int64_t momentum; /* quanta */
  int64_t stress;   /* reserved, zero for liquid */
} fl_face_quanta;

typedef struct {
  double mass_per_quantum;     /* kg, a positive normal power of two */
  double momentum_per_quantum; /* kg m/s, a positive normal power of two */
  uint64_t declared_capacity;  /* declared particle capacity, <= 1024 */
} fl_quantization;

typedef struct {
  uint64_t face_slot;
  uint8_t compatible;
  uint8_t pad[7];
  double normalized_weight;
  double normalized_weight_gradient[3]; /* 1/m */
  double centered_face_offset[3];       /* m */
} fl_compatible_sample;

typedef struct {
  uint8_t available;
  uint8_t pad[7];
  int64_t side_tag;
  double unit_normal[3];
  double wall_velocity[3]; /* m/s */
} fl_wall_sample;

/* Validity: 0 missing, 1 valid, 2 predicted, 3 low mass (LiquidFaceValidity3D). */
typedef struct {
  double velocity_sample_time; /* s */
  double wall_sample_time;     /* s */
  const double* face_velocities;
  const uint8_t* validity;
  const fl_face_tag* face_tags;
  const fl_wall_sample* walls;
} fl_velocity_history;

typedef struct {
  double new_pic_velocity[3];
  double grid_velocity_increment[3];
  double particle_minus_old_pic_velocity[3];
  double fitted_velocity_slopes[9]; /* rows, 1/s */
  double velocity_gradient[9];      /* rows, 1/s */
  uint8_t affine_enabled;
  uint8_t old_pic_fallback;
  uint8_t new_pic_fallback;
  uint8_t low_mass_fallback;
  uint8_t pad[4];
} fl_gathered_particle;

int fl_boundary_create(fl_boundary** out);
int fl_boundary_destroy(fl_boundary* boundary);

/* DepositCompatibleMacQuanta3D: quanta per face slot and 3 x 27 compatible
 * samples per particle (particle, component, stencil (z,y,x) order). */
int fl_boundary_deposit(fl_boundary* boundary, const fl_owned_grid* grid, const fl_boundary_particle* particles,
                        uint64_t particle_count, const fl_face_tag* face_tags, const fl_quantization* quantization,
                        fl_face_quanta* face_quanta, fl_compatible_sample* compatible_stencils,
                        fl_measurement* measurement);

/* NormalizeLiquidMacFaces3D: masses (kg), velocities (m/s, 0 unless valid), validity. */
int fl_boundary_normalize(fl_boundary* boundary, const fl_face_quanta* face_quanta, uint64_t face_count,
                          const fl_quantization* quantization, double minimum_face_mass, double* face_masses,
                          double* face_velocities, uint8_t* validity, fl_measurement* measurement);

/* The CPU table's .forces: predicted = old + dt * acceleration[normal axis], per slot. */
int fl_boundary_forces(fl_boundary* boundary, const fl_owned_grid* grid, const double* old_face_velocities,
                       const double acceleration[3], double step_duration, double* predicted_face_velocities,
                       fl_measurement* measurement);

/* The CPU table's .predict_missing_face: the old history continued at one slot
 * (same-side donors within 2h, wall projection) plus dt * acceleration. */
int fl_boundary_predict_face(fl_boundary* boundary, const fl_owned_grid* grid, const fl_velocity_history* old_history,
                             uint64_t face_slot, int64_t side_tag, const double acceleration[3],
                             double step_duration, double* predicted_face_velocity, fl_measurement* measurement);

/* fl_project_mac_pressure_3d on the boundary object's scratch and stream, which
 * are reserved for the operator's caps when the object is created: the
 * projection allocates nothing. Same arguments, outputs and codes. */
int fl_boundary_project(fl_boundary* boundary, double h, double dt, const int32_t* cell_index,
                        const double* cell_values, uint64_t cell_count, const int32_t* face_index,
                        const int32_t* face_kind, const double* face_values, uint64_t face_count, int max_iterations,
                        double rel_tol, double* pressure, double* corrected_u, double* rhs, double* residual,
                        double* defect, uint64_t* gauge_ordinals, fl_mac_pressure_diagnostics* diagnostics,
                        fl_measurement* measurement);

/* ---- pressure-link assembly (.links) ----
 * BuildLiquidPressureLinks3D (native/src/liquid_boundary_workspace_3d.cc:
 * 189-195 -> liquid_boundary_geometry_3d.cc:1077-1286 after the frozen-view
 * checks of :1289-1380 and the link arithmetic of base/
 * liquid_boundary_geometry_math_3d.h:676-689): the frozen cells become
 * pressure cells; each frozen face becomes a sealed, internal (two liquid
 * endpoints, or a certified internal interface with its jump and mixed
 * density) or Dirichlet air link (pressure-gradient distance theta h with
 * theta clamped to [0.05, 1], exterior pressure = ambient or the air cell's
 * gas pressure plus sigma * curvature). Records in frozen order. */
typedef struct {
  int32_t cell_index[3];
  int32_t pad;
  double signed_distance; /* m, negative in the liquid */
} fl_center_sample;
typedef struct {
  int32_t cell_index[3];
  int32_t pad;
  double fluid_volume;    /* m^3 */
  double center_distance; /* m, negative */
  double curvature;       /* 1/m */
} fl_frozen_cell;
typedef struct {
  int32_t axis;
  int32_t lattice[3];
  uint64_t face_slot;
  double open_area;            /* m^2 */
  double blocked_area;         /* m^2, h^2 - open_area */
  double wall_normal_velocity; /* m/s */
  double prescribed_wall_flux; /* m^3/s, when has_prescribed_wall_flux */
  uint8_t has_prescribed_wall_flux;
  uint8_t is_low_x_piston_face;
  uint8_t pad[6];
} fl_frozen_face;
typedef struct {
  const fl_owned_grid* grid;
  const fl_center_sample* centers; /* strictly increasing (z,y,x) */
  uint64_t center_count;
  const fl_frozen_cell* cells; /* strictly increasing (z,y,x), <= 4096 */
  uint64_t cell_count;
  const fl_frozen_face* faces; /* strictly increasing owned slot, <= 24576 */
  uint64_t face_count;
  double step_duration;   /* s */
  double liquid_density;  /* kg/m^3 */
  double surface_tension; /* N/m */
} fl_frozen_geometry;
typedef struct {
  double target_divergence; /* 1/s */
  double bulk_modulus;      /* Pa, +inf for no compliance */
  double previous_pressure; /* Pa */
  double density;           /* kg/m^3, when has_density */
  uint8_t has_density;
  uint8_t pad[7];
} fl_pressure_cell_fields;
typedef struct {
  int32_t cell_index[3];
  int32_t pad;
  double gas_gauge_pressure; /* Pa */
} fl_air_cell_pressure;
typedef struct {
  uint64_t face_ordinal;
  double tail_fraction;
  double surface_tension;
  double curvature_tail_to_head;
  double normal_viscous_jump_tail_to_head;
} fl_internal_interface;
typedef struct {
  const fl_pressure_cell_fields* cells;     /* frozen cell order */
  const double* predicted_face_velocities;  /* frozen face order, m/s */
  double ambient_pressure;                  /* Pa */
  const double* wetted_piston_face_fluxes;  /* NULL, or one per face (m^3/s) */
  const uint8_t* has_wetted_piston_face_flux;
  const fl_air_cell_pressure* air; /* strictly increasing (z,y,x) */
  uint64_t air_count;
  const fl_internal_interface* interfaces; /* strictly increasing face ordinal */
  uint64_t interface_count;
} fl_pressure_fields;
typedef struct {
  int32_t cell_index[3];
  int32_t pad;
  double fluid_volume, target_divergence, bulk_modulus, previous_pressure, integrated_inward_wall_flux;
} fl_pressure_cell;
/* link_kind: 0 sealed, 1 internal (link_value = jump, Pa), 2 Dirichlet (exterior pressure, Pa). */
typedef struct {
  int32_t axis;
  int32_t lattice[3];
  double open_area, inverse_density, pressure_gradient_distance, predicted_normal_velocity, wall_normal_velocity;
  double link_value;
  double prescribed_wall_flux;
  int32_t link_kind;
  uint8_t has_prescribed_wall_flux;
  uint8_t pad[3];
} fl_pressure_link;

/* ---- geometry freeze (.freeze) ----
 * FreezeLiquidBoundaryGeometry3D (native/src/liquid_boundary_workspace_3d.cc:
 * 186 -> liquid_boundary_geometry_3d.cc:2109-2143 and FreezeCore :765-1075,
 * with the geometry queries of base/liquid_boundary_geometry_math_3d.h:
 * 657-847): each candidate cell's liquid volume from its eight corner
 * distances (six diagonal tetrahedra clipped by the interpolated liquid
 * plane and by the obstacle's planes), the kept cells' faces with their open
 * and blocked areas, the outward curvature of interface cells (exact, or from
 * the centred second differences of the centre distances) and the capillary
 * step bound. Obstacles: none, a translating halfspace, a translating slab or
 * an open tank with its low-x piston (the piston's share of a closed face
 * becomes a prescribed wall flux); sampled solids are not offered here. The host stages the
 * sample lookups and keeps the reference's error order; the device computes
 * every volume, area, curvature and bound. */
typedef struct {
  int32_t corner_index[3]; /* the lattice corner at the cell's low corner */
  int32_t pad;
  double signed_distance; /* m, negative in the liquid */
} fl_corner_sample;
#define FL_OBSTACLE_NONE 0
#define FL_OBSTACLE_HALFSPACE 1
#define FL_OBSTACLE_SLAB 2
#define FL_OBSTACLE_OPEN_TANK 3
typedef struct {
  int32_t kind; /* FL_OBSTACLE_* */
  int32_t pad;
  double unit_normal[3];
  double coordinate;       /* halfspace: start plane coordinate; slab: start centre coordinate (m) */
  double half_width;       /* slab only (m) */
  double wall_velocity[3]; /* m/s */
  /* open tank (AxisAlignedLiquidTank3D): start low x, high x, floor y, low z,
   * high z (m; open above the floor) and the low-x piston's x velocity (m/s) */
  double tank[6];
} fl_obstacle;
typedef struct {
  const fl_owned_grid* grid;
  const int32_t* cell_indices; /* 3 per candidate, strictly increasing (z,y,x), <= 4096 */
  uint64_t cell_count;
  const fl_center_sample* centers; /* strictly increasing (z,y,x) */
  uint64_t center_count;
  const fl_corner_sample* corners; /* strictly increasing (z,y,x) */
  uint64_t corner_count;
  fl_obstacle obstacle;
  double step_duration;   /* s */
  double liquid_density;  /* kg/m^3 */
  double surface_tension; /* N/m */
  double exact_curvature; /* 1/m, when has_exact_curvature */
  uint8_t has_exact_curvature;
  uint8_t pad[7];
} fl_freeze_inputs;
/* cells: room for cell_count records, faces: room for 6 * cell_count; both
 * in frozen order (cells by (z,y,x), faces by owned slot). The capillary
 * bound is +inf without a capillary interface. Outputs are written only on
 * FL_OK; a call allocates nothing. */
int fl_boundary_freeze(fl_boundary* boundary, const fl_freeze_inputs* inputs, fl_frozen_cell* cells,
                       uint64_t* cell_count, fl_frozen_face* faces, uint64_t* face_count,
                       double* capillary_step_bound, fl_measurement* measurement);

/* ---- wetted piston (.wetted_piston) ----
 * ComputeWettedPiston3D (native/src/wetted_piston_3d.cc:342-571 with
 * base/wetted_piston_math_3d.h): the wet area of the open tank's low-x piston
 * under the liquid field, per lattice patch of the piston plane, as
 * outward-rounded [lower, upper] enclosures, and each receiver face's signed
 * flux (positive into the tank): the sum, in (z, y) patch order, of the
 * midpoint-area fluxes of the patches assigned to it. Patches come in (z, y)
 * order, including dry receivers; a wet patch without a receiver joins the
 * receiver directly below it. Frozen cells and faces as fl_boundary_freeze
 * returns them. */
#define FL_PISTON_FIELD_SPHERE 0         /* LiquidAnalyticSphere3D */
#define FL_PISTON_FIELD_PARTICLE_UNION 1 /* LiquidParticleSphereUnion3D over the particle positions */
#define FL_PISTON_FIELD_PLANE 2          /* LiquidHorizontalPlaneSurface3D */
typedef struct {
  int32_t kind; /* FL_PISTON_FIELD_* */
  int32_t pad;
  double sphere_center[3]; /* m, analytic sphere */
  double radius;           /* m, analytic sphere or each particle's sphere */
  double plane_height_y;   /* m, plane */
} fl_piston_field;
typedef struct {
  int32_t lattice_y, lattice_z;
  double area[2]; /* m^2, [lower, upper] */
  uint64_t receiver_face_ordinal;
  uint8_t has_receiver;
  uint8_t pad[7];
  double receiver_area[2]; /* m^2 assigned to this receiver */
  double receiver_flux[2]; /* m^3/s enclosure of its assigned flux */
} fl_piston_patch;
/* patches: room for patch_capacity records (at most 24576 are produced);
 * face_fluxes / has_face_flux: one per frozen face. Outputs are written only
 * on FL_OK; a call allocates nothing. */
int fl_boundary_wetted_piston(fl_boundary* boundary, const fl_owned_grid* grid, const fl_frozen_cell* cells,
                              uint64_t cell_count, const fl_frozen_face* faces, uint64_t face_count,
                              const fl_piston_field* field, const double* particle_positions,
                              uint64_t particle_count, const double tank[6], fl_piston_patch* patches,
                              uint64_t patch_capacity, uint64_t* patch_count, double* face_fluxes,
                              uint8_t* has_face_flux, double whole_area[2], double whole_flux[2],
                              uint64_t* attached_patch_count, fl_measurement* measurement);

int fl_boundary_links(fl_boundary* boundary, const fl_frozen_geometry* geometry, const fl_pressure_fields* fields,
                      fl_pressure_cell* cells, fl_pressure_link* faces, uint64_t* lower_theta_regularization_count,
                      fl_measurement* measurement);

/* GatherLiquidBoundaryParticles3D: one record per particle in input order;
 * fallback_counts = old PIC, new PIC and low-mass fallback particle counts. */
int fl_boundary_gather(fl_boundary* boundary, const fl_owned_grid* grid, const fl_boundary_particle* particles,
                       uint64_t particle_count, double old_time, double new_time,
                       const fl_velocity_history* old_history, const fl_velocity_history* new_history,
                       fl_gathered_particle* gathered, uint64_t fallback_counts[3], fl_measurement* measurement);

#ifdef __cplusplus
}
#endif
#endif
