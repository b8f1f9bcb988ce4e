/* FP64 CPU restatement of FluidiTy's liquid-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. It is loaded by the
 * parity tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline and
 * --impl reference legs; no product code links it.
 *
 * Pinned against (a) the reference's own CPU operators compiled from source
 * (oracle/_ref/libfluidity_ref.so, see oracle/ref/Makefile) and (b) the golden
 * vectors generated from the reference's Python fixtures (tests/golden/).
 *
 * Layout: a dense box of cells [lo, lo+n) per axis. Face arrays for normal axis a
 * have (n[a]+1) entries along a and n[b] along the two other axes, x fastest.
 */
#ifndef FL_ORACLE_H_
#define FL_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double origin[3];
  double h;
  int32_t lo[3];
  int32_t n[3];
} fo_box;

/* Status codes follow the reference's absl codes (0 OK, 3 invalid argument,
 * 9 failed precondition, 10 aborted, 11 out of range, 13 internal). */
enum { FO_OK = 0, FO_INVALID = 3, FO_PRECONDITION = 9, FO_ABORTED = 10, FO_RANGE = 11, FO_INTERNAL = 13 };

size_t fo_face_count(const fo_box* box, int axis);

/* 27 samples of one normal component in (z,y,x) order: faces (axis,x,y,z) and
 * values {weight, offset xyz (m), gradient xyz (1/m)}. */
int fo_stencil(const double origin[3], double h, int axis, const double pos[3], int32_t* faces, double* values);

/* P2G: per face mass and pure momentum (DepositMac3D semantics). mass may be
 * per particle (mass_stride 1) or one shared value (mass_stride 0). */
int fo_p2g(const fo_box* box, const double* x, const double* v, const double* c, const double* mass, int mass_stride,
           size_t np, double* face_mass[3], double* face_momentum[3]);

/* Quantized P2G (DepositMacQuanta3D semantics, nearest-even quanta per contribution). */
int fo_p2g_quanta(const fo_box* box, const double* x, const double* v, const double* c, const double* mass,
                  int mass_stride, size_t np, double mass_per_quantum, double momentum_per_quantum,
                  int64_t* mass_q[3], int64_t* momentum_q[3]);

/* Normalize (u = q/m when m > m_min) and add dt*g on every face. validity (LiquidFaceValidity3D):
 * 0 missing (no mass), 1 valid, 3 low mass (positive mass at or below m_min). */
void fo_normalize_forces(const fo_box* box, double* face_mass[3], double* face_momentum[3], double m_min, double dt,
                         const double g[3], double* u_pred[3], uint8_t* validity[3]);

/* G2P: 24 doubles per particle (PIC velocity, increment, fitted slope rows, gradient rows). */
int fo_g2p(const fo_box* box, const double* x, size_t np, double* u_old[3], double* u_new[3], double* out);

/* General integrated pressure system (ProjectMacPressure3D inputs). */
typedef struct {
  size_t nc, nf;
  const int32_t* cell_index;   /* nc x 3, (z,y,x)-sorted */
  const double* cell_values;   /* nc x 5: volume, target divergence, bulk modulus (0 = inf), previous p, wall flux */
  const int32_t* face_index;   /* nf x 4: axis, x, y, z (head cell) */
  const int32_t* face_kind;    /* 0 sealed, 1 internal, 2 Dirichlet */
  const double* face_values;   /* nf x 6: open area, inverse density, distance, predicted u, wall u, lift */
  double h, dt;
} fo_pressure_inputs;

typedef struct {
  double iterations, true_residual_l2, max_volume_scaled_residual, max_defect, rhs_l2, gauge_count;
} fo_pressure_diag;

/* Assemble b (Neumaier sums), choose gauges, solve to ||b-Ap|| <= rel_tol ||b|| (or the
 * reference gate when rel_tol <= 0) with FP64 Jacobi PCG, then evaluate residual,
 * physical defect and corrected face velocities. */
int fo_pressure_solve(const fo_pressure_inputs* in, double rel_tol, size_t max_iterations, double* pressure,
                      double* residual, double* defect, double* rhs, double* corrected_u, fo_pressure_diag* diag);

/* FP64 evaluation only, for given pressures. */
int fo_pressure_evaluate(const fo_pressure_inputs* in, const double* pressure, double* residual, double* defect,
                         double* rhs, double* corrected_u, fo_pressure_diag* diag);

/* Box scene helpers: solid wall layer on the box boundary, fluid = occupied non-solid cell.
 * cell_type: 0 solid, 1 fluid, 2 air (n[0]*n[1]*n[2], x fastest). */
void fo_classify_cells(const fo_box* box, const double* x, size_t np, uint8_t* cell_type);

/* One full APIC liquid step on the box (P2G, normalize+gravity, wall BC, pressure to
 * rel_tol, G2P with fitted slopes, advect and clamp). Updates x, v, c in place and
 * returns face velocities before/after projection and the pressure on fluid cells. */
typedef struct {
  double dt, density, gravity[3], m_min, rel_tol, clamp_margin;
  size_t max_iterations;
} fo_step_params;

int fo_step(const fo_box* box, const fo_step_params* params, double* x, double* v, double* c, size_t np,
            double* u_pred[3], double* u_new[3], double* cell_pressure, uint8_t* cell_type, fo_pressure_diag* diag);

/* fo_step with the pressure given instead of solved, for replaying one device
 * step at full size: FP32 SoA state in (15 x np), cell_pressure dense over the
 * box, G2P + advection only for particles first, first + stride, ... (15
 * doubles each into sample_out: x, v, C rows after the step). diag holds the
 * FP64 evaluation of the given pressure on the step's own system. */
int fo_step_replay(const fo_box* box, const fo_step_params* params, const float* soa, size_t np,
                   const double* cell_pressure, size_t first, size_t stride, double* u_pred[3], double* u_new[3],
                   uint8_t* cell_type, fo_pressure_diag* diag, double* sample_out);

/* Geometric multigrid V-cycle on the box (FP64 restatement of the GPU preconditioner):
 * red-black Gauss-Seidel, `pre`/`post` sweeps, `levels` levels, piecewise-constant
 * transfer with sum restriction and rediscretized coarse operators, `coarse_sweeps`
 * symmetric sweeps on the coarsest level. Applies z = M^{-1} r on fluid cells.
 * r and z are n-cell dense arrays in units normalized by the face conductance. */
int fo_vcycle(const fo_box* box, const uint8_t* cell_type, int levels, int pre, int post, int coarse_sweeps,
              const double* r, double* z);

#ifdef __cplusplus
}
#endif
#endif
