// Table-against-table harness for the liquid scheduler's backend operations.
// Test infrastructure only (the checker, never the product).
//
// Each bk_* entry runs ONE operation of a LiquidSubstepBackend3D table on host
// arrays: which == 0 the reference's own CPU table (CpuLiquidSubstepBackend3D,
// native/src/liquid_substep_3d_cpu.cc:703-859, compiled from its sources into
// libfluidity_ref.so), which == 1 the B200 table
// (B200LiquidBackend3D::operations(), fluidity_b200/adapter). Both receive the
// same SparseMacGrid3D, the same spans and fresh reference workspaces, so a
// test compares the two tables' outputs directly. The records are the
// reference's own types, passed through as bytes (their layouts match the
// C-ABI's, which the adapter checks at compile time). Every entry returns the
// operation's absl status code (0 = OK) and writes its outputs only on OK.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <vector>

#include "b200_liquid_substep_backend_3d.h"
#include "fluidity/host/liquid_boundary_workspace_3d.h"
#include "fluidity/host/mac_pressure_workspace_3d.h"
#include "fluidity/host/sparse_mac_grid_3d.h"
#include "fluidity/host/wetted_piston_3d.h"

#include <cmath>
#include <optional>

using namespace fluidity;

namespace {

// Host time of the last table operation alone (the harness's own record
// conversion, grid and workspace set-up excluded), in ms.
double g_last_op_ms = 0.0;

template <typename F>
auto TimedOp(F&& op) {
  const auto t0 = std::chrono::steady_clock::now();
  auto r = op();
  g_last_op_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return r;
}


constexpr std::size_t kParticles = 1024;
constexpr std::size_t kFaces = 24576;
constexpr std::size_t kCells = 4096;

std::unique_ptr<B200LiquidBackend3D>& B200() {
  static std::unique_ptr<B200LiquidBackend3D> backend;
  return backend;
}

// The table for `which`, or nullptr (with *code set) when it cannot be made.
const LiquidSubstepBackend3D* Table(int which, int* code) {
  static LiquidSubstepBackend3D cpu = CpuLiquidSubstepBackend3D();
  static LiquidSubstepBackend3D b200{};
  *code = 0;
  if (which == 0) return &cpu;
  if (!B200()) {
    auto made = B200LiquidBackend3D::Create();
    if (!made.ok()) {
      *code = static_cast<int>(made.status().code());
      return nullptr;
    }
    B200() = std::move(*made);
    b200 = B200()->operations();
  }
  return &b200;
}

int Code(const absl::Status& s) { return static_cast<int>(s.code()); }

std::vector<BlockIndex3D> Blocks(const int32_t* blocks, uint64_t nb) {
  std::vector<BlockIndex3D> out(nb);
  for (uint64_t i = 0; i < nb; ++i) out[i] = {blocks[3 * i], blocks[3 * i + 1], blocks[3 * i + 2]};
  return out;
}

absl::StatusOr<SparseMacGrid3D> Grid(const double origin[3], double h, const int32_t* blocks, uint64_t nb) {
  return SparseMacGrid3D::Create({{origin[0], origin[1], origin[2]}, h}, Blocks(blocks, nb), nb);
}

absl::StatusOr<LiquidBoundaryWorkspace3D> Workspace() {
  LiquidStateCapacities3D caps{};
  caps.particles = kParticles;
  caps.blocks = kFaces / 192;
  caps.cells = kCells;
  caps.faces = kFaces;
  return LiquidBoundaryWorkspace3D::Create(caps);
}

template <typename T>
std::span<const T> Span(const void* data, uint64_t count) {
  return std::span<const T>(static_cast<const T*>(data), count);
}

LiquidBoundaryVelocityHistory3D History(double time, const double* velocities, const uint8_t* validity,
                                        const void* tags, const void* walls, uint64_t faces) {
  return LiquidBoundaryVelocityHistory3D{
      .velocity_sample_time = time,
      .wall_sample_time = time,
      .face_velocities = std::span<const double>(velocities, faces),
      .validity = Span<LiquidFaceValidity3D>(validity, faces),
      .face_tags = Span<LiquidBoundaryFaceTag3D>(tags, faces),
      .wall_samples = Span<LiquidPrescribedWallSample3D>(walls, faces),
  };
}

}  // namespace

extern "C" {

// .deposit: quanta (3 x int64 per slot) and 81 compatible samples per particle.
int bk_deposit(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
               const void* particles, uint64_t n, const void* tags, double mass_q, double momentum_q,
               uint64_t declared_capacity, void* quanta_out, void* stencils_out) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  const std::size_t faces = grid->face_count();
  const LiquidBoundaryDepositViewInputs3D inputs{grid->view(), Span<LiquidBoundaryParticle3D>(particles, n),
                                                 Span<LiquidBoundaryFaceTag3D>(tags, faces),
                                                 MacDepositQuantization3D{mass_q, momentum_q, declared_capacity}};
  auto r = TimedOp([&] { return table->deposit(table->context, inputs, *ws); });
  if (!r.ok()) return Code(r.status());
  std::memcpy(quanta_out, r->face_quanta.data(), r->face_quanta.size_bytes());
  std::memcpy(stencils_out, r->compatible_stencils.data(), r->compatible_stencils.size_bytes());
  return 0;
}

// .normalize: masses, velocities and validity per slot.
int bk_normalize(int which, const void* quanta, uint64_t count, double mass_q, double momentum_q,
                 uint64_t declared_capacity, double minimum_face_mass, double* masses, double* velocities,
                 uint8_t* validity) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  auto r = TimedOp([&] {
    return table->normalize(table->context, Span<MacFaceDepositQuanta3D>(quanta, count),
                            MacDepositQuantization3D{mass_q, momentum_q, declared_capacity}, minimum_face_mass, *ws);
  });
  if (!r.ok()) return Code(r.status());
  std::memcpy(masses, r->face_masses.data(), r->face_masses.size_bytes());
  std::memcpy(velocities, r->face_velocities.data(), r->face_velocities.size_bytes());
  std::memcpy(validity, r->validity.data(), r->validity.size_bytes());
  return 0;
}

// .forces: predicted velocity per slot.
int bk_forces(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
              const double* old_velocities, const double acceleration[3], double dt, double* predicted) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  const std::size_t faces = grid->face_count();
  std::vector<double> out(faces, 0.0);
  const auto s = TimedOp([&] { return table->forces(table->context, grid->view(), std::span<const double>(old_velocities, faces),
                               Vec3{acceleration[0], acceleration[1], acceleration[2]}, dt, out); });
  if (!s.ok()) return Code(s);
  std::memcpy(predicted, out.data(), sizeof(double) * faces);
  return 0;
}

// .predict_missing_face on the old history at `time`.
int bk_predict(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb, double time,
               const double* velocities, const uint8_t* validity, const void* tags, const void* walls,
               uint64_t slot, int64_t side, const double acceleration[3], double dt, double* predicted) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  const LiquidMissingFacePredictionInputs3D inputs{
      grid->view(), History(time, velocities, validity, tags, walls, grid->face_count()), slot, side,
      Vec3{acceleration[0], acceleration[1], acceleration[2]}, dt};
  auto r = TimedOp([&] { return table->predict_missing_face(table->context, inputs, *ws); });
  if (!r.ok()) return Code(r.status());
  *predicted = *r;
  return 0;
}

// .gather: one record per particle; counts = old PIC, new PIC, low-mass fallbacks.
int bk_gather(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
              const void* particles, uint64_t n, double old_time, double new_time, const double* old_velocities,
              const uint8_t* old_validity, const void* old_tags, const void* old_walls,
              const double* new_velocities, const uint8_t* new_validity, const void* new_tags,
              const void* new_walls, void* gathered, uint64_t counts[3]) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  const std::size_t faces = grid->face_count();
  const LiquidBoundaryGatherViewInputs3D inputs{
      grid->view(), Span<LiquidBoundaryParticle3D>(particles, n), old_time, new_time,
      History(old_time, old_velocities, old_validity, old_tags, old_walls, faces),
      History(new_time, new_velocities, new_validity, new_tags, new_walls, faces)};
  auto r = TimedOp([&] { return table->gather(table->context, inputs, *ws); });
  if (!r.ok()) return Code(r.status());
  std::memcpy(gathered, r->particles.data(), r->particles.size_bytes());
  counts[0] = r->old_pic_fallback_particle_count;
  counts[1] = r->new_pic_fallback_particle_count;
  counts[2] = r->low_mass_fallback_particle_count;
  return 0;
}

// .project on cells (x,y,z; volume, target divergence, bulk modulus (0 = +inf),
// previous pressure, inward wall flux) and faces in owned-slot order (axis,x,y,z;
// kind 0 sealed / 1 internal / 2 Dirichlet; area, inverse density, distance,
// predicted velocity, wall velocity, jump or exterior pressure; explicit wall
// flux, NaN when absent). diag: iterations, true residual, max |r|/V, max
// defect, gauge count; measure: RHS norm, cell volume, inward explicit flux.
int bk_project(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb, double dt,
               const int32_t* cell_index, const double* cell_values, uint64_t nc, const int32_t* face_index,
               const int32_t* face_kind, const double* face_values, const double* face_flux, uint64_t nf,
               uint64_t max_iterations, double tolerance_scale, double* pressure, double* corrected_u,
               double* rhs, double* residual, double* defect, double diag[5], double measure[3]) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = MacPressureWorkspace3D::Create(kCells, kFaces);
  if (!ws.ok()) return Code(ws.status());
  std::vector<MacPressureCell3D> cells(nc);
  for (uint64_t i = 0; i < nc; ++i) {
    const double* v = cell_values + 5 * i;
    cells[i].cell_index = {cell_index[3 * i], cell_index[3 * i + 1], cell_index[3 * i + 2]};
    cells[i].fluid_volume = v[0];
    cells[i].target_divergence = v[1];
    cells[i].bulk_modulus = v[2] == 0.0 ? HUGE_VAL : v[2];
    cells[i].previous_pressure = v[3];
    cells[i].integrated_inward_wall_flux = v[4];
  }
  std::vector<MacPressureFace3D> faces(nf);
  for (uint64_t f = 0; f < nf; ++f) {
    const double* v = face_values + 6 * f;
    MacPressureFace3D face{};
    face.face_index = {static_cast<FaceNormalAxis>(face_index[4 * f]),
                       {face_index[4 * f + 1], face_index[4 * f + 2], face_index[4 * f + 3]}};
    face.open_area = v[0];
    face.inverse_density = v[1];
    face.pressure_gradient_distance = v[2];
    face.predicted_normal_velocity = v[3];
    face.wall_normal_velocity = v[4];
    if (face_kind[f] == 1) {
      face.pressure_link = InternalMacPressureLink3D{v[5]};
    } else if (face_kind[f] == 2) {
      face.pressure_link = DirichletMacPressureLink3D{v[5]};
    } else {
      face.pressure_link = SealedMacPressureLink3D{};
    }
    if (face_flux && face_flux[f] == face_flux[f]) face.prescribed_wall_flux = face_flux[f];
    faces[f] = face;
  }
  const LiquidPressureProblemView3D problem{cells, faces};
  auto r = TimedOp([&] {
    return table->project(table->context, grid->view(), dt, problem,
                          MacPressureSolverOptions3D{max_iterations, tolerance_scale}, *ws);
  });
  if (!r.ok()) return Code(r.status());
  std::memcpy(pressure, r->cell_pressures.data(), r->cell_pressures.size_bytes());
  std::memcpy(corrected_u, r->corrected_face_velocities.data(), r->corrected_face_velocities.size_bytes());
  std::memcpy(rhs, r->integrated_rhs.data(), r->integrated_rhs.size_bytes());
  std::memcpy(residual, r->true_residuals.data(), r->true_residuals.size_bytes());
  std::memcpy(defect, r->cell_constraint_defects.data(), r->cell_constraint_defects.size_bytes());
  diag[0] = static_cast<double>(r->diagnostics.iteration_count);
  diag[1] = r->diagnostics.true_residual_l2;
  diag[2] = r->diagnostics.max_volume_scaled_residual;
  diag[3] = r->diagnostics.max_cell_constraint_defect;
  diag[4] = static_cast<double>(r->gauge_cell_ordinals.size());
  measure[0] = r->frozen_measurement.integrated_rhs_l2_m3_per_s;
  measure[1] = r->frozen_measurement.pressure_cell_volume_m3;
  measure[2] = r->frozen_measurement.inward_prescribed_wall_flux_m3_per_s;
  return 0;
}

// .links on a frozen view given as plain arrays: centre samples (x,y,z; d),
// frozen cells (x,y,z; volume, centre distance, curvature), frozen faces
// (axis,x,y,z; slot; open area, blocked area, wall velocity, explicit flux or
// NaN; piston flag), pressure fields per cell (target divergence, bulk
// modulus, previous pressure, density or NaN), predicted velocities, wetted
// piston fluxes (NULL, or per face with NaN for none), air pressures (x,y,z;
// p) and interfaces (ordinal; tail fraction, sigma, curvature, viscous jump).
// Outputs: cells (5 doubles each), faces (kind 0/1/2, value, inverse
// density, distance, predicted, wall velocity, open area, flux or NaN: 8
// doubles each) and the lower-theta count.
int bk_links(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
             const int32_t* center_index, const double* center_distance, uint64_t ncenters,
             const int32_t* cell_index, const double* cell_values, uint64_t nc, const int32_t* face_index,
             const uint64_t* face_slot, const double* face_values, const uint8_t* piston, uint64_t nf,
             double step_duration, double density, double sigma, const double* field_values,
             const double* predicted, double ambient, const double* wetted, const int32_t* air_index,
             const double* air_pressure, uint64_t nair, const uint64_t* itf_ordinal, const double* itf_values,
             uint64_t nitf, double* cells_out, double* faces_out, uint64_t* lower) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  std::vector<LiquidCenterDistance3D> centers(ncenters);
  for (uint64_t i = 0; i < ncenters; ++i)
    centers[i] = {{center_index[3 * i], center_index[3 * i + 1], center_index[3 * i + 2]}, center_distance[i]};
  std::vector<FrozenLiquidCell3D> cells(nc);
  for (uint64_t i = 0; i < nc; ++i)
    cells[i] = {{cell_index[3 * i], cell_index[3 * i + 1], cell_index[3 * i + 2]}, cell_values[3 * i],
                cell_values[3 * i + 1], cell_values[3 * i + 2]};
  std::vector<FrozenLiquidFace3D> faces(nf);
  for (uint64_t f = 0; f < nf; ++f) {
    FrozenLiquidFace3D face{};
    face.face_index = {static_cast<FaceNormalAxis>(face_index[4 * f]),
                       {face_index[4 * f + 1], face_index[4 * f + 2], face_index[4 * f + 3]}};
    face.face_slot = face_slot[f];
    face.open_area = face_values[4 * f];
    face.blocked_area = face_values[4 * f + 1];
    face.wall_normal_velocity = face_values[4 * f + 2];
    if (face_values[4 * f + 3] == face_values[4 * f + 3]) face.prescribed_wall_flux = face_values[4 * f + 3];
    face.is_low_x_piston_face = piston[f] != 0;
    faces[f] = face;
  }
  const FrozenLiquidBoundaryGeometryView3D geometry{grid->view(), centers, cells, faces, step_duration, density,
                                                    sigma, 0.0};
  std::vector<LiquidPressureCellFields3D> fields(nc);
  for (uint64_t i = 0; i < nc; ++i) {
    const double* v = field_values + 4 * i;
    fields[i] = {v[0], v[1], v[2], v[3] == v[3] ? std::optional<double>(v[3]) : std::nullopt};
  }
  std::vector<std::optional<double>> wet;
  if (wetted) {
    wet.resize(nf);
    for (uint64_t f = 0; f < nf; ++f)
      if (wetted[f] == wetted[f]) wet[f] = wetted[f];
  }
  std::vector<LiquidAirCellPressure3D> air(nair);
  for (uint64_t k = 0; k < nair; ++k)
    air[k] = {{air_index[3 * k], air_index[3 * k + 1], air_index[3 * k + 2]}, air_pressure[k]};
  std::vector<LiquidInternalInterface3D> itf(nitf);
  for (uint64_t k = 0; k < nitf; ++k) {
    const double* v = itf_values + 4 * k;
    itf[k] = {itf_ordinal[k], v[0], v[1], v[2], v[3]};
  }
  LiquidPressureFields3D pf{};
  pf.cells = fields;
  pf.predicted_face_velocities = std::span<const double>(predicted, nf);
  pf.ambient_pressure = ambient;
  pf.wetted_piston_face_fluxes = wet;
  pf.air_cell_pressures = air;
  pf.internal_interfaces = itf;
  auto r = TimedOp([&] { return table->links(table->context, geometry, pf, *ws); });
  if (!r.ok()) return Code(r.status());
  for (uint64_t i = 0; i < nc; ++i) {
    const auto& c = r->cells[i];
    double* o = cells_out + 5 * i;
    o[0] = c.fluid_volume;
    o[1] = c.target_divergence;
    o[2] = c.bulk_modulus;
    o[3] = c.previous_pressure;
    o[4] = c.integrated_inward_wall_flux;
  }
  for (uint64_t f = 0; f < nf; ++f) {
    const auto& l = r->faces[f];
    double* o = faces_out + 8 * f;
    o[0] = static_cast<double>(l.pressure_link.index() == 0 ? 1 : (l.pressure_link.index() == 1 ? 2 : 0));
    o[1] = l.pressure_link.index() == 0   ? std::get<InternalMacPressureLink3D>(l.pressure_link).pressure_jump
           : l.pressure_link.index() == 1 ? std::get<DirichletMacPressureLink3D>(l.pressure_link).exterior_pressure
                                          : 0.0;
    o[2] = l.inverse_density;
    o[3] = l.pressure_gradient_distance;
    o[4] = l.predicted_normal_velocity;
    o[5] = l.wall_normal_velocity;
    o[6] = l.open_area;
    o[7] = l.prescribed_wall_flux.value_or(std::nan(""));
  }
  *lower = r->lower_theta_regularization_count;
  return 0;
}

// .freeze on candidate cells with centre and corner samples (x,y,z; d),
// obstacle kind 0 none / 1 halfspace / 2 slab (normal, coordinate, half
// width, wall velocity) / 3 open tank (low x, high x, floor y, low z, high z,
// piston velocity) and the exact curvature (NaN for none). Face outputs add
// the prescribed wall flux (NaN for none) and the piston flag. Outputs: cells
// (x,y,z) + (volume, centre distance, curvature), faces (axis,x,y,z) + slot +
// (open, blocked, wall velocity), the counts and the capillary bound.
int bk_freeze(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
              const int32_t* cell_index, uint64_t n, const int32_t* center_index, const double* center_distance,
              uint64_t ncenters, const int32_t* corner_index, const double* corner_distance, uint64_t ncorners,
              int obstacle_kind, const double normal[3], double coordinate, double half_width,
              const double velocity[3], const double tank[6], double step_duration, double density, double sigma,
              double exact_curvature,
              int32_t* cells_index_out, double* cells_out, uint64_t* ncells_out, int32_t* faces_index_out,
              uint64_t* faces_slot_out, double* faces_out, uint64_t* nfaces_out, double* capillary_bound) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  auto ws = Workspace();
  if (!ws.ok()) return Code(ws.status());
  std::vector<CellIndex3D> cells(n);
  for (uint64_t i = 0; i < n; ++i) cells[i] = {cell_index[3 * i], cell_index[3 * i + 1], cell_index[3 * i + 2]};
  std::vector<LiquidCenterDistance3D> centers(ncenters);
  for (uint64_t i = 0; i < ncenters; ++i)
    centers[i] = {{center_index[3 * i], center_index[3 * i + 1], center_index[3 * i + 2]}, center_distance[i]};
  std::vector<LiquidCornerDistance3D> corners(ncorners);
  for (uint64_t i = 0; i < ncorners; ++i)
    corners[i] = {{corner_index[3 * i], corner_index[3 * i + 1], corner_index[3 * i + 2]}, corner_distance[i]};
  LiquidObstacle3D obstacle{};
  const Vec3 nrm{normal[0], normal[1], normal[2]}, vel{velocity[0], velocity[1], velocity[2]};
  if (obstacle_kind == 1) obstacle = TranslatingHalfspace3D{nrm, coordinate, vel};
  if (obstacle_kind == 2) obstacle = TranslatingSlab3D{nrm, coordinate, half_width, vel};
  if (obstacle_kind == 3) obstacle = AxisAlignedLiquidTank3D{tank[0], tank[1], tank[2], tank[3], tank[4], tank[5]};
  LiquidBoundaryGeometryViewInputs3D in{grid->view(), cells, centers, corners, obstacle, step_duration, density,
                                        sigma};
  if (exact_curvature == exact_curvature) in.exact_outward_interface_curvature = exact_curvature;
  auto r = TimedOp([&] { return table->freeze(table->context, in, *ws); });
  if (!r.ok()) return Code(r.status());
  *ncells_out = r->cells.size();
  for (std::size_t i = 0; i < r->cells.size(); ++i) {
    const auto& c = r->cells[i];
    cells_index_out[3 * i] = c.cell_index.x;
    cells_index_out[3 * i + 1] = c.cell_index.y;
    cells_index_out[3 * i + 2] = c.cell_index.z;
    cells_out[3 * i] = c.fluid_volume;
    cells_out[3 * i + 1] = c.center_distance;
    cells_out[3 * i + 2] = c.curvature;
  }
  *nfaces_out = r->faces.size();
  for (std::size_t f = 0; f < r->faces.size(); ++f) {
    const auto& face = r->faces[f];
    faces_index_out[4 * f] = static_cast<int32_t>(face.face_index.axis);
    faces_index_out[4 * f + 1] = face.face_index.lattice_index.x;
    faces_index_out[4 * f + 2] = face.face_index.lattice_index.y;
    faces_index_out[4 * f + 3] = face.face_index.lattice_index.z;
    faces_slot_out[f] = face.face_slot;
    faces_out[5 * f] = face.open_area;
    faces_out[5 * f + 1] = face.blocked_area;
    faces_out[5 * f + 2] = face.wall_normal_velocity;
    faces_out[5 * f + 3] = face.prescribed_wall_flux.value_or(std::nan(""));
    faces_out[5 * f + 4] = face.is_low_x_piston_face ? 1.0 : 0.0;
  }
  *capillary_bound = r->capillary_step_bound;
  return 0;
}

// .wetted_piston on a frozen view given as arrays (cells: x,y,z + volume,
// centre distance, curvature; faces: axis,x,y,z + slot + open, blocked, wall
// velocity, explicit flux or NaN, piston flag), a field (kind 0 sphere with
// centre and radius, 1 particle union with radius over the positions, 2 plane
// at a height; 3 the covariance drop) and the tank. Outputs: 9 doubles per
// patch (y, z, area lower/upper, receiver ordinal or -1, receiver area
// lower/upper, receiver flux lower/upper), face fluxes (NaN for none), the
// whole area and flux enclosures and the attached count.
int bk_wetted_piston(int which, const double origin[3], double h, const int32_t* blocks, uint64_t nb,
                     const int32_t* cell_index, const double* cell_values, uint64_t nc, const int32_t* face_index,
                     const uint64_t* face_slot, const double* face_values, uint64_t nf, int field_kind,
                     const double center[3], double radius, double plane_y, const double* positions, uint64_t np,
                     const double tank[6], double* patches_out, uint64_t* npatches, double* fluxes_out,
                     double whole[4], uint64_t* attached) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  auto grid = Grid(origin, h, blocks, nb);
  if (!grid.ok()) return Code(grid.status());
  LiquidStateCapacities3D caps{};
  caps.particles = kParticles;
  caps.blocks = kFaces / 192;
  caps.cells = kCells;
  caps.faces = kFaces;
  auto ws = WettedPistonWorkspace3D::Create(caps);
  if (!ws.ok()) return Code(ws.status());
  std::vector<FrozenLiquidCell3D> cells(nc);
  for (uint64_t i = 0; i < nc; ++i)
    cells[i] = {{cell_index[3 * i], cell_index[3 * i + 1], cell_index[3 * i + 2]}, cell_values[3 * i],
                cell_values[3 * i + 1], cell_values[3 * i + 2]};
  std::vector<FrozenLiquidFace3D> faces(nf);
  for (uint64_t f = 0; f < nf; ++f) {
    FrozenLiquidFace3D face{};
    face.face_index = {static_cast<FaceNormalAxis>(face_index[4 * f]),
                       {face_index[4 * f + 1], face_index[4 * f + 2], face_index[4 * f + 3]}};
    face.face_slot = face_slot[f];
    face.open_area = face_values[5 * f];
    face.blocked_area = face_values[5 * f + 1];
    face.wall_normal_velocity = face_values[5 * f + 2];
    if (face_values[5 * f + 3] == face_values[5 * f + 3]) face.prescribed_wall_flux = face_values[5 * f + 3];
    face.is_low_x_piston_face = face_values[5 * f + 4] != 0;
    faces[f] = face;
  }
  const std::vector<LiquidCenterDistance3D> centers;
  const FrozenLiquidBoundaryGeometryView3D frozen{grid->view(), centers, cells, faces, 1.0 / 240.0, 1000.0, 0.0, 0.0};
  std::vector<LiquidParticleState3D> particles(np);
  for (uint64_t i = 0; i < np; ++i) particles[i].world_position = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
  LiquidSceneField3D field = LiquidHorizontalPlaneSurface3D{plane_y};
  if (field_kind == 0) field = LiquidAnalyticSphere3D{{center[0], center[1], center[2]}, radius};
  if (field_kind == 1) field = LiquidParticleSphereUnion3D{radius};
  if (field_kind == 3) field = LiquidIsolatedCovarianceDrop3D{radius, 1.0};
  const AxisAlignedLiquidTank3D tk{tank[0], tank[1], tank[2], tank[3], tank[4], tank[5]};
  const WettedPistonInputs3D inputs{field, particles, frozen, tk};
  auto r = TimedOp([&] { return table->wetted_piston(table->context, inputs, *ws); });
  if (!r.ok()) return Code(r.status());
  *npatches = r->patches.size();
  for (std::size_t k = 0; k < r->patches.size(); ++k) {
    const auto& p = r->patches[k];
    double* o = patches_out + 9 * k;
    o[0] = p.lattice_y;
    o[1] = p.lattice_z;
    o[2] = p.area.lower;
    o[3] = p.area.upper;
    o[4] = p.receiver_face_ordinal ? static_cast<double>(*p.receiver_face_ordinal) : -1.0;
    o[5] = p.receiver_area.lower;
    o[6] = p.receiver_area.upper;
    o[7] = p.receiver_flux.lower;
    o[8] = p.receiver_flux.upper;
  }
  for (uint64_t f = 0; f < nf; ++f) fluxes_out[f] = r->face_fluxes[f].value_or(std::nan(""));
  whole[0] = r->whole_area.lower;
  whole[1] = r->whole_area.upper;
  whole[2] = r->whole_flux.lower;
  whole[3] = r->whole_flux.upper;
  *attached = r->attached_patch_count;
  return 0;
}

// Which operations each table fills (bit k: deposit, normalize, predict,
// forces, gather, project, topology, update_particles, links, freeze,
// wetted_piston).
int bk_filled(int which, uint32_t* mask) {
  int code = 0;
  const auto* table = Table(which, &code);
  if (!table) return code;
  const void* ops[] = {reinterpret_cast<const void*>(table->deposit),
                       reinterpret_cast<const void*>(table->normalize),
                       reinterpret_cast<const void*>(table->predict_missing_face),
                       reinterpret_cast<const void*>(table->forces),
                       reinterpret_cast<const void*>(table->gather),
                       reinterpret_cast<const void*>(table->project),
                       reinterpret_cast<const void*>(table->topology),
                       reinterpret_cast<const void*>(table->update_particles),
                       reinterpret_cast<const void*>(table->links),
                       reinterpret_cast<const void*>(table->freeze),
                       reinterpret_cast<const void*>(table->wetted_piston)};
  *mask = 0;
  for (int k = 0; k < 11; ++k)
    if (ops[k]) *mask |= 1u << k;
  return 0;
}

// Host time of the last table operation, ms.
double bk_last_op_ms() { return g_last_op_ms; }

// Drops the B200 table's backend (its device storage) before the process exits.
void bk_release() { B200().reset(); }

}  // extern "C"
