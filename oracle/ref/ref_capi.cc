// C-ABI wrapper around the reference's own CPU operators, compiled from the
// reference sources by oracle/ref/Makefile into oracle/_ref/libfluidity_ref.so.
//
// TEST INFRASTRUCTURE ONLY. This is the checker: the parity tests, smoke() and
// bench.py's cpu_baseline / --impl reference arm load it to compute the
// reference's answers and CPU timings. No product path links or calls it.
//
// Wrapped reference entry points (paths relative to the FluidiTy project):
//   SparseMacGrid3D::Create / FaceSlot / FaceIndex   native/src/sparse_mac_grid_3d.cc:344-409,587-603
//   ComputeParticleSortBin3D                        native/src/sparse_mac_grid_3d.cc:438-449
//   BuildMacFaceGeometryStencil3D                   native/src/sparse_mac_grid_3d.cc:451-548
//   DepositMac3D / DepositMacQuanta3D / GatherMac3D native/src/transfers_3d.cc:139-261
//   ProjectMacPressure3D                            native/src/mac_pressure_3d.cc:6-39
//   NormalizeLiquidMacFaces3D                       native/src/liquid_boundary_transfer_3d.cc:785-805
// Every function returns the absl status code as int (0 = OK).

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <span>
#include <vector>

#include "fluidity/host/liquid_boundary_transfer_3d.h"
#include "fluidity/host/mac_pressure_3d.h"
#include "fluidity/host/sparse_mac_grid_3d.h"
#include "fluidity/host/transfers_3d.h"

using namespace fluidity;

namespace {

UniformMacGeometry3D Geometry(const double origin[3], double h) {
  return {{origin[0], origin[1], origin[2]}, h};
}

std::vector<BlockIndex3D> Blocks(const int32_t* blocks, size_t nb) {
  std::vector<BlockIndex3D> out(nb);
  for (size_t i = 0; i < nb; ++i) out[i] = {blocks[3 * i], blocks[3 * i + 1], blocks[3 * i + 2]};
  return out;
}

// Particle AoS with 19 doubles: sorted(3) trial(3) mass(1) velocity(3) slopes rows(9).
std::vector<MacTransferParticle3D> Particles(const double* p, size_t np) {
  std::vector<MacTransferParticle3D> out(np);
  for (size_t i = 0; i < np; ++i) {
    const double* q = p + 19 * i;
    out[i].sorted_world_position = {q[0], q[1], q[2]};
    out[i].trial_world_position = {q[3], q[4], q[5]};
    out[i].particle_mass = q[6];
    out[i].particle_velocity = {q[7], q[8], q[9]};
    out[i].particle_velocity_slopes = {{q[10], q[11], q[12]}, {q[13], q[14], q[15]}, {q[16], q[17], q[18]}};
  }
  return out;
}

int Code(const absl::Status& s) { return static_cast<int>(s.code()); }

}  // namespace

extern "C" {

// Number of owned face slots (192 per 4^3 block) or a negative status.
long long ref_grid_face_count(const double origin[3], double h, const int32_t* blocks, size_t nb) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return -Code(grid.status());
  return static_cast<long long>(grid->face_count());
}

// Writes (axis, x, y, z) for every owned slot in slot order: face_count x 4 int32.
int ref_grid_face_indices(const double origin[3], double h, const int32_t* blocks, size_t nb, int32_t* out) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return Code(grid.status());
  auto view = grid->view();
  for (size_t s = 0; s < grid->face_count(); ++s) {
    auto f = view.FaceIndex(s);
    if (!f.ok()) return Code(f.status());
    out[4 * s] = static_cast<int32_t>(f->axis);
    out[4 * s + 1] = f->lattice_index.x;
    out[4 * s + 2] = f->lattice_index.y;
    out[4 * s + 3] = f->lattice_index.z;
  }
  return 0;
}

int ref_particle_sort_bin(const double origin[3], double h, const double pos[3], int32_t out[3]) {
  auto bin = ComputeParticleSortBin3D(Geometry(origin, h), {pos[0], pos[1], pos[2]});
  if (!bin.ok()) return Code(bin.status());
  out[0] = bin->x;
  out[1] = bin->y;
  out[2] = bin->z;
  return 0;
}

// 27 samples: face (axis,x,y,z) int32 x4, and doubles weight, offset(3), gradient(3).
int ref_geometry_stencil(const double origin[3], double h, int axis, const double sorted_pos[3],
                         const double trial_pos[3], int32_t* out_faces, double* out_values) {
  auto st = BuildMacFaceGeometryStencil3D(Geometry(origin, h), static_cast<FaceNormalAxis>(axis),
                                          {sorted_pos[0], sorted_pos[1], sorted_pos[2]},
                                          {trial_pos[0], trial_pos[1], trial_pos[2]});
  if (!st.ok()) return Code(st.status());
  for (size_t i = 0; i < 27; ++i) {
    const auto& s = (*st)[i];
    out_faces[4 * i] = static_cast<int32_t>(s.face_index.axis);
    out_faces[4 * i + 1] = s.face_index.lattice_index.x;
    out_faces[4 * i + 2] = s.face_index.lattice_index.y;
    out_faces[4 * i + 3] = s.face_index.lattice_index.z;
    double* v = out_values + 7 * i;
    v[0] = s.weight;
    v[1] = s.face_offset_from_particle.x;
    v[2] = s.face_offset_from_particle.y;
    v[3] = s.face_offset_from_particle.z;
    v[4] = s.weight_gradient.x;
    v[5] = s.weight_gradient.y;
    v[6] = s.weight_gradient.z;
  }
  return 0;
}

// FP64 P2G. out_mass/out_momentum have face_count entries in 4^3 slot order.
int ref_deposit_mac_3d(const double origin[3], double h, const int32_t* blocks, size_t nb, const double* particles,
                       size_t np, double* out_mass, double* out_momentum) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return Code(grid.status());
  auto parts = Particles(particles, np);
  std::vector<MacFaceDeposit3D> faces(grid->face_count());
  auto st = DepositMac3D(*grid, parts, faces);
  if (!st.ok()) return Code(st);
  for (size_t i = 0; i < faces.size(); ++i) {
    out_mass[i] = faces[i].deposited_mass;
    out_momentum[i] = faces[i].deposited_pure_momentum;
  }
  return 0;
}

// Quantized P2G (nearest-even int64 quanta per contribution).
int ref_deposit_mac_quanta_3d(const double origin[3], double h, const int32_t* blocks, size_t nb,
                              const double* particles, size_t np, double mass_per_quantum,
                              double momentum_per_quantum, size_t capacity, int64_t* out_mass_q,
                              int64_t* out_momentum_q) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return Code(grid.status());
  auto parts = Particles(particles, np);
  std::vector<MacFaceDepositQuanta3D> faces(grid->face_count());
  auto st = DepositMacQuanta3D(*grid, parts, {mass_per_quantum, momentum_per_quantum, capacity}, faces);
  if (!st.ok()) return Code(st);
  for (size_t i = 0; i < faces.size(); ++i) {
    out_mass_q[i] = faces[i].mass_quanta_sum;
    out_momentum_q[i] = faces[i].pure_momentum_quanta_sum;
  }
  return 0;
}

// NormalizeLiquidMacFaces3D on per-face quanta (stress channel zero): face
// masses, velocities and validity (LiquidFaceValidity3D as bytes).
extern "C" int ref_normalize_liquid_mac_faces_3d(const int64_t* mass_q, const int64_t* momentum_q, size_t nf,
                                                 double mass_per_quantum, double momentum_per_quantum,
                                                 size_t capacity, double minimum_face_mass, double* out_mass,
                                                 double* out_velocity, uint8_t* out_validity) {
  std::vector<MacFaceDepositQuanta3D> faces(nf);
  for (size_t i = 0; i < nf; ++i) faces[i] = {mass_q[i], momentum_q[i], 0};
  auto r = NormalizeLiquidMacFaces3D(faces, {mass_per_quantum, momentum_per_quantum, capacity}, minimum_face_mass);
  if (!r.ok()) return Code(r.status());
  for (size_t i = 0; i < nf; ++i) {
    out_mass[i] = r->face_masses[i];
    out_velocity[i] = r->face_velocities[i];
    out_validity[i] = static_cast<uint8_t>(r->validity[i]);
  }
  return 0;
}

// FP64 G2P. out has 24 doubles per particle, laid out as MacParticleGatherResult3D:
// new PIC velocity(3), grid increment(3), fitted slope rows(9), interpolant gradient rows(9).
int ref_gather_mac_3d(const double origin[3], double h, const int32_t* blocks, size_t nb, const double* particles,
                      size_t np, const double* old_u, const double* new_u, double* out) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return Code(grid.status());
  auto parts = Particles(particles, np);
  const size_t fc = grid->face_count();
  std::vector<MacParticleGatherResult3D> res(np);
  auto st = GatherMac3D(*grid, parts, std::span<const double>(old_u, fc), std::span<const double>(new_u, fc), res);
  if (!st.ok()) return Code(st);
  for (size_t i = 0; i < np; ++i) {
    const auto& r = res[i];
    double* o = out + 24 * i;
    const double vals[24] = {r.new_pic_velocity.x,
                             r.new_pic_velocity.y,
                             r.new_pic_velocity.z,
                             r.grid_velocity_increment.x,
                             r.grid_velocity_increment.y,
                             r.grid_velocity_increment.z,
                             r.fitted_velocity_slopes.x_row.x,
                             r.fitted_velocity_slopes.x_row.y,
                             r.fitted_velocity_slopes.x_row.z,
                             r.fitted_velocity_slopes.y_row.x,
                             r.fitted_velocity_slopes.y_row.y,
                             r.fitted_velocity_slopes.y_row.z,
                             r.fitted_velocity_slopes.z_row.x,
                             r.fitted_velocity_slopes.z_row.y,
                             r.fitted_velocity_slopes.z_row.z,
                             r.velocity_gradient.x_row.x,
                             r.velocity_gradient.x_row.y,
                             r.velocity_gradient.x_row.z,
                             r.velocity_gradient.y_row.x,
                             r.velocity_gradient.y_row.y,
                             r.velocity_gradient.y_row.z,
                             r.velocity_gradient.z_row.x,
                             r.velocity_gradient.z_row.y,
                             r.velocity_gradient.z_row.z};
    std::memcpy(o, vals, sizeof(vals));
  }
  return 0;
}

// Pressure projection. Cells: int32 (x,y,z) x nc, doubles per cell
//   {fluid_volume, target_divergence, bulk_modulus (0 = +inf), previous_pressure, inward_wall_flux}.
// Faces: int32 (axis,x,y,z) x nf, int32 kind (0 sealed, 1 internal, 2 Dirichlet) and doubles per face
//   {open_area, inverse_density, distance, predicted_u, wall_u, lift}. Faces may come in any order;
//   they are reordered to owned-slot order here and results are returned in the caller's order.
// Outputs: pressure[nc], residual[nc], defect[nc], rhs[nc], corrected_u[nf], diag[5] =
//   {iterations, levels, true_residual_l2, max_volume_scaled_residual, max_defect}.
int ref_project_mac_pressure_3d(const double origin[3], double h, const int32_t* blocks, size_t nb, double dt,
                                const int32_t* cell_index, const double* cell_values, size_t nc,
                                const int32_t* face_index, const int32_t* face_kind, const double* face_values,
                                size_t nf, size_t max_iterations, double tolerance_scale, double* out_pressure,
                                double* out_residual, double* out_defect, double* out_rhs, double* out_corrected_u,
                                double* out_diag) {
  auto grid = SparseMacGrid3D::Create(Geometry(origin, h), Blocks(blocks, nb), nb);
  if (!grid.ok()) return Code(grid.status());
  std::vector<MacPressureCell3D> cells(nc);
  for (size_t i = 0; i < nc; ++i) {
    const double* v = cell_values + 5 * i;
    cells[i].cell_index = {cell_index[3 * i], cell_index[3 * i + 1], cell_index[3 * i + 2]};
    cells[i].fluid_volume = v[0];
    cells[i].target_divergence = v[1];
    cells[i].bulk_modulus = v[2] == 0.0 ? std::numeric_limits<double>::infinity() : v[2];
    cells[i].previous_pressure = v[3];
    cells[i].integrated_inward_wall_flux = v[4];
  }
  std::vector<size_t> slots(nf);
  for (size_t f = 0; f < nf; ++f) {
    FaceIndex3D fi{static_cast<FaceNormalAxis>(face_index[4 * f]),
                   {face_index[4 * f + 1], face_index[4 * f + 2], face_index[4 * f + 3]}};
    auto s = grid->FaceSlot(fi);
    if (!s.ok()) return Code(s.status());
    slots[f] = *s;
  }
  std::vector<size_t> order(nf);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return slots[a] < slots[b]; });
  std::vector<MacPressureFace3D> faces(nf);
  for (size_t k = 0; k < nf; ++k) {
    const size_t f = order[k];
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
    faces[k] = face;
  }
  MacPressureInputs3D inputs{*grid, dt, cells, faces};
  MacPressureSolverOptions3D options{max_iterations, tolerance_scale};
  auto proj = ProjectMacPressure3D(inputs, options);
  if (!proj.ok()) return Code(proj.status());
  for (size_t i = 0; i < nc; ++i) {
    out_pressure[i] = proj->cell_pressures[i];
    out_residual[i] = proj->true_residuals[i];
    out_defect[i] = proj->cell_constraint_defects[i];
    out_rhs[i] = proj->integrated_rhs[i];
  }
  for (size_t k = 0; k < nf; ++k) out_corrected_u[order[k]] = proj->corrected_face_velocities[k];
  out_diag[0] = static_cast<double>(proj->diagnostics.iteration_count);
  out_diag[1] = static_cast<double>(proj->diagnostics.multigrid_level_count);
  out_diag[2] = proj->diagnostics.true_residual_l2;
  out_diag[3] = proj->diagnostics.max_volume_scaled_residual;
  out_diag[4] = proj->diagnostics.max_cell_constraint_defect;
  return 0;
}

}  // extern "C"
