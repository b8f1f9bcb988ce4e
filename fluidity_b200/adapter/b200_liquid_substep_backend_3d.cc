// B200 operations for FluidiTy's liquid scheduler backend table; see the header.
//
// The scheduler's spans pass to the C-ABI unchanged: the C records are
// byte-compatible with the reference's (checked below), so each operation
// converts only the grid view and the histories' span headers, then copies the
// C-ABI's outputs into its own result bank. Argument checks the C-ABI cannot
// see (span extents) come first, in the CPU operations' order
// (liquid_boundary_transfer_3d.cc:46-73, 327-340, 463-484, 519-545).
#include "b200_liquid_substep_backend_3d.h"

#include <cmath>
#include <cstddef>
#include <cstring>
#include <new>
#include <type_traits>
#include <variant>

#include "fluidity/host/liquid_boundary_workspace_3d.h"
#include "fluidity/host/mac_pressure_workspace_3d.h"

namespace fluidity {
namespace {

constexpr std::size_t kParticles = 1024;  // liquid_boundary_transfer_3d.h:16
constexpr std::size_t kFaces = 24576;     // liquid_boundary_transfer_3d.h:17
constexpr std::size_t kPressureCells = 4096;

static_assert(sizeof(BlockIndex3D) == 3 * sizeof(std::int32_t));
static_assert(sizeof(LiquidBoundaryParticle3D) == sizeof(fl_boundary_particle));
static_assert(offsetof(LiquidBoundaryParticle3D, transfer) == 0);
static_assert(offsetof(MacTransferParticle3D, trial_world_position) == offsetof(fl_boundary_particle, trial_position));
static_assert(offsetof(MacTransferParticle3D, particle_mass) == offsetof(fl_boundary_particle, mass));
static_assert(offsetof(MacTransferParticle3D, particle_velocity) == offsetof(fl_boundary_particle, velocity));
static_assert(offsetof(MacTransferParticle3D, particle_velocity_slopes) == offsetof(fl_boundary_particle, slopes));
static_assert(offsetof(LiquidBoundaryParticle3D, side_tag) == offsetof(fl_boundary_particle, side_tag));
static_assert(offsetof(LiquidBoundaryParticle3D, affine_enabled) == offsetof(fl_boundary_particle, affine_enabled));
static_assert(sizeof(LiquidBoundaryFaceTag3D) == sizeof(fl_face_tag));
static_assert(offsetof(LiquidBoundaryFaceTag3D, structurally_eligible) == offsetof(fl_face_tag, structurally_eligible));
static_assert(sizeof(MacFaceDepositQuanta3D) == sizeof(fl_face_quanta));
static_assert(sizeof(CompatibleMacFaceSample3D) == sizeof(fl_compatible_sample));
static_assert(offsetof(CompatibleMacFaceSample3D, compatible) == offsetof(fl_compatible_sample, compatible));
static_assert(offsetof(CompatibleMacFaceSample3D, normalized_weight) ==
              offsetof(fl_compatible_sample, normalized_weight));
static_assert(offsetof(CompatibleMacFaceSample3D, normalized_weight_gradient) ==
              offsetof(fl_compatible_sample, normalized_weight_gradient));
static_assert(offsetof(CompatibleMacFaceSample3D, centered_face_offset) ==
              offsetof(fl_compatible_sample, centered_face_offset));
static_assert(sizeof(LiquidCompatibleStencils3D) == 81 * sizeof(fl_compatible_sample));
static_assert(sizeof(LiquidPrescribedWallSample3D) == sizeof(fl_wall_sample));
static_assert(offsetof(LiquidPrescribedWallSample3D, side_tag) == offsetof(fl_wall_sample, side_tag));
static_assert(offsetof(LiquidPrescribedWallSample3D, unit_normal) == offsetof(fl_wall_sample, unit_normal));
static_assert(offsetof(LiquidPrescribedWallSample3D, wall_velocity) == offsetof(fl_wall_sample, wall_velocity));
static_assert(sizeof(LiquidBoundaryParticleGather3D) == sizeof(fl_gathered_particle));
static_assert(offsetof(LiquidBoundaryParticleGather3D, fitted_velocity_slopes) ==
              offsetof(fl_gathered_particle, fitted_velocity_slopes));
static_assert(offsetof(LiquidBoundaryParticleGather3D, velocity_gradient) ==
              offsetof(fl_gathered_particle, velocity_gradient));
static_assert(offsetof(LiquidBoundaryParticleGather3D, affine_enabled) ==
              offsetof(fl_gathered_particle, affine_enabled));
static_assert(offsetof(LiquidBoundaryParticleGather3D, low_mass_fallback) ==
              offsetof(fl_gathered_particle, low_mass_fallback));
static_assert(sizeof(LiquidFaceValidity3D) == 1);
static_assert(sizeof(LiquidCenterDistance3D) == sizeof(fl_center_sample));
static_assert(offsetof(LiquidCenterDistance3D, signed_distance) == offsetof(fl_center_sample, signed_distance));
static_assert(sizeof(FrozenLiquidCell3D) == sizeof(fl_frozen_cell));
static_assert(sizeof(CellIndex3D) == 3 * sizeof(std::int32_t));
static_assert(sizeof(LiquidCornerDistance3D) == sizeof(fl_corner_sample));
static_assert(offsetof(LiquidCornerDistance3D, signed_distance) == offsetof(fl_corner_sample, signed_distance));
static_assert(offsetof(FrozenLiquidCell3D, curvature) == offsetof(fl_frozen_cell, curvature));
static_assert(sizeof(LiquidAirCellPressure3D) == sizeof(fl_air_cell_pressure));
static_assert(offsetof(LiquidAirCellPressure3D, gas_gauge_pressure) ==
              offsetof(fl_air_cell_pressure, gas_gauge_pressure));
static_assert(sizeof(LiquidInternalInterface3D) == sizeof(fl_internal_interface));
static_assert(offsetof(LiquidInternalInterface3D, normal_viscous_jump_tail_to_head) ==
              offsetof(fl_internal_interface, normal_viscous_jump_tail_to_head));

absl::Status Code(absl::StatusCode code) { return absl::Status(code, ""); }

absl::Status FromFl(int code) {
  return code == FL_OK ? absl::OkStatus() : Code(static_cast<absl::StatusCode>(code));
}

fl_owned_grid OwnedGrid(SparseMacGridView3D grid) {
  const UniformMacGeometry3D geometry = grid.geometry();
  const auto blocks = grid.active_block_indices();
  return fl_owned_grid{{geometry.world_origin.x, geometry.world_origin.y, geometry.world_origin.z},
                       geometry.cell_width,
                       reinterpret_cast<const std::int32_t*>(blocks.data()),
                       blocks.size()};
}

bool PowerOfTwoScale(double scale) {
  int exponent = 0;
  return std::isnormal(scale) && scale > 0.0 && std::frexp(scale, &exponent) == 0.5;
}

// ValidateQuantization (liquid_boundary_transfer_3d.cc:56-73).
absl::Status CheckQuantization(MacDepositQuantization3D q, std::size_t particles) {
  if (!PowerOfTwoScale(q.mass_per_quantum) || !PowerOfTwoScale(q.pure_momentum_per_quantum)) {
    return Code(absl::StatusCode::kInvalidArgument);
  }
  if (q.declared_particle_capacity > kParticles || particles > q.declared_particle_capacity) {
    return Code(absl::StatusCode::kResourceExhausted);
  }
  return absl::OkStatus();
}

fl_quantization Quantization(MacDepositQuantization3D q) {
  return fl_quantization{q.mass_per_quantum, q.pure_momentum_per_quantum, q.declared_particle_capacity};
}

bool HistoryCovers(const LiquidBoundaryVelocityHistory3D& h, std::size_t faces) {
  return h.face_velocities.size() == faces && h.validity.size() == faces && h.face_tags.size() == faces &&
         h.wall_samples.size() == faces;
}

fl_velocity_history History(const LiquidBoundaryVelocityHistory3D& h) {
  return fl_velocity_history{h.velocity_sample_time,
                             h.wall_sample_time,
                             h.face_velocities.data(),
                             reinterpret_cast<const std::uint8_t*>(h.validity.data()),
                             reinterpret_cast<const fl_face_tag*>(h.face_tags.data()),
                             reinterpret_cast<const fl_wall_sample*>(h.wall_samples.data())};
}

double Component(Vec3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

template <typename T>
bool Reserve(std::vector<T>& v, std::size_t n) {
  try {
    v.reserve(n);
  } catch (const std::bad_alloc&) {
    return false;
  }
  return true;
}

}  // namespace

struct B200BackendOps3D {
  static B200LiquidBackend3D& Self(void* context) { return *static_cast<B200LiquidBackend3D*>(context); }

  static absl::StatusOr<LiquidBoundaryFaceDepositsView3D> Deposit(
      void* context,
      const LiquidBoundaryDepositViewInputs3D& inputs,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t faces = inputs.mac_grid.face_count();
    const std::size_t count = inputs.particles.size();
    if (faces > kFaces || count > kParticles) return Code(absl::StatusCode::kResourceExhausted);
    if (const auto status = CheckQuantization(inputs.quantization, count); !status.ok()) return status;
    if (inputs.face_tags.size() != faces) return Code(absl::StatusCode::kInvalidArgument);
    auto& bank = self.deposits_[1 - self.deposit_bank_];
    bank.quanta.resize(faces);
    bank.stencils.resize(count);
    const fl_owned_grid grid = OwnedGrid(inputs.mac_grid);
    const fl_quantization q = Quantization(inputs.quantization);
    const int code = fl_boundary_deposit(
        self.boundary_, &grid, reinterpret_cast<const fl_boundary_particle*>(inputs.particles.data()), count,
        reinterpret_cast<const fl_face_tag*>(inputs.face_tags.data()), &q,
        reinterpret_cast<fl_face_quanta*>(bank.quanta.data()),
        reinterpret_cast<fl_compatible_sample*>(bank.stencils.data()), nullptr
    );
    if (code != FL_OK) return FromFl(code);
    self.deposit_bank_ = 1 - self.deposit_bank_;
    return LiquidBoundaryFaceDepositsView3D{bank.quanta, bank.stencils};
  }

  static absl::StatusOr<NormalizedLiquidMacFacesView3D> Normalize(
      void* context,
      std::span<const MacFaceDepositQuanta3D> quanta,
      MacDepositQuantization3D quantization,
      double minimum_face_mass,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    if (quanta.size() > kFaces) return Code(absl::StatusCode::kResourceExhausted);
    if (const auto status = CheckQuantization(quantization, 0); !status.ok()) return status;
    auto& bank = self.normalized_[1 - self.normalize_bank_];
    bank.masses.resize(quanta.size());
    bank.velocities.resize(quanta.size());
    bank.validity.resize(quanta.size());
    const fl_quantization q = Quantization(quantization);
    const int code = fl_boundary_normalize(
        self.boundary_, reinterpret_cast<const fl_face_quanta*>(quanta.data()), quanta.size(), &q, minimum_face_mass,
        bank.masses.data(), bank.velocities.data(), reinterpret_cast<std::uint8_t*>(bank.validity.data()), nullptr
    );
    if (code != FL_OK) return FromFl(code);
    self.normalize_bank_ = 1 - self.normalize_bank_;
    return NormalizedLiquidMacFacesView3D{bank.masses, bank.velocities, bank.validity};
  }

  static absl::StatusOr<double> PredictMissingFace(
      void* context,
      const LiquidMissingFacePredictionInputs3D& inputs,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t faces = inputs.grid.face_count();
    if (faces > kFaces) return Code(absl::StatusCode::kResourceExhausted);
    if (inputs.face_slot >= faces) return Code(absl::StatusCode::kOutOfRange);
    if (!HistoryCovers(inputs.old_history, faces)) return Code(absl::StatusCode::kInvalidArgument);
    const fl_owned_grid grid = OwnedGrid(inputs.grid);
    const fl_velocity_history history = History(inputs.old_history);
    const double acceleration[3] = {inputs.world_acceleration.x, inputs.world_acceleration.y,
                                    inputs.world_acceleration.z};
    double predicted = 0.0;
    const int code = fl_boundary_predict_face(self.boundary_, &grid, &history, inputs.face_slot, inputs.side_tag,
                                              acceleration, inputs.step_duration, &predicted, nullptr);
    if (code != FL_OK) return FromFl(code);
    return predicted;
  }

  static absl::Status Forces(
      void* context,
      SparseMacGridView3D grid,
      std::span<const double> old_face_velocities,
      Vec3 world_acceleration,
      double step_duration,
      std::span<double> predicted_face_velocities
  ) {
    auto& self = Self(context);
    if (old_face_velocities.size() != grid.face_count() || predicted_face_velocities.size() != grid.face_count()) {
      return Code(absl::StatusCode::kInvalidArgument);
    }
    const fl_owned_grid owned = OwnedGrid(grid);
    const double acceleration[3] = {world_acceleration.x, world_acceleration.y, world_acceleration.z};
    return FromFl(fl_boundary_forces(self.boundary_, &owned, old_face_velocities.data(), acceleration,
                                     step_duration, predicted_face_velocities.data(), nullptr));
  }

  static absl::StatusOr<LiquidBoundaryGatherView3D> Gather(
      void* context,
      const LiquidBoundaryGatherViewInputs3D& inputs,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t faces = inputs.mac_grid.face_count();
    const std::size_t count = inputs.particles.size();
    if (faces > kFaces || count > kParticles) return Code(absl::StatusCode::kResourceExhausted);
    if (!HistoryCovers(inputs.old_history, faces) || !HistoryCovers(inputs.new_history, faces)) {
      return Code(absl::StatusCode::kInvalidArgument);
    }
    auto& bank = self.gathered_[1 - self.gather_bank_];
    bank.particles.resize(count);
    const fl_owned_grid grid = OwnedGrid(inputs.mac_grid);
    const fl_velocity_history old_history = History(inputs.old_history);
    const fl_velocity_history new_history = History(inputs.new_history);
    std::uint64_t counts[3] = {0, 0, 0};
    const int code = fl_boundary_gather(
        self.boundary_, &grid, reinterpret_cast<const fl_boundary_particle*>(inputs.particles.data()), count,
        inputs.old_time, inputs.new_time, &old_history, &new_history,
        reinterpret_cast<fl_gathered_particle*>(bank.particles.data()), counts, nullptr
    );
    if (code != FL_OK) return FromFl(code);
    self.gather_bank_ = 1 - self.gather_bank_;
    return LiquidBoundaryGatherView3D{bank.particles, counts[0], counts[1], counts[2]};
  }


  // The frozen view and the fields with their optional values unpacked into
  // the C-ABI's records; cells, centre samples, air pressures and interfaces
  // pass through (byte-compatible). Results are packed into the reference's
  // pressure-cell and link records.
  // FreezeLiquidBoundaryGeometry3D (liquid_boundary_workspace_3d.cc:186 ->
  // liquid_boundary_geometry_3d.cc:2109-2143): the frozen view in this
  // backend's freeze bank; the centre samples are copied there as the
  // workspace's own freeze does.
  static absl::StatusOr<FrozenLiquidBoundaryGeometryView3D> Freeze(
      void* context,
      const LiquidBoundaryGeometryViewInputs3D& inputs,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t n = inputs.cell_indices.size();
    if (n > kPressureCells || inputs.center_distances.size() > 27 * kPressureCells)
      return Code(absl::StatusCode::kResourceExhausted);
    if (inputs.sampled_solid) return Code(absl::StatusCode::kUnimplemented);
    fl_freeze_inputs in{};
    const fl_owned_grid grid = OwnedGrid(inputs.mac_grid);
    in.grid = &grid;
    in.cell_indices = reinterpret_cast<const std::int32_t*>(inputs.cell_indices.data());
    in.cell_count = n;
    in.centers = reinterpret_cast<const fl_center_sample*>(inputs.center_distances.data());
    in.center_count = inputs.center_distances.size();
    in.corners = reinterpret_cast<const fl_corner_sample*>(inputs.corner_distances.data());
    in.corner_count = inputs.corner_distances.size();
    if (const auto* hs = std::get_if<TranslatingHalfspace3D>(&inputs.obstacle)) {
      in.obstacle = fl_obstacle{FL_OBSTACLE_HALFSPACE, 0, {hs->unit_normal.x, hs->unit_normal.y, hs->unit_normal.z},
                                hs->start_plane_coordinate, 0.0,
                                {hs->wall_velocity.x, hs->wall_velocity.y, hs->wall_velocity.z}};
    } else if (const auto* sl = std::get_if<TranslatingSlab3D>(&inputs.obstacle)) {
      in.obstacle = fl_obstacle{FL_OBSTACLE_SLAB, 0, {sl->unit_normal.x, sl->unit_normal.y, sl->unit_normal.z},
                                sl->start_center_coordinate, sl->half_width,
                                {sl->wall_velocity.x, sl->wall_velocity.y, sl->wall_velocity.z}};
    } else if (const auto* tk = std::get_if<AxisAlignedLiquidTank3D>(&inputs.obstacle)) {
      in.obstacle.kind = FL_OBSTACLE_OPEN_TANK;
      const double t[6] = {tk->start_low_x, tk->high_x, tk->floor_y, tk->low_z, tk->high_z, tk->piston_velocity_x};
      for (int k = 0; k < 6; ++k) in.obstacle.tank[k] = t[k];
    } else {
      in.obstacle.kind = FL_OBSTACLE_NONE;
    }
    in.step_duration = inputs.step_duration;
    in.liquid_density = inputs.liquid_density;
    in.surface_tension = inputs.surface_tension;
    in.has_exact_curvature = inputs.exact_outward_interface_curvature.has_value();
    in.exact_curvature = inputs.exact_outward_interface_curvature.value_or(0.0);
    auto& bank = self.frozen_[1 - self.frozen_bank_];
    bank.cells.resize(n);
    auto& fs = self.freeze_staging_.faces;
    fs.resize(6 * n);
    std::uint64_t nc = 0, nf = 0;
    double bound = 0.0;
    const int code = fl_boundary_freeze(self.boundary_, &in, reinterpret_cast<fl_frozen_cell*>(bank.cells.data()),
                                        &nc, fs.data(), &nf, &bound, nullptr);
    if (code != FL_OK) return FromFl(code);
    bank.cells.resize(nc);
    bank.faces.resize(nf);
    for (std::size_t f = 0; f < nf; ++f) {
      const fl_frozen_face& o = fs[f];
      FrozenLiquidFace3D face{};
      face.face_index = {static_cast<FaceNormalAxis>(o.axis), {o.lattice[0], o.lattice[1], o.lattice[2]}};
      face.face_slot = o.face_slot;
      face.open_area = o.open_area;
      face.blocked_area = o.blocked_area;
      face.wall_normal_velocity = o.wall_normal_velocity;
      if (o.has_prescribed_wall_flux) face.prescribed_wall_flux = o.prescribed_wall_flux;
      face.is_low_x_piston_face = o.is_low_x_piston_face != 0;
      bank.faces[f] = face;
    }
    bank.centers.assign(inputs.center_distances.begin(), inputs.center_distances.end());
    self.frozen_bank_ = 1 - self.frozen_bank_;
    return FrozenLiquidBoundaryGeometryView3D{inputs.mac_grid,
                                              bank.centers,
                                              bank.cells,
                                              bank.faces,
                                              inputs.step_duration,
                                              inputs.liquid_density,
                                              inputs.surface_tension,
                                              bound};
  }

  // ComputeWettedPiston3D (wetted_piston_3d.cc:570-575): the view borrows
  // this backend's piston bank.
  static absl::StatusOr<WettedPistonView3D> WettedPiston(
      void* context,
      const WettedPistonInputs3D& inputs,
      WettedPistonWorkspace3D&
  ) {
    auto& self = Self(context);
    const auto& frozen = inputs.frozen;
    const std::size_t nc = frozen.cells.size(), nf = frozen.faces.size(), np = inputs.particles.size();
    if (nf > kFaces || nc > kPressureCells || np > kParticles) return Code(absl::StatusCode::kResourceExhausted);
    auto& st = self.piston_staging_;
    st.faces.resize(nf);
    for (std::size_t f = 0; f < nf; ++f) {
      const FrozenLiquidFace3D& face = frozen.faces[f];
      fl_frozen_face& o = st.faces[f];
      o = fl_frozen_face{};
      o.axis = static_cast<std::int32_t>(face.face_index.axis);
      o.lattice[0] = face.face_index.lattice_index.x;
      o.lattice[1] = face.face_index.lattice_index.y;
      o.lattice[2] = face.face_index.lattice_index.z;
      o.face_slot = face.face_slot;
      o.open_area = face.open_area;
      o.blocked_area = face.blocked_area;
      o.wall_normal_velocity = face.wall_normal_velocity;
      o.has_prescribed_wall_flux = face.prescribed_wall_flux.has_value();
      o.prescribed_wall_flux = face.prescribed_wall_flux.value_or(0.0);
      o.is_low_x_piston_face = face.is_low_x_piston_face;
    }
    st.positions.resize(3 * np);
    for (std::size_t i = 0; i < np; ++i) {
      st.positions[3 * i] = inputs.particles[i].world_position.x;
      st.positions[3 * i + 1] = inputs.particles[i].world_position.y;
      st.positions[3 * i + 2] = inputs.particles[i].world_position.z;
    }
    fl_piston_field field{};
    field.kind = -1;  // the covariance drop: not a piston field
    if (const auto* sphere = std::get_if<LiquidAnalyticSphere3D>(&inputs.field)) {
      field.kind = FL_PISTON_FIELD_SPHERE;
      field.sphere_center[0] = sphere->world_center.x;
      field.sphere_center[1] = sphere->world_center.y;
      field.sphere_center[2] = sphere->world_center.z;
      field.radius = sphere->radius;
    } else if (const auto* u = std::get_if<LiquidParticleSphereUnion3D>(&inputs.field)) {
      field.kind = FL_PISTON_FIELD_PARTICLE_UNION;
      field.radius = u->radius;
    } else if (const auto* plane = std::get_if<LiquidHorizontalPlaneSurface3D>(&inputs.field)) {
      field.kind = FL_PISTON_FIELD_PLANE;
      field.plane_height_y = plane->world_surface_height_y;
    }
    const double tank[6] = {inputs.tank.start_low_x, inputs.tank.high_x, inputs.tank.floor_y,
                            inputs.tank.low_z,       inputs.tank.high_z, inputs.tank.piston_velocity_x};
    st.patches.resize(kFaces);
    st.fluxes.resize(nf);
    st.has_flux.resize(nf);
    const fl_owned_grid grid = OwnedGrid(frozen.mac_grid);
    std::uint64_t count = 0, attached = 0;
    double whole_area[2], whole_flux[2];
    fl_measurement measured{};
    const int code = fl_boundary_wetted_piston(
        self.boundary_, &grid, reinterpret_cast<const fl_frozen_cell*>(frozen.cells.data()), nc, st.faces.data(), nf,
        &field, st.positions.data(), np, tank, st.patches.data(), st.patches.size(), &count, st.fluxes.data(),
        st.has_flux.data(), whole_area, whole_flux, &attached, &measured);
    if (code != FL_OK) return FromFl(code);
    auto& bank = self.pistons_[1 - self.piston_bank_];
    bank.patches.resize(count);
    for (std::size_t k = 0; k < count; ++k) {
      const fl_piston_patch& o = st.patches[k];
      WettedPistonPatch3D p{};
      p.lattice_y = o.lattice_y;
      p.lattice_z = o.lattice_z;
      p.area = {o.area[0], o.area[1]};
      if (o.has_receiver) p.receiver_face_ordinal = static_cast<std::size_t>(o.receiver_face_ordinal);
      p.receiver_area = {o.receiver_area[0], o.receiver_area[1]};
      p.receiver_flux = {o.receiver_flux[0], o.receiver_flux[1]};
      bank.patches[k] = p;
    }
    bank.face_fluxes.resize(nf);
    for (std::size_t f = 0; f < nf; ++f)
      bank.face_fluxes[f] = st.has_flux[f] ? std::optional<double>(st.fluxes[f]) : std::nullopt;
    self.piston_bank_ = 1 - self.piston_bank_;
    WettedPistonView3D view{};
    view.patches = bank.patches;
    view.face_fluxes = bank.face_fluxes;
    view.whole_area = {whole_area[0], whole_area[1]};
    view.whole_flux = {whole_flux[0], whole_flux[1]};
    view.attached_patch_count = attached;
    view.compiled_architecture = measured.compiled_architecture;
    return view;
  }

  static absl::StatusOr<LiquidPressureProblemView3D> Links(
      void* context,
      const FrozenLiquidBoundaryGeometryView3D& geometry,
      const LiquidPressureFields3D& fields,
      LiquidBoundaryWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t nc = geometry.cells.size(), nf = geometry.faces.size();
    if (nc > kPressureCells || nf > kFaces) return Code(absl::StatusCode::kResourceExhausted);
    // field extents (LinksCore, liquid_boundary_geometry_3d.cc:1086-1094), after the view checks the C-ABI makes
    const bool extents_ok = fields.cells.size() == nc && fields.predicted_face_velocities.size() == nf &&
                            (fields.wetted_piston_face_fluxes.empty() || fields.wetted_piston_face_fluxes.size() == nf);
    auto& st = self.link_staging_;
    st.faces.resize(nf);
    for (std::size_t f = 0; f < nf; ++f) {
      const FrozenLiquidFace3D& face = geometry.faces[f];
      fl_frozen_face& o = st.faces[f];
      o = fl_frozen_face{};
      o.axis = static_cast<std::int32_t>(face.face_index.axis);
      o.lattice[0] = face.face_index.lattice_index.x;
      o.lattice[1] = face.face_index.lattice_index.y;
      o.lattice[2] = face.face_index.lattice_index.z;
      o.face_slot = face.face_slot;
      o.open_area = face.open_area;
      o.blocked_area = face.blocked_area;
      o.wall_normal_velocity = face.wall_normal_velocity;
      o.has_prescribed_wall_flux = face.prescribed_wall_flux.has_value();
      o.prescribed_wall_flux = face.prescribed_wall_flux.value_or(0.0);
      o.is_low_x_piston_face = face.is_low_x_piston_face;
    }
    const std::size_t nfields = std::min(fields.cells.size(), nc);
    st.fields.resize(nc);
    for (std::size_t i = 0; i < nfields; ++i) {
      const LiquidPressureCellFields3D& c = fields.cells[i];
      st.fields[i] = fl_pressure_cell_fields{c.target_divergence, c.bulk_modulus, c.previous_pressure,
                                             c.density.value_or(0.0), static_cast<std::uint8_t>(c.density.has_value()),
                                             {}};
    }
    const bool wetted = !fields.wetted_piston_face_fluxes.empty();
    st.wetted.resize(wetted ? nf : 0);
    st.has_wetted.resize(wetted ? nf : 0);
    for (std::size_t f = 0; wetted && f < std::min(nf, fields.wetted_piston_face_fluxes.size()); ++f) {
      st.wetted[f] = fields.wetted_piston_face_fluxes[f].value_or(0.0);
      st.has_wetted[f] = fields.wetted_piston_face_fluxes[f].has_value();
    }
    const fl_owned_grid grid = OwnedGrid(geometry.mac_grid);
    const fl_frozen_geometry g{&grid,
                               reinterpret_cast<const fl_center_sample*>(geometry.center_distances.data()),
                               geometry.center_distances.size(),
                               reinterpret_cast<const fl_frozen_cell*>(geometry.cells.data()),
                               nc,
                               st.faces.data(),
                               nf,
                               geometry.step_duration,
                               geometry.liquid_density,
                               geometry.surface_tension};
    const fl_pressure_fields pf{st.fields.data(),
                                fields.predicted_face_velocities.data(),
                                fields.ambient_pressure,
                                wetted ? st.wetted.data() : nullptr,
                                wetted ? st.has_wetted.data() : nullptr,
                                reinterpret_cast<const fl_air_cell_pressure*>(fields.air_cell_pressures.data()),
                                fields.air_cell_pressures.size(),
                                reinterpret_cast<const fl_internal_interface*>(fields.internal_interfaces.data()),
                                fields.internal_interfaces.size()};
    st.cells_out.resize(nc);
    st.faces_out.resize(nf);
    std::uint64_t lower = 0;
    int code = FL_OK;
    if (!extents_ok) {
      // the view checks still decide the code when they fail first
      fl_pressure_fields probe = pf;
      probe.ambient_pressure = std::nan("");
      code = fl_boundary_links(self.boundary_, &g, &probe, st.cells_out.data(), st.faces_out.data(), &lower, nullptr);
      return FromFl(code);
    }
    code = fl_boundary_links(self.boundary_, &g, &pf, st.cells_out.data(), st.faces_out.data(), &lower, nullptr);
    if (code != FL_OK) return FromFl(code);
    auto& bank = self.links_[1 - self.links_bank_];
    bank.cells.resize(nc);
    bank.faces.resize(nf);
    for (std::size_t i = 0; i < nc; ++i) {
      const fl_pressure_cell& c = st.cells_out[i];
      bank.cells[i] = MacPressureCell3D{{c.cell_index[0], c.cell_index[1], c.cell_index[2]},
                                        c.fluid_volume,
                                        c.target_divergence,
                                        c.bulk_modulus,
                                        c.previous_pressure,
                                        c.integrated_inward_wall_flux};
    }
    for (std::size_t f = 0; f < nf; ++f) {
      const fl_pressure_link& l = st.faces_out[f];
      MacPressureFace3D face{};
      face.face_index = {static_cast<FaceNormalAxis>(l.axis), {l.lattice[0], l.lattice[1], l.lattice[2]}};
      face.open_area = l.open_area;
      face.inverse_density = l.inverse_density;
      face.pressure_gradient_distance = l.pressure_gradient_distance;
      face.predicted_normal_velocity = l.predicted_normal_velocity;
      face.wall_normal_velocity = l.wall_normal_velocity;
      if (l.link_kind == 1) {
        face.pressure_link = InternalMacPressureLink3D{l.link_value};
      } else if (l.link_kind == 2) {
        face.pressure_link = DirichletMacPressureLink3D{l.link_value};
      } else {
        face.pressure_link = SealedMacPressureLink3D{};
      }
      if (l.has_prescribed_wall_flux) face.prescribed_wall_flux = l.prescribed_wall_flux;
      bank.faces[f] = face;
    }
    self.links_bank_ = 1 - self.links_bank_;
    LiquidPressureProblemView3D view{};
    view.cells = bank.cells;
    view.faces = bank.faces;
    view.lower_theta_regularization_count = lower;
    return view;
  }

  // The pressure problem in the C-ABI's records: bulk modulus +inf as 0 (no
  // compliance) and any other non-positive or non-finite value as NaN (an
  // invalid cell, as the reference rejects it); an explicit wall flux on the
  // face's blocked area as the equivalent wall velocity.
  static absl::StatusOr<MacPressureProjectionView3D> Project(
      void* context,
      SparseMacGridView3D grid,
      double step_duration,
      const LiquidPressureProblemView3D& problem,
      MacPressureSolverOptions3D options,
      MacPressureWorkspace3D&
  ) {
    auto& self = Self(context);
    const std::size_t nc = problem.cells.size(), nf = problem.faces.size();
    if (nc > kPressureCells || nf > kFaces) return Code(absl::StatusCode::kResourceExhausted);
    if (nc == 0) return Code(absl::StatusCode::kInvalidArgument);
    if (!std::isfinite(options.cpu_residual_tolerance_scale) || options.cpu_residual_tolerance_scale < 1e-12 ||
        options.cpu_residual_tolerance_scale > 1.0) {
      return Code(absl::StatusCode::kInvalidArgument);
    }
    const double h = grid.geometry().cell_width;
    const double full_area = h * h;
    auto& s = self.staging_;
    s.cell_index.resize(3 * nc);
    s.cell_values.resize(5 * nc);
    s.face_index.resize(4 * nf);
    s.face_kind.resize(nf);
    s.face_values.resize(6 * nf);
    double volume = 0.0, volume_error = 0.0;
    for (std::size_t i = 0; i < nc; ++i) {
      const MacPressureCell3D& c = problem.cells[i];
      s.cell_index[3 * i] = c.cell_index.x;
      s.cell_index[3 * i + 1] = c.cell_index.y;
      s.cell_index[3 * i + 2] = c.cell_index.z;
      double* v = &s.cell_values[5 * i];
      v[0] = c.fluid_volume;
      v[1] = c.target_divergence;
      v[2] = c.bulk_modulus == HUGE_VAL ? 0.0 : (c.bulk_modulus > 0.0 && std::isfinite(c.bulk_modulus) ? c.bulk_modulus
                                                                                                          : NAN);
      v[3] = c.previous_pressure;
      v[4] = c.integrated_inward_wall_flux;
      const double t = volume + c.fluid_volume;  // Neumaier-compensated total volume
      volume_error += std::abs(volume) >= std::abs(c.fluid_volume) ? (volume - t) + c.fluid_volume
                                                                    : (c.fluid_volume - t) + volume;
      volume = t;
    }
    double inward_flux = 0.0;
    for (std::size_t f = 0; f < nf; ++f) {
      const MacPressureFace3D& face = problem.faces[f];
      // The owner block must be allocated even for a sealed face.
      if (const auto slot = grid.FaceSlot(face.face_index); !slot.ok()) return slot.status();
      s.face_index[4 * f] = static_cast<std::int32_t>(face.face_index.axis);
      s.face_index[4 * f + 1] = face.face_index.lattice_index.x;
      s.face_index[4 * f + 2] = face.face_index.lattice_index.y;
      s.face_index[4 * f + 3] = face.face_index.lattice_index.z;
      double* v = &s.face_values[6 * f];
      v[0] = face.open_area;
      v[1] = face.inverse_density;
      v[2] = face.pressure_gradient_distance;
      v[3] = face.predicted_normal_velocity;
      v[4] = face.wall_normal_velocity;
      if (face.prescribed_wall_flux.has_value()) {
        const double flux = *face.prescribed_wall_flux;
        const double blocked = full_area - face.open_area;
        if (!std::isfinite(flux) || (blocked <= 0.0 && flux != 0.0)) return Code(absl::StatusCode::kInvalidArgument);
        if (blocked > 0.0) v[4] = flux / blocked;
      }
      if (const auto* internal = std::get_if<InternalMacPressureLink3D>(&face.pressure_link)) {
        s.face_kind[f] = 1;
        v[5] = internal->pressure_jump;
      } else if (const auto* dirichlet = std::get_if<DirichletMacPressureLink3D>(&face.pressure_link)) {
        s.face_kind[f] = 2;
        v[5] = dirichlet->exterior_pressure;
      } else {
        s.face_kind[f] = 0;
        v[5] = 0.0;
      }
    }
    auto& bank = self.projections_[1 - self.projection_bank_];
    bank.pressures.resize(nc);
    bank.rhs.resize(nc);
    bank.residuals.resize(nc);
    bank.defects.resize(nc);
    bank.velocities.resize(nf);
    bank.gauges.resize(nc);
    // Scale 1 is the reference's gate 2e-6 + 2e-6 ||b||; a tighter scale
    // solves to 2e-6 scale ||b||, which lies inside the scaled gate.
    const double rel_tol = options.cpu_residual_tolerance_scale < 1.0 ? 2e-6 * options.cpu_residual_tolerance_scale
                                                                       : 0.0;
    fl_mac_pressure_diagnostics d{};
    const int code = fl_boundary_project(
        self.boundary_, h, step_duration, s.cell_index.data(), s.cell_values.data(), nc, s.face_index.data(), s.face_kind.data(),
        s.face_values.data(), nf, static_cast<int>(options.max_iterations), rel_tol, bank.pressures.data(),
        bank.velocities.data(), bank.rhs.data(), bank.residuals.data(), bank.defects.data(),
        reinterpret_cast<std::uint64_t*>(bank.gauges.data()), &d, nullptr
    );
    if (code != FL_OK) return FromFl(code);
    bank.gauges.resize(d.gauge_count);
    for (std::size_t f = 0; f < nf; ++f) {
      const MacPressureFace3D& face = problem.faces[f];
      if (!face.prescribed_wall_flux.has_value()) continue;
      const auto& lattice = face.face_index.lattice_index;
      CellIndex3D tail{lattice.x, lattice.y, lattice.z};
      const int axis = static_cast<int>(face.face_index.axis);
      (axis == 0 ? tail.x : (axis == 1 ? tail.y : tail.z)) -= 1;
      const auto selected = [&](CellIndex3D c) {
        std::size_t lo = 0, hi = nc;
        while (lo < hi) {
          const std::size_t mid = (lo + hi) / 2;
          const CellIndex3D m = problem.cells[mid].cell_index;
          const bool less = m.z != c.z ? m.z < c.z : (m.y != c.y ? m.y < c.y : m.x < c.x);
          if (less) lo = mid + 1; else hi = mid;
        }
        if (lo >= nc) return false;
        const CellIndex3D m = problem.cells[lo].cell_index;
        return m.x == c.x && m.y == c.y && m.z == c.z;
      };
      const CellIndex3D head{lattice.x, lattice.y, lattice.z};
      if (selected(head)) inward_flux += *face.prescribed_wall_flux;
      if (selected(tail)) inward_flux -= *face.prescribed_wall_flux;
    }
    self.projection_bank_ = 1 - self.projection_bank_;
    MacPressureProjectionView3D view{};
    view.cell_pressures = bank.pressures;
    view.corrected_face_velocities = bank.velocities;
    view.integrated_rhs = bank.rhs;
    view.true_residuals = bank.residuals;
    view.cell_constraint_defects = bank.defects;
    view.gauge_cell_ordinals = bank.gauges;
    view.diagnostics.iteration_count = d.iterations;
    view.diagnostics.true_residual_l2 = d.true_residual_l2;
    view.diagnostics.max_volume_scaled_residual = d.max_volume_scaled_residual;
    view.diagnostics.max_cell_constraint_defect = d.max_cell_constraint_defect;
    view.frozen_measurement.integrated_rhs_l2_m3_per_s = d.rhs_l2;
    view.frozen_measurement.pressure_cell_volume_m3 = volume + volume_error;
    view.frozen_measurement.inward_prescribed_wall_flux_m3_per_s = inward_flux;
    return view;
  }
};

absl::StatusOr<std::unique_ptr<B200LiquidBackend3D>> B200LiquidBackend3D::Create() {
  std::unique_ptr<B200LiquidBackend3D> self(new (std::nothrow) B200LiquidBackend3D());
  if (!self) return Code(absl::StatusCode::kResourceExhausted);
  const int code = fl_boundary_create(&self->boundary_);
  if (code != FL_OK) return FromFl(code);
  bool ok = true;
  for (int k = 0; k < 2; ++k) {
    ok = ok && Reserve(self->deposits_[k].quanta, kFaces) && Reserve(self->deposits_[k].stencils, kParticles) &&
         Reserve(self->normalized_[k].masses, kFaces) && Reserve(self->normalized_[k].velocities, kFaces) &&
         Reserve(self->normalized_[k].validity, kFaces) && Reserve(self->gathered_[k].particles, kParticles) &&
         Reserve(self->projections_[k].pressures, kPressureCells) &&
         Reserve(self->projections_[k].velocities, kFaces) && Reserve(self->projections_[k].rhs, kPressureCells) &&
         Reserve(self->projections_[k].residuals, kPressureCells) &&
         Reserve(self->projections_[k].defects, kPressureCells) &&
         Reserve(self->projections_[k].gauges, kPressureCells);
  }
  for (int k = 0; k < 2; ++k)
    ok = ok && Reserve(self->links_[k].cells, kPressureCells) && Reserve(self->links_[k].faces, kFaces) &&
         Reserve(self->frozen_[k].centers, 27 * kPressureCells) && Reserve(self->frozen_[k].cells, kPressureCells) &&
         Reserve(self->frozen_[k].faces, kFaces);
  ok = ok && Reserve(self->freeze_staging_.faces, 6 * kPressureCells);
  for (int k = 0; k < 2; ++k)
    ok = ok && Reserve(self->pistons_[k].patches, kFaces) && Reserve(self->pistons_[k].face_fluxes, kFaces);
  auto& ps = self->piston_staging_;
  ok = ok && Reserve(ps.faces, kFaces) && Reserve(ps.positions, 3 * kParticles) && Reserve(ps.patches, kFaces) &&
       Reserve(ps.fluxes, kFaces) && Reserve(ps.has_flux, kFaces);
  auto& ls = self->link_staging_;
  ok = ok && Reserve(ls.faces, kFaces) && Reserve(ls.fields, kPressureCells) && Reserve(ls.wetted, kFaces) &&
       Reserve(ls.has_wetted, kFaces) && Reserve(ls.cells_out, kPressureCells) && Reserve(ls.faces_out, kFaces);
  auto& s = self->staging_;
  ok = ok && Reserve(s.cell_index, 3 * kPressureCells) && Reserve(s.cell_values, 5 * kPressureCells) &&
       Reserve(s.face_index, 4 * kFaces) && Reserve(s.face_kind, kFaces) && Reserve(s.face_values, 6 * kFaces);
  if (!ok) return Code(absl::StatusCode::kResourceExhausted);
  return self;
}

B200LiquidBackend3D::~B200LiquidBackend3D() {
  if (boundary_) fl_boundary_destroy(boundary_);
}

LiquidSubstepBackend3D B200LiquidBackend3D::operations() {
  LiquidSubstepBackend3D table{};
  table.context = this;
  table.initialize = [](void*, const LiquidState3D&) { return absl::OkStatus(); };
  table.prepare_publication = [](void*, const LiquidState3D&, LiquidClock3D) { return absl::OkStatus(); };
  table.commit_publication = [](void*) noexcept {};
  table.discard_publication = [](void*) noexcept {};
  table.prepare_growth = [](void*, LiquidStateCapacities3D, const LiquidState3D&) { return absl::OkStatus(); };
  table.commit_growth = [](void*) noexcept {};
  table.discard_growth = [](void*) noexcept {};
  table.deposit = &B200BackendOps3D::Deposit;
  table.normalize = &B200BackendOps3D::Normalize;
  table.predict_missing_face = &B200BackendOps3D::PredictMissingFace;
  table.forces = &B200BackendOps3D::Forces;
  table.gather = &B200BackendOps3D::Gather;
  table.freeze = &B200BackendOps3D::Freeze;
  table.wetted_piston = &B200BackendOps3D::WettedPiston;
  table.links = &B200BackendOps3D::Links;
  table.project = &B200BackendOps3D::Project;
  return table;
}

}  // namespace fluidity
