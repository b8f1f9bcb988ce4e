// B200 operations for FluidiTy's liquid scheduler backend table.
//
// Compiled against the reference's headers (native/include) as a maintainer
// adds it to that tree, beside native/cuda/liquid_substep_3d_host.cc whose
// CudaLiquidSubstepBackend3D::operations() (:140-233) it parallels. The table
// it returns fills the operations of the liquid step's transfer and
// projection path with this library's device kernels:
//
//   .deposit               fl_boundary_deposit        (DepositCompatibleMacQuanta3D)
//   .normalize             fl_boundary_normalize      (NormalizeLiquidMacFaces3D)
//   .predict_missing_face  fl_boundary_predict_face   (LiquidBoundaryWorkspace3D::ContinueFace + dt a)
//   .forces                fl_boundary_forces         (the CPU table's ApplyForces)
//   .gather                fl_boundary_gather         (GatherLiquidBoundaryParticles3D)
//   .freeze                fl_boundary_freeze         (FreezeLiquidBoundaryGeometry3D: no obstacle,
//                                                      halfspace, slab or open tank; sampled
//                                                      solids return kUnimplemented)
//   .wetted_piston         fl_boundary_wetted_piston  (ComputeWettedPiston3D)
//   .links                 fl_boundary_links          (BuildLiquidPressureLinks3D)
//   .project               fl_boundary_project        (ProjectMacPressure3D over a pressure problem)
//   .initialize, publication and growth hooks: no device state outlives a call
//
// The scene-geometry, topology and particle-update operations (.sample_*,
// .topology, .project_viscous, .update_particles)
// are outside this library and stay null: the scheduler's
// Create rejects a scene that needs them, and no CPU callback is substituted.
//
// Results borrow the backend's own two banks per region (deposit,
// normalization, gather, freeze, links, projection), reserved at Create for the reference's
// bounded capacities (1024 particles, 24576 faces, 4096 pressure cells); a
// borrow expires on the next successful operation of the same region, as the
// workspace's own do. Attempt operations allocate nothing; errors return
// code-only statuses and publish nothing.
#pragma once

#include <memory>
#include <vector>

#include "fluidity/host/liquid_substep_backend_3d.h"
#include "fluidity/host/wetted_piston_3d.h"
#include "fluidity_b200.h"

namespace fluidity {

class B200LiquidBackend3D {
 public:
  // Reserves the device and host storage; FailedPrecondition without a B200.
  static absl::StatusOr<std::unique_ptr<B200LiquidBackend3D>> Create();
  ~B200LiquidBackend3D();
  B200LiquidBackend3D(const B200LiquidBackend3D&) = delete;
  B200LiquidBackend3D& operator=(const B200LiquidBackend3D&) = delete;

  // The table; its context is this object, which must outlive the scheduler.
  LiquidSubstepBackend3D operations();

  struct DepositBank {
    std::vector<MacFaceDepositQuanta3D> quanta;
    std::vector<LiquidCompatibleStencils3D> stencils;
  };
  struct NormalizeBank {
    std::vector<double> masses;
    std::vector<double> velocities;
    std::vector<LiquidFaceValidity3D> validity;
  };
  struct GatherBank {
    std::vector<LiquidBoundaryParticleGather3D> particles;
  };
  struct ProjectionBank {
    std::vector<double> pressures, velocities, rhs, residuals, defects;
    std::vector<std::size_t> gauges;
  };
  struct LinkBank {
    std::vector<MacPressureCell3D> cells;
    std::vector<MacPressureFace3D> faces;
  };
  struct PistonBank {
    std::vector<WettedPistonPatch3D> patches;
    std::vector<std::optional<double>> face_fluxes;
  };
  // Host staging of the wetted piston's inputs and outputs in the C-ABI's layout.
  struct PistonStaging {
    std::vector<fl_frozen_face> faces;
    std::vector<double> positions;
    std::vector<fl_piston_patch> patches;
    std::vector<double> fluxes;
    std::vector<std::uint8_t> has_flux;
  };
  struct FreezeBank {
    std::vector<LiquidCenterDistance3D> centers;
    std::vector<FrozenLiquidCell3D> cells;
    std::vector<FrozenLiquidFace3D> faces;
  };
  // Host staging of the link assembly's optional-valued records in the C-ABI's layout.
  struct LinkStaging {
    std::vector<fl_frozen_face> faces;
    std::vector<fl_pressure_cell_fields> fields;
    std::vector<double> wetted;
    std::vector<std::uint8_t> has_wetted;
    std::vector<fl_pressure_cell> cells_out;
    std::vector<fl_pressure_link> faces_out;
  };
  // Host staging of the freeze's face records in the C-ABI's layout.
  struct FreezeStaging {
    std::vector<fl_frozen_face> faces;
  };
  // Host staging of a pressure problem in the C-ABI's record layout.
  struct PressureStaging {
    std::vector<std::int32_t> cell_index;
    std::vector<double> cell_values;
    std::vector<std::int32_t> face_index;
    std::vector<std::int32_t> face_kind;
    std::vector<double> face_values;
  };

 private:
  B200LiquidBackend3D() = default;
  friend struct B200BackendOps3D;
  fl_boundary* boundary_ = nullptr;
  DepositBank deposits_[2];
  NormalizeBank normalized_[2];
  GatherBank gathered_[2];
  ProjectionBank projections_[2];
  LinkBank links_[2];
  FreezeBank frozen_[2];
  PistonBank pistons_[2];
  PistonStaging piston_staging_;
  PressureStaging staging_;
  LinkStaging link_staging_;
  FreezeStaging freeze_staging_;
  int deposit_bank_ = 0, normalize_bank_ = 0, gather_bank_ = 0, projection_bank_ = 0, links_bank_ = 0,
      frozen_bank_ = 0, piston_bank_ = 0;
};

}  // namespace fluidity
