// mkb200_compat.hpp — header-only C++ shim with MaterKit's class names over the
// C ABI of mkb200.h, so a MaterKit.cpp-style driver keeps its structure.
//
// Replaces, for the solver path only:
//   mkSpace(xml)                                   MaterKit/inc/mkSpace.h:36
//   readParameters(maxLoops, maxFrame, xml)        MaterKit/inc/mkFunction.h:62
//   mkFluidsMRT / mkFluidsMultiphase: reset, initialize, initialize_geometry,
//   propagate / relaxation* per field, write_vtkfile, check_variables
//                                                  MaterKit/inc/mkFluidsMRT.h:26-49,
//                                                  MaterKit/inc/mkFluidsMultiphase.h:20-59
// The per-field calls of one loop are recorded and the device runs the fused
// loop when the loop's last relaxation is called.  Errors throw mkb200::Error
// (the reference throws mkIOError and relatives).  Direct access to node[i]
// (the mkFluidsUser pattern) is not offered: the state lives on the device.
#ifndef MKB200_COMPAT_HPP
#define MKB200_COMPAT_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "mkb200.h"

namespace mkb200 {

struct Error : std::runtime_error {
  mk_status status;
  Error(mk_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(mk_status s, const mk_handle* h = nullptr) {
  if (s != MK_OK) throw Error(s, h ? mk_last_error(h) : mk_last_global_error());
}

inline void readParameters(int& maxLoops, int& maxFrame, const std::string& xml) {
  int32_t l = 0, f = 0;
  check(mk_read_parameters(xml.c_str(), &l, &f));
  maxLoops = l;
  maxFrame = f;
}

class mkSpace {
 public:
  explicit mkSpace(const std::string& xml) : xml_(xml) {
    mk_options o;
    o.model = o.precision = o.collision = o.lattice = -1;
    o.magic = -1.0;
    o.device = -1;
    o.block_x = o.block_y = 0;
    check(mk_case_params(xml.c_str(), &o, &p_));
  }
  int Mx() const { return p_.nx; }
  int My() const { return p_.ny; }
  int Mz() const { return p_.nz; }
  const std::string& xml() const { return xml_; }

 private:
  std::string xml_;
  mk_params p_;
};

// Common lifecycle of the reference's solver classes.
class mkSolver {
 public:
  explicit mkSolver(const mkSpace& space, int model) : xml_(space.xml()), model_(model) {}
  mkSolver(const mkSolver&) = delete;
  mkSolver& operator=(const mkSolver&) = delete;
  virtual ~mkSolver() {
    if (h_) mk_destroy(h_);
  }
  void reset(const std::string& xml) { xml_ = xml; }
  void initialize(const std::string& xml, int model = -1, int precision = -1) {
    xml_ = xml;
    if (model >= 0) model_ = model;
    mk_options o;
    o.model = model_;
    o.precision = precision;
    o.collision = o.lattice = -1;
    o.magic = -1.0;
    o.device = -1;
    o.block_x = o.block_y = 0;
    if (h_) mk_destroy(h_);
    h_ = nullptr;
    check(mk_create_from_xml(xml_.c_str(), &o, &h_));
  }
  void initialize_geometry() {
    if (!h_) throw Error(MK_ERR_STATE, "initialize() first");
  }
  void write_vtkfile(int loops, const std::string& dir = "vtk") { check(mk_write_vtk(h_, loops, dir.c_str()), h_); }
  mk_diag check_variables(int /*loops*/, char /*plane*/ = 'x') {
    mk_diag d;
    check(mk_diagnostics(h_, &d), h_);
    return d;
  }
  std::vector<double> field(mk_field f) {
    mk_params p;
    check(mk_get_params(h_, &p), h_);
    std::vector<double> v((size_t)p.nx * p.ny * p.nz);
    check(mk_get_field(h_, f, MK_DTYPE_F64, v.data(), v.size() * sizeof(double)), h_);
    return v;
  }
  mk_handle* handle() { return h_; }

 protected:
  // Record one call of the loop; run the device loop when the sequence completes.
  void call(const char* name, const std::vector<std::string>& seq) {
    if (!h_) throw Error(MK_ERR_STATE, "initialize() first");
    if (pending_ >= seq.size() || seq[pending_] != name)
      throw Error(MK_ERR_STATE, std::string(name) + "() out of the reference's per-loop order");
    if (++pending_ == seq.size()) {
      pending_ = 0;
      check(mk_advance(h_, 1), h_);
    }
  }
  std::string xml_;
  int model_;
  mk_handle* h_ = nullptr;
  size_t pending_ = 0;
};

// Flow and dendrite solver (MaterKit/inc/mkFluidsMRT.h).  The model comes from
// initialize(xml, model): MK_MODEL_FLOW (run_flow_Poiseuille),
// MK_MODEL_THERMAL_DENDRITE (run_thermal_dendrite), MK_MODEL_SOLUTAL_DENDRITE
// (run_solutal_dendrite), MK_MODEL_FLOW_DENDRITE (run_flow_thermal_dendrite),
// MK_MODEL_FLOW_SOLUTAL (run_flow_solutal_dendrite) or MK_MODEL_MULTIGRAIN
// (run_multiPhaseField).
class mkFluidsMRT : public mkSolver {
 public:
  explicit mkFluidsMRT(const mkSpace& s) : mkSolver(s, MK_MODEL_FLOW) {}
  void initialize_geometry_Poiseuille() { initialize_geometry(); }
  // mkFluidsLBM::propagate / relaxation (MaterKit.cpp:277-280)
  void propagate() { call("propagate", seq()); }
  void relaxation() { call("relaxation", seq()); }
  // mkPhaseField::propagate / relaxation_anisotropy_thermal, mkThermalField::propagate /
  // relaxation (MaterKit.cpp:775-781)
  void phasefield_propagate() { call("pf_propagate", seq()); }
  void relaxation_anisotropy_thermal() { call("pf_relax", seq()); }
  void thermal_propagate() { call("t_propagate", seq()); }
  void thermal_relaxation() { call("t_relax", seq()); }
  // mkFluidsMRT::propagate_PBB, bdyVelocity, mkThermalField::bdy_flowin
  // (MaterKit.cpp:499-516)
  void propagate_PBB() { call("propagate_PBB", seq()); }
  void bdyVelocity() { call("bdyVelocity", seq()); }
  void bdy_flowin() { call("bdy_flowin", seq()); }
  // mkPhaseField::relaxation_anisotropy_solute(loops), mkSolutalField::propagate /
  // relaxation / bdy_LBflowin (MaterKit.cpp:665-674, 448-456)
  void relaxation_anisotropy_solute(int /*loops*/) { call("pf_relax_solute", seq()); }
  // run_flow_multiphase_dendrite (MaterKit.cpp:377-397): the dendrite's
  // calls that take the two-phase flow.  update_velocity copies the flow's
  // velocity for the thermal relaxation (mkThermalField::update_velocity,
  // mkThermalField.h:36); the phase field does not read the flow.
  void relaxation_anisotropy_thermal(mkSolver& /*flow*/) { relaxation_anisotropy_thermal(); }
  void update_velocity(mkSolver& flow) { check(mk_update_velocity(h_, flow.handle()), h_); }
  void thermal_relaxation(mkSolver& /*flow*/) { thermal_relaxation(); }
  void solutal_propagate() { call("c_propagate", seq()); }
  void solutal_relaxation() { call("c_relax", seq()); }
  void bdy_LBflowin() { call("bdy_LBflowin", seq()); }

 private:
  std::vector<std::string> seq() const {
    if (model_ == MK_MODEL_FLOW_DENDRITE)
      return {"propagate_PBB", "relaxation", "bdyVelocity", "pf_propagate", "pf_relax", "t_propagate", "t_relax",
              "bdy_flowin"};
    if (model_ == MK_MODEL_FLOW_SOLUTAL)  // run_flow_solutal_dendrite (MaterKit.cpp:430-456)
      return {"propagate_PBB", "relaxation", "bdyVelocity", "pf_propagate", "pf_relax_solute", "c_propagate",
              "c_relax", "bdy_LBflowin"};
    if (model_ == MK_MODEL_SOLUTAL_DENDRITE)  // run_solutal_dendrite (MaterKit.cpp:665-674)
      return {"pf_propagate", "pf_relax_solute", "c_propagate", "c_relax"};
    if (model_ == MK_MODEL_THERMAL_DENDRITE)
      return {"pf_propagate", "pf_relax", "t_propagate", "t_relax"};
    if (model_ == MK_MODEL_MULTIGRAIN)  // run_multiPhaseField (MaterKit.cpp:563-567)
      return {"propagate", "relaxation", "t_propagate", "t_relax"};
    return {"propagate", "relaxation"};
  }
};

// Two-phase Allen-Cahn flow (MaterKit/inc/mkFluidsMultiphase.h), run_flow_multiphase
// (MaterKit.cpp:290-331).
class mkFluidsMultiphase : public mkSolver {
 public:
  explicit mkFluidsMultiphase(const mkSpace& s) : mkSolver(s, MK_MODEL_MULTIPHASE) {}
  void propagate() { call("propagate", {"propagate", "relaxation"}); }
  void relaxation() { call("relaxation", {"propagate", "relaxation"}); }
  // The dendrite's solid (phi > 0) becomes this flow's geometry from its next
  // even loop count (mkFluidsMultiphase::update_geometry, mkFluidsMultiphase.h:37).
  void update_geometry(mkSolver& dendrite) { check(mk_update_geometry(h_, dendrite.handle()), h_); }
};

}  // namespace mkb200

#endif
