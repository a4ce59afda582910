// mk_case.cpp — see mk_case.hpp.
//
// Unit conversion of the reference's physical-unit tags (the DLL's own
// conversion is closed; this is the one the XML comments describe):
//   lattice viscosity  nu = kinematicViscosity * mk_dt / mk_dx^2
//   lattice accel.     g  = Gravity * mk_dt^2 / mk_dx
//   phase field        W0_lu = W0 / mk_dx, tau0_lu = t0 / mk_dt           (thermal.xml:56-63)
//                      lambda = 0.8839 W0 / d0 when <lambda> is negative   (thermal.xml:61)
//   diffusivities      D_lu = alphaFluid * mk_dt / mk_dx^2 (in W0^2/tau0 units)
// The optional <b200> element carries lattice-unit values directly and
// overrides all of the above.
#include "mk_case.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "mk_models.hpp"
#include "mk_xml.hpp"

namespace mkc {

void default_params(mk_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->model = MK_MODEL_FLOW;
  p->lattice = MK_D3Q19;
  p->collision = MK_COLL_TRT;
  p->precision = MK_PREC_FP32;
  p->nx = p->ny = p->nz = 1;
  p->bc[0] = p->bc[1] = p->bc[2] = MK_BC_PERIODIC;
  p->max_loops = 300;  // defaults of MaterKit.cpp:190-191
  p->max_frames = 100;
  p->rho0 = 1.0;
  p->tau = 0.8;
  p->magic = 3.0 / 16.0;
  p->rho_l = 1.0;
  p->rho_g = 0.1;
  p->tau_l = 0.8;
  p->tau_g = 0.53;
  p->sigma = 1e-3;
  p->width = 4.0;
  p->mobility = 0.05;
  p->contact_angle = 90.0;
  p->eps4 = 0.05;
  p->W0 = 1.5;
  p->lambda = 10.0;
  p->delta = 0.55;
  p->D = 0.1;
  p->D_s = 1e-4;
  p->k_part = 0.15;
  p->at_coef = 1.0 / (2.0 * std::sqrt(2.0));
  p->tau0 = 0.6267 * p->lambda * p->W0 * p->W0 / p->D;
  p->rng_seed = 0;
  p->aniso = MK_ANISO_CUBIC;
  p->eps2 = 0.0;
  p->wall_axis = -1;
  p->inlet = 0;
  p->grain_kappa = 1.0;
  // grain 1 relaxes towards an equilibrium moving at (0.02, 0, 0) in the
  // reference's multigrain relaxation (mkFluidsUser.cpp:220-226)
  p->grain_u[0] = 0.02;
  p->grain_u[1] = p->grain_u[2] = 0.0;
}

void default_options(mk_options* o) {
  o->model = -1;
  o->precision = -1;
  o->collision = -1;
  o->lattice = -1;
  o->magic = -1.0;
  o->device = -1;
  o->block_x = 0;
  o->block_y = 0;
}

bool read_parameters(const std::string& xml, int* loops, int* frames, std::string& err) {
  mkx::Document doc;
  if (!mkx::parse_file(xml, doc, err)) return false;
  const mkx::Element* r = doc.root.get();
  int l = 300, f = 100;
  if (const mkx::Element* e = r->path("output/numLoops"))
    if (!mkx::read_int(e, l, err)) return false;
  if (const mkx::Element* e = r->path("output/numFrames"))
    if (!mkx::read_int(e, f, err)) return false;
  *loops = l;
  *frames = f;
  return true;
}

namespace {

std::string lower(std::string s) {
  for (auto& c : s) c = (char)tolower((unsigned char)c);
  return s;
}

// Optional scalar: leaves `out` untouched when the element is absent.
bool opt_d(const mkx::Element* r, const char* path, double& out, std::string& err) {
  const mkx::Element* e = r ? r->path(path) : nullptr;
  if (!e) return true;
  return mkx::read_double(e, out, err);
}

bool opt_v(const mkx::Element* r, const char* path, std::vector<double>& out, std::string& err) {
  const mkx::Element* e = r ? r->path(path) : nullptr;
  if (!e) return true;
  return mkx::read_doubles(e, out, err);
}

int parse_bc(const std::string& t) {
  std::string s = lower(t);
  if (s == "periodic" || s == "p") return MK_BC_PERIODIC;
  if (s == "walls" || s == "wall" || s == "w" || s == "bounceback") return MK_BC_WALLS;
  if (s == "closed" || s == "noflux" || s == "zeroflux" || s == "c") return MK_BC_CLOSED;
  return -1;
}

// Seeds of <phasechange><seed> (BoltzTechs - thermal.xml:65-77): number,
// center triples (lattice units), angle triples (degrees, ZYX), radius.
// A centre list shorter than 3 * number places only the seeds whose centre
// is complete (the shipped BoltzTechs - solutal.xml declares 2 seeds and
// gives one centre): number is reduced to the count of full triples.
bool read_seeds(const mkx::Element* seed, mk_params* p, std::string& err) {
  if (!seed) return true;
  int number = 0;
  if (const mkx::Element* e = seed->child("number"))
    if (!mkx::read_int(e, number, err)) return false;
  if (number < 0 || number > MK_MAX_OBJECTS) {
    err = "seed/number out of range";
    return false;
  }
  std::vector<double> c, a, r;
  if (!opt_v(seed, "center", c, err) || !opt_v(seed, "angle", a, err) || !opt_v(seed, "radius", r, err)) return false;
  number = std::min(number, (int)c.size() / 3);
  p->n_objects = number;
  for (int k = 0; k < number; ++k) {
    for (int d = 0; d < 3; ++d) {
      p->obj_center[k][d] = c[3 * k + d];
      p->obj_angle[k][d] = (int)a.size() >= 3 * (k + 1) ? a[3 * k + d] : 0.0;
    }
    p->obj_radius[k] = r.empty() ? 8.0 : ((int)r.size() > k ? r[k] : r.back());
  }
  return true;
}

// Non-overlapping bubbles drawn from splitmix64: radius U[rmin, rmax], centre
// uniform; gap >= `gap` from every other bubble (minimum image on periodic
// axes) and from walled / closed faces.
bool random_bubbles(mk_params* p, int number, double rmin, double rmax, double gap, unsigned long long seed,
                    std::string& err) {
  if (number < 0 || number > MK_MAX_OBJECTS) {
    err = "random/bubbles out of range";
    return false;
  }
  SplitMix64 rng(seed);
  const int n3[3] = {p->nx, p->ny, p->nz};
  for (int b = 0; b < number; ++b) {
    const double R = rmin + (rmax - rmin) * rng.uniform();
    bool placed = false;
    for (int attempt = 0; attempt < 100000 && !placed; ++attempt) {
      double c[3];
      bool ok = true;
      for (int a = 0; a < 3; ++a) {
        if (p->bc[a] == MK_BC_PERIODIC) {
          c[a] = n3[a] * rng.uniform();
        } else {
          // fluid spans [1, n-2] for walls and [0, n-1] for closed faces
          const double lo = (p->bc[a] == MK_BC_WALLS ? 1.0 : 0.0) + R + gap;
          const double hi = (p->bc[a] == MK_BC_WALLS ? n3[a] - 2.0 : n3[a] - 1.0) - R - gap;
          const double u = rng.uniform();
          if (hi < lo) {
            ok = false;
            continue;
          }
          c[a] = lo + (hi - lo) * u;
        }
      }
      if (!ok) continue;
      for (int k = 0; k < b && ok; ++k) {
        double d2 = 0;
        for (int a = 0; a < 3; ++a) {
          double d = std::fabs(c[a] - p->obj_center[k][a]);
          if (p->bc[a] == MK_BC_PERIODIC && d > 0.5 * n3[a]) d = n3[a] - d;
          d2 += d * d;
        }
        const double need = R + p->obj_radius[k] + gap;
        if (d2 < need * need) ok = false;
      }
      if (ok) {
        for (int a = 0; a < 3; ++a) {
          p->obj_center[b][a] = c[a];
          p->obj_angle[b][a] = 0.0;
        }
        p->obj_radius[b] = R;
        placed = true;
      }
    }
    if (!placed) {
      err = "could not place the random bubbles without overlap";
      return false;
    }
  }
  p->n_objects = number;
  p->rng_seed = seed;
  return true;
}

}  // namespace

mk_status validate_params(const mk_params* p, std::string& err) {
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) {
    err = "MeshXYZ must be positive";
    return MK_ERR_ARG;
  }
  // cell indices inside a population plane are 32-bit on the device
  const double cells = (double)p->nx * p->ny * p->nz;
  if (cells >= 2147483647.0 - 64.0) {
    err = "domain too large (at most 2^31 - 65 cells)";
    return MK_ERR_ARG;
  }
  for (int a = 0; a < 3; ++a) {
    if (p->bc[a] < 0 || p->bc[a] > 2) {
      err = "bad boundary kind";
      return MK_ERR_ARG;
    }
    const int n = a == 0 ? p->nx : (a == 1 ? p->ny : p->nz);
    if (p->bc[a] == MK_BC_WALLS && n < 3) {
      err = "a walled axis needs at least 3 cells";
      return MK_ERR_ARG;
    }
  }
  if (p->model < 0 || p->model > MK_MODEL_FLOW_SOLUTAL) {
    err = "unknown model";
    return MK_ERR_ARG;
  }
  if (p->precision < 0 || p->precision > 3) {
    err = "unknown precision";
    return MK_ERR_ARG;
  }
  if (p->wall_axis < -1 || p->wall_axis > 2) {
    err = "wall_axis must be -1, 0, 1 or 2";
    return MK_ERR_ARG;
  }
  if (p->wall_axis >= 0 && p->bc[p->wall_axis] != MK_BC_WALLS) {
    err = "the plate axis must have walled faces";
    return MK_ERR_ARG;
  }
  if (p->wall_axis >= 0 && p->model != MK_MODEL_FLOW && p->model != MK_MODEL_CONVECTION) {
    err = "plates (wall_axis) apply to the flow and convection models";
    return MK_ERR_ARG;
  }
  if (p->model == MK_MODEL_CONVECTION) {
    if (!(p->D > 0)) {
      err = "convection needs a positive scalar diffusivity";
      return MK_ERR_ARG;
    }
    if (p->wall_axis < 0) {
      err = "convection needs a plate axis (wall_axis)";
      return MK_ERR_ARG;
    }
  }
  if (p->inlet) {
    if (p->model != MK_MODEL_FLOW && !mkm::flow_coupled(p->model)) {
      err = "inflow / outflow faces apply to the flow and flow + dendrite models";
      return MK_ERR_ARG;
    }
    if (p->bc[0] != MK_BC_CLOSED || p->nx < 3) {
      err = "inflow / outflow faces need closed x faces and at least 3 cells along x";
      return MK_ERR_ARG;
    }
    if (p->wall_axis == 0) {
      err = "inflow / outflow faces and plates on x exclude each other";
      return MK_ERR_ARG;
    }
  }
  if (p->model == MK_MODEL_FLOW || p->model == MK_MODEL_CONVECTION || mkm::flow_coupled(p->model)) {
    if (p->lattice != MK_D3Q19 && p->lattice != MK_D3Q27) {
      err = "flow lattice must be D3Q19 or D3Q27";
      return MK_ERR_ARG;
    }
    if (p->collision < 0 || p->collision > 2) {
      err = "unknown collision";
      return MK_ERR_ARG;
    }
    if (p->collision == MK_COLL_MRT && p->lattice != MK_D3Q19) {
      err = "MRT is defined for D3Q19 only";
      return MK_ERR_ARG;
    }
    if (!(p->tau > 0.5)) {
      err = "tau must exceed 1/2";
      return MK_ERR_ARG;
    }
    if (p->collision == MK_COLL_TRT && !(p->magic > 0)) {
      err = "TRT magic parameter must be positive";
      return MK_ERR_ARG;
    }
    if (!(p->rho0 > 0)) {
      err = "rho0 must be positive";
      return MK_ERR_ARG;
    }
  } else if (p->model == MK_MODEL_MULTIPHASE) {
    if (!(p->tau_l > 0.5 && p->tau_g > 0.5 && p->rho_l > 0 && p->rho_g > 0 && p->width > 0 && p->mobility > 0)) {
      err = "multiphase parameters out of range (tau > 1/2, densities, W, M > 0)";
      return MK_ERR_ARG;
    }
  }
  if (p->model == MK_MODEL_MULTIGRAIN) {
    if (p->n_objects < 1 || p->n_objects > MK_MAX_OBJECTS) {
      err = "the multigrain model needs 1 to 64 seeds (one order parameter per grain)";
      return MK_ERR_ARG;
    }
    if (!(p->W0 > 0 && p->mobility > 0 && p->D > 0)) {
      err = "multigrain parameters out of range (W0, mobility, D > 0)";
      return MK_ERR_ARG;
    }
  }
  if (mkm::dendrite(p->model)) {
    if (!(p->W0 > 0 && p->tau0 > 0 && p->D > 0)) {
      err = "phase-field parameters out of range (W0, tau0, D > 0)";
      return MK_ERR_ARG;
    }
    if (p->n_objects < 0 || p->n_objects > MK_MAX_OBJECTS) {
      err = "bad seed count";
      return MK_ERR_ARG;
    }
    if (p->aniso < MK_ANISO_CUBIC || p->aniso > MK_ANISO_FACET) {
      err = "unknown anisotropy kind";
      return MK_ERR_ARG;
    }
    if (p->aniso == MK_ANISO_FACET && !(p->eps2 > 0)) {
      err = "facet anisotropy needs a positive cusp width (eps2)";
      return MK_ERR_ARG;
    }
  }
  return MK_OK;
}

mk_status resolve_case(const std::string& xml, const mk_options* opt, mk_params* out, std::string& err) {
  mkx::Document doc;
  if (!mkx::parse_file(xml, doc, err)) return MK_ERR_XML;
  const mkx::Element* r = doc.root.get();
  mk_params p;
  default_params(&p);

  // geometry/MeshXYZ (mkSpace.h:36)
  std::vector<double> mesh;
  if (!r->path("geometry/MeshXYZ")) {
    err = "missing geometry/MeshXYZ";
    return MK_ERR_XML;
  }
  if (!mkx::read_doubles(r->path("geometry/MeshXYZ"), mesh, err)) return MK_ERR_XML;
  if (mesh.size() < 3) {
    err = "geometry/MeshXYZ needs 3 values";
    return MK_ERR_XML;
  }
  p.nx = (int)mesh[0];
  p.ny = (int)mesh[1];
  p.nz = (int)mesh[2];
  int loops = p.max_loops, frames = p.max_frames;
  if (const mkx::Element* e = r->path("output/numLoops"))
    if (!mkx::read_int(e, loops, err)) return MK_ERR_XML;
  if (const mkx::Element* e = r->path("output/numFrames"))
    if (!mkx::read_int(e, frames, err)) return MK_ERR_XML;
  p.max_loops = loops;
  p.max_frames = frames;

  double dx = 1.0, dt = 1.0;
  if (!opt_d(r, "numerics/mk_dx", dx, err) || !opt_d(r, "numerics/mk_dt", dt, err)) return MK_ERR_XML;
  if (!(dx > 0 && dt > 0)) {
    err = "numerics/mk_dx and mk_dt must be positive";
    return MK_ERR_XML;
  }
  std::vector<double> grav;
  if (!opt_v(r, "geometry/Gravity", grav, err)) return MK_ERR_XML;
  double g_lu[3] = {0, 0, 0};
  for (int a = 0; a < 3 && a < (int)grav.size(); ++a) g_lu[a] = grav[a] * dt * dt / dx;

  // model: option > <b200><model> > calcMode
  const mkx::Element* b = r->child("b200");
  int model = -1;
  if (b && b->child("model")) {
    const std::string m = lower(mkx::trimmed(b->child("model")->text));
    if (m == "flow" || m == "poiseuille")
      model = MK_MODEL_FLOW;
    else if (m == "multiphase" || m == "allencahn" || m == "allen_cahn")
      model = MK_MODEL_MULTIPHASE;
    else if (m == "thermal_dendrite" || m == "thermal")
      model = MK_MODEL_THERMAL_DENDRITE;
    else if (m == "solutal_dendrite" || m == "solutal")
      model = MK_MODEL_SOLUTAL_DENDRITE;
    else if (m == "convection" || m == "rbc" || m == "rayleigh_benard")
      model = MK_MODEL_CONVECTION;
    else if (m == "flow_dendrite" || m == "flow_thermal_dendrite")
      model = MK_MODEL_FLOW_DENDRITE;
    else if (m == "flow_solutal_dendrite" || m == "flow_solutal")
      model = MK_MODEL_FLOW_SOLUTAL;
    else if (m == "multigrain" || m == "multiphasefield" || m == "multi_phase_field")
      model = MK_MODEL_MULTIGRAIN;
    else {
      err = "<b200><model>: unknown model '" + m + "'";
      return MK_ERR_XML;
    }
  }
  if (opt && opt->model >= 0) model = opt->model;
  if (model < 0) {
    // calcMode as the reference's driver reads it: a dendrite in a flow
    // (run_flow_thermal_dendrite), a dendrite alone, or a flow alone
    bool dendrite = false, flowfield = false;
    if (const mkx::Element* e = r->path("calcMode/dendrite"))
      if (!mkx::read_bool(e, dendrite, err)) return MK_ERR_XML;
    if (const mkx::Element* e = r->path("calcMode/flowField"))
      if (!mkx::read_bool(e, flowfield, err)) return MK_ERR_XML;
    model = dendrite ? (flowfield ? MK_MODEL_FLOW_DENDRITE : MK_MODEL_THERMAL_DENDRITE) : MK_MODEL_FLOW;
  }
  p.model = model;

  // --- physical-unit tags of the shipped cases
  double omega_f = -1;
  if (!opt_d(r, "numerics/omega_f", omega_f, err)) return MK_ERR_XML;
  if (model == MK_MODEL_CONVECTION) {
    // Rayleigh-Benard (bdy_RBC, mkFluidsUser.cpp:362-392): gravity from
    // geometry/Gravity, the expansion coefficient from temperature/beta,
    // plates normal to y (the reference's bdy_RBC) holding
    // composition/highValue at y = 0 and composition/lowValue at y = My-1
    double nu = -1, alpha = -1, beta = 0, hi = 1.0, lo = 0.0;
    if (!opt_d(r, "phases/fluid/kinematicViscosity", nu, err) || !opt_d(r, "temperature/alphaFluid", alpha, err) ||
        !opt_d(r, "temperature/beta", beta, err) || !opt_d(r, "composition/highValue", hi, err) ||
        !opt_d(r, "composition/lowValue", lo, err))
      return MK_ERR_XML;
    if (nu > 0) p.tau = 3.0 * nu * dt / (dx * dx) + 0.5;
    if (omega_f > 0) p.tau = 1.0 / omega_f;
    if (alpha > 0) p.D = alpha * dt / (dx * dx);
    p.beta = beta;
    p.rho0 = 1.0;
    for (int a = 0; a < 3; ++a) p.force[a] = g_lu[a];
    p.bc[0] = MK_BC_PERIODIC;
    p.bc[1] = MK_BC_WALLS;
    p.bc[2] = MK_BC_PERIODIC;
    p.wall_axis = 1;
    p.wall_value[0] = hi;
    p.wall_value[1] = lo;
    p.s_ref = 0.5 * (hi + lo);
    p.collision = MK_COLL_TRT;
  } else if (model == MK_MODEL_FLOW) {
    double nu = -1, rho = 1.0;
    if (!opt_d(r, "phases/fluid/kinematicViscosity", nu, err)) return MK_ERR_XML;
    if (nu > 0) p.tau = 3.0 * nu * dt / (dx * dx) + 0.5;
    if (omega_f > 0) p.tau = 1.0 / omega_f;
    p.rho0 = 1.0;
    (void)rho;
    std::vector<double> acc;
    if (!opt_v(r, "flow/acceleration", acc, err)) return MK_ERR_XML;
    for (int a = 0; a < 3; ++a) p.force[a] = (a < (int)acc.size() ? acc[a] : 0.0) + g_lu[a];
    // channel walls at y = 0 and y = My-1 (MaterKit/src/mkFluidsUser.cpp:55-58)
    p.bc[0] = MK_BC_PERIODIC;
    p.bc[1] = MK_BC_WALLS;
    p.bc[2] = MK_BC_PERIODIC;
    p.collision = MK_COLL_TRT;
  } else if (model == MK_MODEL_MULTIPHASE) {
    double nu_d = -1, rho_d = -1, nu_r = -1, rho_r = -1, W = -1, M = -1, sig = -1, th = 90;
    if (!opt_d(r, "multiphases/fluidDense/kinematicViscosity", nu_d, err) ||
        !opt_d(r, "multiphases/fluidDense/density", rho_d, err) ||
        !opt_d(r, "multiphases/fluidRare/kinematicViscosity", nu_r, err) ||
        !opt_d(r, "multiphases/fluidRare/density", rho_r, err) || !opt_d(r, "multiphases/W0", W, err) ||
        !opt_d(r, "multiphases/Mobility", M, err) || !opt_d(r, "multiphases/sigma", sig, err) ||
        !opt_d(r, "multiphases/contactAngle", th, err))
      return MK_ERR_XML;
    if (rho_d > 0 && rho_r > 0) {
      p.rho_l = 1.0;
      p.rho_g = rho_r / rho_d;
    }
    if (nu_d > 0) p.tau_l = 3.0 * nu_d * dt / (dx * dx) + 0.5;
    if (nu_r > 0) p.tau_g = 3.0 * nu_r * dt / (dx * dx) + 0.5;
    if (W > 0) p.width = W / dx;
    if (M > 0) p.mobility = M * dt / (dx * dx);
    if (sig > 0) p.sigma = sig;
    p.contact_angle = th;
    std::vector<double> fd;
    if (!opt_v(r, "multiphases/force", fd, err)) return MK_ERR_XML;
    for (int a = 0; a < 3; ++a) {
      const double fa = (a < (int)fd.size() && rho_d > 0) ? fd[a] / rho_d * dt * dt / dx : 0.0;
      p.force[a] = g_lu[a] + fa;
    }
    p.bc[0] = MK_BC_PERIODIC;
    p.bc[1] = MK_BC_WALLS;
    p.bc[2] = MK_BC_PERIODIC;
    p.collision = MK_COLL_MRT;
    if (!read_seeds(r->path("phasechange/seed"), &p, err)) return MK_ERR_XML;
  } else {
    double W0 = 1.0, t0 = 1.0, d0 = -1, lam = -1, eps = p.eps4, alpha = -1, under = p.delta, ini = 1e300;
    if (!opt_d(r, "phasechange/W0", W0, err) || !opt_d(r, "phasechange/t0", t0, err) ||
        !opt_d(r, "phasechange/d0", d0, err) || !opt_d(r, "phasechange/lambda", lam, err) ||
        !opt_d(r, "phasechange/anisotropy", eps, err))
      return MK_ERR_XML;
    p.eps4 = eps;
    p.W0 = W0 / dx;
    p.tau0 = t0 / dt;
    if (lam > 0)
      p.lambda = lam;
    else if (d0 > 0)
      p.lambda = 0.8839 * W0 / d0;
    if (model == MK_MODEL_MULTIGRAIN) {
      // the grains' Allen-Cahn relaxation rate 1/(dt/dx^2/cs^2 + 1/2)
      // (mkFluidsUser.cpp:282): mobility dt/dx^2, 1 in lattice units
      p.mobility = 1.0;
    }
    if (model == MK_MODEL_THERMAL_DENDRITE || model == MK_MODEL_FLOW_DENDRITE || model == MK_MODEL_MULTIGRAIN) {
      if (!opt_d(r, "temperature/alphaFluid", alpha, err) || !opt_d(r, "temperature/undercooling", under, err) ||
          !opt_d(r, "temperature/iniValue", ini, err))
        return MK_ERR_XML;
      if (alpha > 0) p.D = alpha * dt / (dx * dx);
      p.delta = ini < 1e299 ? -ini : under;
    } else {
      double dl = -1, ds = -1, kp = -1, iv = 1e300;
      if (!opt_d(r, "composition/diffFluid", dl, err) || !opt_d(r, "composition/diffSolid", ds, err) ||
          !opt_d(r, "composition/partition", kp, err) || !opt_d(r, "composition/iniValue", iv, err))
        return MK_ERR_XML;
      if (dl > 0) p.D = dl * dt / (dx * dx);
      if (ds >= 0) p.D_s = ds * dt / (dx * dx);
      if (kp > 0) p.k_part = kp;
      if (iv < 1e299) p.delta = -iv;
    }
    p.bc[0] = p.bc[1] = p.bc[2] = MK_BC_CLOSED;
    if (mkm::flow_coupled(model)) {
      // the melt flows in at x = 0 with flow/velocityInlet and out at
      // x = nx - 1 (boundary_vel, mkFluidsUser.cpp:455-617); periodic across
      double nu = -1;
      std::vector<double> vin, acc;
      if (!opt_d(r, "phases/fluid/kinematicViscosity", nu, err) || !opt_v(r, "flow/velocityInlet", vin, err) ||
          !opt_v(r, "flow/acceleration", acc, err))
        return MK_ERR_XML;
      if (nu > 0) p.tau = 3.0 * nu * dt / (dx * dx) + 0.5;
      if (omega_f > 0) p.tau = 1.0 / omega_f;
      for (int a = 0; a < 3; ++a) {
        p.u0[a] = a < (int)vin.size() ? vin[a] * dt / dx : 0.0;
        p.force[a] = (a < (int)acc.size() ? acc[a] : 0.0) + g_lu[a];
      }
      p.rho0 = 1.0;
      p.inlet = 1;
      p.bc[1] = p.bc[2] = MK_BC_PERIODIC;
      p.collision = MK_COLL_TRT;
    }
    if (!read_seeds(r->path("phasechange/seed"), &p, err)) return MK_ERR_XML;
  }

  // --- <b200> lattice-unit overrides
  if (b) {
    if (const mkx::Element* e = b->child("lattice")) {
      const std::string t = lower(mkx::trimmed(e->text));
      if (t == "d3q19")
        p.lattice = MK_D3Q19;
      else if (t == "d3q27")
        p.lattice = MK_D3Q27;
      else {
        err = "<b200><lattice>: unknown '" + t + "'";
        return MK_ERR_XML;
      }
    }
    if (const mkx::Element* e = b->child("collision")) {
      const std::string t = lower(mkx::trimmed(e->text));
      if (t == "bgk")
        p.collision = MK_COLL_BGK;
      else if (t == "trt")
        p.collision = MK_COLL_TRT;
      else if (t == "mrt")
        p.collision = MK_COLL_MRT;
      else {
        err = "<b200><collision>: unknown '" + t + "'";
        return MK_ERR_XML;
      }
    }
    if (const mkx::Element* e = b->child("precision")) {
      const std::string t = lower(mkx::trimmed(e->text));
      if (t == "fp64" || t == "double")
        p.precision = MK_PREC_FP64;
      else if (t == "fp32" || t == "float")
        p.precision = MK_PREC_FP32;
      else if (t == "fp16" || t == "half")
        p.precision = MK_PREC_FP16;
      else if (t == "bf16")
        p.precision = MK_PREC_BF16;
      else {
        err = "<b200><precision>: unknown '" + t + "'";
        return MK_ERR_XML;
      }
    }
    if (const mkx::Element* e = b->child("boundary")) {
      std::string t = e->text;
      std::vector<std::string> toks;
      size_t i = 0;
      while (i < t.size()) {
        while (i < t.size() && isspace((unsigned char)t[i])) ++i;
        size_t j = i;
        while (j < t.size() && !isspace((unsigned char)t[j])) ++j;
        if (j > i) toks.push_back(t.substr(i, j - i));
        i = j;
      }
      if (toks.size() != 3) {
        err = "<b200><boundary> needs 3 values";
        return MK_ERR_XML;
      }
      for (int a = 0; a < 3; ++a) {
        const int bc = parse_bc(toks[a]);
        if (bc < 0) {
          err = "<b200><boundary>: unknown '" + toks[a] + "'";
          return MK_ERR_XML;
        }
        p.bc[a] = bc;
      }
    }
    if (const mkx::Element* e = b->child("anisotropyKind")) {
      const std::string t = lower(mkx::trimmed(e->text));
      if (t == "cubic")
        p.aniso = MK_ANISO_CUBIC;
      else if (t == "cbc")
        p.aniso = MK_ANISO_CBC;
      else if (t == "hcp")
        p.aniso = MK_ANISO_HCP;
      else if (t == "facet")
        p.aniso = MK_ANISO_FACET;
      else {
        err = "<b200><anisotropyKind>: unknown '" + t + "'";
        return MK_ERR_XML;
      }
    }
    std::vector<double> v;
    bool ok = opt_d(b, "eps2", p.eps2, err) && opt_d(b, "magic", p.magic, err) && opt_d(b, "tau", p.tau, err) && opt_d(b, "rho0", p.rho0, err) &&
              opt_d(b, "rhoL", p.rho_l, err) && opt_d(b, "rhoG", p.rho_g, err) && opt_d(b, "tauL", p.tau_l, err) &&
              opt_d(b, "tauG", p.tau_g, err) && opt_d(b, "sigma", p.sigma, err) && opt_d(b, "width", p.width, err) &&
              opt_d(b, "mobility", p.mobility, err) && opt_d(b, "contactAngle", p.contact_angle, err) &&
              opt_d(b, "eps4", p.eps4, err) && opt_d(b, "W0", p.W0, err) && opt_d(b, "lambda", p.lambda, err) &&
              opt_d(b, "delta", p.delta, err) && opt_d(b, "diffusivity", p.D, err) &&
              opt_d(b, "diffSolid", p.D_s, err) && opt_d(b, "partition", p.k_part, err) &&
              opt_d(b, "antiTrapping", p.at_coef, err) && opt_d(b, "grainKappa", p.grain_kappa, err);
    if (!ok) return MK_ERR_XML;
    // tau0 from the thin-interface relation unless given: tau0 = a2 lambda W0^2 / D
    double tau0 = -1;
    if (!opt_d(b, "tau0", tau0, err)) return MK_ERR_XML;
    if (b->child("W0") || b->child("lambda") || b->child("diffusivity") || tau0 > 0)
      p.tau0 = tau0 > 0 ? tau0 : 0.6267 * p.lambda * p.W0 * p.W0 / p.D;
    if (b->child("force")) {
      if (!opt_v(b, "force", v, err)) return MK_ERR_XML;
      for (int a = 0; a < 3; ++a) p.force[a] = a < (int)v.size() ? v[a] : 0.0;
    }
    if (b->child("velocity")) {
      if (!opt_v(b, "velocity", v, err)) return MK_ERR_XML;
      for (int a = 0; a < 3; ++a) p.u0[a] = a < (int)v.size() ? v[a] : 0.0;
    }
    if (b->child("grainVelocity")) {
      if (!opt_v(b, "grainVelocity", v, err)) return MK_ERR_XML;
      for (int a = 0; a < 3; ++a) p.grain_u[a] = a < (int)v.size() ? v[a] : 0.0;
    }
    if (const mkx::Element* e = b->child("wallAxis")) {
      const std::string t = lower(mkx::trimmed(e->text));
      if (t == "x" || t == "0")
        p.wall_axis = 0;
      else if (t == "y" || t == "1")
        p.wall_axis = 1;
      else if (t == "z" || t == "2")
        p.wall_axis = 2;
      else if (t == "none" || t == "-1")
        p.wall_axis = -1;
      else {
        err = "<b200><wallAxis>: unknown '" + t + "'";
        return MK_ERR_XML;
      }
    }
    if (b->child("wallValue")) {
      if (!opt_v(b, "wallValue", v, err)) return MK_ERR_XML;
      if (v.size() != 2) {
        err = "<b200><wallValue> needs 2 values (low plate, high plate)";
        return MK_ERR_XML;
      }
      p.wall_value[0] = v[0];
      p.wall_value[1] = v[1];
    }
    if (b->child("wallVelocity")) {
      if (!opt_v(b, "wallVelocity", v, err)) return MK_ERR_XML;
      if (v.size() != 6) {
        err = "<b200><wallVelocity> needs 6 values (low plate xyz, high plate xyz)";
        return MK_ERR_XML;
      }
      for (int a = 0; a < 3; ++a) {
        p.wall_u[0][a] = v[a];
        p.wall_u[1][a] = v[3 + a];
      }
    }
    if (!opt_d(b, "beta", p.beta, err) || !opt_d(b, "sRef", p.s_ref, err)) return MK_ERR_XML;
    {
      double inl = p.inlet;
      if (!opt_d(b, "inlet", inl, err)) return MK_ERR_XML;
      p.inlet = inl != 0.0 ? 1 : 0;
    }
    if (const mkx::Element* o = b->child("objects")) {
      if (!read_seeds(o, &p, err)) return MK_ERR_XML;
    }
    if (const mkx::Element* rb = b->child("random")) {
      double num = 0, rmin = 8, rmax = 16, gap = 2 * p.width, seed = 0;
      if (!opt_d(rb, "bubbles", num, err) || !opt_d(rb, "radiusMin", rmin, err) ||
          !opt_d(rb, "radiusMax", rmax, err) || !opt_d(rb, "gap", gap, err) || !opt_d(rb, "seed", seed, err))
        return MK_ERR_XML;
      if (!random_bubbles(&p, (int)num, rmin, rmax, gap, (unsigned long long)seed, err)) return MK_ERR_ARG;
    }
  }

  // --- explicit options win
  if (opt) {
    if (opt->precision >= 0) p.precision = opt->precision;
    if (opt->collision >= 0) p.collision = opt->collision;
    if (opt->lattice >= 0) p.lattice = opt->lattice;
    if (opt->magic > 0) p.magic = opt->magic;
  }
  mk_status st = validate_params(&p, err);
  if (st != MK_OK) return st;
  *out = p;
  return MK_OK;
}

// Gas bubbles (phi = 0) in liquid (phi = 1): phi = min_k 1/2 (1 + tanh(2 (d_k - R_k)/W)),
// d_k with the minimum image on periodic axes.  Beyond d - R = 10 W the
// double-precision tanh is exactly 1, so those bubbles are skipped.
static double bubble_phi(const mk_params* p, const double pos[3], const int n3[3]) {
  double ph = 1.0;
  for (int k = 0; k < p->n_objects; ++k) {
    double d2 = 0;
    for (int a = 0; a < 3; ++a) {
      double d = std::fabs(pos[a] - p->obj_center[k][a]);
      if (p->bc[a] == MK_BC_PERIODIC && d > 0.5 * n3[a]) d = n3[a] - d;
      d2 += d * d;
    }
    const double far = p->obj_radius[k] + 10.0 * p->width;
    if (d2 > far * far) continue;
    const double ph_k = 0.5 * (1.0 + std::tanh(2.0 * (std::sqrt(d2) - p->obj_radius[k]) / p->width));
    if (ph_k < ph) ph = ph_k;
  }
  return ph;
}

// Solid seeds (phi = +1) in liquid (phi = -1): the largest of
// -tanh((r_k - R_k)/(sqrt(2) W0)) over the seeds.
// Order parameter of seed k alone: -tanh((r - R) / (sqrt 2 W0)).
static double grain_phi(const mk_params* p, int k, const double pos[3]) {
  double d2 = 0;
  for (int a = 0; a < 3; ++a) {
    const double d = pos[a] - p->obj_center[k][a];
    d2 += d * d;
  }
  return -std::tanh((std::sqrt(d2) - p->obj_radius[k]) / (std::sqrt(2.0) * p->W0));
}

static double seed_phi(const mk_params* p, const double pos[3]) {
  double ph = -1.0;
  for (int k = 0; k < p->n_objects; ++k) {
    double d2 = 0;
    for (int a = 0; a < 3; ++a) {
      const double d = pos[a] - p->obj_center[k][a];
      d2 += d * d;
    }
    const double ph_k = -std::tanh((std::sqrt(d2) - p->obj_radius[k]) / (std::sqrt(2.0) * p->W0));
    if (ph_k > ph) ph = ph_k;
  }
  return ph;
}

mk_status initial_field(const mk_params* p, int field, double* out, size_t ncells, std::string& err) {
  const size_t n = (size_t)p->nx * p->ny * p->nz;
  if (ncells < n) {
    err = "output buffer too small";
    return MK_ERR_ARG;
  }
  const int n3[3] = {p->nx, p->ny, p->nz};
  for (int z = 0; z < p->nz; ++z)
    for (int y = 0; y < p->ny; ++y)
      for (int x = 0; x < p->nx; ++x) {
        const size_t c = (size_t)x + (size_t)p->nx * ((size_t)y + (size_t)p->ny * z);
        const double pos[3] = {(double)x, (double)y, (double)z};
        double v = 0.0;
        switch (field) {
          case MK_FIELD_FLAG:
            v = is_fluid(p, x, y, z) ? MK_FLAG_FLUID : MK_FLAG_WALLS;
            break;
          case MK_FIELD_RHO:
            // the multiphase density follows phi
            v = p->model == MK_MODEL_MULTIPHASE ? p->rho_g + bubble_phi(p, pos, n3) * (p->rho_l - p->rho_g)
                                                : p->rho0;
            break;
          case MK_FIELD_UX:
          case MK_FIELD_UY:
          case MK_FIELD_UZ:
            if (mkm::flow_coupled(p->model)) {
              // u0 scaled by the liquid fraction of the seeded phi
              const double ns = std::min(1.0, std::max(0.0, 0.5 * (1.0 + seed_phi(p, pos))));
              v = (1.0 - ns) * p->u0[field - MK_FIELD_UX];
            } else {
              v = (p->model == MK_MODEL_FLOW || p->model == MK_MODEL_CONVECTION) ? p->u0[field - MK_FIELD_UX] : 0.0;
            }
            break;
          case MK_FIELD_T:
          case MK_FIELD_C:
            if (p->model == MK_MODEL_CONVECTION) {
              // conduction profile between the plates (walls half a cell
              // outside the fluid span) plus one convection-roll mode of
              // amplitude 1e-2 (T_low - T_high) along the first other axis
              const int a = p->wall_axis, b = a == 0 ? 1 : 0;
              const int lo = p->bc[a] == MK_BC_WALLS ? 1 : 0, hi = p->bc[a] == MK_BC_WALLS ? n3[a] - 2 : n3[a] - 1;
              const double H = hi - lo + 1;
              const double sa = std::min(1.0, std::max(0.0, (pos[a] - lo + 0.5) / H));
              const double dT = p->wall_value[0] - p->wall_value[1];
              v = p->wall_value[0] - dT * sa +
                  1e-2 * dT * std::sin(M_PI * sa) * std::cos(2.0 * M_PI * pos[b] / n3[b]);
            } else {
              v = -p->delta;
            }
            break;
          case MK_FIELD_PRESSURE:
          case MK_FIELD_DPHI:
            v = 0.0;
            break;
          case MK_FIELD_GRAIN: {
            int best = 0;
            double bd = 1e300;
            for (int k = 0; k < p->n_objects; ++k) {
              double d2 = 0;
              for (int a = 0; a < 3; ++a) {
                const double d = pos[a] - p->obj_center[k][a];
                d2 += d * d;
              }
              if (d2 < bd) {
                bd = d2;
                best = k;
              }
            }
            v = mkm::dendrite(p->model) ? best : 0;
            if (p->model == MK_MODEL_MULTIGRAIN) {
              // the grain whose order parameter is largest (ties to the lower index)
              double bp = -1e300;
              for (int k = 0; k < p->n_objects; ++k) {
                const double g = grain_phi(p, k, pos);
                if (g > bp) {
                  bp = g;
                  v = k;
                }
              }
            }
            break;
          }
          case MK_FIELD_PHI:
            if (p->model == MK_MODEL_MULTIPHASE) {
              v = bubble_phi(p, pos, n3);
            } else if (p->model == MK_MODEL_FLOW || p->model == MK_MODEL_CONVECTION) {
              v = 0.0;
            } else if (p->model == MK_MODEL_MULTIGRAIN) {
              // aggregate phi = (N - 1) + sum_j phi_j (mkFluidsUser.cpp:162-168)
              v = p->n_objects - 1.0;
              for (int k = 0; k < p->n_objects; ++k) v += grain_phi(p, k, pos);
            } else {
              v = seed_phi(p, pos);
            }
            break;
          default:
            err = "unknown field";
            return MK_ERR_ARG;
        }
        out[c] = v;
      }
  return MK_OK;
}

mk_status ensemble_case(unsigned long long seed, int n, int precision, mk_params* out, std::string& err) {
  if (n < 1 || n > 4096) {
    err = "ensemble size out of range";
    return MK_ERR_ARG;
  }
  SplitMix64 rng(seed);
  const int edges[5] = {48, 64, 80, 96, 128};
  for (int d = 0; d < n; ++d) {
    mk_params p;
    default_params(&p);
    p.model = MK_MODEL_SOLUTAL_DENDRITE;
    p.precision = precision;
    const int L = edges[rng.next() % 5];
    p.nx = p.ny = p.nz = L;
    p.bc[0] = p.bc[1] = p.bc[2] = MK_BC_CLOSED;
    p.max_loops = 3000;
    p.eps4 = 0.02 + 0.04 * rng.uniform();
    p.k_part = 0.15;
    p.D = 0.1;
    p.D_s = 1e-4;
    p.W0 = 1.5;
    p.lambda = 10.0;
    p.delta = 0.55;
    p.tau0 = 0.6267 * p.lambda * p.W0 * p.W0 / p.D;
    p.n_objects = 1 + (int)(rng.next() % 6);
    for (int s = 0; s < p.n_objects; ++s) {
      const double R = 4.0 + 4.0 * rng.uniform();
      for (int a = 0; a < 3; ++a) p.obj_center[s][a] = (R + 2.0) + (L - 1 - 2.0 * (R + 2.0)) * rng.uniform();
      p.obj_radius[s] = R;
      // uniformly random orientation (Shoemake's uniform quaternion) as ZYX angles
      const double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
      const double qx = std::sqrt(1 - u1) * std::sin(2 * M_PI * u2), qy = std::sqrt(1 - u1) * std::cos(2 * M_PI * u2);
      const double qz = std::sqrt(u1) * std::sin(2 * M_PI * u3), qw = std::sqrt(u1) * std::cos(2 * M_PI * u3);
      const double R00 = 1 - 2 * (qy * qy + qz * qz), R10 = 2 * (qx * qy + qz * qw), R20 = 2 * (qx * qz - qy * qw);
      const double R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
      const double r2d = 180.0 / M_PI;
      p.obj_angle[s][0] = std::atan2(R21, R22) * r2d;
      p.obj_angle[s][1] = -std::asin(std::max(-1.0, std::min(1.0, R20))) * r2d;
      p.obj_angle[s][2] = std::atan2(R10, R00) * r2d;
    }
    p.rng_seed = seed;
    mk_status st = validate_params(&p, err);
    if (st != MK_OK) return st;
    out[d] = p;
  }
  return MK_OK;
}

unsigned long long params_hash(const mk_params* p) {
  // FNV-1a over the bytes of the parameter block (precision excluded so a
  // checkpoint can be restored at another storage precision).
  mk_params q = *p;
  q.precision = 0;
  q.max_loops = 0;
  q.max_frames = 0;
  const unsigned char* b = reinterpret_cast<const unsigned char*>(&q);
  unsigned long long h = 1469598103934665603ULL;
  for (size_t i = 0; i < sizeof(q); ++i) {
    h ^= b[i];
    h *= 1099511628211ULL;
  }
  return h;
}

}  // namespace mkc
