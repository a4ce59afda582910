// mk_oracle.cpp — TEST INFRASTRUCTURE ONLY (see mk_oracle.hpp for the model
// definitions and the parity status).  FP64, OpenMP, SoA, two-array pull
// streaming: propagate writes the post-stream ("hlp") populations from the
// neighbours' post-collision ("out") populations, then relaxation writes
// "out" again — the order of MaterKit/src/mkFluidsUser.cpp:68-299.
#include "mk_oracle.hpp"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- lattices
// Velocity set of MaterKit/inc/mkLattice.h:33-35 (e, c, inv), in 3D.
const int E27[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},  {0, 0, 1},  {0, 0, -1},
    {1, 1, 0},   {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},  {1, 0, 1},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {0, 1, 1},   {0, -1, -1}, {0, 1, -1},  {0, -1, 1},  {1, 1, 1},  {-1, -1, -1},
    {1, 1, -1},  {-1, -1, 1}, {1, -1, 1},  {-1, 1, -1}, {-1, 1, 1},  {1, -1, -1}};

inline int inv_dir(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

double weight(int Q, int i) {
  if (Q == 7) return i == 0 ? 0.25 : 0.125;
  if (Q == 19) {
    if (i == 0) return 1.0 / 3.0;
    if (i <= 6) return 1.0 / 18.0;
    return 1.0 / 36.0;
  }
  // D3Q27
  if (i == 0) return 8.0 / 27.0;
  if (i <= 6) return 2.0 / 27.0;
  if (i <= 18) return 1.0 / 54.0;
  return 1.0 / 216.0;
}

// d'Humieres et al. (2002) orthogonal D3Q19 moment basis, the "M" of
// MaterKit/inc/mkLattice.h:89 for the 3D lattice.
struct Mrt19 {
  double M[19][19];
  double inv_norm[19];
  Mrt19() {
    for (int i = 0; i < 19; ++i) {
      const double ex = E27[i][0], ey = E27[i][1], ez = E27[i][2];
      const double e2 = ex * ex + ey * ey + ez * ez;
      M[0][i] = 1.0;
      M[1][i] = 19.0 * e2 - 30.0;
      M[2][i] = (21.0 * e2 * e2 - 53.0 * e2 + 24.0) / 2.0;
      M[3][i] = ex;
      M[4][i] = (5.0 * e2 - 9.0) * ex;
      M[5][i] = ey;
      M[6][i] = (5.0 * e2 - 9.0) * ey;
      M[7][i] = ez;
      M[8][i] = (5.0 * e2 - 9.0) * ez;
      M[9][i] = 3.0 * ex * ex - e2;
      M[10][i] = (3.0 * e2 - 5.0) * (3.0 * ex * ex - e2);
      M[11][i] = ey * ey - ez * ez;
      M[12][i] = (3.0 * e2 - 5.0) * (ey * ey - ez * ez);
      M[13][i] = ex * ey;
      M[14][i] = ey * ez;
      M[15][i] = ex * ez;
      M[16][i] = (ey * ey - ez * ez) * ex;
      M[17][i] = (ez * ez - ex * ex) * ey;
      M[18][i] = (ex * ex - ey * ey) * ez;
    }
    for (int k = 0; k < 19; ++k) {
      double n = 0;
      for (int i = 0; i < 19; ++i) n += M[k][i] * M[k][i];
      inv_norm[k] = 1.0 / n;
    }
  }
};
const Mrt19 MRT;

// Relaxation rates; index 9,11,13,14,15 carry the shear rate.
void mrt_rates(double s_nu, double S[19]) {
  for (int k = 0; k < 19; ++k) S[k] = 1.0;
  S[1] = 1.19;
  S[2] = 1.4;
  S[4] = S[6] = S[8] = 1.2;
  S[10] = S[12] = 1.4;
  S[16] = S[17] = S[18] = 1.98;
  S[9] = S[11] = S[13] = S[14] = S[15] = s_nu;
}

// f* = f - Mi [ S (M(f - feq)) - (I - S/2) M F ]
void mrt_collide(double* f, const double* feq, const double* F, double s_nu) {
  double S[19];
  mrt_rates(s_nu, S);
  double d[19], fneq[19];
  for (int i = 0; i < 19; ++i) fneq[i] = f[i] - feq[i];
  for (int k = 0; k < 19; ++k) {
    double mn = 0, mf = 0;
    for (int i = 0; i < 19; ++i) {
      mn += MRT.M[k][i] * fneq[i];
      mf += MRT.M[k][i] * F[i];
    }
    d[k] = (S[k] * mn - (1.0 - 0.5 * S[k]) * mf) * MRT.inv_norm[k];
  }
  for (int i = 0; i < 19; ++i) {
    double s = 0;
    for (int k = 0; k < 19; ++k) s += MRT.M[k][i] * d[k];
    f[i] -= s;
  }
}

inline double feq2(double w, double eu, double uu) { return w * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu); }

// Rotation "rotate-order ZYX" of the seed angles (BoltzTechs - thermal.xml:71-75):
// R = Rz(az) Ry(ay) Rx(ax), angles in degrees.  Columns are the crystal axes.
void rotation_zyx(const double ang_deg[3], double R[3][3]) {
  const double d2r = M_PI / 180.0;
  const double ax = ang_deg[0] * d2r, ay = ang_deg[1] * d2r, az = ang_deg[2] * d2r;
  const double cx = cos(ax), sx = sin(ax), cy = cos(ay), sy = sin(ay), cz = cos(az), sz = sin(az);
  // Rz*Ry*Rx
  R[0][0] = cz * cy;
  R[0][1] = cz * sy * sx - sz * cx;
  R[0][2] = cz * sy * cx + sz * sx;
  R[1][0] = sz * cy;
  R[1][1] = sz * sy * sx + cz * cx;
  R[1][2] = sz * sy * cx - cz * sx;
  R[2][0] = -sy;
  R[2][1] = cy * sx;
  R[2][2] = cy * cx;
}

}  // namespace

// Model families: the flow + dendrite models carry a flow lattice with porous
// bounce-back and inflow / outflow faces; the solutal models a U-lattice.
static bool flow_coupled(int model) { return model == MK_MODEL_FLOW_DENDRITE || model == MK_MODEL_FLOW_SOLUTAL; }
static bool solutal(int model) { return model == MK_MODEL_SOLUTAL_DENDRITE || model == MK_MODEL_FLOW_SOLUTAL; }

// ------------------------------------------------------------------ state
struct orc_state {
  mk_params p;
  int nx, ny, nz;
  int64_t n;
  int64_t step;
  int Qf;  // populations of lattice 0 (flow / phase field)
  int Qs;  // populations of lattice 1 (AC h / thermal / solutal), 0 if none
  std::vector<uint8_t> flag;
  std::vector<double> f_out, f_hlp;  // lattice 0, [q][cell]
  std::vector<double> s_out, s_hlp;  // lattice 1
  std::vector<double> phi, phi_prev, temp, conc, conc_prev;
  int Qw = 0;                        // flow lattice of the flow + dendrite model, 0 if none
  std::vector<double> w_out, w_hlp;  // its populations
  std::vector<double> vel;           // its velocity, 3 per cell (advects the thermal lattice)
  int Ng = 0;                                   // multigrain: number of grain order parameters
  std::vector<std::vector<double>> gj_out, gj_hlp;  // their D3Q19 lattices, one [q][cell] array per grain
  std::vector<double> phij;                     // their order parameters, [grain][cell]
  std::vector<int> grain;
  std::vector<double> rot;  // 9 per object (R, columns = crystal axes)
  std::vector<uint8_t> pend;  // multiphase: cells to turn solid (orc_update_geometry)
  int pend_set = 0;
};

namespace {

inline int64_t cidx(const orc_state* s, int x, int y, int z) {
  return (int64_t)x + (int64_t)s->nx * ((int64_t)y + (int64_t)s->ny * z);
}

// Neighbour of (x,y,z) along (dx,dy,dz), or -1 when it is solid or outside a
// closed face.  Periodic axes wrap like mkFluidsLBM::neighbor (mkFluidsLBM.h:82).
inline int64_t nbr(const orc_state* s, int x, int y, int z, int dx, int dy, int dz) {
  int c[3] = {x + dx, y + dy, z + dz};
  const int n[3] = {s->nx, s->ny, s->nz};
  for (int a = 0; a < 3; ++a) {
    if (c[a] < 0 || c[a] >= n[a]) {
      if (s->p.bc[a] == MK_BC_PERIODIC)
        c[a] = (c[a] + n[a]) % n[a];
      else
        return -1;
    }
  }
  int64_t j = cidx(s, c[0], c[1], c[2]);
  return s->flag[j] == MK_FLAG_FLUID ? j : -1;
}

// Propagate with half-way bounce-back: hlp_i(x) = out_i(x - e_i), or
// out_inv(i)(x) when x - e_i is not fluid (MaterKit/src/mkFluidsUser.cpp:77-97).
void propagate(const orc_state* s, int Q, const std::vector<double>& out, std::vector<double>& hlp) {
  const int64_t n = s->n;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        if (s->flag[c] != MK_FLAG_FLUID) continue;
        for (int i = 0; i < Q; ++i) {
          const int64_t src = nbr(s, x, y, z, -E27[i][0], -E27[i][1], -E27[i][2]);
          hlp[(int64_t)i * n + c] = src >= 0 ? out[(int64_t)i * n + src] : out[(int64_t)inv_dir(i) * n + c];
        }
      }
}

// Plate corrections of a bounced population (wall_axis >= 0): the flow sees
// a wall moving with wall_u (Ladd: + 6 w rho0 e.u_w, bdyCouette /
// boundary_vel, mkFluidsLBM.h:61-63), a scalar sees the Dirichlet value
// wall_value (anti-bounce-back -t + 2 w T_w, bdy_constT / bdy_RBC,
// mkThermalField.h:37-39).  A population is bounced at the low (high) plate
// when the upwind cell lies below (above) the fluid span of wall_axis.
enum { kWallFlow = 1, kWallScalar = 2 };

// Plate side (0 low, 1 high) of the upwind cell x - e_i, or -1.
inline int plate_side(const orc_state* s, int x, int y, int z, int i) {
  const int a = s->p.wall_axis;
  if (a < 0 || E27[i][a] == 0) return -1;
  const int c3[3] = {x, y, z};
  const int n3[3] = {s->nx, s->ny, s->nz};
  const int p = c3[a] - E27[i][a];
  const int lo = s->p.bc[a] == MK_BC_WALLS ? 1 : 0, hi = s->p.bc[a] == MK_BC_WALLS ? n3[a] - 2 : n3[a] - 1;
  return p < lo ? 0 : (p > hi ? 1 : -1);
}

void propagate_bc(const orc_state* s, int Q, const std::vector<double>& out, std::vector<double>& hlp, int kind) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        if (s->flag[c] != MK_FLAG_FLUID) continue;
        for (int i = 0; i < Q; ++i) {
          const int64_t src = nbr(s, x, y, z, -E27[i][0], -E27[i][1], -E27[i][2]);
          if (src >= 0) {
            hlp[(int64_t)i * n + c] = out[(int64_t)i * n + src];
            continue;
          }
          double v = out[(int64_t)inv_dir(i) * n + c];
          const int side = plate_side(s, x, y, z, i);
          if (side >= 0) {
            const double w = weight(Q, i);
            if (kind == kWallFlow) {
              const double* uw = p.wall_u[side];
              v += 6.0 * w * p.rho0 * (E27[i][0] * uw[0] + E27[i][1] * uw[1] + E27[i][2] * uw[2]);
            } else {
              v = -v + 2.0 * w * p.wall_value[side];
            }
          }
          hlp[(int64_t)i * n + c] = v;
        }
      }
}

// Isotropic gradient and Laplacian of a scalar with D3Q19 weights.  `wall`
// gives the value substituted at a non-fluid neighbour.
template <class WallFn>
void grad_lap(const orc_state* s, const std::vector<double>& f, int x, int y, int z, WallFn wall, double g[3],
              double* lap) {
  const int64_t c = cidx(s, x, y, z);
  const double f0 = f[c];
  g[0] = g[1] = g[2] = 0;
  double l = 0;
  for (int i = 1; i < 19; ++i) {
    const int64_t j = nbr(s, x, y, z, E27[i][0], E27[i][1], E27[i][2]);
    const double fn = j >= 0 ? f[j] : wall(f0);
    const double w = weight(19, i);
    g[0] += w * E27[i][0] * fn;
    g[1] += w * E27[i][1] * fn;
    g[2] += w * E27[i][2] * fn;
    l += w * (fn - f0);
  }
  g[0] *= 3.0;
  g[1] *= 3.0;
  g[2] *= 3.0;
  *lap = 6.0 * l;
}

// ------------------------------------------------------------ FLOW model
void flow_force(const orc_state* s, double F[3]) {
  F[0] = s->p.force[0];
  F[1] = s->p.force[1];
  F[2] = s->p.force[2];
}

// Collision of one cell's Q populations with the Guo force F
// (mkNode::collision_BGK/TRT/MRT*, mkNode.h:74-87); returns u.
void flow_collide(int Q, int coll, double om, double om_m, double* f, const double F[3], double u[3]) {
  double feq[27], Fi[27];
  double rho = 0, j[3] = {0, 0, 0};
  for (int i = 0; i < Q; ++i) {
    rho += f[i];
    j[0] += E27[i][0] * f[i];
    j[1] += E27[i][1] * f[i];
    j[2] += E27[i][2] * f[i];
  }
  for (int a = 0; a < 3; ++a) u[a] = (j[a] + 0.5 * F[a]) / rho;
  const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const double uF = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
  for (int i = 0; i < Q; ++i) {
    const double w = weight(Q, i);
    const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
    const double eF = E27[i][0] * F[0] + E27[i][1] * F[1] + E27[i][2] * F[2];
    feq[i] = rho * feq2(w, eu, uu);
    Fi[i] = w * (3.0 * eF + 9.0 * eu * eF - 3.0 * uF);
  }
  if (coll == MK_COLL_BGK) {
    for (int i = 0; i < Q; ++i) f[i] += -om * (f[i] - feq[i]) + (1.0 - 0.5 * om) * Fi[i];
  } else if (coll == MK_COLL_TRT) {
    double fo[27];
    for (int i = 0; i < Q; ++i) {
      const int k = inv_dir(i);
      const double fp = 0.5 * (f[i] + f[k]), fm = 0.5 * (f[i] - f[k]);
      const double ep = 0.5 * (feq[i] + feq[k]), em = 0.5 * (feq[i] - feq[k]);
      const double Fp = 0.5 * (Fi[i] + Fi[k]), Fm = 0.5 * (Fi[i] - Fi[k]);
      fo[i] = f[i] - om * (fp - ep) - om_m * (fm - em) + (1.0 - 0.5 * om) * Fp + (1.0 - 0.5 * om_m) * Fm;
    }
    for (int i = 0; i < Q; ++i) f[i] = fo[i];
  } else {
    mrt_collide(f, feq, Fi, om);
  }
}

void flow_step(orc_state* s) {
  const int Q = s->Qf;
  const int64_t n = s->n;
  propagate_bc(s, Q, s->f_out, s->f_hlp, kWallFlow);
  double F[3];
  flow_force(s, F);
  const double tau = s->p.tau;
  const double om = 1.0 / tau;
  const double tau_m = 0.5 + s->p.magic / (tau - 0.5);
  const double om_m = 1.0 / tau_m;
  const int coll = s->p.collision;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    double f[27], u[3];
    for (int i = 0; i < Q; ++i) f[i] = s->f_hlp[(int64_t)i * n + c];
    flow_collide(Q, coll, om, om_m, f, F, u);
    for (int i = 0; i < Q; ++i) s->f_out[(int64_t)i * n + c] = f[i];
  }
}

// ------------------------------------------------------ CONVECTION model
// Rayleigh-Benard / natural convection (bdy_RBC, bdy_constT, mkThermalField
// relaxation with advection, Thermal_NusseltRBC: mkThermalField.h:33-40,
// mkFluidsLBM.h:59-68, mkFluidsUser.cpp:362-392): the flow lattice with the
// Boussinesq force F = -rho0 beta (T - T_ref) g (g = force) and a D3Q7
// advection-diffusion lattice t_eq = w T (1 + 4 e.u), omega_T = 1/(4 D + 1/2);
// both streamed with the plate corrections of propagate_bc.
void convection_step(orc_state* s) {
  const int Q = s->Qf;
  const int64_t n = s->n;
  const mk_params& p = s->p;
  propagate_bc(s, Q, s->f_out, s->f_hlp, kWallFlow);
  propagate_bc(s, 7, s->s_out, s->s_hlp, kWallScalar);
  const double om = 1.0 / p.tau;
  const double om_m = 1.0 / (0.5 + p.magic / (p.tau - 0.5));
  const double om_t = 1.0 / (4.0 * p.D + 0.5);
  const double bg[3] = {-p.rho0 * p.beta * p.force[0], -p.rho0 * p.beta * p.force[1], -p.rho0 * p.beta * p.force[2]};
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    double T = 0;
    for (int i = 0; i < 7; ++i) T += s->s_hlp[(int64_t)i * n + c];
    const double F[3] = {bg[0] * (T - p.s_ref), bg[1] * (T - p.s_ref), bg[2] * (T - p.s_ref)};
    double f[27], u[3];
    for (int i = 0; i < Q; ++i) f[i] = s->f_hlp[(int64_t)i * n + c];
    flow_collide(Q, p.collision, om, om_m, f, F, u);
    for (int i = 0; i < Q; ++i) s->f_out[(int64_t)i * n + c] = f[i];
    for (int i = 0; i < 7; ++i) {
      const double ti = s->s_hlp[(int64_t)i * n + c];
      const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
      s->s_out[(int64_t)i * n + c] = ti - om_t * (ti - weight(7, i) * T * (1.0 + 4.0 * eu));
    }
    s->temp[c] = T;
  }
}

// --------------------------------------------------------- MULTIPHASE model
struct MpConst {
  double beta, kappa, tau_h, om_h, cos_t, W;
};

MpConst mp_const(const mk_params& p) {
  MpConst k;
  k.beta = 12.0 * p.sigma / p.width;
  k.kappa = 1.5 * p.sigma * p.width;
  k.tau_h = 3.0 * p.mobility + 0.5;
  k.om_h = 1.0 / k.tau_h;
  k.cos_t = cos(p.contact_angle * M_PI / 180.0);
  k.W = p.width;
  return k;
}

// Force, density and phi gradient of a fluid cell at the stored phi.
struct MpLocal {
  double phi, rho, gphi[3], F[3];
};

MpLocal mp_local(const orc_state* s, const MpConst& k, int x, int y, int z, double pstar) {
  MpLocal L;
  const int64_t c = cidx(s, x, y, z);
  L.phi = s->phi[c];
  const double coef = 4.0 * k.cos_t / k.W;
  double lap;
  grad_lap(
      s, s->phi, x, y, z, [&](double p0) { return p0 + coef * p0 * (1.0 - p0); }, L.gphi, &lap);
  const mk_params& p = s->p;
  const double drho = p.rho_l - p.rho_g;
  L.rho = p.rho_g + L.phi * drho;
  const double mu = 4.0 * k.beta * L.phi * (L.phi - 1.0) * (L.phi - 0.5) - k.kappa * lap;
  for (int a = 0; a < 3; ++a)
    L.F[a] = mu * L.gphi[a] + L.rho * p.force[a] - pstar * (1.0 / 3.0) * drho * L.gphi[a];
  return L;
}

void mp_step(orc_state* s) {
  const int64_t n = s->n;
  propagate(s, 19, s->f_out, s->f_hlp);  // g (pressure / velocity)
  propagate(s, 19, s->s_out, s->s_hlp);  // h (Allen-Cahn)
  // phi = sum h over all fluid cells before any gradient is taken.
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    double ph = 0;
    for (int i = 0; i < 19; ++i) ph += s->s_hlp[(int64_t)i * n + c];
    s->phi[c] = ph;
  }
  const MpConst k = mp_const(s->p);
  const mk_params& p = s->p;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        if (s->flag[c] != MK_FLAG_FLUID) continue;
        double g[19], h[19], geq[19], Fb[19];
        double pstar = 0, j[3] = {0, 0, 0};
        for (int i = 0; i < 19; ++i) {
          g[i] = s->f_hlp[(int64_t)i * n + c];
          h[i] = s->s_hlp[(int64_t)i * n + c];
          pstar += g[i];
          j[0] += E27[i][0] * g[i];
          j[1] += E27[i][1] * g[i];
          j[2] += E27[i][2] * g[i];
        }
        const MpLocal L = mp_local(s, k, x, y, z, pstar);
        double u[3];
        for (int a = 0; a < 3; ++a) u[a] = j[a] + L.F[a] / (2.0 * L.rho);
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double uF = u[0] * L.F[0] + u[1] * L.F[1] + u[2] * L.F[2];
        const double tau = p.tau_g + L.phi * (p.tau_l - p.tau_g);
        const double gn = sqrt(L.gphi[0] * L.gphi[0] + L.gphi[1] * L.gphi[1] + L.gphi[2] * L.gphi[2]);
        double nrm[3];
        for (int a = 0; a < 3; ++a) nrm[a] = L.gphi[a] / (gn + 1e-12);
        const double lam = 4.0 * L.phi * (1.0 - L.phi) / k.W;
        for (int i = 0; i < 19; ++i) {
          const double w = weight(19, i);
          const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
          const double eF = E27[i][0] * L.F[0] + E27[i][1] * L.F[1] + E27[i][2] * L.F[2];
          const double en = E27[i][0] * nrm[0] + E27[i][1] * nrm[1] + E27[i][2] * nrm[2];
          geq[i] = w * (pstar + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
          Fb[i] = w * (3.0 * eF + 9.0 * eu * eF - 3.0 * uF) / L.rho;
          const double heq = L.phi * feq2(w, eu, uu);
          h[i] += -k.om_h * (h[i] - heq) + (1.0 - 0.5 * k.om_h) * w * lam * en;
        }
        mrt_collide(g, geq, Fb, 1.0 / tau);
        for (int i = 0; i < 19; ++i) {
          s->f_out[(int64_t)i * n + c] = g[i];
          s->s_out[(int64_t)i * n + c] = h[i];
        }
      }
}

// ------------------------------------------------------ DENDRITE models
// Nearest-seed grain of a cell (ties to the lower index).
int nearest_seed(const mk_params& p, double x, double y, double z) {
  int best = 0;
  double bd = 1e300;
  for (int k = 0; k < p.n_objects; ++k) {
    const double dx = x - p.obj_center[k][0], dy = y - p.obj_center[k][1], dz = z - p.obj_center[k][2];
    const double d = dx * dx + dy * dy + dz * dz;
    if (d < bd) {
      bd = d;
      best = k;
    }
  }
  return best;
}

// a(n) and its gradient da/dn of the interfacial anisotropy kinds, n the
// crystal-frame unit normal (mkPhaseField::anisotropy / _cbc / _hcp / _facet,
// mkPhaseField.h:61-64; forms of the mk_anisotropy enum in include/mkb200.h):
//   cubic  Karma & Rappel 1998 four-fold: 1 - 3 e4 + 4 e4 s4, s4 = sum n^4
//   cbc    two cubic harmonics (Haxhimali et al., Nat. Mater. 5 (2006) 660):
//          1 + e4 (s4 - 3/5) + e2 (3 s4 + 66 nx^2 ny^2 nz^2 - 17/7)
//   hcp    six-fold in the basal plane plus a c-axis term:
//          1 + e4 Re (nx + i ny)^6 + e2 (2 nz^2 - 1)
//   facet  regularised cusps at the cube directions (the |n_q| faceting form
//          of Eggleston, McFadden & Voorhees, Physica D 150 (2001) 91):
//          1 + e4 (sum sqrt(n_q^2 + e2^2) - sqrt(1 + e2^2) - 2 e2)
void aniso_function(int kind, double e4, double e2, const double n[3], double* a_out, double g[3]) {
  const double x = n[0], y = n[1], z = n[2];
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  double a;
  switch (kind) {
    case MK_ANISO_CBC: {
      const double s4 = x2 * x2 + y2 * y2 + z2 * z2, s6 = x2 * y2 * z2;
      a = 1.0 + e4 * (s4 - 0.6) + e2 * (3.0 * s4 + 66.0 * s6 - 17.0 / 7.0);
      g[0] = 4.0 * e4 * x2 * x + e2 * (12.0 * x2 * x + 132.0 * x * y2 * z2);
      g[1] = 4.0 * e4 * y2 * y + e2 * (12.0 * y2 * y + 132.0 * y * x2 * z2);
      g[2] = 4.0 * e4 * z2 * z + e2 * (12.0 * z2 * z + 132.0 * z * x2 * y2);
      break;
    }
    case MK_ANISO_HCP: {
      const double c6 = x2 * x2 * x2 - 15.0 * x2 * x2 * y2 + 15.0 * x2 * y2 * y2 - y2 * y2 * y2;
      a = 1.0 + e4 * c6 + e2 * (2.0 * z2 - 1.0);
      g[0] = 6.0 * e4 * (x2 * x2 * x - 10.0 * x2 * x * y2 + 5.0 * x * y2 * y2);
      g[1] = -6.0 * e4 * (5.0 * x2 * x2 * y - 10.0 * x2 * y2 * y + y2 * y2 * y);
      g[2] = 4.0 * e2 * z;
      break;
    }
    case MK_ANISO_FACET: {
      const double rx = sqrt(x2 + e2 * e2), ry = sqrt(y2 + e2 * e2), rz = sqrt(z2 + e2 * e2);
      a = 1.0 + e4 * (rx + ry + rz - sqrt(1.0 + e2 * e2) - 2.0 * e2);
      g[0] = e4 * x / rx;
      g[1] = e4 * y / ry;
      g[2] = e4 * z / rz;
      break;
    }
    default: {
      const double s4 = x2 * x2 + y2 * y2 + z2 * z2;
      a = 1.0 - 3.0 * e4 + 4.0 * e4 * s4;
      g[0] = 16.0 * e4 * x2 * x;
      g[1] = 16.0 * e4 * y2 * y;
      g[2] = 16.0 * e4 * z2 * z;
      break;
    }
  }
  *a_out = a;
}

// Anisotropy of a cell: returns a(n) and the lab-frame vector N of the
// anisotropic flux  div(|grad phi|^2 a da/d(grad phi)),
// N_c = |grad phi| a (da/dn - n (n . da/dn)) in the crystal frame, from the
// lab gradient and the grain's rotation (columns = crystal axes).
void anisotropy(const double* R, int kind, double e4, double e2, const double g[3], double* a_out, double N[3]) {
  const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  const double inv = 1.0 / (gn + 1e-12);
  const double nl[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
  double nc[3];
  for (int a = 0; a < 3; ++a) nc[a] = R[0 * 3 + a] * nl[0] + R[1 * 3 + a] * nl[1] + R[2 * 3 + a] * nl[2];
  double a, da[3];
  aniso_function(kind, e4, e2, nc, &a, da);
  const double ndg = nc[0] * da[0] + nc[1] * da[1] + nc[2] * da[2];
  double Nc[3];
  for (int k = 0; k < 3; ++k) Nc[k] = gn * a * (da[k] - nc[k] * ndg);
  for (int a2 = 0; a2 < 3; ++a2) N[a2] = R[a2 * 3 + 0] * Nc[0] + R[a2 * 3 + 1] * Nc[1] + R[a2 * 3 + 2] * Nc[2];
  *a_out = a;
}

// Thermal relaxation of the streamed D3Q7 lattice with latent heat (1/2)
// dphi (mkThermalField::relaxation, mkThermalField.h:34); with a flow lattice
// the equilibrium is advected, w T (1 + 4 e.u) (getTEquPDFs).
void thermal_relax(orc_state* s) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
  const double om_t = 1.0 / (4.0 * p.D + 0.5);
  const bool adv = !s->vel.empty();
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    double T = 0;
    for (int i = 0; i < 7; ++i) T += s->s_hlp[(int64_t)i * n + c];
    const double lat = 0.5 * (s->phi[c] - s->phi_prev[c]);
    for (int i = 0; i < 7; ++i) {
      const double w = weight(7, i);
      const double eu = adv ? E27[i][0] * s->vel[3 * c] + E27[i][1] * s->vel[3 * c + 1] + E27[i][2] * s->vel[3 * c + 2]
                            : 0.0;
      const double ti = s->s_hlp[(int64_t)i * n + c];
      s->s_out[(int64_t)i * n + c] = ti - om_t * (ti - w * T * (1.0 + 4.0 * eu)) + w * lat;
    }
    s->temp[c] = T;
  }
}

void thermal_dendrite_step(orc_state* s) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
  // 1. phase-field propagate, phi^n = sum g (MaterKit/src/mkFluidsUser.cpp:147-172).
  propagate(s, 7, s->f_out, s->f_hlp);
  std::swap(s->phi_prev, s->phi);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) {
      s->phi[c] = s->phi_prev[c];
      continue;
    }
    double ph = 0;
    for (int i = 0; i < 7; ++i) ph += s->f_hlp[(int64_t)i * n + c];
    s->phi[c] = ph;
  }
  // 2. phase-field relaxation with anisotropy and thermal coupling.
  const double D0 = p.W0 * p.W0 / p.tau0;
  const double om_g = 1.0 / (4.0 * D0 + 0.5);
  const double cs2 = 0.25;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        if (s->flag[c] != MK_FLAG_FLUID) continue;
        double gr[3], lap;
        grad_lap(
            s, s->phi, x, y, z, [](double p0) { return p0; }, gr, &lap);
        double a, N[3];
        anisotropy(&s->rot[9 * s->grain[c]], p.aniso, p.eps4, p.eps2, gr, &a, N);
        const double ph = s->phi[c];
        const double dphi = ph - s->phi_prev[c];
        const double one_m = 1.0 - ph * ph;
        const double src = (ph - ph * ph * ph - p.lambda * s->temp[c] * one_m * one_m) / p.tau0 + (1.0 - a * a) * dphi;
        double B[3];
        for (int k = 0; k < 3; ++k) B[k] = -cs2 * ((a * a - 1.0) * gr[k] + N[k]);
        for (int i = 0; i < 7; ++i) {
          const double w = weight(7, i);
          const double eB = E27[i][0] * B[0] + E27[i][1] * B[1] + E27[i][2] * B[2];
          const double gi = s->f_hlp[(int64_t)i * n + c];
          s->f_out[(int64_t)i * n + c] = gi - om_g * (gi - w * ph) + (1.0 - 0.5 * om_g) * w * eB / cs2 + w * src;
        }
      }
  propagate(s, 7, s->s_out, s->s_hlp);
  if (solutal(p.model)) {
    // 3'. solutal propagate + relaxation: variable diffusivity, anti-trapping
    // current in the equilibrium's first moment, rejection and lagged capacity;
    // with a flow lattice the first moment also carries the advective flux U u
    // (the equilibrium w U (1 + 4 e.u) of the liquid).
    const double k = p.k_part;
    const bool adv = !s->vel.empty();
#pragma omp parallel for schedule(static)
    for (int z = 0; z < s->nz; ++z)
      for (int y = 0; y < s->ny; ++y)
        for (int x = 0; x < s->nx; ++x) {
          const int64_t c = cidx(s, x, y, z);
          if (s->flag[c] != MK_FLAG_FLUID) continue;
          double U = 0;
          for (int i = 0; i < 7; ++i) U += s->s_hlp[(int64_t)i * n + c];
          const double ph = s->phi[c];
          const double dphi = ph - s->phi_prev[c];
          double gr[3], lap;
          grad_lap(
              s, s->phi, x, y, z, [](double p0) { return p0; }, gr, &lap);
          // capacity c(phi) applied by dividing the local diffusivity, the
          // anti-trapping flux and the rejection source
          const double cap = (1.0 + k - (1.0 - k) * ph) * 0.5;
          const double gn = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
          // the current is linear in n, so its normal is regularised at 1e-6
          // (not 1e-12) to keep rounding noise where grad phi vanishes out of it
          const double f = -p.at_coef * p.W0 * (1.0 + (1.0 - k) * U) * dphi / ((gn + 1e-6) * cap);
          const double jat[3] = {f * gr[0], f * gr[1], f * gr[2]};
          const double D = (p.D * (1.0 - ph) * 0.5 + p.D_s * (1.0 + ph) * 0.5) / cap;
          const double om = 1.0 / (4.0 * D + 0.5);
          const double src = 0.5 * (1.0 + (1.0 - k) * U) * dphi / cap;
          // TRT: the antisymmetric part relaxes with omega(phi) (sets D), the
          // symmetric part with 1 (the rest population and the pair sums go
          // straight to equilibrium, which keeps the lattice stable where
          // D(phi) -> D_s makes omega approach 2).
          double t[7];
          for (int i = 0; i < 7; ++i) t[i] = s->s_hlp[(int64_t)i * n + c];
          s->s_out[c] = weight(7, 0) * U + weight(7, 0) * src;
          for (int i = 1; i < 7; i += 2) {
            const int j = i + 1;
            const double w = weight(7, i);
            double ej = E27[i][0] * jat[0] + E27[i][1] * jat[1] + E27[i][2] * jat[2];
            if (adv) ej += U * (E27[i][0] * s->vel[3 * c] + E27[i][1] * s->vel[3 * c + 1] + E27[i][2] * s->vel[3 * c + 2]);
            const double sym = w * U;             // (t_i + t_j)/2 after relaxation with rate 1
            const double am = 0.5 * (t[i] - t[j]);  // antisymmetric part
            const double am_new = am - om * (am - w * 4.0 * ej);
            s->s_out[(int64_t)i * n + c] = sym + am_new + w * src;
            s->s_out[(int64_t)j * n + c] = sym - am_new + w * src;
          }
          s->temp[c] = U;
        }
    return;
  }
  thermal_relax(s);
}

// ------------------------------------------------ FLOW + DENDRITE model
// run_flow_thermal_dendrite (MaterKit.cpp:467-527): per loop the flow
// (mkFluidsMRT::propagate_PBB, relaxation, bdyVelocity), then the phase field
// and the thermal lattice (advected by the flow's velocity, bdy_flowin).  The
// porous bounce-back is the partially saturated method of Noble & Torczynski
// (Int. J. Mod. Phys. C 9 (1998) 1189): with the solid fraction
// n_s = clamp((1 + phi)/2) of the previous loop and B = n_s (tau - 1/2) /
// ((1 - n_s) + (tau - 1/2)),
//   f* = f + (1 - B) (f_coll - f) + B (f_inv(i) - f_i + feq_i(rho, 0) - feq_inv(i)(rho, u)).
// The x faces carry the non-equilibrium extrapolation of boundary_vel
// (mkFluidsUser.cpp:455-617): f(b) = f(n) + feq(rho_b, u_b) - feq(rho_n, u_n)
// with n the inner neighbour; inflow at x = 0 (u_b = u0, rho_b = rho_n,
// T_b = -Delta, phi_b = -1), outflow at x = nx - 1 (rho_b = rho0, u_b = u_n,
// T_b = T_n, phi_b = phi_n); the face cell's temperature becomes T_b.
void flow_dendrite_nee(orc_state* s, bool flow_lattice);

void flow_dendrite_flow(orc_state* s) {
  const int Q = s->Qw;
  const int64_t n = s->n;
  const mk_params& p = s->p;
  propagate(s, Q, s->w_out, s->w_hlp);
  const double om = 1.0 / p.tau;
  const double om_m = 1.0 / (0.5 + p.magic / (p.tau - 0.5));
  const double F[3] = {p.force[0], p.force[1], p.force[2]};
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    double f[27], fc[27], u[3];
    double rho = 0;
    for (int i = 0; i < Q; ++i) {
      f[i] = s->w_hlp[(int64_t)i * n + c];
      fc[i] = f[i];
      rho += f[i];
    }
    flow_collide(Q, p.collision, om, om_m, fc, F, u);
    const double ns = std::min(1.0, std::max(0.0, 0.5 * (1.0 + s->phi[c])));
    const double B = ns * (p.tau - 0.5) / ((1.0 - ns) + (p.tau - 0.5));
    const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int i = 0; i < Q; ++i) {
      const int k = inv_dir(i);
      const double w = weight(Q, i);
      const double euk = E27[k][0] * u[0] + E27[k][1] * u[1] + E27[k][2] * u[2];
      const double omega_s = f[k] - f[i] + rho * w - rho * feq2(w, euk, uu);
      s->w_out[(int64_t)i * n + c] = f[i] + (1.0 - B) * (fc[i] - f[i]) + B * omega_s;
    }
    for (int a = 0; a < 3; ++a) s->vel[3 * c + a] = u[a];
  }
  flow_dendrite_nee(s, true);
}

void flow_dendrite_nee(orc_state* s, bool flow_lattice) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
  if (!p.inlet) return;
  for (int side = 0; side < 2; ++side) {
    const int xb = side == 0 ? 0 : s->nx - 1, xn = side == 0 ? 1 : s->nx - 2;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < s->nz; ++z)
      for (int y = 0; y < s->ny; ++y) {
        const int64_t b = cidx(s, xb, y, z), nn = cidx(s, xn, y, z);
        if (s->flag[b] != MK_FLAG_FLUID || s->flag[nn] != MK_FLAG_FLUID) continue;
        if (flow_lattice) {
          const int Q = s->Qw;
          double rho = 0, j[3] = {0, 0, 0};
          for (int i = 0; i < Q; ++i) {
            const double v = s->w_out[(int64_t)i * n + nn];
            rho += v;
            for (int a = 0; a < 3; ++a) j[a] += E27[i][a] * v;
          }
          const double un[3] = {j[0] / rho, j[1] / rho, j[2] / rho};
          const double ub[3] = {side == 0 ? p.u0[0] : un[0], side == 0 ? p.u0[1] : un[1], side == 0 ? p.u0[2] : un[2]};
          const double rb = side == 0 ? rho : p.rho0;
          const double uun = un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
          const double uub = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
          for (int i = 0; i < Q; ++i) {
            const double w = weight(Q, i);
            const double eun = E27[i][0] * un[0] + E27[i][1] * un[1] + E27[i][2] * un[2];
            const double eub = E27[i][0] * ub[0] + E27[i][1] * ub[1] + E27[i][2] * ub[2];
            s->w_out[(int64_t)i * n + b] =
                s->w_out[(int64_t)i * n + nn] + rb * feq2(w, eub, uub) - rho * feq2(w, eun, uun);
          }
          for (int a = 0; a < 3; ++a) s->vel[3 * b + a] = ub[a];
        } else {
          // phase field (no velocity in its equilibrium) and thermal lattice
          double phn = 0, Tn = 0;
          for (int i = 0; i < 7; ++i) {
            phn += s->f_out[(int64_t)i * n + nn];
            Tn += s->s_out[(int64_t)i * n + nn];
          }
          const double phb = side == 0 ? -1.0 : phn, Tb = side == 0 ? -p.delta : Tn;
          const double* un = &s->vel[3 * nn];
          const double* ub = &s->vel[3 * b];
          for (int i = 0; i < 7; ++i) {
            const double w = weight(7, i);
            const double eun = E27[i][0] * un[0] + E27[i][1] * un[1] + E27[i][2] * un[2];
            const double eub = E27[i][0] * ub[0] + E27[i][1] * ub[1] + E27[i][2] * ub[2];
            s->f_out[(int64_t)i * n + b] = s->f_out[(int64_t)i * n + nn] + w * (phb - phn);
            s->s_out[(int64_t)i * n + b] =
                s->s_out[(int64_t)i * n + nn] + w * Tb * (1.0 + 4.0 * eub) - w * Tn * (1.0 + 4.0 * eun);
          }
          s->temp[b] = Tb;  // the face cell holds the boundary temperature
        }
      }
  }
}

// ------------------------------------------------------- MULTIGRAIN model
// run_multiPhaseField (MaterKit.cpp:529-571) with mkFluidsUser::propagate /
// relaxation (mkFluidsUser.cpp:68-299, the multiphase field of "Programming
// Phase-Field Modelling" p. 37 Eq. 4.35), whose arithmetic is readable: one
// lattice per grain j on the reference's flow/phase velocity set (D3Q19 here;
// on a one-cell periodic z axis it reduces exactly to the D2Q9 the reference
// ships with QF = 9, mkGlobalDefs.h:134),
//   phi_j = sum_i g_j,i (streamed, :156-160), phi = (N - 1) + sum_j phi_j (:162-168),
//   n_j = s_j / (|s_j| + eps), s_j = sum_i w_i e_i phi_j(x + e_i) (:201-208),
//   g_j* = g_j - om (g_j - geq_j) + w P_j + (1 - om/2) w lam_j (e.n_j) (:283-297),
// geq_j = w phi_j (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2) with u = grain_u for
// j = 1 and 0 otherwise (:220-226), P_j = -2 p_j kappa_j sum_{k != j} p_k^2,
// p = (1 + phi)/2, kappa_0 = 0, kappa_j = grain_kappa (:231-252), om =
// 1/(M/cs^2 + 1/2) with cs^2 = 1/3 (:282, M = dt/dx^2 = mobility); the growth
// source is off (Q_phi = 0 * ..., :255-263).  The library's source term
// (getAddedPhasePDFs) is the Chai et al. (IJHMT 122 (2018) 631) conservative
// flux with lam_j = (1 - phi_j^2)/(sqrt2 W0), eps = 1e-6.  Then the thermal
// lattice with latent heat (1/2) dphi of the aggregate (mkThermalField::
// propagate / relaxation).  Left out: the aggregate g lattice (its density is
// overwritten by the sum of the grains, :162-168, and never read).
void multigrain_step(orc_state* s) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
  const int N = s->Ng;
  for (int j = 0; j < N; ++j) propagate(s, 19, s->gj_out[j], s->gj_hlp[j]);
  std::swap(s->phi_prev, s->phi);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) {
      s->phi[c] = s->phi_prev[c];
      continue;
    }
    double agg = N - 1.0;
    for (int j = 0; j < N; ++j) {
      double ph = 0;
      for (int i = 0; i < 19; ++i) ph += s->gj_hlp[j][(int64_t)i * n + c];
      s->phij[(int64_t)j * n + c] = ph;
      agg += ph;
    }
    s->phi[c] = agg;
  }
  const double om = 1.0 / (3.0 * p.mobility + 0.5);
  const double fo = 1.0 - 0.5 * om;
  const double inv_w = 1.0 / (std::sqrt(2.0) * p.W0);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        if (s->flag[c] != MK_FLAG_FLUID) continue;
        for (int j = 0; j < N; ++j) {
          const double* f = &s->phij[(int64_t)j * n];
          const double ph = f[c];
          double sv[3] = {0, 0, 0};
          for (int i = 1; i < 19; ++i) {
            const int64_t nb = nbr(s, x, y, z, E27[i][0], E27[i][1], E27[i][2]);
            const double fn = nb >= 0 ? f[nb] : ph;
            for (int a = 0; a < 3; ++a) sv[a] += weight(19, i) * E27[i][a] * fn;
          }
          // regularised at 1e-6: where grad phi_j vanishes (a seed centre on
          // a lattice point) its direction is rounding noise, which the flux
          // would carry at full strength lam
          const double sn = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]) + 1e-6;
          const double nv[3] = {sv[0] / sn, sv[1] / sn, sv[2] / sn};
          const double lam = (1.0 - ph * ph) * inv_w;
          double others = 0;
          for (int k = 0; k < N; ++k)
            if (k != j) {
              const double pk = 0.5 * (1.0 + s->phij[(int64_t)k * n + c]);
              others += pk * pk;
            }
          const double P = j == 0 ? 0.0 : -2.0 * (0.5 * (1.0 + ph)) * others * p.grain_kappa;
          const double u[3] = {j == 1 ? p.grain_u[0] : 0.0, j == 1 ? p.grain_u[1] : 0.0, j == 1 ? p.grain_u[2] : 0.0};
          const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
          for (int i = 0; i < 19; ++i) {
            const double w = weight(19, i);
            const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
            const double en = E27[i][0] * nv[0] + E27[i][1] * nv[1] + E27[i][2] * nv[2];
            const double geq = w * ph * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
            const double g = s->gj_hlp[j][(int64_t)i * n + c];
            s->gj_out[j][(int64_t)i * n + c] = g - om * (g - geq) + w * P + fo * w * lam * en;
          }
        }
      }
  propagate(s, 7, s->s_out, s->s_hlp);
  thermal_relax(s);
}

void flow_dendrite_step(orc_state* s) {
  flow_dendrite_flow(s);       // uses phi of the previous loop
  thermal_dendrite_step(s);    // phase field, then the advected thermal lattice
  flow_dendrite_nee(s, false);
}

}  // namespace

// ------------------------------------------------------------------ C API
static int g_threads = 0;

extern "C" void orc_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}

extern "C" int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

extern "C" orc_state* orc_create(const mk_params* p, const double* phi0, const double* T0, const double* C0,
                                 const double* rho0, const double* ux0, const double* uy0, const double* uz0) {
  orc_state* s = new orc_state();
  s->p = *p;
  s->nx = p->nx;
  s->ny = p->ny;
  s->nz = p->nz;
  s->n = (int64_t)p->nx * p->ny * p->nz;
  s->step = 0;
  const int64_t n = s->n;
  s->flag.assign(n, MK_FLAG_FLUID);
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int c3[3] = {x, y, z};
        const int n3[3] = {s->nx, s->ny, s->nz};
        for (int a = 0; a < 3; ++a)
          if (p->bc[a] == MK_BC_WALLS && (c3[a] == 0 || c3[a] == n3[a] - 1)) s->flag[cidx(s, x, y, z)] = MK_FLAG_WALLS;
      }
  s->phi.assign(n, 0.0);
  if (phi0) std::memcpy(s->phi.data(), phi0, n * sizeof(double));
  s->phi_prev = s->phi;
  s->grain.assign(n, 0);
  s->rot.assign(9 * (size_t)(p->n_objects > 0 ? p->n_objects : 1), 0.0);
  s->rot[0] = s->rot[4] = s->rot[8] = 1.0;
  for (int k = 0; k < p->n_objects; ++k) {
    double R[3][3];
    rotation_zyx(p->obj_angle[k], R);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) s->rot[9 * k + 3 * a + b] = R[a][b];
  }
  if (p->model == MK_MODEL_THERMAL_DENDRITE || p->model == MK_MODEL_SOLUTAL_DENDRITE ||
      flow_coupled(p->model)) {
    for (int z = 0; z < s->nz; ++z)
      for (int y = 0; y < s->ny; ++y)
        for (int x = 0; x < s->nx; ++x) s->grain[cidx(s, x, y, z)] = nearest_seed(*p, x, y, z);
  }

  if (p->model == MK_MODEL_FLOW || p->model == MK_MODEL_CONVECTION) {
    const bool conv = p->model == MK_MODEL_CONVECTION;
    s->Qf = p->lattice;
    s->Qs = conv ? 7 : 0;
    const int Q = s->Qf;
    s->f_out.assign((size_t)Q * n, 0.0);
    s->f_hlp.assign((size_t)Q * n, 0.0);
    if (conv) {
      s->s_out.assign((size_t)7 * n, 0.0);
      s->s_hlp.assign((size_t)7 * n, 0.0);
      s->temp.assign(n, p->s_ref);
      if (T0) std::memcpy(s->temp.data(), T0, n * sizeof(double));
    }
    for (int64_t c = 0; c < n; ++c) {
      const double r = rho0 ? rho0[c] : p->rho0;
      const double u[3] = {ux0 ? ux0[c] : p->u0[0], uy0 ? uy0[c] : p->u0[1], uz0 ? uz0[c] : p->u0[2]};
      const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
      for (int i = 0; i < Q; ++i) {
        const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
        s->f_out[(int64_t)i * n + c] = r * feq2(weight(Q, i), eu, uu);
      }
      if (conv)
        for (int i = 0; i < 7; ++i) {
          const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
          s->s_out[(int64_t)i * n + c] = weight(7, i) * s->temp[c] * (1.0 + 4.0 * eu);
        }
    }
  } else if (p->model == MK_MODEL_MULTIPHASE) {
    s->Qf = 19;
    s->Qs = 19;
    s->f_out.assign((size_t)19 * n, 0.0);  // g = geq(p* = 0, u = 0) = 0
    s->f_hlp.assign((size_t)19 * n, 0.0);
    s->s_out.assign((size_t)19 * n, 0.0);
    s->s_hlp.assign((size_t)19 * n, 0.0);
    for (int64_t c = 0; c < n; ++c)
      for (int i = 0; i < 19; ++i) s->s_out[(int64_t)i * n + c] = weight(19, i) * s->phi[c];
  } else {
    s->Qf = 7;
    s->Qs = 7;
    s->temp.assign(n, -p->delta);
    if (p->model == MK_MODEL_THERMAL_DENDRITE && T0) std::memcpy(s->temp.data(), T0, n * sizeof(double));
    if (solutal(p->model) && C0) std::memcpy(s->temp.data(), C0, n * sizeof(double));
    s->f_out.assign((size_t)7 * n, 0.0);
    s->f_hlp.assign((size_t)7 * n, 0.0);
    s->s_out.assign((size_t)7 * n, 0.0);
    s->s_hlp.assign((size_t)7 * n, 0.0);
    if ((p->model == MK_MODEL_FLOW_DENDRITE || p->model == MK_MODEL_MULTIGRAIN) && T0)
      std::memcpy(s->temp.data(), T0, n * sizeof(double));
    for (int64_t c = 0; c < n; ++c)
      for (int i = 0; i < 7; ++i) {
        s->f_out[(int64_t)i * n + c] = weight(7, i) * s->phi[c];
        s->s_out[(int64_t)i * n + c] = weight(7, i) * s->temp[c];
      }
    if (p->model == MK_MODEL_MULTIGRAIN) {
      // one order parameter per seed, -tanh((r - R)/(sqrt2 W0)), and the
      // aggregate (N - 1) + sum phi_j
      const int N = p->n_objects;
      s->Ng = N;
      s->phij.assign((size_t)N * n, 0.0);
      s->gj_out.assign(N, std::vector<double>((size_t)19 * n, 0.0));
      s->gj_hlp.assign(N, std::vector<double>((size_t)19 * n, 0.0));
      for (int z = 0; z < s->nz; ++z)
        for (int y = 0; y < s->ny; ++y)
          for (int x = 0; x < s->nx; ++x) {
            const int64_t c = cidx(s, x, y, z);
            double agg = N - 1.0;
            for (int j = 0; j < N; ++j) {
              const double dx = x - p->obj_center[j][0], dy = y - p->obj_center[j][1], dz = z - p->obj_center[j][2];
              const double ph =
                  -std::tanh((std::sqrt(dx * dx + dy * dy + dz * dz) - p->obj_radius[j]) / (std::sqrt(2.0) * p->W0));
              s->phij[(int64_t)j * n + c] = ph;
              agg += ph;
              for (int i = 0; i < 19; ++i) s->gj_out[j][(int64_t)i * n + c] = weight(19, i) * ph;
            }
            s->phi[c] = agg;
          }
      s->phi_prev = s->phi;
    }
    if (flow_coupled(p->model)) {
      // the flow starts at rho0 with u0 scaled by the liquid fraction, unless
      // density / velocity fields are given
      s->Qw = p->lattice;
      const int Q = s->Qw;
      s->w_out.assign((size_t)Q * n, 0.0);
      s->w_hlp.assign((size_t)Q * n, 0.0);
      s->vel.assign((size_t)3 * n, 0.0);
      for (int64_t c = 0; c < n; ++c) {
        const double ns = std::min(1.0, std::max(0.0, 0.5 * (1.0 + s->phi[c])));
        const bool given = ux0 && uy0 && uz0;
        const double u[3] = {given ? ux0[c] : (1.0 - ns) * p->u0[0], given ? uy0[c] : (1.0 - ns) * p->u0[1],
                             given ? uz0[c] : (1.0 - ns) * p->u0[2]};
        const double r = rho0 ? rho0[c] : p->rho0;
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        for (int a = 0; a < 3; ++a) s->vel[3 * c + a] = u[a];
        for (int i = 0; i < Q; ++i) {
          const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
          s->w_out[(int64_t)i * n + c] = r * feq2(weight(Q, i), eu, uu);
        }
        // the thermal equilibrium carries the same velocity
        for (int i = 0; i < 7; ++i) {
          const double eu = E27[i][0] * u[0] + E27[i][1] * u[1] + E27[i][2] * u[2];
          s->s_out[(int64_t)i * n + c] = weight(7, i) * s->temp[c] * (1.0 + 4.0 * eu);
        }
      }
    }
  }
  return s;
}

extern "C" void orc_destroy(orc_state* s) { delete s; }

extern "C" int64_t orc_step(const orc_state* s) { return s->step; }

// Coupling of a dendrite and a multiphase flow of one grid (the semantics of
// mk_update_geometry / mk_update_velocity): the flow's fluid cells where the
// dendrite's phi > 0 become solid at the flow's next even loop count
// (cumulative), and the dendrite's scalar lattice takes the flow's velocity.
static void apply_pending_solids(orc_state* s) {
  if (!s->pend_set || (s->step & 1)) return;
  for (int64_t c = 0; c < s->n; ++c)
    if (s->pend[c]) s->flag[c] = MK_FLAG_SOLID;
  s->pend_set = 0;
}

extern "C" int orc_update_geometry(orc_state* flow, const orc_state* dend) {
  if (flow->p.model != MK_MODEL_MULTIPHASE || flow->n != dend->n || flow->nx != dend->nx || flow->ny != dend->ny)
    return 1;
  if (flow->pend.empty()) flow->pend.assign(flow->n, 0);
  for (int64_t c = 0; c < flow->n; ++c)
    if (flow->flag[c] == MK_FLAG_FLUID && dend->phi[c] > 0.0) flow->pend[c] = 1;
  flow->pend_set = 1;
  apply_pending_solids(flow);
  return 0;
}

extern "C" int orc_update_velocity(orc_state* dend, const orc_state* flow) {
  if (flow->p.model != MK_MODEL_MULTIPHASE || flow->n != dend->n) return 1;
  std::vector<double> u((size_t)flow->n);
  dend->vel.assign((size_t)3 * flow->n, 0.0);
  for (int a = 0; a < 3; ++a) {
    orc_get_field(flow, MK_FIELD_UX + a, u.data());
    for (int64_t c = 0; c < flow->n; ++c) dend->vel[(size_t)(3 * c + a)] = u[(size_t)c];
  }
  return 0;
}

extern "C" void orc_advance(orc_state* s, int64_t nsteps) {
  for (int64_t t = 0; t < nsteps; ++t) {
    switch (s->p.model) {
      case MK_MODEL_FLOW:
        flow_step(s);
        break;
      case MK_MODEL_MULTIPHASE:
        apply_pending_solids(s);
        mp_step(s);
        break;
      case MK_MODEL_CONVECTION:
        convection_step(s);
        break;
      case MK_MODEL_FLOW_DENDRITE:
      case MK_MODEL_FLOW_SOLUTAL:
        flow_dendrite_step(s);
        break;
      case MK_MODEL_MULTIGRAIN:
        multigrain_step(s);
        break;
      case MK_MODEL_THERMAL_DENDRITE:
      case MK_MODEL_SOLUTAL_DENDRITE:
        thermal_dendrite_step(s);  // the second lattice follows p.model
        break;
      default:
        return;
    }
    s->step++;
  }
}

extern "C" int orc_get_grain_phi(const orc_state* s, int grain, double* out) {
  if (grain < 0 || grain >= s->Ng) return 1;
  std::memcpy(out, &s->phij[(size_t)grain * s->n], s->n * sizeof(double));
  return 0;
}

extern "C" int orc_get_populations(const orc_state* s, int which, double* out) {
  const std::vector<double>& v = which == 0 ? s->f_out : (which == 1 ? s->s_out : s->w_out);
  if (v.empty()) return 1;
  std::memcpy(out, v.data(), v.size() * sizeof(double));
  return 0;
}

extern "C" int orc_get_field(const orc_state* s, int field, double* out) {
  const int64_t n = s->n;
  const mk_params& p = s->p;
  if (field == MK_FIELD_FLAG && !flow_coupled(p.model)) {
    for (int64_t c = 0; c < n; ++c) out[c] = s->flag[c];
    return 0;
  }
  if (field == MK_FIELD_GRAIN) {
    if (p.model == MK_MODEL_MULTIGRAIN) {
      // the grain whose order parameter is largest (ties to the lower index)
      for (int64_t c = 0; c < n; ++c) {
        int best = 0;
        for (int j = 1; j < s->Ng; ++j)
          if (s->phij[(int64_t)j * n + c] > s->phij[(int64_t)best * n + c]) best = j;
        out[c] = best;
      }
      return 0;
    }
    for (int64_t c = 0; c < n; ++c) out[c] = s->grain[c];
    return 0;
  }
  if (field == MK_FIELD_PHI) {
    std::memcpy(out, s->phi.data(), n * sizeof(double));
    return 0;
  }
  if (flow_coupled(p.model)) {
    if (field == MK_FIELD_FLAG) {
      // reset_flags (mkPhaseField.h:37): solid where phi > 0
      for (int64_t c = 0; c < n; ++c) out[c] = s->flag[c] != MK_FLAG_FLUID ? s->flag[c]
                                                 : (s->phi[c] > 0.0 ? MK_FLAG_SOLID : MK_FLAG_FLUID);
      return 0;
    }
    if (field == MK_FIELD_RHO || field == MK_FIELD_UX || field == MK_FIELD_UY || field == MK_FIELD_UZ) {
      const int Q = s->Qw;
      for (int64_t c = 0; c < n; ++c) {
        if (s->flag[c] != MK_FLAG_FLUID) {
          out[c] = field == MK_FIELD_RHO ? p.rho0 : 0.0;
          continue;
        }
        double rho = 0, j[3] = {0, 0, 0};
        for (int i = 0; i < Q; ++i) {
          const double f = s->w_out[(int64_t)i * n + c];
          rho += f;
          for (int a = 0; a < 3; ++a) j[a] += E27[i][a] * f;
        }
        out[c] = field == MK_FIELD_RHO ? rho : (j[field - MK_FIELD_UX] - 0.5 * p.force[field - MK_FIELD_UX]) / rho;
      }
      return 0;
    }
  }
  if (p.model == MK_MODEL_CONVECTION && field == MK_FIELD_T) {
    std::memcpy(out, s->temp.data(), n * sizeof(double));
    return 0;
  }
  if (p.model == MK_MODEL_FLOW || p.model == MK_MODEL_CONVECTION) {
    if (field != MK_FIELD_RHO && field != MK_FIELD_UX && field != MK_FIELD_UY && field != MK_FIELD_UZ) return 1;
    double F[3];
    flow_force(s, F);
    const int Q = s->Qf;
    for (int64_t c = 0; c < n; ++c) {
      if (s->flag[c] != MK_FLAG_FLUID) {
        out[c] = field == MK_FIELD_RHO ? p.rho0 : 0.0;
        continue;
      }
      if (p.model == MK_MODEL_CONVECTION) {
        // the buoyancy of the stored (post-collision) scalar
        double T = 0;
        for (int i = 0; i < 7; ++i) T += s->s_out[(int64_t)i * n + c];
        for (int a = 0; a < 3; ++a) F[a] = -p.rho0 * p.beta * p.force[a] * (T - p.s_ref);
      }
      double rho = 0, j[3] = {0, 0, 0};
      for (int i = 0; i < Q; ++i) {
        const double f = s->f_out[(int64_t)i * n + c];
        rho += f;
        j[0] += E27[i][0] * f;
        j[1] += E27[i][1] * f;
        j[2] += E27[i][2] * f;
      }
      if (field == MK_FIELD_RHO)
        out[c] = rho;
      else {
        const int a = field - MK_FIELD_UX;
        out[c] = (j[a] - 0.5 * F[a]) / rho;
      }
    }
    return 0;
  }
  if (p.model == MK_MODEL_MULTIPHASE) {
    if (field != MK_FIELD_RHO && field != MK_FIELD_UX && field != MK_FIELD_UY && field != MK_FIELD_UZ &&
        field != MK_FIELD_PRESSURE)
      return 1;
    const MpConst k = mp_const(p);
    for (int z = 0; z < s->nz; ++z)
      for (int y = 0; y < s->ny; ++y)
        for (int x = 0; x < s->nx; ++x) {
          const int64_t c = cidx(s, x, y, z);
          if (field == MK_FIELD_RHO) {
            out[c] = p.rho_g + s->phi[c] * (p.rho_l - p.rho_g);
            continue;
          }
          if (s->flag[c] != MK_FLAG_FLUID) {
            out[c] = 0.0;
            continue;
          }
          double pstar = 0, j[3] = {0, 0, 0};
          for (int i = 0; i < 19; ++i) {
            const double g = s->f_out[(int64_t)i * n + c];
            pstar += g;
            j[0] += E27[i][0] * g;
            j[1] += E27[i][1] * g;
            j[2] += E27[i][2] * g;
          }
          if (field == MK_FIELD_PRESSURE) {
            out[c] = pstar;
            continue;
          }
          const MpLocal L = mp_local(s, k, x, y, z, pstar);
          const int a = field - MK_FIELD_UX;
          out[c] = j[a] - L.F[a] / (2.0 * L.rho);
        }
    return 0;
  }
  // dendrites
  if (field == MK_FIELD_T || field == MK_FIELD_C) {
    if ((field == MK_FIELD_T) != !solutal(p.model)) return 1;
    std::memcpy(out, s->temp.data(), n * sizeof(double));
    return 0;
  }
  if (field == MK_FIELD_DPHI) {
    for (int64_t c = 0; c < n; ++c) out[c] = s->phi[c] - s->phi_prev[c];
    return 0;
  }
  return 1;
}

extern "C" void orc_anisotropy(int kind, double e4, double e2, const double* n, double* a, double* g) {
  aniso_function(kind, e4, e2, n, a, g);
}

// ------------------------------------------------------------------ ADJOINT
// Discrete adjoint of the thermal dendrite loop (thermal_dendrite_step),
// reverse mode over stored states.  The state at the start of loop n is
// Y = (F = f_out, S = s_out, P = phi (= phi^(n-1)), U = temp (= u^n)); the loss
// is a function of P after the last loop.
namespace {

// d2a/dn2 and the derivatives of a and da/dn with respect to e4, for the
// kinds of aniso_function.
void aniso_second(int kind, double e4, double e2, const double n[3], double H[3][3], double* a_e4,
                  double da_e4[3]) {
  const double x = n[0], y = n[1], z = n[2];
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  for (int q = 0; q < 3; ++q)
    for (int r = 0; r < 3; ++r) H[q][r] = 0.0;
  switch (kind) {
    case MK_ANISO_CBC: {
      const double s4 = x2 * x2 + y2 * y2 + z2 * z2;
      H[0][0] = 12.0 * e4 * x2 + e2 * (36.0 * x2 + 132.0 * y2 * z2);
      H[1][1] = 12.0 * e4 * y2 + e2 * (36.0 * y2 + 132.0 * x2 * z2);
      H[2][2] = 12.0 * e4 * z2 + e2 * (36.0 * z2 + 132.0 * x2 * y2);
      H[0][1] = H[1][0] = 264.0 * e2 * x * y * z2;
      H[0][2] = H[2][0] = 264.0 * e2 * x * z * y2;
      H[1][2] = H[2][1] = 264.0 * e2 * y * z * x2;
      *a_e4 = s4 - 0.6;
      da_e4[0] = 4.0 * x2 * x;
      da_e4[1] = 4.0 * y2 * y;
      da_e4[2] = 4.0 * z2 * z;
      break;
    }
    case MK_ANISO_HCP: {
      const double h00 = 6.0 * e4 * (5.0 * x2 * x2 - 30.0 * x2 * y2 + 5.0 * y2 * y2);
      H[0][0] = h00;
      H[1][1] = -h00;
      H[0][1] = H[1][0] = 6.0 * e4 * (-20.0 * x2 * x * y + 20.0 * x * y2 * y);
      H[2][2] = 4.0 * e2;
      *a_e4 = x2 * x2 * x2 - 15.0 * x2 * x2 * y2 + 15.0 * x2 * y2 * y2 - y2 * y2 * y2;
      da_e4[0] = 6.0 * (x2 * x2 * x - 10.0 * x2 * x * y2 + 5.0 * x * y2 * y2);
      da_e4[1] = -6.0 * (5.0 * x2 * x2 * y - 10.0 * x2 * y2 * y + y2 * y2 * y);
      da_e4[2] = 0.0;
      break;
    }
    case MK_ANISO_FACET: {
      const double r[3] = {sqrt(x2 + e2 * e2), sqrt(y2 + e2 * e2), sqrt(z2 + e2 * e2)};
      for (int q = 0; q < 3; ++q) {
        H[q][q] = e4 * e2 * e2 / (r[q] * r[q] * r[q]);
        da_e4[q] = n[q] / r[q];
      }
      *a_e4 = r[0] + r[1] + r[2] - sqrt(1.0 + e2 * e2) - 2.0 * e2;
      break;
    }
    default: {
      H[0][0] = 48.0 * e4 * x2;
      H[1][1] = 48.0 * e4 * y2;
      H[2][2] = 48.0 * e4 * z2;
      *a_e4 = -3.0 + 4.0 * (x2 * x2 + y2 * y2 + z2 * z2);
      da_e4[0] = 16.0 * x2 * x;
      da_e4[1] = 16.0 * y2 * y;
      da_e4[2] = 16.0 * z2 * z;
      break;
    }
  }
}

// Below this |grad phi| the normal n = grad phi / (|grad phi| + 1e-12) is
// rounding noise, and its exact derivative (~1 / (|grad phi| + 1e-12)) makes
// the adjoint of the (1 - a^2) dphi source grow without bound over long runs
// (measured: 1e32 after 2000 loops at 96^3, while central differences stay
// near 3e5).  There the reverse sweep keeps the direct eps4 derivative of a
// and N and drops their derivative through n.
const double kAdjGradCut = 1e-8;

// Reverse of anisotropy(): from the adjoints ab of a and Nb of N, adds the
// adjoint of the lab gradient to gb and that of e4 to *e4b.
void anisotropy_vjp(const double* R, int kind, double e4, double e2, const double g[3], double ab, const double Nb[3],
                    double gb[3], double* e4b) {
  const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  const double inv = 1.0 / (gn + 1e-12);
  const double nl[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
  double nc[3];
  for (int q = 0; q < 3; ++q) nc[q] = R[0 * 3 + q] * nl[0] + R[1 * 3 + q] * nl[1] + R[2 * 3 + q] * nl[2];
  double a, da[3];
  aniso_function(kind, e4, e2, nc, &a, da);
  const double ndg = nc[0] * da[0] + nc[1] * da[1] + nc[2] * da[2];
  // N = R Nc, Nc = gn a (da - nc ndg)
  double Ncb[3];
  for (int q = 0; q < 3; ++q) Ncb[q] = R[0 * 3 + q] * Nb[0] + R[1 * 3 + q] * Nb[1] + R[2 * 3 + q] * Nb[2];
  double ct = 0, cn = 0;
  for (int q = 0; q < 3; ++q) {
    ct += Ncb[q] * (da[q] - nc[q] * ndg);
    cn += Ncb[q] * nc[q];
  }
  double gnb = a * ct;
  const double abt = ab + gn * ct;
  double dab[3], ncb[3];
  const double ndgb = -gn * a * cn;
  for (int q = 0; q < 3; ++q) {
    dab[q] = gn * a * Ncb[q] + ndgb * nc[q];
    ncb[q] = -gn * a * Ncb[q] * ndg + ndgb * da[q];
  }
  // (a, da) = f(nc)
  double H[3][3], a_e4, da_e4[3];
  aniso_second(kind, e4, e2, nc, H, &a_e4, da_e4);
  for (int q = 0; q < 3; ++q) ncb[q] += abt * da[q] + H[q][0] * dab[0] + H[q][1] * dab[1] + H[q][2] * dab[2];
  *e4b += abt * a_e4 + dab[0] * da_e4[0] + dab[1] * da_e4[1] + dab[2] * da_e4[2];
  if (gn < kAdjGradCut) return;
  // nc = R^T nl
  double nlb[3];
  for (int r = 0; r < 3; ++r) nlb[r] = R[r * 3 + 0] * ncb[0] + R[r * 3 + 1] * ncb[1] + R[r * 3 + 2] * ncb[2];
  // nl = g inv, inv = 1/(gn + 1e-12), gn = |g|
  const double invb = nlb[0] * g[0] + nlb[1] * g[1] + nlb[2] * g[2];
  for (int q = 0; q < 3; ++q) gb[q] += inv * nlb[q];
  gnb -= inv * inv * invb;
  if (gn > 0)
    for (int q = 0; q < 3; ++q) gb[q] += gnb * g[q] / gn;
}

// Transpose of propagate(): outb_k(y) = hlpb_k(y + e_k), or hlpb_inv(k)(y)
// when y + e_k is not fluid.
void propagate_adjoint(const orc_state* s, int Q, const std::vector<double>& hlpb, std::vector<double>& outb) {
  const int64_t n = s->n;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const int64_t c = cidx(s, x, y, z);
        for (int i = 0; i < Q; ++i) {
          if (s->flag[c] != MK_FLAG_FLUID) {
            outb[(int64_t)i * n + c] = 0.0;
            continue;
          }
          const int64_t d = nbr(s, x, y, z, E27[i][0], E27[i][1], E27[i][2]);
          outb[(int64_t)i * n + c] = d >= 0 ? hlpb[(int64_t)i * n + d] : hlpb[(int64_t)inv_dir(i) * n + c];
        }
      }
}

struct AdjSnap {
  std::vector<double> F, S, P, U;
};

}  // namespace

// Loss L = sum (phi - target)^2 of phi after `steps` loops from the current
// state, and dL/d eps4, dL/d Delta (a uniform shift of the initial u by
// -Delta) and dL/d tau_T (omega_T = 1/tau_T; tau0 held fixed).  out = {L,
// dL/deps4, dL/dDelta, dL/dtau_T}.  Thermal dendrite only; leaves the state
// advanced by `steps` loops.
extern "C" int orc_backward(orc_state* s, const double* target, int64_t steps, double* out) {
  if (s->p.model != MK_MODEL_THERMAL_DENDRITE || steps < 1) return 1;
  const int64_t n = s->n;
  const mk_params& p = s->p;
  std::vector<AdjSnap> Y((size_t)steps + 1);
  auto snap = [&](AdjSnap& y) {
    y.F = s->f_out;
    y.S = s->s_out;
    y.P = s->phi;
    y.U = s->temp;
  };
  snap(Y[0]);
  for (int64_t t = 0; t < steps; ++t) {
    thermal_dendrite_step(s);
    s->step++;
    snap(Y[(size_t)t + 1]);
  }
  double loss = 0;
  std::vector<double> Pb(n), Ub(n, 0.0), Fb(7 * n, 0.0), Sb(7 * n, 0.0);
  for (int64_t c = 0; c < n; ++c) {
    const double d = s->phi[c] - target[c];
    loss += d * d;
    Pb[c] = 2.0 * d;
  }
  const double D0 = p.W0 * p.W0 / p.tau0;
  const double om_g = 1.0 / (4.0 * D0 + 0.5);
  const double om_t = 1.0 / (4.0 * p.D + 0.5);
  const double cs2 = 0.25;
  const double fo = (1.0 - 0.5 * om_g) / cs2;
  double e4b = 0, omtb = 0;
  std::vector<double> fh(7 * n), sh(7 * n), fhb(7 * n), shb(7 * n), phib(n), Pbn(n), Ubn(n), gbar(3 * n);
  for (int64_t t = steps - 1; t >= 0; --t) {
    const AdjSnap& y = Y[(size_t)t];
    const std::vector<double>& phin = Y[(size_t)t + 1].P;  // phi^t
    propagate(s, 7, y.F, fh);
    propagate(s, 7, y.S, sh);
    std::fill(fhb.begin(), fhb.end(), 0.0);
    std::fill(shb.begin(), shb.end(), 0.0);
    std::fill(Pbn.begin(), Pbn.end(), 0.0);
    std::fill(Ubn.begin(), Ubn.end(), 0.0);
    std::fill(gbar.begin(), gbar.end(), 0.0);
    for (int64_t c = 0; c < n; ++c) phib[c] = Pb[c];  // the loop's phi^t becomes P
    double e4_acc = 0, om_acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : e4_acc, om_acc)
    for (int z = 0; z < s->nz; ++z)
      for (int yy = 0; yy < s->ny; ++yy)
        for (int x = 0; x < s->nx; ++x) {
          const int64_t c = cidx(s, x, yy, z);
          if (s->flag[c] != MK_FLAG_FLUID) continue;
          // thermal relaxation t* = t - om_t (t - w T) + w dphi / 2, U' = T
          double T = 0, Mt = 0;
          for (int i = 0; i < 7; ++i) {
            T += sh[(int64_t)i * n + c];
            Mt += weight(7, i) * Sb[(int64_t)i * n + c];
          }
          for (int i = 0; i < 7; ++i) {
            const double sbi = Sb[(int64_t)i * n + c];
            shb[(int64_t)i * n + c] = (1.0 - om_t) * sbi + om_t * Mt + Ub[c];
            om_acc += sbi * (weight(7, i) * T - sh[(int64_t)i * n + c]);
          }
          double dphib = 0.5 * Mt;
          // phase-field relaxation
          const double ph = phin[c];
          const double dphi = ph - y.P[c];
          const double u = y.U[c];
          const double one_m = 1.0 - ph * ph;
          double gr[3], lap;
          grad_lap(
              s, phin, x, yy, z, [](double p0) { return p0; }, gr, &lap);
          const double* R = &s->rot[9 * s->grain[c]];
          double a, N[3];
          anisotropy(R, p.aniso, p.eps4, p.eps2, gr, &a, N);
          double Mg = 0, Vg[3] = {0, 0, 0};
          for (int i = 0; i < 7; ++i) {
            const double fb = Fb[(int64_t)i * n + c];
            const double w = weight(7, i);
            Mg += w * fb;
            for (int q = 0; q < 3; ++q) Vg[q] += w * E27[i][q] * fb;
            fhb[(int64_t)i * n + c] = (1.0 - om_g) * fb;
          }
          const double src_phi = (1.0 - 3.0 * ph * ph + 4.0 * p.lambda * u * ph * one_m) / p.tau0;
          double phb = om_g * Mg + Mg * src_phi;
          Ubn[c] = -Mg * p.lambda * one_m * one_m / p.tau0;
          dphib += (1.0 - a * a) * Mg;
          phb += dphib;
          Pbn[c] -= dphib;
          const double beta[3] = {fo * Vg[0], fo * Vg[1], fo * Vg[2]};
          const double bg = beta[0] * gr[0] + beta[1] * gr[1] + beta[2] * gr[2];
          const double ab = -cs2 * 2.0 * a * bg - 2.0 * a * dphi * Mg;
          const double Nb[3] = {-cs2 * beta[0], -cs2 * beta[1], -cs2 * beta[2]};
          double gb[3] = {-cs2 * (a * a - 1.0) * beta[0], -cs2 * (a * a - 1.0) * beta[1],
                          -cs2 * (a * a - 1.0) * beta[2]};
          anisotropy_vjp(R, p.aniso, p.eps4, p.eps2, gr, ab, Nb, gb, &e4_acc);
          for (int q = 0; q < 3; ++q) gbar[3 * c + q] = gb[q];
          phib[c] += phb;
        }
    e4b += e4_acc;
    omtb += om_acc;
    // gr(x) = 3 sum_k w_k e_k phi~(x + e_k), phi~ = phi(x) at a non-fluid neighbour
#pragma omp parallel for schedule(static)
    for (int z = 0; z < s->nz; ++z)
      for (int yy = 0; yy < s->ny; ++yy)
        for (int x = 0; x < s->nx; ++x) {
          const int64_t c = cidx(s, x, yy, z);
          if (s->flag[c] != MK_FLAG_FLUID) continue;
          double acc = 0;
          for (int k = 1; k < 19; ++k) {
            const double w3 = 3.0 * weight(19, k);
            const int64_t src = nbr(s, x, yy, z, -E27[k][0], -E27[k][1], -E27[k][2]);
            if (src >= 0)
              acc += w3 * (E27[k][0] * gbar[3 * src] + E27[k][1] * gbar[3 * src + 1] + E27[k][2] * gbar[3 * src + 2]);
            if (nbr(s, x, yy, z, E27[k][0], E27[k][1], E27[k][2]) < 0)
              acc += w3 * (E27[k][0] * gbar[3 * c] + E27[k][1] * gbar[3 * c + 1] + E27[k][2] * gbar[3 * c + 2]);
          }
          phib[c] += acc;
        }
    // phi^t = sum of the streamed g (fluid), a copy of P (elsewhere)
    for (int64_t c = 0; c < n; ++c) {
      if (s->flag[c] == MK_FLAG_FLUID) {
        for (int i = 0; i < 7; ++i) fhb[(int64_t)i * n + c] += phib[c];
      } else {
        Pbn[c] += phib[c];
      }
    }
    propagate_adjoint(s, 7, fhb, Fb);
    propagate_adjoint(s, 7, shb, Sb);
    Pb.swap(Pbn);
    Ub.swap(Ubn);
  }
  // initial state: S_i = w_i u0, U = u0, u0 = -Delta (fluid cells)
  double sum_u = 0;
  for (int64_t c = 0; c < n; ++c) {
    if (s->flag[c] != MK_FLAG_FLUID) continue;
    for (int i = 0; i < 7; ++i) sum_u += weight(7, i) * Sb[(int64_t)i * n + c];
    sum_u += Ub[c];
  }
  out[0] = loss;
  out[1] = e4b;
  out[2] = -sum_u;
  out[3] = -om_t * om_t * omtb;
  return 0;
}

// ===================================================== reference-structure
// The same method with the reference's data structure: every field of a node
// in one object, mirroring the member list of mkNode (MaterKit/inc/mkNode.h:
// 128-215: the f / g / h / x population vectors of 19 values each, the
// equilibrium and neighbour vectors, velocity, density, phase and temperature
// fields, the multigrain and solute vectors), an array of those objects, and
// node sweeps `omp parallel for schedule(static, 16)` (MK_OMP_CHUNKSIZE,
// MaterKit/src/mkFluidsUser.cpp:70).  Used as the CPU baseline closest to the
// reference's own memory traffic (its solver bodies are in the closed DLL);
// for the flow model and the thermal dendrite it reproduces orc_advance bit
// for bit (the same per-cell arithmetic, in the same order).
namespace {

struct AosNode {
  double f_out[19], f_hlp[19], f_equ[19];
  double vel[3], vel_old[3];
  double density, omega_f;
  double g_out[19], g_hlp[19], g_nbr[19];
  double phi, phi_old, d_phi;
  std::vector<double> gVec_out, gVec_hlp, gVec_nbr;  // multigrain lattices (empty here)
  std::vector<double> phiVec, phiVec_old, d_phiVec;
  double N_v[3], D_p, A2s, phi_n[3], normal[3];
  double h_out[19], h_hlp[19];
  double temperature;
  double index_nb[19];
  double x_out[19], x_hlp[19];
  std::vector<double> X_potents, X_solutes, X_DCs;  // solute vectors (empty here)
  double ptl_mp, prs_mp, rho_mp, eta, k_d;
  int flag, grain_id;
};

constexpr int kChunk = 16;

}  // namespace

struct orc_aos {
  orc_state geo;  // parameters, flags, grains and rotations only
  std::vector<AosNode> node;
};

namespace {

// The streaming of mkFluidsUser.cpp:77-97 on one population vector member.
template <double (AosNode::*OUT)[19], double (AosNode::*HLP)[19]>
void aos_propagate(orc_aos* a, int Q) {
  const orc_state* s = &a->geo;
  const int64_t n = s->n;
  AosNode* nd = a->node.data();
#pragma omp parallel for schedule(static, kChunk)
  for (int64_t c = 0; c < n; ++c) {
    if (nd[c].flag != MK_FLAG_FLUID) continue;
    const int x = (int)(c % s->nx), y = (int)((c / s->nx) % s->ny), z = (int)(c / ((int64_t)s->nx * s->ny));
    for (int i = 0; i < Q; ++i) {
      const int64_t src = nbr(s, x, y, z, -E27[i][0], -E27[i][1], -E27[i][2]);
      (nd[c].*HLP)[i] = src >= 0 ? (nd[src].*OUT)[i] : (nd[c].*OUT)[inv_dir(i)];
    }
  }
}

// grad_lap on the nodes' phi (the same sums as grad_lap, in the same order).
void aos_grad_lap(const orc_aos* a, int x, int y, int z, double g[3], double* lap) {
  const orc_state* s = &a->geo;
  const AosNode* nd = a->node.data();
  const double f0 = nd[cidx(s, x, y, z)].phi;
  g[0] = g[1] = g[2] = 0;
  double l = 0;
  for (int i = 1; i < 19; ++i) {
    const int64_t j = nbr(s, x, y, z, E27[i][0], E27[i][1], E27[i][2]);
    const double fn = j >= 0 ? nd[j].phi : f0;
    const double w = weight(19, i);
    g[0] += w * E27[i][0] * fn;
    g[1] += w * E27[i][1] * fn;
    g[2] += w * E27[i][2] * fn;
    l += w * (fn - f0);
  }
  g[0] *= 3.0;
  g[1] *= 3.0;
  g[2] *= 3.0;
  *lap = 6.0 * l;
}

void aos_flow_step(orc_aos* a) {
  const orc_state* s = &a->geo;
  const int Q = s->Qf;
  aos_propagate<&AosNode::f_out, &AosNode::f_hlp>(a, Q);
  double F[3];
  flow_force(s, F);
  const double tau = s->p.tau, om = 1.0 / tau;
  const double om_m = 1.0 / (0.5 + s->p.magic / (tau - 0.5));
  const int coll = s->p.collision;
  AosNode* nd = a->node.data();
#pragma omp parallel for schedule(static, kChunk)
  for (int64_t c = 0; c < s->n; ++c) {
    AosNode& q = nd[c];
    if (q.flag != MK_FLAG_FLUID) continue;
    double f[27], u[3];
    for (int i = 0; i < Q; ++i) f[i] = q.f_hlp[i];
    flow_collide(Q, coll, om, om_m, f, F, u);
    for (int i = 0; i < Q; ++i) q.f_out[i] = f[i];
    double rho = 0;
    for (int i = 0; i < Q; ++i) rho += q.f_hlp[i];
    q.density = rho;
    for (int k = 0; k < 3; ++k) {
      q.vel_old[k] = q.vel[k];
      q.vel[k] = u[k];
    }
  }
}

void aos_thermal_dendrite_step(orc_aos* a) {
  const orc_state* s = &a->geo;
  const mk_params& p = s->p;
  AosNode* nd = a->node.data();
  aos_propagate<&AosNode::g_out, &AosNode::g_hlp>(a, 7);
#pragma omp parallel for schedule(static, kChunk)
  for (int64_t c = 0; c < s->n; ++c) {
    AosNode& q = nd[c];
    q.phi_old = q.phi;
    if (q.flag != MK_FLAG_FLUID) continue;
    double ph = 0;
    for (int i = 0; i < 7; ++i) ph += q.g_hlp[i];
    q.phi = ph;
  }
  const double D0 = p.W0 * p.W0 / p.tau0;
  const double om_g = 1.0 / (4.0 * D0 + 0.5);
  const double cs2 = 0.25;
#pragma omp parallel for schedule(static, kChunk)
  for (int64_t c = 0; c < s->n; ++c) {
    AosNode& q = nd[c];
    if (q.flag != MK_FLAG_FLUID) continue;
    const int x = (int)(c % s->nx), y = (int)((c / s->nx) % s->ny), z = (int)(c / ((int64_t)s->nx * s->ny));
    double gr[3], lap;
    aos_grad_lap(a, x, y, z, gr, &lap);
    double an, N[3];
    anisotropy(&s->rot[9 * q.grain_id], p.aniso, p.eps4, p.eps2, gr, &an, N);
    const double ph = q.phi;
    const double dphi = ph - q.phi_old;
    const double one_m = 1.0 - ph * ph;
    const double src = (ph - ph * ph * ph - p.lambda * q.temperature * one_m * one_m) / p.tau0 + (1.0 - an * an) * dphi;
    double B[3];
    for (int k = 0; k < 3; ++k) B[k] = -cs2 * ((an * an - 1.0) * gr[k] + N[k]);
    for (int k = 0; k < 3; ++k) {
      q.phi_n[k] = gr[k];
      q.normal[k] = N[k];
    }
    q.d_phi = dphi;
    for (int i = 0; i < 7; ++i) {
      const double w = weight(7, i);
      const double eB = E27[i][0] * B[0] + E27[i][1] * B[1] + E27[i][2] * B[2];
      const double gi = q.g_hlp[i];
      q.g_out[i] = gi - om_g * (gi - w * ph) + (1.0 - 0.5 * om_g) * w * eB / cs2 + w * src;
    }
  }
  aos_propagate<&AosNode::h_out, &AosNode::h_hlp>(a, 7);
  const double om_t = 1.0 / (4.0 * p.D + 0.5);
#pragma omp parallel for schedule(static, kChunk)
  for (int64_t c = 0; c < s->n; ++c) {
    AosNode& q = nd[c];
    if (q.flag != MK_FLAG_FLUID) continue;
    double T = 0;
    for (int i = 0; i < 7; ++i) T += q.h_hlp[i];
    const double lat = 0.5 * (q.phi - q.phi_old);
    for (int i = 0; i < 7; ++i) {
      const double w = weight(7, i);
      const double ti = q.h_hlp[i];
      q.h_out[i] = ti - om_t * (ti - w * T * (1.0 + 4.0 * 0.0)) + w * lat;
    }
    q.temperature = T;
  }
}

}  // namespace

extern "C" size_t orc_aos_node_bytes(void) { return sizeof(AosNode); }

extern "C" orc_aos* orc_aos_create(const orc_state* s) {
  const int m = s->p.model;
  if (!((m == MK_MODEL_FLOW && s->Qf == 19 && s->p.wall_axis < 0) || m == MK_MODEL_THERMAL_DENDRITE)) return nullptr;
  orc_aos* a = new orc_aos();
  a->geo.p = s->p;
  a->geo.nx = s->nx;
  a->geo.ny = s->ny;
  a->geo.nz = s->nz;
  a->geo.n = s->n;
  a->geo.step = s->step;
  a->geo.Qf = s->Qf;
  a->geo.Qs = s->Qs;
  a->geo.flag = s->flag;
  a->geo.grain = s->grain;
  a->geo.rot = s->rot;
  const int64_t n = s->n;
  a->node.resize((size_t)n);
  for (int64_t c = 0; c < n; ++c) {
    AosNode& q = a->node[(size_t)c];  // value-initialised: every number starts at 0
    q.flag = s->flag[c];
    q.grain_id = s->grain.empty() ? 0 : s->grain[c];
    if (m == MK_MODEL_FLOW) {
      for (int i = 0; i < s->Qf; ++i) q.f_out[i] = s->f_out[(int64_t)i * n + c];
    } else {
      for (int i = 0; i < 7; ++i) {
        q.g_out[i] = s->f_out[(int64_t)i * n + c];
        q.h_out[i] = s->s_out[(int64_t)i * n + c];
      }
      q.phi = s->phi[c];
      q.phi_old = s->phi_prev[c];
      q.temperature = s->temp[c];
    }
  }
  return a;
}

extern "C" void orc_aos_destroy(orc_aos* a) { delete a; }

extern "C" void orc_aos_advance(orc_aos* a, int64_t nsteps) {
  for (int64_t t = 0; t < nsteps; ++t) {
    if (a->geo.p.model == MK_MODEL_FLOW)
      aos_flow_step(a);
    else
      aos_thermal_dendrite_step(a);
    a->geo.step += 1;
  }
}

// Post-collision populations in the layout of orc_get_populations ([q][cell];
// which 0: the flow lattice or the phase-field lattice, 1: the thermal one),
// or the phase field / temperature (field MK_FIELD_PHI / MK_FIELD_T).
extern "C" int orc_aos_get_populations(const orc_aos* a, int which, double* out) {
  const int64_t n = a->geo.n;
  const bool flow = a->geo.p.model == MK_MODEL_FLOW;
  if (which < 0 || which > 1 || (flow && which == 1)) return -1;
  const int Q = flow ? a->geo.Qf : 7;
  for (int64_t c = 0; c < n; ++c) {
    const AosNode& q = a->node[(size_t)c];
    const double* v = flow ? q.f_out : (which == 0 ? q.g_out : q.h_out);
    for (int i = 0; i < Q; ++i) out[(int64_t)i * n + c] = v[i];
  }
  return 0;
}

extern "C" int orc_aos_get_field(const orc_aos* a, int field, double* out) {
  if (field != MK_FIELD_PHI && field != MK_FIELD_T) return -1;
  for (int64_t c = 0; c < a->geo.n; ++c)
    out[c] = field == MK_FIELD_PHI ? a->node[(size_t)c].phi : a->node[(size_t)c].temperature;
  return 0;
}
