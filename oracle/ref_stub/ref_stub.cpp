// Bodies of the closed-library functions that the reference's readable
// multigrain solver (MaterKit/src/mkFluidsUser.cpp: propagate, relaxation)
// calls, restated from the published forms, and a C entry point that runs
// that solver on given initial order parameters.  Test infrastructure: built
// into oracle/_ref by oracle/Makefile (target `ref`) together with the
// reference's mkFluidsUser.cpp, compiled where it lies; the fixture generator
// tests/golden/make_multigrain_ref.py and bench.py's CPU baseline legs load
// the result.
//
// Restated here (not readable in the reference):
//   lattice        D2Q9 (QF 9) or D3Q19 (QF 19) velocities and weights, cs^2 = 1/3
//   getEquPDFs     w_i rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2)
//   getAddedPhasePDFs  the conservative phase-field source of Chai et al.
//                  (Int. J. Heat Mass Transfer 122 (2018) 631):
//                  (1 - omega/2) w_i lam e_i.n, lam = (1 - phi^2)/(sqrt2 W0)
//   neighbor       periodic wrap on every axis
//   reset_flags    leaves every node fluid (the multigrain case has no solid)
//   epsilon        1e-6, the regularisation of the grain normal
// The harness runs one OpenMP thread unless mgref_set_threads says otherwise:
// relaxation() keeps omega_g firstprivate and sets it after its first use, so
// the first node each thread relaxes sees omega_g = 1 in its source term
// (thread-count dependent in the reference); the fixtures exclude the light
// cone of that node.  Timing runs may use every host thread.
#include <omp.h>

#include <cstring>

#include "mkFluidsUser.h"

namespace {
double g_W0 = 1.0;
const mkLattice* g_lat = nullptr;
int g_threads = 1;
double g_loop_seconds = 0.0;
}  // namespace

mkReal mkPDFs::density() const {
  mkReal s = 0;
  for (int i = 0; i < QF; ++i) s += v[i];
  return s;
}

mkVector3d mkPDFs::velocity(const mkReal& rho) const {
  mkVector3d j;
  for (int i = 0; i < QF; ++i) j += g_lat->c[i] * v[i];
  return j / rho;
}

mkPDFs mkPDFs::operator+(const mkPDFs& o) const {
  mkPDFs r;
  for (int i = 0; i < QF; ++i) r.v[i] = v[i] + o.v[i];
  return r;
}

mkPDFs mkPDFs::operator-(const mkPDFs& o) const {
  mkPDFs r;
  for (int i = 0; i < QF; ++i) r.v[i] = v[i] - o.v[i];
  return r;
}

mkPDFs mkPDFs::operator*(mkReal s) const {
  mkPDFs r;
  for (int i = 0; i < QF; ++i) r.v[i] = v[i] * s;
  return r;
}

void mkLattice::initialize(const mkReal&) {
  int n = 0;
  auto add = [&](int x, int y, int z, double w) {
    e[n][0] = x, e[n][1] = y, e[n][2] = z;
    c[n] = mkVector3d(x, y, z);
    weight[n] = w;
    ++n;
  };
  add(0, 0, 0, QF == 9 ? 4.0 / 9.0 : 1.0 / 3.0);
  const double wa = QF == 9 ? 1.0 / 9.0 : 1.0 / 18.0, wd = 1.0 / 36.0;
  for (int a = 0; a < (QF == 9 ? 2 : 3); ++a)
    for (int s = 1; s >= -1; s -= 2) add(a == 0 ? s : 0, a == 1 ? s : 0, a == 2 ? s : 0, wa);
  for (int a = 0; a < (QF == 9 ? 1 : 3); ++a)  // diagonals of the planes xy, xz, yz
    for (int s = 1; s >= -1; s -= 2)
      for (int t = 1; t >= -1; t -= 2) {
        const int p = a == 2 ? 1 : 0, q = a == 0 ? 1 : 2;
        int d[3] = {0, 0, 0};
        d[p] = s;
        d[q] = t;
        add(d[0], d[1], d[2], wd);
      }
  for (int i = 0; i < QF; ++i)
    for (int k = 0; k < QF; ++k)
      if (e[k][0] == -e[i][0] && e[k][1] == -e[i][1] && e[k][2] == -e[i][2]) inv[i] = k;
  cs_squ = 1.0 / 3.0;
  g_lat = this;
}

mkPDFs mkNode::getEquPDFs(const mkReal& rho, const mkVector3d& u) {
  mkPDFs f;
  const double uu = u.x * u.x + u.y * u.y + u.z * u.z;
  for (int i = 0; i < QF; ++i) {
    const double eu = g_lat->c[i].x * u.x + g_lat->c[i].y * u.y + g_lat->c[i].z * u.z;
    f[i] = g_lat->weight[i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
  }
  return f;
}

mkPDFs mkNode::getAddedPhasePDFs(const mkReal& omega, const mkReal& ph, const mkVector3d& n) {
  mkPDFs f;
  const double lam = (1.0 - ph * ph) / (std::sqrt(2.0) * g_W0);
  for (int i = 0; i < QF; ++i) {
    const double en = g_lat->c[i].x * n.x + g_lat->c[i].y * n.y + g_lat->c[i].z * n.z;
    f[i] = (1.0 - 0.5 * omega) * g_lat->weight[i] * lam * en;
  }
  return f;
}

int mkFluidsLBM::neighbor(const int& x, const int& y, const int& z, const int& i) {
  const int a = (x + lattice.e[i][0] + Mx) % Mx, b = (y + lattice.e[i][1] + My) % My,
            c = (z + lattice.e[i][2] + Mz) % Mz;
  return (a * My + b) * Mz + c;
}

bool mkFluidsLBM::compute_normal_LB(mkVector3d& normal, const int& x, const int& y, const int& z) {
  mkVector3d g;
  for (int i = 0; i < QF; ++i) g += lattice.c[i] * (lattice.weight[i] * node[neighbor(x, y, z, i)].phi);
  normal = -g / (g.length() + epsilon);
  return true;
}

void mkFluidsLBM::reset_flags() {}

// Runs `loops` loops of propagate() + relaxation() on an nx x ny x nz
// periodic domain of `ngr` grains.  phi0 / out: ngr planes of nx*ny*nz
// values, x fastest (the reference's nodes are z fastest).  The populations
// start at rest equilibrium w_i phi_j.  Returns 0, or 1 for a shape the
// lattice cannot run (QF 9 needs nz = 1).
extern "C" int mgref_lattice(void) { return QF; }

// OpenMP threads of the next runs (1 by default: the fixtures' setting).
extern "C" void mgref_set_threads(int n) { g_threads = n > 0 ? n : 1; }

// Wall time of the propagate + relaxation loops of the last run, seconds.
extern "C" double mgref_loop_seconds(void) { return g_loop_seconds; }

extern "C" int mgref_run(int nx, int ny, int nz, int ngr, double W0, const double* phi0, int loops, double* out) {
  if (nx < 1 || ny < 1 || nz < 1 || ngr < 1 || (QF == 9 && nz != 1)) return 1;
  omp_set_num_threads(g_threads);
  g_W0 = W0;
  const int64_t n = (int64_t)nx * ny * nz;
  std::vector<mkNode> nodes((size_t)n);
  mkFluidsUser u;
  u.Mx = nx, u.My = ny, u.Mz = nz;
  u.node = nodes.data();
  u.lattice.initialize(1.0);
  u.phase_number = ngr;
  const mkVector3d rest(0, 0, 0);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        mkNode& q = nodes[(size_t)((x * ny + y) * nz + z)];
        const int64_t m = x + (int64_t)nx * (y + (int64_t)ny * z);
        q.gVec_out.assign(ngr, mkPDFs());
        q.gVec_hlp.assign(ngr, mkPDFs());
        q.gVec_nbr.assign(ngr, mkPDFs());
        q.phiVec.assign(ngr, 0.0);
        q.d_phiVec.assign(ngr, 0.0);
        double agg = ngr - 1.0;
        for (int j = 0; j < ngr; ++j) {
          const double ph = phi0[j * n + m];
          q.phiVec[j] = ph;
          q.gVec_out[j] = q.getEquPDFs(ph, rest);
          agg += ph;
        }
        q.phi = agg;
        q.g_out = q.getEquPDFs(agg, rest);
      }
  const double t0 = omp_get_wtime();
  for (int t = 0; t < loops; ++t) {
    u.propagate();
    u.relaxation();
  }
  g_loop_seconds = omp_get_wtime() - t0;
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        const mkNode& q = nodes[(size_t)((x * ny + y) * nz + z)];
        const int64_t m = x + (int64_t)nx * (y + (int64_t)ny * z);
        for (int j = 0; j < ngr; ++j) out[j * n + m] = q.phiVec[j];
      }
  u.node = nullptr;
  return 0;
}
