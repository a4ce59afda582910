// Stand-in declarations for compiling the reference's readable multigrain
// solver, MaterKit/src/mkFluidsUser.cpp, outside its closed library.
//
// Test infrastructure: this header and ref_stub.cpp build oracle/_ref only
// (the fixture generator tests/golden/make_multigrain_ref.py and bench.py's
// CPU baseline legs load it); nothing in the product includes them.  The
// reference's mkFluidsUser.cpp is compiled where it lies and includes
// "mkFluidsUser.h" by name, so this file carries
// exactly the names that source uses (classes, members and functions of
// MaterKit/inc/mkFluidsLBM.h, mkNode.h, mkLattice.h, mkPhaseField.h and
// mkFluidsUser.h) and nothing of the library itself: the bodies of the
// library's functions that the multigrain path calls (lattice, equilibrium,
// the Chai phase-field source, the neighbour wrap, reset_flags) are restated
// in ref_stub.cpp from the published forms, and everything the path does
// not reach is an empty body.  All members are public so the harness can set
// the state up directly.
#ifndef MK_REF_STUB_MKFLUIDSUSER_H
#define MK_REF_STUB_MKFLUIDSUSER_H

#include <cmath>
#include <string>
#include <vector>

// mkFluidsUser.cpp names std::vector unqualified
using namespace std;

// Velocity set of the flow / phase lattices: 9 (D2Q9) is the value the
// reference ships (MaterKit/inc/mkGlobalDefs.h:134); 19 gives the D3Q19 build.
#ifndef QF
#define QF 9
#endif
#define MK_OMP_CHUNKSIZE 16  // MaterKit/inc/mkGlobalDefs.h:18

typedef double mkReal;

// node flags (MaterKit/inc/mkGlobalDefs.h:140-145)
enum { is_fluid = 0, is_solid = 2, is_walls = 3 };

inline mkReal mkSQ(const mkReal& v) { return v * v; }

class mkVector3d {
 public:
  mkReal x = 0, y = 0, z = 0;
  mkVector3d() = default;
  mkVector3d(mkReal a, mkReal b, mkReal c) : x(a), y(b), z(c) {}
  void set(mkReal a, mkReal b, mkReal c) { x = a, y = b, z = c; }
  void set(const mkVector3d& v) { *this = v; }
  mkReal length() const { return std::sqrt(x * x + y * y + z * z); }
  mkVector3d& operator+=(const mkVector3d& v) {
    x += v.x, y += v.y, z += v.z;
    return *this;
  }
  mkVector3d operator-() const { return mkVector3d(-x, -y, -z); }
  mkVector3d operator+(const mkVector3d& v) const { return mkVector3d(x + v.x, y + v.y, z + v.z); }
  mkVector3d operator-(const mkVector3d& v) const { return mkVector3d(x - v.x, y - v.y, z - v.z); }
  mkVector3d operator*(mkReal s) const { return mkVector3d(x * s, y * s, z * s); }
  mkVector3d operator/(mkReal s) const { return mkVector3d(x / s, y / s, z / s); }
};

// QF populations of one node
class mkPDFs {
 public:
  mkReal v[QF] = {};
  mkReal& operator[](int i) { return v[i]; }
  const mkReal& operator[](int i) const { return v[i]; }
  mkReal density() const;
  mkVector3d velocity(const mkReal& rho) const;
  mkPDFs operator+(const mkPDFs& o) const;
  mkPDFs operator-(const mkPDFs& o) const;
  mkPDFs operator*(mkReal s) const;
};

class mkLattice {
 public:
  int inv[QF];
  mkVector3d c[QF];
  int e[QF][3];
  mkPDFs weight;
  mkReal cs_squ = 1.0 / 3.0;
  void initialize(const mkReal& omega);
};

class mkNode {
 public:
  mkPDFs getEquPDFs(const mkReal& rho, const mkVector3d& vel);
  mkPDFs getAddedPhasePDFs(const mkReal& omega, const mkReal& phi, const mkVector3d& normal);
  void initialFlag(int f) { flag = f; }
  int getGrainId() const { return 0; }

  int flag = is_fluid;
  mkPDFs f_out, f_hlp;
  mkVector3d vel;
  double density = 1.0;
  mkPDFs g_out, g_hlp, g_nbr;
  double phi = 0, d_phi = 0;
  std::vector<mkPDFs> gVec_out, gVec_hlp, gVec_nbr;
  std::vector<double> phiVec, d_phiVec;
  double temperature = 0;
  std::vector<double> X_potents, X_solutes;
};

class mkSpace {};

class mkFluidsLBM {
 public:
  mkFluidsLBM() = default;
  explicit mkFluidsLBM(const mkSpace&) {}
  virtual ~mkFluidsLBM() = default;
  void initialize(const std::string&) {}
  int neighbor(const int& x, const int& y, const int& z, const int& i);
  bool compute_normal_LB(mkVector3d& normal, const int& x, const int& y, const int& z);
  void reset_flags();

  mkNode* node = nullptr;
  int Mx = 0, My = 0, Mz = 0;
  mkLattice lattice;
  mkReal omega_f = 1.0;
  mkReal mk_dt = 1.0, mk_dx = 1.0, mk_lambda = 0.0;
  mkReal epsilon = 1e-6;
  int phase_number = 1;
  std::vector<mkReal> mk_X_high = std::vector<mkReal>(1, 0.0), mk_X_low = std::vector<mkReal>(1, 0.0);
  mkVector3d vel_in;
};

class mkFlowField : virtual public mkFluidsLBM {
 public:
  void initialize(const std::string&) {}
};
class mkThermalField : virtual public mkFluidsLBM {
 public:
  void initialize(const std::string&) {}
};
class mkSolutalField : virtual public mkFluidsLBM {
 public:
  void initialize(const std::string&) {}
};
class mkPhaseField : virtual public mkFluidsLBM {
 public:
  void initialize_seeds(const std::string&) {}
};

class mkFluidsMRT : virtual public mkFlowField,
                    virtual public mkThermalField,
                    virtual public mkSolutalField,
                    virtual public mkPhaseField {
 public:
  mkFluidsMRT() = default;
  explicit mkFluidsMRT(const mkSpace&) {}
};

// The method list of MaterKit/inc/mkFluidsUser.h.
class mkFluidsUser : virtual public mkFluidsMRT {
 public:
  mkFluidsUser();
  mkFluidsUser(const mkSpace& space);
  ~mkFluidsUser();
  void initialize(const std::string& xmlfname);
  void initialize_geometry();
  void propagate();
  void relaxation();
  void bdy_constX();
  void bdy_nonflux();
  void bdy_RBC();
  void boundary_vel();
  void boundary_Couette();
};

#endif
