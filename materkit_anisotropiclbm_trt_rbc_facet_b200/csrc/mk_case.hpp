// mk_case.hpp — BoltzTechs XML case → resolved lattice-unit parameters and
// initial fields.  Host code only; no CUDA.
//
// This is the reference's case set-up path: mkSpace(xml) (MaterKit/inc/mkSpace.h:36),
// readParameters (MaterKit/inc/mkFunction.h:62), the per-field initialize(xml)
// (MaterKit/inc/mkFluidsMRT.h:39, mkPhaseField.h:39, mkThermalField.h:31,
// mkFluidsMultiphase.h:30) and initialize_geometry (mkFluidsMRT.h:40).
#ifndef MK_CASE_HPP
#define MK_CASE_HPP

#include <string>
#include <vector>

#include "../../include/mkb200.h"

namespace mkc {

// splitmix64 generator used for every seeded synthetic case.
struct SplitMix64 {
  unsigned long long s;
  explicit SplitMix64(unsigned long long seed) : s(seed) {}
  unsigned long long next() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void default_params(mk_params* p);
void default_options(mk_options* o);

// Read output/numLoops and output/numFrames (readParameters).
bool read_parameters(const std::string& xml, int* loops, int* frames, std::string& err);

// Resolve an XML case with optional overrides.  Returns MK_OK or an error
// status with a message.
mk_status resolve_case(const std::string& xml, const mk_options* opt, mk_params* out, std::string& err);

// Check a parameter set; MK_ERR_ARG with a message when invalid.
mk_status validate_params(const mk_params* p, std::string& err);

// Initial macroscopic field of the case, dense x-fastest.
mk_status initial_field(const mk_params* p, int field, double* out, size_t ncells, std::string& err);

// Whether cell (x,y,z) is fluid under the per-axis boundary kinds.
inline bool is_fluid(const mk_params* p, int x, int y, int z) {
  const int c[3] = {x, y, z};
  const int n[3] = {p->nx, p->ny, p->nz};
  for (int a = 0; a < 3; ++a)
    if (p->bc[a] == MK_BC_WALLS && (c[a] == 0 || c[a] == n[a] - 1)) return false;
  return true;
}

// Seeded solutal ensemble (config 4): n domain parameter sets.
mk_status ensemble_case(unsigned long long seed, int n, int precision, mk_params* out, std::string& err);

// A stable hash of the parameters (checkpoint compatibility).
unsigned long long params_hash(const mk_params* p);

}  // namespace mkc

#endif
