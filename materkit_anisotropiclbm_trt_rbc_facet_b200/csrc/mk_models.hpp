// mk_models.hpp — families of solver models (host and device).
#ifndef MK_MODELS_HPP
#define MK_MODELS_HPP

#include "../../include/mkb200.h"

namespace mkm {

// A flow lattice with porous bounce-back and inflow / outflow faces beside the
// phase field (run_flow_thermal_dendrite / run_flow_solutal_dendrite).
inline constexpr bool flow_coupled(int m) { return m == MK_MODEL_FLOW_DENDRITE || m == MK_MODEL_FLOW_SOLUTAL; }
// The scalar lattice is the solutal U-lattice (else thermal).
inline constexpr bool solutal(int m) { return m == MK_MODEL_SOLUTAL_DENDRITE || m == MK_MODEL_FLOW_SOLUTAL; }
// A single phase field with seeds and a thermal or solutal lattice.
inline constexpr bool dendrite(int m) {
  return m == MK_MODEL_THERMAL_DENDRITE || m == MK_MODEL_SOLUTAL_DENDRITE || flow_coupled(m);
}

}  // namespace mkm

#endif
