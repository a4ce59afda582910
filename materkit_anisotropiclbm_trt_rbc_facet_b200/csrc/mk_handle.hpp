// mk_handle.hpp — the handle behind the opaque mk_handle of include/mkb200.h,
// and the error helpers the entry-point files share (mk_api.cpp, mk_slab.cpp).
#ifndef MK_HANDLE_HPP
#define MK_HANDLE_HPP

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>

#include "../../include/mkb200.h"
#include "mk_engine.hpp"

struct mk_handle {
  mke::Engine e;
  std::string err;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two loops captured, keyed by start parity
  // last mk_tip_track result (velocity = change per loop since then)
  int64_t tip_step = -1;
  int32_t tip_seed = -1;
  double tip_iso = 0.0;
  double tip_len[6] = {0, 0, 0, 0, 0, 0};
  // first diagnostics of the handle (reference of the drift in the metrics log)
  bool have_d0 = false;
  double d0_mass = 0.0, d0_phi = 0.0;
};

namespace mka {

// NVTX range around an entry point (visible in Nsight Systems / ncu timelines;
// without a tool attached the push / pop cost a few instructions).
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

// Status with a message in the calling thread's slot (mk_last_global_error).
mk_status set_global(mk_status s, const std::string& m);
// Status of a failed CUDA call, message in the handle (if any) and the
// thread's slot; clears the runtime's last-error record.
mk_status cuda_fail(mk_handle* h, cudaError_t st, const char* where);
// Whether a CUDA device is present (else the reason).
bool have_device(std::string& why);

}  // namespace mka

#endif
