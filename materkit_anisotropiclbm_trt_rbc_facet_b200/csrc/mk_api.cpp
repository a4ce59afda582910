// mk_api.cpp — the extern "C" entry points of include/mkb200.h.
//
// Each entry point maps one step of the reference's lifecycle (header of
// include/mkb200.h) onto the device engine.  Failures return an mk_status and
// leave a message in the handle (mk_last_error) or, for calls without a
// handle, in a thread-local slot (mk_last_global_error).  There is no CPU
// fallback: without a CUDA device mk_create* returns MK_ERR_NODEVICE.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mkb200.h"
#include "mk_case.hpp"
#include "mk_engine.hpp"
#include "mk_handle.hpp"
#include "mk_models.hpp"

namespace mka {


// JSON-lines metrics log (mk_set_metrics_log): one object per timed advance
// and per diagnostics call, appended under a process-wide lock.
std::mutex g_metrics_mu;
std::string g_metrics_path;

void metrics_line(const std::string& body) {
  std::lock_guard<std::mutex> lock(g_metrics_mu);
  if (g_metrics_path.empty()) return;
  FILE* f = fopen(g_metrics_path.c_str(), "a");
  if (!f) return;
  fprintf(f, "{%s}\n", body.c_str());
  fclose(f);
}

std::string fmt(const char* k, double v) {
  char b[96];
  snprintf(b, sizeof b, "\"%s\": %.17g", k, v);
  return b;
}

thread_local std::string g_err;

mk_status set_global(mk_status s, const std::string& m) {
  g_err = m;
  return s;
}

mk_status cuda_fail(mk_handle* h, cudaError_t st, const char* where) {
  // clear the runtime's last-error record (a failed allocation leaves it set,
  // and a later launch check would report it again); sticky errors stay
  cudaGetLastError();
  std::string m = std::string(where) + ": " + cudaGetErrorString(st);
  if (h) h->err = m;
  g_err = m;
  if (st == cudaErrorMemoryAllocation) return MK_ERR_OOM;
  return MK_ERR_CUDA;
}

// Entry points a slab handle does not offer (its loop runs through the
// slab protocol, with exchanges between the kernels).
mk_status slab_refuse(mk_handle* h, const char* what) {
  h->err = std::string(what) + ": not available on a slab handle (advance it with mk_slab_run and the exchanges)";
  return MK_ERR_STATE;
}

bool have_device(std::string& why) {
  int n = 0;
  cudaError_t st = cudaGetDeviceCount(&n);
  if (st != cudaSuccess || n == 0) {
    why = std::string("no CUDA device: ") + (st != cudaSuccess ? cudaGetErrorString(st) : "count is 0");
    cudaGetLastError();
    return false;
  }
  return true;
}

mk_status copy_field(mk_handle* h, int field, std::vector<double>& out) {
  cudaError_t st = mke::engine_field(h->e, field);
  if (st == cudaErrorInvalidValue) {
    h->err = "field not available for this model";
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "field");
  out.resize((size_t)h->e.ncell);
  st = cudaMemcpyAsync(out.data(), h->e.field, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "field copy");
  st = cudaStreamSynchronize(h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "field sync");
  return MK_OK;
}

}  // namespace mka

using namespace mka;

namespace mke {
void set_global_error(const std::string& m) { g_err = m; }
}  // namespace mke

extern "C" {

int32_t mk_abi_version(void) { return MKB200_ABI_VERSION; }

mk_status mk_set_device(int32_t device) {
  std::string why;
  if (!have_device(why)) return set_global(MK_ERR_NODEVICE, why);
  cudaError_t st = cudaSetDevice(device);
  if (st != cudaSuccess) return cuda_fail(nullptr, st, "set_device");
  return MK_OK;
}

const char* mk_version_string(void) { return "mkb200 1.0 (sm_100a)"; }

const char* mk_last_global_error(void) { return g_err.c_str(); }

mk_status mk_set_metrics_log(const char* path) {
  std::lock_guard<std::mutex> lock(g_metrics_mu);
  g_metrics_path = path ? path : "";
  if (!g_metrics_path.empty()) {
    FILE* f = fopen(g_metrics_path.c_str(), "a");
    if (!f) {
      g_err = std::string("cannot open metrics log ") + g_metrics_path;
      g_metrics_path.clear();
      return MK_ERR_IO;
    }
    fclose(f);
  }
  return MK_OK;
}

mk_status mk_read_parameters(const char* xml_path, int32_t* max_loops, int32_t* max_frames) {
  if (!xml_path || !max_loops || !max_frames) return set_global(MK_ERR_ARG, "null argument");
  std::string err;
  int l, f;
  if (!mkc::read_parameters(xml_path, &l, &f, err)) return set_global(MK_ERR_XML, err);
  *max_loops = l;
  *max_frames = f;
  return MK_OK;
}

mk_status mk_case_params(const char* xml_path, const mk_options* opt, mk_params* out) {
  if (!xml_path || !out) return set_global(MK_ERR_ARG, "null argument");
  std::string err;
  mk_status s = mkc::resolve_case(xml_path, opt, out, err);
  if (s != MK_OK) return set_global(s, err);
  return MK_OK;
}

mk_status mk_case_initial_field(const mk_params* p, int32_t field, double* out, size_t ncells) {
  if (!p || !out) return set_global(MK_ERR_ARG, "null argument");
  std::string err;
  mk_status s = mkc::validate_params(p, err);
  if (s != MK_OK) return set_global(s, err);
  s = mkc::initial_field(p, field, out, ncells, err);
  if (s != MK_OK) return set_global(s, err);
  return MK_OK;
}

mk_status mk_create(const mk_params* p, mk_handle** out) {
  const Range nvtx_range("mk_create");
  if (!p || !out) return set_global(MK_ERR_ARG, "null argument");
  *out = nullptr;
  std::string err;
  mk_status s = mkc::validate_params(p, err);
  if (s != MK_OK) return set_global(s, err);
  if (!have_device(err)) return set_global(MK_ERR_NODEVICE, err);
  mk_handle* h = new mk_handle();
  int dev = 0;
  cudaGetDevice(&dev);
  cudaError_t st = mke::engine_alloc(h->e, *p, dev, 0, 0, err);
  if (st != cudaSuccess) {
    mk_status r = err.empty() ? cuda_fail(h, st, "allocate") : set_global(MK_ERR_ARG, err);
    mke::engine_free(h->e);
    delete h;
    return r;
  }
  // initial state (initialize + initialize_geometry)
  const size_t n = (size_t)h->e.ncell;
  const bool flow = p->model == MK_MODEL_FLOW || p->model == MK_MODEL_CONVECTION;
  const bool scalar = p->model == MK_MODEL_THERMAL_DENDRITE || p->model == MK_MODEL_SOLUTAL_DENDRITE ||
                      p->model == MK_MODEL_CONVECTION || mkm::flow_coupled(p->model) ||
                      p->model == MK_MODEL_MULTIGRAIN;
  std::vector<double> phi(flow ? 0 : n), temp(scalar ? n : 0), rho(flow ? n : 0);
  if (!flow) mkc::initial_field(p, MK_FIELD_PHI, phi.data(), n, err);
  if (scalar) mkc::initial_field(p, MK_FIELD_T, temp.data(), n, err);
  if (flow) mkc::initial_field(p, MK_FIELD_RHO, rho.data(), n, err);
  st = mke::engine_set_state(h->e, flow ? nullptr : phi.data(), scalar ? temp.data() : nullptr,
                             flow ? rho.data() : nullptr, nullptr, nullptr, nullptr);
  if (st != cudaSuccess) {
    mk_status r = cuda_fail(h, st, "initialise");
    mke::engine_free(h->e);
    delete h;
    return r;
  }
  *out = h;
  return MK_OK;
}

mk_status mk_create_from_xml(const char* xml_path, const mk_options* opt, mk_handle** out) {
  if (!xml_path || !out) return set_global(MK_ERR_ARG, "null argument");
  mk_params p;
  mk_status s = mk_case_params(xml_path, opt, &p);
  if (s != MK_OK) return s;
  s = mk_create(&p, out);
  if (s == MK_OK && opt && (opt->block_x > 0 || opt->block_y > 0)) {
    const int bx = opt->block_x > 0 ? opt->block_x : (*out)->e.block_x;
    const int by = opt->block_y > 0 ? opt->block_y : 256 / bx;
    if (bx * by > 1024 || bx % 32 != 0 || by < 1) {
      mk_destroy(*out);
      *out = nullptr;
      return set_global(MK_ERR_ARG, "block shape must be a multiple of 32 in x and at most 1024 threads");
    }
    (*out)->e.block_x = bx;
    (*out)->e.block_y = by;
  }
  return s;
}

mk_status mk_destroy(mk_handle* h) {
  if (!h) return MK_ERR_ARG;
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  mke::engine_free(h->e);
  delete h;
  return MK_OK;
}

const char* mk_last_error(const mk_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

mk_status mk_get_params(const mk_handle* h, mk_params* out) {
  if (!h || !out) return MK_ERR_ARG;
  *out = h->e.p;
  return MK_OK;
}

int64_t mk_get_step(const mk_handle* h) { return h ? h->e.step : -1; }

mk_status mk_advance(mk_handle* h, int64_t nsteps) {
  const Range nvtx_range("mk_advance");
  if (!h || nsteps < 0) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_advance");
  for (int64_t t = 0; t < nsteps; ++t) {
    cudaError_t st = mke::engine_step(h->e, nullptr);
    if (st != cudaSuccess) return cuda_fail(h, st, "advance");
  }
  return MK_OK;
}

mk_status mk_advance_graph(mk_handle* h, int64_t nsteps) {
  const Range nvtx_range("mk_advance_graph");
  if (!h || nsteps < 0) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_advance_graph");
  mke::Engine& e = h->e;
  int64_t left = nsteps;
  if (left > 0 && e.wave_skip >= 0) {
    // a pending test fault (mk_inject_fault) applies to one eager loop only
    const mk_status s = mk_advance(h, 1);
    if (s != MK_OK) return s;
    --left;
  }
  if (left > 0 && e.mpending_set) {
    // dynamic solids change at an even loop count: reach one eagerly
    if (e.step & 1) {
      const mk_status s = mk_advance(h, 1);
      if (s != MK_OK) return s;
      --left;
    }
    cudaError_t st = mke::mp_apply_solids(e);
    if (st != cudaSuccess) return cuda_fail(h, st, "dynamic solids");
  }
  while (left >= 2) {
    const int par = (int)(e.step & 1);
    for (int attempt = 0; !h->graph[par]; ++attempt) {
      const int64_t step0 = e.step, l0 = e.launches;
      const int cur0 = e.phi_cur;
      cudaGraph_t g = nullptr;
      cudaError_t st = cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal);
      if (st != cudaSuccess) return cuda_fail(h, st, "capture begin");
      e.capturing = 1;
      mke::engine_step(e, nullptr);
      mke::engine_step(e, nullptr);
      e.capturing = 0;
      st = cudaStreamEndCapture(e.stream, &g);
      e.step = step0;
      e.launches = l0;
      e.phi_cur = cur0;
      if (st == cudaSuccess) {
        st = cudaGraphInstantiate(&h->graph[par], g, 0);
        cudaGraphDestroy(g);
      }
      if (st != cudaSuccess) {
        if (attempt == 0 && e.wave) {
          // the fused loop's cooperative launch could not be captured: the
          // graph takes the two-kernel loop instead
          cudaGetLastError();
          e.wave = 0;
          for (auto& gx : h->graph)
            if (gx) {
              cudaGraphExecDestroy(gx);
              gx = nullptr;
            }
          continue;
        }
        return cuda_fail(h, st, "graph capture");
      }
    }
    cudaError_t st = cudaGraphLaunch(h->graph[par], e.stream);
    if (st != cudaSuccess) return cuda_fail(h, st, "graph launch");
    e.step += 2;
    e.launches += 2 * mke::engine_launches_per_step(e);
    left -= 2;
  }
  if (left) return mk_advance(h, left);
  return MK_OK;
}

// After the stream is idle: report a bounded device wait of the fused
// multiphase loop that ran out since the last check.
mk_status check_waits(mk_handle* h) {
  bool timed_out = false;
  cudaError_t st = mke::engine_check_waits(h->e, &timed_out);
  if (st != cudaSuccess) return cuda_fail(h, st, "wait check");
  if (timed_out) {
    h->err = "a bounded device wait of the fused multiphase loop ran out (a tile's phi planes were never "
             "published); the loops since the last check are invalid";
    return MK_ERR_TIMEOUT;
  }
  return MK_OK;
}

mk_status mk_sync(mk_handle* h) {
  if (!h) return MK_ERR_ARG;
  cudaError_t st = cudaStreamSynchronize(h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "sync");
  return check_waits(h);
}

mk_status mk_set_fused(mk_handle* h, int32_t fused) {
  if (!h) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_set_fused");
  if (fused < 0 || fused > 1) {
    h->err = "loop form must be 0 or 1";
    return MK_ERR_ARG;
  }
  if (fused && !h->e.wave_ok) {
    h->err = "this case does not admit the fused multiphase loop (multiphase model, x extent a multiple of 4, "
             "at least 8 planes in z)";
    return MK_ERR_ARG;
  }
  if (fused != h->e.wave) {
    h->e.wave = fused;
    for (auto& g : h->graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  return MK_OK;
}

int32_t mk_get_fused(const mk_handle* h) { return h && h->e.wave_ok && h->e.wave ? 1 : 0; }

mk_status mk_set_row_staging(mk_handle* h, int32_t on) {
  if (!h) return MK_ERR_ARG;
  if (on < 0 || on > 1) {
    h->err = "row staging must be 0 or 1";
    return MK_ERR_ARG;
  }
  if (on && !h->e.rows_ok) {
    h->err = "this case does not admit the row-staged collision (multiphase model, x rows of at most 256 cells "
             "and a multiple of 16 bytes)";
    return MK_ERR_ARG;
  }
  if (on != h->e.rows) {
    h->e.rows = on;
    for (auto& g : h->graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  return MK_OK;
}

int32_t mk_get_row_staging(const mk_handle* h) { return h && h->e.rows_ok && h->e.rows ? 1 : 0; }

namespace {

bool couple_ok(const mke::Engine& f, const mke::Engine& d) {
  const int dm = d.p.model;
  return f.p.model == MK_MODEL_MULTIPHASE && (dm == MK_MODEL_THERMAL_DENDRITE || dm == MK_MODEL_SOLUTAL_DENDRITE) &&
         f.nx == d.nx && f.ny == d.ny && f.nz == d.nz && f.device == d.device && !f.slab && !d.slab;
}

void drop_graphs(mk_handle* h) {
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

}  // namespace

mk_status mk_update_geometry(mk_handle* flow, mk_handle* dendrite) {
  const Range nvtx_range("mk_update_geometry");
  if (!flow || !dendrite) return MK_ERR_ARG;
  if (!couple_ok(flow->e, dendrite->e)) {
    flow->err = "update_geometry: a multiphase handle and a thermal or solutal dendrite handle of one grid and device";
    return MK_ERR_ARG;
  }
  mke::Engine& f = flow->e;
  const bool fresh = !f.msolid;
  // the dendrite's current phi, ordered before the flow's next work
  cudaError_t st = cudaStreamSynchronize(dendrite->e.stream);
  if (st != cudaSuccess) return cuda_fail(dendrite, st, "update_geometry");
  const mke::Engine& d = dendrite->e;
  st = mke::mp_solid_from_phi(f, d.phi[d.phi_cur], d.phi_elem == 8 ? 1 : 0);
  if (st == cudaSuccess) st = cudaStreamSynchronize(f.stream);  // done with the dendrite's phi
  if (st != cudaSuccess) return cuda_fail(flow, st, "update_geometry");
  if (fresh) drop_graphs(flow);  // the captured geometry had no solids
  return MK_OK;
}

mk_status mk_update_velocity(mk_handle* dendrite, mk_handle* flow) {
  const Range nvtx_range("mk_update_velocity");
  if (!flow || !dendrite) return MK_ERR_ARG;
  if (!couple_ok(flow->e, dendrite->e)) {
    dendrite->err = "update_velocity: a thermal or solutal dendrite handle and a multiphase handle of one grid and device";
    return MK_ERR_ARG;
  }
  const bool fresh = !dendrite->e.vel;
  cudaError_t st = mke::engine_set_velocity(dendrite->e, flow->e);
  if (st != cudaSuccess) return cuda_fail(dendrite, st, "update_velocity");
  if (fresh) drop_graphs(dendrite);  // the captured loop had no advection
  return MK_OK;
}

mk_status mk_get_tuning(const mk_handle* h, mk_tuning* out) {
  if (!h || !out) return MK_ERR_ARG;
  const mke::Engine& e = h->e;
  out->block_x = e.block_x;
  out->block_y = e.block_y;
  out->minb = e.minb;
  out->fused = e.wave_ok && e.wave ? 1 : 0;
  out->row_staged = e.rows_ok && e.rows ? 1 : 0;
  out->phi_tile = e.tma_ok && e.tma ? 1 : 0;
  return MK_OK;
}

mk_status mk_set_tuning(mk_handle* h, const mk_tuning* t) {
  if (!h || !t) return MK_ERR_ARG;
  mke::Engine& e = h->e;
  auto bad = [&](const char* m) {
    h->err = std::string("tuning: ") + m;
    return MK_ERR_ARG;
  };
  if (t->block_x < 32 || t->block_x % 32 != 0 || t->block_y < 1 || t->block_x * t->block_y > 1024)
    return bad("block shape must be a multiple of 32 in x and at most 1024 threads");
  if ((t->fused != 0 && t->fused != 1) || (t->row_staged != 0 && t->row_staged != 1) ||
      (t->phi_tile != 0 && t->phi_tile != 1))
    return bad("fused, row_staged and phi_tile are 0 or 1");
  if (t->fused + t->row_staged + t->phi_tile > 1) return bad("at most one of fused, row_staged and phi_tile");
  const int mb_max = e.p.model == MK_MODEL_MULTIPHASE ? 5 : 2;
  if (t->minb < 1 || t->minb > mb_max) return bad("minb must be 1 or 2 (multiphase: 1 to 5)");
  if (t->fused && !e.wave_ok) return bad("this case does not admit the fused multiphase loop");
  if (t->row_staged && !e.rows_ok) return bad("this case does not admit the row-staged collision");
  if (t->phi_tile && !e.tma_ok) return bad("this case does not admit the TMA phi tile (nx a multiple of 4, no slab)");
  if (t->fused && e.slab) return slab_refuse(h, "mk_set_tuning (fused)");
  e.block_x = t->block_x;
  e.block_y = t->block_y;
  e.minb = t->minb;
  e.wave = t->fused;
  e.rows = t->row_staged;
  e.tma = t->phi_tile;
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  return MK_OK;
}

mk_status mk_inject_fault(mk_handle* h, int32_t kind) {
  if (!h) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_inject_fault");
  if (kind != 1) {
    h->err = "unknown fault kind";
    return MK_ERR_ARG;
  }
  if (!(h->e.wave && h->e.wave_ok)) {
    h->err = "fault kind 1 needs a case that runs the fused multiphase loop";
    return MK_ERR_ARG;
  }
  h->e.wave_skip = 0;
  return MK_OK;
}

mk_status mk_get_stream(mk_handle* h, void** stream) {
  if (!h || !stream) return MK_ERR_ARG;
  *stream = (void*)h->e.stream;
  return MK_OK;
}

mk_status mk_get_field(mk_handle* h, int32_t field, int32_t dtype, void* host_dst, size_t bytes) {
  const Range nvtx_range("mk_get_field");
  if (!h || !host_dst) return MK_ERR_ARG;
  const size_t n = (size_t)h->e.ncell;
  const size_t need = n * (dtype == MK_DTYPE_F64 ? 8 : 4);
  if (dtype != MK_DTYPE_F64 && dtype != MK_DTYPE_F32) {
    h->err = "dtype must be MK_DTYPE_F64 or MK_DTYPE_F32";
    return MK_ERR_ARG;
  }
  if (bytes < need) {
    h->err = "destination buffer too small";
    return MK_ERR_ARG;
  }
  cudaError_t st = dtype == MK_DTYPE_F64 ? mke::engine_field(h->e, field) : mke::engine_field_f32(h->e, field);
  if (st == cudaErrorInvalidValue) {
    h->err = "field not available for this model";
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "field");
  const void* src = dtype == MK_DTYPE_F64 ? (const void*)h->e.field : (const void*)h->e.field32;
  st = cudaMemcpyAsync(host_dst, src, need, cudaMemcpyDeviceToHost, h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "field copy");
  st = cudaStreamSynchronize(h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "field sync");
  return MK_OK;
}

mk_status mk_get_grain_field(mk_handle* h, int32_t grain, int32_t dtype, void* host_dst, size_t bytes) {
  if (!h || !host_dst) return MK_ERR_ARG;
  const size_t n = (size_t)h->e.ncell;
  if (dtype != MK_DTYPE_F64 && dtype != MK_DTYPE_F32) {
    h->err = "dtype must be MK_DTYPE_F64 or MK_DTYPE_F32";
    return MK_ERR_ARG;
  }
  const size_t need = n * (dtype == MK_DTYPE_F64 ? 8 : 4);
  if (bytes < need) {
    h->err = "destination buffer too small";
    return MK_ERR_ARG;
  }
  cudaError_t st = mke::engine_grain_field(h->e, grain);
  if (st == cudaErrorInvalidValue) {
    h->err = "not a multigrain case, or grain index out of range";
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "grain field");
  if (dtype == MK_DTYPE_F32) {
    std::vector<double> tmp(n);
    st = cudaMemcpyAsync(tmp.data(), h->e.field, n * sizeof(double), cudaMemcpyDeviceToHost, h->e.stream);
    if (st == cudaSuccess) st = cudaStreamSynchronize(h->e.stream);
    if (st != cudaSuccess) return cuda_fail(h, st, "grain field copy");
    float* out = (float*)host_dst;
    for (size_t c = 0; c < n; ++c) out[c] = (float)tmp[c];
    return MK_OK;
  }
  st = cudaMemcpyAsync(host_dst, h->e.field, need, cudaMemcpyDeviceToHost, h->e.stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "grain field copy");
  return MK_OK;
}

mk_status mk_set_state(mk_handle* h, const double* phi, const double* temp, const double* conc, const double* rho,
                       const double* ux, const double* uy, const double* uz) {
  if (!h) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_set_state");
  const mk_params& p = h->e.p;
  const size_t n = (size_t)h->e.ncell;
  std::string err;
  std::vector<double> dphi, dt;
  if (!phi) {
    dphi.resize(n);
    mkc::initial_field(&p, MK_FIELD_PHI, dphi.data(), n, err);
    phi = dphi.data();
  }
  const double* tt = mkm::solutal(p.model) ? conc : temp;
  if (!tt) {
    dt.resize(n);
    mkc::initial_field(&p, MK_FIELD_T, dt.data(), n, err);
    tt = dt.data();
  }
  cudaError_t st = mke::engine_set_state(h->e, phi, tt, rho, ux, uy, uz);
  if (st != cudaSuccess) return cuda_fail(h, st, "set_state");
  return MK_OK;
}

mk_status mk_set_state_f32(mk_handle* h, const float* phi, const float* temp, const float* conc) {
  if (!h) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_set_state_f32");
  const mk_params& p = h->e.p;
  const size_t n = (size_t)h->e.ncell;
  std::string err;
  std::vector<float> dphi;
  if (!phi) {  // keep the case's initial order parameter
    std::vector<double> tmp(n);
    mkc::initial_field(&p, MK_FIELD_PHI, tmp.data(), n, err);
    dphi.assign(tmp.begin(), tmp.end());
    phi = dphi.data();
  }
  const float* tt = mkm::solutal(p.model) ? conc : temp;
  cudaError_t st = mke::engine_set_state_f32(h->e, phi, tt);
  if (st == cudaSuccess) st = cudaStreamSynchronize(h->e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "set_state_f32");
  return MK_OK;
}

mk_status mk_write_vtk(mk_handle* h, int64_t loops, const char* dir) {
  const Range nvtx_range("mk_write_vtk");
  if (!h || !dir) return MK_ERR_ARG;
  const mk_params& p = h->e.p;
  const int64_t n = h->e.ncell;
  const int m = p.model;
  std::vector<double> rho(n, 1.0), grain(n, 0.0), phi(n, 0.0), dphi(n, 0.0), conc(n, 0.0), temp(n, 0.0), ux(n, 0.0),
      uy(n, 0.0), uz(n, 0.0);
  mk_status s;
  if (m == MK_MODEL_FLOW || m == MK_MODEL_MULTIPHASE || m == MK_MODEL_CONVECTION || mkm::flow_coupled(m)) {
    if ((s = copy_field(h, MK_FIELD_RHO, rho)) != MK_OK) return s;
    if ((s = copy_field(h, MK_FIELD_UX, ux)) != MK_OK) return s;
    if ((s = copy_field(h, MK_FIELD_UY, uy)) != MK_OK) return s;
    if ((s = copy_field(h, MK_FIELD_UZ, uz)) != MK_OK) return s;
  }
  if ((s = copy_field(h, MK_FIELD_GRAIN, grain)) != MK_OK) return s;
  if ((s = copy_field(h, MK_FIELD_PHI, phi)) != MK_OK) return s;
  if (m == MK_MODEL_CONVECTION && (s = copy_field(h, MK_FIELD_T, temp)) != MK_OK) return s;
  if (mkm::dendrite(m) || m == MK_MODEL_MULTIGRAIN) {
    const bool th = !mkm::solutal(m);
    if ((s = copy_field(h, MK_FIELD_DPHI, dphi)) != MK_OK) return s;
    if ((s = copy_field(h, th ? MK_FIELD_T : MK_FIELD_C, th ? temp : conc)) != MK_OK) return s;
  }
  std::ostringstream fn;
  fn << dir << "/fluid_t" << loops << ".vtk";
  std::ofstream o(fn.str().c_str());
  if (!o) {
    h->err = "cannot open " + fn.str();
    return MK_ERR_IO;
  }
  // Format of MaterKit/src/mkFluidsUser.cpp:728-939 (x fastest, default stream precision).
  o << "# vtk DataFile Version 3.0\n";
  o << "fluid_state\n";
  o << "ASCII\n";
  o << "DATASET RECTILINEAR_GRID\n";
  o << "DIMENSIONS " << p.nx << " " << p.ny << " " << p.nz << "\n";
  o << "X_COORDINATES " << p.nx << " float\n";
  for (int x = 0; x < p.nx; ++x) o << x + 0.5 << " ";
  o << "\n";
  o << "Y_COORDINATES " << p.ny << " float\n";
  for (int y = 0; y < p.ny; ++y) o << y + 0.5 << " ";
  o << "\n";
  o << "Z_COORDINATES " << p.nz << " float\n";
  for (int z = 0; z < p.nz; ++z) o << z + 0.5 << " ";
  o << "\n";
  o << "POINT_DATA " << n << "\n";
  auto scal = [&](const char* name, const std::vector<double>& v) {
    o << "SCALARS " << name << " float 1\n";
    o << "LOOKUP_TABLE default\n";
    for (int64_t c = 0; c < n; ++c) o << v[c] << "\n";
  };
  std::vector<double> tmp(n);
  for (int64_t c = 0; c < n; ++c) tmp[c] = rho[c] - 1;
  scal("density_difference", tmp);
  scal("grain_id", grain);
  scal("order_parameter", phi);
  scal("delta_order_parameter", dphi);
  scal("X0_solutes", conc);
  scal("X0_potentials", conc);
  const double kp = p.k_part;
  for (int64_t c = 0; c < n; ++c) tmp[c] = (conc[c] * (1 - kp) + 1) * 0.5 * (1 + kp - (1 - kp) * phi[c]);
  scal("X0_solutes_dim", tmp);
  scal("temperature", temp);
  o << "VECTORS velocity_vector float\n";
  for (int64_t c = 0; c < n; ++c) o << ux[c] << " " << uy[c] << " " << uz[c] << "\n";
  o.close();
  if (!o) {
    h->err = "write failed for " + fn.str();
    return MK_ERR_IO;
  }
  return MK_OK;
}

mk_status mk_interface_points(mk_handle* h, double iso, double* xyz, double* scalar, int64_t capacity,
                              int64_t* count) {
  if (!h || !count || capacity < 0 || (capacity > 0 && !xyz)) return MK_ERR_ARG;
  cudaError_t st = mke::engine_interface(h->e, iso, xyz, scalar, capacity, count);
  if (st == cudaErrorInvalidValue) {
    h->err = "this model has no order parameter";
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "interface_points");
  return MK_OK;
}

mk_status mk_tip_track(mk_handle* h, int32_t seed, double iso, mk_tip* out) {
  if (!h || !out) return MK_ERR_ARG;
  double len[6];
  cudaError_t st = mke::engine_tip(h->e, seed, iso, len);
  if (st == cudaErrorInvalidValue) {
    h->err = "no order parameter, or seed index out of range";
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "tip_track");
  const int64_t step = h->e.step;
  const bool prev = h->tip_step >= 0 && h->tip_seed == seed && h->tip_iso == iso && step > h->tip_step;
  out->step = step;
  for (int q = 0; q < 6; ++q) {
    out->length[q] = len[q];
    out->velocity[q] = prev ? (len[q] - h->tip_len[q]) / (double)(step - h->tip_step) : 0.0;
    h->tip_len[q] = len[q];
  }
  h->tip_step = step;
  h->tip_seed = seed;
  h->tip_iso = iso;
  return MK_OK;
}

mk_status mk_diagnostics(mk_handle* h, mk_diag* out) {
  const Range nvtx_range("mk_diagnostics");
  if (!h || !out) return MK_ERR_ARG;
  double v[mke::DG_N];
  cudaError_t st = mke::engine_diag(h->e, v);
  if (st != cudaSuccess) return cuda_fail(h, st, "diagnostics");
  const mk_status w = check_waits(h);
  if (w != MK_OK) return w;
  std::memset(out, 0, sizeof(*out));
  out->step = h->e.step;
  out->mass = v[mke::DG_MASS];
  out->momentum[0] = v[mke::DG_MX];
  out->momentum[1] = v[mke::DG_MY];
  out->momentum[2] = v[mke::DG_MZ];
  out->phi_sum = v[mke::DG_PHI];
  out->solid_frac = v[mke::DG_FLUID] > 0 ? v[mke::DG_SOLID] / v[mke::DG_FLUID] : 0.0;
  out->heat = v[mke::DG_HEAT];
  out->solute = v[mke::DG_SOLUTE];
  out->max_speed = v[mke::DG_MAXU];
  out->n_bad = (int32_t)v[mke::DG_BAD];
  if (!h->have_d0) {
    h->have_d0 = true;
    h->d0_mass = out->mass;
    h->d0_phi = out->phi_sum;
  }
  metrics_line("\"event\": \"diagnostics\", " + fmt("model", h->e.p.model) + ", " + fmt("step", (double)out->step) +
               ", " + fmt("mass", out->mass) + ", " + fmt("phi_sum", out->phi_sum) + ", " +
               fmt("mass_drift", h->d0_mass != 0 ? (out->mass - h->d0_mass) / h->d0_mass : 0.0) + ", " +
               fmt("phi_drift", h->d0_phi != 0 ? (out->phi_sum - h->d0_phi) / h->d0_phi : 0.0) + ", " +
               fmt("solid_frac", out->solid_frac) + ", " + fmt("max_speed", out->max_speed) + ", " +
               fmt("n_bad", out->n_bad));
  if (out->n_bad > 0) {
    h->err = "diverged: non-finite or non-positive state in " + std::to_string(out->n_bad) + " cells";
    return MK_ERR_DIVERGED;
  }
  return MK_OK;
}

mk_status mk_nusselt(mk_handle* h, double* nu) {
  if (!h || !nu) return MK_ERR_ARG;
  const mk_params& p = h->e.p;
  if (p.model != MK_MODEL_CONVECTION) {
    h->err = "Nusselt number: convection cases only";
    return MK_ERR_ARG;
  }
  const double dT = p.wall_value[0] - p.wall_value[1];
  if (dT == 0.0) {
    h->err = "Nusselt number: the plates hold the same value";
    return MK_ERR_ARG;
  }
  double v[mke::DG_N];
  cudaError_t st = mke::engine_diag(h->e, v);
  if (st != cudaSuccess) return cuda_fail(h, st, "nusselt");
  const int a = p.wall_axis;
  const int n3[3] = {p.nx, p.ny, p.nz};
  const double H = p.bc[a] == MK_BC_WALLS ? n3[a] - 2 : n3[a];
  // Nu = 1 + <u_a T> H / (kappa dT): the convective part of the heat flux
  // across the layer over the conductive flux kappa dT / H
  *nu = 1.0 + (v[mke::DG_FLUX] / v[mke::DG_FLUID]) * H / (p.D * dT);
  return MK_OK;
}

// Checkpoint layout: magic, version, params hash, step, phi_cur, precision,
// byte counts, then raw population planes, phi buffers and T/U, the FP32 rest
// plane (16-bit multiphase) and the flow lattice of the flow + dendrite model
// (sizes implied by the parameters the hash covers).
static const char kMagic[8] = {'M', 'K', 'B', '2', '0', '0', 'C', 'K'};

mk_status mk_checkpoint(mk_handle* h, const char* path) {
  const Range nvtx_range("mk_checkpoint");
  if (!h || !path) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_checkpoint");
  mke::Engine& e = h->e;
  cudaError_t st = cudaStreamSynchronize(e.stream);
  if (st != cudaSuccess) return cuda_fail(h, st, "checkpoint sync");
  FILE* f = fopen(path, "wb");
  if (!f) {
    h->err = std::string("cannot open ") + path;
    return MK_ERR_IO;
  }
  const uint64_t hash = mkc::params_hash(&e.p);
  const int32_t ver = 1, prec = e.p.precision, cur = e.phi_cur;
  const int64_t step = e.step;
  const uint64_t b0 = mke::engine_pop_bytes(e, 0), b1 = mke::engine_pop_bytes(e, 1);
  const uint64_t bp = (uint64_t)e.ncell * e.phi_elem;
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&hash, 8, 1, f) == 1 &&
            fwrite(&step, 8, 1, f) == 1 && fwrite(&cur, 4, 1, f) == 1 && fwrite(&prec, 4, 1, f) == 1 &&
            fwrite(&b0, 8, 1, f) == 1 && fwrite(&b1, 8, 1, f) == 1 && fwrite(&bp, 8, 1, f) == 1;
  std::vector<char> buf;
  auto dump = [&](const void* dptr, uint64_t bytes) {
    if (!ok || !dptr || !bytes) return;
    buf.resize(bytes);
    if (cudaMemcpy(buf.data(), dptr, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
      ok = false;
      return;
    }
    ok = fwrite(buf.data(), 1, bytes, f) == bytes;
  };
  dump(e.pop0, b0);
  dump(e.pop1, b1);
  dump(e.phi[0], bp);
  dump(e.phi[1], e.phi[1] ? bp : 0);
  dump(e.temp, e.temp ? bp : 0);
  dump(e.rest1, e.rest1 ? (uint64_t)e.ncell * sizeof(float) : 0);
  dump(e.pop2, mke::engine_pop_bytes(e, 2));
  dump(e.phij, e.phij ? (uint64_t)e.p.n_objects * bp : 0);
  fclose(f);
  if (!ok) {
    h->err = std::string("checkpoint write failed: ") + path;
    return MK_ERR_IO;
  }
  return MK_OK;
}

mk_status mk_restore(mk_handle* h, const char* path) {
  const Range nvtx_range("mk_restore");
  if (!h || !path) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_restore");
  mke::Engine& e = h->e;
  FILE* f = fopen(path, "rb");
  if (!f) {
    h->err = std::string("cannot open ") + path;
    return MK_ERR_IO;
  }
  char mg[8];
  int32_t ver = 0, prec = 0, cur = 0;
  uint64_t hash = 0, b0 = 0, b1 = 0, bp = 0;
  int64_t step = 0;
  bool ok = fread(mg, 1, 8, f) == 8 && std::memcmp(mg, kMagic, 8) == 0 && fread(&ver, 4, 1, f) == 1 && ver == 1 &&
            fread(&hash, 8, 1, f) == 1 && fread(&step, 8, 1, f) == 1 && fread(&cur, 4, 1, f) == 1 &&
            fread(&prec, 4, 1, f) == 1 && fread(&b0, 8, 1, f) == 1 && fread(&b1, 8, 1, f) == 1 &&
            fread(&bp, 8, 1, f) == 1;
  if (!ok) {
    fclose(f);
    h->err = "not a checkpoint or truncated header";
    return MK_ERR_IO;
  }
  if (hash != mkc::params_hash(&e.p) || prec != e.p.precision || b0 != mke::engine_pop_bytes(e, 0) ||
      b1 != mke::engine_pop_bytes(e, 1) || bp != (uint64_t)e.ncell * e.phi_elem || step < 0 || (cur != 0 && cur != 1)) {
    fclose(f);
    h->err = "checkpoint does not match this case (parameters, precision or sizes differ)";
    return MK_ERR_ARG;
  }
  std::vector<char> buf;
  auto load = [&](void* dptr, uint64_t bytes) {
    if (!ok || !dptr || !bytes) return;
    buf.resize(bytes);
    if (fread(buf.data(), 1, bytes, f) != bytes) {
      ok = false;
      return;
    }
    ok = cudaMemcpy(dptr, buf.data(), bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  load(e.pop0, b0);
  load(e.pop1, b1);
  load(e.phi[0], bp);
  load(e.phi[1], e.phi[1] ? bp : 0);
  load(e.temp, e.temp ? bp : 0);
  load(e.rest1, e.rest1 ? (uint64_t)e.ncell * sizeof(float) : 0);
  load(e.pop2, mke::engine_pop_bytes(e, 2));
  load(e.phij, e.phij ? (uint64_t)e.p.n_objects * bp : 0);
  fclose(f);
  if (!ok) {
    h->err = "checkpoint truncated";
    return MK_ERR_IO;
  }
  e.step = step;
  e.phi_cur = cur;
  return MK_OK;
}

mk_status mk_profile_steps(mk_handle* h, int64_t nsteps, const char* kernel, double* kernel_ms, double* step_ms,
                           int64_t* kernel_launches) {
  if (!h || nsteps <= 0 || !kernel || !kernel_ms || !step_ms) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_profile_steps");
  mke::Engine& e = h->e;
  const int kps = mke::engine_kernels_per_step(e);
  int slot = -1;
  for (int k = 0; k < kps; ++k)
    if (std::strcmp(mke::engine_kernel_name(e, k), kernel) == 0) slot = k;
  if (slot < 0) {
    h->err = std::string("no kernel named ") + kernel;
    return MK_ERR_ARG;
  }
  const size_t per = (size_t)2 * kps;
  std::vector<cudaEvent_t> ev((size_t)nsteps * per);
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, e.stream);
  for (int64_t s = 0; s < nsteps; ++s) mke::engine_step(e, &ev[(size_t)s * per]);
  cudaEventRecord(t1, e.stream);
  cudaError_t st = cudaEventSynchronize(t1);
  double kt = 0;
  if (st == cudaSuccess) {
    for (int64_t s = 0; s < nsteps; ++s) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[(size_t)s * per + 2 * slot], ev[(size_t)s * per + 2 * slot + 1]);
      kt += ms;
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, t0, t1);
    *step_ms = tot;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (st != cudaSuccess) return cuda_fail(h, st, "profile");
  *kernel_ms = kt;
  if (kernel_launches) *kernel_launches = nsteps;
  return MK_OK;
}

mk_status mk_time_advance(mk_handle* h, int64_t nsteps, int32_t use_graph, double* ms) {
  const Range nvtx_range("mk_time_advance");
  if (!h || nsteps < 0 || !ms) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_time_advance");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, h->e.stream);
  mk_status s = use_graph ? mk_advance_graph(h, nsteps) : mk_advance(h, nsteps);
  cudaEventRecord(t1, h->e.stream);
  cudaError_t st = cudaEventSynchronize(t1);
  float f = 0;
  if (st == cudaSuccess) cudaEventElapsedTime(&f, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (s != MK_OK) return s;
  if (st != cudaSuccess) return cuda_fail(h, st, "time_advance");
  *ms = f;
  if (f > 0) {
    const double cells = (double)h->e.ncell;
    metrics_line("\"event\": \"time_advance\", " + fmt("model", h->e.p.model) + ", " +
                 fmt("precision", h->e.p.precision) + ", " + fmt("step", (double)h->e.step) + ", " +
                 fmt("loops", (double)nsteps) + ", " + fmt("ms", f) + ", " +
                 fmt("mlups", cells * nsteps / (f * 1e-3) / 1e6) + ", " +
                 fmt("gbs", mke::engine_bytes_per_cell(h->e) * cells * nsteps / (f * 1e-3) / 1e9) + ", " +
                 fmt("launches_per_loop", mke::engine_kernels_per_step(h->e)));
  }
  return MK_OK;
}

mk_status mk_autotune(mk_handle* h, int32_t trial_steps, int32_t* block_x, int32_t* block_y, int32_t* minb,
                      double* ms_per_step) {
  const Range nvtx_range("mk_autotune");
  if (!h || trial_steps < 1) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_autotune");
  mke::TuneResult r;
  cudaError_t st = mke::engine_autotune(h->e, trial_steps, &r);
  if (st != cudaSuccess) return cuda_fail(h, st, "autotune");
  // captured graphs hold the old launch shape
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  if (block_x) *block_x = r.block_x;
  if (block_y) *block_y = r.block_y;
  if (minb) *minb = r.minb;
  if (ms_per_step) *ms_per_step = r.ms_per_step;
  return MK_OK;
}

mk_status mk_backward(mk_handle* h, const mk_loss* loss, mk_grad* out) {
  const Range nvtx_range("mk_backward");
  if (!h || !loss || !out || !loss->target_phi) return MK_ERR_ARG;
  if (h->e.slab) return slab_refuse(h, "mk_backward");
  std::string err;
  double r[5] = {0, 0, 0, 0, 0};
  cudaError_t st = mke::engine_backward(h->e, loss->target_phi, loss->steps, loss->checkpoint_every, r, err);
  if (st == cudaErrorInvalidValue && !err.empty()) {
    h->err = err;
    return MK_ERR_ARG;
  }
  if (st != cudaSuccess) return cuda_fail(h, st, "backward");
  out->loss = r[0];
  out->d_eps4 = r[1];
  out->d_delta = r[2];
  out->d_tau_t = r[3];
  out->forward_loops = (int64_t)r[4];
  return MK_OK;
}

mk_status mk_host_alloc(size_t bytes, void** out) {
  if (!out) return set_global(MK_ERR_ARG, "null argument");
  cudaError_t st = cudaHostAlloc(out, bytes, cudaHostAllocDefault);
  if (st != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(nullptr, st, "host_alloc");
  }
  return MK_OK;
}

mk_status mk_host_free(void* p) {
  if (!p) return MK_OK;
  cudaError_t st = cudaFreeHost(p);
  if (st != cudaSuccess) return cuda_fail(nullptr, st, "host_free");
  return MK_OK;
}

double mk_bytes_per_cell(const mk_handle* h) { return h ? mke::engine_bytes_per_cell(h->e) : 0.0; }

int64_t mk_fluid_cells(const mk_handle* h) {
  if (!h) return 0;
  const mk_params& p = h->e.p;
  int64_t f[3] = {p.nx, p.ny, p.nz};
  for (int a = 0; a < 3; ++a)
    if (p.bc[a] == MK_BC_WALLS) f[a] -= 2;
  if (h->e.slab) {
    // the owned planes, less the global wall planes among them
    const mke::Engine& e = h->e;
    f[2] = 0;
    for (int z = e.zg0; z < e.zg0 + e.nz - 2; ++z)
      if (p.bc[2] != MK_BC_WALLS || (z != 0 && z != e.nzg - 1)) ++f[2];
  }
  return f[0] * f[1] * f[2];
}

int32_t mk_launches_per_step(const mk_handle* h) { return h ? mke::engine_launches_per_step(h->e) : 0; }

}  // extern "C"
