// mk_engine.hpp — internal interface between the C ABI (mk_api.cpp) and the
// kernels (mk_kernels.cu).  Not installed; no torch types anywhere.
#ifndef MK_ENGINE_HPP
#define MK_ENGINE_HPP

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/mkb200.h"

namespace mke {

// Number of FP64 diagnostic accumulators.
enum {
  DG_MASS = 0,
  DG_MX,
  DG_MY,
  DG_MZ,
  DG_PHI,
  DG_SOLID,
  DG_HEAT,
  DG_SOLUTE,
  DG_MAXU,
  DG_BAD,
  DG_FLUID,
  DG_FLUX,  // sum of u_axis T (convection: the convective heat flux across the plates)
  DG_N
};

struct Engine {
  mk_params p;
  int nx, ny, nz;
  int64_t ncell;
  int64_t stride;     // population plane stride in cells
  int elem;           // bytes per stored population
  int phi_elem;       // bytes per phi / temperature value (8 for FP64, else 4)
  int Q0, Q1;         // populations of lattice 0 and 1 (0 if absent)
  int Q2;             // populations of lattice 2: the flow of the flow + dendrite model, else 0
  int64_t step;       // completed loops
  int phi_cur;        // dendrites: index of the current phi buffer
  cudaStream_t stream;
  int device;
  int block_x, block_y;
  int minb;           // occupancy variant of the dominant kernel (1 or 2 resident blocks per SM)
  // device buffers
  void* pop0;
  void* pop1;
  void* pop2;         // flow lattice of the flow + dendrite model (deviations f - w rho0)
  void* vel;          // flow + dendrite: the loop's collision velocity, 3 planes of ncell (phi type), read by
                      // the thermal lattice and the boundary kernel
  void* phij;         // multigrain: the grains' order parameters, N planes of ncell (phi type), else null
  double* gseeds;     // multigrain: x, y, z, R per grain (initial state), else null
  float* rest1;       // FP32 rest population of lattice 1 (multiphase h) with 16-bit storage, else null
  void* phi[2];
  void* temp;
  double* seeds;      // n_objects * 12 doubles: centre (3), rotation (9, row-major, columns = crystal axes)
  void* rot;          // the rotations alone in the arithmetic type (double for FP64, else float)
  unsigned char* grain;  // per-cell nearest-seed index (dendrites with more than one seed), else null
  double* partial;    // diagnostics scratch, DG_N doubles per block
  int partial_blocks;
  double* dsum;       // DG_N doubles
  double* field;      // ncell doubles (field output staging)
  float* field32;     // ncell floats (FP32 field output staging, allocated on first use)
  float* stage32;     // 2 * ncell floats (FP32 state upload staging, allocated on first use)
  // launch counters
  int64_t launches;
  // fused multiphase step: one cooperative launch per loop (k_mp_wave)
  int wave;              // multiphase loop form: 0 phi kernel + collision kernel, 1 fused
  int wave_ok;           // the case admits the fused loop (x extent a multiple of 4, nz >= 8, grid co-resident)
  int wave_sx, wave_sy;  // tiles: 32-cell x segments times y bands
  int wave_rows;         // rows of the tallest band
  int wave_threads;      // threads per CTA
  size_t wave_smem;      // dynamic shared memory (the phi ring)
  unsigned* wave_flags;  // per-tile publication counters (zeroed before every launch)
  int* wave_err;         // error word of the bounded waits (0 = none)
  int wave_skip;         // test hook: tile that publishes nothing in the next fused loop (-1: none)
  // row-staged collision of the two-kernel multiphase loop (k_mp_rows): whole
  // x rows of all 38 populations staged through shared memory by the
  // bulk-copy engine, `rows_ns` rows in flight per CTA
  int rows_ok;           // the case admits it (x rows of at most 256 cells, a multiple of 16 bytes)
  int rows;              // 1: the collision runs row-staged
  int rows_ns, rows_grid, rows_threads;
  size_t rows_stage, rows_smem;
  // collision with its phi tile (and halo) staged by one TMA tensor load per
  // block: the case admits it (the map encoded: nx a multiple of 4, no
  // slab), the form is chosen, and the 3-D tensor map over phi (the driver's
  // 128-byte CUtensorMap)
  int tma_ok;
  int tma;
  alignas(64) unsigned char tma_map[128];
  // dynamic solids of a multiphase flow coupled to a dendrite
  // (mk_update_geometry): the solid flags, the fluid cells next to a solid,
  // and the flags of the next update, applied at the next even loop count
  unsigned char* msolid;
  unsigned char* mnear;
  unsigned char* mpending;
  int mpending_set;
  int capturing;         // a loop is being captured into a graph (no host-side state changes)
  // z-slab of a larger multiphase domain (mk_create_slab): the local planes
  // 1 .. nz - 2 are the global planes zg0 .. zg0 + nz - 3 of nzg planes; the
  // planes 0 and nz - 1 are ghosts filled by the exchanges
  int slab;              // 1 for a slab handle
  int zg0, nzg;          // first owned global plane, global plane count
  int rank, nranks;      // this slab and the slab count
  int slab_next;         // next action of the loop protocol (MK_SLAB_*)
  void* slab_halo;       // the runs a return exchange delivers: 2 faces x 2 lattices x 5 populations x nx ny,
                         // merged into the owned boundary planes by mk_slab_done
};

// Population plane stride of a domain of ncell cells (a multiple of 64 cells).
inline int64_t pop_stride(int64_t ncell) { return (ncell + 63) / 64 * 64; }

// Bytes of one stored population / of one phi value for a storage precision.
inline int pop_elem(int precision) {
  return precision == MK_PREC_FP64 ? 8 : (precision == MK_PREC_FP32 ? 4 : 2);
}
inline int phi_elem_of(int precision) { return precision == MK_PREC_FP64 ? 8 : 4; }

// Message returned by mk_last_global_error on this thread.
void set_global_error(const std::string& m);

// Grain table of a dendrite case: 12 doubles per object (centre, then the
// row-major rotation whose columns are the crystal axes).
void seed_table(const mk_params& p, std::vector<double>& sd);

// Allocate and zero device buffers for p.  Returns cudaSuccess or an error.
cudaError_t engine_alloc(Engine& e, const mk_params& p, int device, int block_x, int block_y, std::string& err);
void engine_free(Engine& e);

// Initialise populations, phi and T/U from host macroscopic fields (ncell
// doubles each; NULL uses the value the case defines as uniform default).
cudaError_t engine_set_state(Engine& e, const double* phi, const double* temp, const double* rho, const double* ux,
                             const double* uy, const double* uz);

// Same from FP32 host arrays (phi and T/U; NULL keeps the uniform default).
cudaError_t engine_set_state_f32(Engine& e, const float* phi, const float* temp);

// Field as FP32 into e.field32 (device).
cudaError_t engine_field_f32(Engine& e, int field);

// One loop.  When `ev` is non-null, ev[2k], ev[2k+1] bracket the k-th kernel.
cudaError_t engine_step(Engine& e, cudaEvent_t* ev);
// Kernel phases of one loop (the profiler's slots) and the launches they take.
int engine_kernels_per_step(const Engine& e);
int engine_launches_per_step(const Engine& e);
const char* engine_kernel_name(const Engine& e, int k);

// Compute a macroscopic field of the current state into e.field (device).
cudaError_t engine_field(Engine& e, int field);
// A thermal or solutal dendrite advected by a multiphase flow of the same
// grid: the flow's velocity into d.vel (allocated on first use), after which
// the dendrite's scalar lattice carries it.  Synchronous.
cudaError_t engine_set_velocity(Engine& d, Engine& f);
// Multigrain: grain j's order parameter into e.field (device).
cudaError_t engine_grain_field(Engine& e, int grain);

// Multiphase loop (mk_multiphase.cu): choose the fused loop's tiling for the
// case (sets wave_ok and the wave_* fields), and launch one loop.
void mp_configure(Engine& e);
void mp_launch(Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev);
// Dynamic solids: set the pending flags from a dendrite's phi (solid where
// phi > 0, cumulative), on the handle's stream; and apply pending flags
// (solid, near) when the loop count is even.  The dendrite's phi is FP64
// (phi_double) or FP32.
cudaError_t mp_solid_from_phi(Engine& e, const void* dend_phi, int phi_double);
cudaError_t mp_apply_solids(Engine& e);

// One kernel of the two-kernel loop at the parity of e.step: part 0 the phi
// kernel, part 1 the collision (slab handles run the loop in its parts, with
// the exchanges between them).
cudaError_t mp_launch_part(Engine& e, int part);

// After a synchronisation: whether a bounded device wait of the fused loop
// gave up since the last check (clears the record).  Returns the CUDA status
// of the read; *timed_out is set when a wait ran out.
cudaError_t engine_check_waits(Engine& e, bool* timed_out);

// FP64 diagnostics (two-pass reduction into e.dsum); host copy in out[DG_N].
cudaError_t engine_diag(Engine& e, double* out);

// Autotuner: times `trial_steps` loops of every candidate launch shape and
// occupancy variant (two warm-up loops, then the faster of two timed repeats)
// on a saved copy of the state, restores the state and keeps the fastest.
// Returns the chosen configuration and its ms per loop.
struct TuneResult {
  int block_x, block_y, minb;
  double ms_per_step;
  int candidates;
};
cudaError_t engine_autotune(Engine& e, int trial_steps, TuneResult* out);

// Raw state for checkpoints: populations in their storage format.
size_t engine_pop_bytes(const Engine& e, int which);

double engine_bytes_per_cell(const Engine& e);

// phi = iso contour points (mk_interface_points) and tip lengths along the
// six axis rays from a seed centre (mk_tip_track); mk_interface.cu.
cudaError_t engine_interface(Engine& e, double iso, double* xyz, double* sc, int64_t capacity, int64_t* count);
cudaError_t engine_tip(Engine& e, int seed, double iso, double out[6]);

// Discrete adjoint of `steps` thermal dendrite loops from the current state
// with checkpoints every `every` loops (<= 0: 100).  out = {loss, dL/deps4,
// dL/dDelta, dL/dtau_T, forward loops run}.  Leaves the state after the
// forward run.  cudaErrorInvalidValue with `err` set for unsupported cases.
cudaError_t engine_backward(Engine& e, const double* h_target, int64_t steps, int64_t every, double* out,
                            std::string& err);

}  // namespace mke

#endif
