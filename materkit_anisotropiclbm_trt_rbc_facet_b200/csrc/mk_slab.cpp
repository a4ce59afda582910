// mk_slab.cpp — z-slab decomposition of one multiphase domain (the mk_slab_*
// entry points of include/mkb200.h).
//
// A slab owns global planes z0 .. z0 + nown - 1 as its local planes
// 1 .. nown and keeps one ghost plane on each side (local 0 and nown + 1).
// The kernels are the whole-domain ones; the slab geometry (Geom::slab) makes
// the ghost cells non-fluid but valid streaming targets, so every link that
// leaves the slab reads or writes a ghost slot, and the exchanges below move
// exactly those slots between neighbours:
//
//   AA parity    reads across the face          writes across the face
//   even loop    none (own slots)               none
//   odd loop     ghost slots of e_z = -1 (ghost  ghost slots of e_z = -1 (ghost
//                0) and e_z = +1 (top ghost)     0) and e_z = +1 (top ghost)
//
// FILL copies the neighbours' even-loop results into those ghost slots before
// an odd loop; RETURN moves the odd loop's ghost writes to the planes that own
// them.  The initial state is placed as the output of an odd loop, so a slab
// starts with a RETURN.  PHI copies the boundary phi planes after the phi
// kernel of every loop (the collision's gradient and Laplacian stencil).
//
// A RETURN run lands in the slab's halo buffer, not in the owned plane: a slot
// of a boundary plane whose source cell across the face is not fluid (an x or
// y wall column, a cell beyond a closed face, a global wall plane) was written
// by its own cell's bounce-back, and the neighbour's ghost slot there holds
// nothing.  The merge kernel (k_slab_merge, launched by mk_slab_done) copies a
// slot only where the cell's link to its source is open.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mkb200.h"
#include "mk_case.hpp"
#include "mk_device.cuh"
#include "mk_engine.hpp"
#include "mk_handle.hpp"
#include "mk_shared.cuh"

using namespace mka;

namespace {

bool split(int nz, int r, int n, int& z0, int& nown) {
  if (n < 1 || r < 0 || r >= n || nz < n) return false;
  const int q = nz / n, m = nz % n;
  nown = q + (r < m ? 1 : 0);
  z0 = r * q + std::min(r, m);
  return true;
}

// What a plan needs of a slab.
struct SlabGeo {
  int nx, ny, nown, rank, nranks, bc2;
  int64_t stride;
  int elem, phi_elem;
};

SlabGeo geo_of(const mk_params& global, int rank, int nranks, int nown) {
  SlabGeo s;
  s.nx = global.nx;
  s.ny = global.ny;
  s.nown = nown;
  s.rank = rank;
  s.nranks = nranks;
  s.bc2 = global.bc[2];
  s.stride = mke::pop_stride((int64_t)global.nx * global.ny * (nown + 2));
  s.elem = mke::pop_elem(global.precision);
  s.phi_elem = mke::phi_elem_of(global.precision);
  return s;
}

constexpr int kUp = 0, kDown = 1;

int tag_of(int dir, int array, int pop) { return 128 * dir + 32 * array + pop; }

// The D3Q19 directions crossing a z face, by the sign of e_z, in index order.
struct FacePops {
  int p[2][5];  // [0]: e_z = +1 (arrive through the lower face), [1]: e_z = -1 (through the upper)
};

FacePops face_pops() {
  FacePops f;
  int a = 0, b = 0;
  for (int i = 0; i < 19; ++i) {
    if (mkd::ez(i) == 1) f.p[0][a++] = i;
    if (mkd::ez(i) == -1) f.p[1][b++] = i;
  }
  return f;
}

// Element offset of a return run in the halo buffer: face 0 the lower face
// (its runs merge into plane 1), face 1 the upper (into plane nown).
__host__ __device__ int64_t halo_offset(int face, int lattice, int k, int64_t plane) {
  return ((int64_t)(face * 2 + lattice) * 5 + k) * plane;
}

// The transfers of one stage, sorted by (peer, tag, receive before send).
std::vector<mk_slab_xfer> plan(const SlabGeo& s, int stage) {
  const bool periodic = s.bc2 == MK_BC_PERIODIC;
  const int below = s.rank > 0 ? s.rank - 1 : (periodic ? s.nranks - 1 : -1);
  const int above = s.rank < s.nranks - 1 ? s.rank + 1 : (periodic ? 0 : -1);
  const int64_t plane = (int64_t)s.nx * s.ny;
  const int top = s.nown, ghost_top = s.nown + 1;
  std::vector<mk_slab_xfer> out;
  auto add = [&](int peer, int send, int dir, int array, int pop, int lz) {
    mk_slab_xfer x;
    std::memset(&x, 0, sizeof x);
    x.peer = peer;
    x.send = send;
    x.tag = tag_of(dir, array, pop);
    x.array = array;
    x.offset = (array == 2 ? 0 : (int64_t)pop * s.stride) + (int64_t)lz * plane;
    x.count = plane;
    x.bytes = plane * (array == 2 ? s.phi_elem : s.elem);
    x.ptr = nullptr;
    out.push_back(x);
  };
  // a return run received into the halo buffer (array 3)
  auto add_halo = [&](int peer, int dir, int lattice, int pop, int face, int k) {
    add(peer, 0, dir, lattice, pop, 0);
    out.back().array = 3;
    out.back().offset = halo_offset(face, lattice, k, plane);
  };
  const FacePops fp = face_pops();
  const int(&up)[5] = fp.p[0];
  const int(&dn)[5] = fp.p[1];
  if (stage == MK_SLAB_PHI) {
    if (above >= 0) add(above, 1, kUp, 2, 0, top);
    if (below >= 0) add(below, 0, kUp, 2, 0, 0);
    if (below >= 0) add(below, 1, kDown, 2, 0, 1);
    if (above >= 0) add(above, 0, kDown, 2, 0, ghost_top);
  } else {
    for (int a = 0; a < 2; ++a)
      for (int k = 0; k < 5; ++k) {
        if (stage == MK_SLAB_FILL) {
          // upward: the top owned plane's e_z = -1 slots into ghost 0 above;
          // downward: plane 1's e_z = +1 slots into the top ghost below
          if (above >= 0) add(above, 1, kUp, a, dn[k], top);
          if (below >= 0) add(below, 0, kUp, a, dn[k], 0);
          if (below >= 0) add(below, 1, kDown, a, up[k], 1);
          if (above >= 0) add(above, 0, kDown, a, up[k], ghost_top);
        } else {
          // upward: the top ghost's e_z = +1 slots into plane 1 above;
          // downward: ghost 0's e_z = -1 slots into the top owned plane below
          // (both received into the halo buffer and merged)
          if (above >= 0) add(above, 1, kUp, a, up[k], ghost_top);
          if (below >= 0) add_halo(below, kUp, a, up[k], 0, k);
          if (below >= 0) add(below, 1, kDown, a, dn[k], 0);
          if (above >= 0) add_halo(above, kDown, a, dn[k], 1, k);
        }
      }
  }
  std::sort(out.begin(), out.end(), [](const mk_slab_xfer& a, const mk_slab_xfer& b) {
    if (a.peer != b.peer) return a.peer < b.peer;
    if (a.tag != b.tag) return a.tag < b.tag;
    return a.send < b.send;
  });
  return out;
}

mk_status copy_plan(const std::vector<mk_slab_xfer>& v, mk_slab_xfer* out, int32_t capacity, int32_t* count) {
  *count = (int32_t)v.size();
  if ((int32_t)v.size() > capacity || (!out && !v.empty())) return MK_ERR_ARG;
  std::copy(v.begin(), v.end(), out);
  return MK_OK;
}

bool valid_stage(int stage) { return stage == MK_SLAB_FILL || stage == MK_SLAB_PHI || stage == MK_SLAB_RETURN; }

SlabGeo geo_of(const mke::Engine& e) {
  mk_params g = e.p;
  g.nz = e.nzg;
  return geo_of(g, e.rank, e.nranks, e.nz - 2);
}

std::vector<mk_slab_xfer> transfers(const mke::Engine& e, int stage) {
  std::vector<mk_slab_xfer> v = plan(geo_of(e), stage);
  for (mk_slab_xfer& x : v) {
    void* const bases[4] = {e.pop0, e.pop1, e.phi[0], e.slab_halo};
    char* base = (char*)bases[x.array];
    x.ptr = base + x.offset * (x.array == 2 ? e.phi_elem : e.elem);
  }
  return v;
}

const char* action_name(int a) {
  switch (a) {
    case MK_SLAB_FILL:
      return "MK_SLAB_FILL";
    case MK_SLAB_PHI:
      return "MK_SLAB_PHI";
    case MK_SLAB_RETURN:
      return "MK_SLAB_RETURN";
    case MK_SLAB_RUN_PHI:
      return "MK_SLAB_RUN_PHI";
    case MK_SLAB_RUN_COLLIDE:
      return "MK_SLAB_RUN_COLLIDE";
    default:
      return "unknown";
  }
}

mk_status out_of_order(mk_handle* h, int asked) {
  h->err = std::string("slab protocol: ") + action_name(asked) + " asked, next is " + action_name(h->e.slab_next);
  return MK_ERR_STATE;
}

mk_status slab_state(mk_handle* h) {
  h->err = "not a slab handle (mk_create_slab makes one)";
  return MK_ERR_STATE;
}

// Merge the received return runs into the owned boundary planes: one thread
// per cell of a plane and run (blockIdx.z = face * 10 + lattice * 5 + k).  W
// is an unsigned integer of the storage size (the slots are copied as bits).
struct MergeArgs {
  int pops[2][5];
  int nown;
  int faces;  // bit 0: a neighbour below, bit 1: above
};

template <class W>
__global__ void k_slab_merge(W* __restrict__ G, W* __restrict__ H, const W* __restrict__ halo, const mkd::Geom g,
                             const MergeArgs m) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int q = blockIdx.z;
  const int face = q / 10, lattice = (q / 5) % 2, k = q % 5;
  if (x >= g.nx || !((m.faces >> face) & 1)) return;
  const int z = face == 0 ? 1 : m.nown;
  if (!g.fluid(x, y, z)) return;
  const int i = m.pops[face][k];
  const mkd::Nbr nb(g, x, y, z);
  // closed source: the cell wrote the slot itself (bounce-back)
  if (!nb.fluid(-mkd::ex(i), -mkd::ey(i), -mkd::ez(i))) return;
  const int64_t plane = (int64_t)g.nx * g.ny;
  const int64_t c = x + (int64_t)g.nx * (y + (int64_t)g.ny * z);
  W* A = lattice ? H : G;
  A[(int64_t)i * g.stride + c] = halo[halo_offset(face, lattice, k, plane) + x + (int64_t)g.nx * y];
}

template <class W>
cudaError_t launch_merge(mke::Engine& e, const mkd::Geom& g, const MergeArgs& m) {
  const dim3 block(128), grid((e.nx + 127) / 128, e.ny, 20);
  k_slab_merge<W><<<grid, block, 0, e.stream>>>((W*)e.pop0, (W*)e.pop1, (const W*)e.slab_halo, g, m);
  e.launches += 1;
  return cudaGetLastError();
}

cudaError_t slab_merge(mke::Engine& e) {
  const SlabGeo sg = geo_of(e);
  const bool periodic = sg.bc2 == MK_BC_PERIODIC;
  MergeArgs m;
  const FacePops fp = face_pops();
  std::memcpy(m.pops, fp.p, sizeof m.pops);
  m.nown = sg.nown;
  m.faces = ((sg.rank > 0 || periodic) ? 1 : 0) | ((sg.rank < sg.nranks - 1 || periodic) ? 2 : 0);
  if (!m.faces) return cudaSuccess;
  const mkd::Geom g = mks::make_geom(e);
  switch (e.elem) {
    case 8:
      return launch_merge<unsigned long long>(e, g, m);
    case 4:
      return launch_merge<unsigned int>(e, g, m);
    default:
      return launch_merge<unsigned short>(e, g, m);
  }
}

// State after a completed exchange (a return exchange merges its runs first).
cudaError_t advance_done(mke::Engine& e, int stage) {
  if (stage == MK_SLAB_RETURN) {
    cudaError_t st = slab_merge(e);
    if (st != cudaSuccess) return st;
  }
  e.slab_next = stage == MK_SLAB_PHI ? MK_SLAB_RUN_COLLIDE : MK_SLAB_RUN_PHI;
  return cudaSuccess;
}

}  // namespace

extern "C" {

mk_status mk_slab_split(int32_t nz, int32_t rank, int32_t nranks, int32_t* z0, int32_t* nz_own) {
  if (!z0 || !nz_own) return set_global(MK_ERR_ARG, "null argument");
  int a = 0, b = 0;
  if (!split(nz, rank, nranks, a, b)) return set_global(MK_ERR_ARG, "slab split: need 0 <= rank < nranks <= nz");
  *z0 = a;
  *nz_own = b;
  return MK_OK;
}

mk_status mk_slab_plan(const mk_params* global, int32_t rank, int32_t nranks, int32_t stage, mk_slab_xfer* out,
                       int32_t capacity, int32_t* count) {
  if (!global || !count) return set_global(MK_ERR_ARG, "null argument");
  *count = 0;
  if (!valid_stage(stage)) return set_global(MK_ERR_ARG, "slab plan: stage must be FILL, PHI or RETURN");
  int z0 = 0, nown = 0;
  if (!split(global->nz, rank, nranks, z0, nown))
    return set_global(MK_ERR_ARG, "slab split: need 0 <= rank < nranks <= nz");
  const std::vector<mk_slab_xfer> v = plan(geo_of(*global, rank, nranks, nown), stage);
  if (copy_plan(v, out, capacity, count) != MK_OK) return set_global(MK_ERR_ARG, "slab plan: capacity too small");
  return MK_OK;
}

mk_status mk_create_slab(const mk_params* global, int32_t rank, int32_t nranks, mk_handle** out) {
  const Range nvtx_range("mk_create_slab");
  if (!global || !out) return set_global(MK_ERR_ARG, "null argument");
  *out = nullptr;
  std::string err;
  mk_status s = mkc::validate_params(global, err);
  if (s != MK_OK) return set_global(s, err);
  if (global->model != MK_MODEL_MULTIPHASE) return set_global(MK_ERR_ARG, "slabs: the multiphase model only");
  int z0 = 0, nown = 0;
  if (!split(global->nz, rank, nranks, z0, nown))
    return set_global(MK_ERR_ARG, "slab split: need 0 <= rank < nranks <= nz");
  if (!have_device(err)) return set_global(MK_ERR_NODEVICE, err);
  mk_params lp = *global;
  lp.nz = nown + 2;
  mk_handle* h = new mk_handle();
  int dev = 0;
  cudaGetDevice(&dev);
  cudaError_t st = mke::engine_alloc(h->e, lp, dev, 0, 0, err);
  if (st != cudaSuccess) {
    mk_status r = err.empty() ? cuda_fail(h, st, "allocate") : set_global(MK_ERR_ARG, err);
    mke::engine_free(h->e);
    delete h;
    return r;
  }
  mke::Engine& e = h->e;
  e.slab = 1;
  e.zg0 = z0;
  e.nzg = global->nz;
  e.rank = rank;
  e.nranks = nranks;
  e.wave = 0;
  e.wave_ok = 0;  // the fused loop has no exchange points
  e.tma_ok = 0;   // the TMA phi tile is validated on whole domains only
  e.tma = 0;
  const size_t halo_bytes = (size_t)20 * global->nx * global->ny * e.elem;
  if ((st = cudaMalloc(&e.slab_halo, halo_bytes)) != cudaSuccess ||
      (st = cudaMemsetAsync(e.slab_halo, 0, halo_bytes, e.stream)) != cudaSuccess) {
    mk_status r = cuda_fail(h, st, "allocate");
    mke::engine_free(e);
    delete h;
    return r;
  }
  // the global initial phi, cut to the slab and its ghost planes
  const int64_t plane = (int64_t)global->nx * global->ny;
  std::vector<double> gphi((size_t)(plane * global->nz)), phi((size_t)(plane * (nown + 2)));
  s = mkc::initial_field(global, MK_FIELD_PHI, gphi.data(), gphi.size(), err);
  if (s != MK_OK) {
    mke::engine_free(e);
    delete h;
    return set_global(s, err);
  }
  for (int lz = 0; lz < nown + 2; ++lz) {
    int gz = z0 + lz - 1;
    if (global->bc[2] == MK_BC_PERIODIC)
      gz = (gz + global->nz) % global->nz;
    else
      gz = std::min(std::max(gz, 0), global->nz - 1);  // beyond a closed end: never read
    std::copy(gphi.begin() + gz * plane, gphi.begin() + (gz + 1) * plane, phi.begin() + lz * plane);
  }
  st = mke::engine_set_state(e, phi.data(), nullptr, nullptr, nullptr, nullptr, nullptr);
  if (st != cudaSuccess) {
    mk_status r = cuda_fail(h, st, "initialise");
    mke::engine_free(e);
    delete h;
    return r;
  }
  e.slab_next = MK_SLAB_RETURN;
  *out = h;
  return MK_OK;
}

mk_status mk_slab_info(const mk_handle* h, int32_t* rank, int32_t* nranks, int32_t* z0, int32_t* nz_own,
                       int32_t* nz_global) {
  if (!h) return MK_ERR_ARG;
  if (!h->e.slab) return MK_ERR_STATE;
  if (rank) *rank = h->e.rank;
  if (nranks) *nranks = h->e.nranks;
  if (z0) *z0 = h->e.zg0;
  if (nz_own) *nz_own = h->e.nz - 2;
  if (nz_global) *nz_global = h->e.nzg;
  return MK_OK;
}

int32_t mk_slab_next(const mk_handle* h) { return h && h->e.slab ? h->e.slab_next : -1; }

mk_status mk_slab_transfers(const mk_handle* h, int32_t stage, mk_slab_xfer* out, int32_t capacity, int32_t* count) {
  if (!h || !count) return MK_ERR_ARG;
  *count = 0;
  if (!h->e.slab) return MK_ERR_STATE;
  if (!valid_stage(stage)) return MK_ERR_ARG;
  return copy_plan(transfers(h->e, stage), out, capacity, count);
}

mk_status mk_slab_done(mk_handle* h, int32_t stage) {
  if (!h) return MK_ERR_ARG;
  if (!h->e.slab) return slab_state(h);
  if (!valid_stage(stage)) return MK_ERR_ARG;
  if (stage != h->e.slab_next) return out_of_order(h, stage);
  cudaError_t st = advance_done(h->e, stage);
  if (st != cudaSuccess) return cuda_fail(h, st, "slab merge");
  return MK_OK;
}

mk_status mk_slab_run(mk_handle* h, int32_t action) {
  const Range nvtx_range("mk_slab_run");
  if (!h) return MK_ERR_ARG;
  mke::Engine& e = h->e;
  if (!e.slab) return slab_state(h);
  if (action != MK_SLAB_RUN_PHI && action != MK_SLAB_RUN_COLLIDE) return MK_ERR_ARG;
  if (action != e.slab_next) return out_of_order(h, action);
  const int part = action == MK_SLAB_RUN_PHI ? 0 : 1;
  const int64_t loop = e.step;
  cudaError_t st = mke::mp_launch_part(e, part);
  if (st != cudaSuccess) return cuda_fail(h, st, "slab run");
  if (part == 0)
    e.slab_next = MK_SLAB_PHI;
  else
    e.slab_next = (loop & 1) ? MK_SLAB_RETURN : MK_SLAB_FILL;
  return MK_OK;
}

mk_status mk_slab_exchange_local(mk_handle* const* hs, int32_t n, int32_t stage) {
  const Range nvtx_range("mk_slab_exchange_local");
  if (!hs || n < 1) return set_global(MK_ERR_ARG, "slab exchange: need n >= 1 handles");
  if (!valid_stage(stage)) return set_global(MK_ERR_ARG, "slab exchange: stage must be FILL, PHI or RETURN");
  for (int r = 0; r < n; ++r) {
    const mk_handle* h = hs[r];
    if (!h) return set_global(MK_ERR_ARG, "slab exchange: null handle");
    const mke::Engine& e = h->e;
    if (!e.slab || e.rank != r || e.nranks != n || e.nzg != hs[0]->e.nzg || e.nx != hs[0]->e.nx ||
        e.ny != hs[0]->e.ny || e.p.precision != hs[0]->e.p.precision || e.p.bc[2] != hs[0]->e.p.bc[2])
      return set_global(MK_ERR_ARG, "slab exchange: hs[r] must be rank r of one decomposition");
    if (e.slab_next != stage)
      return set_global(MK_ERR_STATE, std::string("slab exchange: rank ") + std::to_string(r) + " expects " +
                                          action_name(e.slab_next));
  }
  // every source is complete before any copy starts
  for (int r = 0; r < n; ++r) {
    cudaError_t st = cudaStreamSynchronize(hs[r]->e.stream);
    if (st != cudaSuccess) return cuda_fail(hs[r], st, "slab exchange sync");
  }
  std::vector<std::vector<mk_slab_xfer>> lists((size_t)n);
  for (int r = 0; r < n; ++r) lists[(size_t)r] = transfers(hs[r]->e, stage);
  for (int r = 0; r < n; ++r) {
    mke::Engine& dst = hs[r]->e;
    for (const mk_slab_xfer& x : lists[(size_t)r]) {
      if (x.send) continue;
      const mk_slab_xfer* src = nullptr;
      for (const mk_slab_xfer& y : lists[(size_t)x.peer])
        if (y.send && y.peer == r && y.tag == x.tag) src = &y;
      if (!src || src->bytes != x.bytes) return set_global(MK_ERR_STATE, "slab exchange: unmatched transfer");
      const mke::Engine& se = hs[x.peer]->e;
      cudaError_t st = se.device == dst.device
                           ? cudaMemcpyAsync(x.ptr, src->ptr, (size_t)x.bytes, cudaMemcpyDeviceToDevice, dst.stream)
                           : cudaMemcpyPeerAsync(x.ptr, dst.device, src->ptr, se.device, (size_t)x.bytes, dst.stream);
      if (st != cudaSuccess) return cuda_fail(hs[r], st, "slab exchange copy");
    }
  }
  // no slab writes a source run again before every copy has landed
  for (int r = 0; r < n; ++r) {
    cudaError_t st = cudaStreamSynchronize(hs[r]->e.stream);
    if (st != cudaSuccess) return cuda_fail(hs[r], st, "slab exchange sync");
  }
  for (int r = 0; r < n; ++r) {
    cudaError_t st = advance_done(hs[r]->e, stage);
    if (st != cudaSuccess) return cuda_fail(hs[r], st, "slab merge");
  }
  return MK_OK;
}

}  // extern "C"
