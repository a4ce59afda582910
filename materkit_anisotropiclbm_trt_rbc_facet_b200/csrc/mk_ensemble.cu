// mk_ensemble.cu — many dendrite domains advanced as one packed lattice.
//
// The reference runs a parameter sweep of dendrite cases one after the other
// (run_solutal_dendrite / run_thermal_dendrite, MaterKit.cpp:633-687 and
// 743-788; each a full mkSpace + mkPhaseField + mkThermalField lifecycle).
// Small and unevenly sized domains cannot fill 148 SMs one at a time, so the
// ensemble packs them:
//
//   * every population plane, phi buffer and scalar field is one array over
//     the concatenated cells of all domains (domain d occupies
//     [off_d, off_d + nx ny nz), x fastest inside it);
//   * every domain's cell count is a multiple of 256, so each 256-cell tile
//     lies in one domain; a tile -> domain table and a per-domain record
//     (geometry, offset, grain-table start, kernel coefficients) give each
//     block its domain with two cached loads;
//   * one loop is two persistent grid-stride launches over all tiles (phi sum,
//     then the coupled phase-field + thermal/solutal update), the same cell
//     code as the single-domain kernels (mk_dendrite.cuh), so a domain of the
//     ensemble evolves bit for bit like the same case run alone;
//   * mk_ensemble_advance replays two loops as one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mkb200.h"
#include "mk_case.hpp"
#include "mk_dendrite.cuh"
#include "mk_engine.hpp"

using namespace mkd;

namespace {

constexpr int TILE = 256;

// Per-domain record.  g.stride is the packed plane stride.
struct DomInfo {
  Geom g;
  int off;                // first packed cell of the domain
  int seed0;              // first grain of the domain in the packed grain tables
  double ref_t;           // rest value of the T/U lattice (-Delta of the domain)
  float inv_nx, inv_nxy;  // 1/nx, 1/(nx ny) rounded to FP32
};

// q = floor(a / b) for 0 <= a < 2^24 from the FP32 reciprocal of b: the
// product is within one unit of the quotient, one correction makes it exact.
__device__ __forceinline__ int div_small(int a, int b, float inv_b, int& rem) {
  int q = __float2int_rz((float)a * inv_b);
  int r = a - q * b;
  if (r < 0) {
    q -= 1;
    r += b;
  } else if (r >= b) {
    q += 1;
    r -= b;
  }
  rem = r;
  return q;
}

// Coordinates of this thread's cell in tile t of domain `di`.
__device__ __forceinline__ void tile_xyz(const DomInfo& di, int t, int& x, int& y, int& z) {
  const int local = t * TILE - di.off + (int)threadIdx.x;
  int r;
  z = div_small(local, di.g.nx * di.g.ny, di.inv_nxy, r);
  y = div_small(r, di.g.nx, di.inv_nx, x);
}

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(TILE)
    k_ens_phi(const S* __restrict__ G, const P* __restrict__ phi_old, P* __restrict__ phi_new,
              const DomInfo* __restrict__ dom, const int* __restrict__ tile_dom, const int ntiles,
              const typename Stor<S>::T ref_g) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const DomInfo di = dom[__ldg(tile_dom + t)];
    int x, y, z;
    tile_xyz(di, t, x, y, z);
    if (!di.g.fluid(x, y, z)) {
      const int c = t * TILE + (int)threadIdx.x;
      phi_new[c] = phi_old[c];
      continue;
    }
    if (fastw_cell(di.g, x, y, z)) {
      FastW fa = make_fastw(di.g, x, y, z);
      fa.c += di.off;
      pf_phi_cell<S, P, PARITY>(G, phi_new, di.g.stride, fa, fa.c, ref_g);
    } else {
      Nbr nb(di.g, x, y, z);
      nb.base = di.off;
      pf_phi_cell<S, P, PARITY>(G, phi_new, di.g.stride, nb, nb.idx(0, 0, 0), ref_g);
    }
  }
}

// The phi pass with two cells per thread (TILE / 2 threads per tile, cells x
// and x + 1 of one row; every domain's nx even): pf_phi_pair where both cells
// are fluid and on the interior path, else pf_phi_cell per cell; phi is
// bit-identical to k_ens_phi.
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(TILE / 2)
    k_ens_phi2(const S* __restrict__ G, const P* __restrict__ phi_old, P* __restrict__ phi_new,
               const DomInfo* __restrict__ dom, const int* __restrict__ tile_dom, const int ntiles,
               const typename Stor<S>::T ref_g) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const DomInfo di = dom[__ldg(tile_dom + t)];
    const int c0 = t * TILE + 2 * (int)threadIdx.x;
    const int local = c0 - di.off;
    int r, x, y;
    const int z = div_small(local, di.g.nx * di.g.ny, di.inv_nxy, r);
    y = div_small(r, di.g.nx, di.inv_nx, x);
    const bool f0 = di.g.fluid(x, y, z), f1 = di.g.fluid(x + 1, y, z);
    if (f0 && f1 && fastw_cell(di.g, x, y, z) && fastw_cell(di.g, x + 1, y, z)) {
      FastW a = make_fastw(di.g, x, y, z), b = make_fastw(di.g, x + 1, y, z);
      a.c += di.off;
      b.c += di.off;
      pf_phi_pair<S, P, PARITY>(G, phi_new, di.g.stride, a, b, ref_g);
      continue;
    }
    for (int k = 0; k < 2; ++k) {
      const int xx = x + k, c = c0 + k;
      if (!(k == 0 ? f0 : f1)) {
        phi_new[c] = phi_old[c];
        continue;
      }
      if (fastw_cell(di.g, xx, y, z)) {
        FastW fa = make_fastw(di.g, xx, y, z);
        fa.c += di.off;
        pf_phi_cell<S, P, PARITY>(G, phi_new, di.g.stride, fa, fa.c, ref_g);
      } else {
        Nbr nb(di.g, xx, y, z);
        nb.base = di.off;
        pf_phi_cell<S, P, PARITY>(G, phi_new, di.g.stride, nb, nb.idx(0, 0, 0), ref_g);
      }
    }
  }
}

// The even loop's phi pass when every cell of every domain is fluid (no wall
// axis; ensemble domains carry no solid mask): an even loop reads only a
// cell's own slots, so phi is a flat sum over the packed index, two cells per
// thread, with no domain lookup or coordinates (pf_phi_pair at parity 0 uses
// the cell index alone; bit-identical to k_ens_phi).
template <class S, class P>
__global__ void __launch_bounds__(TILE)
    k_ens_phi_flat(const S* __restrict__ G, P* __restrict__ phi_new, const int64_t stride, const int ncell,
                   const typename Stor<S>::T ref_g) {
  for (int64_t c = 2 * (int64_t)(blockIdx.x * blockDim.x + threadIdx.x); c < ncell;
       c += 2 * (int64_t)gridDim.x * blockDim.x) {
    FastW a{};
    a.c = (int)c;
    pf_phi_pair<S, P, 0>(G, phi_new, stride, a, a, ref_g);
  }
}

// Four resident 256-thread blocks per SM (64 registers) for the 32-bit and
// 16-bit variants; the FP64 one keeps its registers.
template <class S, class P, int PARITY, bool SOL, bool GEN>
__global__ void __launch_bounds__(TILE, sizeof(typename Stor<S>::T) == 8 ? 2 : 4)
    k_ens_collide(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phi_new,
                  const P* __restrict__ phi_old, P* __restrict__ temp, const unsigned char* __restrict__ grain,
                  const typename Stor<S>::T* __restrict__ rot, const DomInfo* __restrict__ dom,
                  const DendK<typename Stor<S>::T>* __restrict__ kd, const int* __restrict__ tile_dom,
                  const int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int d = __ldg(tile_dom + t);
    const DomInfo di = dom[d];
    int x, y, z;
    tile_xyz(di, t, x, y, z);
    if (!di.g.fluid(x, y, z)) continue;
    const DendK<typename Stor<S>::T> k = kd[d];
    const typename Stor<S>::T* rd = rot + 9 * di.seed0;
    if (fastw_cell(di.g, x, y, z)) {
      FastW fa = make_fastw(di.g, x, y, z);
      fa.c += di.off;
      dend_cell<S, P, PARITY, SOL, GEN>(G, Tp, phi_new, phi_old, temp, grain, rd, di.g.stride, fa, fa.c, k);
    } else {
      Nbr nb(di.g, x, y, z);
      nb.base = di.off;
      dend_cell<S, P, PARITY, SOL, GEN>(G, Tp, phi_new, phi_old, temp, grain, rd, di.g.stride, nb, nb.idx(0, 0, 0),
                                        k);
    }
  }
}

// Initial state from packed FP64 phi and T/U: the dendrite branch of the
// single-domain initialiser.
template <class S>
__global__ void __launch_bounds__(TILE)
    k_ens_init(S* __restrict__ G, S* __restrict__ Tp, typename PhiOf<S>::type* __restrict__ phi0,
               typename PhiOf<S>::type* __restrict__ phi1, typename PhiOf<S>::type* __restrict__ temp,
               const double* __restrict__ in_phi, const double* __restrict__ in_t, const DomInfo* __restrict__ dom,
               const int* __restrict__ tile_dom, const int ntiles, const double ref_g) {
  typedef typename PhiOf<S>::type P;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const DomInfo di = dom[__ldg(tile_dom + t)];
    int x, y, z;
    tile_xyz(di, t, x, y, z);
    const int c = t * TILE + (int)threadIdx.x;
    const double ph = in_phi[c], tv = in_t[c];
    phi0[c] = P(ph);
    phi1[c] = P(ph);
    temp[c] = P(tv);
    if (!di.g.fluid(x, y, z)) continue;
    Nbr nb(di.g, x, y, z);
    nb.base = di.off;
    put_eq<S, 7>(G, di.g, nb, c, ph, 0.0, 0.0, 0.0, 0.0, ref_g);
    put_eq<S, 7>(Tp, di.g, nb, c, tv, 0.0, 0.0, 0.0, 0.0, di.ref_t);
  }
}

// One domain's field: a (minus b) for phi / dphi / T / U; grain or flag from
// the geometry.
template <class P, class O>
__global__ void k_ens_field(const P* __restrict__ a, const P* __restrict__ b, const Geom g, const int off,
                            const int mode, const double* __restrict__ seeds, const int nobj, O* __restrict__ out) {
  const int n = g.nx * g.ny * g.nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v;
    if (mode == 0) {
      v = b ? double(a[off + i]) - double(b[off + i]) : double(a[off + i]);
    } else {
      const int z = i / (g.nx * g.ny), r = i - z * g.nx * g.ny, y = r / g.nx, x = r - y * g.nx;
      if (mode == 1)
        v = g.fluid(x, y, z) ? MK_FLAG_FLUID : MK_FLAG_WALLS;
      else
        v = nobj > 0 ? nearest_seed(seeds, nobj, x, y, z) : 0;
    }
    out[i] = O(v);
  }
}

int store_bytes(int prec) { return prec == MK_PREC_FP64 ? 8 : (prec == MK_PREC_FP32 ? 4 : 2); }

}  // namespace

struct mk_ensemble {
  std::vector<mk_params> params;
  std::vector<int> off;  // first packed cell per domain
  int n = 0, model = 0, precision = 0, elem = 0, phi_elem = 0;
  int64_t ncell = 0, stride = 0;
  int ntiles = 0;
  int device = 0, sms = 148;
  int grid_phi[2] = {1, 1}, grid_col[2] = {1, 1};  // persistent launch sizes per parity
  int grid_flat = 1;
  bool gen_aniso = false;  // some domain has a non-cubic anisotropy kind
  bool pair = false;       // every domain's nx even: the phi pass is k_ens_phi2
  bool flat_even = false;  // no domain has a wall axis: the even loop's phi pass is k_ens_phi_flat
  cudaStream_t stream = nullptr;
  void* pop0 = nullptr;
  void* pop1 = nullptr;
  void* phi[2] = {nullptr, nullptr};
  void* temp = nullptr;
  double* seeds = nullptr;
  void* rot = nullptr;             // rotations in the arithmetic type, 9 per grain
  unsigned char* grain = nullptr;  // packed per-cell grain index
  DomInfo* dom = nullptr;
  void* kd = nullptr;
  int* tile_dom = nullptr;
  void* field = nullptr;  // largest domain, 8 bytes per cell
  int64_t step = 0;
  int phi_cur = 0;
  int64_t launches = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  std::string err;
};

namespace {

mk_status ens_cuda_fail(mk_ensemble* e, cudaError_t st, const char* where) {
  const std::string m = std::string(where) + ": " + cudaGetErrorString(st);
  if (e) e->err = m;
  mke::set_global_error(m);
  return st == cudaErrorMemoryAllocation ? MK_ERR_OOM : MK_ERR_CUDA;
}

mk_status ens_arg(mk_ensemble* e, const std::string& m) {
  if (e) e->err = m;
  mke::set_global_error(m);
  return MK_ERR_ARG;
}

// Blocks of a persistent launch: resident blocks per SM x SMs, at most one per tile.
template <class K>
int persistent_grid(const mk_ensemble& e, K kernel, int threads = TILE) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return (int)std::min<int64_t>(e.ntiles, (int64_t)per_sm * e.sms);
}

// One loop.  When `ev` is non-null, ev[0..1] bracket the phi launch and
// ev[2..3] the collide launch.
template <class S, bool SOL, bool GEN>
void loop_t(mk_ensemble& e, cudaEvent_t* ev) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const int parity = (int)(e.step & 1);
  S* G = (S*)e.pop0;
  S* Tp = (S*)e.pop1;
  P* phi_old = (P*)e.phi[e.phi_cur];
  P* phi_new = (P*)e.phi[1 - e.phi_cur];
  const DendK<T>* kd = (const DendK<T>*)e.kd;
  const T ref_g = T(-1.0);
  if (ev) cudaEventRecord(ev[0], e.stream);
  if (parity == 0 && e.flat_even) {
    k_ens_phi_flat<S, P><<<e.grid_flat, TILE, 0, e.stream>>>(G, phi_new, e.stride, (int)e.ncell, ref_g);
  } else if (e.pair) {
    if (parity == 0)
      k_ens_phi2<S, P, 0><<<e.grid_phi[0], TILE / 2, 0, e.stream>>>(G, phi_old, phi_new, e.dom, e.tile_dom,
                                                                    e.ntiles, ref_g);
    else
      k_ens_phi2<S, P, 1><<<e.grid_phi[1], TILE / 2, 0, e.stream>>>(G, phi_old, phi_new, e.dom, e.tile_dom,
                                                                    e.ntiles, ref_g);
  } else if (parity == 0) {
    k_ens_phi<S, P, 0><<<e.grid_phi[0], TILE, 0, e.stream>>>(G, phi_old, phi_new, e.dom, e.tile_dom, e.ntiles,
                                                             ref_g);
  } else {
    k_ens_phi<S, P, 1><<<e.grid_phi[1], TILE, 0, e.stream>>>(G, phi_old, phi_new, e.dom, e.tile_dom, e.ntiles,
                                                             ref_g);
  }
  if (ev) {
    cudaEventRecord(ev[1], e.stream);
    cudaEventRecord(ev[2], e.stream);
  }
  if (parity == 0)
    k_ens_collide<S, P, 0, SOL, GEN><<<e.grid_col[0], TILE, 0, e.stream>>>(G, Tp, phi_new, phi_old, (P*)e.temp, e.grain,
                                                                       (const T*)e.rot, e.dom, kd, e.tile_dom,
                                                                       e.ntiles);
  else
    k_ens_collide<S, P, 1, SOL, GEN><<<e.grid_col[1], TILE, 0, e.stream>>>(G, Tp, phi_new, phi_old, (P*)e.temp, e.grain,
                                                                       (const T*)e.rot, e.dom, kd, e.tile_dom,
                                                                       e.ntiles);
  if (ev) cudaEventRecord(ev[3], e.stream);
  e.phi_cur = 1 - e.phi_cur;
  e.step += 1;
  e.launches += 2;
}

template <class S>
void loop_s(mk_ensemble& e, cudaEvent_t* ev) {
  const bool sol = e.model == MK_MODEL_SOLUTAL_DENDRITE;
  if (e.gen_aniso) {
    if (sol)
      loop_t<S, true, true>(e, ev);
    else
      loop_t<S, false, true>(e, ev);
  } else {
    if (sol)
      loop_t<S, true, false>(e, ev);
    else
      loop_t<S, false, false>(e, ev);
  }
}

void ens_loop(mk_ensemble& e, cudaEvent_t* ev = nullptr) {
  switch (e.precision) {
    case MK_PREC_FP64:
      loop_s<double>(e, ev);
      break;
    case MK_PREC_FP32:
      loop_s<float>(e, ev);
      break;
    case MK_PREC_FP16:
      loop_s<__half>(e, ev);
      break;
    default:
      loop_s<__nv_bfloat16>(e, ev);
      break;
  }
}

template <class S>
void size_grids(mk_ensemble& e) {
  typedef typename PhiOf<S>::type P;
  const bool sol = e.model == MK_MODEL_SOLUTAL_DENDRITE;
  // each parity has its own register footprint, hence its own resident count
  e.grid_flat = persistent_grid(e, k_ens_phi_flat<S, P>);
  if (e.pair) {
    e.grid_phi[0] = persistent_grid(e, k_ens_phi2<S, P, 0>, TILE / 2);
    e.grid_phi[1] = persistent_grid(e, k_ens_phi2<S, P, 1>, TILE / 2);
  } else {
    e.grid_phi[0] = persistent_grid(e, k_ens_phi<S, P, 0>);
    e.grid_phi[1] = persistent_grid(e, k_ens_phi<S, P, 1>);
  }
  for (int par = 0; par < 2; ++par) {
    int g;
    if (e.gen_aniso)
      g = sol ? persistent_grid(e, par ? k_ens_collide<S, P, 1, true, true> : k_ens_collide<S, P, 0, true, true>)
              : persistent_grid(e, par ? k_ens_collide<S, P, 1, false, true> : k_ens_collide<S, P, 0, false, true>);
    else
      g = sol ? persistent_grid(e, par ? k_ens_collide<S, P, 1, true, false> : k_ens_collide<S, P, 0, true, false>)
              : persistent_grid(e, par ? k_ens_collide<S, P, 1, false, false> : k_ens_collide<S, P, 0, false, false>);
    e.grid_col[par] = g;
  }
}

// Per-domain coefficients and the rotations, in the arithmetic type.
template <class S>
cudaError_t upload_kd(mk_ensemble& e, const std::vector<double>& seeds) {
  typedef typename Stor<S>::T T;
  std::vector<DendK<T>> k(e.n);
  for (int d = 0; d < e.n; ++d) k[d] = dend_params<T>(e.params[d], -1.0, -e.params[d].delta);
  const size_t ngr = seeds.size() / 12;
  std::vector<T> r(9 * ngr);
  for (size_t g = 0; g < ngr; ++g)
    for (int q = 0; q < 9; ++q) r[9 * g + q] = T(seeds[12 * g + 3 + q]);
  cudaError_t st = cudaMalloc(&e.kd, k.size() * sizeof(DendK<T>));
  if (st != cudaSuccess) return st;
  if ((st = cudaMalloc(&e.rot, r.size() * sizeof(T))) != cudaSuccess) return st;
  st = cudaMemcpyAsync(e.kd, k.data(), k.size() * sizeof(DendK<T>), cudaMemcpyHostToDevice, e.stream);
  if (st != cudaSuccess) return st;
  st = cudaMemcpyAsync(e.rot, r.data(), r.size() * sizeof(T), cudaMemcpyHostToDevice, e.stream);
  if (st != cudaSuccess) return st;
  return cudaStreamSynchronize(e.stream);
}

template <class S>
void init_t(mk_ensemble& e, const double* d_phi, const double* d_t) {
  typedef typename PhiOf<S>::type P;
  k_ens_init<S><<<persistent_grid(e, k_ens_init<S>), TILE, 0, e.stream>>>(
      (S*)e.pop0, (S*)e.pop1, (P*)e.phi[0], (P*)e.phi[1], (P*)e.temp, d_phi, d_t, e.dom, e.tile_dom, e.ntiles, -1.0);
}

void ens_free(mk_ensemble* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (cudaGraphExec_t& g : e->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  void* ptrs[] = {e->pop0,  e->pop1, e->phi[0], e->phi[1],     e->temp, e->seeds,
                  e->rot,   e->grain, e->dom,   e->kd, e->tile_dom, e->field};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}


// Field of one domain into e.field (device), as FP64 or FP32.
template <class S, class O>
cudaError_t field_t(mk_ensemble& e, int d, int field) {
  typedef typename PhiOf<S>::type P;
  const mk_params& p = e.params[d];
  Geom g;
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.bc0 = p.bc[0];
  g.bc1 = p.bc[1];
  g.bc2 = p.bc[2];
  g.stride = e.stride;
  const P* cur = (const P*)e.phi[e.phi_cur];
  const P* prev = (const P*)e.phi[1 - e.phi_cur];
  const P* a = nullptr;
  const P* b = nullptr;
  int mode = 0;
  switch (field) {
    case MK_FIELD_PHI:
      a = cur;
      break;
    case MK_FIELD_DPHI:
      a = cur;
      b = prev;
      break;
    case MK_FIELD_T:
    case MK_FIELD_C:
      if ((field == MK_FIELD_T) != (e.model == MK_MODEL_THERMAL_DENDRITE)) return cudaErrorInvalidValue;
      a = (const P*)e.temp;
      break;
    case MK_FIELD_FLAG:
      mode = 1;
      break;
    case MK_FIELD_GRAIN:
      mode = 2;
      break;
    default:
      return cudaErrorInvalidValue;
  }
  int seed0 = 0;
  for (int q = 0; q < d; ++q) seed0 += std::max(1, e.params[q].n_objects);
  const int n = p.nx * p.ny * p.nz;
  k_ens_field<P, O><<<(n + 255) / 256, 256, 0, e.stream>>>(a, b, g, e.off[d], mode, e.seeds + 12 * seed0,
                                                           p.n_objects, (O*)e.field);
  return cudaGetLastError();
}

template <class S>
cudaError_t field_s(mk_ensemble& e, int d, int field, int dtype) {
  return dtype == MK_DTYPE_F64 ? field_t<S, double>(e, d, field) : field_t<S, float>(e, d, field);
}

cudaError_t ens_field(mk_ensemble& e, int d, int field, int dtype) {
  switch (e.precision) {
    case MK_PREC_FP64:
      return field_s<double>(e, d, field, dtype);
    case MK_PREC_FP32:
      return field_s<float>(e, d, field, dtype);
    case MK_PREC_FP16:
      return field_s<__half>(e, d, field, dtype);
    default:
      return field_s<__nv_bfloat16>(e, d, field, dtype);
  }
}

template <class S>
cudaError_t setup_t(mk_ensemble& e, const double* d_phi, const double* d_t, const std::vector<double>& seeds) {
  size_grids<S>(e);
  cudaError_t st = upload_kd<S>(e, seeds);
  if (st != cudaSuccess) return st;
  init_t<S>(e, d_phi, d_t);
  return cudaGetLastError();
}

cudaError_t ens_setup(mk_ensemble& e, const double* d_phi, const double* d_t, const std::vector<double>& seeds) {
  switch (e.precision) {
    case MK_PREC_FP64:
      return setup_t<double>(e, d_phi, d_t, seeds);
    case MK_PREC_FP32:
      return setup_t<float>(e, d_phi, d_t, seeds);
    case MK_PREC_FP16:
      return setup_t<__half>(e, d_phi, d_t, seeds);
    default:
      return setup_t<__nv_bfloat16>(e, d_phi, d_t, seeds);
  }
}

// Checks of an ensemble parameter set; empty string when valid.
std::string check_ensemble(const mk_params* params, int n) {
  if (n < 1) return "ensemble needs at least one domain";
  const int model = params[0].model, prec = params[0].precision;
  if (model != MK_MODEL_THERMAL_DENDRITE && model != MK_MODEL_SOLUTAL_DENDRITE)
    return "ensemble domains must be thermal or solutal dendrite cases";
  int64_t total = 0;
  for (int d = 0; d < n; ++d) {
    const mk_params& p = params[d];
    std::string err;
    if (mkc::validate_params(&p, err) != MK_OK) return "domain " + std::to_string(d) + ": " + err;
    if (p.model != model) return "domain " + std::to_string(d) + ": all domains must share the model";
    if (p.precision != prec) return "domain " + std::to_string(d) + ": all domains must share the precision";
    const int64_t c = (int64_t)p.nx * p.ny * p.nz;
    if (c % TILE != 0)
      return "domain " + std::to_string(d) + ": cell count " + std::to_string(c) + " is not a multiple of 256";
    if (c >= ((int64_t)1 << 24)) return "domain " + std::to_string(d) + ": more than 2^24 cells";
    total += c;
  }
  if (total > ((int64_t)1 << 31) - 65) return "ensemble exceeds 2^31 - 65 cells";
  return std::string();
}

}  // namespace

extern "C" {

mk_status mk_ensemble_case_params(uint64_t seed, int32_t n_domains, int32_t precision, mk_params* out) {
  if (!out) return ens_arg(nullptr, "null argument");
  if (precision < MK_PREC_FP64 || precision > MK_PREC_BF16) return ens_arg(nullptr, "unknown precision");
  std::string err;
  const mk_status s = mkc::ensemble_case((unsigned long long)seed, n_domains, precision, out, err);
  if (s != MK_OK) mke::set_global_error(err);
  return s;
}

mk_status mk_ensemble_create(const mk_params* params, int32_t n_domains, mk_ensemble** out) {
  if (!params || !out) return ens_arg(nullptr, "null argument");
  *out = nullptr;
  const std::string why = check_ensemble(params, n_domains);
  if (!why.empty()) return ens_arg(nullptr, why);
  int ndev = 0;
  cudaError_t st = cudaGetDeviceCount(&ndev);
  if (st != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    mke::set_global_error(std::string("no CUDA device: ") +
                          (st != cudaSuccess ? cudaGetErrorString(st) : "count is 0"));
    return MK_ERR_NODEVICE;
  }
  mk_ensemble* e = new mk_ensemble();
  e->params.assign(params, params + n_domains);
  e->n = n_domains;
  e->model = params[0].model;
  e->precision = params[0].precision;
  e->elem = store_bytes(e->precision);
  e->pair = true;
  e->flat_even = true;
  for (int d = 0; d < n_domains; ++d) {
    e->gen_aniso = e->gen_aniso || params[d].aniso != MK_ANISO_CUBIC;
    e->pair = e->pair && params[d].nx % 2 == 0;
    for (int a = 0; a < 3; ++a) e->flat_even = e->flat_even && params[d].bc[a] != MK_BC_WALLS;
  }
  e->phi_elem = e->precision == MK_PREC_FP64 ? 8 : 4;
  cudaGetDevice(&e->device);
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device);
  // packing: offsets, tile table, domain records, grain table
  std::vector<DomInfo> dom(n_domains);
  std::vector<double> seeds;
  int64_t off = 0, maxc = 0;
  for (int d = 0; d < n_domains; ++d) {
    const mk_params& p = params[d];
    const int64_t c = (int64_t)p.nx * p.ny * p.nz;
    e->off.push_back((int)off);
    DomInfo& di = dom[d];
    di.g.nx = p.nx;
    di.g.ny = p.ny;
    di.g.nz = p.nz;
    di.g.bc0 = p.bc[0];
    di.g.bc1 = p.bc[1];
    di.g.bc2 = p.bc[2];
    di.off = (int)off;
    di.seed0 = (int)(seeds.size() / 12);
    di.ref_t = -p.delta;
    di.inv_nx = 1.0f / (float)p.nx;
    di.inv_nxy = 1.0f / (float)(p.nx * p.ny);
    std::vector<double> sd;
    mke::seed_table(p, sd);
    seeds.insert(seeds.end(), sd.begin(), sd.end());
    off += c;
    maxc = std::max(maxc, c);
  }
  e->ncell = off;
  e->stride = off;  // a multiple of 256
  e->ntiles = (int)(off / TILE);
  for (DomInfo& di : dom) di.g.stride = e->stride;
  std::vector<int> tile_dom(e->ntiles);
  for (int d = 0; d < n_domains; ++d) {
    const int64_t c = (int64_t)params[d].nx * params[d].ny * params[d].nz;
    for (int64_t t = e->off[d] / TILE; t < (e->off[d] + c) / TILE; ++t) tile_dom[t] = d;
  }
  // initial fields (mkSpace + initialize of every domain), packed
  // (independent per domain: host threads take domains in turn)
  std::vector<double> h_init((size_t)2 * off);
  {
    const int nth = std::max(1, std::min<int>(n_domains, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; ++t)
      pool.emplace_back([&, t]() {
        for (int d = t; d < n_domains; d += nth) {
          const size_t c = (size_t)params[d].nx * params[d].ny * params[d].nz;
          std::string err;
          mkc::initial_field(&params[d], MK_FIELD_PHI, h_init.data() + e->off[d], c, err);
          mkc::initial_field(&params[d], MK_FIELD_T, h_init.data() + off + e->off[d], c, err);
        }
      });
    for (std::thread& th : pool) th.join();
  }
  double* d_init = nullptr;
  auto fail = [&](cudaError_t s, const char* where) {
    const mk_status r = ens_cuda_fail(nullptr, s, where);
    if (d_init) cudaFree(d_init);
    ens_free(e);
    return r;
  };
  if ((st = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(st, "stream");
  const size_t pop_bytes = (size_t)7 * e->stride * e->elem, sc_bytes = (size_t)off * e->phi_elem;
  if ((st = cudaMalloc(&e->pop0, pop_bytes)) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc(&e->pop1, pop_bytes)) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc(&e->phi[0], sc_bytes)) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc(&e->phi[1], sc_bytes)) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc(&e->temp, sc_bytes)) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc((void**)&e->seeds, seeds.size() * sizeof(double))) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc((void**)&e->dom, dom.size() * sizeof(DomInfo))) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc((void**)&e->tile_dom, tile_dom.size() * sizeof(int))) != cudaSuccess)
    return fail(st, "allocate");
  if ((st = cudaMalloc(&e->field, (size_t)maxc * sizeof(double))) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMalloc((void**)&d_init, h_init.size() * sizeof(double))) != cudaSuccess) return fail(st, "allocate");
  if ((st = cudaMemsetAsync(e->pop0, 0, pop_bytes, e->stream)) != cudaSuccess) return fail(st, "clear");
  if ((st = cudaMemsetAsync(e->pop1, 0, pop_bytes, e->stream)) != cudaSuccess) return fail(st, "clear");
  if ((st = cudaMemcpyAsync(e->seeds, seeds.data(), seeds.size() * sizeof(double), cudaMemcpyHostToDevice,
                            e->stream)) != cudaSuccess)
    return fail(st, "upload");
  if ((st = cudaMemcpyAsync(e->dom, dom.data(), dom.size() * sizeof(DomInfo), cudaMemcpyHostToDevice, e->stream)) !=
      cudaSuccess)
    return fail(st, "upload");
  if ((st = cudaMemcpyAsync(e->tile_dom, tile_dom.data(), tile_dom.size() * sizeof(int), cudaMemcpyHostToDevice,
                            e->stream)) != cudaSuccess)
    return fail(st, "upload");
  if ((st = cudaMemcpyAsync(d_init, h_init.data(), h_init.size() * sizeof(double), cudaMemcpyHostToDevice,
                            e->stream)) != cudaSuccess)
    return fail(st, "upload");
  if ((st = cudaMalloc((void**)&e->grain, (size_t)off)) != cudaSuccess) return fail(st, "allocate");
  for (int d = 0; d < n_domains; ++d) {
    const int64_t c = (int64_t)params[d].nx * params[d].ny * params[d].nz;
    k_grain_map<<<(int)std::min<int64_t>((c + 255) / 256, 4096), 256, 0, e->stream>>>(
        dom[d].g, e->seeds + 12 * dom[d].seed0, params[d].n_objects, e->off[d], e->grain);
  }
  if ((st = cudaGetLastError()) != cudaSuccess) return fail(st, "grain map");
  if ((st = ens_setup(*e, d_init, d_init + off, seeds)) != cudaSuccess) return fail(st, "initialise");
  if ((st = cudaStreamSynchronize(e->stream)) != cudaSuccess) return fail(st, "initialise");
  cudaFree(d_init);
  e->step = 0;
  e->phi_cur = 0;
  *out = e;
  return MK_OK;
}

mk_status mk_ensemble_destroy(mk_ensemble* e) {
  if (!e) return MK_ERR_ARG;
  ens_free(e);
  return MK_OK;
}

const char* mk_ensemble_last_error(const mk_ensemble* e) { return e ? e->err.c_str() : ""; }

mk_status mk_ensemble_advance(mk_ensemble* e, int64_t nsteps) {
  if (!e || nsteps < 0) return MK_ERR_ARG;
  int64_t left = nsteps;
  while (left >= 2) {
    const int par = (int)(e->step & 1);
    if (!e->graph[par]) {
      const int64_t step0 = e->step, l0 = e->launches;
      const int cur0 = e->phi_cur;
      cudaGraph_t g;
      cudaError_t st = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
      if (st != cudaSuccess) return ens_cuda_fail(e, st, "capture begin");
      ens_loop(*e);
      ens_loop(*e);
      st = cudaStreamEndCapture(e->stream, &g);
      e->step = step0;
      e->launches = l0;
      e->phi_cur = cur0;
      if (st != cudaSuccess) return ens_cuda_fail(e, st, "capture end");
      st = cudaGraphInstantiate(&e->graph[par], g, 0);
      cudaGraphDestroy(g);
      if (st != cudaSuccess) return ens_cuda_fail(e, st, "graph instantiate");
    }
    const cudaError_t st = cudaGraphLaunch(e->graph[par], e->stream);
    if (st != cudaSuccess) return ens_cuda_fail(e, st, "graph launch");
    e->step += 2;
    e->launches += 4;
    left -= 2;
  }
  if (left) {
    ens_loop(*e);
    const cudaError_t st = cudaGetLastError();
    if (st != cudaSuccess) return ens_cuda_fail(e, st, "launch");
  }
  return MK_OK;
}

mk_status mk_ensemble_time_advance(mk_ensemble* e, int64_t nsteps, double* ms) {
  if (!e || nsteps < 0 || !ms) return MK_ERR_ARG;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, e->stream);
  const mk_status s = mk_ensemble_advance(e, nsteps);
  cudaEventRecord(t1, e->stream);
  const cudaError_t st = cudaEventSynchronize(t1);
  float f = 0;
  if (st == cudaSuccess) cudaEventElapsedTime(&f, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (s != MK_OK) return s;
  if (st != cudaSuccess) return ens_cuda_fail(e, st, "time_advance");
  *ms = f;
  return MK_OK;
}

mk_status mk_ensemble_get_field(mk_ensemble* e, int32_t domain, int32_t field, int32_t dtype, void* host_dst,
                                size_t bytes) {
  if (!e || !host_dst) return MK_ERR_ARG;
  if (domain < 0 || domain >= e->n) return ens_arg(e, "domain index out of range");
  if (dtype != MK_DTYPE_F64 && dtype != MK_DTYPE_F32) return ens_arg(e, "dtype must be MK_DTYPE_F64 or MK_DTYPE_F32");
  const mk_params& p = e->params[domain];
  const size_t need = (size_t)p.nx * p.ny * p.nz * (dtype == MK_DTYPE_F64 ? 8 : 4);
  if (bytes < need) return ens_arg(e, "destination buffer too small");
  cudaError_t st = ens_field(*e, domain, field, dtype);
  if (st == cudaErrorInvalidValue) {
    cudaGetLastError();
    return ens_arg(e, "field not available for this model");
  }
  if (st != cudaSuccess) return ens_cuda_fail(e, st, "field");
  if ((st = cudaMemcpyAsync(host_dst, e->field, need, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess)
    return ens_cuda_fail(e, st, "field copy");
  if ((st = cudaStreamSynchronize(e->stream)) != cudaSuccess) return ens_cuda_fail(e, st, "field sync");
  return MK_OK;
}

mk_status mk_ensemble_profile_steps(mk_ensemble* e, int64_t nsteps, const char* kernel, double* kernel_ms,
                                    double* step_ms) {
  if (!e || nsteps <= 0 || !kernel || !kernel_ms || !step_ms) return MK_ERR_ARG;
  int slot = -1;
  if (std::strcmp(kernel, "phi") == 0) slot = 0;
  if (std::strcmp(kernel, "collide") == 0) slot = 1;
  if (slot < 0) return ens_arg(e, std::string("no kernel named ") + kernel);
  std::vector<cudaEvent_t> ev((size_t)nsteps * 4);
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, e->stream);
  for (int64_t s = 0; s < nsteps; ++s) ens_loop(*e, &ev[(size_t)s * 4]);
  cudaEventRecord(t1, e->stream);
  const cudaError_t st = cudaEventSynchronize(t1);
  double kt = 0;
  float tot = 0;
  if (st == cudaSuccess) {
    for (int64_t s = 0; s < nsteps; ++s) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[(size_t)s * 4 + 2 * slot], ev[(size_t)s * 4 + 2 * slot + 1]);
      kt += ms;
    }
    cudaEventElapsedTime(&tot, t0, t1);
  }
  for (auto& x : ev) cudaEventDestroy(x);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (st != cudaSuccess) return ens_cuda_fail(e, st, "profile");
  *kernel_ms = kt;
  *step_ms = tot;
  return MK_OK;
}

int64_t mk_ensemble_launches(const mk_ensemble* e) { return e ? e->launches : -1; }

int64_t mk_ensemble_cells(const mk_ensemble* e) { return e ? e->ncell : -1; }

int64_t mk_ensemble_step(const mk_ensemble* e) { return e ? e->step : -1; }

}  // extern "C"
