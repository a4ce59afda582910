// mk_shared.cuh — host/device helpers shared by the kernel translation units
// (mk_kernels.cu, mk_multiphase.cu): geometry of a handle, rest values of
// the lattices, and the multiphase cell pieces that field output and
// diagnostics reuse (the phi sum of a cell, the phi stencil and force).
#ifndef MK_SHARED_CUH
#define MK_SHARED_CUH

#include <cmath>

#include "mk_device.cuh"
#include "mk_engine.hpp"

namespace mks {

using namespace mkd;

// Rest values of the two lattices: populations are held as f_i - w_i ref.
struct Refs {
  double r0, r1;
};

inline Geom make_geom(const mke::Engine& e) {
  Geom g;
  g.nx = e.nx;
  g.ny = e.ny;
  g.nz = e.nz;
  g.bc0 = e.p.bc[0];
  g.bc1 = e.p.bc[1];
  g.bc2 = e.p.bc[2];
  g.stride = e.stride;
  g.slab = e.slab;
  g.zg0 = e.zg0;
  g.nzg = e.nzg;
  g.solid = e.msolid;
  g.near = e.mnear;
  return g;
}

inline void launch_dims(const mke::Engine& e, dim3& grid, dim3& block) {
  block = dim3(e.block_x, e.block_y, 1);
  grid = dim3((e.nx + e.block_x - 1) / e.block_x, (e.ny + e.block_y - 1) / e.block_y, e.nz);
}

// Rest values of the lattices (populations are held as f_i - w_i ref).
inline Refs refs_of(const mk_params& p) {
  Refs r{0.0, 0.0};
  if (p.model == MK_MODEL_FLOW) {
    r.r0 = p.rho0;
  } else if (p.model == MK_MODEL_CONVECTION) {
    r.r0 = p.rho0;
    r.r1 = p.s_ref;  // t: the buoyancy reference value
  } else if (p.model == MK_MODEL_MULTIPHASE) {
    r.r0 = 0.0;  // g: rest state p* = 0, u = 0
    r.r1 = 1.0;  // h: liquid phi = 1
  } else {
    r.r0 = -1.0;      // g: liquid phi = -1
    r.r1 = -p.delta;  // t/U: far-field value
  }
  return r;
}

// ========================================================= MULTIPHASE (K4)
// The pressure lattice g rests at 0 (p* = 0, u = 0), so its deviation is g
// itself; the Allen-Cahn lattice h rests at the liquid, h_i = w_i (phi = 1).
template <class T>
struct MpK {
  T beta, kappa, om_h, coef_wet, inv_w4, rho_l, rho_g, tau_l, tau_g, gx, gy, gz;
  T ref_h;  // 1
};

// With 16-bit storage the Allen-Cahn rest population h_0 (always stored at
// its own cell, in both AA parities) lives in an FP32 plane H0 and absorbs the
// rounding residual of the cell's 18 moving populations, so sum(h) — the
// conserved phase volume — is kept to FP32 rounding.
template <class S>
struct Rest32 {
  static constexpr bool on = Stor<S>::bytes == 2;
};

template <class S, class P, int PARITY, class NB>
__device__ __forceinline__ void mp_phi_cell(const S* __restrict__ H, const float* __restrict__ H0, P* __restrict__ phi,
                                            int64_t stride, const NB& nb, int c, typename Stor<S>::T ref_h) {
  typedef typename Stor<S>::T T;
  T s = Rest32<S>::on ? T(H0[c]) : ld_in<S, 19>(H, stride, nb, PARITY, c, 0);
  if constexpr (Stor<S>::scaled) {
    // 16-bit storage holds h'/w: sum the axis and the diagonal classes in
    // stored units and scale once per class (2 multiplies instead of 18)
    T sa = T(0), sd = T(0);
#pragma unroll
    for (int i = 1; i < 7; ++i) sa += ld_in_raw<S, 19>(H, stride, nb, PARITY, c, i);
#pragma unroll
    for (int i = 7; i < 19; ++i) sd += ld_in_raw<S, 19>(H, stride, nb, PARITY, c, i);
    s += T(wq<19>(1)) * sa + T(wq<19>(7)) * sd;
  } else {
#pragma unroll
    for (int i = 1; i < 19; ++i) s += ld_in<S, 19>(H, stride, nb, PARITY, c, i);
  }
  phi[c] = P(ref_h + s);
}


// Where a collision reads phi: its own cell (center) and the neighbour
// (dx, dy, dz) (at).  PhiGlobal reads the phi array, which no kernel writes
// while a two-kernel step's collision runs; the fused step reads a shared
// memory ring of staged planes instead (PhiRing, below).
template <class P, class NB>
struct PhiGlobal {
  const P* __restrict__ phi;
  const NB& nb;
  int c;
  __device__ __forceinline__ P center() const { return phi[c]; }
  __device__ __forceinline__ P at(int dx, int dy, int dz) const { return __ldg(phi + nb_idx(nb, dx, dy, dz)); }
};

// Density, phi gradient and total force of a fluid cell (shared by the
// collision and by field output so both see identical values).
template <class T, class P, class NB, class PH>
__device__ __forceinline__ void mp_force_src(const PH& src, const NB& nb, const MpK<T>& k, T pstar, T& ph, T& rho,
                                             T (&gp)[3], T (&F)[3]) {
  ph = T(src.center());
  const T wall = ph + k.coef_wet * ph * (T(1) - ph);
  T gx = T(0), gy = T(0), gz = T(0), l = T(0);
#pragma unroll
  for (int i = 1; i < 19; ++i) {
    const T fn = nb_fluid(nb, ex(i), ey(i), ez(i)) ? T(src.at(ex(i), ey(i), ez(i))) : wall;
    const T w = T(wq<19>(i));
    if (ex(i)) gx += (w * T(ex(i))) * fn;
    if (ey(i)) gy += (w * T(ey(i))) * fn;
    if (ez(i)) gz += (w * T(ez(i))) * fn;
    l += w * (fn - ph);
  }
  gp[0] = T(3) * gx;
  gp[1] = T(3) * gy;
  gp[2] = T(3) * gz;
  const T lap = T(6) * l;
  const T drho = k.rho_l - k.rho_g;
  rho = k.rho_g + ph * drho;
  const T mu = T(4) * k.beta * ph * (ph - T(1)) * (ph - T(0.5)) - k.kappa * lap;
  const T pg = pstar * (T(1) / T(3)) * drho;
  F[0] = mu * gp[0] + rho * k.gx - pg * gp[0];
  F[1] = mu * gp[1] + rho * k.gy - pg * gp[1];
  F[2] = mu * gp[2] + rho * k.gz - pg * gp[2];
}

template <class T, class P, class NB>
__device__ __forceinline__ void mp_force(const P* __restrict__ phi, const NB& nb, int c, const MpK<T>& k, T pstar,
                                         T& ph, T& rho, T (&gp)[3], T (&F)[3]) {
  mp_force_src<T, P, NB>(PhiGlobal<P, NB>{phi, nb, c}, nb, k, pstar, ph, rho, gp, F);
}

template <class T>
MpK<T> mp_coef(const mk_params& p, Refs r) {
  MpK<T> k;
  k.beta = T(12.0 * p.sigma / p.width);
  k.kappa = T(1.5 * p.sigma * p.width);
  k.om_h = T(1.0 / (3.0 * p.mobility + 0.5));
  k.coef_wet = T(4.0 * std::cos(p.contact_angle * M_PI / 180.0) / p.width);
  k.inv_w4 = T(4.0 / p.width);
  k.rho_l = T(p.rho_l);
  k.rho_g = T(p.rho_g);
  k.tau_l = T(p.tau_l);
  k.tau_g = T(p.tau_g);
  k.gx = T(p.force[0]);
  k.gy = T(p.force[1]);
  k.gz = T(p.force[2]);
  k.ref_h = T(r.r1);
  return k;
}

}  // namespace mks

#endif
