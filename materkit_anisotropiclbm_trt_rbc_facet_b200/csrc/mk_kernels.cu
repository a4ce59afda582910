// mk_kernels.cu — sm_100a kernels of the coupled step and their launchers.
//
// K1 k_flow          fused collide + AA stream, D3Q19/D3Q27, BGK/TRT/MRT, Guo
//                    forcing, half-way bounce-back           (mkFluidsLBM::propagate/
//                    relaxation, mkFluidsLBM.h:47-49; mkNode::collision_*, mkNode.h:74-87)
// K4 k_mp_phi        phi = sum h of the streamed Allen-Cahn populations
//    k_mp_collide    MRT pressure/velocity lattice + conservative Allen-Cahn lattice,
//                    surface tension, gravity, wetting       (mkFluidsMultiphase::propagate/
//                    relaxation, mkFluidsMultiphase.h:52-57; getEquPDFsLiang/PhiLiang, mkNode.h:38-40)
// K3 k_pf_phi        phi = sum g of the streamed phase-field populations
// K2/K3 k_dend_collide  anisotropic phase field + D3Q7 thermal ADE with latent heat
//                    (mkPhaseField::relaxation_anisotropy_thermal, mkPhaseField.h:46;
//                    mkThermalField::propagate/relaxation, mkThermalField.h:33-34)
// K6 k_diag_*        FP64 warp-shuffle reductions (check_variables, mkFluidsLBM.h:55)
//
// All kernels are HBM-bound stencils: one thread per cell, x fastest, so a
// warp touches 32 consecutive cells of every population plane.  No tensor
// cores: the step is not a contraction.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "mk_device.cuh"
#include "mk_engine.hpp"
#include "mk_models.hpp"
#include "mk_shared.cuh"

using namespace mkd;
using namespace mks;

namespace {

// ================================================================ FLOW (K1)
template <class T>
struct FlowK {
  T om, om_m, Fx, Fy, Fz;
  T ref;  // rho0
};

// Moments, velocity (half-force corrected) and collision of one cell's Q
// deviations f_i - w_i rho0 in place, with the Guo force F.
template <class T, int Q, int COLL>
__device__ __forceinline__ void flow_relax(T (&f)[Q], const FlowK<T>& k, const T Fx, const T Fy, const T Fz, T& ux,
                                           T& uy, T& uz) {
  T drho = T(0), jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    drho += f[i];
    if (ex(i)) jx += T(ex(i)) * f[i];
    if (ey(i)) jy += T(ey(i)) * f[i];
    if (ez(i)) jz += T(ez(i)) * f[i];
  }
  const T rho = k.ref + drho;
  const T irho = div_fast(T(1), rho);
  ux = (jx + T(0.5) * Fx) * irho;
  uy = (jy + T(0.5) * Fy) * irho;
  uz = (jz + T(0.5) * Fz) * irho;
  const T uu = ux * ux + uy * uy + uz * uz;
  if constexpr (COLL == MK_COLL_MRT && Q == 19) {
    MrtIn<T> q;  // equilibrium deviation: w [drho + rho (3eu + 4.5(eu)^2 - 1.5u^2)]
    q.a0 = drho - T(1.5) * rho * uu;
    q.bx = rho * ux;
    q.by = rho * uy;
    q.bz = rho * uz;
    q.qxx = rho * ux * ux;
    q.qyy = rho * uy * uy;
    q.qzz = rho * uz * uz;
    q.qxy = rho * ux * uy;
    q.qxz = rho * ux * uz;
    q.qyz = rho * uy * uz;
    q.Fx = Fx;
    q.Fy = Fy;
    q.Fz = Fz;
    q.ux = ux;
    q.uy = uy;
    q.uz = uz;
    q.sF = T(1);
    q.s_nu = k.om;
    mrt19_collide_moments<T>(f, q);
    return;
  }
  const T uF = ux * Fx + uy * Fy + uz * Fz;
  T feq[Q], Fi[Q];  // equilibrium deviations and Guo force terms
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const T w = T(wq<Q>(i));
    const T eu = T(ex(i)) * ux + T(ey(i)) * uy + T(ez(i)) * uz;
    const T eF = T(ex(i)) * Fx + T(ey(i)) * Fy + T(ez(i)) * Fz;
    feq[i] = w * (drho + rho * (T(3) * eu + T(4.5) * eu * eu - T(1.5) * uu));
    Fi[i] = w * (T(3) * eF + T(9) * eu * eF - T(3) * uF);
  }
  if (COLL == MK_COLL_BGK) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] += -k.om * (f[i] - feq[i]) + (T(1) - T(0.5) * k.om) * Fi[i];
  } else if (COLL == MK_COLL_TRT) {
    T fo[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const int j = inv(i);
      const T fp = T(0.5) * (f[i] + f[j]), fm = T(0.5) * (f[i] - f[j]);
      const T ep = T(0.5) * (feq[i] + feq[j]), em = T(0.5) * (feq[i] - feq[j]);
      const T Fp = T(0.5) * (Fi[i] + Fi[j]), Fm = T(0.5) * (Fi[i] - Fi[j]);
      fo[i] = f[i] - k.om * (fp - ep) - k.om_m * (fm - em) + (T(1) - T(0.5) * k.om) * Fp +
              (T(1) - T(0.5) * k.om_m) * Fm;
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = fo[i];
  }
}

template <class S, int Q, int COLL, int PARITY>
__global__ void __launch_bounds__(256) k_flow(S* __restrict__ A, const Geom g, const FlowK<typename Stor<S>::T> k) {
  typedef typename Stor<S>::T T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const Nbr nb(g, x, y, z);
  const int c = nb.idx(0, 0, 0);
  T f[Q];  // deviations f_i - w_i rho0
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = ld_in<S, Q>(A, g.stride, nb, PARITY, c, i);
  T ux, uy, uz;
  flow_relax<T, Q, COLL>(f, k, k.Fx, k.Fy, k.Fz, ux, uy, uz);
#pragma unroll
  for (int i = 0; i < Q; ++i) st_out<S, Q>(A, g.stride, nb, PARITY, c, i, f[i]);
}

// ================================================== CONVECTION (RBC, a3/a7)
// Flow lattice with the Boussinesq force F = -rho0 beta (T - T_ref) g and a
// D3Q7 advection-diffusion lattice t_eq = w T (1 + 4 e.u) (mkThermalField
// relaxation with the flow's velocity), both held as deviations (f - w rho0,
// t - w T_ref).  Populations bounced at a plate of `axis` get the plate's
// correction on read: + 6 w rho0 e.u_w for the flow (a moving wall; Couette,
// bdyCouette), t -> -t + 2 w (T_w - T_ref) for the scalar (Dirichlet anti-
// bounce-back; bdy_constT / bdy_RBC).  SCALAR = false is the flow model with
// moving plates and its constant body force.
template <class T>
struct ConvK {
  FlowK<T> f;       // om, om_m, Fx..Fz (flow model body force), ref = rho0
  T om_t, ref_t;    // scalar relaxation rate and rest value (T_ref)
  T bg[3];          // -rho0 beta g
  T tw2[2];         // 2 (T_w - T_ref) of the low / high plate
  T uw6[2][3];      // 6 rho0 u_w of the low / high plate
  int axis, lo, hi; // plate axis and the fluid span on it
};

__device__ __forceinline__ int e_on(int i, int axis) { return axis == 0 ? ex(i) : (axis == 1 ? ey(i) : ez(i)); }

template <class S, int Q, int COLL, int PARITY, bool SCALAR, bool WALLS, class NB>
__device__ __forceinline__ void conv_cell(S* __restrict__ F, S* __restrict__ Tp, const int64_t stride, const NB& nb,
                                          const int c, const int coord, const ConvK<typename Stor<S>::T>& k) {
  typedef typename Stor<S>::T T;
  T f[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    f[i] = ld_in<S, Q>(F, stride, nb, PARITY, c, i);
    if (WALLS && !nb_fluid(nb, -ex(i), -ey(i), -ez(i))) {
      const int ea = e_on(i, k.axis);
      const int p = coord - ea;
      const int side = ea == 0 ? -1 : (p < k.lo ? 0 : (p > k.hi ? 1 : -1));
      if (side >= 0)
        f[i] += T(wq<Q>(i)) * (T(ex(i)) * k.uw6[side][0] + T(ey(i)) * k.uw6[side][1] + T(ez(i)) * k.uw6[side][2]);
    }
  }
  T t[7], dT = T(0);
  if constexpr (SCALAR) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      t[i] = ld_in<S, 7>(Tp, stride, nb, PARITY, c, i);
      if (WALLS && !nb_fluid(nb, -ex(i), -ey(i), -ez(i))) {
        const int ea = e_on(i, k.axis);
        const int p = coord - ea;
        const int side = ea == 0 ? -1 : (p < k.lo ? 0 : (p > k.hi ? 1 : -1));
        if (side >= 0) t[i] = -t[i] + T(wq<7>(i)) * k.tw2[side];
      }
      dT += t[i];
    }
  }
  T ux, uy, uz;
  if constexpr (SCALAR)
    flow_relax<T, Q, COLL>(f, k.f, k.bg[0] * dT, k.bg[1] * dT, k.bg[2] * dT, ux, uy, uz);
  else
    flow_relax<T, Q, COLL>(f, k.f, k.f.Fx, k.f.Fy, k.f.Fz, ux, uy, uz);
#pragma unroll
  for (int i = 0; i < Q; ++i) st_out<S, Q>(F, stride, nb, PARITY, c, i, f[i]);
  if constexpr (SCALAR) {
    const T Tabs = k.ref_t + dT;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      const T w = T(wq<7>(i));
      const T eu = T(ex(i)) * ux + T(ey(i)) * uy + T(ez(i)) * uz;
      st_out<S, 7>(Tp, stride, nb, PARITY, c, i, t[i] - k.om_t * (t[i] - w * (dT + T(4) * Tabs * eu)));
    }
  }
}

template <class S, int Q, int COLL, int PARITY, bool SCALAR>
__global__ void __launch_bounds__(256)
    k_conv(S* __restrict__ F, S* __restrict__ Tp, const Geom g, const ConvK<typename Stor<S>::T> k) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const int coord = k.axis == 0 ? x : (k.axis == 1 ? y : z);
  if (fast_cell(g, x, y, z)) {
    const Fast fa = make_fast(g, x, y, z);
    conv_cell<S, Q, COLL, PARITY, SCALAR, false>(F, Tp, g.stride, fa, fa.c, coord, k);
  } else {
    const Nbr nb(g, x, y, z);
    conv_cell<S, Q, COLL, PARITY, SCALAR, true>(F, Tp, g.stride, nb, nb.idx(0, 0, 0), coord, k);
  }
}

}  // namespace

#include "mk_dendrite.cuh"

namespace {

// ============================================== FLOW + DENDRITE (a1/a7/a8)
// run_flow_thermal_dendrite (MaterKit.cpp:467-527): per loop the flow lattice
// with the partially saturated porous bounce-back (mkFluidsMRT::propagate_PBB
// and relaxation), the phase field, the thermal lattice advected by the flow,
// then the inflow/outflow faces (bdyVelocity, bdy_flowin).  The porous
// bounce-back follows Noble & Torczynski (Int. J. Mod. Phys. C 9 (1998)
// 1189): with the solid fraction n_s = clamp((1 + phi)/2) of the previous
// loop and B = n_s (tau - 1/2) / ((1 - n_s) + (tau - 1/2)),
//   f* = f_coll + B (Omega_s - (f_coll - f)),
//   Omega_s = f_inv(i) - f_i + feq_i(rho, 0) - feq_inv(i)(rho, u).
template <class T>
struct FdK {
  FlowK<T> f;     // flow lattice coefficients (ref = rho0)
  T half;         // tau - 1/2
  T u0[3];        // inflow velocity
  T ref_g, ref_t; // rest values of the phase-field and thermal lattices (-1, -Delta)
  int inlet;      // 1: inflow at x = 0, outflow at x = nx - 1
};

// BGK / TRT collision with the porous bounce-back, over opposite pairs
// (i, j = inv i; BGK is TRT with omega- = omega+).  With e_j = -e_i the pair's
// symmetric and antisymmetric equilibrium parts are w (drho + rho (4.5 eu^2 -
// 1.5 u^2)) and w rho 3 eu, the Guo force parts w (9 eu eF - 3 u.F) and w 3 eF.
// The porous term f* = f_coll + B (f_inv(i) - rho w_i P_i - f_coll),
// P_i = -3 e_i.u + 4.5 (e_i.u)^2 - 1.5 u^2 (rho w_i - feq_inv(i)(rho, u) =
// -rho w_i P_i), is the Noble-Torczynski form with f_i cancelled; it is
// evaluated only when a lane of the warp has B > 0.  FORCE = false drops the
// force terms (a zero body force).
// Mass and momentum deviations of Q populations; SC: f holds f'/w (16-bit
// stored units), summed per weight class and scaled once per class.
__host__ __device__ constexpr int wclass_rep(int i) { return i == 0 ? 0 : (i <= 6 ? 1 : (i <= 18 ? 7 : 19)); }

template <class T, int Q, bool SC>
__device__ __forceinline__ void flow_moments(const T (&f)[Q], T& drho, T& jx, T& jy, T& jz) {
  T d[4] = {T(0), T(0), T(0), T(0)}, x[4] = {T(0), T(0), T(0), T(0)}, y[4] = {T(0), T(0), T(0), T(0)},
    z[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int c = SC ? (i == 0 ? 0 : (i <= 6 ? 1 : (i <= 18 ? 2 : 3))) : 0;
    d[c] += f[i];
    if (ex(i)) x[c] += T(ex(i)) * f[i];
    if (ey(i)) y[c] += T(ey(i)) * f[i];
    if (ez(i)) z[c] += T(ez(i)) * f[i];
  }
  if constexpr (SC) {
    const T w0 = T(wq<Q>(0)), w1 = T(wq<Q>(1)), w2 = T(wq<Q>(7)), w3 = Q == 27 ? T(wq<Q>(19)) : T(0);
    drho = w0 * d[0] + w1 * d[1] + w2 * d[2] + w3 * d[3];
    jx = w1 * x[1] + w2 * x[2] + w3 * x[3];
    jy = w1 * y[1] + w2 * y[2] + w3 * y[3];
    jz = w1 * z[1] + w2 * z[2] + w3 * z[3];
  } else {
    drho = d[0];
    jx = x[0];
    jy = y[0];
    jz = z[0];
  }
}

template <class T, int Q, int COLL, bool FORCE, bool SC = false>
__device__ __forceinline__ void fd_relax(T (&f)[Q], const FlowK<T>& k, const T ns, const T half, T& ux, T& uy,
                                         T& uz) {
  T drho, jx, jy, jz;
  flow_moments<T, Q, SC>(f, drho, jx, jy, jz);
  const T rho = k.ref + drho;
  const T irho = div_fast(T(1), rho);
  ux = FORCE ? (jx + T(0.5) * k.Fx) * irho : jx * irho;
  uy = FORCE ? (jy + T(0.5) * k.Fy) * irho : jy * irho;
  uz = FORCE ? (jz + T(0.5) * k.Fz) * irho : jz * irho;
  const T uu = ux * ux + uy * uy + uz * uz;
  const T uF = FORCE ? ux * k.Fx + uy * k.Fy + uz * k.Fz : T(0);
  const T om_p = k.om, om_m = COLL == MK_COLL_TRT ? k.om_m : k.om;
  const T gp = T(1) - T(0.5) * om_p, gm = T(1) - T(0.5) * om_m;
  const T B = ns > T(0) ? ns * half / ((T(1) - ns) + half) : T(0);
  // lanes past the row end or on walls have returned: vote among the active
  // lanes only (a lane with B > 0 always votes itself in)
  const bool psm = __any_sync(__activemask(), B > T(0));
  const T base = drho - T(1.5) * rho * uu;  // symmetric equilibrium part / w, less the 4.5 eu^2 term
  {
    const T w = SC ? T(1) : T(wq<Q>(0));  // SC: every term below carries w, divided out
    T fc = f[0] - om_p * (f[0] - w * base);
    if (FORCE) fc += gp * w * T(-3) * uF;
    if (psm) fc += B * (f[0] - rho * w * T(-1.5) * uu - fc);
    f[0] = fc;
  }
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const int j = i + 1;
    const T w = SC ? T(1) : T(wq<Q>(i));
    const T eu = T(ex(i)) * ux + T(ey(i)) * uy + T(ez(i)) * uz;
    const T fp = T(0.5) * (f[i] + f[j]), fm = T(0.5) * (f[i] - f[j]);
    const T ep = w * (base + T(4.5) * rho * eu * eu), em = w * T(3) * rho * eu;
    T dp = -om_p * (fp - ep), dm = -om_m * (fm - em);
    if (FORCE) {
      const T eF = T(ex(i)) * k.Fx + T(ey(i)) * k.Fy + T(ez(i)) * k.Fz;
      dp += gp * w * (T(9) * eu * eF - T(3) * uF);
      dm += gm * w * T(3) * eF;
    }
    T ci = f[i] + dp + dm, cj = f[j] + dp - dm;
    if (psm) {
      const T q = T(4.5) * eu * eu - T(1.5) * uu;
      const T gi = f[j] - rho * w * (q - T(3) * eu);
      const T gj = f[i] - rho * w * (q + T(3) * eu);
      ci += B * (gi - ci);
      cj += B * (gj - cj);
    }
    f[i] = ci;
    f[j] = cj;
  }
}

// Flow lattice of one cell: collision with the porous bounce-back of the
// crystal (solid fraction of the previous loop's phi).  MRT collides in
// moment space and applies the porous term after it, reading the
// pre-collision populations again (each slot is read and written by this
// cell alone in the AA layout, and no store has happened yet).  The
// collision velocity goes to vel[3][ncell] for the thermal lattice and the
// boundary pass.
template <class S, class P, int Q, int COLL, int PARITY, bool FORCE, bool NEE, class NB>
__device__ __forceinline__ void fd_flow_cell(S* __restrict__ W, const P* __restrict__ phi_old, P* __restrict__ vel,
                                             const int64_t stride, const int64_t ncell, const NB& nb, const int c,
                                             const int x, const int nx, const FdK<typename Stor<S>::T>& k) {
  typedef typename Stor<S>::T T;
  // SC: 16-bit storage with BGK/TRT works in the stored units f'/w (the
  // weights enter only the class sums of the moments)
  constexpr bool SC = Stor<S>::scaled && COLL != MK_COLL_MRT;
  T f[Q];  // deviations f_i - w_i rho0 (or f'/w), post-collision after the relaxation
#pragma unroll
  for (int i = 0; i < Q; ++i)
    f[i] = SC ? ld_in_raw<S, Q>(W, stride, nb, PARITY, c, i) : ld_in<S, Q>(W, stride, nb, PARITY, c, i);
  T ux, uy, uz;
  const T ns = fmin(T(1), fmax(T(0), T(0.5) * (T(1) + T(phi_old[c]))));
  if constexpr (COLL == MK_COLL_MRT && Q == 19) {
    flow_relax<T, Q, COLL>(f, k.f, k.f.Fx, k.f.Fy, k.f.Fz, ux, uy, uz);
    if (ns > T(0)) {
      const T B = ns * k.half / ((T(1) - ns) + k.half);
      T drho = T(0);
#pragma unroll
      for (int i = 0; i < Q; ++i) drho += ld_in<S, Q>(W, stride, nb, PARITY, c, i);
      const T rho = k.f.ref + drho;
      const T uu = ux * ux + uy * uy + uz * uz;
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const T eu = T(ex(i)) * ux + T(ey(i)) * uy + T(ez(i)) * uz;
        const T fk = ld_in<S, Q>(W, stride, nb, PARITY, c, inv(i));
        f[i] += B * (fk - rho * T(wq<Q>(i)) * (T(-3) * eu + T(4.5) * eu * eu - T(1.5) * uu) - f[i]);
      }
    }
  } else {
    fd_relax<T, Q, COLL, FORCE, SC>(f, k.f, ns, k.half, ux, uy, uz);
  }
  if constexpr (NEE) {
    // inflow / outflow faces in registers: the cell at x = 0 (x = nx - 1)
    // takes the post-collision populations of its inner neighbour, the next
    // (previous) lane of its warp, f(b) = f(n) + feq(rho_b, u_b) - feq(rho_n, u_n),
    // inflow u_b = u0, rho_b = rho_n; outflow rho_b = rho0, u_b = u_n; the face
    // cell's velocity becomes u_b
    const unsigned act = __activemask();
    const bool edge = x == 0 || x == nx - 1;
    if (__any_sync(act, edge)) {
      const int lane = threadIdx.x & 31;
      const int src = x == 0 ? lane + 1 : lane - 1;
      // every lane sums its own post-collision moments; the face lanes take
      // their neighbour's four sums, then its populations one by one
      T drho, jx, jy, jz;
      flow_moments<T, Q, SC>(f, drho, jx, jy, jz);
      drho = __shfl_sync(act, drho, src);
      jx = __shfl_sync(act, jx, src);
      jy = __shfl_sync(act, jy, src);
      jz = __shfl_sync(act, jz, src);
      const T rn = k.f.ref + drho;
      const T un[3] = {jx / rn, jy / rn, jz / rn};
      const bool in = x == 0;
      const T ub[3] = {in ? k.u0[0] : un[0], in ? k.u0[1] : un[1], in ? k.u0[2] : un[2]};
      const T rb = in ? rn : k.f.ref;
      const T uun = un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
      const T uub = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const T v = __shfl_sync(act, f[i], src);
        if (edge) {
          const T w = SC ? T(1) : T(wq<Q>(i));
          const T eun = T(ex(i)) * un[0] + T(ey(i)) * un[1] + T(ez(i)) * un[2];
          const T eub = T(ex(i)) * ub[0] + T(ey(i)) * ub[1] + T(ez(i)) * ub[2];
          f[i] = v + w * ((rb - rn) + rb * (T(3) * eub + T(4.5) * eub * eub - T(1.5) * uub) -
                          rn * (T(3) * eun + T(4.5) * eun * eun - T(1.5) * uun));
        }
      }
      if (edge) {
        ux = ub[0];
        uy = ub[1];
        uz = ub[2];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    if constexpr (SC)
      st_out_raw<S, Q>(W, stride, nb, PARITY, c, i, f[i]);
    else
      st_out<S, Q>(W, stride, nb, PARITY, c, i, f[i]);
  }
  vel[c] = P(ux);
  vel[ncell + c] = P(uy);
  vel[2 * ncell + c] = P(uz);
}

template <class S, class P, int Q, int COLL, int PARITY, bool FORCE, bool NEE>
__global__ void __launch_bounds__(256)
    k_fd_flow(S* __restrict__ W, const P* __restrict__ phi_old, P* __restrict__ vel, const Geom g,
              const FdK<typename Stor<S>::T> k) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    fd_flow_cell<S, P, Q, COLL, PARITY, FORCE, NEE>(W, phi_old, vel, g.stride, ncell, fa, fa.c, x, g.nx, k);
  } else {
    const Nbr nb(g, x, y, z);
    fd_flow_cell<S, P, Q, COLL, PARITY, FORCE, NEE>(W, phi_old, vel, g.stride, ncell, nb, nb.idx(0, 0, 0), x, g.nx,
                                                    k);
  }
}

// Phase field and thermal lattice with the equilibrium advected by the
// loop's flow velocity.
// With the face pass (NEE) the cell keeps both lattices' outputs until the
// shuffles: four resident blocks per SM (64 registers, a few spilled bytes)
// measured faster (128^3 FP32 81.5 -> 72.1 us) than the default allocation.
template <class S, class P, int PARITY, bool GEN, bool NEE, bool SOL>
__global__ void __launch_bounds__(256, NEE ? 4 : 1)
    k_fd_dend(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phi_new, const P* __restrict__ phi_old,
              P* __restrict__ temp, const P* __restrict__ vel, const unsigned char* __restrict__ grain,
              const typename Stor<S>::T* __restrict__ rot, const Geom g, const DendK<typename Stor<S>::T> k) {
  typedef typename Stor<S>::T T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    const int c = fa.c;
    dend_cell<S, P, PARITY, SOL, GEN, FastW, true, NEE>(G, Tp, phi_new, phi_old, temp, grain, rot, g.stride, fa, c,
                                                          k, T(vel[c]), T(vel[ncell + c]), T(vel[2 * ncell + c]), x,
                                                          g.nx);
  } else {
    const Nbr nb(g, x, y, z);
    const int c = nb.idx(0, 0, 0);
    dend_cell<S, P, PARITY, SOL, GEN, Nbr, true, NEE>(G, Tp, phi_new, phi_old, temp, grain, rot, g.stride, nb, c, k,
                                                        T(vel[c]), T(vel[ncell + c]), T(vel[2 * ncell + c]), x, g.nx);
  }
}

// Non-equilibrium extrapolation of the x faces after the loop's collisions
// (boundary_vel, mkFluidsUser.cpp:455-617; bdy_flowin): with n the inner
// neighbour of the face cell b,
//   flow      f(b) = f(n) + feq(rho_b, u_b) - feq(rho_n, u_n)
//   phase     g(b) = g(n) + w (phi_b - phi_n)
//   thermal   t(b) = t(n) + w T_b (1 + 4 e.u_b) - w T_n (1 + 4 e.u_n)
// inflow (x = 0): u_b = u0, rho_b = rho_n, phi_b = -1, T_b = -Delta;
// outflow (x = nx - 1): rho_b = rho0, u_b = u_n, phi_b = phi_n, T_b = T_n;
// the face cell's temperature becomes T_b.
// rho_n, u_n, phi_n, T_n are moments of the post-collision populations of n,
// except the thermal u_n, the collision velocity of n (vel).  One thread
// per face cell; each writes only its own cell's outgoing slots and reads only
// those of x = 1 / x = nx - 2, so no two threads touch one slot.
template <class S, class P, int Q>
__global__ void __launch_bounds__(128)
    k_fd_nee(S* __restrict__ W, S* __restrict__ G, S* __restrict__ Tp, P* __restrict__ temp,
             const P* __restrict__ vel, const Geom g, int64_t steps_done, const FdK<typename Stor<S>::T> k) {
  typedef typename Stor<S>::T T;
  const int plane = g.ny * g.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * plane) return;
  const int side = t >= plane ? 1 : 0;
  const int yz = t - side * plane;
  const int y = yz % g.ny, z = yz / g.ny;
  const int xb = side == 0 ? 0 : g.nx - 1, xn = side == 0 ? 1 : g.nx - 2;
  if (!g.fluid(xb, y, z) || !g.fluid(xn, y, z)) return;
  const Nbr nbb(g, xb, y, z), nbn(g, xn, y, z);
  const int cb = nbb.idx(0, 0, 0), cn = nbn.idx(0, 0, 0);
  // flow lattice
  T fn[Q];
  T drho = T(0), jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    fn[i] = ld_out<S, Q>(W, g.stride, nbn, steps_done, cn, i);
    drho += fn[i];
    if (ex(i)) jx += T(ex(i)) * fn[i];
    if (ey(i)) jy += T(ey(i)) * fn[i];
    if (ez(i)) jz += T(ez(i)) * fn[i];
  }
  const T rn = k.f.ref + drho;
  const T un[3] = {jx / rn, jy / rn, jz / rn};
  const T ub[3] = {side == 0 ? k.u0[0] : un[0], side == 0 ? k.u0[1] : un[1], side == 0 ? k.u0[2] : un[2]};
  const T rb = side == 0 ? rn : k.f.ref;
  const T uun = un[0] * un[0] + un[1] * un[1] + un[2] * un[2];
  const T uub = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const T w = T(wq<Q>(i));
    const T eun = T(ex(i)) * un[0] + T(ey(i)) * un[1] + T(ez(i)) * un[2];
    const T eub = T(ex(i)) * ub[0] + T(ey(i)) * ub[1] + T(ez(i)) * ub[2];
    const T d = w * ((rb - rn) + rb * (T(3) * eub + T(4.5) * eub * eub - T(1.5) * uub) -
                     rn * (T(3) * eun + T(4.5) * eun * eun - T(1.5) * uun));
    st_layout<S, Q>(W, g.stride, nbb, steps_done, cb, i, fn[i] + d);
  }
  // phase-field and thermal lattices
  T gn[7], tn[7], sg = T(0), st = T(0);
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    gn[i] = ld_out<S, 7>(G, g.stride, nbn, steps_done, cn, i);
    tn[i] = ld_out<S, 7>(Tp, g.stride, nbn, steps_done, cn, i);
    sg += gn[i];
    st += tn[i];
  }
  const T phn = k.ref_g + sg, Tn = k.ref_t + st;
  const T phb = side == 0 ? T(-1) : phn, Tb = side == 0 ? k.ref_t : Tn;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  const T vn[3] = {T(vel[cn]), T(vel[ncell + cn]), T(vel[2 * ncell + cn])};
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    const T w = T(wq<7>(i));
    const T evn = T(ex(i)) * vn[0] + T(ey(i)) * vn[1] + T(ez(i)) * vn[2];
    const T evb = T(ex(i)) * ub[0] + T(ey(i)) * ub[1] + T(ez(i)) * ub[2];
    st_layout<S, 7>(G, g.stride, nbb, steps_done, cb, i, gn[i] + w * (phb - phn));
    st_layout<S, 7>(Tp, g.stride, nbb, steps_done, cb, i,
                    tn[i] + w * (Tb * (T(1) + T(4) * evb) - Tn * (T(1) + T(4) * evn)));
  }
  temp[cb] = P(Tb);
}

// ====================================================== MULTIGRAIN (f-3)
// run_multiPhaseField with mkFluidsUser::propagate / relaxation
// (mkFluidsUser.cpp:68-299): one D3Q19 lattice per grain (pop0 planes
// 19j .. 19j+18, held as g - w (-1); on a one-cell periodic z axis D3Q19
// reduces exactly to the D2Q9 set the reference ships), phi_j = sum g_j
// (streamed), the aggregate phi = (N - 1) + sum phi_j, and per grain
//   g_j* = g_j - om (g_j - geq_j) + w P_j + (1 - om/2) w lam_j (e.n_j),
// geq_j = w phi_j (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2) with u = grain_u for
// j = 1 and 0 otherwise (mkFluidsUser.cpp:220-226), P_j = -2 p_j kappa_j
// (sum_k p_k^2 - p_j^2), p = (1 + phi)/2, kappa_0 = 0; n_j = s_j / (|s_j| +
// 1e-6) with s_j = sum_i w_i e_i phi_j(x + e_i) (:201-208); lam_j = (1 -
// phi_j^2)/(sqrt2 W0); om = 1/(3 M + 1/2) (:282).
// The thermal lattice relaxes with latent heat (1/2) dphi of the aggregate.
template <class T>
struct MgK {
  T om, fo, inv_w, kappa, om_t, ref_t;
  T ux, uy, uz, uu;  // grain 1's equilibrium velocity and its square
  int ngr;
};

// One thread per (cell, grain): block z = plane + nz * (grain - j0).  A loop
// over the grains inside a thread keeps the per-direction neighbour offsets
// of the odd loop live across it (80-92 registers, 31-37% occupancy, 1.10 ms
// FP16 / 0.42 ms FP32 per odd-loop phi launch at 128^3 with 8 grains).
template <class S, class P, int PARITY, class NB>
__device__ __forceinline__ void mg_phi_cell(const S* __restrict__ Gj, P* __restrict__ phij, const int64_t stride,
                                            const NB& nb, const int c) {
  typedef typename Stor<S>::T T;
  T sum = T(-1);
  if constexpr (Stor<S>::scaled) {  // stored units, one multiply per weight class
    T sa = T(0), sd = T(0);
#pragma unroll
    for (int i = 1; i < 7; ++i) sa += ld_in_raw<S, 19>(Gj, stride, nb, PARITY, c, i);
#pragma unroll
    for (int i = 7; i < 19; ++i) sd += ld_in_raw<S, 19>(Gj, stride, nb, PARITY, c, i);
    sum += T(wq<19>(0)) * ld_in_raw<S, 19>(Gj, stride, nb, PARITY, c, 0) + T(wq<19>(1)) * sa + T(wq<19>(7)) * sd;
  } else {
#pragma unroll
    for (int i = 0; i < 19; ++i) sum += ld_in<S, 19>(Gj, stride, nb, PARITY, c, i);
  }
  phij[c] = P(sum);
}

// phi_j of every fluid cell.
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256) k_mg_phi(const S* __restrict__ G, P* __restrict__ phij, const Geom g, int j0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = (int)(blockIdx.z % (unsigned)g.nz);
  const int j = j0 + (int)(blockIdx.z / (unsigned)g.nz);
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  const S* Gj = G + (int64_t)j * 19 * g.stride;
  P* pj = phij + (int64_t)j * ncell;
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    mg_phi_cell<S, P, PARITY>(Gj, pj, g.stride, fa, fa.c);
  } else {
    const Nbr nb(g, x, y, z);
    mg_phi_cell<S, P, PARITY>(Gj, pj, g.stride, nb, nb.idx(0, 0, 0));
  }
}

// k_mg_phi with 16-bit storage, two cells of a row per thread (nx even):
// each slot pair of the even loop and each of the odd loop's slots without an
// x shift is one 32-bit load, phi_j is stored as a float2; each cell's sums
// keep mg_phi_cell's order (bit-identical).  A pair with a cell off the
// interior path or not fluid takes mg_phi_cell per cell.
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256) k_mg_phi2(const S* __restrict__ G, P* __restrict__ phij, const Geom g, int j0) {
  typedef typename Stor<S>::T T;
  static_assert(Stor<S>::scaled, "the pair form is the 16-bit one");
  const int x = 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = (int)(blockIdx.z % (unsigned)g.nz);
  const int j = j0 + (int)(blockIdx.z / (unsigned)g.nz);
  if (x >= g.nx || y >= g.ny) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  const S* Gj = G + (int64_t)j * 19 * g.stride;
  P* pj = phij + (int64_t)j * ncell;
  const bool f0 = g.fluid(x, y, z), f1 = g.fluid(x + 1, y, z);
  if (f0 && f1 && fastw_cell(g, x, y, z) && fastw_cell(g, x + 1, y, z)) {
    const FastW a = make_fastw(g, x, y, z), b = make_fastw(g, x + 1, y, z);
    T v0[19], v1[19];
#pragma unroll
    for (int i = 0; i < 19; ++i) {
      if (PARITY == 0 || ex(i) == 0) {
        ldr_pair(Gj + off_in<19>(g.stride, a, PARITY, a.c, i), v0[i], v1[i]);
      } else {
        v0[i] = ld_in_raw<S, 19>(Gj, g.stride, a, PARITY, a.c, i);
        v1[i] = ld_in_raw<S, 19>(Gj, g.stride, b, PARITY, b.c, i);
      }
    }
    T sa0 = T(0), sd0 = T(0), sa1 = T(0), sd1 = T(0);
#pragma unroll
    for (int i = 1; i < 7; ++i) {
      sa0 += v0[i];
      sa1 += v1[i];
    }
#pragma unroll
    for (int i = 7; i < 19; ++i) {
      sd0 += v0[i];
      sd1 += v1[i];
    }
    T sum0 = T(-1), sum1 = T(-1);
    sum0 += T(wq<19>(0)) * v0[0] + T(wq<19>(1)) * sa0 + T(wq<19>(7)) * sd0;
    sum1 += T(wq<19>(0)) * v1[0] + T(wq<19>(1)) * sa1 + T(wq<19>(7)) * sd1;
    st_pair(pj + a.c, P(sum0), P(sum1));
    return;
  }
#pragma unroll 1
  for (int k = 0; k < 2; ++k) {
    const int xx = x + k;
    if (!(k == 0 ? f0 : f1)) continue;
    if (fastw_cell(g, xx, y, z)) {
      const FastW fa = make_fastw(g, xx, y, z);
      mg_phi_cell<S, P, PARITY>(Gj, pj, g.stride, fa, fa.c);
    } else {
      const Nbr nb(g, xx, y, z);
      mg_phi_cell<S, P, PARITY>(Gj, pj, g.stride, nb, nb.idx(0, 0, 0));
    }
  }
}

// Per cell, once: the aggregate phi = (N - 1) + sum phi_j into phi_new and
// S2 = sum_k p_k^2, p = (1 + phi)/2, into plane N of phij (the grains'
// threads of the collision read it instead of all N order parameters each).
// A solid cell keeps its aggregate.
template <class S, class P>
__global__ void __launch_bounds__(256) k_mg_sums(P* __restrict__ phij, const P* __restrict__ phi_old,
                                                 P* __restrict__ phi_new, const Geom g, int ngr) {
  typedef typename Stor<S>::T T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  const int64_t c = g.idx(x, y, z);
  if (!g.fluid(x, y, z)) {
    phi_new[c] = phi_old[c];
    return;
  }
  T S2 = T(0), agg = T(ngr - 1);
  for (int q = 0; q < ngr; ++q) {
    const T fq = T(phij[(int64_t)q * ncell + c]);
    const T pk = T(0.5) * (T(1) + fq);
    S2 += pk * pk;
    agg += fq;
  }
  phi_new[c] = P(agg);
  phij[(int64_t)ngr * ncell + c] = P(S2);
}

// Grain j of one cell: its D3Q19 gradient, overlap penalty and relaxation.
// Grain 0's thread also relaxes the thermal lattice with the latent heat
// (1/2) dphi of the aggregate.
template <class S, class P, int PARITY, class NB>
__device__ __forceinline__ void mg_cell(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phij,
                                        const P* __restrict__ phi_new, const P* __restrict__ phi_old,
                                        P* __restrict__ temp, const int64_t stride, const int64_t ncell, const NB& nb,
                                        const int c, const int j, const MgK<typename Stor<S>::T>& k) {
  typedef typename Stor<S>::T T;
  S* Gj = G + (int64_t)j * 19 * stride;
  // FP32 / FP64: the grain's slots (and grain 0's thermal slots) go to L2
  // while the stencil and the penalty are computed (compiled out with 16-bit
  // storage, where it measured no gain)
  if constexpr (Stor<S>::bytes >= 4) {
#pragma unroll
    for (int i = 0; i < 19; ++i) pf_in<S, 19>(Gj, stride, nb, PARITY, c, i);
    if (j == 0) {
#pragma unroll
      for (int i = 0; i < 7; ++i) pf_in<S, 7>(Tp, stride, nb, PARITY, c, i);
    }
  }
  const T S2 = T(phij[(int64_t)k.ngr * ncell + c]);
  const P* f = phij + (int64_t)j * ncell;
  const T ph = T(f[c]);
  T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
  for (int i = 1; i < 19; ++i) {
    const T fn = nb_fluid(nb, ex(i), ey(i), ez(i)) ? T(__ldg(f + nb_idx(nb, ex(i), ey(i), ez(i)))) : ph;
    const T w = T(wq<19>(i));
    if (ex(i)) gx += (w * T(ex(i))) * fn;
    if (ey(i)) gy += (w * T(ey(i))) * fn;
    if (ez(i)) gz += (w * T(ez(i))) * fn;
  }
  // regularised at 1e-6: where grad phi_j vanishes (a seed centre on a
  // lattice point) its direction is rounding noise
  const T gs = sqrt(gx * gx + gy * gy + gz * gz) + T(1e-6);
  const T inv = Stor<S>::bytes == 2 ? div_fast(T(1), gs) : T(1) / gs;
  const T lam = (T(1) - ph * ph) * k.inv_w * k.fo;
  const T pj = T(0.5) * (T(1) + ph);
  const T Pj = j == 0 ? T(0) : T(-2) * pj * (S2 - pj * pj) * k.kappa;
  const T dph = ph + T(1);  // phi_j - ref
  const bool moving = j == 1;
  T gv[19];
#pragma unroll
  for (int i = 0; i < 19; ++i) gv[i] = ld_in<S, 19>(Gj, stride, nb, PARITY, c, i);
#pragma unroll
  for (int i = 0; i < 19; ++i) {
    const T w = T(wq<19>(i));
    const T en = (T(ex(i)) * gx + T(ey(i)) * gy + T(ez(i)) * gz) * inv;
    T eq = dph;  // geq - w ref, over w
    if (moving) {
      const T eu = T(ex(i)) * k.ux + T(ey(i)) * k.uy + T(ez(i)) * k.uz;
      eq += ph * (T(3) * eu + T(4.5) * eu * eu - T(1.5) * k.uu);
    }
    st_out<S, 19>(Gj, stride, nb, PARITY, c, i, gv[i] - k.om * (gv[i] - w * eq) + w * Pj + w * lam * en);
  }
  if (j != 0) return;
  // thermal lattice with latent heat (1/2) dphi of the aggregate
  T t[7], dT = T(0);
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    t[i] = ld_in<S, 7>(Tp, stride, nb, PARITY, c, i);
    dT += t[i];
  }
  const T lat = T(0.5) * (T(phi_new[c]) - T(phi_old[c]));
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    const T w = T(wq<7>(i));
    st_out<S, 7>(Tp, stride, nb, PARITY, c, i, t[i] - k.om_t * (t[i] - w * dT) + w * lat);
  }
  temp[c] = P(k.ref_t + dT);
}

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256)
    k_mg_collide(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phij, const P* __restrict__ phi_new,
                 const P* __restrict__ phi_old, P* __restrict__ temp, const Geom g, const MgK<typename Stor<S>::T> k,
                 int j0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = (int)(blockIdx.z % (unsigned)g.nz);
  const int j = j0 + (int)(blockIdx.z / (unsigned)g.nz);
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    mg_cell<S, P, PARITY>(G, Tp, phij, phi_new, phi_old, temp, g.stride, ncell, fa, fa.c, j, k);
  } else {
    const Nbr nb(g, x, y, z);
    mg_cell<S, P, PARITY>(G, Tp, phij, phi_new, phi_old, temp, g.stride, ncell, nb, nb.idx(0, 0, 0), j, k);
  }
}

// Initial state: grain j's order parameter -tanh((r_j - R_j)/(sqrt2 W0)) from
// its seed (gseeds: x, y, z, R per grain), the aggregate, T, and the
// equilibria of all lattices.
template <class S, class InT>
__global__ void k_mg_init(S* A0, S* A1, typename PhiOf<S>::type* phij, typename PhiOf<S>::type* phi0,
                          typename PhiOf<S>::type* phi1, typename PhiOf<S>::type* temp, const InT* __restrict__ in_t,
                          double d_t, const double* __restrict__ gseeds, int ngr, double W0, const Geom g,
                          int64_t ncell, Refs refs) {
  typedef typename PhiOf<S>::type P;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  const bool fl = g.fluid(x, y, z);
  const Nbr nb(g, x, y, z);
  double agg = ngr - 1.0;
  for (int j = 0; j < ngr; ++j) {
    const double dx = x - gseeds[4 * j], dy = y - gseeds[4 * j + 1], dz = z - gseeds[4 * j + 2];
    const double ph = -tanh((sqrt(dx * dx + dy * dy + dz * dz) - gseeds[4 * j + 3]) / (sqrt(2.0) * W0));
    phij[(int64_t)j * ncell + c] = P(ph);
    agg += ph;
    if (fl) put_eq<S, 19>(A0 + (int64_t)j * 19 * g.stride, g, nb, (int)c, ph, 0.0, 0.0, 0.0, 0.0, refs.r0);
  }
  phi0[c] = P(agg);
  phi1[c] = P(agg);
  const double tv = in_t ? double(in_t[c]) : d_t;
  temp[c] = P(tv);
  if (fl) put_eq<S, 7>(A1, g, nb, (int)c, tv, 0.0, 0.0, 0.0, 0.0, refs.r1);
}

// Grain field: the grain whose order parameter is largest (ties to the lower index).
template <class P>
__global__ void k_field_mg_grain(const P* __restrict__ phij, int ngr, int64_t n, double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int best = 0;
  P bv = phij[c];
  for (int j = 1; j < ngr; ++j) {
    const P v = phij[(int64_t)j * n + c];
    if (v > bv) {
      bv = v;
      best = j;
    }
  }
  out[c] = best;
}

// ===================================================================== INIT
template <class S, class InT>
__global__ void k_init(int model, int Q0, S* A0, S* A1, S* A2, int Q2, float* H0, typename PhiOf<S>::type* phi0,
                       typename PhiOf<S>::type* phi1, typename PhiOf<S>::type* temp, const InT* __restrict__ in_phi,
                       const InT* __restrict__ in_t, const InT* __restrict__ in_rho,
                       const InT* __restrict__ in_u, double d_rho, double d_ux, double d_uy, double d_uz,
                       double d_t, const Geom g, int64_t ncell, Refs refs) {
  typedef typename PhiOf<S>::type P;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  const double ph = in_phi ? in_phi[c] : 0.0;
  const double ux = in_u ? in_u[c] : d_ux, uy = in_u ? in_u[ncell + c] : d_uy, uz = in_u ? in_u[2 * ncell + c] : d_uz;
  if (phi0) phi0[c] = P(ph);
  if (phi1) phi1[c] = P(ph);
  const double tv = in_t ? in_t[c] : d_t;
  if (temp) temp[c] = P(tv);
  if (!g.fluid(x, y, z)) return;
  const Nbr nb(g, x, y, z);
  const int ci = (int)c;
  if (model == MK_MODEL_FLOW || model == MK_MODEL_CONVECTION) {
    const double r = in_rho ? in_rho[c] : d_rho;
    if (Q0 == 19)
      put_eq<S, 19>(A0, g, nb, ci, r, ux, uy, uz, 0.0, refs.r0);
    else
      put_eq<S, 27>(A0, g, nb, ci, r, ux, uy, uz, 0.0, refs.r0);
    if (model == MK_MODEL_CONVECTION) {
      // t_eq = w T (1 + 4 e.u), held as t - w T_ref
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        const double eu = ex(i) * ux + ey(i) * uy + ez(i) * uz;
        st_layout<S, 7>(A1, g.stride, nb, 0, ci, i,
                        typename Stor<S>::T(wq<7>(i) * ((tv - refs.r1) + 4.0 * tv * eu)));
      }
    }
  } else if (model == MK_MODEL_MULTIPHASE) {
    // g = geq(p* = 0, u) = w (3eu + 4.5eu^2 - 1.5u^2); h = phi w (1 + ...)
    put_eq<S, 19>(A0, g, nb, ci, 1.0, ux, uy, uz, -1.0, refs.r0);
    put_eq<S, 19>(A1, g, nb, ci, ph, ux, uy, uz, 0.0, refs.r1);
    if (H0) H0[c] = float(wq<19>(0) * ((ph - refs.r1) - 1.5 * ph * (ux * ux + uy * uy + uz * uz)));
  } else if (mkm::flow_coupled(model)) {
    // the flow starts at rho0 with u0 scaled by the liquid fraction (unless
    // given); the thermal equilibrium carries the same velocity
    const double ns = fmin(1.0, fmax(0.0, 0.5 * (1.0 + ph)));
    const double vx = in_u ? ux : (1.0 - ns) * d_ux, vy = in_u ? uy : (1.0 - ns) * d_uy,
                 vz = in_u ? uz : (1.0 - ns) * d_uz;
    const double r = in_rho ? in_rho[c] : d_rho;
    put_eq<S, 7>(A0, g, nb, ci, ph, 0.0, 0.0, 0.0, 0.0, refs.r0);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      const double eu = ex(i) * vx + ey(i) * vy + ez(i) * vz;
      st_layout<S, 7>(A1, g.stride, nb, 0, ci, i, typename Stor<S>::T(wq<7>(i) * ((tv - refs.r1) + 4.0 * tv * eu)));
    }
    if (Q2 == 19)
      put_eq<S, 19>(A2, g, nb, ci, r, vx, vy, vz, 0.0, d_rho);
    else
      put_eq<S, 27>(A2, g, nb, ci, r, vx, vy, vz, 0.0, d_rho);
  } else {
    put_eq<S, 7>(A0, g, nb, ci, ph, 0.0, 0.0, 0.0, 0.0, refs.r0);
    put_eq<S, 7>(A1, g, nb, ci, tv, 0.0, 0.0, 0.0, 0.0, refs.r1);
  }
}

// =================================================================== FIELDS
// Buoyancy coefficients of the stored scalar (convection): F = bg (T - T_ref).
struct Buoy {
  double bg[3], ref;
};

// Stored (post-collision) scalar T of a convection cell.
template <class S>
__device__ __forceinline__ double conv_T(const S* __restrict__ Tp, const Geom& g, const Nbr& nb, int64_t steps_done,
                                         int c, double ref) {
  double t = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i) t += double(ld_out<S, 7>(Tp, g.stride, nb, steps_done, c, i));
  return ref + t;
}

template <class S, int Q>
__global__ void k_field_flow(const S* __restrict__ A, const S* __restrict__ Tp, const Buoy bu, const Geom g,
                             int64_t steps_done, int field, double Fx, double Fy, double Fz, double rho0,
                             double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  if (!g.fluid(x, y, z)) {
    out[c] = field == MK_FIELD_RHO ? rho0 : (field == MK_FIELD_T ? bu.ref : 0.0);
    return;
  }
  const Nbr nb(g, x, y, z);
  if (Tp) {
    const double T = conv_T<S>(Tp, g, nb, steps_done, (int)c, bu.ref);
    if (field == MK_FIELD_T) {
      out[c] = T;
      return;
    }
    Fx = bu.bg[0] * (T - bu.ref);
    Fy = bu.bg[1] * (T - bu.ref);
    Fz = bu.bg[2] * (T - bu.ref);
  }
  double drho = 0, j[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const double f = double(ld_out<S, Q>(A, g.stride, nb, steps_done, (int)c, i));
    drho += f;
    j[0] += ex(i) * f;
    j[1] += ey(i) * f;
    j[2] += ez(i) * f;
  }
  const double rho = rho0 + drho;
  const double F[3] = {Fx, Fy, Fz};
  out[c] = field == MK_FIELD_RHO ? rho : (j[field - MK_FIELD_UX] - 0.5 * F[field - MK_FIELD_UX]) / rho;
}

template <class S>
__global__ void k_field_mp(const S* __restrict__ G, const typename PhiOf<S>::type* __restrict__ phi, const Geom g,
                           int64_t steps_done, int field, const MpK<typename Stor<S>::T> k, double* __restrict__ out) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  if (field == MK_FIELD_RHO) {
    out[c] = double(k.rho_g) + double(phi[c]) * (double(k.rho_l) - double(k.rho_g));
    return;
  }
  if (!g.fluid(x, y, z)) {
    out[c] = 0.0;
    return;
  }
  const Nbr nb(g, x, y, z);
  T pstar = T(0), j[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int i = 0; i < 19; ++i) {
    const T v = ld_out<S, 19>(G, g.stride, nb, steps_done, (int)c, i);
    pstar += v;
    j[0] += T(ex(i)) * v;
    j[1] += T(ey(i)) * v;
    j[2] += T(ez(i)) * v;
  }
  if (field == MK_FIELD_PRESSURE) {
    out[c] = double(pstar);
    return;
  }
  T ph, rho, gp[3], F[3];
  mp_force<T, P>(phi, nb, (int)c, k, pstar, ph, rho, gp, F);
  const int a = field - MK_FIELD_UX;
  out[c] = double(j[a] - F[a] / (T(2) * rho));
}

template <class P>
__global__ void k_field_copy(const P* __restrict__ a, const P* __restrict__ b, int64_t n, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = b ? double(a[i]) - double(b[i]) : double(a[i]);
}

template <class P>
__global__ void k_double_to_plane(const double* __restrict__ a, P* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = P(a[i]);
}

__global__ void k_to_f32(const double* __restrict__ a, int64_t n, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)a[i];
}

__global__ void k_field_geom(const Geom g, int field, const double* __restrict__ seeds, int nobj,
                             double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  if (field == MK_FIELD_FLAG)
    out[c] = g.fluid(x, y, z) ? MK_FLAG_FLUID : ((g.solid && g.solid[c]) ? MK_FLAG_SOLID : MK_FLAG_WALLS);
  else
    out[c] = nobj > 0 ? nearest_seed(seeds, nobj, x, y, z) : 0;
}

// Cell flags of the flow + dendrite model (reset_flags, mkPhaseField.h:37):
// solid where phi > 0, walls where the geometry has them, else fluid.
template <class P>
__global__ void k_field_fdflag(const Geom g, const P* __restrict__ phi, double* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int64_t c = g.idx(x, y, z);
  out[c] = !g.fluid(x, y, z) ? MK_FLAG_WALLS : (double(phi[c]) > 0.0 ? MK_FLAG_SOLID : MK_FLAG_FLUID);
}

// ============================================================ DIAGNOSTICS (K6)
__device__ __forceinline__ void warp_reduce(double (&v)[mke::DG_N]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < mke::DG_N; ++q) {
      const double r = __shfl_down_sync(0xffffffffu, v[q], o);
      v[q] = q == mke::DG_MAXU ? fmax(v[q], r) : v[q] + r;
    }
  }
}

// Block-level reduction of per-thread partials into partial[blockIdx.x].
__device__ __forceinline__ void block_reduce_store(double (&v)[mke::DG_N], double* __restrict__ partial) {
  __shared__ double sh[32][mke::DG_N];
  warp_reduce(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < mke::DG_N; ++q) sh[wid][q] = v[q];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < mke::DG_N; ++q) v[q] = lane < nw ? sh[lane][q] : (q == mke::DG_MAXU ? 0.0 : 0.0);
    warp_reduce(v);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < mke::DG_N; ++q) partial[(int64_t)blockIdx.x * mke::DG_N + q] = v[q];
  }
}

__device__ __forceinline__ void cell_coords(const Geom& g, int64_t c, int& x, int& y, int& z) {
  x = (int)(c % g.nx);
  const int64_t r = c / g.nx;
  y = (int)(r % g.ny);
  z = (int)(r / g.ny);
}

template <class S, int Q>
__global__ void __launch_bounds__(256) k_diag_flow(const S* __restrict__ A, const S* __restrict__ Tp, const Buoy bu,
                                                   int axis, const Geom g, int64_t steps_done, double Fx0,
                                                   double Fy0, double Fz0, double rho0, int64_t n,
                                                   double* __restrict__ partial) {
  double v[mke::DG_N];
#pragma unroll
  for (int q = 0; q < mke::DG_N; ++q) v[q] = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_coords(g, c, x, y, z);
    if (!g.fluid(x, y, z)) continue;
    const Nbr nb(g, x, y, z);
    double drho = 0, j[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double f = double(ld_out<S, Q>(A, g.stride, nb, steps_done, (int)c, i));
      drho += f;
      j[0] += ex(i) * f;
      j[1] += ey(i) * f;
      j[2] += ez(i) * f;
    }
    double Fx = Fx0, Fy = Fy0, Fz = Fz0, T = 0;
    if (Tp) {
      T = conv_T<S>(Tp, g, nb, steps_done, (int)c, bu.ref);
      Fx = bu.bg[0] * (T - bu.ref);
      Fy = bu.bg[1] * (T - bu.ref);
      Fz = bu.bg[2] * (T - bu.ref);
    }
    const double rho = rho0 + drho;
    const double mx = j[0] - 0.5 * Fx, my = j[1] - 0.5 * Fy, mz = j[2] - 0.5 * Fz;
    const bool bad = !(rho > 0.0) || !isfinite(rho) || !isfinite(mx) || !isfinite(my) || !isfinite(mz) ||
                     (Tp && !isfinite(T));
    v[mke::DG_MASS] += rho;
    v[mke::DG_MX] += mx;
    v[mke::DG_MY] += my;
    v[mke::DG_MZ] += mz;
    v[mke::DG_FLUID] += 1.0;
    v[mke::DG_BAD] += bad ? 1.0 : 0.0;
    if (!bad) v[mke::DG_MAXU] = fmax(v[mke::DG_MAXU], sqrt(mx * mx + my * my + mz * mz) / rho);
    if (Tp) {
      v[mke::DG_HEAT] += T;
      v[mke::DG_FLUX] += (axis == 0 ? mx : (axis == 1 ? my : mz)) / rho * T;
    }
  }
  block_reduce_store(v, partial);
}

template <class S>
__global__ void __launch_bounds__(256) k_diag_mp(const S* __restrict__ G, const typename PhiOf<S>::type* __restrict__ phi,
                                                 const Geom g, int64_t steps_done, const MpK<typename Stor<S>::T> k,
                                                 int64_t n, double* __restrict__ partial) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  double v[mke::DG_N];
#pragma unroll
  for (int q = 0; q < mke::DG_N; ++q) v[q] = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_coords(g, c, x, y, z);
    if (!g.fluid(x, y, z)) continue;
    const Nbr nb(g, x, y, z);
    T pstar = T(0), j[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int i = 0; i < 19; ++i) {
      const T f = ld_out<S, 19>(G, g.stride, nb, steps_done, (int)c, i);
      pstar += f;
      j[0] += T(ex(i)) * f;
      j[1] += T(ey(i)) * f;
      j[2] += T(ez(i)) * f;
    }
    T ph, rho, gp[3], F[3];
    mp_force<T, P>(phi, nb, (int)c, k, pstar, ph, rho, gp, F);
    double u[3];
    for (int a = 0; a < 3; ++a) u[a] = double(j[a] - F[a] / (T(2) * rho));
    const double r = double(rho), p = double(ph);
    const bool bad = !isfinite(p) || !isfinite(double(pstar)) || !(r > 0.0) || !isfinite(u[0]) || !isfinite(u[1]) ||
                     !isfinite(u[2]);
    v[mke::DG_MASS] += r;
    v[mke::DG_MX] += r * u[0];
    v[mke::DG_MY] += r * u[1];
    v[mke::DG_MZ] += r * u[2];
    v[mke::DG_PHI] += p;
    v[mke::DG_SOLID] += p < 0.5 ? 1.0 : 0.0;
    v[mke::DG_FLUID] += 1.0;
    v[mke::DG_BAD] += bad ? 1.0 : 0.0;
    if (!bad) v[mke::DG_MAXU] = fmax(v[mke::DG_MAXU], sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
  }
  block_reduce_store(v, partial);
}

// Flow + dendrite: the flow lattice's mass, momentum and speed with the phase
// field's and the thermal lattice's sums.
template <class S, class P, int Q>
__global__ void __launch_bounds__(256) k_diag_fd(const S* __restrict__ W, const P* __restrict__ phi,
                                                 const P* __restrict__ phi_prev, const P* __restrict__ temp,
                                                 const Geom g, int64_t steps_done, double Fx, double Fy, double Fz,
                                                 double rho0, int solutal, int64_t n, double* __restrict__ partial) {
  double v[mke::DG_N];
#pragma unroll
  for (int q = 0; q < mke::DG_N; ++q) v[q] = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_coords(g, c, x, y, z);
    if (!g.fluid(x, y, z)) continue;
    const Nbr nb(g, x, y, z);
    double drho = 0, j[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double f = double(ld_out<S, Q>(W, g.stride, nb, steps_done, (int)c, i));
      drho += f;
      j[0] += ex(i) * f;
      j[1] += ey(i) * f;
      j[2] += ez(i) * f;
    }
    const double rho = rho0 + drho;
    const double mx = j[0] - 0.5 * Fx, my = j[1] - 0.5 * Fy, mz = j[2] - 0.5 * Fz;
    const double p = double(phi[c]), pp = double(phi_prev[c]), t = double(temp[c]);
    const bool bad = !(rho > 0.0) || !isfinite(rho) || !isfinite(mx) || !isfinite(my) || !isfinite(mz) ||
                     !isfinite(p) || !isfinite(t);
    v[mke::DG_MASS] += rho;
    v[mke::DG_MX] += mx;
    v[mke::DG_MY] += my;
    v[mke::DG_MZ] += mz;
    v[mke::DG_PHI] += p;
    v[mke::DG_SOLID] += p > 0.0 ? 1.0 : 0.0;
    if (solutal)
      v[mke::DG_SOLUTE] += t;
    else
      v[mke::DG_HEAT] += t - 0.5 * pp;
    v[mke::DG_FLUID] += 1.0;
    v[mke::DG_BAD] += bad ? 1.0 : 0.0;
    if (!bad) v[mke::DG_MAXU] = fmax(v[mke::DG_MAXU], sqrt(mx * mx + my * my + mz * mz) / rho);
  }
  block_reduce_store(v, partial);
}

template <class P>
__global__ void __launch_bounds__(256) k_diag_dend(const P* __restrict__ phi, const P* __restrict__ phi_prev,
                                                   const P* __restrict__ temp, const Geom g, int solutal, int64_t n,
                                                   double* __restrict__ partial) {
  double v[mke::DG_N];
#pragma unroll
  for (int q = 0; q < mke::DG_N; ++q) v[q] = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_coords(g, c, x, y, z);
    if (!g.fluid(x, y, z)) continue;
    const double p = double(phi[c]), pp = double(phi_prev[c]), t = double(temp[c]);
    const bool bad = !isfinite(p) || !isfinite(t);
    v[mke::DG_PHI] += p;
    v[mke::DG_SOLID] += p > 0.0 ? 1.0 : 0.0;
    if (solutal)
      v[mke::DG_SOLUTE] += t;
    else
      v[mke::DG_HEAT] += t - 0.5 * pp;
    v[mke::DG_FLUID] += 1.0;
    v[mke::DG_BAD] += bad ? 1.0 : 0.0;
  }
  block_reduce_store(v, partial);
}

// Second pass: one block sums the partials in a fixed order (deterministic).
__global__ void k_diag_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
  double v[mke::DG_N];
#pragma unroll
  for (int q = 0; q < mke::DG_N; ++q) v[q] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < mke::DG_N; ++q) {
      const double r = partial[(int64_t)b * mke::DG_N + q];
      v[q] = q == mke::DG_MAXU ? fmax(v[q], r) : v[q] + r;
    }
  __shared__ double sh[32][mke::DG_N];
  warp_reduce(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < mke::DG_N; ++q) sh[wid][q] = v[q];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    for (int q = 0; q < mke::DG_N; ++q) v[q] = lane < nw ? sh[lane][q] : 0.0;
    warp_reduce(v);
    if (lane == 0)
      for (int q = 0; q < mke::DG_N; ++q) out[q] = v[q];
  }
}

// ================================================================ launchers
template <class T>
FlowK<T> flow_coef(const mk_params& p, double ref) {
  FlowK<T> k;
  k.om = T(1.0 / p.tau);
  k.om_m = T(1.0 / (0.5 + p.magic / (p.tau - 0.5)));
  k.Fx = T(p.force[0]);
  k.Fy = T(p.force[1]);
  k.Fz = T(p.force[2]);
  k.ref = T(ref);
  return k;
}

template <class T>
DendK<T> dend_coef(const mk_params& p, Refs r) {
  return dend_params<T>(p, r.r0, r.r1);
}

Buoy buoy_of(const mk_params& p) {
  Buoy b;
  for (int a = 0; a < 3; ++a) b.bg[a] = -p.rho0 * p.beta * p.force[a];
  b.ref = p.s_ref;
  return b;
}

template <class T>
ConvK<T> conv_coef(const mk_params& p) {
  ConvK<T> k;
  k.f = flow_coef<T>(p, p.rho0);
  k.om_t = T(1.0 / (4.0 * p.D + 0.5));
  k.ref_t = T(p.s_ref);
  for (int a = 0; a < 3; ++a) k.bg[a] = T(-p.rho0 * p.beta * p.force[a]);
  const int ax = p.wall_axis >= 0 ? p.wall_axis : 0;
  const int n3[3] = {p.nx, p.ny, p.nz};
  k.axis = ax;
  k.lo = p.bc[ax] == MK_BC_WALLS ? 1 : 0;
  k.hi = p.bc[ax] == MK_BC_WALLS ? n3[ax] - 2 : n3[ax] - 1;
  for (int sd = 0; sd < 2; ++sd) {
    k.tw2[sd] = T(2.0 * (p.wall_value[sd] - p.s_ref));
    for (int a = 0; a < 3; ++a) k.uw6[sd][a] = T(6.0 * p.rho0 * p.wall_u[sd][a]);
  }
  return k;
}

template <class S, int Q, int COLL, bool SCALAR>
void launch_conv_t(mke::Engine& e, int parity, dim3 grid, dim3 block) {
  typedef typename Stor<S>::T T;
  const Geom g = make_geom(e);
  const ConvK<T> k = conv_coef<T>(e.p);
  if (parity == 0)
    k_conv<S, Q, COLL, 0, SCALAR><<<grid, block, 0, e.stream>>>((S*)e.pop0, (S*)e.pop1, g, k);
  else
    k_conv<S, Q, COLL, 1, SCALAR><<<grid, block, 0, e.stream>>>((S*)e.pop0, (S*)e.pop1, g, k);
}

template <class S, bool SCALAR>
void launch_conv(mke::Engine& e, int parity, dim3 grid, dim3 block) {
  const int Q = e.p.lattice, C = e.p.collision;
  if (Q == 19) {
    if (C == MK_COLL_BGK)
      launch_conv_t<S, 19, MK_COLL_BGK, SCALAR>(e, parity, grid, block);
    else if (C == MK_COLL_TRT)
      launch_conv_t<S, 19, MK_COLL_TRT, SCALAR>(e, parity, grid, block);
    else
      launch_conv_t<S, 19, MK_COLL_MRT, SCALAR>(e, parity, grid, block);
  } else {
    if (C == MK_COLL_BGK)
      launch_conv_t<S, 27, MK_COLL_BGK, SCALAR>(e, parity, grid, block);
    else
      launch_conv_t<S, 27, MK_COLL_TRT, SCALAR>(e, parity, grid, block);
  }
}

template <class S, int Q, int COLL>
void launch_flow_t(mke::Engine& e, int parity, dim3 grid, dim3 block) {
  typedef typename Stor<S>::T T;
  const Geom g = make_geom(e);
  const FlowK<T> k = flow_coef<T>(e.p, refs_of(e.p).r0);
  S* A = (S*)e.pop0;
  if (parity == 0)
    k_flow<S, Q, COLL, 0><<<grid, block, 0, e.stream>>>(A, g, k);
  else
    k_flow<S, Q, COLL, 1><<<grid, block, 0, e.stream>>>(A, g, k);
}

template <class S>
void launch_flow(mke::Engine& e, int parity, dim3 grid, dim3 block) {
  const int Q = e.p.lattice, C = e.p.collision;
  if (Q == 19) {
    if (C == MK_COLL_BGK)
      launch_flow_t<S, 19, MK_COLL_BGK>(e, parity, grid, block);
    else if (C == MK_COLL_TRT)
      launch_flow_t<S, 19, MK_COLL_TRT>(e, parity, grid, block);
    else
      launch_flow_t<S, 19, MK_COLL_MRT>(e, parity, grid, block);
  } else {
    if (C == MK_COLL_BGK)
      launch_flow_t<S, 27, MK_COLL_BGK>(e, parity, grid, block);
    else
      launch_flow_t<S, 27, MK_COLL_TRT>(e, parity, grid, block);
  }
}

template <class S>
void launch_dend(mke::Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  const DendK<T> k = dend_coef<T>(e.p, r);
  S* G = (S*)e.pop0;
  S* Tp = (S*)e.pop1;
  P* phi_old = (P*)e.phi[e.phi_cur];
  P* phi_new = (P*)e.phi[1 - e.phi_cur];
  P* temp = (P*)e.temp;
  if (ev) cudaEventRecord(ev[0], e.stream);
  if (parity == 0)
    k_pf_phi<S, P, 0><<<grid, block, 0, e.stream>>>(G, phi_old, phi_new, g, T(r.r0));
  else
    k_pf_phi<S, P, 1><<<grid, block, 0, e.stream>>>(G, phi_old, phi_new, g, T(r.r0));
  if (ev) {
    cudaEventRecord(ev[1], e.stream);
    cudaEventRecord(ev[2], e.stream);
  }
  const bool sol = e.p.model == MK_MODEL_SOLUTAL_DENDRITE;
  const bool gen = e.p.aniso != MK_ANISO_CUBIC;
  if (e.vel) {
    // an external velocity (mk_update_velocity): the scalar lattice advected
    // as in the flow + dendrite models, no inflow faces
    const P* vel = (const P*)e.vel;
#define MK_DENDV(PAR, GEN, SOL)                                                                                 \
  k_fd_dend<S, P, PAR, GEN, false, SOL><<<grid, block, 0, e.stream>>>(G, Tp, phi_new, phi_old, temp, vel, e.grain, \
                                                                      (const T*)e.rot, g, k)
    if (parity == 0) {
      if (sol)
        gen ? MK_DENDV(0, true, true) : MK_DENDV(0, false, true);
      else
        gen ? MK_DENDV(0, true, false) : MK_DENDV(0, false, false);
    } else {
      if (sol)
        gen ? MK_DENDV(1, true, true) : MK_DENDV(1, false, true);
      else
        gen ? MK_DENDV(1, true, false) : MK_DENDV(1, false, false);
    }
#undef MK_DENDV
    if (ev) cudaEventRecord(ev[3], e.stream);
    return;
  }
#define MK_DEND(PAR, SOL, GEN)                                                                              \
  k_dend_collide<S, P, PAR, SOL, GEN><<<grid, block, 0, e.stream>>>(G, Tp, phi_new, phi_old, temp, e.grain, \
                                                                    (const T*)e.rot, g, k)
  if (parity == 0) {
    if (sol)
      gen ? MK_DEND(0, true, true) : MK_DEND(0, true, false);
    else
      gen ? MK_DEND(0, false, true) : MK_DEND(0, false, false);
  } else {
    if (sol)
      gen ? MK_DEND(1, true, true) : MK_DEND(1, true, false);
    else
      gen ? MK_DEND(1, false, true) : MK_DEND(1, false, false);
  }
#undef MK_DEND
  if (ev) cudaEventRecord(ev[3], e.stream);
}

template <class T>
FdK<T> fd_coef(const mk_params& p, Refs r) {
  FdK<T> k;
  k.f = flow_coef<T>(p, p.rho0);
  k.half = T(p.tau - 0.5);
  for (int a = 0; a < 3; ++a) k.u0[a] = T(p.u0[a]);
  k.ref_g = T(r.r0);
  k.ref_t = T(r.r1);
  k.inlet = p.inlet ? 1 : 0;
  return k;
}

// Whether the inflow / outflow faces are applied in registers by the flow and
// phase-field kernels (warp shuffles between a face cell and its inner
// neighbour, which share a warp unless x = nx - 1 starts one) rather than by
// the separate boundary kernel.
bool fd_faces_in_warp(const mke::Engine& e) { return e.p.inlet && e.nx % 32 != 1; }

template <class S, int Q, int COLL>
void launch_fd_flow(mke::Engine& e, int parity, dim3 grid, dim3 block) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const FdK<T> k = fd_coef<T>(e.p, refs_of(e.p));
  const P* phi_old = (const P*)e.phi[e.phi_cur];
  const bool force = e.p.force[0] != 0.0 || e.p.force[1] != 0.0 || e.p.force[2] != 0.0;
  const bool nee = fd_faces_in_warp(e);
#define MK_FDF(PAR, FRC, NEE) \
  k_fd_flow<S, P, Q, COLL, PAR, FRC, NEE><<<grid, block, 0, e.stream>>>((S*)e.pop2, phi_old, (P*)e.vel, g, k)
#define MK_FDF2(PAR, FRC) nee ? MK_FDF(PAR, FRC, true) : MK_FDF(PAR, FRC, false)
  if (parity == 0)
    force ? MK_FDF2(0, true) : MK_FDF2(0, false);
  else
    force ? MK_FDF2(1, true) : MK_FDF2(1, false);
#undef MK_FDF2
#undef MK_FDF
}

// Flow + dendrite loop: phi of the streamed phase field, the flow lattice,
// the phase field with the advected thermal lattice, and the inflow/outflow
// faces (in the two collision kernels, or a separate kernel when a face cell
// and its inner neighbour can fall in different warps).
template <class S>
void launch_fd(mke::Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  S* G = (S*)e.pop0;
  P* phi_old = (P*)e.phi[e.phi_cur];
  P* phi_new = (P*)e.phi[1 - e.phi_cur];
  if (ev) cudaEventRecord(ev[0], e.stream);
  if (parity == 0)
    k_pf_phi<S, P, 0><<<grid, block, 0, e.stream>>>(G, phi_old, phi_new, g, T(r.r0));
  else
    k_pf_phi<S, P, 1><<<grid, block, 0, e.stream>>>(G, phi_old, phi_new, g, T(r.r0));
  if (ev) {
    cudaEventRecord(ev[1], e.stream);
    cudaEventRecord(ev[2], e.stream);
  }
  const int Q = e.p.lattice, C = e.p.collision;
  if (Q == 19) {
    if (C == MK_COLL_BGK)
      launch_fd_flow<S, 19, MK_COLL_BGK>(e, parity, grid, block);
    else if (C == MK_COLL_TRT)
      launch_fd_flow<S, 19, MK_COLL_TRT>(e, parity, grid, block);
    else
      launch_fd_flow<S, 19, MK_COLL_MRT>(e, parity, grid, block);
  } else {
    if (C == MK_COLL_BGK)
      launch_fd_flow<S, 27, MK_COLL_BGK>(e, parity, grid, block);
    else
      launch_fd_flow<S, 27, MK_COLL_TRT>(e, parity, grid, block);
  }
  if (ev) {
    cudaEventRecord(ev[3], e.stream);
    cudaEventRecord(ev[4], e.stream);
  }
  {
    const DendK<T> kd = dend_coef<T>(e.p, r);
    const bool gen = e.p.aniso != MK_ANISO_CUBIC;
    const P* vel = (const P*)e.vel;
    const bool nee = fd_faces_in_warp(e);
    const bool sol = mkm::solutal(e.p.model);
#define MK_FDD(PAR, GEN, NEE, SOL)                                                                                 \
  k_fd_dend<S, P, PAR, GEN, NEE, SOL><<<grid, block, 0, e.stream>>>(G, (S*)e.pop1, phi_new, phi_old, (P*)e.temp, \
                                                                    vel, e.grain, (const T*)e.rot, g, kd)
#define MK_FDD2(PAR, GEN, SOL) nee ? MK_FDD(PAR, GEN, true, SOL) : MK_FDD(PAR, GEN, false, SOL)
#define MK_FDD3(PAR, SOL) gen ? MK_FDD2(PAR, true, SOL) : MK_FDD2(PAR, false, SOL)
    if (parity == 0)
      sol ? MK_FDD3(0, true) : MK_FDD3(0, false);
    else
      sol ? MK_FDD3(1, true) : MK_FDD3(1, false);
#undef MK_FDD3
#undef MK_FDD2
#undef MK_FDD
  }
  if (ev) cudaEventRecord(ev[5], e.stream);
  if (e.p.inlet && !fd_faces_in_warp(e)) {
    if (ev) cudaEventRecord(ev[6], e.stream);
    const FdK<T> k = fd_coef<T>(e.p, r);
    const int nt = 2 * e.ny * e.nz;
    if (Q == 19)
      k_fd_nee<S, P, 19><<<(nt + 127) / 128, 128, 0, e.stream>>>((S*)e.pop2, G, (S*)e.pop1, (P*)e.temp, (const P*)e.vel, g,
                                                                 e.step + 1, k);
    else
      k_fd_nee<S, P, 27><<<(nt + 127) / 128, 128, 0, e.stream>>>((S*)e.pop2, G, (S*)e.pop1, (P*)e.temp, (const P*)e.vel, g,
                                                                 e.step + 1, k);
    if (ev) cudaEventRecord(ev[7], e.stream);
  }
}

// Grains per multigrain launch: block z = plane + nz * grain stays <= 65535.
inline int mg_grains_per_launch(const mke::Engine& e) { return std::max(1, 65535 / std::max(1, e.nz)); }

template <class T>
MgK<T> mg_coef(const mk_params& p, Refs r) {
  MgK<T> k;
  // omega_g = 1/(dt/dx^2/cs^2 + 1/2), cs^2 = 1/3 (mkFluidsUser.cpp:282; M = dt/dx^2)
  k.om = T(1.0 / (3.0 * p.mobility + 0.5));
  k.fo = T(1.0 - 0.5 / (3.0 * p.mobility + 0.5));
  k.ux = T(p.grain_u[0]);
  k.uy = T(p.grain_u[1]);
  k.uz = T(p.grain_u[2]);
  k.uu = T(p.grain_u[0] * p.grain_u[0] + p.grain_u[1] * p.grain_u[1] + p.grain_u[2] * p.grain_u[2]);
  k.inv_w = T(1.0 / (std::sqrt(2.0) * p.W0));
  k.kappa = T(p.grain_kappa);
  k.om_t = T(1.0 / (4.0 * p.D + 0.5));
  k.ref_t = T(r.r1);
  k.ngr = p.n_objects;
  return k;
}

template <class S>
void launch_mg(mke::Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  S* G = (S*)e.pop0;
  P* phij = (P*)e.phij;
  P* phi_old = (P*)e.phi[e.phi_cur];
  P* phi_new = (P*)e.phi[1 - e.phi_cur];
  // block z = plane + nz * grain, at most 65535: grains in chunks of ppl
  const int ngr = e.p.n_objects, ppl = mg_grains_per_launch(e);
  const MgK<T> k = mg_coef<T>(e.p, r);
  if (ev) cudaEventRecord(ev[0], e.stream);
  for (int j0 = 0; j0 < ngr; j0 += ppl) {
    const dim3 gz(grid.x, grid.y, (unsigned)(e.nz * std::min(ppl, ngr - j0)));
    bool paired = false;
    if constexpr (Stor<S>::bytes == 2) {
      if (e.nx % 2 == 0) {
        const dim3 g2((unsigned)((e.nx / 2 + (int)block.x - 1) / (int)block.x), gz.y, gz.z);
        if (parity == 0)
          k_mg_phi2<S, P, 0><<<g2, block, 0, e.stream>>>(G, phij, g, j0);
        else
          k_mg_phi2<S, P, 1><<<g2, block, 0, e.stream>>>(G, phij, g, j0);
        paired = true;
      }
    }
    if (paired) continue;
    if (parity == 0)
      k_mg_phi<S, P, 0><<<gz, block, 0, e.stream>>>(G, phij, g, j0);
    else
      k_mg_phi<S, P, 1><<<gz, block, 0, e.stream>>>(G, phij, g, j0);
  }
  if (ev) {
    cudaEventRecord(ev[1], e.stream);
    cudaEventRecord(ev[2], e.stream);
  }
  k_mg_sums<S, P><<<grid, block, 0, e.stream>>>(phij, phi_old, phi_new, g, ngr);
  if (ev) {
    cudaEventRecord(ev[3], e.stream);
    cudaEventRecord(ev[4], e.stream);
  }
  for (int j0 = 0; j0 < ngr; j0 += ppl) {
    const dim3 gz(grid.x, grid.y, (unsigned)(e.nz * std::min(ppl, ngr - j0)));
    if (parity == 0)
      k_mg_collide<S, P, 0><<<gz, block, 0, e.stream>>>(G, (S*)e.pop1, phij, phi_new, phi_old, (P*)e.temp, g, k, j0);
    else
      k_mg_collide<S, P, 1><<<gz, block, 0, e.stream>>>(G, (S*)e.pop1, phij, phi_new, phi_old, (P*)e.temp, g, k, j0);
  }
  if (ev) cudaEventRecord(ev[5], e.stream);
}

template <class S>
void step_t(mke::Engine& e, cudaEvent_t* ev) {
  dim3 grid, block;
  launch_dims(e, grid, block);
  const int parity = (int)(e.step & 1);
  switch (e.p.model) {
    case MK_MODEL_FLOW:
      if (ev) cudaEventRecord(ev[0], e.stream);
      if (e.p.wall_axis >= 0)
        launch_conv<S, false>(e, parity, grid, block);  // moving plates
      else
        launch_flow<S>(e, parity, grid, block);
      if (ev) cudaEventRecord(ev[1], e.stream);
      e.launches += 1;
      break;
    case MK_MODEL_CONVECTION:
      if (ev) cudaEventRecord(ev[0], e.stream);
      launch_conv<S, true>(e, parity, grid, block);
      if (ev) cudaEventRecord(ev[1], e.stream);
      e.launches += 1;
      break;
    case MK_MODEL_MULTIPHASE:
      if (e.mpending_set && !e.capturing) mke::mp_apply_solids(e);
      mke::mp_launch(e, parity, grid, block, ev);
      e.launches += engine_kernels_per_step(e);
      break;
    case MK_MODEL_MULTIGRAIN:
      launch_mg<S>(e, parity, grid, block, ev);
      e.phi_cur = 1 - e.phi_cur;
      e.launches += engine_launches_per_step(e);
      break;
    case MK_MODEL_FLOW_DENDRITE:
    case MK_MODEL_FLOW_SOLUTAL:
      launch_fd<S>(e, parity, grid, block, ev);
      e.phi_cur = 1 - e.phi_cur;
      e.launches += (e.p.inlet && !fd_faces_in_warp(e)) ? 4 : 3;
      break;
    default:
      launch_dend<S>(e, parity, grid, block, ev);
      e.phi_cur = 1 - e.phi_cur;
      e.launches += 2;
      break;
  }
  e.step += 1;
}

template <class S, class InT>
cudaError_t set_state_t(mke::Engine& e, const InT* d_phi, const InT* d_t, const InT* d_rho, const InT* d_u) {
  typedef typename PhiOf<S>::type P;
  dim3 grid, block;
  launch_dims(e, grid, block);
  const Geom g = make_geom(e);
  if (e.p.model == MK_MODEL_MULTIGRAIN) {
    // the grains' order parameters start from their seeds (phi is their aggregate)
    k_mg_init<S, InT><<<grid, block, 0, e.stream>>>((S*)e.pop0, (S*)e.pop1, (P*)e.phij, (P*)e.phi[0], (P*)e.phi[1],
                                                    (P*)e.temp, d_t, -e.p.delta, e.gseeds, e.p.n_objects, e.p.W0, g,
                                                    e.ncell, refs_of(e.p));
    return cudaGetLastError();
  }
  k_init<S, InT><<<grid, block, 0, e.stream>>>(e.p.model, e.Q0, (S*)e.pop0, (S*)e.pop1, (S*)e.pop2, e.Q2, e.rest1,
                                               (P*)e.phi[0],
                                               (P*)e.phi[1],
                                          (P*)e.temp, d_phi, d_t, d_rho, d_u, e.p.rho0, e.p.u0[0], e.p.u0[1],
                                          e.p.u0[2], e.p.model == MK_MODEL_CONVECTION ? e.p.s_ref : -e.p.delta, g,
                                          e.ncell, refs_of(e.p));
  return cudaGetLastError();
}

template <class S>
cudaError_t field_t(mke::Engine& e, int field) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  dim3 grid, block;
  launch_dims(e, grid, block);
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  const int m = e.p.model;
  const int nb = (int)((e.ncell + 255) / 256);
  if (field == MK_FIELD_GRAIN && m == MK_MODEL_MULTIGRAIN) {
    k_field_mg_grain<P><<<nb, 256, 0, e.stream>>>((const P*)e.phij, e.p.n_objects, e.ncell, e.field);
    return cudaGetLastError();
  }
  if (field == MK_FIELD_FLAG && mkm::flow_coupled(m)) {
    k_field_fdflag<P><<<grid, block, 0, e.stream>>>(g, (const P*)e.phi[e.phi_cur], e.field);
    return cudaGetLastError();
  }
  if (field == MK_FIELD_FLAG || field == MK_FIELD_GRAIN) {
    const int nobj = mkm::dendrite(m) ? e.p.n_objects : 0;
    k_field_geom<<<grid, block, 0, e.stream>>>(g, field, e.seeds, nobj, e.field);
    return cudaGetLastError();
  }
  if (field == MK_FIELD_PHI) {
    k_field_copy<P><<<nb, 256, 0, e.stream>>>((const P*)e.phi[e.phi_cur], nullptr, e.ncell, e.field);
    return cudaGetLastError();
  }
  if (m == MK_MODEL_FLOW || m == MK_MODEL_CONVECTION) {
    const bool conv = m == MK_MODEL_CONVECTION;
    if (field != MK_FIELD_RHO && field != MK_FIELD_UX && field != MK_FIELD_UY && field != MK_FIELD_UZ &&
        !(conv && field == MK_FIELD_T))
      return cudaErrorInvalidValue;
    const S* Tp = conv ? (const S*)e.pop1 : nullptr;
    const Buoy bu = buoy_of(e.p);
    if (e.p.lattice == 19)
      k_field_flow<S, 19><<<grid, block, 0, e.stream>>>((const S*)e.pop0, Tp, bu, g, e.step, field, e.p.force[0],
                                                        e.p.force[1], e.p.force[2], e.p.rho0, e.field);
    else
      k_field_flow<S, 27><<<grid, block, 0, e.stream>>>((const S*)e.pop0, Tp, bu, g, e.step, field, e.p.force[0],
                                                        e.p.force[1], e.p.force[2], e.p.rho0, e.field);
    return cudaGetLastError();
  }
  if (mkm::flow_coupled(m) &&
      (field == MK_FIELD_RHO || field == MK_FIELD_UX || field == MK_FIELD_UY || field == MK_FIELD_UZ)) {
    const Buoy bu = buoy_of(e.p);
    if (e.Q2 == 19)
      k_field_flow<S, 19><<<grid, block, 0, e.stream>>>((const S*)e.pop2, nullptr, bu, g, e.step, field, e.p.force[0],
                                                        e.p.force[1], e.p.force[2], e.p.rho0, e.field);
    else
      k_field_flow<S, 27><<<grid, block, 0, e.stream>>>((const S*)e.pop2, nullptr, bu, g, e.step, field, e.p.force[0],
                                                        e.p.force[1], e.p.force[2], e.p.rho0, e.field);
    return cudaGetLastError();
  }
  if (m == MK_MODEL_MULTIPHASE) {
    if (field != MK_FIELD_RHO && field != MK_FIELD_UX && field != MK_FIELD_UY && field != MK_FIELD_UZ &&
        field != MK_FIELD_PRESSURE)
      return cudaErrorInvalidValue;
    k_field_mp<S><<<grid, block, 0, e.stream>>>((const S*)e.pop0, (const P*)e.phi[0], g, e.step, field,
                                                mp_coef<T>(e.p, r), e.field);
    return cudaGetLastError();
  }
  if (field == MK_FIELD_T || field == MK_FIELD_C) {
    if ((field == MK_FIELD_T) != (m == MK_MODEL_THERMAL_DENDRITE || m == MK_MODEL_FLOW_DENDRITE ||
                                  m == MK_MODEL_MULTIGRAIN))
      return cudaErrorInvalidValue;
    k_field_copy<P><<<nb, 256, 0, e.stream>>>((const P*)e.temp, nullptr, e.ncell, e.field);
    return cudaGetLastError();
  }
  if (field == MK_FIELD_DPHI) {
    k_field_copy<P><<<nb, 256, 0, e.stream>>>((const P*)e.phi[e.phi_cur], (const P*)e.phi[1 - e.phi_cur], e.ncell,
                                              e.field);
    return cudaGetLastError();
  }
  return cudaErrorInvalidValue;
}

template <class S>
cudaError_t diag_t(mke::Engine& e) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  const int nb = e.partial_blocks;
  const int m = e.p.model;
  if (m == MK_MODEL_FLOW || m == MK_MODEL_CONVECTION) {
    const S* Tp = m == MK_MODEL_CONVECTION ? (const S*)e.pop1 : nullptr;
    const Buoy bu = buoy_of(e.p);
    const int ax = e.p.wall_axis >= 0 ? e.p.wall_axis : 0;
    if (e.p.lattice == 19)
      k_diag_flow<S, 19><<<nb, 256, 0, e.stream>>>((const S*)e.pop0, Tp, bu, ax, g, e.step, e.p.force[0],
                                                   e.p.force[1], e.p.force[2], e.p.rho0, e.ncell, e.partial);
    else
      k_diag_flow<S, 27><<<nb, 256, 0, e.stream>>>((const S*)e.pop0, Tp, bu, ax, g, e.step, e.p.force[0],
                                                   e.p.force[1], e.p.force[2], e.p.rho0, e.ncell, e.partial);
  } else if (mkm::flow_coupled(m)) {
    const P* ph = (const P*)e.phi[e.phi_cur];
    const P* pp = (const P*)e.phi[1 - e.phi_cur];
    if (e.Q2 == 19)
      k_diag_fd<S, P, 19><<<nb, 256, 0, e.stream>>>((const S*)e.pop2, ph, pp, (const P*)e.temp, g, e.step,
                                                    e.p.force[0], e.p.force[1], e.p.force[2], e.p.rho0,
                                                    mkm::solutal(m) ? 1 : 0, e.ncell, e.partial);
    else
      k_diag_fd<S, P, 27><<<nb, 256, 0, e.stream>>>((const S*)e.pop2, ph, pp, (const P*)e.temp, g, e.step,
                                                    e.p.force[0], e.p.force[1], e.p.force[2], e.p.rho0,
                                                    mkm::solutal(m) ? 1 : 0, e.ncell, e.partial);
  } else if (m == MK_MODEL_MULTIPHASE) {
    k_diag_mp<S><<<nb, 256, 0, e.stream>>>((const S*)e.pop0, (const P*)e.phi[0], g, e.step, mp_coef<T>(e.p, r),
                                           e.ncell, e.partial);
  } else {
    k_diag_dend<P><<<nb, 256, 0, e.stream>>>((const P*)e.phi[e.phi_cur], (const P*)e.phi[1 - e.phi_cur],
                                             (const P*)e.temp, g, mkm::solutal(m) ? 1 : 0, e.ncell,
                                             e.partial);
  }
  k_diag_final<<<1, 256, 0, e.stream>>>(e.partial, nb, e.dsum);
  return cudaGetLastError();
}

}  // namespace

namespace mke {

// Grain table: centre + rotation per object (R = Rz Ry Rx of the ZYX angles in
// degrees, as in the oracle); one identity entry when there are none.
void seed_table(const mk_params& p, std::vector<double>& sd) {
  const int nobj = p.n_objects > 0 ? p.n_objects : 1;
  sd.assign((size_t)12 * nobj, 0.0);
  for (int k = 0; k < nobj; ++k) {
    double* s = &sd[12 * k];
    if (k < p.n_objects) {
      s[0] = p.obj_center[k][0];
      s[1] = p.obj_center[k][1];
      s[2] = p.obj_center[k][2];
    }
    const double d2r = M_PI / 180.0;
    const double ax = (k < p.n_objects ? p.obj_angle[k][0] : 0) * d2r, ay = (k < p.n_objects ? p.obj_angle[k][1] : 0) * d2r,
                 az = (k < p.n_objects ? p.obj_angle[k][2] : 0) * d2r;
    const double cx = std::cos(ax), sx = std::sin(ax), cy = std::cos(ay), sy = std::sin(ay), cz = std::cos(az),
                 sz = std::sin(az);
    double* R = s + 3;
    R[0] = cz * cy;
    R[1] = cz * sy * sx - sz * cx;
    R[2] = cz * sy * cx + sz * sx;
    R[3] = sz * cy;
    R[4] = sz * sy * sx + cz * cx;
    R[5] = sz * sy * cx - cz * sx;
    R[6] = -sy;
    R[7] = cy * sx;
    R[8] = cy * cx;
  }
}

cudaError_t engine_alloc(Engine& e, const mk_params& p, int device, int block_x, int block_y, std::string& err) {
  std::memset(&e, 0, sizeof(e));
  e.p = p;
  e.nx = p.nx;
  e.ny = p.ny;
  e.nz = p.nz;
  e.ncell = (int64_t)p.nx * p.ny * p.nz;
  e.stride = pop_stride(e.ncell);
  e.elem = pop_elem(p.precision);
  e.phi_elem = phi_elem_of(p.precision);
  e.device = device;
  if (p.model == MK_MODEL_FLOW || p.model == MK_MODEL_CONVECTION) {
    e.Q0 = p.lattice;
    e.Q1 = p.model == MK_MODEL_CONVECTION ? 7 : 0;
  } else if (p.model == MK_MODEL_MULTIPHASE) {
    e.Q0 = 19;
    e.Q1 = 19;
  } else {
    e.Q0 = 7;
    e.Q1 = 7;
  }
  if (p.model == MK_MODEL_MULTIGRAIN) e.Q0 = 19 * p.n_objects;  // one D3Q19 lattice per grain
  e.Q2 = mkm::flow_coupled(p.model) ? p.lattice : 0;
  // Launch shape: a full warp row along x, rows stacked in y to 256 threads.
  int bx = block_x > 0 ? block_x : (p.nx >= 128 ? 128 : (p.nx >= 64 ? 64 : 32));
  int by = block_y > 0 ? block_y : 256 / bx;
  if (bx * by > 1024 || bx < 1 || by < 1) {
    err = "invalid block shape";
    return cudaErrorInvalidValue;
  }
  e.block_x = bx;
  e.block_y = by;
  e.minb = 2;
  cudaError_t st = cudaSetDevice(device);
  if (st != cudaSuccess) return st;
  st = cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking);
  if (st != cudaSuccess) return st;
  auto alloc = [&](void** ptr, size_t bytes) -> cudaError_t {
    if (bytes == 0) {
      *ptr = nullptr;
      return cudaSuccess;
    }
    cudaError_t s = cudaMalloc(ptr, bytes);
    if (s != cudaSuccess) return s;
    return cudaMemsetAsync(*ptr, 0, bytes, e.stream);
  };
  if ((st = alloc(&e.pop0, (size_t)e.Q0 * e.stride * e.elem)) != cudaSuccess) return st;
  if ((st = alloc(&e.pop1, (size_t)e.Q1 * e.stride * e.elem)) != cudaSuccess) return st;
  if ((st = alloc(&e.pop2, (size_t)e.Q2 * e.stride * e.elem)) != cudaSuccess) return st;
  const bool fd = mkm::flow_coupled(p.model);
  if ((st = alloc(&e.vel, fd ? (size_t)3 * e.ncell * e.phi_elem : 0)) != cudaSuccess) return st;
  if (p.model == MK_MODEL_MULTIPHASE && e.elem == 2) {
    if ((st = alloc((void**)&e.rest1, (size_t)e.ncell * sizeof(float))) != cudaSuccess) return st;
  } else {
    e.rest1 = nullptr;
  }
  if ((st = alloc(&e.phi[0], (size_t)e.ncell * e.phi_elem)) != cudaSuccess) return st;
  const bool dend = mkm::dendrite(p.model) || p.model == MK_MODEL_MULTIGRAIN;
  const bool mg = p.model == MK_MODEL_MULTIGRAIN;
  // N order parameters and the per-cell sum of p_k^2 (plane N)
  if ((st = alloc(&e.phij, mg ? (size_t)(p.n_objects + 1) * e.ncell * e.phi_elem : 0)) != cudaSuccess) return st;
  if (mg) {
    std::vector<double> gs((size_t)4 * p.n_objects);
    for (int k = 0; k < p.n_objects; ++k) {
      for (int a = 0; a < 3; ++a) gs[4 * k + a] = p.obj_center[k][a];
      gs[4 * k + 3] = p.obj_radius[k];
    }
    if ((st = cudaMalloc((void**)&e.gseeds, gs.size() * sizeof(double))) != cudaSuccess) return st;
    if ((st = cudaMemcpy(e.gseeds, gs.data(), gs.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
      return st;
  }
  if ((st = alloc(&e.phi[1], dend ? (size_t)e.ncell * e.phi_elem : 0)) != cudaSuccess) return st;
  if (!dend) e.phi[1] = nullptr;
  if ((st = alloc(&e.temp, dend ? (size_t)e.ncell * e.phi_elem : 0)) != cudaSuccess) return st;
  std::vector<double> sd;
  seed_table(p, sd);
  if ((st = cudaMalloc((void**)&e.seeds, sd.size() * sizeof(double))) != cudaSuccess) return st;
  if ((st = cudaMemcpyAsync(e.seeds, sd.data(), sd.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream)) !=
      cudaSuccess)
    return st;
  // rotations in the arithmetic type (9 per grain) and the per-cell grain map
  const int nrot = (int)(sd.size() / 12);
  std::vector<double> rd((size_t)9 * nrot);
  std::vector<float> rf((size_t)9 * nrot);
  for (int k = 0; k < nrot; ++k)
    for (int q = 0; q < 9; ++q) {
      rd[9 * k + q] = sd[12 * k + 3 + q];
      rf[9 * k + q] = (float)sd[12 * k + 3 + q];
    }
  const bool rot64 = p.precision == MK_PREC_FP64;
  const size_t rbytes = rot64 ? rd.size() * sizeof(double) : rf.size() * sizeof(float);
  if ((st = cudaMalloc(&e.rot, rbytes)) != cudaSuccess) return st;
  if ((st = cudaMemcpyAsync(e.rot, rot64 ? (const void*)rd.data() : (const void*)rf.data(), rbytes,
                            cudaMemcpyHostToDevice, e.stream)) != cudaSuccess)
    return st;
  if (dend && p.n_objects > 1) {
    if ((st = cudaMalloc((void**)&e.grain, (size_t)e.ncell)) != cudaSuccess) return st;
    Geom g;
    g.nx = p.nx;
    g.ny = p.ny;
    g.nz = p.nz;
    g.bc0 = p.bc[0];
    g.bc1 = p.bc[1];
    g.bc2 = p.bc[2];
    g.stride = e.stride;
    k_grain_map<<<(int)std::min<int64_t>((e.ncell + 255) / 256, 4096), 256, 0, e.stream>>>(g, e.seeds, p.n_objects, 0,
                                                                                         e.grain);
    if ((st = cudaGetLastError()) != cudaSuccess) return st;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  e.partial_blocks = sms * 8;
  if ((st = cudaMalloc((void**)&e.partial, (size_t)e.partial_blocks * DG_N * sizeof(double))) != cudaSuccess)
    return st;
  if ((st = cudaMalloc((void**)&e.dsum, DG_N * sizeof(double))) != cudaSuccess) return st;
  if ((st = cudaMalloc((void**)&e.field, (size_t)e.ncell * sizeof(double))) != cudaSuccess) return st;
  e.wave_skip = -1;
  if (p.model == MK_MODEL_MULTIPHASE) {
    mp_configure(e);
    if (e.wave_ok) {
      if ((st = alloc((void**)&e.wave_flags, (size_t)e.wave_sx * e.wave_sy * sizeof(unsigned))) != cudaSuccess) return st;
      e.wave = 0;  // the two-kernel loop until mk_set_fused or the autotuner chooses the fused one
    }
    // the error word of the bounded waits (fused loop, row-staged collision,
    // TMA phi tile)
    if (e.wave_ok || e.rows_ok || e.tma_ok)
      if ((st = alloc((void**)&e.wave_err, sizeof(int))) != cudaSuccess) return st;
    e.rows = 0;
  }
  // host-side copy of sd must outlive the async copy
  st = cudaStreamSynchronize(e.stream);
  return st;
}

void engine_free(Engine& e) {
  if (e.stream) cudaStreamSynchronize(e.stream);
  void* ptrs[] = {e.pop0, e.pop1, e.pop2, e.vel, e.phij, e.gseeds, e.rest1, e.phi[0], e.phi[1], e.temp, e.seeds, e.rot, e.grain, e.partial, e.dsum, e.field,
                  e.field32, e.stage32, e.wave_flags, e.wave_err, e.slab_halo, e.msolid, e.mnear, e.mpending};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (e.stream) cudaStreamDestroy(e.stream);
  std::memset(&e, 0, sizeof(e));
}

cudaError_t engine_set_state(Engine& e, const double* phi, const double* temp, const double* rho, const double* ux,
                             const double* uy, const double* uz) {
  // Stage host fields in one device buffer: phi | T | rho | ux uy uz.
  const size_t n = (size_t)e.ncell;
  double* d = nullptr;
  cudaError_t st = cudaMalloc((void**)&d, 6 * n * sizeof(double));
  if (st != cudaSuccess) return st;
  const double* src[6] = {phi, temp, rho, ux, uy, uz};
  for (int q = 0; q < 6; ++q)
    if (src[q] && (st = cudaMemcpyAsync(d + q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice, e.stream)) !=
                      cudaSuccess) {
      cudaFree(d);
      return st;
    }
  const bool has_u = ux && uy && uz;
  const double* dphi = phi ? d : nullptr;
  const double* dt = temp ? d + n : nullptr;
  const double* drho = rho ? d + 2 * n : nullptr;
  const double* du = has_u ? d + 3 * n : nullptr;
  e.step = 0;
  e.phi_cur = 0;
  switch (e.p.precision) {
    case MK_PREC_FP64:
      st = set_state_t<double, double>(e, dphi, dt, drho, du);
      break;
    case MK_PREC_FP32:
      st = set_state_t<float, double>(e, dphi, dt, drho, du);
      break;
    case MK_PREC_FP16:
      st = set_state_t<__half, double>(e, dphi, dt, drho, du);
      break;
    default:
      st = set_state_t<__nv_bfloat16, double>(e, dphi, dt, drho, du);
      break;
  }
  cudaError_t s2 = cudaStreamSynchronize(e.stream);
  cudaFree(d);
  return st != cudaSuccess ? st : s2;
}

cudaError_t engine_set_state_f32(Engine& e, const float* phi, const float* temp) {
  // Host arrays go straight into a persistent FP32 staging buffer (a pinned
  // source makes these plain DMA copies), then one init kernel.
  const size_t n = (size_t)e.ncell;
  cudaError_t st;
  if (!e.stage32 && (st = cudaMalloc((void**)&e.stage32, 2 * n * sizeof(float))) != cudaSuccess) return st;
  if (phi && (st = cudaMemcpyAsync(e.stage32, phi, n * sizeof(float), cudaMemcpyHostToDevice, e.stream)) !=
                 cudaSuccess)
    return st;
  if (temp && (st = cudaMemcpyAsync(e.stage32 + n, temp, n * sizeof(float), cudaMemcpyHostToDevice, e.stream)) !=
                  cudaSuccess)
    return st;
  const float* dphi = phi ? e.stage32 : nullptr;
  const float* dt = temp ? e.stage32 + n : nullptr;
  e.step = 0;
  e.phi_cur = 0;
  switch (e.p.precision) {
    case MK_PREC_FP64:
      return set_state_t<double, float>(e, dphi, dt, nullptr, nullptr);
    case MK_PREC_FP32:
      return set_state_t<float, float>(e, dphi, dt, nullptr, nullptr);
    case MK_PREC_FP16:
      return set_state_t<__half, float>(e, dphi, dt, nullptr, nullptr);
    default:
      return set_state_t<__nv_bfloat16, float>(e, dphi, dt, nullptr, nullptr);
  }
}

cudaError_t engine_field_f32(Engine& e, int field) {
  cudaError_t st = engine_field(e, field);
  if (st != cudaSuccess) return st;
  if (!e.field32 && (st = cudaMalloc((void**)&e.field32, (size_t)e.ncell * sizeof(float))) != cudaSuccess) return st;
  const int nb = (int)((e.ncell + 255) / 256);
  k_to_f32<<<nb, 256, 0, e.stream>>>(e.field, e.ncell, e.field32);
  return cudaGetLastError();
}

cudaError_t engine_step(Engine& e, cudaEvent_t* ev) {
  switch (e.p.precision) {
    case MK_PREC_FP64:
      step_t<double>(e, ev);
      break;
    case MK_PREC_FP32:
      step_t<float>(e, ev);
      break;
    case MK_PREC_FP16:
      step_t<__half>(e, ev);
      break;
    default:
      step_t<__nv_bfloat16>(e, ev);
      break;
  }
  return cudaGetLastError();
}

static bool one_kernel(const Engine& e) { return e.p.model == MK_MODEL_FLOW || e.p.model == MK_MODEL_CONVECTION; }

static bool fused_mp(const Engine& e) { return e.p.model == MK_MODEL_MULTIPHASE && e.wave && e.wave_ok; }

int engine_kernels_per_step(const Engine& e) {
  if (mkm::flow_coupled(e.p.model)) return (e.p.inlet && !fd_faces_in_warp(e)) ? 4 : 3;
  if (e.p.model == MK_MODEL_MULTIGRAIN) return 3;
  return (one_kernel(e) || fused_mp(e)) ? 1 : 2;
}

int engine_launches_per_step(const Engine& e) {
  if (e.p.model == MK_MODEL_MULTIGRAIN) {
    const int ppl = mg_grains_per_launch(e);
    return 2 * ((e.p.n_objects + ppl - 1) / ppl) + 1;
  }
  return engine_kernels_per_step(e);
}

const char* engine_kernel_name(const Engine& e, int k) {
  if (one_kernel(e) || fused_mp(e)) return "collide";
  if (mkm::flow_coupled(e.p.model)) {
    static const char* const names[4] = {"phi", "flow", "collide", "boundary"};
    return k >= 0 && k < 4 ? names[k] : "";
  }
  if (e.p.model == MK_MODEL_MULTIGRAIN) {
    static const char* const names[3] = {"phi", "sums", "collide"};
    return k >= 0 && k < 3 ? names[k] : "";
  }
  return k == 0 ? "phi" : "collide";
}

cudaError_t engine_set_velocity(Engine& d, Engine& f) {
  const int dm = d.p.model;
  if (!(dm == MK_MODEL_THERMAL_DENDRITE || dm == MK_MODEL_SOLUTAL_DENDRITE) || f.p.model != MK_MODEL_MULTIPHASE ||
      d.nx != f.nx || d.ny != f.ny || d.nz != f.nz || d.device != f.device || d.slab || f.slab)
    return cudaErrorInvalidValue;
  const int64_t n = d.ncell;
  cudaError_t st = cudaSuccess;
  if (!d.vel) {
    if ((st = cudaMalloc(&d.vel, (size_t)3 * n * d.phi_elem)) != cudaSuccess) return st;
    if ((st = cudaMemsetAsync(d.vel, 0, (size_t)3 * n * d.phi_elem, d.stream)) != cudaSuccess) return st;
  }
  const int blocks = (int)((n + 255) / 256);
  for (int a = 0; a < 3; ++a) {
    if ((st = engine_field(f, MK_FIELD_UX + a)) != cudaSuccess) return st;
    if ((st = cudaStreamSynchronize(f.stream)) != cudaSuccess) return st;
    if (d.phi_elem == 8)
      k_double_to_plane<double><<<blocks, 256, 0, d.stream>>>(f.field, (double*)d.vel + a * n, n);
    else
      k_double_to_plane<float><<<blocks, 256, 0, d.stream>>>(f.field, (float*)d.vel + a * n, n);
    if ((st = cudaGetLastError()) != cudaSuccess) return st;
    if ((st = cudaStreamSynchronize(d.stream)) != cudaSuccess) return st;  // f.field is reused
  }
  return cudaSuccess;
}

cudaError_t engine_field(Engine& e, int field) {
  switch (e.p.precision) {
    case MK_PREC_FP64:
      return field_t<double>(e, field);
    case MK_PREC_FP32:
      return field_t<float>(e, field);
    case MK_PREC_FP16:
      return field_t<__half>(e, field);
    default:
      return field_t<__nv_bfloat16>(e, field);
  }
}

cudaError_t engine_grain_field(Engine& e, int grain) {
  if (e.p.model != MK_MODEL_MULTIGRAIN || grain < 0 || grain >= e.p.n_objects) return cudaErrorInvalidValue;
  const int nb = (int)((e.ncell + 255) / 256);
  if (e.phi_elem == 8)
    k_field_copy<double><<<nb, 256, 0, e.stream>>>((const double*)e.phij + (int64_t)grain * e.ncell, nullptr, e.ncell,
                                                   e.field);
  else
    k_field_copy<float><<<nb, 256, 0, e.stream>>>((const float*)e.phij + (int64_t)grain * e.ncell, nullptr, e.ncell,
                                                  e.field);
  return cudaGetLastError();
}

cudaError_t engine_check_waits(Engine& e, bool* timed_out) {
  *timed_out = false;
  if (!e.wave_err) return cudaSuccess;
  int v = 0;
  cudaError_t st = cudaMemcpyAsync(&v, e.wave_err, sizeof(int), cudaMemcpyDeviceToHost, e.stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
  if (st != cudaSuccess) return st;
  if (v != 0) {
    *timed_out = true;
    st = cudaMemsetAsync(e.wave_err, 0, sizeof(int), e.stream);
    if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
  }
  return st;
}

cudaError_t engine_diag(Engine& e, double* out) {
  cudaError_t st;
  switch (e.p.precision) {
    case MK_PREC_FP64:
      st = diag_t<double>(e);
      break;
    case MK_PREC_FP32:
      st = diag_t<float>(e);
      break;
    case MK_PREC_FP16:
      st = diag_t<__half>(e);
      break;
    default:
      st = diag_t<__nv_bfloat16>(e);
      break;
  }
  if (st != cudaSuccess) return st;
  st = cudaMemcpyAsync(out, e.dsum, DG_N * sizeof(double), cudaMemcpyDeviceToHost, e.stream);
  if (st != cudaSuccess) return st;
  return cudaStreamSynchronize(e.stream);
}

cudaError_t engine_autotune(Engine& e, int trial_steps, TuneResult* out) {
  if (trial_steps < 1) trial_steps = 1;
  const size_t b0 = engine_pop_bytes(e, 0), b1 = engine_pop_bytes(e, 1), b2 = engine_pop_bytes(e, 2),
               bp = (size_t)e.ncell * e.phi_elem;
  void* const bufs[8] = {e.pop0, e.pop1, e.phi[0], e.phi[1], e.temp, e.rest1, e.pop2, e.phij};
  const size_t sizes[8] = {b0, b1, bp, e.phi[1] ? bp : 0, e.temp ? bp : 0,
                           e.rest1 ? (size_t)e.ncell * sizeof(float) : 0, b2,
                           e.phij ? (size_t)e.p.n_objects * bp : 0};
  size_t total = 0;
  for (size_t s : sizes) total += s;
  char* save = nullptr;
  cudaError_t st = cudaMalloc((void**)&save, total);
  if (st != cudaSuccess) return st;
  auto copy = [&](bool to_save) -> cudaError_t {
    size_t off = 0;
    for (int q = 0; q < 8; ++q) {
      if (!sizes[q]) continue;
      cudaError_t s2 = to_save ? cudaMemcpyAsync(save + off, bufs[q], sizes[q], cudaMemcpyDeviceToDevice, e.stream)
                               : cudaMemcpyAsync(bufs[q], save + off, sizes[q], cudaMemcpyDeviceToDevice, e.stream);
      if (s2 != cudaSuccess) return s2;
      off += sizes[q];
    }
    return cudaSuccess;
  };
  const int64_t step0 = e.step, l0 = e.launches;
  const int cur0 = e.phi_cur, bx0 = e.block_x, by0 = e.block_y, mb0 = e.minb;
  // pending dynamic solids are not applied by the trial loops
  const int pend0 = e.mpending_set;
  e.capturing = 1;
  if ((st = copy(true)) != cudaSuccess) {
    e.capturing = 0;
    cudaFree(save);
    return st;
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  // 64-, 128- and 256-thread blocks, a warp-multiple row along x
  const int shapes[9][2] = {{32, 2}, {64, 1}, {32, 4}, {64, 2}, {128, 1}, {32, 8}, {64, 4}, {128, 2}, {256, 1}};
  // occupancy variants: 1, 2 (256-thread launch bounds), and for the
  // multiphase collision 3, 4, 5 (registers capped at 112, 96, 80)
  const int nmb = e.p.model == MK_MODEL_MULTIPHASE ? 5 : 1;
  double best = 1e300;
  int bbx = bx0, bby = by0, bmb = mb0, ncand = 0, bwave = 0, brows = 0, btma = 0;
  // time the configuration now in e (warm-up of both AA parities, then the
  // faster of two timed repeats: one slow repeat must not decide), restore
  // the state and keep the configuration if it is the fastest so far
  auto trial = [&]() {
    engine_step(e, nullptr);
    engine_step(e, nullptr);
    float ms = 1e30f;
    for (int rep = 0; rep < 2 && st == cudaSuccess; ++rep) {
      cudaEventRecord(t0, e.stream);
      for (int s = 0; s < trial_steps; ++s) engine_step(e, nullptr);
      cudaEventRecord(t1, e.stream);
      st = cudaEventSynchronize(t1);
      if (st == cudaSuccess) st = cudaGetLastError();
      float m = 0;
      if (st == cudaSuccess) cudaEventElapsedTime(&m, t0, t1);
      ms = std::min(ms, m);
    }
    ++ncand;
    if (st == cudaSuccess && ms / trial_steps < best) {
      best = ms / trial_steps;
      bbx = e.block_x;
      bby = e.block_y;
      bmb = e.minb;
      bwave = e.wave;
      brows = e.rows;
      btma = e.tma;
    }
    e.step = step0;
    e.phi_cur = cur0;
    e.launches = l0;
    if (st == cudaSuccess) st = copy(false);
  };
  // candidate -1: the fused multiphase loop (its tiling is fixed by the case);
  // candidate -2: the row-staged collision, -3: the TMA phi tile (the block
  // shape given is the phi kernel's)
  for (int si = -3; si < 9 && st == cudaSuccess; ++si) {
    if ((si == -1 && !e.wave_ok) || (si == -2 && !e.rows_ok) || (si == -3 && !e.tma_ok)) continue;
    const int bx = si < 0 ? bx0 : shapes[si][0];
    if (si >= 0 && bx > 32 && bx / 2 >= e.nx) continue;  // no wider than the row
    for (int mb = 1; mb <= (si < 0 ? 1 : nmb) && st == cudaSuccess; ++mb) {
      e.wave = si == -1 ? 1 : 0;
      e.rows = si == -2 ? 1 : 0;
      e.tma = si == -3 ? 1 : 0;
      e.block_x = bx;
      e.block_y = si < 0 ? by0 : shapes[si][1];
      e.minb = (nmb > 1 && si >= 0) ? mb : mb0;
      trial();
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e.capturing = 0;
  e.mpending_set = pend0;
  cudaError_t s3 = cudaStreamSynchronize(e.stream);
  cudaFree(save);
  if (st != cudaSuccess) return st;
  if (s3 != cudaSuccess) return s3;
  e.block_x = bbx;
  e.block_y = bby;
  e.minb = bmb;
  e.wave = bwave;
  e.rows = brows;
  e.tma = btma;
  if (out) {
    // a fused multiphase loop has no block shape or occupancy variant: 0, 0, 0;
    // the row-staged collision has no occupancy variant: minb 0
    out->block_x = bwave ? 0 : bbx;
    out->block_y = bwave ? 0 : bby;
    out->minb = (bwave || brows || btma) ? 0 : bmb;
    out->ms_per_step = best;
    out->candidates = ncand;
  }
  return cudaSuccess;
}

size_t engine_pop_bytes(const Engine& e, int which) {
  return (size_t)(which == 0 ? e.Q0 : (which == 1 ? e.Q1 : e.Q2)) * e.stride * e.elem;
}

double engine_bytes_per_cell(const Engine& e) {
  // Compulsory traffic: every population read once and written once; phi
  // written once and read once where a model has it.
  // An FP32 rest plane (16-bit multiphase storage) moves 4 B instead of 2 B.
  const double S = e.elem;
  const double phi = (e.p.model == MK_MODEL_FLOW || e.p.model == MK_MODEL_CONVECTION) ? 0.0 : 2.0 * e.phi_elem;
  const double rest = e.rest1 ? 2.0 * (4.0 - S) : 0.0;
  const double grains = e.phij ? 2.0 * e.p.n_objects * e.phi_elem : 0.0;  // phi_j written, then read
  return 2.0 * (e.Q0 + e.Q1 + e.Q2) * S + phi + rest + grains;
}

}  // namespace mke
