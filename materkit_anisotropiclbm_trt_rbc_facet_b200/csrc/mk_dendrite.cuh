// mk_dendrite.cuh — phase-field + thermal / solutal cell update of one loop,
// shared by the single-domain kernels (mk_kernels.cu) and the packed
// multi-domain ensemble (mk_ensemble.cu).
#ifndef MK_DENDRITE_CUH
#define MK_DENDRITE_CUH

#include "mk_device.cuh"
#include "../../include/mkb200.h"

namespace mkd {

// ========================================================== DENDRITE (K2/K3)
// Both D3Q7 lattices are held as deviations from the far-field liquid:
// g_i - w_i ref_g (ref_g = -1) and t_i - w_i ref_t (ref_t = -Delta).
template <class T>
struct DendK {
  T om_g, om_t, inv_tau0, lambda, eps4, eps2;
  int nobj, aniso;
  T ref_g, ref_t;
  T k_part, D_l, D_s, at_w0;  // solutal lattice
};

// phi of a streamed cell: the sum of its seven phase-field populations.
template <class S, class P, int PARITY, class NB>
__device__ __forceinline__ void pf_phi_cell(const S* __restrict__ G, P* __restrict__ phi_new, const int64_t stride,
                                            const NB& nb, const int c, const typename Stor<S>::T ref_g) {
  typedef typename Stor<S>::T T;
  T s = T(0);
  if constexpr (Stor<S>::scaled) {
    // 16-bit storage holds f'/w: sum each weight class in stored units and
    // scale once per class (2 multiplies instead of 7)
    T sa = T(0);
#pragma unroll
    for (int i = 1; i < 7; ++i) sa += ld_in_raw<S, 7>(G, stride, nb, PARITY, c, i);
    s = T(wq<7>(0)) * ld_in_raw<S, 7>(G, stride, nb, PARITY, c, 0) + T(wq<7>(1)) * sa;
  } else {
#pragma unroll
    for (int i = 0; i < 7; ++i) s += ld_in<S, 7>(G, stride, nb, PARITY, c, i);
  }
  phi_new[c] = P(ref_g + s);
}

// phi of the two cells a and b (b = a + 1 in x, a.c even, both fluid and on
// the FastW path): each slot pair of the even loop and each of the odd loop's
// slots without an x shift is one aligned pair load (the slot planes' stride
// is even); each cell's sum keeps pf_phi_cell's order, so both values are
// bit-identical to it.
template <class S, class P, int PARITY>
__device__ __forceinline__ void pf_phi_pair(const S* __restrict__ G, P* __restrict__ phi_new, const int64_t stride,
                                            const FastW& a, const FastW& b, const typename Stor<S>::T ref_g) {
  typedef typename Stor<S>::T T;
  T v0[7], v1[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    if (PARITY == 0 || ex(i) == 0) {
      ldr_pair(G + off_in<7>(stride, a, PARITY, a.c, i), v0[i], v1[i]);
    } else {
      v0[i] = ld_in_raw<S, 7>(G, stride, a, PARITY, a.c, i);
      v1[i] = ld_in_raw<S, 7>(G, stride, b, PARITY, b.c, i);
    }
  }
  T s0 = T(0), s1 = T(0);
  if constexpr (Stor<S>::scaled) {
    T sa0 = T(0), sa1 = T(0);
#pragma unroll
    for (int i = 1; i < 7; ++i) {
      sa0 += v0[i];
      sa1 += v1[i];
    }
    s0 = T(wq<7>(0)) * v0[0] + T(wq<7>(1)) * sa0;
    s1 = T(wq<7>(0)) * v1[0] + T(wq<7>(1)) * sa1;
  } else {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      s0 += v0[i];
      s1 += v1[i];
    }
  }
  st_pair(phi_new + a.c, P(ref_g + s0), P(ref_g + s1));
}

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256) k_pf_phi(const S* __restrict__ G, const P* __restrict__ phi_old,
                                                P* __restrict__ phi_new, const Geom g, typename Stor<S>::T ref_g) {
  typedef typename Stor<S>::T T;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  // planes in descending order: the collision kernel that follows walks them
  // ascending and starts on the planes whose populations this kernel read
  // last (still in L2)
  const int z = g.nz - 1 - (int)blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  if (!g.fluid(x, y, z)) {
    const int64_t c = g.idx(x, y, z);
    phi_new[c] = phi_old[c];
    return;
  }
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    pf_phi_cell<S, P, PARITY>(G, phi_new, g.stride, fa, fa.c, ref_g);
  } else {
    const Nbr nb(g, x, y, z);
    pf_phi_cell<S, P, PARITY>(G, phi_new, g.stride, nb, nb.idx(0, 0, 0), ref_g);
  }
}

// Nearest seed (ties to the lower index), in FP64 like the oracle.
__device__ __forceinline__ int nearest_seed(const double* __restrict__ seeds, int nobj, int x, int y, int z) {
  int best = 0;
  double bd = 1e300;
  for (int k = 0; k < nobj; ++k) {
    const double dx = x - __ldg(seeds + 12 * k + 0), dy = y - __ldg(seeds + 12 * k + 1),
                 dz = z - __ldg(seeds + 12 * k + 2);
    const double d = dx * dx + dy * dy + dz * dz;
    if (d < bd) {
      bd = d;
      best = k;
    }
  }
  return best;
}

// a(n) and da/dn of the anisotropy kinds (mk_anisotropy), n the crystal-frame
// unit normal (mkPhaseField::anisotropy / _cbc / _hcp / _facet,
// mkPhaseField.h:61-64).  The kind is uniform over a launch, so the switch
// never diverges.
template <class T>
__device__ __forceinline__ void aniso_function(int kind, T e4, T e2, const T (&n)[3], T& a, T (&g)[3]) {
  const T x = n[0], y = n[1], z = n[2];
  const T x2 = x * x, y2 = y * y, z2 = z * z;
  switch (kind) {
    case MK_ANISO_CBC: {
      const T s4 = x2 * x2 + y2 * y2 + z2 * z2, s6 = x2 * y2 * z2;
      a = T(1) + e4 * (s4 - T(0.6)) + e2 * (T(3) * s4 + T(66) * s6 - T(17.0 / 7.0));
      g[0] = T(4) * e4 * x2 * x + e2 * (T(12) * x2 * x + T(132) * x * y2 * z2);
      g[1] = T(4) * e4 * y2 * y + e2 * (T(12) * y2 * y + T(132) * y * x2 * z2);
      g[2] = T(4) * e4 * z2 * z + e2 * (T(12) * z2 * z + T(132) * z * x2 * y2);
      break;
    }
    case MK_ANISO_HCP: {
      const T c6 = x2 * x2 * x2 - T(15) * x2 * x2 * y2 + T(15) * x2 * y2 * y2 - y2 * y2 * y2;
      a = T(1) + e4 * c6 + e2 * (T(2) * z2 - T(1));
      g[0] = T(6) * e4 * (x2 * x2 * x - T(10) * x2 * x * y2 + T(5) * x * y2 * y2);
      g[1] = T(-6) * e4 * (T(5) * x2 * x2 * y - T(10) * x2 * y2 * y + y2 * y2 * y);
      g[2] = T(4) * e2 * z;
      break;
    }
    case MK_ANISO_FACET: {
      const T rx = sqrt(x2 + e2 * e2), ry = sqrt(y2 + e2 * e2), rz = sqrt(z2 + e2 * e2);
      a = T(1) + e4 * (rx + ry + rz - sqrt(T(1) + e2 * e2) - T(2) * e2);
      g[0] = e4 * x / rx;
      g[1] = e4 * y / ry;
      g[2] = e4 * z / rz;
      break;
    }
    default: {
      const T s4 = x2 * x2 + y2 * y2 + z2 * z2;
      a = T(1) - T(3) * e4 + T(4) * e4 * s4;
      g[0] = T(16) * e4 * x2 * x;
      g[1] = T(16) * e4 * y2 * y;
      g[2] = T(16) * e4 * z2 * z;
      break;
    }
  }
}

// a(n) and the lab-frame vector N of the anisotropic flux (Karma-Rappel):
// N_c = |grad phi| a (da/dn - n (n . da/dn)) in the crystal frame.  `Rm` is
// the grain's rotation (row-major, columns = crystal axes) in the arithmetic
// type.
// GEN = false compiles the four-fold cubic kind alone (the form of the
// reference's default anisotropy()); GEN = true takes any kind at run time.
template <class T, bool GEN = true>
__device__ __forceinline__ void anisotropy(const T* __restrict__ Rm, int kind, T eps4, T eps2, const T (&gr)[3],
                                           T& a, T (&N)[3]) {
  T R[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) R[q] = __ldg(Rm + q);
  const T gn = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
  const T inv = div_fast(T(1), gn + T(1e-12));
  const T nl0 = gr[0] * inv, nl1 = gr[1] * inv, nl2 = gr[2] * inv;
  T nc[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) nc[q] = R[0 * 3 + q] * nl0 + R[1 * 3 + q] * nl1 + R[2 * 3 + q] * nl2;
  T Nc[3];
  if constexpr (!GEN) {
    (void)kind;
    (void)eps2;
    const T s4 = nc[0] * nc[0] * nc[0] * nc[0] + nc[1] * nc[1] * nc[1] * nc[1] + nc[2] * nc[2] * nc[2] * nc[2];
    a = T(1) - T(3) * eps4 + T(4) * eps4 * s4;
#pragma unroll
    for (int q = 0; q < 3; ++q) Nc[q] = gn * a * T(16) * eps4 * (nc[q] * nc[q] * nc[q] - nc[q] * s4);
  } else {
    T da[3];
    aniso_function<T>(kind, eps4, eps2, nc, a, da);
    const T ndg = nc[0] * da[0] + nc[1] * da[1] + nc[2] * da[2];
#pragma unroll
    for (int q = 0; q < 3; ++q) Nc[q] = gn * a * (da[q] - nc[q] * ndg);
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) N[q] = R[q * 3 + 0] * Nc[0] + R[q * 3 + 1] * Nc[1] + R[q * 3 + 2] * Nc[2];
}

// One loop of a dendrite cell: the phase-field lattice, then the thermal
// (SOL = false) or solutal (SOL = true) lattice.  `grain` is the per-cell
// grain index (read only with more than one grain), `rot` the rotations of
// the cell's domain, 9 values per grain.  ADV = true advects the scalar
// equilibrium with the flow velocity (vx, vy, vz): t_eq = w T (1 + 4 e.u)
// (mkThermalField::relaxation with a flow lattice, getTEquPDFs); for the
// solutal lattice the advective flux U u joins the anti-trapping current in
// the equilibrium's first moment (the liquid's w U (1 + 4 e.u)).
// NEE = true (with ADV) also applies the inflow / outflow faces of the flow
// + dendrite models in registers: the cell at x = 0 (x = nx - 1) takes the
// post-collision g, t of its inner neighbour — the next (previous) lane of
// its warp, so nx % 32 != 1 and the row starts a warp — by shuffles:
//   g(b) = g(n) + w (phi_b - phi_n),
//   t(b) = t(n) + w T_b (1 + 4 e.u_b) - w T_n (1 + 4 e.u_n),
// inflow phi_b = -1, T_b = ref_t; outflow phi_b = phi_n, T_b = T_n; u_b is
// the face cell's own (vx, vy, vz), u_n the neighbour's; temp(b) = T_b (T is
// the supersaturation U for the solutal lattice: bdy_LBflowin,
// mkSolutalField.h:53).
template <class S, class P, int PARITY, bool SOL, bool GEN, class NB, bool ADV = false, bool NEE = false>
__device__ __forceinline__ void dend_cell(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phi_new,
                                          const P* __restrict__ phi_old, P* __restrict__ temp,
                                          const unsigned char* __restrict__ grain,
                                          const typename Stor<S>::T* __restrict__ rot, const int64_t stride,
                                          const NB& nb, const int c, const DendK<typename Stor<S>::T>& k,
                                          typename Stor<S>::T vx = 0, typename Stor<S>::T vy = 0,
                                          typename Stor<S>::T vz = 0, int x = 0, int nx = 0) {
  static_assert(!NEE || ADV, "the face pass belongs to the advected scalar lattice");
  typedef typename Stor<S>::T T;
  // FP32 / FP64: both lattices' slots go to L2 now, while the phi stencil
  // and the anisotropy are computed (the kernel waits on load latency;
  // measured 128^3 FP32 collide 58 -> 53 us).  With 16-bit storage the extra
  // instructions cost more than they hide (ensemble BF16 0.98 -> 1.06 ms).
  if constexpr (Stor<S>::bytes >= 4) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      pf_in<S, 7>(G, stride, nb, PARITY, c, i);
      pf_in<S, 7>(Tp, stride, nb, PARITY, c, i);
    }
  }
  const T ph = T(phi_new[c]);
  T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
  for (int i = 1; i < 19; ++i) {
    const T fn = nb_fluid(nb, ex(i), ey(i), ez(i)) ? T(__ldg(phi_new + nb_idx(nb, ex(i), ey(i), ez(i)))) : ph;
    const T w = T(wq<19>(i));
    if (ex(i)) gx += (w * T(ex(i))) * fn;
    if (ey(i)) gy += (w * T(ey(i))) * fn;
    if (ez(i)) gz += (w * T(ez(i))) * fn;
  }
  const T gr[3] = {T(3) * gx, T(3) * gy, T(3) * gz};
  const int gid = k.nobj > 1 ? (int)__ldg(grain + c) : 0;
  T a, N[3];
  anisotropy<T, GEN>(rot + 9 * gid, k.aniso, k.eps4, k.eps2, gr, a, N);
  const T dphi = ph - T(phi_old[c]);
  const T u_old = T(temp[c]);
  const T one_m = T(1) - ph * ph;
  const T src = (ph - ph * ph * ph - k.lambda * u_old * one_m * one_m) * k.inv_tau0 + (T(1) - a * a) * dphi;
  const T cs2 = T(0.25);
  const T B0 = -cs2 * ((a * a - T(1)) * gr[0] + N[0]);
  const T B1 = -cs2 * ((a * a - T(1)) * gr[1] + N[1]);
  const T B2 = -cs2 * ((a * a - T(1)) * gr[2] + N[2]);
  const T fo = (T(1) - T(0.5) * k.om_g) / cs2;
  // SU: 16-bit storage holds f'/w; both lattices are then updated in those
  // stored units (every term of the BGK/TRT updates below carries the factor
  // w_i, so dividing by it leaves no weights to apply per population), and
  // the weight enters only the class sum of T.  Off with the face pass.
  constexpr bool SU = Stor<S>::scaled && !NEE;
  // phase-field lattice, all seven loaded before any store (in-place safety)
  T gv[7];
#pragma unroll
  for (int i = 0; i < 7; ++i)
    gv[i] = SU ? ld_in_raw<S, 7>(G, stride, nb, PARITY, c, i) : ld_in<S, 7>(G, stride, nb, PARITY, c, i);
  const T dph = ph - k.ref_g;
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    const T w = SU ? T(1) : T(wq<7>(i));
    const T eB = T(ex(i)) * B0 + T(ey(i)) * B1 + T(ez(i)) * B2;
    const T go = gv[i] - k.om_g * (gv[i] - w * dph) + fo * w * eB + w * src;
    if constexpr (NEE)
      gv[i] = go;  // stored after the face pass below
    else if constexpr (SU)
      st_out_raw<S, 7>(G, stride, nb, PARITY, c, i, go);
    else
      st_out<S, 7>(G, stride, nb, PARITY, c, i, go);
  }
  T t[7];
  T dT = T(0);
  if constexpr (SU) {
    T sa = T(0);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      t[i] = ld_in_raw<S, 7>(Tp, stride, nb, PARITY, c, i);
      if (i > 0) sa += t[i];
    }
    dT = T(wq<7>(0)) * t[0] + T(wq<7>(1)) * sa;
  } else {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      t[i] = ld_in<S, 7>(Tp, stride, nb, PARITY, c, i);
      dT += t[i];
    }
  }
  if constexpr (SOL) {
    // solutal lattice (TRT): capacity c(phi) applied to D(phi), the
    // anti-trapping current (first moment of the equilibrium) and the
    // rejection source; pair sums relax to equilibrium with rate 1, pair
    // differences with omega(phi)
    // three divisions: su, then fj = -2 a_t W0 su / (|grad phi| + 1e-6) and
    // om = 1 / (4 D + 1/2) = c / (4 c D + c/2) with c D the numerator of D
    // (FP32: the fast division, well inside the single-precision tolerance)
    const T U = k.ref_t + dT;
    const T km = T(1) - k.k_part;
    const T cap = (T(1) + k.k_part - km * ph) * T(0.5);
    const T gn = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
    const T su = div_fast(T(0.5) * (T(1) + km * U) * dphi, cap);
    const T fj = div_fast(T(-2) * k.at_w0 * su, gn + T(1e-6));
    const T cD = k.D_l * (T(1) - ph) * T(0.5) + k.D_s * (T(1) + ph) * T(0.5);
    const T om = div_fast(cap, T(4) * cD + T(0.5) * cap);
    {
      const T w0 = SU ? T(1) : T(wq<7>(0));
      if constexpr (NEE)
        t[0] = w0 * dT + w0 * su;  // stored after the face pass below
      else if constexpr (SU)
        st_out_raw<S, 7>(Tp, stride, nb, PARITY, c, 0, w0 * dT + w0 * su);
      else
        st_out<S, 7>(Tp, stride, nb, PARITY, c, 0, w0 * dT + w0 * su);
    }
#pragma unroll
    for (int i = 1; i < 7; i += 2) {
      const int j = i + 1;
      const T w = SU ? T(1) : T(wq<7>(i));
      T ej = fj * (T(ex(i)) * gr[0] + T(ey(i)) * gr[1] + T(ez(i)) * gr[2]);
      if constexpr (ADV) ej += U * (T(ex(i)) * vx + T(ey(i)) * vy + T(ez(i)) * vz);
      const T sym = w * dT;
      const T am = T(0.5) * (t[i] - t[j]);
      const T am_new = am - om * (am - w * T(4) * ej);
      if constexpr (NEE) {
        t[i] = sym + am_new + w * su;
        t[j] = sym - am_new + w * su;
      } else if constexpr (SU) {
        st_out_raw<S, 7>(Tp, stride, nb, PARITY, c, i, sym + am_new + w * su);
        st_out_raw<S, 7>(Tp, stride, nb, PARITY, c, j, sym - am_new + w * su);
      } else {
        st_out<S, 7>(Tp, stride, nb, PARITY, c, i, sym + am_new + w * su);
        st_out<S, 7>(Tp, stride, nb, PARITY, c, j, sym - am_new + w * su);
      }
    }
  } else {
    // thermal lattice: relaxation with latent heat (1/2) dphi
    const T lat = T(0.5) * dphi;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      const T w = SU ? T(1) : T(wq<7>(i));
      T eq = dT;
      if constexpr (ADV) {
        const T eu = T(ex(i)) * vx + T(ey(i)) * vy + T(ez(i)) * vz;
        if (i > 0) eq += T(4) * (k.ref_t + dT) * eu;
      }
      const T to = t[i] - k.om_t * (t[i] - w * eq) + w * lat;
      if constexpr (NEE)
        t[i] = to;
      else if constexpr (SU)
        st_out_raw<S, 7>(Tp, stride, nb, PARITY, c, i, to);
      else
        st_out<S, 7>(Tp, stride, nb, PARITY, c, i, to);
    }
  }
  T Tc = k.ref_t + dT;
  if constexpr (NEE) {
    const unsigned act = __activemask();
    const bool edge = x == 0 || x == nx - 1;
    if (__any_sync(act, edge)) {
      const int lane = threadIdx.x & 31;
      const int src = x == 0 ? lane + 1 : lane - 1;
      T sg = T(0), st = T(0);
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        sg += gv[i];
        st += t[i];
      }
      sg = __shfl_sync(act, sg, src);
      st = __shfl_sync(act, st, src);
      const T un0 = __shfl_sync(act, vx, src), un1 = __shfl_sync(act, vy, src), un2 = __shfl_sync(act, vz, src);
      const T phn = k.ref_g + sg, Tn = k.ref_t + st;
      const T phb = x == 0 ? T(-1) : phn, Tb = x == 0 ? k.ref_t : Tn;
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        const T gn = __shfl_sync(act, gv[i], src), tn = __shfl_sync(act, t[i], src);
        if (edge) {
          const T w = T(wq<7>(i));
          const T evn = T(ex(i)) * un0 + T(ey(i)) * un1 + T(ez(i)) * un2;
          const T evb = T(ex(i)) * vx + T(ey(i)) * vy + T(ez(i)) * vz;
          gv[i] = gn + w * (phb - phn);
          t[i] = tn + w * (Tb * (T(1) + T(4) * evb) - Tn * (T(1) + T(4) * evn));
        }
      }
      if (edge) Tc = Tb;
    }
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      st_out<S, 7>(G, stride, nb, PARITY, c, i, gv[i]);
      st_out<S, 7>(Tp, stride, nb, PARITY, c, i, t[i]);
    }
  }
  temp[c] = P(Tc);
}

// 16-bit storage: five resident 256-thread blocks per SM (48 registers, a few
// spilled bytes) for more loads in flight; measured 128^3 FP16 collide
// 47.4 -> 46.4 us.
template <class S, class P, int PARITY, bool SOL, bool GEN>
__global__ void __launch_bounds__(256, Stor<S>::bytes == 2 ? 5 : 1)
    k_dend_collide(S* __restrict__ G, S* __restrict__ Tp, const P* __restrict__ phi_new, const P* __restrict__ phi_old,
                   P* __restrict__ temp, const unsigned char* __restrict__ grain,
                   const typename Stor<S>::T* __restrict__ rot, const Geom g, const DendK<typename Stor<S>::T> k) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  if (fastw_cell(g, x, y, z)) {
    const FastW fa = make_fastw(g, x, y, z);
    dend_cell<S, P, PARITY, SOL, GEN>(G, Tp, phi_new, phi_old, temp, grain, rot, g.stride, fa, fa.c, k);
  } else {
    const Nbr nb(g, x, y, z);
    dend_cell<S, P, PARITY, SOL, GEN>(G, Tp, phi_new, phi_old, temp, grain, rot, g.stride, nb, nb.idx(0, 0, 0), k);
  }
}

// Per-cell grain index: the nearest seed in FP64, ties to the lower index
// (computed once; the seeds do not move).
static __global__ void k_grain_map(const Geom g, const double* __restrict__ seeds, int nobj, int base,
                            unsigned char* __restrict__ grain) {
  const int n = g.nx * g.ny * g.nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int z = i / (g.nx * g.ny), r = i - z * g.nx * g.ny, y = r / g.nx, x = r - y * g.nx;
    grain[base + i] = (unsigned char)(nobj > 1 ? nearest_seed(seeds, nobj, x, y, z) : 0);
  }
}


// Kernel coefficients of a dendrite case (host side).
template <class T>
inline DendK<T> dend_params(const mk_params& p, double ref_g, double ref_t) {
  DendK<T> k;
  const double D0 = p.W0 * p.W0 / p.tau0;
  k.om_g = T(1.0 / (4.0 * D0 + 0.5));
  k.om_t = T(1.0 / (4.0 * p.D + 0.5));
  k.inv_tau0 = T(1.0 / p.tau0);
  k.lambda = T(p.lambda);
  k.eps4 = T(p.eps4);
  k.eps2 = T(p.eps2);
  k.nobj = p.n_objects;
  k.aniso = p.aniso;
  k.ref_g = T(ref_g);
  k.ref_t = T(ref_t);
  k.k_part = T(p.k_part);
  k.D_l = T(p.D);
  k.D_s = T(p.D_s);
  k.at_w0 = T(p.at_coef * p.W0);
  return k;
}

}  // namespace mkd

#endif
