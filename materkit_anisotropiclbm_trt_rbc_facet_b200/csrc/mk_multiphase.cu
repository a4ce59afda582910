// mk_multiphase.cu — the two-phase Allen-Cahn loop (K4): the phi kernel and
// the collision kernel, and the fused one-launch loop, with their launchers
// (mkFluidsMultiphase::propagate/relaxation, mkFluidsMultiphase.h:52-57;
// getEquPDFsLiang/PhiLiang, mkNode.h:38-40).
#include <cuda.h>  // CUtensorMap and its encoding enums (resolved through the runtime)

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "mk_device.cuh"
#include "mk_engine.hpp"
#include "mk_shared.cuh"
#include "mk_wave.cuh"

using namespace mkd;
using namespace mks;

namespace {

// The neighbourhood and the cell index made to depend on a value computed
// late in the collision, so no slot address derived from them exists before
// it (the asm emits nothing).  Applied in the even loop with FP64 and 16-bit
// storage, where it lowers the registers and raises the warps per SM:
// 186 -> 152 registers FP64, 120 -> 96 FP16 / BF16; 256^3 collide FP64
// 1.894 -> 1.759 ms, FP16 0.766 -> 0.746 ms.  With FP32 storage it measured
// 0.912 -> 0.925 ms and in the odd loop it raised the registers, so those
// keep the plain form.
template <class T>
__device__ __forceinline__ void dep(Fast& f, int& c, T v) {
  if constexpr (sizeof(T) == 8)
    asm volatile("" : "+r"(f.c), "+r"(c) : "d"(v));
  else
    asm volatile("" : "+r"(f.c), "+r"(c) : "f"(v));
}
template <class T>
__device__ __forceinline__ void dep(Nbr& f, int& c, T v) {
  if constexpr (sizeof(T) == 8)
    asm volatile("" : "+r"(f.base), "+r"(c) : "d"(v));
  else
    asm volatile("" : "+r"(f.base), "+r"(c) : "f"(v));
}

// The planes z_lo .. z_lo + gridDim.z - 1.
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256) k_mp_phi(const S* __restrict__ H, const float* __restrict__ H0,
                                                P* __restrict__ phi, const Geom g, typename Stor<S>::T ref_h,
                                                const int z_lo) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  // planes in descending order: the collision kernel that follows walks them
  // ascending, so it starts on the planes whose h this kernel read last
  // (still in L2), and it ends where the next loop's phi kernel starts
  const int z = z_lo + (int)(gridDim.z - 1 - blockIdx.z);
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  if (fast_cell(g, x, y, z)) {
    const Fast fa = make_fast(g, x, y, z);
    mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, fa, fa.c, ref_h);
  } else {
    const Nbr nb(g, x, y, z);
    mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, nb, nb.idx(0, 0, 0), ref_h);
  }
}

// Two stored 16-bit values at p (p 4-byte aligned) as floats.
__device__ __forceinline__ float2 ldr2(const __half* p) { return __half22float2(*reinterpret_cast<const __half2*>(p)); }
__device__ __forceinline__ float2 ldr2(const __nv_bfloat16* p) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}

// The phi kernel with 16-bit storage, two cells per thread (x even, nx
// even): a 16-bit load per slot moves half the bytes of an FP32 one, so
// each slot pair that is 4-byte aligned (every slot of the even loop, the
// odd loop's directions without an x component) is one 32-bit load; the odd
// loop's x-shifted slots stay 16-bit loads per cell.  Each cell's sums run
// in mp_phi_cell's order, so phi is bit-identical.  Pairs with a cell off
// the interior path or not fluid take mp_phi_cell per cell.
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256) k_mp_phi2(const S* __restrict__ H, const float* __restrict__ H0,
                                                 P* __restrict__ phi, const Geom g, typename Stor<S>::T ref_h,
                                                 const int z_lo) {
  const int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = z_lo + (int)(gridDim.z - 1 - blockIdx.z);
  if (x >= g.nx || y >= g.ny) return;
  const bool f0 = g.fluid(x, y, z), f1 = g.fluid(x + 1, y, z);
  if (f0 && f1 && fast_cell(g, x, y, z) && fast_cell(g, x + 1, y, z)) {
    const Fast a = make_fast(g, x, y, z), b = make_fast(g, x + 1, y, z);
    const int64_t st = g.stride;
    const float2 r0 = *reinterpret_cast<const float2*>(H0 + a.c);
    float sa0 = 0.f, sa1 = 0.f, sd0 = 0.f, sd1 = 0.f;
#pragma unroll
    for (int i = 1; i < 19; ++i) {
      float v0, v1;
      if (PARITY == 0 || ex(i) == 0) {
        const int64_t o = PARITY == 0 ? (int64_t)i * st + a.c : (int64_t)inv(i) * st + a.idx(0, -ey(i), -ez(i));
        const float2 v = ldr2(H + o);
        v0 = v.x;
        v1 = v.y;
      } else {
        v0 = Stor<S>::ldr(H + (int64_t)inv(i) * st + a.idx(-ex(i), -ey(i), -ez(i)));
        v1 = Stor<S>::ldr(H + (int64_t)inv(i) * st + b.idx(-ex(i), -ey(i), -ez(i)));
      }
      if (i < 7) {
        sa0 += v0;
        sa1 += v1;
      } else {
        sd0 += v0;
        sd1 += v1;
      }
    }
    float s0 = r0.x, s1 = r0.y;
    s0 += float(wq<19>(1)) * sa0 + float(wq<19>(7)) * sd0;
    s1 += float(wq<19>(1)) * sa1 + float(wq<19>(7)) * sd1;
    *reinterpret_cast<float2*>(phi + a.c) = make_float2(ref_h + s0, ref_h + s1);
    return;
  }
  for (int k = 0; k < 2; ++k) {
    const int xx = x + k;
    if (!(k == 0 ? f0 : f1)) continue;
    if (fast_cell(g, xx, y, z)) {
      const Fast fa = make_fast(g, xx, y, z);
      mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, fa, fa.c, ref_h);
    } else {
      const Nbr nb(g, xx, y, z);
      mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, nb, nb.idx(0, 0, 0), ref_h);
    }
  }
}

// Where a collision reads its pre-collision populations: straight from the
// lattices in global memory (GlobalLd), or from rows the bulk-copy engine
// staged in shared memory (RowLd, below).  g(i) / h(0) return f'_i, hr(i)
// the stored value (f'_i, or f'_i / w_i in 16-bit storage), h0() the FP32
// rest population of 16-bit storage.
template <class S, int PARITY, class NB>
struct GlobalLd {
  typedef typename Stor<S>::T T;
  const S* __restrict__ G;
  const S* __restrict__ H;
  const float* __restrict__ H0;
  int64_t stride;
  const NB& nb;
  int c;
  // the Allen-Cahn slots go to L2 now (FP32 / FP64; with 16-bit storage the
  // prefetch measured 2% slower) and are loaded once the pressure lattice is
  // stored, so the two lattices' populations are never live together
  // (register pressure sets the occupancy of this kernel)
  __device__ __forceinline__ void prefetch() const {
    if constexpr (Stor<S>::bytes >= 4) {
#pragma unroll
      for (int i = 1; i < 19; ++i) pf_in<S, 19>(H, stride, nb, PARITY, c, i);
    }
  }
  __device__ __forceinline__ T g(int i) const { return ld_in<S, 19>(G, stride, nb, PARITY, c, i); }
  __device__ __forceinline__ T h(int i) const { return ld_in<S, 19>(H, stride, nb, PARITY, c, i); }
  __device__ __forceinline__ T hr(int i) const { return ld_in_raw<S, 19>(H, stride, nb, PARITY, c, i); }
  // the same slot through another neighbourhood value (see dep)
  __device__ __forceinline__ T hr2(int i, const NB& nb2, int c2) const {
    return ld_in_raw<S, 19>(H, stride, nb2, PARITY, c2, i);
  }
  __device__ __forceinline__ T h0() const { return T(H0[c]); }
};

// One loop of a fluid cell.  Every population load (19 g, 19 h) is issued
// before any store: the loads are the latency the kernel must hide, and a
// store into the same array in between would stop the compiler from hoisting
// the later loads (in place, on odd loops a direction's result goes to the
// slot its opposite direction is read from).
template <class S, class P, int PARITY, class NB, class PH, class LD>
__device__ __forceinline__ void mp_collide_cell(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0,
                                                const PH& phi_src, const int64_t stride, const NB& nb,
                                                const int c, const MpK<typename Stor<S>::T>& k, const LD& ld) {
  typedef typename Stor<S>::T T;
  constexpr bool LATE = PARITY == 0 && Stor<S>::bytes != 4;  // see dep
  ld.prefetch();
  T gp_[19];  // g (rests at 0)
#pragma unroll
  for (int i = 0; i < 19; ++i) gp_[i] = ld.g(i);
  T m[19];  // MRT moments: m[0] = p*, (m[3], m[5], m[7]) = j
  mrt19_moments<T>(gp_, m);
  const T pstar = m[0], jx = m[3], jy = m[5], jz = m[7];
  T ph, rho, gphi[3], F[3];
  mp_force_src<T, P, NB>(phi_src, nb, k, pstar, ph, rho, gphi, F);
  const T irho = div_fast(T(1), rho);
  const T ux = jx + T(0.5) * F[0] * irho;
  const T uy = jy + T(0.5) * F[1] * irho;
  const T uz = jz + T(0.5) * F[2] * irho;
  const T uu = ux * ux + uy * uy + uz * uz;
  // ---- pressure/velocity lattice: moment-space MRT with the Guo force / rho
  {
    MrtIn<T> q;
    q.a0 = pstar - T(1.5) * uu;
    q.bx = ux;
    q.by = uy;
    q.bz = uz;
    q.qxx = ux * ux;
    q.qyy = uy * uy;
    q.qzz = uz * uz;
    q.qxy = ux * uy;
    q.qxz = ux * uz;
    q.qyz = uy * uz;
    q.Fx = F[0];
    q.Fy = F[1];
    q.Fz = F[2];
    q.ux = ux;
    q.uy = uy;
    q.uz = uz;
    q.sF = irho;
    q.s_nu = div_fast(T(1), k.tau_g + ph * (k.tau_l - k.tau_g));
    mrt19_relax_back<T>(gp_, m, q);
    NB nbg = nb;
    int cg = c;
    if constexpr (LATE) dep(nbg, cg, gp_[0]);
#pragma unroll
    for (int i = 0; i < 19; ++i) st_out<S, 19>(G, stride, nbg, PARITY, cg, i, gp_[i]);
  }
  const T gn = sqrt(gphi[0] * gphi[0] + gphi[1] * gphi[1] + gphi[2] * gphi[2]);
  const T inv_gn = div_fast(T(1), gn + T(1e-12));
  const T nx_ = gphi[0] * inv_gn, ny_ = gphi[1] * inv_gn, nz_ = gphi[2] * inv_gn;
  const T lam = k.inv_w4 * ph * (T(1) - ph);
  // ---- Allen-Cahn lattice (BGK + sharpening flux), pair by pair, in the
  // stored units (h' = h - w, or h'/w for 16-bit storage, sig = w or 1):
  //   h*' = (1 - om) h' + sig [om (X_even +- X_odd) +- Y],
  //   heq_i - w_i = w_i [X_even + X_odd], X_even = (phi - 1) + phi (4.5(eu)^2 - 1.5u^2),
  //   X_odd = 3 phi eu, the sharpening flux w_i Y = w_i (1 - om/2) lam (e.n)
  constexpr bool SC = Stor<S>::scaled;
  T h[19];
  NB nbh = nb;
  int ch = c;
  if constexpr (LATE) dep(nbh, ch, gp_[18]);
  h[0] = Rest32<S>::on ? ld.h0() : ld.h(0);
#pragma unroll
  for (int i = 1; i < 19; ++i) h[i] = ld.hr2(i, nbh, ch);
  const T om_h = k.om_h;
  const T one_om = T(1) - om_h;
  const T src = (T(1) - T(0.5) * om_h) * lam;
  const T dph = ph - k.ref_h;
  T res_a = T(0), res_d = T(0);  // what the 16-bit stores rounded away, per weight class (Rest32 only)
  if constexpr (std::is_same<T, float>::value) {
    // FP32 arithmetic: two pairs per packed instruction, the pairs of equal
    // weight grouped (+-x with +-y, then the four diagonal planes two by
    // two); the +-z pair goes alone
    auto store = [&](int i, float v, bool axis) {
      if constexpr (Rest32<S>::on) {
        const float r = v - st_out_raw_rt<S, 19>(H, stride, nbh, PARITY, ch, i, v);
        if (axis)
          res_a += r;
        else
          res_d += r;
      } else {
        st_out_raw<S, 19>(H, stride, nbh, PARITY, ch, i, v);
      }
    };
    const float2 b_ph = bc2(ph), b_dph = bc2(dph), b_uu = bc2(-1.5f * uu), b_one_om = bc2(one_om);
    const float2 b_om = bc2(om_h), b_3phom = bc2(3.0f * ph * om_h), b_src = bc2(src), b_m1 = bc2(-1.0f);
    auto group = [&](int p, int q, float2 eu, float2 en, float sg) {
      const float2 t = fma2(bc2(4.5f), mul2(eu, eu), b_uu);
      const float2 E = mul2(b_om, fma2(b_ph, t, b_dph));          // om X_even
      const float2 Pq = fma2(b_3phom, eu, mul2(b_src, en));       // om X_odd + Y
      float2 a = add2(E, Pq), b = fma2(Pq, b_m1, E);
      if (!SC) {
        a = mul2(bc2(sg), a);
        b = mul2(bc2(sg), b);
      }
      const float2 hi = make_float2(h[2 * p - 1], h[2 * q - 1]), hj = make_float2(h[2 * p], h[2 * q]);
      const float2 vi = fma2(b_one_om, hi, a), vj = fma2(b_one_om, hj, b);
      const bool ax = p <= 3;
      store(2 * p - 1, vi.x, ax);
      store(2 * p, vj.x, ax);
      store(2 * q - 1, vi.y, ax);
      store(2 * q, vj.y, ax);
    };
    const float wa = float(wq<19>(1)), wd = float(wq<19>(7));
    group(1, 2, make_float2(ux, uy), make_float2(nx_, ny_), wa);
    group(4, 5, make_float2(ux + uy, ux - uy), make_float2(nx_ + ny_, nx_ - ny_), wd);
    group(6, 7, make_float2(ux + uz, ux - uz), make_float2(nx_ + nz_, nx_ - nz_), wd);
    group(8, 9, make_float2(uy + uz, uy - uz), make_float2(ny_ + nz_, ny_ - nz_), wd);
    {
      // +-z alone
      const float sg = SC ? 1.0f : wa;
      const float eu = uz, en = nz_;
      const float E = om_h * (dph + ph * (4.5f * eu * eu - 1.5f * uu));
      const float Pq = 3.0f * ph * om_h * eu + src * en;
      store(5, one_om * h[5] + sg * (E + Pq), true);
      store(6, one_om * h[6] + sg * (E - Pq), true);
    }
  } else {
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const int i = 2 * p - 1, j = 2 * p;
    const T sig = SC ? T(1) : T(wq<19>(i));
    const T eu = T(ex(i)) * ux + T(ey(i)) * uy + T(ez(i)) * uz;
    const T en = T(ex(i)) * nx_ + T(ey(i)) * ny_ + T(ez(i)) * nz_;
    const T xe = dph + ph * (T(4.5) * eu * eu - T(1.5) * uu);
    const T xo = ph * (T(3) * eu);
    const T y = src * en;
    const T vi = one_om * h[i] + sig * (om_h * (xe + xo) + y);
    const T vj = one_om * h[j] + sig * (om_h * (xe - xo) - y);
    if constexpr (Rest32<S>::on) {
      const T r = (vi - st_out_raw_rt<S, 19>(H, stride, nbh, PARITY, ch, i, vi)) +
                  (vj - st_out_raw_rt<S, 19>(H, stride, nbh, PARITY, ch, j, vj));
      if (p <= 3)
        res_a += r;
      else
        res_d += r;
    } else {
      st_out_raw<S, 19>(H, stride, nbh, PARITY, ch, i, vi);
      st_out_raw<S, 19>(H, stride, nbh, PARITY, ch, j, vj);
    }
  }
  }
  {
    const T w = T(wq<19>(0));
    const T h0 = h[0];
    const T heq = w * (dph - T(1.5) * ph * uu);
    const T v0 = h0 - om_h * (h0 - heq);
    if constexpr (Rest32<S>::on)
      H0[c] = float(v0 + (T(wq<19>(1)) * res_a + T(wq<19>(7)) * res_d));
    else
      st_out<S, 19>(H, stride, nb, PARITY, c, 0, v0);
  }
}

// One fluid cell of the thread-per-cell collision (planes z_lo ..
// z_lo + gridDim.z - 1).  Interior rows take the Fast addressing.
template <class S, class P, int PARITY>
__device__ __forceinline__ void mp_collide_thread(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0,
                                                  const P* __restrict__ phi, const Geom& g,
                                                  const MpK<typename Stor<S>::T>& k, int z_lo) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = z_lo + (int)blockIdx.z;
  if (x >= g.nx || y >= g.ny || !g.fluid(x, y, z)) return;
  if (fast_cell(g, x, y, z)) {
    const Fast fa = make_fast(g, x, y, z);
    mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Fast>{phi, fa, fa.c}, g.stride, fa, fa.c, k,
                                  GlobalLd<S, PARITY, Fast>{G, H, H0, g.stride, fa, fa.c});
  } else {
    const Nbr nb(g, x, y, z);
    const int c = nb.idx(0, 0, 0);
    mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Nbr>{phi, nb, c}, g.stride, nb, c, k,
                                  GlobalLd<S, PARITY, Nbr>{G, H, H0, g.stride, nb, c});
  }
}

// Occupancy variants of the collision: MINB 1 or 2 resident 256-thread blocks
// per SM (1 keeps every value in registers, 2 doubles the warps per SM at the
// price of a few spills); k_mp_collide_r caps the registers at R (with
// 64-thread blocks 112 gives 18 warps per SM, 96 gives 20, 80 gives 24).
// The autotuner picks (minb 3, 4, 5 select R = 112, 96, 80).
template <class S, class P, int PARITY, int MINB>
__global__ void __launch_bounds__(256, MINB) k_mp_collide(S* __restrict__ G, S* __restrict__ H,
                                                          float* __restrict__ H0, const P* __restrict__ phi,
                                                          const Geom g, const MpK<typename Stor<S>::T> k,
                                                          const int z_lo) {
  mp_collide_thread<S, P, PARITY>(G, H, H0, phi, g, k, z_lo);
}
template <class S, class P, int PARITY, int R>
__global__ void __maxnreg__(R) k_mp_collide_r(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0,
                                              const P* __restrict__ phi, const Geom g,
                                              const MpK<typename Stor<S>::T> k, const int z_lo) {
  mp_collide_thread<S, P, PARITY>(G, H, H0, phi, g, k, z_lo);
}

// ------------------------------------------- row-staged collision (rows)
// The two-kernel loop's collision with its population loads handed to the
// bulk-copy engine.  A CTA owns whole x rows (one thread per cell) and keeps
// `ns` rows in flight: for each row it stages the 19 g and 19 h source rows
// (and the FP32 rest row of 16-bit storage) into shared memory with
// cp.async.bulk, completing on the row's mbarrier, while it computes the row
// staged before.  The bytes in flight no longer depend on how many warps the
// collision's registers leave resident.
//
// The source row of direction i: on even loops the cell's own row of plane i;
// on odd loops the row (y - e_y, z - e_z) of plane inv(i), or the own row of
// plane i when that row link is closed (wall, closed face, slab end).  The x
// shift of an odd loop is a column offset in shared memory (periodic x wraps
// inside the staged row); a closed x link (walled or closed x, at the row
// ends only) reads the own slot from global memory.  Every slot a row's
// cells read is read and later written by that cell alone (AA ownership), so
// staging ahead races with nothing.  The per-cell arithmetic is
// mp_collide_cell's, on the same values: the result is bit-identical to
// k_mp_collide.
struct RowPlan {
  int nrows;      // fluid rows (y, z)
  int ylo, nyf;   // fluid y span
  int zlo;        // first fluid plane
  int xlo, xhi;   // fluid x span
  int xper;       // x periodic
  int xf;         // a fluid x (row link tests)
  int ns;         // rows in flight per CTA
  int stage;      // bytes of one staged row
};

template <class S, int PARITY>
struct RowLd {
  typedef typename Stor<S>::T T;
  const S* sg;         // staged g rows [19][nx]
  const S* sh;         // staged h rows [19][nx]
  const float* sh0;    // staged FP32 rest row (16-bit storage)
  int x, nx;
  unsigned rowok;      // odd loops: bit i set when the row link of direction i is open
  int xm, xp;          // column of the x - 1 / x + 1 source, -1 when that link is closed
  const S* __restrict__ G;
  const S* __restrict__ H;
  int64_t stride;
  int c;
  __device__ __forceinline__ void prefetch() const {}
  // shared-memory column of direction i's source, -1 for the cell's own slot in global memory
  __device__ __forceinline__ int col(int i) const {
    if (PARITY == 0 || ex(i) == 0 || !((rowok >> i) & 1u)) return x;
    return ex(i) > 0 ? xm : xp;
  }
  __device__ __forceinline__ T g(int i) const {
    const int q = col(i);
    return Stor<S>::ld(q >= 0 ? sg + i * nx + q : G + i * stride + c, T(wq<19>(i)));
  }
  __device__ __forceinline__ T h(int i) const {
    const int q = col(i);
    return Stor<S>::ld(q >= 0 ? sh + i * nx + q : H + i * stride + c, T(wq<19>(i)));
  }
  __device__ __forceinline__ T hr(int i) const {
    const int q = col(i);
    return Stor<S>::ldr(q >= 0 ? sh + i * nx + q : H + i * stride + c);
  }
  template <class NB2>
  __device__ __forceinline__ T hr2(int i, const NB2&, int) const { return hr(i); }
  __device__ __forceinline__ T h0() const { return T(sh0[x]); }
};

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256, 2) k_mp_rows(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0,
                                                    const P* __restrict__ phi, const Geom g,
                                                    const MpK<typename Stor<S>::T> k, const RowPlan rp,
                                                    int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);        // ns <= 4 barriers
  unsigned* s_rowok = reinterpret_cast<unsigned*>(smem + 64);  // per stage
  unsigned char* stage0 = smem + 128;
  const int nx = g.nx, tid = threadIdx.x;
  const int nct = gridDim.x, b = blockIdx.x;
  const int mine = b < rp.nrows ? (rp.nrows - b + nct - 1) / nct : 0;
  if (mine == 0) return;  // the whole CTA, before any barrier
  const int ns = rp.ns;
  constexpr bool R32 = Rest32<S>::on;
  const unsigned row_bytes = (unsigned)nx * sizeof(S);
  if (tid == 0) {
    for (int s = 0; s < ns; ++s) mkw::mbar_init(&bar[s], 1);
    mkw::fence_mbar_init();
  }
  __syncthreads();
  auto row_yz = [&](int kk, int& y, int& z) {
    const int r = b + kk * nct;
    y = rp.ylo + r % rp.nyf;
    z = rp.zlo + r / rp.nyf;
  };
  // warp 0: stage the source rows of this CTA's kk-th row into stage kk % ns,
  // lane i the two rows of direction i (lane 19 the FP32 rest row)
  auto issue = [&](int kk) {
    const int s = kk % ns, lane = tid & 31;
    int y, z;
    row_yz(kk, y, z);
    unsigned char* st = stage0 + (size_t)s * rp.stage;
    S* sg = reinterpret_cast<S*>(st);
    S* sh = sg + 19 * nx;
    const int64_t own = g.idx(0, y, z);
    mkw::fence_proxy_async_shared();  // the stage's earlier reads before the engine's writes
    if (lane == 0) {
      const unsigned bytes = (R32 ? 37u : 38u) * row_bytes + (R32 ? (unsigned)nx * 4u : 0u);
      mkw::mbar_arrive_expect(&bar[s], bytes);
    }
    __syncwarp();
    bool open = false;
    if (lane < 19) {
      const int i = lane;
      // element offset of the source row in the lattice arrays
      int64_t nb = own, off = (int64_t)i * g.stride + own;
      if (PARITY == 1 && g.nbr(rp.xf, y, z, 0, -ey(i), -ez(i), nb)) {
        open = true;
        off = (int64_t)inv(i) * g.stride + (nb - rp.xf);
      }
      mkw::bulk_g2s(sg + i * nx, G + off, row_bytes, &bar[s]);
      if (!R32 || i > 0) mkw::bulk_g2s(sh + i * nx, H + off, row_bytes, &bar[s]);
    } else if (R32 && lane == 19) {
      mkw::bulk_g2s(sh + 19 * nx, H0 + own, (unsigned)nx * 4u, &bar[s]);
    }
    const unsigned ok = __ballot_sync(0xffffffffu, open);  // bit i: direction i's row link is open
    if (lane == 0) s_rowok[s] = ok;
  };
  if (tid < 32)
    for (int kk = 0; kk < ns && kk < mine; ++kk) issue(kk);
  int kk = 0;
  for (; kk < mine; ++kk) {
    const int s = kk % ns;
    const bool landed = mkw::mbar_wait(&bar[s], (unsigned)((kk / ns) & 1), err);
    if (!__syncthreads_and(landed)) break;  // one decision for the CTA
    int y, z;
    row_yz(kk, y, z);
    const int x = tid;
    if (x < nx && x >= rp.xlo && x <= rp.xhi) {
      const S* sg = reinterpret_cast<const S*>(stage0 + (size_t)s * rp.stage);
      const S* sh = sg + 19 * nx;
      const float* sh0 = reinterpret_cast<const float*>(sh + 19 * nx);
      int xm = x - 1, xp = x + 1;
      if (rp.xper) {
        xm = x == 0 ? nx - 1 : xm;
        xp = x == nx - 1 ? 0 : xp;
      } else {
        xm = xm >= rp.xlo ? xm : -1;
        xp = xp <= rp.xhi ? xp : -1;
      }
      const unsigned rowok = s_rowok[s];
      if (fast_cell(g, x, y, z)) {
        const Fast fa = make_fast(g, x, y, z);
        mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Fast>{phi, fa, fa.c}, g.stride, fa, fa.c, k,
                                      RowLd<S, PARITY>{sg, sh, sh0, x, nx, rowok, xm, xp, G, H, g.stride, fa.c});
      } else {
        const Nbr nb(g, x, y, z);
        const int c = nb.idx(0, 0, 0);
        mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Nbr>{phi, nb, c}, g.stride, nb, c, k,
                                      RowLd<S, PARITY>{sg, sh, sh0, x, nx, rowok, xm, xp, G, H, g.stride, c});
      }
    }
    __syncthreads();  // every thread is done with stage s
    if (tid < 32 && kk + ns < mine) issue(kk + ns);
  }
  // a wait gave up: let the copies already issued land before the CTA exits
  if (kk < mine && tid == 0) {
    const int issued = kk + ns < mine ? kk + ns : mine;
    for (int q = kk; q < issued; ++q) mkw::mbar_wait(&bar[q % ns], (unsigned)((q / ns) & 1), err);
  }
}

// ------------------------------------------------- fused multiphase step
// One cooperative launch per loop.  Each CTA owns a tile column: a 32-cell x
// segment times a band of rows, marching through z.  For its own cells it
// computes phi = 1 + sum h' from exactly the slots the cell's collision reads
// later (in both AA parities every slot is read and written by one cell
// only), so computing phi ahead of the collision races with nothing.  A tile
// publishes phi `look` planes ahead of its collision plane (a release store of
// its count of finished planes), the bulk-copy engine stages the tile's phi
// rows plus a one-cell halo (one row of each neighbour band, four columns of
// each neighbour segment, periodic wrap resolved by the row addresses) into a
// four-plane shared-memory ring two planes ahead, and the collision reads its
// 19-point phi stencil from the ring.  h is read from HBM once per loop (the
// phi pass's read is reused from L2 by the collision `look` planes later), so
// the loop moves the compulsory 312 B/cell (FP32) instead of the 388 B/cell
// of the separate phi kernel.
//
// Publication order of the planes: 0, 1, ..., nz-1, or nz-1, 0, ..., nz-2 with
// a periodic z axis (the collision of plane 0 then needs plane nz-1 first).
// The prologue publishes the first `look` planes (look + 1 when periodic).
// Iteration z publishes the next one, stages sequence position z + 2 and
// collides plane z; a neighbour published the planes staged at iteration z
// one iteration earlier, so the waits are satisfied on arrival in steady
// state.  The grid never exceeds the co-resident capacity (cooperative
// launch), and every wait is bounded (mk_wave.cuh).
struct Wave {
  int sx, sy;        // x segments (32 cells) and y bands per segment: tile = band * sx + segment
  int look;          // planes published ahead of the collision plane (>= 3)
  int pz;            // 1: periodic z
  int pitch;         // ring row pitch in phi elements
  int rows_max;      // rows of the tallest band
  unsigned* flags;   // per tile: planes published in this launch (zeroed before every launch)
  int* err;          // error word (mkw::ERR_*), checked by the host
  int skip_tile;     // test hook: this tile never publishes (-1: none)
};

template <class P>
struct PhiRing {
  const P* lo;   // plane z - 1
  const P* mid;  // plane z
  const P* hi;   // plane z + 1
  int li, pitch;
  __device__ __forceinline__ P center() const { return mid[li]; }
  __device__ __forceinline__ P at(int dx, int dy, int dz) const {
    const P* s = dz < 0 ? lo : (dz > 0 ? hi : mid);
    return s[li + dy * pitch + dx];
  }
};

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(256, 2) k_mp_wave(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0,
                                                    P* __restrict__ phi, const Geom g,
                                                    const MpK<typename Stor<S>::T> k, const Wave w) {
  extern __shared__ __align__(128) unsigned char wave_smem[];
  __shared__ __align__(8) uint64_t bars[4];
  __shared__ int nbr_tile[8];
  P* const ring = reinterpret_cast<P*>(wave_smem);
  const int tile = blockIdx.x;
  const int seg = tile % w.sx, band = tile / w.sx;
  const int x0 = seg * 32;
  const int width = min(32, g.nx - x0);
  const int y0 = (int)((int64_t)band * g.ny / w.sy), y1 = (int)((int64_t)(band + 1) * g.ny / w.sy);
  const int rows = y1 - y0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int slot_elems = (w.rows_max + 2) * w.pitch;
  const int nz = g.nz;
  const bool publisher = tile != w.skip_tile;

  if (threadIdx.x < 8) {
    const int d = threadIdx.x < 4 ? threadIdx.x : threadIdx.x + 1;  // the 3 x 3 neighbourhood without its centre
    int ns = seg + d % 3 - 1, nb = band + d / 3 - 1;
    bool ok = true;
    if (ns < 0 || ns >= w.sx) {
      if (g.bc0 == 0)
        ns = (ns + w.sx) % w.sx;
      else
        ok = false;
    }
    if (nb < 0 || nb >= w.sy) {
      if (g.bc1 == 0)
        nb = (nb + w.sy) % w.sy;
      else
        ok = false;
    }
    nbr_tile[threadIdx.x] = ok ? nb * w.sx + ns : -1;
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < 4; ++s) mkw::mbar_init(&bars[s], 1);
    mkw::fence_mbar_init();
  }
  __syncthreads();

  const int P0 = w.look + w.pz;  // planes published by the prologue
  auto pub_plane = [&](int kk) { return w.pz ? (kk == 0 ? nz - 1 : kk - 1) : kk; };
  auto pub_index = [&](int q) { return w.pz ? (q == nz - 1 ? 0 : q + 1) : q; };

  // phi of this tile's fluid cells in plane p (the phi kernel's arithmetic)
  auto phi_plane = [&](int p) {
    for (int r = warp; r < rows; r += nwarps) {
      const int x = x0 + lane, y = y0 + r;
      if (lane < width && g.fluid(x, y, p)) {
        if (fast_cell(g, x, y, p)) {
          const Fast fa = make_fast(g, x, y, p);
          mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, fa, fa.c, k.ref_h);
        } else {
          const Nbr nb(g, x, y, p);
          mp_phi_cell<S, P, PARITY>(H, H0, phi, g.stride, nb, nb.idx(0, 0, 0), k.ref_h);
        }
      }
    }
  };
  // warp 0, lanes 0..7: wait until every neighbour tile has published `need` planes
  auto wait_neighbours = [&](unsigned need) {
    if (threadIdx.x < 8) {
      const int t = nbr_tile[threadIdx.x];
      if (t >= 0) mkw::wait_count(w.flags + t, need, w.err);
    }
  };
  // thread 0: stage sequence position q (-1 <= q <= nz) of phi into its ring slot
  auto stage = [&](int q) {
    const int slot = (q + 1) & 3;
    uint64_t* bar = &bars[slot];
    P* dst0 = ring + (size_t)slot * slot_elems;
    int plane = q;
    if (w.pz) plane = (q + nz) % nz;
    const bool have = plane >= 0 && plane < nz;
    // bytes first (one arrival announcing them), then the copies
    unsigned bytes = 0;
    const int xl = x0 - 4, xr = x0 + width + 4;  // [xl, xr) with the halo
    const int lo_mid = max(xl, 0), hi_mid = min(xr, g.nx);
    const bool wrap_l = xl < 0 && g.bc0 == 0, wrap_r = xr > g.nx && g.bc0 == 0;
    int nrows = 0;
    if (have)
      for (int lr = 0; lr < rows + 2; ++lr) {
        const int y = y0 - 1 + lr;
        if ((y < 0 || y >= g.ny) && g.bc1 != 0) continue;
        ++nrows;
      }
    if (have)
      bytes = (unsigned)(nrows * ((hi_mid - lo_mid) + (wrap_l ? 4 : 0) + (wrap_r ? 4 : 0)) * (int)sizeof(P));
    mkw::mbar_arrive_expect(bar, bytes);
    if (!have) return;
    const int64_t pbase = (int64_t)plane * g.nx * g.ny;
    for (int lr = 0; lr < rows + 2; ++lr) {
      int y = y0 - 1 + lr;
      if (y < 0 || y >= g.ny) {
        if (g.bc1 != 0) continue;
        y = (y + g.ny) % g.ny;
      }
      const P* src = phi + pbase + (int64_t)y * g.nx;
      P* dst = dst0 + (size_t)lr * w.pitch;
      mkw::bulk_g2s(dst + (lo_mid - xl), src + lo_mid, (unsigned)((hi_mid - lo_mid) * sizeof(P)), bar);
      if (wrap_l) mkw::bulk_g2s(dst, src + (g.nx - 4), (unsigned)(4 * sizeof(P)), bar);
      if (wrap_r) mkw::bulk_g2s(dst + 4 + width, src, (unsigned)(4 * sizeof(P)), bar);
    }
  };
  auto parity_of = [](int q) { return (unsigned)(((q + 1) >> 2) & 1); };
  auto slot_ptr = [&](int q) { return ring + (size_t)((q + 1) & 3) * slot_elems; };

  // ---- prologue: publish the first P0 planes, stage positions -1, 0, 1
  for (int kk = 0; kk < P0 && kk < nz; ++kk) phi_plane(pub_plane(kk));
  __syncthreads();
  if (threadIdx.x == 0 && publisher) mkw::st_release(w.flags + tile, (unsigned)min(P0, nz));
  wait_neighbours((unsigned)min(P0, nz));
  __syncthreads();
  if (threadIdx.x == 0) {
    mkw::fence_proxy_async_global();
    stage(-1);
    stage(0);
    stage(1);
  }
  mkw::mbar_wait(&bars[0], parity_of(-1), w.err);
  mkw::mbar_wait(&bars[1], parity_of(0), w.err);

  for (int z = 0; z < nz; ++z) {
    // neighbours' publication of the plane staged below (done one iteration ago)
    const int q2 = z + 2;
    const int plane2 = w.pz ? q2 % nz : q2;
    const bool staged2 = q2 <= nz && plane2 < nz;
    if (staged2) wait_neighbours((unsigned)(pub_index(plane2) + 1));
    // publish the next plane
    const int kk = P0 + z;
    const bool pub = kk < nz;
    if (pub) phi_plane(pub_plane(kk));
    __syncthreads();  // also: every thread is done with collision z - 1 (ring slot of position z - 2)
    if (threadIdx.x == 0) {
      // the release store after the CTA barrier orders every thread's phi
      // stores of the plane before the count (cumulativity of release)
      if (pub && publisher) mkw::st_release(w.flags + tile, (unsigned)(kk + 1));
      mkw::fence_proxy_async_global();
      mkw::fence_proxy_async_shared();
      if (q2 <= nz) stage(q2);
    }
    mkw::mbar_wait(&bars[(z + 2) & 3], parity_of(z + 1), w.err);
    // collision of plane z from the ring (positions z - 1, z, z + 1)
    const P* lo = slot_ptr(z - 1);
    const P* mid = slot_ptr(z);
    const P* hi = slot_ptr(z + 1);
    for (int r = warp; r < rows; r += nwarps) {
      const int x = x0 + lane, y = y0 + r;
      if (lane < width && g.fluid(x, y, z)) {
        const PhiRing<P> src{lo, mid, hi, (r + 1) * w.pitch + lane + 4, w.pitch};
        if (fast_cell(g, x, y, z)) {
          const Fast fa = make_fast(g, x, y, z);
          mp_collide_cell<S, P, PARITY>(G, H, H0, src, g.stride, fa, fa.c, k,
                                        GlobalLd<S, PARITY, Fast>{G, H, H0, g.stride, fa, fa.c});
        } else {
          const Nbr nb(g, x, y, z);
          const int c = nb.idx(0, 0, 0);
          mp_collide_cell<S, P, PARITY>(G, H, H0, src, g.stride, nb, c, k,
                                        GlobalLd<S, PARITY, Nbr>{G, H, H0, g.stride, nb, c});
        }
      }
    }
  }
  // the last staged position (nz + 1 is never staged; nz was waited above)
}

// The fused loop's tiling for this case (see k_mp_wave): 32-cell x segments
// times y bands, with as many bands as the co-resident capacity of the
// kernel allows, so every tile is one CTA and all CTAs are resident together.
template <class S>
void wave_config(mke::Engine& e) {
  typedef typename PhiOf<S>::type P;
  e.wave_ok = 0;
  if (e.p.model != MK_MODEL_MULTIPHASE || e.nx % 4 != 0 || e.nz < 8) return;
  int dev = e.device, sms = 0, coop = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (sms <= 0 || !coop) return;
  const int sx = (e.nx + 31) / 32;
  const int pitch = 40;
  // occupancy of the larger launch (256 threads, 16 rows), both parities
  size_t smem_max = (size_t)4 * (16 + 2) * pitch * sizeof(P);
  const void* kerns[2] = {(const void*)k_mp_wave<S, P, 0>, (const void*)k_mp_wave<S, P, 1>};
  int per_sm = 1 << 20;
  for (const void* kern : kerns) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 256, smem_max) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    per_sm = std::min(per_sm, b);
  }
  const int cap = per_sm * sms;
  if (per_sm < 1 || sx > cap) return;
  const int sy = std::min(e.ny, cap / sx);
  const int rows = (e.ny + sy - 1) / sy;
  if (rows > 16) return;
  e.wave_sx = sx;
  e.wave_sy = sy;
  e.wave_rows = rows;
  e.wave_threads = 32 * std::min(rows, 8);  // one warp per row
  e.wave_smem = (size_t)4 * (rows + 2) * pitch * sizeof(P);
  for (const void* kern : kerns)
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.wave_smem) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
  e.wave_ok = 1;
}

// Row-staged collision: eligibility, rows in flight and grid for the case.
template <class S>
void rows_config(mke::Engine& e) {
  typedef typename PhiOf<S>::type P;
  e.rows_ok = 0;
  const int nx = e.nx;
  if (e.p.model != MK_MODEL_MULTIPHASE || nx > 256 || ((size_t)nx * sizeof(S)) % 16 != 0 || nx < 3) return;
  const bool r32 = Rest32<S>::on;
  size_t stage = (size_t)38 * nx * sizeof(S) + (r32 ? (size_t)nx * 4 : 0);
  stage = (stage + 127) / 128 * 128;
  const int threads = (nx + 31) / 32 * 32;
  int dev = e.device, sms = 0, smem_sm = 0, smem_blk = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (sms <= 0) return;
  const void* kerns[2] = {(const void*)k_mp_rows<S, P, 0>, (const void*)k_mp_rows<S, P, 1>};
  // CTAs per SM the registers allow, then as many rows in flight (2..4) as
  // that many CTAs' shared memory holds
  int per_sm = 1 << 20;
  for (const void* kern : kerns) {
    int bsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bsm, kern, threads, 0) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    per_sm = std::min(per_sm, bsm);
  }
  if (per_sm < 1) return;
  int ns = 0, cta = per_sm;
  for (; cta >= 1 && ns < 2; --cta) {
    const size_t budget = std::min<size_t>((size_t)smem_sm / cta - 1024, (size_t)smem_blk);
    ns = (int)std::min<size_t>(4, (budget - 128) / stage);
    if (ns >= 2) break;
  }
  if (ns < 2) return;
  const size_t smem = 128 + (size_t)ns * stage;
  for (const void* kern : kerns)
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
  int resident = 1 << 20;
  for (const void* kern : kerns) {
    int bsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bsm, kern, threads, smem) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    resident = std::min(resident, bsm);
  }
  if (resident < 1) return;
  e.rows_ns = ns;
  e.rows_stage = stage;
  e.rows_smem = smem;
  e.rows_threads = threads;
  e.rows_grid = resident * sms;
  e.rows_ok = 1;
}

// The fluid rows of the case as the row-staged kernel enumerates them (the
// spans Geom::fluid gives: walls drop the end cells of an axis, a slab its
// ghost planes and any global wall plane it holds).
inline RowPlan row_plan(const mke::Engine& e, const Geom& g) {
  auto span = [](int n, int bc, int& lo, int& hi) {
    lo = bc == MK_BC_WALLS ? 1 : 0;
    hi = bc == MK_BC_WALLS ? n - 2 : n - 1;
  };
  RowPlan rp;
  span(g.nx, g.bc0, rp.xlo, rp.xhi);
  int yhi = 0, zlo = 0, zhi = 0;
  span(g.ny, g.bc1, rp.ylo, yhi);
  if (g.slab) {
    zlo = 1;
    zhi = g.nz - 2;
    if (g.bc2 == MK_BC_WALLS) {
      if (g.zg0 == 0) zlo = 2;
      if (g.zg0 + g.nz - 3 == g.nzg - 1) zhi = g.nz - 3;
    }
  } else {
    span(g.nz, g.bc2, zlo, zhi);
  }
  rp.nyf = std::max(0, yhi - rp.ylo + 1);
  rp.zlo = zlo;
  rp.nrows = rp.nyf * std::max(0, zhi - zlo + 1);
  rp.xper = g.bc0 == MK_BC_PERIODIC;
  rp.xf = rp.xlo;
  rp.ns = e.rows_ns;
  rp.stage = (int)e.rows_stage;
  return rp;
}

// ------------------------------------------- TMA-staged phi tile (phi_tile)
// The two-kernel loop's collision with the phi stencil read from shared
// memory: one 3-D TMA tensor load per block stages the block's phi tile and
// its one-cell halo (x rounded out to 16 bytes, y +-1, z +-1) for a 64 x 4
// block in one plane.  Interior cells (the Fast path, no periodic wrap along
// x) read their 19 phi values from the tile; every other cell reads global
// memory as in k_mp_collide.  The values are the same, so the result is
// bit-identical.  The tensor map covers this GPU's own phi buffer; no
// multicast.
constexpr int kTileX = 64, kTileY = 4, kTileHX = 4;
constexpr int kTileW = kTileX + 2 * kTileHX, kTileH = kTileY + 2;

// The stencil's first access (center) waits for the tile, so the cell's
// population loads, issued before it, overlap the tile's transfer; a wait
// that gives up (recorded in *err) falls back to global memory.
template <class P>
struct PhiTile {
  const P* t;
  uint64_t* bar;
  int* err;
  const P* phi;  // global phi, the fallback
  const Fast& fa;
  int lx, ly;  // the cell's column and row in the tile
  mutable bool tile_ok;
  __device__ __forceinline__ P center() const {
    tile_ok = mkw::mbar_wait(bar, 0, err);
    return tile_ok ? t[(kTileH + ly) * kTileW + lx] : phi[fa.c];
  }
  __device__ __forceinline__ P at(int dx, int dy, int dz) const {
    return tile_ok ? t[((1 + dz) * kTileH + ly + dy) * kTileW + lx + dx] : __ldg(phi + fa.idx(dx, dy, dz));
  }
};

template <class S, class P, int PARITY>
__global__ void __launch_bounds__(kTileX* kTileY, 2)
    k_mp_collide_tma(S* __restrict__ G, S* __restrict__ H, float* __restrict__ H0, const P* __restrict__ phi,
                     const Geom g, const MpK<typename Stor<S>::T> k, const __grid_constant__ CUtensorMap tmap,
                     int* err) {
  __shared__ alignas(128) P tile[3 * kTileH * kTileW];
  __shared__ alignas(8) uint64_t bar;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY, z = blockIdx.z;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  if (lead) {
    mkw::mbar_init(&bar, 1);
    mkw::fence_mbar_init();
  }
  __syncthreads();
  if (lead) {
    mkw::mbar_arrive_expect(&bar, (unsigned)sizeof(tile));
    mkw::tma_load_3d(tile, &tmap, x0 - kTileHX, y0 - 1, z - 1, &bar);
  }
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x < g.nx && y < g.ny && g.fluid(x, y, z)) {
    if (fast_cell(g, x, y, z)) {
      const Fast fa = make_fast(g, x, y, z);
      if (x >= 1 && x <= g.nx - 2)
        mp_collide_cell<S, P, PARITY>(
            G, H, H0, PhiTile<P>{tile, &bar, err, phi, fa, (int)threadIdx.x + kTileHX, (int)threadIdx.y + 1, false},
            g.stride, fa, fa.c, k, GlobalLd<S, PARITY, Fast>{G, H, H0, g.stride, fa, fa.c});
      else
        mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Fast>{phi, fa, fa.c}, g.stride, fa, fa.c, k,
                                      GlobalLd<S, PARITY, Fast>{G, H, H0, g.stride, fa, fa.c});
    } else {
      const Nbr nb(g, x, y, z);
      const int c = nb.idx(0, 0, 0);
      mp_collide_cell<S, P, PARITY>(G, H, H0, PhiGlobal<P, Nbr>{phi, nb, c}, g.stride, nb, c, k,
                                    GlobalLd<S, PARITY, Nbr>{G, H, H0, g.stride, nb, c});
    }
  }
  // the block's shared memory must outlive the tile's transfer, whether or
  // not any of its cells read the tile (bounded)
  if (lead) mkw::mbar_wait(&bar, 0, err);
}

// The tensor map over phi (nx x ny x nz, x fastest): admitted when the row
// stride is a multiple of 16 bytes (nx a multiple of 4) and the driver
// encodes the map; slabs are not admitted.
template <class P>
void tma_config(mke::Engine& e) {
  e.tma_ok = 0;
  e.tma = 0;
  if (e.slab || e.nx % 4 != 0 || e.nx < 4) return;
  typedef CUresult (*Encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode encode = []() -> Encode {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return (Encode)fn;
  }();
  if (!encode) return;
  const cuuint64_t dims[3] = {(cuuint64_t)e.nx, (cuuint64_t)e.ny, (cuuint64_t)e.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)e.nx * sizeof(P), (cuuint64_t)e.nx * e.ny * sizeof(P)};
  const cuuint32_t box[3] = {(cuuint32_t)kTileW, (cuuint32_t)kTileH, 3u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r =
      encode(reinterpret_cast<CUtensorMap*>(e.tma_map),
             sizeof(P) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, e.phi[0], dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  e.tma_ok = r == CUDA_SUCCESS ? 1 : 0;
}

template <class S>
void launch_mp_tma(mke::Engine& e, int parity, const Geom& g, const MpK<typename Stor<S>::T>& k) {
  typedef typename PhiOf<S>::type P;
  const dim3 grid((e.nx + kTileX - 1) / kTileX, (e.ny + kTileY - 1) / kTileY, e.nz), block(kTileX, kTileY);
  const CUtensorMap& m = *reinterpret_cast<const CUtensorMap*>(e.tma_map);
  S* G = (S*)e.pop0;
  S* H = (S*)e.pop1;
  const P* phi = (const P*)e.phi[0];
  if (parity == 0)
    k_mp_collide_tma<S, P, 0><<<grid, block, 0, e.stream>>>(G, H, e.rest1, phi, g, k, m, e.wave_err);
  else
    k_mp_collide_tma<S, P, 1><<<grid, block, 0, e.stream>>>(G, H, e.rest1, phi, g, k, m, e.wave_err);
}

template <class S>
void launch_mp_rows(mke::Engine& e, int parity, const Geom& g, const MpK<typename Stor<S>::T>& k) {
  typedef typename PhiOf<S>::type P;
  const RowPlan rp = row_plan(e, g);
  if (rp.nrows == 0 || rp.xhi < rp.xlo) return;
  S* G = (S*)e.pop0;
  S* H = (S*)e.pop1;
  const P* phi = (const P*)e.phi[0];
  const int grid = std::min(e.rows_grid, rp.nrows);
  if (parity == 0)
    k_mp_rows<S, P, 0><<<grid, e.rows_threads, e.rows_smem, e.stream>>>(G, H, e.rest1, phi, g, k, rp, e.wave_err);
  else
    k_mp_rows<S, P, 1><<<grid, e.rows_threads, e.rows_smem, e.stream>>>(G, H, e.rest1, phi, g, k, rp, e.wave_err);
}

template <class S>
void launch_mp_wave(mke::Engine& e, int parity, cudaEvent_t* ev) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  const Geom g = make_geom(e);
  const MpK<T> k = mp_coef<T>(e.p, refs_of(e.p));
  Wave w;
  w.sx = e.wave_sx;
  w.sy = e.wave_sy;
  w.look = 3;  // >= 3: a tile publishes before it waits within an iteration
  w.pz = e.p.bc[2] == MK_BC_PERIODIC ? 1 : 0;
  w.pitch = 40;
  w.rows_max = e.wave_rows;
  w.flags = e.wave_flags;
  w.err = e.wave_err;
  w.skip_tile = e.wave_skip;
  e.wave_skip = -1;
  const int tiles = w.sx * w.sy;
  if (ev) cudaEventRecord(ev[0], e.stream);
  cudaMemsetAsync(e.wave_flags, 0, (size_t)tiles * sizeof(unsigned), e.stream);
  S* G = (S*)e.pop0;
  S* H = (S*)e.pop1;
  float* H0 = e.rest1;
  P* phi = (P*)e.phi[0];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles);
  cfg.blockDim = dim3(e.wave_threads);
  cfg.dynamicSmemBytes = e.wave_smem;
  cfg.stream = e.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (parity == 0)
    cudaLaunchKernelEx(&cfg, k_mp_wave<S, P, 0>, G, H, H0, phi, g, k, w);
  else
    cudaLaunchKernelEx(&cfg, k_mp_wave<S, P, 1>, G, H, H0, phi, g, k, w);
  if (ev) cudaEventRecord(ev[1], e.stream);
}

// The phi kernel over planes z_lo .. z_lo + nzr - 1 on `st`.
template <class S>
void launch_phi_range(mke::Engine& e, int parity, dim3 grid, dim3 block, int z_lo, int nzr, cudaStream_t st) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  if (nzr <= 0) return;
  const Geom g = make_geom(e);
  const Refs r = refs_of(e.p);
  grid.z = nzr;
  S* H = (S*)e.pop1;
  P* phi = (P*)e.phi[0];
  if constexpr (Stor<S>::bytes == 2) {
    if (e.nx % 2 == 0) {  // two cells per thread
      dim3 g2 = grid;
      g2.x = (unsigned)((e.nx / 2 + block.x - 1) / block.x);
      if (parity == 0)
        k_mp_phi2<S, P, 0><<<g2, block, 0, st>>>(H, e.rest1, phi, g, T(r.r1), z_lo);
      else
        k_mp_phi2<S, P, 1><<<g2, block, 0, st>>>(H, e.rest1, phi, g, T(r.r1), z_lo);
      return;
    }
  }
  if (parity == 0)
    k_mp_phi<S, P, 0><<<grid, block, 0, st>>>(H, e.rest1, phi, g, T(r.r1), z_lo);
  else
    k_mp_phi<S, P, 1><<<grid, block, 0, st>>>(H, e.rest1, phi, g, T(r.r1), z_lo);
}

// The thread-per-cell collision over planes z_lo .. z_lo + nzr - 1 on `st`,
// in the occupancy variant e.minb.
template <class S>
void launch_collide_range(mke::Engine& e, int parity, dim3 grid, dim3 block, int z_lo, int nzr, cudaStream_t st) {
  typedef typename Stor<S>::T T;
  typedef typename PhiOf<S>::type P;
  if (nzr <= 0) return;
  const Geom g = make_geom(e);
  const MpK<T> k = mp_coef<T>(e.p, refs_of(e.p));
  grid.z = nzr;
  S* G = (S*)e.pop0;
  S* H = (S*)e.pop1;
  const P* phi = (const P*)e.phi[0];
  if (e.minb == 1) {
    if (parity == 0)
      k_mp_collide<S, P, 0, 1><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
    else
      k_mp_collide<S, P, 1, 1><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
  } else if (e.minb >= 3 && e.minb <= 5) {
    // register-capped variants
    auto go = [&](auto rr) {
      constexpr int R = decltype(rr)::value;
      if (parity == 0)
        k_mp_collide_r<S, P, 0, R><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
      else
        k_mp_collide_r<S, P, 1, R><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
    };
    if (e.minb == 3)
      go(std::integral_constant<int, 112>{});
    else if (e.minb == 4)
      go(std::integral_constant<int, 96>{});
    else
      go(std::integral_constant<int, 80>{});
  } else {
    if (parity == 0)
      k_mp_collide<S, P, 0, 2><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
    else
      k_mp_collide<S, P, 1, 2><<<grid, block, 0, st>>>(G, H, e.rest1, phi, g, k, z_lo);
  }
}

// parts: bit 0 the phi kernel, bit 1 the collision (3: the whole loop)
template <class S>
void launch_mp(mke::Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev, int parts = 3) {
  typedef typename Stor<S>::T T;
  if (parts == 3 && e.wave && e.wave_ok) {
    launch_mp_wave<S>(e, parity, ev);
    return;
  }
  if (ev) cudaEventRecord(ev[0], e.stream);
  if (parts & 1) launch_phi_range<S>(e, parity, grid, block, 0, e.nz, e.stream);
  if (ev) {
    cudaEventRecord(ev[1], e.stream);
    cudaEventRecord(ev[2], e.stream);
  }
  if (!(parts & 2)) {
    if (ev) cudaEventRecord(ev[3], e.stream);
    return;
  }
  if (e.rows && e.rows_ok) {
    const Geom g = make_geom(e);
    launch_mp_rows<S>(e, parity, g, mp_coef<T>(e.p, refs_of(e.p)));
  } else if (e.tma && e.tma_ok) {
    const Geom g = make_geom(e);
    launch_mp_tma<S>(e, parity, g, mp_coef<T>(e.p, refs_of(e.p)));
  } else {
    launch_collide_range<S>(e, parity, grid, block, 0, e.nz, e.stream);
  }
  if (ev) cudaEventRecord(ev[3], e.stream);
}

// Dynamic solids: pending |= (a fluid cell of the static geometry with the
// dendrite's phi > 0).
template <class P>
__global__ void k_solid_from_phi(const P* __restrict__ dphi, const Geom g, unsigned char* __restrict__ pending,
                                 int64_t n) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % g.nx), y = (int)((c / g.nx) % g.ny), z = (int)(c / ((int64_t)g.nx * g.ny));
    if (g.fluid(x, y, z) && double(dphi[c]) > 0.0) pending[c] = 1;
  }
}

// near = a fluid cell with a D3Q19 neighbour that is solid (g carries the
// static geometry; `solid` the new flags).
__global__ void k_near_solid(const Geom g, const unsigned char* __restrict__ solid, unsigned char* __restrict__ near,
                             int64_t n) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % g.nx), y = (int)((c / g.nx) % g.ny), z = (int)(c / ((int64_t)g.nx * g.ny));
    unsigned char v = 0;
    if (!solid[c] && g.fluid(x, y, z)) {
#pragma unroll
      for (int i = 1; i < 19; ++i) {
        int64_t j;
        if (g.nbr(x, y, z, ex(i), ey(i), ez(i), j) && solid[j]) v = 1;
      }
    }
    near[c] = v;
  }
}

// Re-streams the links that the cells turning solid close.  At an even loop
// count the in-place layout holds each fluid cell's streamed (pre-collision)
// populations in its own slots, streamed with the geometry of the last loop:
// slot i of a cell c whose upwind neighbour c - e_i turns solid now holds
// that neighbour's outgoing population.  With the new geometry that link
// bounces back: it must hold c's own outgoing population in direction
// inv(i), which the last odd loop wrote into the neighbour's slot inv(i)
// (the link was open then).  The new solids' slots are only read and the
// fluid cells' only written, so the copy is race-free; a raw element copy is
// exact in every storage format (w_i = w_inv(i)).  `g` carries the solids
// of the last loop, `pending` the new set (a superset).
template <class W>
__global__ void k_solid_restream(W* __restrict__ G, W* __restrict__ H, const Geom g,
                                 const unsigned char* __restrict__ pending, int64_t n) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % g.nx), y = (int)((c / g.nx) % g.ny), z = (int)(c / ((int64_t)g.nx * g.ny));
    if (pending[c] || !g.fluid(x, y, z)) continue;
#pragma unroll
    for (int i = 1; i < 19; ++i) {
      int64_t j;
      if (g.nbr(x, y, z, -ex(i), -ey(i), -ez(i), j) && pending[j]) {
        G[(int64_t)i * g.stride + c] = G[(int64_t)inv(i) * g.stride + j];
        H[(int64_t)i * g.stride + c] = H[(int64_t)inv(i) * g.stride + j];
      }
    }
  }
}

}  // namespace

namespace mke {

cudaError_t mp_solid_from_phi(Engine& e, const void* dend_phi, int phi_double) {
  if (e.p.model != MK_MODEL_MULTIPHASE || e.slab) return cudaErrorInvalidValue;
  const size_t n = (size_t)e.ncell;
  cudaError_t st = cudaSuccess;
  for (unsigned char** a : {&e.msolid, &e.mnear, &e.mpending})
    if (!*a) {
      if ((st = cudaMalloc((void**)a, n)) != cudaSuccess) return st;
      if ((st = cudaMemsetAsync(*a, 0, n, e.stream)) != cudaSuccess) return st;
    }
  Geom g = make_geom(e);
  g.solid = nullptr;  // the static geometry
  g.near = nullptr;
  const int blocks = (int)std::min<int64_t>((e.ncell + 255) / 256, 4096);
  if (phi_double)
    k_solid_from_phi<double><<<blocks, 256, 0, e.stream>>>((const double*)dend_phi, g, e.mpending, e.ncell);
  else
    k_solid_from_phi<float><<<blocks, 256, 0, e.stream>>>((const float*)dend_phi, g, e.mpending, e.ncell);
  if ((st = cudaGetLastError()) != cudaSuccess) return st;
  e.mpending_set = 1;
  // the staged and fused forms assume a static geometry
  e.wave = e.wave_ok = 0;
  e.rows = e.rows_ok = 0;
  return mp_apply_solids(e);
}

cudaError_t mp_apply_solids(Engine& e) {
  if (!e.mpending_set || (e.step & 1)) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((e.ncell + 255) / 256, 4096);
  Geom g = make_geom(e);  // the solids of the last loop
  g.near = nullptr;
  switch (pop_elem(e.p.precision)) {
    case 8:
      k_solid_restream<uint64_t><<<blocks, 256, 0, e.stream>>>((uint64_t*)e.pop0, (uint64_t*)e.pop1, g, e.mpending,
                                                               e.ncell);
      break;
    case 4:
      k_solid_restream<uint32_t><<<blocks, 256, 0, e.stream>>>((uint32_t*)e.pop0, (uint32_t*)e.pop1, g, e.mpending,
                                                               e.ncell);
      break;
    default:
      k_solid_restream<uint16_t><<<blocks, 256, 0, e.stream>>>((uint16_t*)e.pop0, (uint16_t*)e.pop1, g, e.mpending,
                                                               e.ncell);
      break;
  }
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) return st;
  if ((st = cudaMemcpyAsync(e.msolid, e.mpending, (size_t)e.ncell, cudaMemcpyDeviceToDevice, e.stream)) !=
      cudaSuccess)
    return st;
  g.solid = nullptr;
  k_near_solid<<<blocks, 256, 0, e.stream>>>(g, e.msolid, e.mnear, e.ncell);
  e.mpending_set = 0;
  return cudaGetLastError();
}

void mp_configure(Engine& e) {
  switch (e.p.precision) {
    case MK_PREC_FP64:
      wave_config<double>(e);
      rows_config<double>(e);
      tma_config<double>(e);
      break;
    case MK_PREC_FP32:
      wave_config<float>(e);
      rows_config<float>(e);
      tma_config<float>(e);
      break;
    case MK_PREC_FP16:
      wave_config<__half>(e);
      rows_config<__half>(e);
      tma_config<float>(e);
      break;
    default:
      wave_config<__nv_bfloat16>(e);
      rows_config<__nv_bfloat16>(e);
      tma_config<float>(e);
      break;
  }
}

void mp_launch(Engine& e, int parity, dim3 grid, dim3 block, cudaEvent_t* ev) {
  switch (e.p.precision) {
    case MK_PREC_FP64:
      launch_mp<double>(e, parity, grid, block, ev);
      break;
    case MK_PREC_FP32:
      launch_mp<float>(e, parity, grid, block, ev);
      break;
    case MK_PREC_FP16:
      launch_mp<__half>(e, parity, grid, block, ev);
      break;
    default:
      launch_mp<__nv_bfloat16>(e, parity, grid, block, ev);
      break;
  }
}

cudaError_t mp_launch_part(Engine& e, int part) {
  if (part != 0 && part != 1) return cudaErrorInvalidValue;
  dim3 grid, block;
  launch_dims(e, grid, block);
  const int parity = (int)(e.step & 1);
  const int parts = part == 0 ? 1 : 2;
  switch (e.p.precision) {
    case MK_PREC_FP64:
      launch_mp<double>(e, parity, grid, block, nullptr, parts);
      break;
    case MK_PREC_FP32:
      launch_mp<float>(e, parity, grid, block, nullptr, parts);
      break;
    case MK_PREC_FP16:
      launch_mp<__half>(e, parity, grid, block, nullptr, parts);
      break;
    default:
      launch_mp<__nv_bfloat16>(e, parity, grid, block, nullptr, parts);
      break;
  }
  e.launches += 1;
  if (part == 1) e.step += 1;
  return cudaGetLastError();
}

}  // namespace mke
