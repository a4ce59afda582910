// mk_device.cuh — lattice tables, storage traits and geometry shared by the
// sm_100a kernels.
//
// Memory layout in HBM: structure of arrays, one plane per population,
// A[q * stride + cell] with cell = x + nx (y + ny z) and stride rounded up to
// a multiple of 64 cells, so every population plane starts 256-byte aligned.
// Streaming is in place with the AA pattern (Bailey et al. 2009): an even
// loop reads and writes only the cell's own slots (A[i][c] in, A[inv i][c]
// out); an odd loop reads A[inv i][c - e_i] and writes A[i][c + e_i].  Each
// population is therefore read once and written once per loop, and no second
// population array exists.  Half-way bounce-back (MaterKit/src/mkFluidsUser.cpp:
// 77-97 streams with bounce-back in the same sweep) folds into the odd loop's
// addressing: a link to a non-fluid neighbour reads/writes the cell's own
// opposite slot instead.
#ifndef MK_DEVICE_CUH
#define MK_DEVICE_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <utility>

namespace mkd {

// ------------------------------------------------------------- lattices
// Direction order identical to the oracle and the public header docs:
// rest, +-x, +-y, +-z, xy/xz/yz edges, 8 corners; opposite directions adjacent.
__host__ __device__ constexpr int ex(int i) {
  constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
  return t[i];
}
__host__ __device__ constexpr int ey(int i) {
  constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
  return t[i];
}
__host__ __device__ constexpr int ez(int i) {
  constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
  return t[i];
}
__host__ __device__ constexpr int inv(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

template <int Q>
__host__ __device__ constexpr double wq(int i) {
  return Q == 7 ? (i == 0 ? 0.25 : 0.125)
                : (Q == 19 ? (i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0))
                           : (i == 0 ? 8.0 / 27.0 : (i <= 6 ? 2.0 / 27.0 : (i <= 18 ? 1.0 / 54.0 : 1.0 / 216.0))));
}

// d'Humieres 2002 D3Q19 moment matrix entry M[k][i] (integer valued).
__host__ __device__ constexpr int mrt_m(int k, int i) {
  const int x = ex(i), y = ey(i), z = ez(i);
  const int e2 = x * x + y * y + z * z;
  switch (k) {
    case 0: return 1;
    case 1: return 19 * e2 - 30;
    case 2: return (21 * e2 * e2 - 53 * e2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * e2 - 9) * x;
    case 5: return y;
    case 6: return (5 * e2 - 9) * y;
    case 7: return z;
    case 8: return (5 * e2 - 9) * z;
    case 9: return 3 * x * x - e2;
    case 10: return (3 * e2 - 5) * (3 * x * x - e2);
    case 11: return y * y - z * z;
    case 12: return (3 * e2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    default: return (x * x - y * y) * z;
  }
}
__host__ __device__ constexpr int mrt_norm(int k) {
  int s = 0;
  for (int i = 0; i < 19; ++i) s += mrt_m(k, i) * mrt_m(k, i);
  return s;
}
// Fixed rates; the shear rows (9, 11, 13, 14, 15) take the runtime rate.
__host__ __device__ constexpr double mrt_rate(int k) {
  return k == 1 ? 1.19 : (k == 2 ? 1.4 : ((k == 4 || k == 6 || k == 8) ? 1.2 : ((k == 10 || k == 12) ? 1.4 : (k >= 16 ? 1.98 : 1.0))));
}
__host__ __device__ constexpr bool mrt_is_shear(int k) { return k == 9 || k == 11 || k == 13 || k == 14 || k == 15; }

// ---- moment-space MRT with analytic equilibria -------------------------
// For an equilibrium  f_eq,i = w_i [a0 + 3 e_i.b + 4.5 (e_i e_i):Q]  and a
// Guo force term  F_i = s_F w_i [3 e_i.F + 9 (e_i.u)(e_i.F) - 3 u.F]  the
// moments M f_eq and M F are linear in (a0, b, Q) and (F, u F) with the
// integer tables below (weights scaled by 36).  Everything is evaluated at
// compile time, so one collision costs the pair-split transform M f, 19
// relaxations and the pair-split back-transform.
__host__ __device__ constexpr int w36(int i) { return i == 0 ? 12 : (i <= 6 ? 2 : 1); }
__host__ __device__ constexpr int mrt_a36(int k) {
  int s = 0;
  for (int i = 0; i < 19; ++i) s += mrt_m(k, i) * w36(i);
  return s;
}
__host__ __device__ constexpr int mrt_b36(int k, int a) {
  int s = 0;
  for (int i = 0; i < 19; ++i) s += mrt_m(k, i) * w36(i) * (a == 0 ? ex(i) : (a == 1 ? ey(i) : ez(i)));
  return s;
}
__host__ __device__ constexpr int mrt_c36(int k, int a, int b) {
  int s = 0;
  for (int i = 0; i < 19; ++i)
    s += mrt_m(k, i) * w36(i) * (a == 0 ? ex(i) : (a == 1 ? ey(i) : ez(i))) *
         (b == 0 ? ex(i) : (b == 1 ? ey(i) : ez(i)));
  return s;
}
__host__ __device__ constexpr bool mrt_even(int k) { return k <= 2 || (k >= 9 && k <= 15); }

template <int K>
struct MrtRow {
  static constexpr int a = mrt_a36(K);
  static constexpr int bx = mrt_b36(K, 0), by = mrt_b36(K, 1), bz = mrt_b36(K, 2);
  static constexpr int cxx = mrt_c36(K, 0, 0), cyy = mrt_c36(K, 1, 1), czz = mrt_c36(K, 2, 2);
  static constexpr int cxy = mrt_c36(K, 0, 1), cxz = mrt_c36(K, 0, 2), cyz = mrt_c36(K, 1, 2);
  static constexpr int norm = mrt_norm(K);
};

template <class T>
struct MrtIn {
  T a0, bx, by, bz;                 // equilibrium: a0 and the vector b
  T qxx, qyy, qzz, qxy, qxz, qyz;   // equilibrium: symmetric tensor Q (full off-diagonal value)
  T Fx, Fy, Fz, ux, uy, uz, sF;     // force, velocity of the force term, scale
  T s_nu;                           // shear rate
};

// d_K = (s_K (m_K - meq_K) - (1 - s_K/2) mF_K) / |M_K|^2
template <class T, int K>
__host__ __device__ __forceinline__ T mrt_relax(T mk, const MrtIn<T>& q) {
  typedef MrtRow<K> R;
  constexpr double c = 1.0 / 36.0;
  T meq = T(0), mf = T(0);
  if constexpr (R::a != 0) meq += T(R::a * c) * q.a0;
  if constexpr (R::bx != 0) meq += T(3.0 * R::bx * c) * q.bx;
  if constexpr (R::by != 0) meq += T(3.0 * R::by * c) * q.by;
  if constexpr (R::bz != 0) meq += T(3.0 * R::bz * c) * q.bz;
  if constexpr (R::cxx != 0) meq += T(4.5 * R::cxx * c) * q.qxx;
  if constexpr (R::cyy != 0) meq += T(4.5 * R::cyy * c) * q.qyy;
  if constexpr (R::czz != 0) meq += T(4.5 * R::czz * c) * q.qzz;
  if constexpr (R::cxy != 0) meq += T(9.0 * R::cxy * c) * q.qxy;
  if constexpr (R::cxz != 0) meq += T(9.0 * R::cxz * c) * q.qxz;
  if constexpr (R::cyz != 0) meq += T(9.0 * R::cyz * c) * q.qyz;
  // force moments: 3 B.F + 9 u.C.F - 3 A u.F
  if constexpr (R::bx != 0) mf += T(3.0 * R::bx * c) * q.Fx;
  if constexpr (R::by != 0) mf += T(3.0 * R::by * c) * q.Fy;
  if constexpr (R::bz != 0) mf += T(3.0 * R::bz * c) * q.Fz;
  if constexpr (R::cxx != 0) mf += T(9.0 * R::cxx * c) * (q.ux * q.Fx);
  if constexpr (R::cyy != 0) mf += T(9.0 * R::cyy * c) * (q.uy * q.Fy);
  if constexpr (R::czz != 0) mf += T(9.0 * R::czz * c) * (q.uz * q.Fz);
  if constexpr (R::cxy != 0) mf += T(9.0 * R::cxy * c) * (q.ux * q.Fy + q.uy * q.Fx);
  if constexpr (R::cxz != 0) mf += T(9.0 * R::cxz * c) * (q.ux * q.Fz + q.uz * q.Fx);
  if constexpr (R::cyz != 0) mf += T(9.0 * R::cyz * c) * (q.uy * q.Fz + q.uz * q.Fy);
  if constexpr (R::a != 0) mf -= T(3.0 * R::a * c) * (q.ux * q.Fx + q.uy * q.Fy + q.uz * q.Fz);
  const T s = mrt_is_shear(K) ? q.s_nu : T(mrt_rate(K));
  return (s * (mk - meq) - (T(1) - T(0.5) * s) * (q.sF * mf)) * T(1.0 / R::norm);
}

template <class T, int... Ks>
__host__ __device__ __forceinline__ void mrt_relax_all(const T (&m)[19], T (&d)[19], const MrtIn<T>& q,
                                              std::integer_sequence<int, Ks...>) {
  ((d[Ks] = mrt_relax<T, Ks>(m[Ks], q)), ...);
}

// In-place D3Q19 MRT collision in moment space (pair-split transforms).
template <class T>
__host__ __device__ __forceinline__ void mrt19_collide_moments(T (&f)[19], const MrtIn<T>& q) {
  T s[10], a[10];
  s[0] = f[0];
  a[0] = T(0);
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    s[p] = f[2 * p - 1] + f[2 * p];
    a[p] = f[2 * p - 1] - f[2 * p];
  }
  T m[19];
#pragma unroll
  for (int k = 0; k < 19; ++k) {
    T acc = T(0);
    if (mrt_even(k)) {
      if (mrt_m(k, 0) != 0) acc += T(mrt_m(k, 0)) * s[0];
#pragma unroll
      for (int p = 1; p <= 9; ++p)
        if (mrt_m(k, 2 * p - 1) != 0) acc += T(mrt_m(k, 2 * p - 1)) * s[p];
    } else {
#pragma unroll
      for (int p = 1; p <= 9; ++p)
        if (mrt_m(k, 2 * p - 1) != 0) acc += T(mrt_m(k, 2 * p - 1)) * a[p];
    }
    m[k] = acc;
  }
  T d[19];
  mrt_relax_all<T>(m, d, q, std::make_integer_sequence<int, 19>{});
  T d0 = T(0);
#pragma unroll
  for (int k = 0; k < 19; ++k)
    if (mrt_even(k) && mrt_m(k, 0) != 0) d0 += T(mrt_m(k, 0)) * d[k];
  f[0] -= d0;
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    T E = T(0), O = T(0);
#pragma unroll
    for (int k = 0; k < 19; ++k) {
      if (mrt_m(k, 2 * p - 1) == 0) continue;
      if (mrt_even(k))
        E += T(mrt_m(k, 2 * p - 1)) * d[k];
      else
        O += T(mrt_m(k, 2 * p - 1)) * d[k];
    }
    f[2 * p - 1] -= E + O;
    f[2 * p] -= E - O;
  }
}

// The same collision with the two transforms written out in the pair-split
// basis, sharing partial sums (face sum, edge sum, the x/y/z edge fluxes), so
// the forward transform is ~45 additions and the back transform ~60.  Pairs:
// p = 1..3 the +-x, +-y, +-z faces; p = 4..9 the xy(+,+), xy(+,-), xz(+,+),
// xz(+,-), yz(+,+), yz(+,-) edges (direction 2p-1, opposite 2p).
// The 19 moments m = M f of the d'Humieres basis by pair-split sums (m[0]
// is sum f, m[3], m[5], m[7] the three momentum components).
template <class T>
__host__ __device__ __forceinline__ void mrt19_moments(const T (&f)[19], T (&m)[19]) {
  T s[10], a[10];
  s[0] = f[0];
  a[0] = T(0);
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    s[p] = f[2 * p - 1] + f[2 * p];
    a[p] = f[2 * p - 1] - f[2 * p];
  }
  const T Sf = s[1] + s[2] + s[3];
  const T Se = (s[4] + s[5]) + (s[6] + s[7]) + (s[8] + s[9]);
  m[0] = s[0] + Sf + Se;
  m[1] = T(-30) * s[0] - T(11) * Sf + T(8) * Se;
  m[2] = T(12) * s[0] - T(4) * Sf + Se;
  const T t9 = T(2) * s[1] - s[2] - s[3];
  const T u9 = (s[4] + s[5]) + (s[6] + s[7]) - T(2) * (s[8] + s[9]);
  m[9] = t9 + u9;
  m[10] = T(-2) * t9 + u9;
  const T t11 = s[2] - s[3];
  const T u11 = (s[4] + s[5]) - (s[6] + s[7]);
  m[11] = t11 + u11;
  m[12] = T(-2) * t11 + u11;
  m[13] = s[4] - s[5];
  m[14] = s[8] - s[9];
  m[15] = s[6] - s[7];
  const T Ax = (a[4] + a[5]) + (a[6] + a[7]);
  const T Ay = (a[4] - a[5]) + (a[8] + a[9]);
  const T Az = (a[6] - a[7]) + (a[8] - a[9]);
  m[3] = a[1] + Ax;
  m[4] = T(-4) * a[1] + Ax;
  m[5] = a[2] + Ay;
  m[6] = T(-4) * a[2] + Ay;
  m[7] = a[3] + Az;
  m[8] = T(-4) * a[3] + Az;
  m[16] = (a[4] + a[5]) - (a[6] + a[7]);
  m[17] = (a[5] - a[4]) + (a[8] + a[9]);
  m[18] = (a[6] - a[7]) - (a[8] - a[9]);
}

// f -= M^T d with d the relaxed, force-corrected moment updates of m.
template <class T>
__host__ __device__ __forceinline__ void mrt19_relax_back(T (&f)[19], const T (&m)[19], const MrtIn<T>& q) {
  T d[19];
  mrt_relax_all<T>(m, d, q, std::make_integer_sequence<int, 19>{});
  // back transform f -= M^T d, even part E and odd part O per pair
  f[0] -= d[0] - T(30) * d[1] + T(12) * d[2];
  const T cf = d[0] - T(11) * d[1] - T(4) * d[2];
  const T ce = d[0] + T(8) * d[1] + d[2];
  const T g9 = d[9] + d[10];
  const T h11 = d[11] + d[12];
  T E[10], O[10];
  E[1] = cf + T(2) * d[9] - T(4) * d[10];
  E[2] = cf - d[9] + T(2) * d[10] + d[11] - T(2) * d[12];
  E[3] = cf - d[9] + T(2) * d[10] - d[11] + T(2) * d[12];
  E[4] = ce + g9 + h11 + d[13];
  E[5] = ce + g9 + h11 - d[13];
  E[6] = ce + g9 - h11 + d[15];
  E[7] = ce + g9 - h11 - d[15];
  E[8] = ce - T(2) * g9 + d[14];
  E[9] = ce - T(2) * g9 - d[14];
  const T jx = d[3] + d[4], jy = d[5] + d[6], jz = d[7] + d[8];
  O[1] = d[3] - T(4) * d[4];
  O[2] = d[5] - T(4) * d[6];
  O[3] = d[7] - T(4) * d[8];
  O[4] = jx + jy + d[16] - d[17];
  O[5] = jx - jy + d[16] + d[17];
  O[6] = jx + jz - d[16] + d[18];
  O[7] = jx - jz - d[16] - d[18];
  O[8] = jy + jz + d[17] - d[18];
  O[9] = jy - jz + d[17] + d[18];
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    f[2 * p - 1] -= E[p] + O[p];
    f[2 * p] -= E[p] - O[p];
  }
}

// In-place D3Q19 MRT collision in moment space (pair-split transforms).
template <class T>
__host__ __device__ __forceinline__ void mrt19_collide_fact(T (&f)[19], const MrtIn<T>& q) {
  T m[19];
  mrt19_moments<T>(f, m);
  mrt19_relax_back<T>(f, m, q);
}

// f -= Mi [ S M (f - feq) - (I - S/2) M F ]   (all loops unrolled; M is
// integer so the compiler folds every zero).
template <class T>
__host__ __device__ __forceinline__ void mrt19_collide(T (&f)[19], const T (&feq)[19], const T (&F)[19], T s_nu) {
  T d[19];
#pragma unroll
  for (int k = 0; k < 19; ++k) {
    T mn = T(0), mf = T(0);
#pragma unroll
    for (int i = 0; i < 19; ++i) {
      if (mrt_m(k, i) != 0) {
        mn += T(mrt_m(k, i)) * (f[i] - feq[i]);
        mf += T(mrt_m(k, i)) * F[i];
      }
    }
    const T s = mrt_is_shear(k) ? s_nu : T(mrt_rate(k));
    d[k] = (s * mn - (T(1) - T(0.5) * s) * mf) * T(1.0 / mrt_norm(k));
  }
#pragma unroll
  for (int i = 0; i < 19; ++i) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 19; ++k)
      if (mrt_m(k, i) != 0) acc += T(mrt_m(k, i)) * d[k];
    f[i] -= acc;
  }
}

// ------------------------------------------------- packed FP32 pairs (sm_100)
// a / b: IEEE division in FP64, the fast approximate division in FP32 (about
// two ulp, far inside the single-precision parity bounds; the denominators in
// the kernels — densities, |grad phi| + eps, capacities, relaxation times —
// are nowhere near its 2^126 limit).  An IEEE FP32 division is a
// multi-instruction sequence with a slow path; the 16-bit kernels are
// instruction-bound.
__device__ __forceinline__ double div_fast(double a, double b) { return a / b; }
__device__ __forceinline__ float div_fast(float a, float b) { return __fdividef(a, b); }

// Blackwell executes two FP32 lanes per FADD2 / FMUL2 / FFMA2 instruction
// (round to nearest, no contraction beyond the written FMA).  Used where the
// same arithmetic runs over two population pairs.
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// -------------------------------------------------------- storage traits
// Every lattice is held as its deviation from the rest state,
//   f'_i = f_i - w_i ref      (ref = rho0, phi = 1, phi = -1, u = -Delta, ...),
// and the kernels do their arithmetic on f' (moments of f' plus the rest
// value; equilibria minus w_i ref).  Near rest the deviation is small, so FP32
// keeps the digits of the velocity moments that raw f_i ~ w_i would round
// away, and the 16-bit formats hold f'_i / w_i, a plane-independent O(1)
// quantity inside the normal range of FP16.  FP64 and FP32 store f', FP16 and
// BF16 store f'/w; collision arithmetic is FP64 or FP32.
// st_rt stores like st and returns the value a later ld will see (used to
// carry the 16-bit rounding residual into an FP32 rest population).
template <class S>
struct Stor;
template <>
struct Stor<double> {
  typedef double T;
  static constexpr int bytes = 8;
  static constexpr bool scaled = false;
  __device__ __forceinline__ static double ldr(const double* p) { return *p; }
  __device__ __forceinline__ static void str(double* p, double v) { *p = v; }
  __device__ __forceinline__ static double ld(const double* p, double) { return *p; }
  __device__ __forceinline__ static void st(double* p, double v, double) { *p = v; }
  __device__ __forceinline__ static double st_rt(double* p, double v, double) {
    *p = v;
    return v;
  }
};
template <>
struct Stor<float> {
  typedef float T;
  static constexpr int bytes = 4;
  static constexpr bool scaled = false;
  __device__ __forceinline__ static float ldr(const float* p) { return *p; }
  __device__ __forceinline__ static void str(float* p, float v) { *p = v; }
  __device__ __forceinline__ static float ld(const float* p, float) { return *p; }
  __device__ __forceinline__ static void st(float* p, float v, float) { *p = v; }
  __device__ __forceinline__ static float st_rt(float* p, float v, float) {
    *p = v;
    return v;
  }
};
template <>
struct Stor<__half> {
  typedef float T;
  static constexpr int bytes = 2;
  static constexpr bool scaled = true;  // stores f'/w
  __device__ __forceinline__ static float ldr(const __half* p) { return __half2float(*p); }
  __device__ __forceinline__ static void str(__half* p, float v) { *p = __float2half_rn(v); }
  // store and return what a later ldr reads
  __device__ __forceinline__ static float str_rt(__half* p, float v) {
    const __half h = __float2half_rn(v);
    *p = h;
    return __half2float(h);
  }
  __device__ __forceinline__ static float ld(const __half* p, float w) { return w * __half2float(*p); }
  __device__ __forceinline__ static void st(__half* p, float v, float w) { *p = __float2half_rn(v * (1.0f / w)); }
  __device__ __forceinline__ static float st_rt(__half* p, float v, float w) {
    const __half h = __float2half_rn(v * (1.0f / w));
    *p = h;
    return w * __half2float(h);
  }
};
template <>
struct Stor<__nv_bfloat16> {
  typedef float T;
  static constexpr int bytes = 2;
  static constexpr bool scaled = true;  // stores f'/w
  __device__ __forceinline__ static float ldr(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  __device__ __forceinline__ static void str(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
  __device__ __forceinline__ static float str_rt(__nv_bfloat16* p, float v) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    *p = h;
    return __bfloat162float(h);
  }
  __device__ __forceinline__ static float ld(const __nv_bfloat16* p, float w) { return w * __bfloat162float(*p); }
  __device__ __forceinline__ static void st(__nv_bfloat16* p, float v, float w) {
    *p = __float2bfloat16_rn(v * (1.0f / w));
  }
  __device__ __forceinline__ static float st_rt(__nv_bfloat16* p, float v, float w) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v * (1.0f / w));
    *p = h;
    return w * __bfloat162float(h);
  }
};

// -------------------------------------------------------------- geometry
// Boundary kinds per axis: 0 periodic, 1 walls (cells 0 and n-1 solid),
// 2 closed faces (all cells fluid, the faces bounce back).
//
// z-slab of a larger domain (slab = 1): the local planes 1 .. nz - 2 are the
// global planes zg0 .. zg0 + nz - 3 of a domain of nzg planes, and the local
// planes 0 and nz - 1 are ghost copies of the neighbour slabs' boundary
// planes.  Ghost cells are never updated (fluid() is false there), but a
// neighbour link into a ghost plane is valid wherever the global domain has
// that neighbour, so streaming reads and writes the ghost slots; the z wrap of
// a periodic global axis goes through the ghosts, never through the index.
//
// Dynamic solids (a multiphase flow coupled to a growing dendrite): `solid`
// flags cells that left the fluid (1), and `near` the fluid cells with a
// solid neighbour; both NULL when the domain has none.  A solid cell is not
// fluid, a link into it bounces back, and a cell next to one takes the
// general neighbourhood (Nbr) instead of the interior-row addressing.
struct Geom {
  int nx, ny, nz;
  int bc0, bc1, bc2;
  int64_t stride;  // population plane stride (cells)
  int slab = 0, zg0 = 0, nzg = 0;
  const unsigned char* solid = nullptr;
  const unsigned char* near = nullptr;

  // global z of local plane z (slab), and whether a global plane is a cell of
  // the domain that streams (not beyond a non-periodic face, not a wall)
  __device__ __forceinline__ int gz(int z) const { return zg0 + z - 1; }
  __device__ __forceinline__ bool gz_open(int q) const {
    if (bc2 != 0 && (q < 0 || q >= nzg)) return false;
    if (bc2 == 1 && (q == 0 || q == nzg - 1)) return false;
    return true;
  }

  __device__ __forceinline__ bool fluid(int x, int y, int z) const {
    if (solid && solid[idx(x, y, z)]) return false;
    if (bc0 == 1 && (x == 0 || x == nx - 1)) return false;
    if (bc1 == 1 && (y == 0 || y == ny - 1)) return false;
    if (slab) return z >= 1 && z <= nz - 2 && gz_open(gz(z));
    if (bc2 == 1 && (z == 0 || z == nz - 1)) return false;
    return true;
  }
  __device__ __forceinline__ int64_t idx(int x, int y, int z) const {
    return (int64_t)x + (int64_t)nx * ((int64_t)y + (int64_t)ny * z);
  }
  // Neighbour index along (dx,dy,dz); false when it is non-fluid or outside a
  // closed face.  Periodic axes wrap (mkFluidsLBM::neighbor, mkFluidsLBM.h:82).
  __device__ __forceinline__ bool nbr(int x, int y, int z, int dx, int dy, int dz, int64_t& out) const {
    int cx = x + dx, cy = y + dy, cz = z + dz;
    if (dx != 0) {
      if (cx < 0 || cx >= nx) {
        if (bc0 != 0) return false;
        cx = cx < 0 ? cx + nx : cx - nx;
      }
      if (bc0 == 1 && (cx == 0 || cx == nx - 1)) return false;
    }
    if (dy != 0) {
      if (cy < 0 || cy >= ny) {
        if (bc1 != 0) return false;
        cy = cy < 0 ? cy + ny : cy - ny;
      }
      if (bc1 == 1 && (cy == 0 || cy == ny - 1)) return false;
    }
    if (dz != 0) {
      if (slab) {
        if (cz < 0 || cz >= nz || !gz_open(gz(cz))) return false;
      } else {
        if (cz < 0 || cz >= nz) {
          if (bc2 != 0) return false;
          cz = cz < 0 ? cz + nz : cz - nz;
        }
        if (bc2 == 1 && (cz == 0 || cz == nz - 1)) return false;
      }
    }
    out = idx(cx, cy, cz);
    return !(solid && solid[out]);
  }
};

// Neighbourhood of one cell, resolved once per thread: per axis the three
// candidate coordinates (already multiplied by the axis stride) and whether
// each is fluid; a 27-bit mask answers "is neighbour (dx,dy,dz) fluid".
// Cell indices are 32-bit (domains are limited to < 2^31 cells); only the
// population-plane offset i * stride is 64-bit.
struct Nbr {
  int ox[3], oy[3], oz[3];
  unsigned ok;
  int base = 0;  // offset of the domain inside a packed multi-domain index

  __device__ __forceinline__ static void axis(int n, int bc, int c, int mul, int (&o)[3], bool (&v)[3]) {
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      int cc = c + d;
      bool valid = true;
      if (cc < 0 || cc >= n) {
        if (bc == 0) {
          cc = cc < 0 ? cc + n : cc - n;
        } else {
          valid = false;
          cc = c;
        }
      }
      if (bc == 1 && (cc == 0 || cc == n - 1)) valid = false;
      o[d + 1] = cc * mul;
      v[d + 1] = valid;
    }
  }

  // z of a slab: no wrap (the ghosts hold the neighbours), validity from the
  // global plane
  __device__ __forceinline__ static void axis_slab(const Geom& g, int z, int (&o)[3], bool (&v)[3]) {
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const int cc = z + d;
      const bool in = cc >= 0 && cc < g.nz;
      v[d + 1] = in && g.gz_open(g.gz(cc));
      o[d + 1] = (in ? cc : z) * (g.nx * g.ny);
    }
  }

  __device__ __forceinline__ Nbr(const Geom& g, int x, int y, int z) {
    bool vx[3], vy[3], vz[3];
    axis(g.nx, g.bc0, x, 1, ox, vx);
    axis(g.ny, g.bc1, y, g.nx, oy, vy);
    if (g.slab)
      axis_slab(g, z, oz, vz);
    else
      axis(g.nz, g.bc2, z, g.nx * g.ny, oz, vz);
    ok = 0u;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
          if (vx[dx] && vy[dy] && vz[dz]) ok |= 1u << (dx + 3 * dy + 9 * dz);
    if (g.solid) {
      // links into dynamic solids close
#pragma unroll
      for (int b = 0; b < 27; ++b)
        if (((ok >> b) & 1u) && g.solid[ox[b % 3] + oy[(b / 3) % 3] + oz[b / 9]]) ok &= ~(1u << b);
    }
  }
  __device__ __forceinline__ int idx(int dx, int dy, int dz) const {
    return base + ox[dx + 1] + oy[dy + 1] + oz[dz + 1];
  }
  __device__ __forceinline__ bool fluid(int dx, int dy, int dz) const {
    return (ok >> ((dx + 1) + 3 * (dy + 1) + 9 * (dz + 1))) & 1u;
  }
};

// Addressing of a cell whose y and z neighbours are all fluid and need no
// periodic wrap (every row of the domain interior, so a warp — one row
// segment — takes this path as a whole).  x neighbours come from two
// wrap-aware offsets; no fluid tests, no selects.
struct Fast {
  int c, xm, xp, nx, nxy;
  __device__ __forceinline__ int xo(int d) const { return d < 0 ? xm : (d > 0 ? xp : 0); }
  __device__ __forceinline__ int idx(int dx, int dy, int dz) const { return c + xo(dx) + dy * nx + dz * nxy; }
};

// Whether (x,y,z) may use Fast: y, z strictly inside the fluid span of their
// axis, x inside it or on a periodic axis.
__device__ __forceinline__ bool fast_cell(const Geom& g, int x, int y, int z) {
  if (g.near && g.near[g.idx(x, y, z)]) return false;
  auto inside = [](int c, int n, int bc) {
    const int lo = bc == 1 ? 2 : 1;
    const int hi = bc == 1 ? n - 3 : n - 2;
    return c >= lo && c <= hi;
  };
  // a slab plane needs no z wrap; its z neighbours must all be open globally
  const bool zin = g.slab ? (g.bc2 == 0 || inside(g.gz(z), g.nzg, g.bc2)) : inside(z, g.nz, g.bc2);
  return inside(y, g.ny, g.bc1) && zin && (g.bc0 == 0 ? g.nx >= 3 : inside(x, g.nx, g.bc0));
}

__device__ __forceinline__ Fast make_fast(const Geom& g, int x, int y, int z) {
  Fast f;
  f.nx = g.nx;
  f.nxy = g.nx * g.ny;
  f.c = x + g.nx * (y + g.ny * z);
  f.xm = x == 0 ? g.nx - 1 : -1;
  f.xp = x == g.nx - 1 ? -(g.nx - 1) : 1;
  return f;
}

// Interior-row addressing for domains whose x faces are closed or walled:
// as Fast, plus the validity of the two x neighbours, so the cells at the
// ends of a row stay on the same code path as the rest of their warp (the
// bounce-back select is emitted only for directions with ex != 0).
struct FastW : Fast {
  bool okm, okp;  // x-1 / x+1 neighbour is fluid
};

// Whether (x,y,z) may use FastW: y and z strictly inside the fluid span of
// their axis (x is free).
__device__ __forceinline__ bool fastw_cell(const Geom& g, int x, int y, int z) {
  if (g.near && g.near[g.idx(x, y, z)]) return false;
  auto inside = [](int c, int n, int bc) {
    const int lo = bc == 1 ? 2 : 1;
    const int hi = bc == 1 ? n - 3 : n - 2;
    return c >= lo && c <= hi;
  };
  const bool zin = g.slab ? (g.bc2 == 0 || inside(g.gz(z), g.nzg, g.bc2)) : inside(z, g.nz, g.bc2);
  return inside(y, g.ny, g.bc1) && zin;
}

__device__ __forceinline__ FastW make_fastw(const Geom& g, int x, int y, int z) {
  FastW f;
  f.nx = g.nx;
  f.nxy = g.nx * g.ny;
  f.c = x + g.nx * (y + g.ny * z);
  if (g.bc0 == 0) {
    f.xm = x == 0 ? g.nx - 1 : -1;
    f.xp = x == g.nx - 1 ? -(g.nx - 1) : 1;
    f.okm = f.okp = true;
  } else {
    const int lo = g.bc0 == 1 ? 1 : 0, hi = g.bc0 == 1 ? g.nx - 2 : g.nx - 1;
    f.xm = -1;
    f.xp = 1;
    f.okm = x - 1 >= lo;
    f.okp = x + 1 <= hi;
  }
  return f;
}

__device__ __forceinline__ bool fastw_fluid(const FastW& fa, int dx) { return dx < 0 ? fa.okm : (dx > 0 ? fa.okp : true); }

template <int Q>
__device__ __forceinline__ int64_t off_in(int64_t stride, const FastW& fa, int parity, int, int i) {
  if (parity == 0) return (int64_t)i * stride + fa.c;
  if (ex(i) == 0) return (int64_t)inv(i) * stride + fa.idx(-ex(i), -ey(i), -ez(i));
  const bool f = fastw_fluid(fa, -ex(i));
  return (int64_t)(f ? inv(i) : i) * stride + (f ? fa.idx(-ex(i), -ey(i), -ez(i)) : fa.c);
}
template <int Q>
__device__ __forceinline__ int64_t off_out(int64_t stride, const FastW& fa, int parity, int, int i) {
  if (parity == 0) return (int64_t)inv(i) * stride + fa.c;
  if (ex(i) == 0) return (int64_t)i * stride + fa.idx(ex(i), ey(i), ez(i));
  const bool f = fastw_fluid(fa, ex(i));
  return (int64_t)(f ? i : inv(i)) * stride + (f ? fa.idx(ex(i), ey(i), ez(i)) : fa.c);
}

template <int Q>
__device__ __forceinline__ int64_t off_in(int64_t stride, const Fast& fa, int parity, int, int i) {
  if (parity == 0) return (int64_t)i * stride + fa.c;
  return (int64_t)inv(i) * stride + fa.idx(-ex(i), -ey(i), -ez(i));
}
template <int Q>
__device__ __forceinline__ int64_t off_out(int64_t stride, const Fast& fa, int parity, int, int i) {
  if (parity == 0) return (int64_t)inv(i) * stride + fa.c;
  return (int64_t)i * stride + fa.idx(ex(i), ey(i), ez(i));
}

// Element offset of the slot population i of the cell at `c` is read from
// (pre-collision) at the given AA parity.  The bounce-back alternative is a
// select, not a branch, so every access is one load or store.
template <int Q>
__device__ __forceinline__ int64_t off_in(int64_t stride, const Nbr& nb, int parity, int c, int i) {
  if (parity == 0) return (int64_t)i * stride + c;
  const bool f = nb.fluid(-ex(i), -ey(i), -ez(i));
  const int cell = f ? nb.idx(-ex(i), -ey(i), -ez(i)) : c;
  return (int64_t)(f ? inv(i) : i) * stride + cell;
}

// Element offset of the slot the post-collision population i is written to.
template <int Q>
__device__ __forceinline__ int64_t off_out(int64_t stride, const Nbr& nb, int parity, int c, int i) {
  if (parity == 0) return (int64_t)inv(i) * stride + c;
  const bool f = nb.fluid(ex(i), ey(i), ez(i));
  const int cell = f ? nb.idx(ex(i), ey(i), ez(i)) : c;
  return (int64_t)(f ? i : inv(i)) * stride + cell;
}

// Pre-collision deviation f'_i of the cell at `c` (= nb.idx(0,0,0)); `nb` is
// a general neighbourhood (Nbr) or an interior-row one (Fast).
template <class S, int Q, class NB>
__device__ __forceinline__ typename Stor<S>::T ld_in(const S* __restrict__ A, int64_t stride, const NB& nb,
                                                      int parity, int c, int i) {
  return Stor<S>::ld(A + off_in<Q>(stride, nb, parity, c, i), typename Stor<S>::T(wq<Q>(i)));
}

// Bring the slot that population i of the cell at `c` is read from into L2
// (no register, no wait), for a load that comes later in the thread.
template <class S, int Q, class NB>
__device__ __forceinline__ void pf_in(const S* __restrict__ A, int64_t stride, const NB& nb, int parity, int c, int i) {
  const S* p = A + off_in<Q>(stride, nb, parity, c, i);
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// The stored value itself: f'_i, or f'_i / w_i for the 16-bit formats
// (Stor<S>::scaled), for arithmetic that works in the stored units.
// Two adjacent stored values at p as ldr reads them (p aligned to twice the
// element size): one 16-, 8- or 4-byte load.
__device__ __forceinline__ void ldr_pair(const double* p, double& a, double& b) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ldr_pair(const float* p, float& a, float& b) {
  const float2 v = *reinterpret_cast<const float2*>(p);
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ldr_pair(const __half* p, float& a, float& b) {
  const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void ldr_pair(const __nv_bfloat16* p, float& a, float& b) {
  const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void st_pair(double* p, double a, double b) { *reinterpret_cast<double2*>(p) = make_double2(a, b); }
__device__ __forceinline__ void st_pair(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }

template <class S, int Q, class NB>
__device__ __forceinline__ typename Stor<S>::T ld_in_raw(const S* __restrict__ A, int64_t stride, const NB& nb,
                                                          int parity, int c, int i) {
  return Stor<S>::ldr(A + off_in<Q>(stride, nb, parity, c, i));
}
template <class S, int Q, class NB>
__device__ __forceinline__ void st_out_raw(S* __restrict__ A, int64_t stride, const NB& nb, int parity, int c, int i,
                                           typename Stor<S>::T v) {
  Stor<S>::str(A + off_out<Q>(stride, nb, parity, c, i), v);
}
template <class S, int Q, class NB>
__device__ __forceinline__ typename Stor<S>::T st_out_raw_rt(S* __restrict__ A, int64_t stride, const NB& nb,
                                                              int parity, int c, int i, typename Stor<S>::T v) {
  return Stor<S>::str_rt(A + off_out<Q>(stride, nb, parity, c, i), v);
}

// Store the post-collision deviation f'_i of the cell at `c`.
template <class S, int Q, class NB>
__device__ __forceinline__ void st_out(S* __restrict__ A, int64_t stride, const NB& nb, int parity, int c, int i,
                                       typename Stor<S>::T v) {
  Stor<S>::st(A + off_out<Q>(stride, nb, parity, c, i), v, typename Stor<S>::T(wq<Q>(i)));
}

// Store and return the value a later load will see.
template <class S, int Q, class NB>
__device__ __forceinline__ typename Stor<S>::T st_out_rt(S* __restrict__ A, int64_t stride, const NB& nb, int parity,
                                                          int c, int i, typename Stor<S>::T v) {
  return Stor<S>::st_rt(A + off_out<Q>(stride, nb, parity, c, i), v, typename Stor<S>::T(wq<Q>(i)));
}

// Neighbour queries common to both neighbourhood kinds.
__device__ __forceinline__ bool nb_fluid(const Nbr& nb, int dx, int dy, int dz) { return nb.fluid(dx, dy, dz); }
__device__ __forceinline__ bool nb_fluid(const Fast&, int, int, int) { return true; }
__device__ __forceinline__ int nb_idx(const Nbr& nb, int dx, int dy, int dz) { return nb.idx(dx, dy, dz); }
__device__ __forceinline__ int nb_idx(const Fast& fa, int dx, int dy, int dz) { return fa.idx(dx, dy, dz); }
__device__ __forceinline__ bool nb_fluid(const FastW& fa, int dx, int, int) { return fastw_fluid(fa, dx); }
__device__ __forceinline__ int nb_idx(const FastW& fa, int dx, int dy, int dz) { return fa.idx(dx, dy, dz); }

// Post-collision deviation f'_i of a cell in the layout left after
// `steps_done` loops (field output, diagnostics): the slot the last loop
// wrote it to.
template <class S, int Q>
__device__ __forceinline__ typename Stor<S>::T ld_out(const S* __restrict__ A, int64_t stride, const Nbr& nb,
                                                       int64_t steps_done, int c, int i) {
  return Stor<S>::ld(A + off_out<Q>(stride, nb, (int)((steps_done + 1) & 1), c, i), typename Stor<S>::T(wq<Q>(i)));
}

// Inverse of ld_out: place a post-collision deviation so that the next loop
// (parity = steps_done & 1) reads it as the streamed value.
template <class S, int Q>
__device__ __forceinline__ void st_layout(S* __restrict__ A, int64_t stride, const Nbr& nb, int64_t steps_done, int c,
                                          int i, typename Stor<S>::T v) {
  Stor<S>::st(A + off_out<Q>(stride, nb, (int)((steps_done + 1) & 1), c, i), v, typename Stor<S>::T(wq<Q>(i)));
}

// Equilibrium placement of the initial state.
// Stores the deviation of  f_i = base_scale w (1 + 3eu + 4.5eu^2 - 1.5u^2) + w p_extra
// from w ref, placed as the post-collision state of loop 0.
template <class S, int Q>
__device__ __forceinline__ void put_eq(S* A, const Geom& g, const Nbr& nb, int c, double base_scale, double ux,
                                       double uy, double uz, double p_extra, double ref) {
  typedef typename Stor<S>::T T;
  const double uu = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const double w = wq<Q>(i);
    const double eu = ex(i) * ux + ey(i) * uy + ez(i) * uz;
    const double v = w * ((base_scale - ref + p_extra) + base_scale * (3.0 * eu + 4.5 * eu * eu - 1.5 * uu));
    st_layout<S, Q>(A, g.stride, nb, 0, c, i, T(v));
  }
}

// Storage type of phi and the scalar fields: FP64 with FP64 populations, else FP32.
template <class S>
struct PhiOf {
  typedef float type;
};
template <>
struct PhiOf<double> {
  typedef double type;
};

}  // namespace mkd

#endif
