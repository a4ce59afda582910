// mk_adjoint.cu — discrete adjoint of the thermal dendrite loop (mk_backward).
//
// Loss L = sum_x (phi(x) - target(x))^2 of phi after `steps` loops; gradients
// with respect to the anisotropy strength eps4, the undercooling Delta (the
// initial u = -Delta) and the thermal relaxation time tau_T = 1/omega_T
// (tau0 held fixed).  The reference has no gradients; this is the inverse-
// design use of run_thermal_dendrite (MaterKit.cpp:743-788).
//
// Reverse mode over the loop as the kernels run it (mk_dendrite.cuh):
// state at the start of loop n = streamed populations g^n, t^n, phi^(n-1)
// (the phi_old plane) and u^n (the T plane).  Forward states are kept as
// checkpoints every K loops; each segment is recomputed forward (storing its
// K + 1 states in HBM, about 113 MB per 96^3 FP64 state) and reversed with two
// kernels per loop:
//
//   k_adj_cell  adjoints of the post-collision populations pulled from the
//               next loop's adjoints (the transpose of the streaming, bounce-
//               back included), the local reverse of the thermal and phase-
//               field relaxations, the reverse of the anisotropy (Hessian of
//               a(n)), and per-block partial sums of dL/deps4, dL/domega_T;
//   k_adj_phi   the transpose of the D3Q19 gradient stencil (gather of the
//               neighbours' grad-phi adjoints) and phi = ref + sum g.
//
// The adjoint arithmetic is FP64 for FP64 and FP32 storage.  The formulas are
// those of the oracle's orc_backward, checked there against central
// differences.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mkb200.h"
#include "mk_dendrite.cuh"
#include "mk_engine.hpp"

using namespace mkd;

namespace {

constexpr int BX = 32, BY = 8;

struct AdjK {
  double om_g, om_t, fo, inv_tau0, lambda, eps4, eps2;
  int aniso, nobj;
};

// d2a/dn2 and the derivatives of a and da/dn with respect to e4.
__device__ void aniso_second(int kind, double e4, double e2, const double (&n)[3], double (&H)[3][3], double& a_e4,
                             double (&da_e4)[3]) {
  const double x = n[0], y = n[1], z = n[2];
  const double x2 = x * x, y2 = y * y, z2 = z * z;
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int r = 0; r < 3; ++r) H[q][r] = 0.0;
  switch (kind) {
    case MK_ANISO_CBC: {
      const double s4 = x2 * x2 + y2 * y2 + z2 * z2;
      H[0][0] = 12.0 * e4 * x2 + e2 * (36.0 * x2 + 132.0 * y2 * z2);
      H[1][1] = 12.0 * e4 * y2 + e2 * (36.0 * y2 + 132.0 * x2 * z2);
      H[2][2] = 12.0 * e4 * z2 + e2 * (36.0 * z2 + 132.0 * x2 * y2);
      H[0][1] = H[1][0] = 264.0 * e2 * x * y * z2;
      H[0][2] = H[2][0] = 264.0 * e2 * x * z * y2;
      H[1][2] = H[2][1] = 264.0 * e2 * y * z * x2;
      a_e4 = s4 - 0.6;
      da_e4[0] = 4.0 * x2 * x;
      da_e4[1] = 4.0 * y2 * y;
      da_e4[2] = 4.0 * z2 * z;
      break;
    }
    case MK_ANISO_HCP: {
      const double h00 = 6.0 * e4 * (5.0 * x2 * x2 - 30.0 * x2 * y2 + 5.0 * y2 * y2);
      H[0][0] = h00;
      H[1][1] = -h00;
      H[0][1] = H[1][0] = 6.0 * e4 * (-20.0 * x2 * x * y + 20.0 * x * y2 * y);
      H[2][2] = 4.0 * e2;
      a_e4 = x2 * x2 * x2 - 15.0 * x2 * x2 * y2 + 15.0 * x2 * y2 * y2 - y2 * y2 * y2;
      da_e4[0] = 6.0 * (x2 * x2 * x - 10.0 * x2 * x * y2 + 5.0 * x * y2 * y2);
      da_e4[1] = -6.0 * (5.0 * x2 * x2 * y - 10.0 * x2 * y2 * y + y2 * y2 * y);
      da_e4[2] = 0.0;
      break;
    }
    case MK_ANISO_FACET: {
      const double r[3] = {sqrt(x2 + e2 * e2), sqrt(y2 + e2 * e2), sqrt(z2 + e2 * e2)};
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        H[q][q] = e4 * e2 * e2 / (r[q] * r[q] * r[q]);
        da_e4[q] = n[q] / r[q];
      }
      a_e4 = r[0] + r[1] + r[2] - sqrt(1.0 + e2 * e2) - 2.0 * e2;
      break;
    }
    default: {
      H[0][0] = 48.0 * e4 * x2;
      H[1][1] = 48.0 * e4 * y2;
      H[2][2] = 48.0 * e4 * z2;
      a_e4 = -3.0 + 4.0 * (x2 * x2 + y2 * y2 + z2 * z2);
      da_e4[0] = 16.0 * x2 * x;
      da_e4[1] = 16.0 * y2 * y;
      da_e4[2] = 16.0 * z2 * z;
      break;
    }
  }
}

// Below this |grad phi| the normal n = grad phi / (|grad phi| + 1e-12) is
// rounding noise and its exact derivative (~1 / (|grad phi| + 1e-12)) makes
// the adjoint of the (1 - a^2) dphi source grow without bound over long runs
// (1e32 after 2000 loops at 96^3 against central differences near 3e5).
// There the reverse keeps the direct eps4 derivative of a and N and drops
// their derivative through n (the oracle does the same).
constexpr double kAdjGradCut = 1e-8;

// Reverse of anisotropy(): adds the adjoint of the lab gradient to gb and
// returns the adjoint of e4, from the adjoints ab of a and Nb of N.
__device__ double anisotropy_vjp(const double* __restrict__ R, int kind, double e4, double e2, const double (&g)[3],
                                 double ab, const double (&Nb)[3], double (&gb)[3]) {
  const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  const double inv = 1.0 / (gn + 1e-12);
  const double nl[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
  double nc[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) nc[q] = R[0 * 3 + q] * nl[0] + R[1 * 3 + q] * nl[1] + R[2 * 3 + q] * nl[2];
  double a, da[3];
  aniso_function<double>(kind, e4, e2, nc, a, da);
  const double ndg = nc[0] * da[0] + nc[1] * da[1] + nc[2] * da[2];
  double Ncb[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) Ncb[q] = R[0 * 3 + q] * Nb[0] + R[1 * 3 + q] * Nb[1] + R[2 * 3 + q] * Nb[2];
  double ct = 0, cn = 0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    ct += Ncb[q] * (da[q] - nc[q] * ndg);
    cn += Ncb[q] * nc[q];
  }
  double gnb = a * ct;
  const double abt = ab + gn * ct;
  const double ndgb = -gn * a * cn;
  double dab[3], ncb[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    dab[q] = gn * a * Ncb[q] + ndgb * nc[q];
    ncb[q] = -gn * a * Ncb[q] * ndg + ndgb * da[q];
  }
  double H[3][3], a_e4, da_e4[3];
  aniso_second(kind, e4, e2, nc, H, a_e4, da_e4);
#pragma unroll
  for (int q = 0; q < 3; ++q) ncb[q] += abt * da[q] + H[q][0] * dab[0] + H[q][1] * dab[1] + H[q][2] * dab[2];
  const double e4b = abt * a_e4 + dab[0] * da_e4[0] + dab[1] * da_e4[1] + dab[2] * da_e4[2];
  if (gn < kAdjGradCut) return e4b;
  double nlb[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) nlb[r] = R[r * 3 + 0] * ncb[0] + R[r * 3 + 1] * ncb[1] + R[r * 3 + 2] * ncb[2];
  const double invb = nlb[0] * g[0] + nlb[1] * g[1] + nlb[2] * g[2];
#pragma unroll
  for (int q = 0; q < 3; ++q) gb[q] += inv * nlb[q];
  gnb -= inv * inv * invb;
  if (gn > 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) gb[q] += gnb * g[q] / gn;
  return e4b;
}

// Block sum of two values into partial[2 * block] (fixed order: warp
// shuffles, then the warps in index order).
__device__ void block_sum2(double v0, double v1, double* __restrict__ partial) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_down_sync(0xffffffffu, v0, o);
    v1 += __shfl_down_sync(0xffffffffu, v1, o);
  }
  __shared__ double sh[2][32];
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = t & 31, wid = t >> 5, nw = (blockDim.x * blockDim.y + 31) >> 5;
  if (lane == 0) {
    sh[0][wid] = v0;
    sh[1][wid] = v1;
  }
  __syncthreads();
  if (t == 0) {
    double s0 = 0, s1 = 0;
    for (int w = 0; w < nw; ++w) {
      s0 += sh[0][w];
      s1 += sh[1][w];
    }
    const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    partial[2 * b] = s0;
    partial[2 * b + 1] = s1;
  }
}

// acc[q] += sum of the block partials, in a fixed order.
__global__ void k_adj_final(const double* __restrict__ partial, int nblocks, double* __restrict__ acc) {
  __shared__ double sh[2][256];
  double s0 = 0, s1 = 0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    s0 += partial[2 * b];
    s1 += partial[2 * b + 1];
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    acc[0] += sh[0][0];
    acc[1] += sh[1][0];
  }
}

// Seed of the reverse sweep: dL/dg_j = 2 (phi - target) for every j of a
// fluid cell (phi after the last loop is ref + sum g of that loop); all other
// adjoints zero.  Also the per-block loss partials.
template <class P>
__global__ void k_adj_seed(const P* __restrict__ phi, const double* __restrict__ target, const Geom g,
                           double* __restrict__ Lg, double* __restrict__ Lt, double* __restrict__ LP,
                           double* __restrict__ LU, double* __restrict__ partial) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double l = 0;
  if (x < g.nx && y < g.ny) {
    const int64_t c = g.idx(x, y, z);
    const double d = double(phi[c]) - target[c];
    l = d * d;
    const double s = g.fluid(x, y, z) ? 2.0 * d : 0.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      Lg[i * g.stride + c] = s;
      Lt[i * g.stride + c] = 0.0;
    }
    LP[c] = 0.0;
    LU[c] = 0.0;
  }
  block_sum2(l, 0.0, partial);
}

// Reverse of the local part of loop n.  In: the next loop's adjoints (Lg1,
// Lt1, LP1, LU1) and the forward state of loop n (streamed t^n from the raw
// AA planes, phi^(n-1), u^n, and phi^n).  Out: (1 - omega_g) times the
// post-collision g adjoint (Lg0, completed by k_adj_phi), Lt0, LP0, LU0, the
// local phi adjoint Lph and the grad-phi adjoint Gb (3 planes).
template <class S, class P, int PARITY>
__global__ void __launch_bounds__(BX* BY)
    k_adj_cell(const S* __restrict__ Tp, const P* __restrict__ phi_old, const P* __restrict__ temp,
               const P* __restrict__ phi_n, const unsigned char* __restrict__ grain, const double* __restrict__ seeds,
               const double* __restrict__ Lg1, const double* __restrict__ Lt1, const double* __restrict__ LP1,
               const double* __restrict__ LU1, double* __restrict__ Lg0, double* __restrict__ Lt0,
               double* __restrict__ LP0, double* __restrict__ LU0, double* __restrict__ Lph, double* __restrict__ Gb,
               double* __restrict__ partial, const Geom g, const AdjK k) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double e4_acc = 0, om_acc = 0;
  if (x < g.nx && y < g.ny) {
    const int c = (int)g.idx(x, y, z);
    const int64_t st = g.stride;
    if (!g.fluid(x, y, z)) {
      // phi of a non-fluid cell is a copy of P: its adjoint goes to P
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        Lg0[i * st + c] = 0.0;
        Lt0[i * st + c] = 0.0;
      }
      LP0[c] = 0.0;
      LU0[c] = 0.0;
      Lph[c] = LP1[c];
      Gb[c] = Gb[st + c] = Gb[2 * st + c] = 0.0;
    } else {
      const Nbr nb(g, x, y, z);
      // adjoints of the post-collision populations: the transpose of the
      // streaming (x + e_i, or the bounced slot inv(i) of x)
      double mg[7], mt[7];
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        const bool f = nb.fluid(ex(i), ey(i), ez(i));
        const int64_t o = f ? (int64_t)i * st + nb.idx(ex(i), ey(i), ez(i)) : (int64_t)inv(i) * st + c;
        mg[i] = Lg1[o];
        mt[i] = Lt1[o];
      }
      // thermal relaxation: t* = t - om_t (t - w T) + w dphi / 2, u' = T
      double t[7], dT = 0, Mt = 0;
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        t[i] = double(ld_in<S, 7>(Tp, st, nb, PARITY, c, i));
        dT += t[i];
        Mt += wq<7>(i) * mt[i];
      }
      const double lu1 = LU1[c];
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        Lt0[i * st + c] = (1.0 - k.om_t) * mt[i] + k.om_t * Mt + lu1;
        om_acc += mt[i] * (wq<7>(i) * dT - t[i]);
      }
      double dphib = 0.5 * Mt;
      // phase-field relaxation
      const double ph = double(phi_n[c]);
      const double dphi = ph - double(phi_old[c]);
      const double u = double(temp[c]);
      const double one_m = 1.0 - ph * ph;
      double gx = 0, gy = 0, gz = 0;
#pragma unroll
      for (int i = 1; i < 19; ++i) {
        const double fn = nb.fluid(ex(i), ey(i), ez(i)) ? double(phi_n[nb.idx(ex(i), ey(i), ez(i))]) : ph;
        const double w = wq<19>(i);
        if (ex(i)) gx += (w * ex(i)) * fn;
        if (ey(i)) gy += (w * ey(i)) * fn;
        if (ez(i)) gz += (w * ez(i)) * fn;
      }
      const double gr[3] = {3.0 * gx, 3.0 * gy, 3.0 * gz};
      const int gid = k.nobj > 1 ? (int)grain[c] : 0;
      const double* R = seeds + 12 * gid + 3;
      double a, N[3];
      anisotropy<double>(R, k.aniso, k.eps4, k.eps2, gr, a, N);
      double Mg = 0, Vg[3] = {0, 0, 0};
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        const double w = wq<7>(i);
        Mg += w * mg[i];
        Vg[0] += w * ex(i) * mg[i];
        Vg[1] += w * ey(i) * mg[i];
        Vg[2] += w * ez(i) * mg[i];
        Lg0[i * st + c] = (1.0 - k.om_g) * mg[i];
      }
      const double src_phi = (1.0 - 3.0 * ph * ph + 4.0 * k.lambda * u * ph * one_m) * k.inv_tau0;
      double phb = k.om_g * Mg + Mg * src_phi + LP1[c];
      LU0[c] = -Mg * k.lambda * one_m * one_m * k.inv_tau0;
      dphib += (1.0 - a * a) * Mg;
      phb += dphib;
      LP0[c] = -dphib;
      const double cs2 = 0.25;
      const double beta[3] = {k.fo * Vg[0], k.fo * Vg[1], k.fo * Vg[2]};
      const double bg = beta[0] * gr[0] + beta[1] * gr[1] + beta[2] * gr[2];
      const double ab = -cs2 * 2.0 * a * bg - 2.0 * a * dphi * Mg;
      const double Nb[3] = {-cs2 * beta[0], -cs2 * beta[1], -cs2 * beta[2]};
      double gb[3] = {-cs2 * (a * a - 1.0) * beta[0], -cs2 * (a * a - 1.0) * beta[1], -cs2 * (a * a - 1.0) * beta[2]};
      e4_acc = anisotropy_vjp(R, k.aniso, k.eps4, k.eps2, gr, ab, Nb, gb);
      // grad phi substitutes phi(x) at non-fluid neighbours: those terms stay here
#pragma unroll
      for (int i = 1; i < 19; ++i)
        if (!nb.fluid(ex(i), ey(i), ez(i)))
          phb += 3.0 * wq<19>(i) * (ex(i) * gb[0] + ey(i) * gb[1] + ez(i) * gb[2]);
      Lph[c] = phb;
      Gb[c] = gb[0];
      Gb[st + c] = gb[1];
      Gb[2 * st + c] = gb[2];
    }
  }
  block_sum2(e4_acc, om_acc, partial);
}

// Transpose of grad phi (gather of the neighbours' Gb) and of
// phi = ref + sum g: completes Lg0; a non-fluid cell's phi adjoint goes to P.
__global__ void __launch_bounds__(BX* BY)
    k_adj_phi(const double* __restrict__ Lph, const double* __restrict__ Gb, double* __restrict__ Lg0,
              double* __restrict__ LP0, const Geom g) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const int c = (int)g.idx(x, y, z);
  const int64_t st = g.stride;
  if (!g.fluid(x, y, z)) {
    LP0[c] += Lph[c];
    return;
  }
  const Nbr nb(g, x, y, z);
  double acc = Lph[c];
#pragma unroll
  for (int i = 1; i < 19; ++i)
    if (nb.fluid(-ex(i), -ey(i), -ez(i))) {
      const int s = nb.idx(-ex(i), -ey(i), -ez(i));
      acc += 3.0 * wq<19>(i) * (ex(i) * Gb[s] + ey(i) * Gb[st + s] + ez(i) * Gb[2 * st + s]);
    }
#pragma unroll
  for (int i = 0; i < 7; ++i) Lg0[i * st + c] += acc;
}

// -dL/dDelta partials: sum over fluid cells of sum_i w_i Lt_i + LU.
__global__ void k_adj_delta(const double* __restrict__ Lt, const double* __restrict__ LU, const Geom g,
                            double* __restrict__ partial) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  double v = 0;
  if (x < g.nx && y < g.ny && g.fluid(x, y, z)) {
    const int64_t c = g.idx(x, y, z);
#pragma unroll
    for (int i = 0; i < 7; ++i) v += wq<7>(i) * Lt[i * g.stride + c];
    v += LU[c];
  }
  block_sum2(v, 0.0, partial);
}

// Raw copy of the state at the start of a loop.
struct Snap {
  void* pop0 = nullptr;
  void* pop1 = nullptr;
  void* phi = nullptr;   // phi[phi_cur] = phi^(n-1)
  void* temp = nullptr;  // u^n
  int64_t step = 0;
  int phi_cur = 0;
};

}  // namespace

namespace mke {

cudaError_t engine_backward(Engine& e, const double* h_target, int64_t steps, int64_t every, double* out,
                            std::string& err) {
  if (e.p.model != MK_MODEL_THERMAL_DENDRITE) {
    err = "mk_backward: thermal dendrite cases only";
    return cudaErrorInvalidValue;
  }
  if (e.p.precision != MK_PREC_FP64 && e.p.precision != MK_PREC_FP32) {
    err = "mk_backward: FP64 or FP32 storage only";
    return cudaErrorInvalidValue;
  }
  if (steps < 1 || !h_target) {
    err = "mk_backward: needs a target and at least one loop";
    return cudaErrorInvalidValue;
  }
  const int64_t K = every > 0 ? every : 100;
  const bool f64 = e.p.precision == MK_PREC_FP64;
  const size_t b0 = (size_t)e.Q0 * e.stride * e.elem, b1 = (size_t)e.Q1 * e.stride * e.elem;
  const size_t bs = (size_t)e.ncell * e.phi_elem;
  const int64_t nrev = steps - 1;  // reverse loops n = steps-2 .. 0
  const int64_t nck = nrev > 0 ? (nrev - 1) / K + 1 : 0;
  const int64_t nseg = nrev > 0 ? std::min<int64_t>(K, nrev) + 1 : 0;
  std::vector<void*> owned;
  cudaError_t st = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) -> cudaError_t {
    cudaError_t s = cudaMalloc(p, bytes);
    if (s == cudaSuccess) owned.push_back(*p);
    return s;
  };
  auto cleanup = [&]() {
    cudaStreamSynchronize(e.stream);
    for (void* p : owned) cudaFree(p);
  };
  auto alloc_snap = [&](Snap& s) -> cudaError_t {
    cudaError_t r;
    if ((r = alloc(&s.pop0, b0)) != cudaSuccess) return r;
    if ((r = alloc(&s.pop1, b1)) != cudaSuccess) return r;
    if ((r = alloc(&s.phi, bs)) != cudaSuccess) return r;
    return alloc(&s.temp, bs);
  };
  auto take = [&](Snap& s) -> cudaError_t {
    cudaError_t r;
    if ((r = cudaMemcpyAsync(s.pop0, e.pop0, b0, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(s.pop1, e.pop1, b1, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(s.phi, e.phi[e.phi_cur], bs, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess)
      return r;
    if ((r = cudaMemcpyAsync(s.temp, e.temp, bs, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    s.step = e.step;
    s.phi_cur = e.phi_cur;
    return cudaSuccess;
  };
  auto put = [&](const Snap& s) -> cudaError_t {
    cudaError_t r;
    if ((r = cudaMemcpyAsync(e.pop0, s.pop0, b0, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(e.pop1, s.pop1, b1, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(e.phi[s.phi_cur], s.phi, bs, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess)
      return r;
    if ((r = cudaMemcpyAsync(e.temp, s.temp, bs, cudaMemcpyDeviceToDevice, e.stream)) != cudaSuccess) return r;
    e.step = s.step;
    e.phi_cur = s.phi_cur;
    return cudaSuccess;
  };
#define MK_TRY(x)             \
  if ((st = (x)) != cudaSuccess) { \
    cleanup();                \
    return st;                \
  }
  std::vector<Snap> ck((size_t)nck), seg((size_t)nseg);
  Snap fin;
  for (Snap& s : ck) MK_TRY(alloc_snap(s));
  for (Snap& s : seg) MK_TRY(alloc_snap(s));
  MK_TRY(alloc_snap(fin));
  // adjoint planes (FP64, logical layout q * stride + cell)
  const size_t pl = (size_t)e.stride * sizeof(double);
  double *Lg[2], *Lt[2], *LP[2], *LU[2], *Lph, *Gb, *target, *partial, *acc;
  for (int b = 0; b < 2; ++b) {
    MK_TRY(alloc((void**)&Lg[b], 7 * pl));
    MK_TRY(alloc((void**)&Lt[b], 7 * pl));
    MK_TRY(alloc((void**)&LP[b], pl));
    MK_TRY(alloc((void**)&LU[b], pl));
  }
  MK_TRY(alloc((void**)&Lph, pl));
  MK_TRY(alloc((void**)&Gb, 3 * pl));
  MK_TRY(alloc((void**)&target, (size_t)e.ncell * sizeof(double)));
  const dim3 block(BX, BY, 1), grid((e.nx + BX - 1) / BX, (e.ny + BY - 1) / BY, e.nz);
  const int nblocks = (int)(grid.x * grid.y * grid.z);
  MK_TRY(alloc((void**)&partial, (size_t)nblocks * 2 * sizeof(double)));
  // acc: [0] dL/deps4, [1] dL/domega_T, [2] loss, [4] -dL/dDelta ([3], [5] unused)
  MK_TRY(alloc((void**)&acc, 6 * sizeof(double)));
  MK_TRY(cudaMemsetAsync(acc, 0, 6 * sizeof(double), e.stream));
  MK_TRY(cudaMemcpyAsync(target, h_target, (size_t)e.ncell * sizeof(double), cudaMemcpyHostToDevice, e.stream));

  // 1. forward with checkpoints
  for (int64_t n = 0; n < steps; ++n) {
    if (n < nrev && n % K == 0) MK_TRY(take(ck[(size_t)(n / K)]));
    MK_TRY(engine_step(e, nullptr));
  }
  MK_TRY(take(fin));

  Geom g;
  g.nx = e.nx;
  g.ny = e.ny;
  g.nz = e.nz;
  g.bc0 = e.p.bc[0];
  g.bc1 = e.p.bc[1];
  g.bc2 = e.p.bc[2];
  g.stride = e.stride;
  AdjK k;
  const double D0 = e.p.W0 * e.p.W0 / e.p.tau0;
  k.om_g = 1.0 / (4.0 * D0 + 0.5);
  k.om_t = 1.0 / (4.0 * e.p.D + 0.5);
  k.fo = (1.0 - 0.5 * k.om_g) / 0.25;
  k.inv_tau0 = 1.0 / e.p.tau0;
  k.lambda = e.p.lambda;
  k.eps4 = e.p.eps4;
  k.eps2 = e.p.eps2;
  k.aniso = e.p.aniso;
  k.nobj = e.p.n_objects;

  // 2. loss and seed (phi after the last loop)
  if (f64)
    k_adj_seed<double><<<grid, block, 0, e.stream>>>((const double*)e.phi[e.phi_cur], target, g, Lg[0], Lt[0], LP[0],
                                                     LU[0], partial);
  else
    k_adj_seed<float><<<grid, block, 0, e.stream>>>((const float*)e.phi[e.phi_cur], target, g, Lg[0], Lt[0], LP[0],
                                                    LU[0], partial);
  k_adj_final<<<1, 256, 0, e.stream>>>(partial, nblocks, acc + 2);
  MK_TRY(cudaGetLastError());

  // 3. reverse, segment by segment
  int cur = 0;  // adjoints of loop n + 1 live in [cur]
  for (int64_t kk = nck - 1; kk >= 0; --kk) {
    const int64_t s0 = kk * K, s1 = std::min<int64_t>(s0 + K, nrev);  // reverse loops s1-1 .. s0
    MK_TRY(put(ck[(size_t)kk]));
    MK_TRY(take(seg[0]));
    for (int64_t n = s0; n < s1; ++n) {
      MK_TRY(engine_step(e, nullptr));
      MK_TRY(take(seg[(size_t)(n - s0 + 1)]));
    }
    for (int64_t n = s1 - 1; n >= s0; --n) {
      const Snap& X = seg[(size_t)(n - s0)];
      const Snap& Xn = seg[(size_t)(n - s0 + 1)];
      const int nxt = 1 - cur;
      const int par = (int)(X.step & 1);
#define MK_ADJ_CELL(S, P, PAR)                                                                                    \
  k_adj_cell<S, P, PAR><<<grid, block, 0, e.stream>>>(                                                           \
      (const S*)X.pop1, (const P*)X.phi, (const P*)X.temp, (const P*)Xn.phi, e.grain, e.seeds, Lg[cur], Lt[cur], \
      LP[cur], LU[cur], Lg[nxt], Lt[nxt], LP[nxt], LU[nxt], Lph, Gb, partial, g, k)
      if (f64) {
        if (par == 0)
          MK_ADJ_CELL(double, double, 0);
        else
          MK_ADJ_CELL(double, double, 1);
      } else {
        if (par == 0)
          MK_ADJ_CELL(float, float, 0);
        else
          MK_ADJ_CELL(float, float, 1);
      }
#undef MK_ADJ_CELL
      k_adj_final<<<1, 256, 0, e.stream>>>(partial, nblocks, acc);
      k_adj_phi<<<grid, block, 0, e.stream>>>(Lph, Gb, Lg[nxt], LP[nxt], g);
      MK_TRY(cudaGetLastError());
      cur = nxt;
    }
  }
  // 4. dL/dDelta from the adjoints of loop 0's streamed t and u
  k_adj_delta<<<grid, block, 0, e.stream>>>(Lt[cur], LU[cur], g, partial);
  k_adj_final<<<1, 256, 0, e.stream>>>(partial, nblocks, acc + 4);
  MK_TRY(cudaGetLastError());
  double h_acc[6] = {0, 0, 0, 0, 0, 0};
  MK_TRY(cudaMemcpyAsync(h_acc, acc, 6 * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
  // 5. leave the state after the forward run
  MK_TRY(put(fin));
  MK_TRY(cudaStreamSynchronize(e.stream));
#undef MK_TRY
  out[0] = h_acc[2];                        // loss
  out[1] = h_acc[0];                        // dL/deps4
  out[2] = -h_acc[4];                       // dL/dDelta
  out[3] = -k.om_t * k.om_t * h_acc[1];     // dL/dtau_T
  out[4] = (double)(steps + nrev);          // forward loops run (first pass + recompute)
  cleanup();
  return cudaSuccess;
}

}  // namespace mke
