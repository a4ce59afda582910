// mk_interface.cu — the phi = iso interface on the device: contour points and
// tip lengths, in place of the ParaView contour step of the reference's
// post-processing (SaveContourBatch.py: Contour of `order_parameter` at 0 on
// each fluid_t<loops>.vtk, saved as loops<loops>.csv).
//
// Contour points are the vertices a marching-cubes contour of the VTK grid
// places before triangulation: one per grid edge (cell c to c + e_a, a = x, y,
// z, no periodic wrap — the VTK grid has none) whose end values straddle the
// iso value, at a + t e_a with t = (iso - phi_a) / (phi_b - phi_a), in the VTK
// coordinates (cell index + 0.5).  Point order is deterministic: by cell
// index, then axis — each block counts its points, the host scans the block
// counts, and each block writes its points at its offset in thread order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mk_device.cuh"
#include "mk_engine.hpp"

using namespace mkd;

namespace {

constexpr int kThreads = 256;

// Edge crossings of the cell c = (x, y, z) along +x, +y, +z (bit a set when
// the edge along axis a crosses).
template <class P>
__device__ __forceinline__ unsigned cell_crossings(const P* __restrict__ phi, int nx, int ny, int nz, int64_t c,
                                                   double iso, double (&t)[3]) {
  const int x = (int)(c % nx);
  const int64_t r = c / nx;
  const int y = (int)(r % ny), z = (int)(r / ny);
  const double a = double(phi[c]);
  const bool ia = a < iso;
  unsigned m = 0u;
  const bool has[3] = {x + 1 < nx, y + 1 < ny, z + 1 < nz};
  const int64_t off[3] = {1, (int64_t)nx, (int64_t)nx * ny};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    t[k] = 0.0;
    if (!has[k]) continue;
    const double b = double(phi[c + off[k]]);
    if ((b < iso) != ia) {
      m |= 1u << k;
      t[k] = (iso - a) / (b - a);
    }
  }
  return m;
}

template <class P>
__global__ void __launch_bounds__(kThreads) k_iface_count(const P* __restrict__ phi, int nx, int ny, int nz,
                                                          int64_t n, double iso, int* __restrict__ counts) {
  const int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  int k = 0;
  if (c < n) {
    double t[3];
    k = __popc(cell_crossings(phi, nx, ny, nz, c, iso, t));
  }
  __shared__ int sh[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) k += __shfl_down_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
    counts[blockIdx.x] = s;
  }
}

// Writes 4 doubles per point (x, y, z, interpolated scalar or 0) at
// offsets[block] + the exclusive prefix of the block's threads.
template <class P>
__global__ void __launch_bounds__(kThreads) k_iface_write(const P* __restrict__ phi, const P* __restrict__ sc,
                                                          int nx, int ny, int nz, int64_t n, double iso,
                                                          const int64_t* __restrict__ offsets,
                                                          double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  unsigned m = 0u;
  double t[3] = {0.0, 0.0, 0.0};
  if (c < n) m = cell_crossings(phi, nx, ny, nz, c, iso, t);
  const int k = __popc(m);
  // exclusive prefix over the block in thread order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = k;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  __shared__ int wsum[kThreads / 32];
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  int base = 0;
  for (int w = 0; w < wid; ++w) base += wsum[w];
  if (!m) return;
  int64_t pos = offsets[blockIdx.x] + base + incl - k;
  const int x = (int)(c % nx);
  const int64_t r = c / nx;
  const int y = (int)(r % ny), z = (int)(r / ny);
  const int64_t off[3] = {1, (int64_t)nx, (int64_t)nx * ny};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!(m & (1u << a))) continue;
    double* o = out + 4 * pos;
    o[0] = x + 0.5 + (a == 0 ? t[a] : 0.0);
    o[1] = y + 0.5 + (a == 1 ? t[a] : 0.0);
    o[2] = z + 0.5 + (a == 2 ? t[a] : 0.0);
    o[3] = sc ? double(sc[c]) + t[a] * (double(sc[c + off[a]]) - double(sc[c])) : 0.0;
    ++pos;
  }
}

// phi along the four grid lines parallel to each axis that surround the line
// through the centre: line (j, l) of axis a runs through (b0 + j, c0 + l) of
// the two other axes.  out holds, per axis, 4 lines of n_a values.
template <class P>
__global__ void k_tip_lines(const P* __restrict__ phi, int nx, int ny, int nz, int bx0, int by0, int bz0, int bx1,
                            int by1, int bz1, double* __restrict__ out) {
  const int n3[3] = {nx, ny, nz};
  const int tot = 4 * (nx + ny + nz);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += gridDim.x * blockDim.x) {
    int a = 0, r = i;
    while (r >= 4 * n3[a]) {
      r -= 4 * n3[a];
      ++a;
    }
    const int line = r / n3[a], k = r - line * n3[a];
    const int j = line & 1, l = line >> 1;
    int x, y, z;
    if (a == 0) {
      x = k;
      y = j ? by1 : by0;
      z = l ? bz1 : bz0;
    } else if (a == 1) {
      y = k;
      x = j ? bx1 : bx0;
      z = l ? bz1 : bz0;
    } else {
      z = k;
      x = j ? bx1 : bx0;
      y = l ? by1 : by0;
    }
    out[i] = double(phi[(int64_t)x + (int64_t)nx * ((int64_t)y + (int64_t)ny * z)]);
  }
}

}  // namespace

namespace mke {

static bool has_order_parameter(const Engine& e) {
  return e.p.model == MK_MODEL_MULTIPHASE || e.p.model == MK_MODEL_THERMAL_DENDRITE ||
         e.p.model == MK_MODEL_SOLUTAL_DENDRITE || e.p.model == MK_MODEL_FLOW_DENDRITE ||
         e.p.model == MK_MODEL_FLOW_SOLUTAL || e.p.model == MK_MODEL_MULTIGRAIN;
}

template <class P>
static cudaError_t interface_t(Engine& e, double iso, double* xyz, double* sc, int64_t capacity, int64_t* count) {
  const P* phi = (const P*)e.phi[e.phi_cur];
  const P* scal = (const P*)e.temp;  // T or C of the dendrite models, else null
  const int64_t n = e.ncell;
  const int nb = (int)((n + kThreads - 1) / kThreads);
  int* d_counts = nullptr;
  int64_t* d_off = nullptr;
  double* d_pts = nullptr;
  cudaError_t st = cudaMalloc((void**)&d_counts, (size_t)nb * sizeof(int));
  if (st != cudaSuccess) return st;
  std::vector<int> counts(nb);
  std::vector<int64_t> off(nb);
  k_iface_count<P><<<nb, kThreads, 0, e.stream>>>(phi, e.nx, e.ny, e.nz, n, iso, d_counts);
  st = cudaGetLastError();
  if (st == cudaSuccess)
    st = cudaMemcpyAsync(counts.data(), d_counts, (size_t)nb * sizeof(int), cudaMemcpyDeviceToHost, e.stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
  int64_t total = 0;
  for (int b = 0; b < nb; ++b) {
    off[b] = total;
    total += counts[b];
  }
  *count = total;
  const int64_t nw = std::min<int64_t>(total, capacity);
  if (st == cudaSuccess && nw > 0) {
    st = cudaMalloc((void**)&d_off, (size_t)nb * sizeof(int64_t));
    if (st == cudaSuccess) st = cudaMalloc((void**)&d_pts, (size_t)total * 4 * sizeof(double));
    if (st == cudaSuccess)
      st = cudaMemcpyAsync(d_off, off.data(), (size_t)nb * sizeof(int64_t), cudaMemcpyHostToDevice, e.stream);
    if (st == cudaSuccess) {
      k_iface_write<P><<<nb, kThreads, 0, e.stream>>>(phi, scal, e.nx, e.ny, e.nz, n, iso, d_off, d_pts);
      st = cudaGetLastError();
    }
    std::vector<double> h((size_t)nw * 4);
    if (st == cudaSuccess)
      st = cudaMemcpyAsync(h.data(), d_pts, (size_t)nw * 4 * sizeof(double), cudaMemcpyDeviceToHost, e.stream);
    if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
    if (st == cudaSuccess)
      for (int64_t i = 0; i < nw; ++i) {
        if (xyz)
          for (int q = 0; q < 3; ++q) xyz[3 * i + q] = h[4 * i + q];
        if (sc) sc[i] = h[4 * i + 3];
      }
  }
  cudaFree(d_counts);
  if (d_off) cudaFree(d_off);
  if (d_pts) cudaFree(d_pts);
  return st;
}

cudaError_t engine_interface(Engine& e, double iso, double* xyz, double* sc, int64_t capacity, int64_t* count) {
  if (!has_order_parameter(e)) return cudaErrorInvalidValue;
  return e.phi_elem == 8 ? interface_t<double>(e, iso, xyz, sc, capacity, count)
                         : interface_t<float>(e, iso, xyz, sc, capacity, count);
}

// Outermost crossing of the sampled line s (inside = s >= iso) walking away
// from the centre coordinate cc in direction dir; the distance from cc, 0 when
// the centre sample is outside, the distance to the last sample when the
// inside reaches the end of the line.
static double ray_length(const std::vector<double>& s, double cc, int dir, double iso) {
  const int n = (int)s.size();
  if (dir > 0) {
    const int k0 = std::max(0, std::min(n - 1, (int)std::ceil(cc)));
    if (s[k0] < iso) return 0.0;
    int k = k0;
    while (k + 1 < n && s[k + 1] >= iso) ++k;
    if (k + 1 >= n) return (n - 1) - cc;
    return k + (s[k] - iso) / (s[k] - s[k + 1]) - cc;
  }
  const int k0 = std::max(0, std::min(n - 1, (int)std::floor(cc)));
  if (s[k0] < iso) return 0.0;
  int k = k0;
  while (k - 1 >= 0 && s[k - 1] >= iso) --k;
  if (k - 1 < 0) return cc;
  return cc - (k - (s[k] - iso) / (s[k] - s[k - 1]));
}

cudaError_t engine_tip(Engine& e, int seed, double iso, double out[6]) {
  if (!has_order_parameter(e) || seed < 0 || seed >= std::max(1, e.p.n_objects)) return cudaErrorInvalidValue;
  const double c[3] = {e.p.n_objects > 0 ? e.p.obj_center[seed][0] : 0.5 * (e.nx - 1),
                       e.p.n_objects > 0 ? e.p.obj_center[seed][1] : 0.5 * (e.ny - 1),
                       e.p.n_objects > 0 ? e.p.obj_center[seed][2] : 0.5 * (e.nz - 1)};
  const int n3[3] = {e.nx, e.ny, e.nz};
  int b0[3], b1[3];
  double w[3];
  for (int a = 0; a < 3; ++a) {
    const double cc = std::min(std::max(c[a], 0.0), (double)(n3[a] - 1));
    b0[a] = (int)std::floor(cc);
    b1[a] = std::min(b0[a] + 1, n3[a] - 1);
    w[a] = cc - b0[a];
  }
  const int tot = 4 * (e.nx + e.ny + e.nz);
  double* d = nullptr;
  cudaError_t st = cudaMalloc((void**)&d, (size_t)tot * sizeof(double));
  if (st != cudaSuccess) return st;
  const int blocks = (tot + 255) / 256;
  if (e.phi_elem == 8)
    k_tip_lines<double><<<blocks, 256, 0, e.stream>>>((const double*)e.phi[e.phi_cur], e.nx, e.ny, e.nz, b0[0],
                                                      b0[1], b0[2], b1[0], b1[1], b1[2], d);
  else
    k_tip_lines<float><<<blocks, 256, 0, e.stream>>>((const float*)e.phi[e.phi_cur], e.nx, e.ny, e.nz, b0[0],
                                                     b0[1], b0[2], b1[0], b1[1], b1[2], d);
  st = cudaGetLastError();
  std::vector<double> h(tot);
  if (st == cudaSuccess)
    st = cudaMemcpyAsync(h.data(), d, (size_t)tot * sizeof(double), cudaMemcpyDeviceToHost, e.stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
  cudaFree(d);
  if (st != cudaSuccess) return st;
  size_t base = 0;
  for (int a = 0; a < 3; ++a) {
    // bilinear weights of the two transverse axes (j along the first, l along the second)
    const int ta = a == 0 ? 1 : 0, tb = a == 2 ? 1 : 2;
    const double wj = w[ta], wl = w[tb];
    const int n = n3[a];
    std::vector<double> s(n);
    for (int k = 0; k < n; ++k) {
      const double v00 = h[base + 0 * n + k], v10 = h[base + 1 * n + k], v01 = h[base + 2 * n + k],
                   v11 = h[base + 3 * n + k];
      s[k] = (1 - wj) * (1 - wl) * v00 + wj * (1 - wl) * v10 + (1 - wj) * wl * v01 + wj * wl * v11;
    }
    out[2 * a] = ray_length(s, c[a], +1, iso);
    out[2 * a + 1] = ray_length(s, c[a], -1, iso);
    base += (size_t)4 * n;
  }
  return cudaSuccess;
}

}  // namespace mke
