// Gauss-point viscosity and density from material points: the reference's
// default coefficient projection (coefficient_projection_type 1, "Q1") on one
// rank, src/material_point_utils.c:1090-1190 and 957-1088.
//
//   node sums over the markers of each element:  A1 += N_i eta_p,
//   A2 += N_i rho_p, B += N_i, with N_i the Q1 basis at the marker's local
//   coordinates on the element's 8 vertices (Q2 nodes 0,2,6,8,18,20,24,26)
//   and 1 on its other 19 nodes;  A1 /= B, A2 /= B;  at each Gauss point the
//   Q1 interpolant of the vertex values, clamped to the range of the
//   element's 27 node values.
//
// Deterministic without atomics: markers are sorted by element (stable radix
// sort, so each element keeps its markers in input order), one warp sums an
// element's markers into per-element node partials (lane = node), and a
// per-node gather adds the (<= 8) element partials in a fixed order.  Node
// arrays are indexed compactly over the element box's own nodes.
#pragma once

#include <cstdint>

namespace ptk {

// Q1 basis of pTatinConstructNI_Q1_3D (src/material_point_utils.c:503-520),
// vertex v = k*4 + j*2 + i.
__device__ __forceinline__ double mk_q1(int v, double x, double y, double z)
{
  const double a = (v & 1) ? 1.0 + x : 1.0 - x;
  const double b = (v & 2) ? 1.0 + y : 1.0 - y;
  const double c = (v & 4) ? 1.0 + z : 1.0 - z;
  return 0.125 * a * b * c;
}

// Q2 node of vertex v
__device__ __forceinline__ int mk_vertex_node(int v) { return 2 * (v & 1) + 6 * ((v >> 1) & 1) + 18 * (v >> 2); }

// Sort keys and payload: key = element index, with every index outside
// [0, nel) mapped to nel so that a radix sort over the bits of nel suffices;
// payload = marker index.
__global__ void mk_keys_kernel(const int32_t *__restrict__ wil, int64_t n, int32_t nel, int32_t *__restrict__ key,
                               int32_t *__restrict__ idx)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t w = wil[i];
    key[i] = (w >= 0 && w < nel) ? w : nel;
    idx[i] = (int32_t)i;
  }
}

// start[e] = first sorted position with key >= e, e = 0..nel
__global__ void mk_starts_kernel(const int32_t *__restrict__ keys, int64_t n, int64_t nel, int64_t *__restrict__ start)
{
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e <= nel; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < e) lo = mid + 1;
      else hi = mid;
    }
    start[e] = lo;
  }
}

// One warp per element, lane i < 27 = node i: part[(e*27 + i)*3 + {0,1,2}] =
// sums over the element's markers of (N_i eta, N_i rho, N_i).  The warp reads
// up to 32 markers at a time (one per lane) and broadcasts them, so the sum
// over markers runs in marker order without a chain of dependent loads.
__global__ void __launch_bounds__(128) mk_element_kernel(int64_t nel, const int64_t *__restrict__ start,
                                                         const int32_t *__restrict__ order,
                                                         const double *__restrict__ xi, const double *__restrict__ eta,
                                                         const double *__restrict__ rho, double *__restrict__ part)
{
  const int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= nel) return;  // whole warp
  // lane's vertex (or -1): nodes 0,2,6,8,18,20,24,26 are vertices 0..7
  const int c = lane % 3, b = (lane / 3) % 3, a = lane / 9;
  const int v = (lane < 27 && c != 1 && b != 1 && a != 1) ? (c >> 1) + 2 * (b >> 1) + 4 * (a >> 1) : -1;
  double s1 = 0.0, s2 = 0.0, sb = 0.0;
  const int64_t m0 = start[e], m1 = start[e + 1];
  for (int64_t c0 = m0; c0 < m1; c0 += 32) {
    const int cnt = (int)min((int64_t)32, m1 - c0);
    double x0 = 0.0, x1 = 0.0, x2 = 0.0, ee = 0.0, rr = 0.0;
    if (lane < cnt) {
      const int64_t p = order[c0 + lane];
      x0 = xi[3 * p];
      x1 = xi[3 * p + 1];
      x2 = xi[3 * p + 2];
      ee = eta[p];
      rr = rho[p];
    }
    for (int k = 0; k < cnt; k++) {
      const double y0 = __shfl_sync(0xffffffffu, x0, k), y1 = __shfl_sync(0xffffffffu, x1, k);
      const double y2 = __shfl_sync(0xffffffffu, x2, k), ek = __shfl_sync(0xffffffffu, ee, k);
      const double rk = __shfl_sync(0xffffffffu, rr, k);
      const double N = v >= 0 ? mk_q1(v, y0, y1, y2) : 1.0;
      s1 += N * ek;
      s2 += N * rk;
      sb += N;
    }
  }
  if (lane < 27) {
    double *o = part + (e * 27 + lane) * 3;
    o[0] = s1;
    o[1] = s2;
    o[2] = sb;
  }
}

// Per node of the element box (compact index i + j X + k X Y, X = 2mx+1):
// add the element partials in a fixed order, divide.
__global__ void mk_node_kernel(int mx, int my, int mz, const double *__restrict__ part, double *__restrict__ v1,
                               double *__restrict__ v2)
{
  // node count < 2^31 (checked by the caller): 32-bit index arithmetic
  const unsigned X = 2 * mx + 1, Y = 2 * my + 1;
  const unsigned nn = X * Y * (2 * mz + 1);
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += gridDim.x * blockDim.x) {
    const unsigned txy = t / X;
    const int i = (int)(t - txy * X), j = (int)(txy % Y), k = (int)(txy / Y);
    int ex[2], lx[2], nx = 0, ey[2], ly[2], ny = 0, ez[2], lz[2], nz = 0;
    if (i & 1) { ex[0] = i >> 1; lx[0] = 1; nx = 1; }
    else {
      if (i > 0) { ex[nx] = (i >> 1) - 1; lx[nx++] = 2; }
      if ((i >> 1) < mx) { ex[nx] = i >> 1; lx[nx++] = 0; }
    }
    if (j & 1) { ey[0] = j >> 1; ly[0] = 1; ny = 1; }
    else {
      if (j > 0) { ey[ny] = (j >> 1) - 1; ly[ny++] = 2; }
      if ((j >> 1) < my) { ey[ny] = j >> 1; ly[ny++] = 0; }
    }
    if (k & 1) { ez[0] = k >> 1; lz[0] = 1; nz = 1; }
    else {
      if (k > 0) { ez[nz] = (k >> 1) - 1; lz[nz++] = 2; }
      if ((k >> 1) < mz) { ez[nz] = k >> 1; lz[nz++] = 0; }
    }
    double a1 = 0.0, a2 = 0.0, b = 0.0;
    for (int cz = 0; cz < nz; cz++)
      for (int cy = 0; cy < ny; cy++)
        for (int cx = 0; cx < nx; cx++) {
          const int64_t e = ex[cx] + (int64_t)mx * (ey[cy] + (int64_t)my * ez[cz]);
          const double *o = part + (e * 27 + lx[cx] + 3 * ly[cy] + 9 * lz[cz]) * 3;
          a1 += o[0];
          a2 += o[1];
          b += o[2];
        }
    v1[t] = a1 / b;
    v2[t] = a2 / b;
  }
}

// Gauss point q of element e: Q1 interpolant of the vertex values, clamped to
// the element's 27 node values.  One warp per element: lane n < 27 reads node
// n once, the range is a warp reduction, the vertex values are broadcast, and
// lane q writes Gauss point q.  Abscissae of QuadratureCreateGauss_3pnt_3D
// (src/quadrature.c:136-167).
__global__ void __launch_bounds__(128) mk_qp_kernel(int mx, int my, int mz, const double *__restrict__ v1,
                                                    const double *__restrict__ v2, double *__restrict__ eta_qp,
                                                    double *__restrict__ rho_qp)
{
  // element count < 2^31 (checked by the caller): 32-bit index arithmetic
  const unsigned nel = (unsigned)mx * my * mz;
  const unsigned e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= nel) return;  // whole warp
  const int X = 2 * mx + 1, Y = 2 * my + 1;
  const unsigned exy = e / mx;
  const int ei = (int)(e - exy * mx), ej = (int)(exy % my), ek = (int)(exy / my);
  const int64_t base = 2 * (int64_t)ei + 2 * (int64_t)ej * X + 2 * (int64_t)ek * X * Y;
  // lanes 27..31 read node 0 again, so the range reduction needs no sentinel
  const int n = lane < 27 ? lane : 0;
  const int64_t nd = base + (n % 3) + ((n / 3) % 3) * (int64_t)X + (n / 9) * (int64_t)X * Y;
  const double a = v1[nd], b = v2[nd];
  double lo1 = a, hi1 = a, lo2 = b, hi2 = b;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo1 = fmin(lo1, __shfl_xor_sync(0xffffffffu, lo1, o));
    hi1 = fmax(hi1, __shfl_xor_sync(0xffffffffu, hi1, o));
    lo2 = fmin(lo2, __shfl_xor_sync(0xffffffffu, lo2, o));
    hi2 = fmax(hi2, __shfl_xor_sync(0xffffffffu, hi2, o));
  }
  const double g[3] = {-0.774596669241483, 0.0, 0.774596669241483};
  const double x = g[n % 3], y = g[(n / 3) % 3], z = g[n / 9];
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const int vn = mk_vertex_node(v);
    const double N = mk_q1(v, x, y, z);
    s1 += N * __shfl_sync(0xffffffffu, a, vn);
    s2 += N * __shfl_sync(0xffffffffu, b, vn);
  }
  if (lane >= 27) return;
  if (s1 < lo1) s1 = lo1;
  if (s1 > hi1) s1 = hi1;
  if (s2 < lo2) s2 = lo2;
  if (s2 > hi2) s2 = hi2;
  if (eta_qp) eta_qp[27 * (int64_t)e + lane] = s1;
  if (rho_qp) rho_qp[27 * (int64_t)e + lane] = s2;
}

}  // namespace ptk
