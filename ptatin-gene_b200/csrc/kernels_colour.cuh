// Element kernels with an 8-colour deterministic scatter.
//
// Elements are split by the parity of (ei, ej, ek); two elements of one
// colour are at least two elements apart along some axis and share no node,
// so one launch per colour can read-modify-write y without atomics and the
// summation order at every node is fixed (colour 0..7).  This replaces the
// reference CUDA back-end's greedy host colouring (src/stokes_operators_cuda.cu:
// 337-397), which yields the same 8 classes on a structured grid.
//
// One thread owns one element; the element's 27 nodes are gathered straight
// from the reference layouts (interleaved coordinates / velocity).
#pragma once

#include <cstdint>

#include "q2_core.cuh"

namespace ptk {

// A rank's element box inside its ghosted local node box.  Element
// (ei, ej, ek) has node n = a*9 + b*3 + c at
//   off + (2ei + c) + (2ej + b) X + (2ek + a) XY,   off = ox + oy X + oz XY
// (the table of src/dmda_element_q2p1.c:395-455 with i = esi-gsi + 2ei).
struct Box {
  int mx, my, mz;
  int64_t X, XY, off;
};

struct ColourGrid {
  Box b;
  int cx, cy, cz;      // colour (parity per axis)
  int ncx, ncy, ncz;   // elements of this colour per axis
};

__host__ inline ColourGrid colour_grid(const Box &b, int colour)
{
  ColourGrid g;
  g.b = b;
  g.cx = colour & 1; g.cy = (colour >> 1) & 1; g.cz = (colour >> 2) & 1;
  g.ncx = (b.mx - g.cx + 1) / 2;
  g.ncy = (b.my - g.cy + 1) / 2;
  g.ncz = (b.mz - g.cz + 1) / 2;
  return g;
}

__device__ __forceinline__ void element_nodes(const Box &bx, int ei, int ej, int ek, int64_t nid[27])
{
  const int64_t base = bx.off + 2 * (int64_t)ei + 2 * (int64_t)ej * bx.X + 2 * (int64_t)ek * bx.XY;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int c = 0; c < 3; c++) nid[9 * a + 3 * b + c] = base + c + b * bx.X + a * bx.XY;
}

__device__ __forceinline__ bool colour_element(const ColourGrid &g, int64_t t, int &ei, int &ej, int &ek)
{
  const int64_t n = (int64_t)g.ncx * g.ncy * g.ncz;
  if (t >= n) return false;
  ei = g.cx + 2 * (int)(t % g.ncx);
  ej = g.cy + 2 * (int)((t / g.ncx) % g.ncy);
  ek = g.cz + 2 * (int)(t / ((int64_t)g.ncx * g.ncy));
  return true;
}

// J[d][l][q] = d x_l / d xi_d at the 27 Gauss points.
template <typename T>
__device__ __forceinline__ void element_jacobian(const T *__restrict__ coords, const int64_t nid[27], T Jg[3][3][27],
                                                 T Xq[3][27])
{
#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    T f[27];
#pragma unroll
    for (int n = 0; n < 27; n++) f[n] = coords[3 * nid[n] + l];
    q2::interp(f, Xq[l]);
    q2::grad_colloc(Xq[l], Jg[0][l], Jg[1][l], Jg[2][l]);
  }
}

// ---------------------------------------------------------------------------
// A11
// ---------------------------------------------------------------------------
template <typename T, bool MASKED>
__global__ void __launch_bounds__(128) a11_colour_kernel(ColourGrid g, const T *__restrict__ coords,
                                                         const T *__restrict__ eta, const T *__restrict__ u,
                                                         const uint8_t *__restrict__ mask, T *__restrict__ y)
{
  int ei, ej, ek;
  if (!colour_element(g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const int64_t e = ei + (int64_t)g.b.mx * (ej + (int64_t)g.b.my * ek);
  int64_t nid[27];
  element_nodes(g.b, ei, ej, ek, nid);

  T Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);

  T Ug[3][3][27];
#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    T f[27], I[27];
#pragma unroll
    for (int n = 0; n < 27; n++) {
      const int64_t k = 3 * nid[n] + l;
      T v = u[k];
      if (MASKED && mask[k]) v = T(0);
      f[n] = v;
    }
    q2::interp(f, I);
    q2::grad_colloc(I, Ug[0][l], Ug[1][l], Ug[2][l]);
  }

#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    T J[3][3], adj[3][3], G[3][3], d[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) {
        J[k][l] = Jg[k][l][q];
        G[k][l] = Ug[k][l][q];
      }
    const T det = q2::adjugate(J, adj);
    const T c = T(q2::weight(q)) * eta[27 * e + q] / det;
    q2::qp_viscous(adj, c, G, d);
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) Ug[k][l][q] = d[k][l];
  }

#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    T r[27], f[27];
    q2::grad_colloc_t(Ug[0][l], Ug[1][l], Ug[2][l], r);
    q2::interp_t(r, f);
#pragma unroll
    for (int n = 0; n < 27; n++) y[3 * nid[n] + l] += f[n];
  }
}

// ---------------------------------------------------------------------------
// diag(A11):  Y[3n+d] += w det eta (|grad N_n|^2 + (dN_n/dx_d)^2)
// (src/stokes_q2p1_mf_operators_diag_def.c:120-205)
// ---------------------------------------------------------------------------

// Reference-coordinate basis gradients at the Gauss points, [q][n][d].
__constant__ double c_dN[27][27][3];

__global__ void __launch_bounds__(128) diag_colour_kernel(ColourGrid g, const double *__restrict__ coords,
                                                          const double *__restrict__ eta, double *__restrict__ y)
{
  int ei, ej, ek;
  if (!colour_element(g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const int64_t e = ei + (int64_t)g.b.mx * (ej + (int64_t)g.b.my * ek);
  int64_t nid[27];
  element_nodes(g.b, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  double acc[27][3];
#pragma unroll
  for (int n = 0; n < 27; n++) acc[n][0] = acc[n][1] = acc[n][2] = 0.0;
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    const double det = q2::adjugate(J, adj);
    // w det eta |adj gN / det|^2 = (w eta / det) |adj gN|^2
    const double c = q2::weight(q) * eta[27 * e + q] / det;
#pragma unroll
    for (int n = 0; n < 27; n++) {
      const double g0 = c_dN[q][n][0], g1 = c_dN[q][n][1], g2 = c_dN[q][n][2];
      const double x0 = adj[0][0] * g0 + adj[0][1] * g1 + adj[0][2] * g2;
      const double x1 = adj[1][0] * g0 + adj[1][1] * g1 + adj[1][2] * g2;
      const double x2 = adj[2][0] * g0 + adj[2][1] * g1 + adj[2][2] * g2;
      const double s0 = x0 * x0, s1 = x1 * x1, s2 = x2 * x2;
      const double tot = (s0 + s1) + s2;
      acc[n][0] += c * (tot + s0);
      acc[n][1] += c * (tot + s1);
      acc[n][2] += c * (tot + s2);
    }
  }
#pragma unroll
  for (int n = 0; n < 27; n++)
#pragma unroll
    for (int d = 0; d < 3; d++) y[3 * nid[n] + d] += acc[n][d];
}

// ---------------------------------------------------------------------------
// P1 "global relative" pressure basis (src/element_utils_q2.c:183-224):
// Np = {1, (x_q - mean)/Lx, (y_q - mean)/Ly, (z_q - mean)/Lz}.
// Returns the per-element offsets/scales; x_q comes from Xq.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void p1grel_frame(const double *__restrict__ coords, const int64_t nid[27],
                                             double mean[3], double invL[3])
{
#pragma unroll
  for (int l = 0; l < 3; l++) {
    double s = 0.0;
#pragma unroll
    for (int n = 0; n < 27; n++) s += coords[3 * nid[n] + l];
    mean[l] = (1.0 / 27.0) * s;
  }
  invL[0] = 1.0 / (coords[3 * nid[14]] - coords[3 * nid[12]]);
  invL[1] = 1.0 / (coords[3 * nid[16] + 1] - coords[3 * nid[10] + 1]);
  invL[2] = 1.0 / (coords[3 * nid[22] + 2] - coords[3 * nid[4] + 2]);
}

// ---------------------------------------------------------------------------
// A21 (B u):  Yp[e,i] = -sum_q w det div(u)_q Np_i(q)
//             = -sum_q w Np_i(q) trace(adj Gu)      (det cancels)
// No scatter conflicts: one thread writes its own 4 pressure dofs.
// ---------------------------------------------------------------------------
template <bool MASKED>
__global__ void __launch_bounds__(128) a21_kernel(Box bx, const double *__restrict__ coords,
                                                  const double *__restrict__ u, const uint8_t *__restrict__ mask,
                                                  double *__restrict__ yp)
{
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)bx.mx * bx.my * bx.mz) return;
  const int ei = (int)(e % bx.mx), ej = (int)((e / bx.mx) % bx.my), ek = (int)(e / ((int64_t)bx.mx * bx.my));
  int64_t nid[27];
  element_nodes(bx, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  double mean[3], invL[3];
  p1grel_frame(coords, nid, mean, invL);

  double Ug[3][3][27];
#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    double f[27], I[27];
#pragma unroll
    for (int n = 0; n < 27; n++) {
      const int64_t k = 3 * nid[n] + l;
      double v = u[k];
      if (MASKED && mask[k]) v = 0.0;
      f[n] = v;
    }
    q2::interp(f, I);
    q2::grad_colloc(I, Ug[0][l], Ug[1][l], Ug[2][l]);
  }
  double Y[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    (void)q2::adjugate(J, adj);
    double tr = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) tr += adj[k][0] * Ug[0][k][q] + adj[k][1] * Ug[1][k][q] + adj[k][2] * Ug[2][k][q];
    const double f = -q2::weight(q) * tr;
    Y[0] += f;
    Y[1] += f * ((Xq[0][q] - mean[0]) * invL[0]);
    Y[2] += f * ((Xq[1][q] - mean[1]) * invL[1]);
    Y[3] += f * ((Xq[2][q] - mean[2]) * invL[2]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) yp[4 * e + i] = Y[i];
}

// ---------------------------------------------------------------------------
// A12 (B^T p):  Yu[n,l] = -sum_q w det p_q dN_n/dx_l,
//   dv[k][l] = -w p_q adj[l][k],  Yu_l = (B x B x B)^T sum_k Dc_k^T dv[k][l]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) a12_colour_kernel(ColourGrid g, const double *__restrict__ coords,
                                                         const double *__restrict__ p, double *__restrict__ yu)
{
  int ei, ej, ek;
  if (!colour_element(g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const int64_t e = ei + (int64_t)g.b.mx * (ej + (int64_t)g.b.my * ek);
  int64_t nid[27];
  element_nodes(g.b, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  double mean[3], invL[3];
  p1grel_frame(coords, nid, mean, invL);
  const double p0 = p[4 * e], p1 = p[4 * e + 1], p2 = p[4 * e + 2], p3 = p[4 * e + 3];
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    (void)q2::adjugate(J, adj);
    const double pq = p0 + p1 * ((Xq[0][q] - mean[0]) * invL[0]) + p2 * ((Xq[1][q] - mean[1]) * invL[1]) +
                      p3 * ((Xq[2][q] - mean[2]) * invL[2]);
    const double s = -q2::weight(q) * pq;
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) Jg[k][l][q] = s * adj[l][k];
  }
#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    double r[27], f[27];
    q2::grad_colloc_t(Jg[0][l], Jg[1][l], Jg[2][l], r);
    q2::interp_t(r, f);
#pragma unroll
    for (int n = 0; n < 27; n++) yu[3 * nid[n] + l] += f[n];
  }
}

// ---------------------------------------------------------------------------
// Body-force load of the momentum residual (src/stokes_form_function.c:201-213):
//   F[n,l] += sum_q w_q det(J_q) N_n(q) Fu_l(q),  fu = [27 nel][3]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) body_force_colour_kernel(ColourGrid g, const double *__restrict__ coords,
                                                                const double *__restrict__ fu, double *__restrict__ F)
{
  int ei, ej, ek;
  if (!colour_element(g, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ei, ej, ek)) return;
  const int64_t e = ei + (int64_t)g.b.mx * (ej + (int64_t)g.b.my * ek);
  int64_t nid[27];
  element_nodes(g.b, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  double wd[27];
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    wd[q] = q2::weight(q) * q2::adjugate(J, adj);
  }
#pragma unroll 1
  for (int l = 0; l < 3; l++) {
    double r[27], f[27];
#pragma unroll
    for (int q = 0; q < 27; q++) r[q] = wd[q] * fu[3 * (27 * e + q) + l];
    q2::interp_t(r, f);
#pragma unroll
    for (int n = 0; n < 27; n++) F[3 * nid[n] + l] += f[n];
  }
}

}  // namespace ptk
