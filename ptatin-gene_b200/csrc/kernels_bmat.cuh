// Stored divergence blocks for B u (A21) and B^T p (A12) on one-rank boxes.
//
// Per element, B_e is the 4 x 81 block of the discrete divergence,
//     B_e[i][3n+l] = -sum_q w_q det J_q Np_i(q) dN_n/dx_l(q)
//                  = -sum_q w_q Np_i(q) (adj(J_q) grad_xi N_n)_l,
// with the P1GRel pressure basis Np = {1, x^, y^, z^} of
// P3D_ConstructNi_P1GRel_3D (src/element_utils_q2.c:183-224): the element
// operator of MatMultMF_Stokes_MixedFEM3d_A21 / _A12
// (src/stokes_q2p1_mf_operators_def.c:423-538).  Row i is the B^T element
// operator of a12_colour_kernel applied to the unit pressure vector e_i,
// stored column-major [e][j][i] (a column's four entries are one 32-byte
// sector), 2.6 KB per element in FP64; it depends on the coordinates only.
//
// B u is then a 4 x 81 GEMV per element (one warp, lanes over the columns, a
// fixed-order warp reduction; no scatter: the pressure dofs are element-local)
// and B^T p a node-centred sum over the (<= 8) elements of each node of their
// 4-term column products, in a fixed order -- both deterministic, both a
// stream over B_e instead of a recomputation of the geometry per apply.
#pragma once

#include <cstdint>

#include "kernels_colour.cuh"
#include "q2_core.cuh"

namespace ptk {

constexpr int BMAT_LD = 324;  // 4 x 81 per element

__global__ void __launch_bounds__(128) bmat_kernel(Box bx, const double *__restrict__ coords, double *__restrict__ Be)
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
  // per Gauss point: Jg[k][l][q] <- -w adj[l][k];  Xq[d][q] <- (x_d(q) - mean_d) / L_d
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    (void)q2::adjugate(J, adj);
    const double s = -q2::weight(q);
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) Jg[k][l][q] = s * adj[l][k];
#pragma unroll
    for (int d = 0; d < 3; d++) Xq[d][q] = (Xq[d][q] - mean[d]) * invL[d];
  }
  double *out = Be + e * BMAT_LD;
#pragma unroll 1
  for (int i = 0; i < 4; i++)
#pragma unroll 1
    for (int l = 0; l < 3; l++) {
      double dv[3][27], r[27], f[27];
#pragma unroll
      for (int k = 0; k < 3; k++)
#pragma unroll
        for (int q = 0; q < 27; q++) dv[k][q] = i == 0 ? Jg[k][l][q] : Jg[k][l][q] * Xq[i - 1][q];
      q2::grad_colloc_t(dv[0], dv[1], dv[2], r);
      q2::interp_t(r, f);
#pragma unroll
      for (int n = 0; n < 27; n++) out[(3 * n + l) * 4 + i] = f[n];
    }
}

// yp[4e+i] = sum_j B_e[i][j] u_j (MASKED: Dirichlet entries of u taken as 0).
// One warp per element.  The block is read as 162 16-byte pairs (B_e[j][0..1]
// or B_e[j][2..3]), 32 consecutive pairs per warp load: even lanes sum rows 0
// and 1, odd lanes rows 2 and 3, then a fixed xor-tree reduction over the
// lanes of each parity.
template <bool MASKED>
__global__ void __launch_bounds__(128) bmat_a21_kernel(Box bx, const double *__restrict__ Be,
                                                       const double *__restrict__ u,
                                                       const uint8_t *__restrict__ mask, double *__restrict__ yp)
{
  const int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= (int64_t)bx.mx * bx.my * bx.mz) return;  // whole warp
  const int ei = (int)(e % bx.mx), ej = (int)((e / bx.mx) % bx.my), ek = (int)(e / ((int64_t)bx.mx * bx.my));
  const int64_t node0 = bx.off + 2 * (int64_t)ei + 2 * (int64_t)ej * bx.X + 2 * (int64_t)ek * bx.XY;
  const double2 *b2 = reinterpret_cast<const double2 *>(Be + e * BMAT_LD);
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int it = 0; it < 6; it++) {
    const int idx = lane + 32 * it;
    if (idx < 162) {
      const int j = idx >> 1, n = j / 3, l = j - 3 * n;
      const int64_t k = 3 * (node0 + (n % 3) + ((n / 3) % 3) * bx.X + (n / 9) * bx.XY) + l;
      double v = u[k];
      if (MASKED && mask[k]) v = 0.0;
      const double2 c = b2[idx];
      s0 = fma(c.x, v, s0);
      s1 = fma(c.y, v, s1);
    }
  }
#pragma unroll
  for (int o = 16; o > 1; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (lane < 2) {
    double *y = yp + 4 * e + 2 * lane;
    y[0] = s0;
    y[1] = s1;
  }
}

// B^T p node by node: y_k = sum over the (<= 8) elements of node k, in the
// order of ebe_gather_kernel, of sum_i B_e[i][j] p[4e+i] (j = the node's dof in
// element e), with no per-element output array (ACC: added to y).
// One-rank boxes (node box = element box).
template <bool ACC>
__global__ void bmat_a12_gather_kernel(Box b, const double *__restrict__ Be, const double *__restrict__ p,
                                       double *__restrict__ y)
{
  const int64_t n = 3 * b.XY * (2 * (int64_t)b.mz + 1);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % 3);
    const int64_t node = t / 3;
    const int i = (int)(node % b.X), j = (int)((node / b.X) % (2 * b.my + 1)), k = (int)(node / b.XY);
    int ex[2], lx[2], nx = 0, ey[2], ly[2], ny = 0, ez[2], lz[2], nz = 0;
    if (i & 1) { ex[0] = i >> 1; lx[0] = 1; nx = 1; }
    else {
      if (i > 0) { ex[nx] = (i >> 1) - 1; lx[nx++] = 2; }
      if ((i >> 1) < b.mx) { ex[nx] = i >> 1; lx[nx++] = 0; }
    }
    if (j & 1) { ey[0] = j >> 1; ly[0] = 1; ny = 1; }
    else {
      if (j > 0) { ey[ny] = (j >> 1) - 1; ly[ny++] = 2; }
      if ((j >> 1) < b.my) { ey[ny] = j >> 1; ly[ny++] = 0; }
    }
    if (k & 1) { ez[0] = k >> 1; lz[0] = 1; nz = 1; }
    else {
      if (k > 0) { ez[nz] = (k >> 1) - 1; lz[nz++] = 2; }
      if ((k >> 1) < b.mz) { ez[nz] = k >> 1; lz[nz++] = 0; }
    }
    double acc = 0.0;
    for (int c = 0; c < nz; c++)
      for (int bb = 0; bb < ny; bb++)
        for (int a = 0; a < nx; a++) {
          const int64_t e = ex[a] + (int64_t)b.mx * (ey[bb] + (int64_t)b.my * ez[c]);
          const double *be = Be + e * BMAT_LD + 4 * (3 * (lx[a] + 3 * ly[bb] + 9 * lz[c]) + l);
          const double2 c01 = *reinterpret_cast<const double2 *>(be);
          const double2 c23 = *reinterpret_cast<const double2 *>(be + 2);
          const double *pe = p + 4 * e;
          acc += fma(c23.y, pe[3], fma(c23.x, pe[2], fma(c01.y, pe[1], c01.x * pe[0])));
        }
    y[t] = ACC ? y[t] + acc : acc;
  }
}

}  // namespace ptk
