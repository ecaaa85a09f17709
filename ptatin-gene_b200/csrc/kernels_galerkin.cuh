// Galerkin coarse-level element matrices for the multigrid hierarchy: the
// reference's OP_TYPE_MFGALERKIN / OP_TYPE_GALERKIN coarse operators
// (src/ptatin_driver_linear_ts.c:64-380, 713-800), built element by element.
//
// On nested Q2 meshes a coarse element E is the union of 8 fine children c,
// and the Q2 interpolation from E's 27 nodes to a child's 27 nodes is local
// to E.  So the Galerkin operator P^T A P is the assembly of coarse element
// matrices
//     A_E = sum_c P_c^T (M_c A_c M_c) P_c,
// with A_c the child's 81x81 matrix, M_c its Dirichlet mask (the fine
// Dirichlet dofs are zeroed by the prolongation and the restriction) and P_c
// = Pz (x) Py (x) Px the child's 1-D interpolation tensor, per component.
// This is the reference's cell problem (MatAssembleMFGalerkin: the fine
// cell's element matrices assembled and PtAP'd with the cell interpolation)
// without forming a global matrix.
//
// A_c comes either from the fine level's quadrature (MF = true: coordinates
// and Gauss-point viscosity, the fine level runs matrix-free) or from the
// fine level's own stored element matrices (MF = false: a Galerkin level
// below another one).  With g_n = adj(J) grad_xi N_n and c = w eta / det J,
//     A[(n,a),(m,b)] = sum_q c_q (delta_ab g_n . g_m + g_n[b] g_m[a]),
// the element matrix of 2 eta eps(u):eps(v).
//
// One CTA of 256 threads per coarse element; matrices in the packed
// symmetric layout of kernels_ebe.cuh, FP64.
#pragma once

#include <cstdint>

#include "kernels_colour.cuh"
#include "kernels_ebe.cuh"
#include "q2_core.cuh"

namespace ptk {

struct GalerkinArgs {
  Box fb;                       // fine level (node strides, element counts)
  int cmx, cmy, cmz;            // coarse level elements per axis
  const double *coords;         // MF: fine node coordinates
  const double *eta;            // MF: fine Gauss-point viscosity [27 nel_f]
  const double *Af;             // !MF: fine element matrices, packed [nel_f][EBE_LD]
  const uint8_t *mask;          // fine Dirichlet mask [3 N_f] or null
  double *Ac;                   // out: coarse element matrices, packed [nel_c][EBE_LD]
};

constexpr int GAL_THREADS = 256;

// smem (doubles): child matrix, work matrix, g table [q][n][3], c[q], child coords
constexpr size_t galerkin_smem_bytes()
{
  return sizeof(double) * (2 * 6561 + 27 * 27 * 3 + 27 + 81) + 96;
}

// 1-D Q2 interpolation from a coarse element's nodes M to child h's nodes m:
// fine node m of child h sits at coarse xi = -1 + h + m/2.
// (m and M are compile-time constants where it is called, so this is a select on h.)
__device__ __forceinline__ double gal_p1(int h, int m, int M)
{
  if (m == 0) return h ? (M == 1 ? 1.0 : 0.0) : (M == 0 ? 1.0 : 0.0);
  if (m == 2) return h ? (M == 2 ? 1.0 : 0.0) : (M == 1 ? 1.0 : 0.0);
  return h ? (M == 0 ? -0.125 : (M == 1 ? 0.75 : 0.375)) : (M == 0 ? 0.375 : (M == 1 ? 0.75 : -0.125));
}

// 1-D Q2 basis (nodes -1, 0, 1) and its derivative at Gauss point p.
__device__ __forceinline__ double gal_n1(int p, int m)
{
  const double x = (p - 1) * q2::GS;
  return m == 0 ? 0.5 * x * (x - 1.0) : (m == 1 ? 1.0 - x * x : 0.5 * x * (x + 1.0));
}
__device__ __forceinline__ double gal_d1(int p, int m)
{
  const double x = (p - 1) * q2::GS;
  return m == 0 ? x - 0.5 : (m == 1 ? -2.0 * x : x + 0.5);
}

// Apply the 1-D interpolation tensor of child (hx, hy, hz) to a 27-vector in
// place, in the transposed direction (fine values in, coarse values out):
// w[M] = sum_m P[m][M] v[m].
__device__ __forceinline__ void gal_pt27(int hx, int hy, int hz, double v[27])
{
  double t[27];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int I = 0; I < 3; I++) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++) s = fma(gal_p1(hx, i, I), v[i + 3 * j + 9 * k], s);
        t[I + 3 * j + 9 * k] = s;
      }
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int J = 0; J < 3; J++)
#pragma unroll
      for (int I = 0; I < 3; I++) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 3; j++) s = fma(gal_p1(hy, j, J), t[I + 3 * j + 9 * k], s);
        v[I + 3 * J + 9 * k] = s;
      }
#pragma unroll
  for (int K = 0; K < 3; K++)
#pragma unroll
    for (int J = 0; J < 3; J++)
#pragma unroll
      for (int I = 0; I < 3; I++) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) s = fma(gal_p1(hz, k, K), v[I + 3 * J + 9 * k], s);
        t[I + 3 * J + 9 * K] = s;
      }
#pragma unroll
  for (int n = 0; n < 27; n++) v[n] = t[n];
}

template <bool MF>
__global__ void __launch_bounds__(GAL_THREADS) galerkin_kernel(GalerkinArgs a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *A = reinterpret_cast<double *>(smem_raw);  // child matrix, then P^T (.) P
  double *B = A + 6561;                              // A P
  double *G = B + 6561;                              // g[q][n][3]
  double *cq = G + 27 * 27 * 3;
  double *xe = cq + 27;
  uint8_t *mk = reinterpret_cast<uint8_t *>(xe + 81);
  const int t = threadIdx.x;
  const int64_t E = blockIdx.x;
  const int I = (int)(E % a.cmx), J = (int)((E / a.cmx) % a.cmy), K = (int)(E / ((int64_t)a.cmx * a.cmy));
  double acc[26];
#pragma unroll
  for (int k = 0; k < 26; k++) acc[k] = 0.0;

#pragma unroll 1
  for (int ch = 0; ch < 8; ch++) {
    const int hx = ch & 1, hy = (ch >> 1) & 1, hz = ch >> 2;
    const int ei = 2 * I + hx, ej = 2 * J + hy, ek = 2 * K + hz;
    const int64_t e = ei + (int64_t)a.fb.mx * (ej + (int64_t)a.fb.my * ek);
    const int64_t node0 = a.fb.off + 2 * (int64_t)ei + 2 * (int64_t)ej * a.fb.X + 2 * (int64_t)ek * a.fb.XY;
    if (t < 81) {
      const int n = t / 3, l = t % 3;
      const int64_t k = 3 * (node0 + (n % 3) + ((n / 3) % 3) * a.fb.X + (n / 9) * a.fb.XY) + l;
      mk[t] = a.mask ? a.mask[k] : 0;
      if (MF) xe[t] = a.coords[k];
    }
    __syncthreads();
    if (MF) {
      // per Gauss point: c = w eta / det and g_n = adj(J) grad_xi N_n
      if (t < 27) {
        const int q = t, pc = q % 3, pb = (q / 3) % 3, pa = q / 9;
        double Jm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int n = 0; n < 27; n++) {
          const int ni = n % 3, nj = (n / 3) % 3, nk = n / 9;
          const double d0 = gal_d1(pc, ni) * gal_n1(pb, nj) * gal_n1(pa, nk);
          const double d1 = gal_n1(pc, ni) * gal_d1(pb, nj) * gal_n1(pa, nk);
          const double d2 = gal_n1(pc, ni) * gal_n1(pb, nj) * gal_d1(pa, nk);
          for (int l = 0; l < 3; l++) {
            const double x = xe[3 * n + l];
            Jm[0][l] = fma(d0, x, Jm[0][l]);
            Jm[1][l] = fma(d1, x, Jm[1][l]);
            Jm[2][l] = fma(d2, x, Jm[2][l]);
          }
        }
        double adj[3][3];
        const double det = q2::adjugate(Jm, adj);
        cq[q] = q2::weight(q) * a.eta[27 * e + q] / det;
        for (int n = 0; n < 27; n++) {
          const int ni = n % 3, nj = (n / 3) % 3, nk = n / 9;
          const double d[3] = {gal_d1(pc, ni) * gal_n1(pb, nj) * gal_n1(pa, nk),
                               gal_n1(pc, ni) * gal_d1(pb, nj) * gal_n1(pa, nk),
                               gal_n1(pc, ni) * gal_n1(pb, nj) * gal_d1(pa, nk)};
          for (int l = 0; l < 3; l++) G[(q * 27 + n) * 3 + l] = adj[l][0] * d[0] + adj[l][1] * d[1] + adj[l][2] * d[2];
        }
      }
      __syncthreads();
      for (int p = t; p < 729; p += GAL_THREADS) {
        const int n = p / 27, m = p % 27;
        double S = 0.0, T[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int q = 0; q < 27; q++) {
          const double *gn = G + (q * 27 + n) * 3, *gm = G + (q * 27 + m) * 3;
          const double c = cq[q];
          const double gn0 = c * gn[0], gn1 = c * gn[1], gn2 = c * gn[2];
          const double gm0 = gm[0], gm1 = gm[1], gm2 = gm[2];
          S = fma(gn0, gm0, fma(gn1, gm1, fma(gn2, gm2, S)));
          T[0][0] = fma(gn0, gm0, T[0][0]); T[0][1] = fma(gn1, gm0, T[0][1]); T[0][2] = fma(gn2, gm0, T[0][2]);
          T[1][0] = fma(gn0, gm1, T[1][0]); T[1][1] = fma(gn1, gm1, T[1][1]); T[1][2] = fma(gn2, gm1, T[1][2]);
          T[2][0] = fma(gn0, gm2, T[2][0]); T[2][1] = fma(gn1, gm2, T[2][1]); T[2][2] = fma(gn2, gm2, T[2][2]);
        }
        // row dof (n, ra), column dof (m, cb): delta S + g_n[cb] g_m[ra]  (T[ra][cb])
#pragma unroll
        for (int ra = 0; ra < 3; ra++)
#pragma unroll
          for (int cb = 0; cb < 3; cb++) {
            const int i = 3 * n + ra, j = 3 * m + cb;
            const double v = (ra == cb ? S : 0.0) + T[ra][cb];
            A[j * 81 + i] = (mk[i] || mk[j]) ? 0.0 : v;
          }
      }
    } else {
      const double *src = a.Af + e * EBE_LD;
      for (int idx = t; idx < 6561; idx += GAL_THREADS) {
        const int j = idx / 81, i = idx - 81 * j;
        A[idx] = (mk[i] || mk[j]) ? 0.0 : src[ebe_sym(i, j)];
      }
    }
    __syncthreads();
    // B = A P: row i, column component b, 27 column nodes -> 27 coarse nodes
    if (t < 243) {
      const int i = t % 81, b = t / 81;
      double v[27];
#pragma unroll
      for (int m = 0; m < 27; m++) v[m] = A[(3 * m + b) * 81 + i];
      gal_pt27(hx, hy, hz, v);
#pragma unroll
      for (int M = 0; M < 27; M++) B[(3 * M + b) * 81 + i] = v[M];
    }
    __syncthreads();
    // A <- P^T B: column j, row component r, 27 row nodes -> 27 coarse nodes
    if (t < 243) {
      const int j = t % 81, r = t / 81;
      double v[27];
#pragma unroll
      for (int n = 0; n < 27; n++) v[n] = B[j * 81 + 3 * n + r];
      gal_pt27(hx, hy, hz, v);
#pragma unroll
      for (int N = 0; N < 27; N++) A[j * 81 + 3 * N + r] = v[N];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 26; k++) {
      const int idx = t + GAL_THREADS * k;
      if (idx < 6561) acc[k] += A[idx];
    }
    __syncthreads();
  }
  // upper triangle, packed (the sum is symmetric up to rounding)
  double *out = a.Ac + E * EBE_LD;
#pragma unroll
  for (int k = 0; k < 26; k++) {
    const int idx = t + GAL_THREADS * k;
    const int j = idx / 81, i = idx - 81 * j;
    if (idx < 6561 && i <= j) out[j * (j + 1) / 2 + i] = acc[k];
  }
  if (t < EBE_LD - 3321) out[3321 + t] = 0.0;
}

template <typename TO>
__global__ void convert_kernel(const double *__restrict__ a, TO *__restrict__ b, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (TO)a[i];
}

}  // namespace ptk
