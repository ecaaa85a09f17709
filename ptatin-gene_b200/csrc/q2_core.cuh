// Element-level arithmetic of the Q2-P1disc Stokes operator, shared by the
// CUDA kernels and by the host-compiled self-check (tests/test_core_host.py
// compiles this header with g++).  Everything here is per element and
// register-resident; the kernels decide how elements map to threads.
//
// Notation (same as the reference's tensor path, src/stokes_operators_tensor.c):
//   node n = k*9 + j*3 + i  (i along xi, j along eta, k along zeta)
//   qp   q = a*9 + b*3 + c  (c along xi, b along eta, a along zeta)
//   B[q][n] = Q2 Lagrange basis n at Gauss node q     (tensor.c:195-198)
//   D[q][n] = its derivative                          (tensor.c:199-201)
//
// Instead of the reference's three D(x)B(x)B contractions per gradient
// (tensor.c:246-255, 9 contractions of 3 stages each) the field is first
// interpolated to the Gauss points with B(x)B(x)B and then differentiated
// with the collocation matrix Dc = D B^-1 along each axis.  Dc B = D holds
// exactly, so grad = Dc_axis (B(x)B(x)B) in exact arithmetic; it costs 6
// one-dimensional passes per field instead of 9 and exploits B's sparse
// middle row (the middle Gauss point is the middle node: B[1] = [0,1,0]).
// The transpose uses (B(x)B(x)B)^T (sum_d Dc_d^T dv_d).
//
// The quadrature-point action uses the adjugate of J (J^-1 = adj/det), so
// one reciprocal per point replaces the reference's nine scaled cofactors
// (tensor.c:94-179):  with A = adj(J) grad_xi(u) = det * grad_x(u),
//   dv[k][l] = (w eta / det) * sum_j (A + A^T)[j][l] adj[j][k].
#pragma once

#ifdef __CUDACC__
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD inline
#endif

namespace q2 {

// sqrt(3/5), correctly rounded.
constexpr double GS = 0.77459666924148337704;
// B rows 0 and 2 (row 1 is [0, 1, 0]); B[2][n] = B[0][2-n].
constexpr double B0 = 0.5 * (0.6 + GS);
constexpr double B1 = 0.4;
constexpr double B2 = 0.5 * (0.6 - GS);
// Collocation derivative at the Gauss points:
//   Dc = [[-3h, 4h, -h], [-h, 0, h], [h, -4h, 3h]],  h = 1/(2 sqrt(3/5)).
constexpr double DH = 0.5 / GS;
constexpr double W0 = 5.0 / 9.0;
constexpr double W1 = 8.0 / 9.0;

// ---------------------------------------------------------------------------
// One-dimensional passes on a line (x0, x1, x2) with stride S inside an array.
// ---------------------------------------------------------------------------

// y = B x
template <typename T>
PT_HD void lineB(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T b0 = T(B0), b1 = T(B1), b2 = T(B2);
  const T m = b1 * x1;
  y0 = b0 * x0 + (m + b2 * x2);
  y1 = x1;
  y2 = b2 * x0 + (m + b0 * x2);
}

// y = B^T x
template <typename T>
PT_HD void lineBt(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T b0 = T(B0), b1 = T(B1), b2 = T(B2);
  y0 = b0 * x0 + b2 * x2;
  y1 = b1 * (x0 + x2) + x1;
  y2 = b2 * x0 + b0 * x2;
}

// y = Dc x
template <typename T>
PT_HD void lineD(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T h = T(DH);
  const T d = x2 - x0;              // Dc row 1: h (x2 - x0)
  const T t = (x0 + x2) - T(2) * x1;  // second difference
  y1 = h * d;
  y0 = y1 - T(2) * h * t;           // -3h x0 + 4h x1 - h x2
  y2 = y1 + T(2) * h * t;           //  h x0 - 4h x1 + 3h x2
}

// y (+)= Dc^T x
template <typename T, bool ACC>
PT_HD void lineDt(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T h = T(DH);
  const T o = x0 - x2;
  const T s = (x0 + x1) + x2;
  // Dc^T = [[-3h, -h, h], [4h, 0, -4h], [-h, h, 3h]]
  const T r0 = -(h * s) - T(2) * h * o;
  const T r1 = T(4) * h * o;
  const T r2 = (h * s) - T(2) * h * o;
  if (ACC) { y0 += r0; y1 += r1; y2 += r2; }
  else { y0 = r0; y1 = r1; y2 = r2; }
}

// ---------------------------------------------------------------------------
// 3-D passes on 27-value element arrays.
// ---------------------------------------------------------------------------

// I = (B x B x B) f  (nodes -> Gauss points)
template <typename T>
PT_HD void interp(const T f[27], T I[27])
{
  T t[27];
#pragma unroll
  for (int kj = 0; kj < 9; kj++)  // along i (xi)
    lineB(f[3 * kj], f[3 * kj + 1], f[3 * kj + 2], t[3 * kj], t[3 * kj + 1], t[3 * kj + 2]);
#pragma unroll
  for (int k = 0; k < 3; k++)  // along j (eta)
#pragma unroll
    for (int c = 0; c < 3; c++)
      lineB(t[9 * k + c], t[9 * k + 3 + c], t[9 * k + 6 + c], I[9 * k + c], I[9 * k + 3 + c], I[9 * k + 6 + c]);
#pragma unroll
  for (int bc = 0; bc < 9; bc++)  // along k (zeta)
    lineB(I[bc], I[9 + bc], I[18 + bc], t[bc], t[9 + bc], t[18 + bc]);
#pragma unroll
  for (int q = 0; q < 27; q++) I[q] = t[q];
}

// g[d] = Dc along axis d of I (d = 0 xi, 1 eta, 2 zeta)
template <typename T>
PT_HD void grad_colloc(const T I[27], T g0[27], T g1[27], T g2[27])
{
#pragma unroll
  for (int ab = 0; ab < 9; ab++)
    lineD(I[3 * ab], I[3 * ab + 1], I[3 * ab + 2], g0[3 * ab], g0[3 * ab + 1], g0[3 * ab + 2]);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      lineD(I[9 * a + c], I[9 * a + 3 + c], I[9 * a + 6 + c], g1[9 * a + c], g1[9 * a + 3 + c], g1[9 * a + 6 + c]);
#pragma unroll
  for (int bc = 0; bc < 9; bc++)
    lineD(I[bc], I[9 + bc], I[18 + bc], g2[bc], g2[9 + bc], g2[18 + bc]);
}

// r = sum_d Dc_d^T v_d
template <typename T>
PT_HD void grad_colloc_t(const T v0[27], const T v1[27], const T v2[27], T r[27])
{
#pragma unroll
  for (int ab = 0; ab < 9; ab++)
    lineDt<T, false>(v0[3 * ab], v0[3 * ab + 1], v0[3 * ab + 2], r[3 * ab], r[3 * ab + 1], r[3 * ab + 2]);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      lineDt<T, true>(v1[9 * a + c], v1[9 * a + 3 + c], v1[9 * a + 6 + c], r[9 * a + c], r[9 * a + 3 + c], r[9 * a + 6 + c]);
#pragma unroll
  for (int bc = 0; bc < 9; bc++)
    lineDt<T, true>(v2[bc], v2[9 + bc], v2[18 + bc], r[bc], r[9 + bc], r[18 + bc]);
}

// f = (B x B x B)^T r  (Gauss points -> nodes)
template <typename T>
PT_HD void interp_t(const T r[27], T f[27])
{
  T t[27];
#pragma unroll
  for (int bc = 0; bc < 9; bc++)
    lineBt(r[bc], r[9 + bc], r[18 + bc], t[bc], t[9 + bc], t[18 + bc]);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      lineBt(t[9 * k + c], t[9 * k + 3 + c], t[9 * k + 6 + c], f[9 * k + c], f[9 * k + 3 + c], f[9 * k + 6 + c]);
#pragma unroll
  for (int kj = 0; kj < 9; kj++)
    lineBt(f[3 * kj], f[3 * kj + 1], f[3 * kj + 2], t[3 * kj], t[3 * kj + 1], t[3 * kj + 2]);
#pragma unroll
  for (int n = 0; n < 27; n++) f[n] = t[n];
}

// Tensor-product Gauss weight of qp q.
PT_HD double weight(int q)
{
  const int a = q / 9, b = (q / 3) % 3, c = q % 3;
  const double w[3] = {W0, W1, W0};
  return w[a] * w[b] * w[c];
}

// adj(J) and det(J) for J[d][l] = d x_l / d xi_d.
template <typename T>
PT_HD T adjugate(const T J[3][3], T adj[3][3])
{
  adj[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  adj[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  adj[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  adj[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  adj[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  adj[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  adj[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  adj[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  adj[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  return J[0][0] * adj[0][0] + J[0][1] * adj[1][0] + J[0][2] * adj[2][0];
}

// Viscous quadrature action at one point:
//   in  Gu[d][l] = d u_l / d xi_d, adj/c with c = w*eta/det
//   out dv[k][l] = c * sum_j (A + A^T)[j][l] adj[j][k],  A = adj Gu
template <typename T>
PT_HD void qp_viscous(const T adj[3][3], T c, const T Gu[3][3], T dv[3][3])
{
  T A[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) A[k][l] = adj[k][0] * Gu[0][l] + adj[k][1] * Gu[1][l] + adj[k][2] * Gu[2][l];
  const T c2 = c + c;
  T S[3][3];
  S[0][0] = c2 * A[0][0];
  S[1][1] = c2 * A[1][1];
  S[2][2] = c2 * A[2][2];
  S[0][1] = S[1][0] = c * (A[0][1] + A[1][0]);
  S[0][2] = S[2][0] = c * (A[0][2] + A[2][0]);
  S[1][2] = S[2][1] = c * (A[1][2] + A[2][1]);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) dv[k][l] = S[0][l] * adj[0][k] + S[1][l] * adj[1][k] + S[2][l] * adj[2][k];
}

}  // namespace q2
