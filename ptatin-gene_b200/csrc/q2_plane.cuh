// Quadrature-plane arithmetic of the streaming A11 kernel, host+device so the
// CPU self-check (tests/core_host_check.cpp) runs the same code.
//
// Per element and quadrature plane a (the Gauss point index along zeta):
//   forward   node planes N_k (k = 0..2, 9 values [j*3+i] each) of one velocity
//             component -> the scaled reference gradient at the 9 Gauss points
//             of plane a:  G0 = d/dxi, G1 = d/deta, G2 = d/dzeta, all times 1/h.
//             zeta: Q = sum_k B[a][k] N_k,  R = sum_k (D[a][k]/h) N_k;
//             then (B x B) on Q and R, collocated Dc/h along xi and eta on BxB Q.
//   action    dv = (A + A^T) K with A = K G at each point (K from the set-up).
//   backward  the transpose: contributions C_k (9 values each) to the node
//             planes k = 0..2 of one component.
// With K = h sqrt(w eta / det J) adj(J) the result is exactly the reference's
// element action (src/stokes_operators_tensor.c:181-286); see kernels_stream.cuh.
#pragma once

#include <cmath>

#include "q2_core.cuh"

namespace q2 {

// D/h rows at the Gauss points (h = DH, s = sqrt(3/5)):
//   a=0 [-1.2-s, 2.4, s-1.2], a=1 [-s, 0, s], a=2 [1.2-s, -2.4, 1.2+s]
constexpr double DZ00 = -1.2 - GS, DZ01 = 2.4, DZ02 = GS - 1.2;
constexpr double DZ20 = 1.2 - GS, DZ21 = -2.4, DZ22 = 1.2 + GS;

// y = (Dc/h) x,  Dc/h = [[-3, 4, -1], [-1, 0, 1], [1, -4, 3]]
template <typename T>
PT_HD void sD(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T d = x2 - x0;
  const T t = (x0 + x2) - T(2) * x1;
  y1 = d;
  y0 = d - T(2) * t;
  y2 = d + T(2) * t;
}

// y (+)= (Dc/h)^T x
template <typename T, bool ACC>
PT_HD void sDt(T x0, T x1, T x2, T &y0, T &y1, T &y2)
{
  const T o = x0 - x2;
  const T s = (x0 + x1) + x2;
  const T r0 = -s - T(2) * o;
  const T r1 = T(4) * o;
  const T r2 = s - T(2) * o;
  if (ACC) { y0 += r0; y1 += r1; y2 += r2; }
  else { y0 = r0; y1 = r1; y2 = r2; }
}

// zeta contraction of one (j,i) node column for plane A: Q and R.
template <typename T, int A>
PT_HD void zeta_fwd(T n0, T n1, T n2, T &q, T &r)
{
  if (A == 1) {
    q = n1;
    r = T(GS) * (n2 - n0);
  } else if (A == 0) {
    q = T(B0) * n0 + (T(B1) * n1 + T(B2) * n2);
    r = T(DZ00) * n0 + (T(DZ01) * n1 + T(DZ02) * n2);
  } else {
    q = T(B2) * n0 + (T(B1) * n1 + T(B0) * n2);
    r = T(DZ20) * n0 + (T(DZ21) * n1 + T(DZ22) * n2);
  }
}

// its transpose: contributions of (q, r) to the node planes k = 0, 1, 2
template <typename T, int A>
PT_HD void zeta_bwd(T q, T r, T &c0, T &c1, T &c2)
{
  if (A == 1) {
    c0 = -T(GS) * r; c1 = q; c2 = T(GS) * r;
  } else if (A == 0) {
    c0 = T(B0) * q + T(DZ00) * r; c1 = T(B1) * q + T(DZ01) * r; c2 = T(B2) * q + T(DZ02) * r;
  } else {
    c0 = T(B2) * q + T(DZ20) * r; c1 = T(B1) * q + T(DZ21) * r; c2 = T(B0) * q + T(DZ22) * r;
  }
}

// Q, R [j*3+i] -> G0, G1, G2 [b*3+c]
template <typename T>
PT_HD void plane_fwd(const T Q[9], const T R[9], T G0[9], T G1[9], T G2[9])
{
  T Qx[9], Rx[9], I[9];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    lineB(Q[3 * j], Q[3 * j + 1], Q[3 * j + 2], Qx[3 * j], Qx[3 * j + 1], Qx[3 * j + 2]);
    lineB(R[3 * j], R[3 * j + 1], R[3 * j + 2], Rx[3 * j], Rx[3 * j + 1], Rx[3 * j + 2]);
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    lineB(Qx[c], Qx[3 + c], Qx[6 + c], I[c], I[3 + c], I[6 + c]);
    lineB(Rx[c], Rx[3 + c], Rx[6 + c], G2[c], G2[3 + c], G2[6 + c]);
  }
#pragma unroll
  for (int b = 0; b < 3; b++) sD(I[3 * b], I[3 * b + 1], I[3 * b + 2], G0[3 * b], G0[3 * b + 1], G0[3 * b + 2]);
#pragma unroll
  for (int c = 0; c < 3; c++) sD(I[c], I[3 + c], I[6 + c], G1[c], G1[3 + c], G1[6 + c]);
}

// transpose of plane_fwd: G0, G1, G2 [b*3+c] -> Qt, Rt [j*3+i]
template <typename T>
PT_HD void plane_bwd(const T G0[9], const T G1[9], const T G2[9], T Qt[9], T Rt[9])
{
  T Sx[9], Qe[9], Re[9];
#pragma unroll
  for (int b = 0; b < 3; b++) sDt<T, false>(G0[3 * b], G0[3 * b + 1], G0[3 * b + 2], Sx[3 * b], Sx[3 * b + 1], Sx[3 * b + 2]);
#pragma unroll
  for (int c = 0; c < 3; c++) sDt<T, true>(G1[c], G1[3 + c], G1[6 + c], Sx[c], Sx[3 + c], Sx[6 + c]);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    lineBt(Sx[c], Sx[3 + c], Sx[6 + c], Qe[c], Qe[3 + c], Qe[6 + c]);
    lineBt(G2[c], G2[3 + c], G2[6 + c], Re[c], Re[3 + c], Re[6 + c]);
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    lineBt(Qe[3 * j], Qe[3 * j + 1], Qe[3 * j + 2], Qt[3 * j], Qt[3 * j + 1], Qt[3 * j + 2]);
    lineBt(Re[3 * j], Re[3 * j + 1], Re[3 * j + 2], Rt[3 * j], Rt[3 * j + 1], Rt[3 * j + 2]);
  }
}

// Viscous action at point p of a plane: G[d][l][p] <- dv'[d][l] = ((K G)+(K G)^T) K
template <typename T>
PT_HD void qp_action_K(const T Kq[9], T G[3][3][9], int p)
{
  T A[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) A[k][l] = Kq[3 * k] * G[0][l][p] + (Kq[3 * k + 1] * G[1][l][p] + Kq[3 * k + 2] * G[2][l][p]);
  T S[3][3];
  S[0][0] = A[0][0] + A[0][0];
  S[1][1] = A[1][1] + A[1][1];
  S[2][2] = A[2][2] + A[2][2];
  S[0][1] = S[1][0] = A[0][1] + A[1][0];
  S[0][2] = S[2][0] = A[0][2] + A[2][0];
  S[1][2] = S[2][1] = A[1][2] + A[2][1];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) G[k][l][p] = S[0][l] * Kq[k] + (S[1][l] * Kq[3 + k] + S[2][l] * Kq[6 + k]);
}

// ---------------------------------------------------------------------------
// diag(A11) from K (the streaming diagonal kernel).
//
// For basis function n and velocity component m the A11 action above applied
// to u = N_n e_m gives, at each point, A[k][l] = delta_lm a_k with
//   a_k(n,q) = sum_d K[3k+d](q) g'_d(n,q),   g' = h^-1 grad_xi N_n,
// and the diagonal entry sum_q sum_k (a_k + delta_km a_m) a_k, i.e.
//   diag(n, m) = Q_m(n) + sum_k Q_k(n),   Q_k(n) = sum_q a_k(n,q)^2
// (the reference's w det eta (|grad N|^2 + (dN/dx_m)^2) of
// src/stokes_q2p1_mf_operators_diag_def.c:120-205 in K form).
//
// Q_k is a quadratic form in g': with r = row k of K at a point,
//   a_k^2 = sum_{d,e} r_d r_e g'_d g'_e,
// and g'_d g'_e factorises per axis: along axis t it is E(g,i)^2 if d = e = t,
// E(g,i) B(g,i) if exactly one of d, e is t and B(g,i)^2 otherwise (B the Q2
// basis and E = D/h its scaled derivative at Gauss abscissa g, node i).  So
// the six products r_d r_e (cross terms doubled) of a Gauss plane are
// contracted along xi, then along eta and summed by their zeta factor
// (BB: de = 00, 11, 01; EB: 02, 12; EE: 22), and the zeta factors of the
// plane spread the three sums over the node planes: ~400 operations per
// plane and component instead of 27 x 9 x 4 for the point-by-node sum.
// ---------------------------------------------------------------------------
namespace dg {
// B(g,i) and E(g,i) = D(g,i)/h (rows of q2::B* and the DZ constants above)
PT_HD constexpr double xb(int g, int i)
{
  return g == 1 ? (i == 1 ? 1.0 : 0.0) : (i == 1 ? B1 : (((g == 0) == (i == 0)) ? B0 : B2));
}
PT_HD constexpr double xe(int g, int i)
{
  return g == 1 ? (i == 0 ? -GS : (i == 1 ? 0.0 : GS))
                : (g == 0 ? (i == 0 ? DZ00 : (i == 1 ? DZ01 : DZ02)) : (i == 0 ? DZ20 : (i == 1 ? DZ21 : DZ22)));
}
PT_HD constexpr double bb(int g, int i) { return xb(g, i) * xb(g, i); }
PT_HD constexpr double eb(int g, int i) { return xe(g, i) * xb(g, i); }
PT_HD constexpr double ee(int g, int i) { return xe(g, i) * xe(g, i); }

// acc += f c, skipped where the compile-time factor c is zero (the middle
// Gauss point: B = [0 1 0], E = [-s 0 s], so EB = 0 there)
template <typename T>
PT_HD void cacc(T &acc, T f, double c)
{
  if (c != 0.0) acc += f * T(c);
}
}  // namespace dg

// Q[k*9 + j*3 + i] = sum over the 9 points p = b*3 + c (b along eta, c along
// xi) of one Gauss plane of a(n,p)^2 for node n = (i,j,k), a = r . g'.
// kr(p, d) returns component d of the row of K at point p; z[s][k] are the
// plane's zeta factors (s = 0: B^2, 1: E B, 2: E^2 at its Gauss abscissa).
template <typename T, typename KR>
PT_HD void diag_form_plane(KR kr, const T z[3][3], T Q[27])
{
  using namespace dg;
  T Z[3][9];  // [BB, EB, EE][j*3+i]
#pragma unroll
  for (int b = 0; b < 3; b++) {
    T X[6][3];  // products [00, 11, 22, 01, 02, 12] contracted along xi, [i]
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int p = 3 * b + c;
      const T k0 = kr(p, 0), k1 = kr(p, 1), k2 = kr(p, 2);
      const T t0 = k0 + k0, t1 = k1 + k1;
      const T f00 = k0 * k0, f11 = k1 * k1, f22 = k2 * k2, f01 = t0 * k1, f02 = t0 * k2, f12 = t1 * k2;
#pragma unroll
      for (int i = 0; i < 3; i++) {
        if (c == 0) {  // every factor of the first abscissa is non-zero
          X[0][i] = f00 * T(ee(0, i));
          X[1][i] = f11 * T(bb(0, i));
          X[2][i] = f22 * T(bb(0, i));
          X[3][i] = f01 * T(eb(0, i));
          X[4][i] = f02 * T(eb(0, i));
          X[5][i] = f12 * T(bb(0, i));
        } else {
          cacc(X[0][i], f00, ee(c, i));
          cacc(X[1][i], f11, bb(c, i));
          cacc(X[2][i], f22, bb(c, i));
          cacc(X[3][i], f01, eb(c, i));
          cacc(X[4][i], f02, eb(c, i));
          cacc(X[5][i], f12, bb(c, i));
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        T &zbb = Z[0][3 * j + i], &zeb = Z[1][3 * j + i], &zee = Z[2][3 * j + i];
        if (b == 0) {
          zbb = X[0][i] * T(bb(0, j)) + (X[1][i] * T(ee(0, j)) + X[3][i] * T(eb(0, j)));
          zeb = X[4][i] * T(bb(0, j)) + X[5][i] * T(eb(0, j));
          zee = X[2][i] * T(bb(0, j));
        } else {
          cacc(zbb, X[0][i], bb(b, j));
          cacc(zbb, X[1][i], ee(b, j));
          cacc(zbb, X[3][i], eb(b, j));
          cacc(zeb, X[4][i], bb(b, j));
          cacc(zeb, X[5][i], eb(b, j));
          cacc(zee, X[2][i], bb(b, j));
        }
      }
  }
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int ji = 0; ji < 9; ji++) Q[9 * k + ji] = z[0][k] * Z[0][ji] + (z[1][k] * Z[1][ji] + z[2][k] * Z[2][ji]);
}

// K at one Gauss point from J (d x_l / d xi_d) and the weight*eta product.
// Returns false when c = w eta / det is not positive and finite.
template <typename T>
PT_HD bool geom_K(const double J[3][3], double w_eta, T Kq[9])
{
  double adj[3][3];
  const double det = adjugate(J, adj);
  const double c = w_eta / det;
  const bool ok = (c > 0.0) && (c < 1.0e308);
  const double f = DH * (ok ? sqrt(c) : 0.0);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int l = 0; l < 3; l++) Kq[3 * k + l] = (T)(f * adj[k][l]);
  return ok;
}

}  // namespace q2
