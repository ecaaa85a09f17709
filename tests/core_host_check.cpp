// Host build of the element arithmetic in ptatin-gene_b200/csrc/q2_core.cuh,
// used by tests/test_core_host.py to check the kernels' per-element algorithm
// against the CPU oracle without a GPU.  Element loop, gathers and scatters
// are plain serial C++ here; only the per-element math is shared with the
// CUDA kernels.
#include <cstdint>
#include <cstring>

#include "q2_core.cuh"
#include "q2_plane.cuh"

template <typename T>
static void a11_mesh(int mx, int my, int mz, const double *coords, const double *eta, const double *u,
                     double *y)
{
  const int64_t X = 2 * mx + 1, Y = 2 * my + 1;
  for (int ek = 0; ek < mz; ek++)
    for (int ej = 0; ej < my; ej++)
      for (int ei = 0; ei < mx; ei++) {
        const int64_t e = ei + (int64_t)mx * (ej + (int64_t)my * ek);
        int64_t nid[27];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
              nid[9 * a + 3 * b + c] = (2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y;
        T xf[3][27], uf[3][27], I[27], Jg[3][3][27], Ug[3][3][27];
        for (int n = 0; n < 27; n++)
          for (int l = 0; l < 3; l++) {
            xf[l][n] = (T)coords[3 * nid[n] + l];
            uf[l][n] = (T)u[3 * nid[n] + l];
          }
        for (int l = 0; l < 3; l++) {
          q2::interp(xf[l], I);
          q2::grad_colloc(I, Jg[0][l], Jg[1][l], Jg[2][l]);
          q2::interp(uf[l], I);
          q2::grad_colloc(I, Ug[0][l], Ug[1][l], Ug[2][l]);
        }
        T dv[3][3][27];
        for (int q = 0; q < 27; q++) {
          T J[3][3], adj[3][3], G[3][3], d[3][3];
          for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) {
              J[k][l] = Jg[k][l][q];
              G[k][l] = Ug[k][l][q];
            }
          const T det = q2::adjugate(J, adj);
          const T c = (T)q2::weight(q) * (T)eta[27 * e + q] / det;
          q2::qp_viscous(adj, c, G, d);
          for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) dv[k][l][q] = d[k][l];
        }
        for (int l = 0; l < 3; l++) {
          T r[27], f[27];
          q2::grad_colloc_t(dv[0][l], dv[1][l], dv[2][l], r);
          q2::interp_t(r, f);
          for (int n = 0; n < 27; n++) y[3 * nid[n] + l] += (double)f[n];
        }
      }
}

extern "C" void core_a11_f64(int mx, int my, int mz, const double *coords, const double *eta,
                             const double *u, double *y)
{
  a11_mesh<double>(mx, my, mz, coords, eta, u, y);
}

extern "C" void core_a11_f32(int mx, int my, int mz, const double *coords, const double *eta,
                             const double *u, double *y)
{
  a11_mesh<float>(mx, my, mz, coords, eta, u, y);
}

// The streaming kernel's algorithm (csrc/q2_plane.cuh): K per Gauss point from
// the geometry, then per quadrature plane forward / action / transpose.
template <typename T>
static int a11_plane_mesh(int mx, int my, int mz, const double *coords, const double *eta, const double *u,
                          double *y)
{
  const int64_t X = 2 * mx + 1, Y = 2 * my + 1;
  int bad = 0;
  for (int ek = 0; ek < mz; ek++)
    for (int ej = 0; ej < my; ej++)
      for (int ei = 0; ei < mx; ei++) {
        const int64_t e = ei + (int64_t)mx * (ej + (int64_t)my * ek);
        int64_t nid[27];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
              nid[9 * a + 3 * b + c] = (2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y;
        // geometry (FP64) -> K
        double xf[27], I[27], Jg[3][3][27];
        for (int l = 0; l < 3; l++) {
          for (int n = 0; n < 27; n++) xf[n] = coords[3 * nid[n] + l];
          q2::interp(xf, I);
          q2::grad_colloc(I, Jg[0][l], Jg[1][l], Jg[2][l]);
        }
        T K[27][9];
        for (int q = 0; q < 27; q++) {
          double J[3][3];
          for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
          if (!q2::geom_K(J, q2::weight(q) * eta[27 * e + q], K[q])) bad++;
        }
        T N[3][3][27];  // [comp][k-plane][j*3+i] -> use [l][k][9]
        for (int l = 0; l < 3; l++)
          for (int k = 0; k < 3; k++)
            for (int ji = 0; ji < 9; ji++) N[l][k][ji] = (T)u[3 * nid[9 * k + ji] + l];
        T out[3][3][9];
        for (int l = 0; l < 3; l++)
          for (int k = 0; k < 3; k++)
            for (int ji = 0; ji < 9; ji++) out[l][k][ji] = T(0);
        for (int a = 0; a < 3; a++) {
          T G[3][3][9];
          for (int l = 0; l < 3; l++) {
            T Q[9], R[9];
            for (int ji = 0; ji < 9; ji++) {
              if (a == 0) q2::zeta_fwd<T, 0>(N[l][0][ji], N[l][1][ji], N[l][2][ji], Q[ji], R[ji]);
              if (a == 1) q2::zeta_fwd<T, 1>(N[l][0][ji], N[l][1][ji], N[l][2][ji], Q[ji], R[ji]);
              if (a == 2) q2::zeta_fwd<T, 2>(N[l][0][ji], N[l][1][ji], N[l][2][ji], Q[ji], R[ji]);
            }
            q2::plane_fwd(Q, R, G[0][l], G[1][l], G[2][l]);
          }
          for (int p = 0; p < 9; p++) q2::qp_action_K(K[9 * a + p], G, p);
          for (int l = 0; l < 3; l++) {
            T Qt[9], Rt[9];
            q2::plane_bwd(G[0][l], G[1][l], G[2][l], Qt, Rt);
            for (int ji = 0; ji < 9; ji++) {
              T c0, c1, c2;
              if (a == 0) q2::zeta_bwd<T, 0>(Qt[ji], Rt[ji], c0, c1, c2);
              if (a == 1) q2::zeta_bwd<T, 1>(Qt[ji], Rt[ji], c0, c1, c2);
              if (a == 2) q2::zeta_bwd<T, 2>(Qt[ji], Rt[ji], c0, c1, c2);
              out[l][0][ji] += c0;
              out[l][1][ji] += c1;
              out[l][2][ji] += c2;
            }
          }
        }
        for (int l = 0; l < 3; l++)
          for (int k = 0; k < 3; k++)
            for (int ji = 0; ji < 9; ji++) y[3 * nid[9 * k + ji] + l] += (double)out[l][k][ji];
      }
  return bad;
}

extern "C" int core_a11_plane_f64(int mx, int my, int mz, const double *coords, const double *eta,
                                  const double *u, double *y)
{
  return a11_plane_mesh<double>(mx, my, mz, coords, eta, u, y);
}

extern "C" int core_a11_plane_f32(int mx, int my, int mz, const double *coords, const double *eta,
                                  const double *u, double *y)
{
  return a11_plane_mesh<float>(mx, my, mz, coords, eta, u, y);
}

// The streaming diagonal kernel's algorithm (q2::diag_form_plane): K per
// Gauss point, then per quadrature plane and velocity component the
// sum-factorised quadratic form Q_m; diag(n, l) = Q_l(n) + sum_m Q_m(n).
extern "C" int core_diag_plane_f64(int mx, int my, int mz, const double *coords, const double *eta, double *y)
{
  const int64_t X = 2 * mx + 1, Y = 2 * my + 1;
  int bad = 0;
  double zf[3][3][3];  // [plane A][BB, EB, EE][k]
  for (int a = 0; a < 3; a++)
    for (int k = 0; k < 3; k++) {
      zf[a][0][k] = q2::dg::bb(a, k);
      zf[a][1][k] = q2::dg::eb(a, k);
      zf[a][2][k] = q2::dg::ee(a, k);
    }
  for (int ek = 0; ek < mz; ek++)
    for (int ej = 0; ej < my; ej++)
      for (int ei = 0; ei < mx; ei++) {
        const int64_t e = ei + (int64_t)mx * (ej + (int64_t)my * ek);
        int64_t nid[27];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            for (int c = 0; c < 3; c++)
              nid[9 * a + 3 * b + c] = (2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y;
        double xf[27], I[27], Jg[3][3][27];
        for (int l = 0; l < 3; l++) {
          for (int n = 0; n < 27; n++) xf[n] = coords[3 * nid[n] + l];
          q2::interp(xf, I);
          q2::grad_colloc(I, Jg[0][l], Jg[1][l], Jg[2][l]);
        }
        double K[27][9];
        for (int q = 0; q < 27; q++) {
          double J[3][3];
          for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
          if (!q2::geom_K(J, q2::weight(q) * eta[27 * e + q], K[q])) bad++;
        }
        for (int a = 0; a < 3; a++) {
          double S[27] = {0};
          for (int m = 0; m < 3; m++) {
            double Q[27];
            q2::diag_form_plane<double>([&](int p, int d) { return K[9 * a + p][3 * m + d]; }, zf[a], Q);
            for (int n = 0; n < 27; n++) {
              y[3 * nid[n] + m] += Q[n];
              S[n] += Q[n];
            }
          }
          for (int n = 0; n < 27; n++)
            for (int l = 0; l < 3; l++) y[3 * nid[n] + l] += S[n];
        }
      }
  return bad;
}
