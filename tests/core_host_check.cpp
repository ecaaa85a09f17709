// Host build of the element arithmetic in ptatin-gene_b200/csrc/q2_core.cuh,
// used by tests/test_core_host.py to check the kernels' per-element algorithm
// against the CPU oracle without a GPU.  Element loop, gathers and scatters
// are plain serial C++ here; only the per-element math is shared with the
// CUDA kernels.
#include <cstdint>
#include <cstring>

#include "q2_core.cuh"

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
