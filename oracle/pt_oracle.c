/*
 * CPU oracle for the pTatin3D matrix-free Q2-P1disc Stokes operator.
 * TEST INFRASTRUCTURE ONLY -- see pt_oracle.h for scope, layouts and the
 * reference file:line each routine restates.
 *
 * Build: gcc -O2 -fopenmp -fPIC -shared pt_oracle.c -o liboracle.so -lm
 * (-O2 without -ffast-math keeps IEEE evaluation order, which matters for a
 * checker; -march is not used so results do not depend on the host ISA).
 */
#include "pt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NPE 27
#define NQP 27

int ora_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Quadrature and basis tables                                               */
/* ------------------------------------------------------------------------ */

/*
 * 3-point Gauss-Legendre rule on [-1,1].  The tensor and AVX paths obtain it
 * from PETSc's PetscDTGaussQuadrature(3,-1,1,x,w) (stokes_operators_tensor.c:194,
 * PETSc 3.8.3).  PETSc computes the rule numerically (Golub-Welsch: eigen-
 * decomposition of the symmetric tridiagonal Jacobi matrix with off-diagonals
 * k/sqrt(4k^2-1)); for n=3 the eigenvalues are 0 and +-sqrt(3/5) and the
 * weights 2*v0^2 are 5/9, 8/9, 5/9.  The closed form is used here; it can
 * differ from PETSc's numerical value in the last ulp only.
 */
void ora_gauss3(double x[3], double w[3])
{
  const double s = sqrt(3.0 / 5.0);
  x[0] = -s; x[1] = 0.0; x[2] = s;
  w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
}

/*
 * B[q][n] = Q2 Lagrange basis n at Gauss node q; D = its derivative
 * (stokes_operators_tensor.c:195-202).
 */
static void tensor_tables(double B[3][3], double D[3][3], double w[NQP], double x1[3])
{
  double w1[3];
  int i, j, k;
  ora_gauss3(x1, w1);
  for (i = 0; i < 3; i++) {
    B[i][0] = .5 * (x1[i] * x1[i] - x1[i]);
    B[i][1] = 1 - x1[i] * x1[i];
    B[i][2] = .5 * (x1[i] * x1[i] + x1[i]);
    D[i][0] = x1[i] - .5;
    D[i][1] = -2 * x1[i];
    D[i][2] = x1[i] + .5;
  }
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++)
      for (k = 0; k < 3; k++) w[(i * 3 + j) * 3 + k] = w1[i] * w1[j] * w1[k];
}

/* Q2 basis values at xi (element_utils_q2.c, P3D_ConstructNi_Q2_3D). */
static void q2_ni(const double xi[3], double Ni[NPE])
{
  double b[3][3];
  int d, i, j, k, cnt = 0;
  for (d = 0; d < 3; d++) {
    double t = xi[d];
    b[d][0] = 0.5 * t * (t - 1.0);
    b[d][1] = (1.0 + t) * (1.0 - t);
    b[d][2] = 0.5 * (1.0 + t) * t;
  }
  for (k = 0; k < 3; k++)
    for (j = 0; j < 3; j++)
      for (i = 0; i < 3; i++) Ni[cnt++] = b[0][i] * b[1][j] * b[2][k];
}

/*
 * 3x3x3 Gauss rule with the truncated constants and the derivative tables of
 * the "ref" path (element_utils_q2.c:276-333, P3D_prepare_elementQ2_3x3).
 */
static void ref_tables(double WEIGHT[NQP], double XI[NQP][3], double GNI[NQP][3][NPE])
{
  const double s = 0.774596669241483;
  const double w_1 = 0.555555555555556;
  const double w_0 = 0.888888888888889;
  double od_xi[3], od_w[3];
  int i, j, k, p, cnt = 0;
  od_xi[0] = -s; od_xi[1] = 0.0; od_xi[2] = s;
  od_w[0] = w_1; od_w[1] = w_0; od_w[2] = w_1;
  for (k = 0; k < 3; k++)
    for (j = 0; j < 3; j++)
      for (i = 0; i < 3; i++) {
        XI[cnt][0] = od_xi[i]; XI[cnt][1] = od_xi[j]; XI[cnt][2] = od_xi[k];
        WEIGHT[cnt] = od_w[i] * od_w[j] * od_w[k];
        cnt++;
      }
  for (p = 0; p < NQP; p++) {
    double GNix[3][3], Nix[3][3];
    int ix;
    for (ix = 0; ix < 3; ix++) {
      double t = XI[p][ix];
      Nix[ix][0] = 0.5 * t * (t - 1.0);
      Nix[ix][1] = (1.0 + t) * (1.0 - t);
      Nix[ix][2] = 0.5 * (1.0 + t) * t;
      GNix[ix][0] = t - 0.5;
      GNix[ix][1] = -2.0 * t;
      GNix[ix][2] = 0.5 * (1.0 + 2.0 * t);
    }
    cnt = 0;
    for (k = 0; k < 3; k++)
      for (j = 0; j < 3; j++)
        for (i = 0; i < 3; i++) {
          GNI[p][0][cnt] = GNix[0][i] * Nix[1][j] * Nix[2][k];
          GNI[p][1][cnt] = Nix[0][i] * GNix[1][j] * Nix[2][k];
          GNI[p][2][cnt] = Nix[0][i] * Nix[1][j] * GNix[2][k];
          cnt++;
        }
  }
}

/* ------------------------------------------------------------------------ */
/* Mesh topology                                                              */
/* ------------------------------------------------------------------------ */

/*
 * Element e = ei + ej*mx + ek*mx*my -> 27 node ids, lexicographic with the
 * local i index fastest and a stride of 2 nodes per element
 * (dmda_element_q2p1.c:395-455 on one rank: esi=gsi=0).
 */
void ora_elements_q2(int mx, int my, int mz, int32_t *elnidx)
{
  const int64_t X = 2 * mx + 1, Y = 2 * my + 1;
  int64_t e = 0;
  int ei, ej, ek, a, b, c;
  for (ek = 0; ek < mz; ek++)
    for (ej = 0; ej < my; ej++)
      for (ei = 0; ei < mx; ei++) {
        for (a = 0; a < 3; a++)
          for (b = 0; b < 3; b++)
            for (c = 0; c < 3; c++)
              elnidx[27 * e + a * 9 + b * 3 + c] =
                  (int32_t)((2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y);
        e++;
      }
}

static inline void element_nodes(int mx, int my, int64_t e, int64_t nid[NPE])
{
  const int64_t X = 2 * (int64_t)mx + 1, Y = 2 * (int64_t)my + 1;
  const int64_t ei = e % mx, ej = (e / mx) % my, ek = e / ((int64_t)mx * my);
  int a, b, c;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++)
        nid[a * 9 + b * 3 + c] = (2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y;
}

/* ------------------------------------------------------------------------ */
/* Geometry of the "ref" path (element_utils_q2.c:399-476, STANDARD variant)  */
/* ------------------------------------------------------------------------ */

static void ref_geometry(const double el_coords[3 * NPE], double GNI[NQP][3][NPE],
                         double detJ[NQP], double dNudx[NQP][NPE], double dNudy[NQP][NPE],
                         double dNudz[NQP][NPE])
{
  int k, p;
  for (p = 0; p < NQP; p++) {
    double J[3][3] = {{0}}, iJ[3][3];
    double t4, t6, t8, t10, t12, t14, t17;
    for (k = 0; k < NPE; k++) {
      double xc = el_coords[3 * k + 0], yc = el_coords[3 * k + 1], zc = el_coords[3 * k + 2];
      J[0][0] += GNI[p][0][k] * xc; J[0][1] += GNI[p][0][k] * yc; J[0][2] += GNI[p][0][k] * zc;
      J[1][0] += GNI[p][1][k] * xc; J[1][1] += GNI[p][1][k] * yc; J[1][2] += GNI[p][1][k] * zc;
      J[2][0] += GNI[p][2][k] * xc; J[2][1] += GNI[p][2][k] * yc; J[2][2] += GNI[p][2][k] * zc;
    }
    detJ[p] = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1])
            - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0])
            + J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    t4 = J[2][0] * J[0][1];
    t6 = J[2][0] * J[0][2];
    t8 = J[1][0] * J[0][1];
    t10 = J[1][0] * J[0][2];
    t12 = J[0][0] * J[1][1];
    t14 = J[0][0] * J[1][2];
    t17 = 0.1e1 / (t4 * J[1][2] - t6 * J[1][1] - t8 * J[2][2] + t10 * J[2][1] + t12 * J[2][2] - t14 * J[2][1]);
    iJ[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * t17;
    iJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) * t17;
    iJ[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * t17;
    iJ[1][0] = -(-J[2][0] * J[1][2] + J[1][0] * J[2][2]) * t17;
    iJ[1][1] = (-t6 + J[0][0] * J[2][2]) * t17;
    iJ[1][2] = -(-t10 + t14) * t17;
    iJ[2][0] = (-J[2][0] * J[1][1] + J[1][0] * J[2][1]) * t17;
    iJ[2][1] = -(-t4 + J[0][0] * J[2][1]) * t17;
    iJ[2][2] = (-t8 + t12) * t17;
    for (k = 0; k < NPE; k++) {
      dNudx[p][k] = iJ[0][0] * GNI[p][0][k] + iJ[0][1] * GNI[p][1][k] + iJ[0][2] * GNI[p][2][k];
      dNudy[p][k] = iJ[1][0] * GNI[p][0][k] + iJ[1][1] * GNI[p][1][k] + iJ[1][2] * GNI[p][2][k];
      dNudz[p][k] = iJ[2][0] * GNI[p][0][k] + iJ[2][1] * GNI[p][1][k] + iJ[2][2] * GNI[p][2][k];
    }
  }
}

/*
 * P1 "global relative" pressure basis at reference point xi
 * (element_utils_q2.c:183-224, selected by include/ptatin3d_defs.h:54,83-85):
 * Np = {1, xh, yh, zh}, xh = (x(xi) - mean of the 27 nodes) / L, with
 * Lx = x14 - x12, Ly = y16 - y10, Lz = z22 - z4.
 */
static void p1grel_ni(const double xi[3], const double coords[3 * NPE], double Ni[4])
{
  double Ng[NPE], xg[3] = {0, 0, 0}, ax = 0, ay = 0, az = 0, Lx, Ly, Lz;
  int i;
  q2_ni(xi, Ng);
  for (i = 0; i < NPE; i++) {
    xg[0] = xg[0] + Ng[i] * coords[3 * i];
    xg[1] = xg[1] + Ng[i] * coords[3 * i + 1];
    xg[2] = xg[2] + Ng[i] * coords[3 * i + 2];
    ax = ax + coords[3 * i];
    ay = ay + coords[3 * i + 1];
    az = az + coords[3 * i + 2];
  }
  ax = (1.0 / 27.0) * ax;
  ay = (1.0 / 27.0) * ay;
  az = (1.0 / 27.0) * az;
  Lx = coords[3 * 14] - coords[3 * 12];
  Ly = coords[3 * 16 + 1] - coords[3 * 10 + 1];
  Lz = coords[3 * 22 + 2] - coords[3 * 4 + 2];
  Ni[0] = 1.0;
  Ni[1] = (xg[0] - ax) / Lx;
  Ni[2] = (xg[1] - ay) / Ly;
  Ni[3] = (xg[2] - az) / Lz;
}

/* ------------------------------------------------------------------------ */
/* Tensor-product kernels (stokes_operators_tensor.c:40-179)                 */
/* ------------------------------------------------------------------------ */

typedef enum { GRAD, GRAD_TRANSPOSE } GradMode;

/* y[l,a,b,c] += T[a,k] S[b,j] R[c,i] x[l,k,j,i] for the 3 fields l. */
static void tensor_contract(double Rf[3][3], double Sf[3][3], double Tf[3][3], GradMode g,
                            double x[3][NQP], double y[3][NQP])
{
  double R[3][3], S[3][3], T[3][3], u[3][NQP], v[3][NQP];
  int i, j, k, l, kj, ji, a, b, c;
  for (j = 0; j < 3; j++)
    for (i = 0; i < 3; i++) {
      R[i][j] = g == GRAD ? Rf[i][j] : Rf[j][i];
      S[i][j] = g == GRAD ? Sf[i][j] : Sf[j][i];
      T[i][j] = g == GRAD ? Tf[i][j] : Tf[j][i];
    }
  memset(u, 0, sizeof u);
  for (l = 0; l < 3; l++)
    for (kj = 0; kj < 9; kj++)
      for (i = 0; i < 3; i++)
        for (c = 0; c < 3; c++) u[l][kj * 3 + c] += R[c][i] * x[l][kj * 3 + i];
  memset(v, 0, sizeof v);
  for (l = 0; l < 3; l++)
    for (k = 0; k < 3; k++)
      for (j = 0; j < 3; j++)
        for (c = 0; c < 3; c++)
          for (b = 0; b < 3; b++) v[l][(k * 3 + b) * 3 + c] += S[b][j] * u[l][(k * 3 + j) * 3 + c];
  for (k = 0; k < 3; k++)
    for (l = 0; l < 3; l++)
      for (a = 0; a < 3; a++)
        for (ji = 0; ji < 9; ji++) y[l][a * 9 + ji] += T[a][k] * v[l][k * 9 + ji];
}

/* Replace dx (= d x_k / d xi_j, stored dx[j][k]) by its inverse; store det. */
static void jacobian_invert(double dx[3][3][NQP], double dxdet[NQP])
{
  int i, j, k;
  for (i = 0; i < NQP; i++) {
    double a[3][3], b0, b3, b6, det, idet;
    for (j = 0; j < 3; j++)
      for (k = 0; k < 3; k++) a[j][k] = dx[j][k][i];
    b0 = (a[1][1] * a[2][2] - a[2][1] * a[1][2]);
    b3 = -(a[1][0] * a[2][2] - a[2][0] * a[1][2]);
    b6 = (a[1][0] * a[2][1] - a[2][0] * a[1][1]);
    det = a[0][0] * b0 + a[0][1] * b3 + a[0][2] * b6;
    idet = 1.0 / det;
    dx[0][0][i] = idet * b0;
    dx[0][1][i] = -idet * (a[0][1] * a[2][2] - a[2][1] * a[0][2]);
    dx[0][2][i] = idet * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
    dx[1][0][i] = idet * b3;
    dx[1][1][i] = idet * (a[0][0] * a[2][2] - a[2][0] * a[0][2]);
    dx[1][2][i] = -idet * (a[0][0] * a[1][2] - a[1][0] * a[0][2]);
    dx[2][0][i] = idet * b6;
    dx[2][1][i] = -idet * (a[0][0] * a[2][1] - a[2][0] * a[0][1]);
    dx[2][2][i] = idet * (a[0][0] * a[1][1] - a[1][0] * a[0][1]);
    dxdet[i] = det;
  }
}

/* tau = 2 eta sym(grad u); dv[k][l] = w det sum_j tau[j][l] dxi_k/dx_j. */
static void quadrature_action(const double *eta, double dx[3][3][NQP], double dxdet[NQP],
                              const double w[NQP], double du[3][3][NQP], double dv[3][3][NQP])
{
  int i, l, k;
  for (i = 0; i < NQP; i++) {
    double dux[3][3], Du[6], Dv[6], dvx[3][3];
    for (l = 0; l < 3; l++)
      for (k = 0; k < 3; k++)
        dux[k][l] = du[0][l][i] * dx[k][0][i] + du[1][l][i] * dx[k][1][i] + du[2][l][i] * dx[k][2][i];
    Du[0] = dux[0][0];
    Du[1] = dux[1][1];
    Du[2] = dux[2][2];
    Du[3] = 0.5 * (dux[0][1] + dux[1][0]);
    Du[4] = 0.5 * (dux[0][2] + dux[2][0]);
    Du[5] = 0.5 * (dux[1][2] + dux[2][1]);
    for (k = 0; k < 6; k++) Dv[k] = 2 * eta[i] * Du[k];
    dvx[0][0] = Dv[0]; dvx[0][1] = Dv[3]; dvx[0][2] = Dv[4];
    dvx[1][0] = Dv[3]; dvx[1][1] = Dv[1]; dvx[1][2] = Dv[5];
    dvx[2][0] = Dv[4]; dvx[2][1] = Dv[5]; dvx[2][2] = Dv[2];
    for (l = 0; l < 3; l++)
      for (k = 0; k < 3; k++)
        dv[k][l][i] = w[i] * dxdet[i] *
                      (dvx[0][l] * dx[0][k][i] + dvx[1][l] * dx[1][k][i] + dvx[2][l] * dx[2][k][i]);
  }
}

/*
 * Tensor A11 (stokes_operators_tensor.c:181-286).  The reference batches 4
 * elements per vector (NEV) and pads with the last element; the per-element
 * arithmetic is the same, so one element per iteration is used here.  The
 * scatter is serialised exactly as the reference's "omp critical".
 */
void ora_a11_tensor(int mx, int my, int mz, const double *coords, const double *eta,
                    const double *u, double *y)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double B[3][3], D[3][3], w[NQP], x1[3];
  int64_t e;
  tensor_tables(B, D, w, x1);
#pragma omp parallel for schedule(static)
  for (e = 0; e < nel; e++) {
    double elu[3][NQP], elx[3][NQP], elv[3][NQP];
    double dx[3][3][NQP], dxdet[NQP], du[3][3][NQP], dv[3][3][NQP];
    int64_t nid[NPE];
    int i, l;
    element_nodes(mx, my, e, nid);
    for (i = 0; i < NPE; i++)
      for (l = 0; l < 3; l++) {
        elx[l][i] = coords[3 * nid[i] + l];
        elu[l][i] = u[3 * nid[i] + l];
      }
    memset(dx, 0, sizeof dx);
    tensor_contract(D, B, B, GRAD, elx, dx[0]);
    tensor_contract(B, D, B, GRAD, elx, dx[1]);
    tensor_contract(B, B, D, GRAD, elx, dx[2]);
    jacobian_invert(dx, dxdet);
    memset(du, 0, sizeof du);
    tensor_contract(D, B, B, GRAD, elu, du[0]);
    tensor_contract(B, D, B, GRAD, elu, du[1]);
    tensor_contract(B, B, D, GRAD, elu, du[2]);
    quadrature_action(&eta[NQP * e], dx, dxdet, w, du, dv);
    memset(elv, 0, sizeof elv);
    tensor_contract(D, B, B, GRAD_TRANSPOSE, dv[0], elv);
    tensor_contract(B, D, B, GRAD_TRANSPOSE, dv[1], elv);
    tensor_contract(B, B, D, GRAD_TRANSPOSE, dv[2], elv);
#pragma omp critical
    for (i = 0; i < NPE; i++)
      for (l = 0; l < 3; l++) y[3 * nid[i] + l] += elv[l][i];
  }
}

/* ------------------------------------------------------------------------ */
/* "ref" element loops (stokes_operators_mf.c)                               */
/* ------------------------------------------------------------------------ */

static void gather_coords(const double *coords, const int64_t nid[NPE], double el[3 * NPE])
{
  int i;
  for (i = 0; i < NPE; i++) {
    el[3 * i] = coords[3 * nid[i]];
    el[3 * i + 1] = coords[3 * nid[i] + 1];
    el[3 * i + 2] = coords[3 * nid[i] + 2];
  }
}

/* A11 "ref" (stokes_operators_mf.c:237-351 with the B11 per-qp kernel,
 * stokes_q2p1_mf_operators_def.c:151-257). */
void ora_a11_ref(int mx, int my, int mz, const double *coords, const double *eta,
                 const double *u, double *y)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double WEIGHT[NQP], XI[NQP][3], GNI[NQP][3][NPE];
  int64_t e;
  ref_tables(WEIGHT, XI, GNI);
  for (e = 0; e < nel; e++) {
    double elc[3 * NPE], ux[NPE], uy[NPE], uz[NPE], Ye[3 * NPE];
    double detJ[NQP], dNdx[NQP][NPE], dNdy[NQP][NPE], dNdz[NQP][NPE];
    int64_t nid[NPE];
    int k, p;
    element_nodes(mx, my, e, nid);
    gather_coords(coords, nid, elc);
    for (k = 0; k < NPE; k++) {
      ux[k] = u[3 * nid[k]];
      uy[k] = u[3 * nid[k] + 1];
      uz[k] = u[3 * nid[k] + 2];
    }
    ref_geometry(elc, GNI, detJ, dNdx, dNdy, dNdz);
    memset(Ye, 0, sizeof Ye);
    for (p = 0; p < NQP; p++) {
      const double fac = WEIGHT[p] * detJ[p], eg = eta[NQP * e + p];
      double sr[6] = {0, 0, 0, 0, 0, 0}, tau[6];
      for (k = 0; k < NPE; k++) {
        sr[0] += ux[k] * dNdx[p][k];
        sr[1] += uy[k] * dNdy[p][k];
        sr[2] += uz[k] * dNdz[p][k];
        sr[3] += ux[k] * dNdy[p][k] + uy[k] * dNdx[p][k];
        sr[4] += ux[k] * dNdz[p][k] + uz[k] * dNdx[p][k];
        sr[5] += uy[k] * dNdz[p][k] + uz[k] * dNdy[p][k];
      }
      tau[0] = 2.0 * eg * sr[0];
      tau[1] = 2.0 * eg * sr[1];
      tau[2] = 2.0 * eg * sr[2];
      tau[3] = eg * sr[3];
      tau[4] = eg * sr[4];
      tau[5] = eg * sr[5];
      for (k = 0; k < NPE; k++) {
        Ye[3 * k] += fac * (dNdx[p][k] * tau[0] + dNdy[p][k] * tau[3] + dNdz[p][k] * tau[4]);
        Ye[3 * k + 1] += fac * (dNdx[p][k] * tau[3] + dNdy[p][k] * tau[1] + dNdz[p][k] * tau[5]);
        Ye[3 * k + 2] += fac * (dNdx[p][k] * tau[4] + dNdy[p][k] * tau[5] + dNdz[p][k] * tau[2]);
      }
    }
    for (k = 0; k < NPE; k++) {
      y[3 * nid[k]] += Ye[3 * k];
      y[3 * nid[k] + 1] += Ye[3 * k + 1];
      y[3 * nid[k] + 2] += Ye[3 * k + 2];
    }
  }
}

/*
 * Momentum residual FormFunctionLocal_U (stokes_form_function.c:99-243) on one
 * rank, restated: per element and Gauss point, with the ref-path geometry,
 *   fac = w detJ,  p_q = fac * sum_i Np_i p_i  (P1GRel basis, :163-166),
 *   strain exx.. from dN/dx (:169-178), stresses 2 eta fac exx, eta fac exy
 *   (:183-192),
 *   Fe[3k+0] += dNdx (sxx - p_q) + dNdy sxy + dNdz sxz    (and y, z; :194-198)
 *   Be[3k+c] += fac N_k Fu_c                               (:201-205)
 * and Ru += Fe - Be (:209-213).  u is used as given (the caller inserts the
 * Dirichlet values); fu is the Gauss-point body force, 3 per point.
 */
void ora_residual_u(int mx, int my, int mz, const double *coords, const double *eta, const double *fu,
                    const double *u, const double *pr, double *ru)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double WEIGHT[NQP], XI[NQP][3], GNI[NQP][3][NPE], NI[NQP][NPE];
  int64_t e;
  int p;
  ref_tables(WEIGHT, XI, GNI);
  for (p = 0; p < NQP; p++) q2_ni(XI[p], NI[p]);
  for (e = 0; e < nel; e++) {
    double elc[3 * NPE], ux[NPE], uy[NPE], uz[NPE], Fe[3 * NPE], Be[3 * NPE], NIp[NQP][4];
    double detJ[NQP], dNdx[NQP][NPE], dNdy[NQP][NPE], dNdz[NQP][NPE];
    int64_t nid[NPE];
    int k;
    element_nodes(mx, my, e, nid);
    gather_coords(coords, nid, elc);
    for (k = 0; k < NPE; k++) {
      ux[k] = u[3 * nid[k]];
      uy[k] = u[3 * nid[k] + 1];
      uz[k] = u[3 * nid[k] + 2];
    }
    for (p = 0; p < NQP; p++) p1grel_ni(XI[p], elc, NIp[p]);
    ref_geometry(elc, GNI, detJ, dNdx, dNdy, dNdz);
    memset(Fe, 0, sizeof Fe);
    memset(Be, 0, sizeof Be);
    for (p = 0; p < NQP; p++) {
      const double fac = WEIGHT[p] * detJ[p], eg = eta[NQP * e + p];
      double pq = 0.0, exx = 0, eyy = 0, ezz = 0, exy = 0, exz = 0, eyz = 0;
      double d1, d2, sxx, syy, szz, sxy, sxz, syz;
      for (k = 0; k < 4; k++) pq += NIp[p][k] * pr[4 * e + k];
      pq = pq * fac;
      for (k = 0; k < NPE; k++) {
        exx += dNdx[p][k] * ux[k];
        eyy += dNdy[p][k] * uy[k];
        ezz += dNdz[p][k] * uz[k];
        exy += dNdy[p][k] * ux[k] + dNdx[p][k] * uy[k];
        exz += dNdz[p][k] * ux[k] + dNdx[p][k] * uz[k];
        eyz += dNdz[p][k] * uy[k] + dNdy[p][k] * uz[k];
      }
      d1 = 2.0 * eg * fac;
      d2 = eg * fac;
      sxx = d1 * exx; syy = d1 * eyy; szz = d1 * ezz;
      sxy = d2 * exy; sxz = d2 * exz; syz = d2 * eyz;
      for (k = 0; k < NPE; k++) {
        Fe[3 * k] += dNdx[p][k] * (sxx - pq) + dNdy[p][k] * sxy + dNdz[p][k] * sxz;
        Fe[3 * k + 1] += dNdy[p][k] * (syy - pq) + dNdx[p][k] * sxy + dNdz[p][k] * syz;
        Fe[3 * k + 2] += dNdz[p][k] * (szz - pq) + dNdx[p][k] * sxz + dNdy[p][k] * syz;
      }
      for (k = 0; k < NPE; k++) {
        Be[3 * k] += fac * NI[p][k] * fu[3 * (NQP * e + p)];
        Be[3 * k + 1] += fac * NI[p][k] * fu[3 * (NQP * e + p) + 1];
        Be[3 * k + 2] += fac * NI[p][k] * fu[3 * (NQP * e + p) + 2];
      }
    }
    for (k = 0; k < NPE; k++) {
      ru[3 * nid[k]] += Fe[3 * k] - Be[3 * k];
      ru[3 * nid[k] + 1] += Fe[3 * k + 1] - Be[3 * k + 1];
      ru[3 * nid[k] + 2] += Fe[3 * k + 2] - Be[3 * k + 2];
    }
  }
}

/* diag(A11) (stokes_operators_mf.c:71-135, diag_def.c:120-205). */
void ora_a11_diag(int mx, int my, int mz, const double *coords, const double *eta, double *y)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double WEIGHT[NQP], XI[NQP][3], GNI[NQP][3][NPE];
  int64_t e;
  ref_tables(WEIGHT, XI, GNI);
  for (e = 0; e < nel; e++) {
    double elc[3 * NPE], Ye[3 * NPE];
    double detJ[NQP], dNdx[NQP][NPE], dNdy[NQP][NPE], dNdz[NQP][NPE];
    int64_t nid[NPE];
    int k, p;
    element_nodes(mx, my, e, nid);
    gather_coords(coords, nid, elc);
    ref_geometry(elc, GNI, detJ, dNdx, dNdy, dNdz);
    memset(Ye, 0, sizeof Ye);
    for (p = 0; p < NQP; p++) {
      const double fac = WEIGHT[p] * detJ[p], eg = eta[NQP * e + p];
      for (k = 0; k < NPE; k++) {
        const double gx = dNdx[p][k] * dNdx[p][k], gy = dNdy[p][k] * dNdy[p][k],
                     gz = dNdz[p][k] * dNdz[p][k];
        Ye[3 * k] += fac * (eg * gy + eg * gz + 2.0 * eg * gx);
        Ye[3 * k + 1] += fac * (eg * gx + eg * gz + 2.0 * eg * gy);
        Ye[3 * k + 2] += fac * (eg * gx + eg * gy + 2.0 * eg * gz);
      }
    }
    for (k = 0; k < NPE; k++) {
      y[3 * nid[k]] += Ye[3 * k];
      y[3 * nid[k] + 1] += Ye[3 * k + 1];
      y[3 * nid[k] + 2] += Ye[3 * k + 2];
    }
  }
}

/* A21 = B u (stokes_operators_mf.c:862-937, def.c:517-538). */
void ora_a21_ref(int mx, int my, int mz, const double *coords, const double *u, double *yp)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double WEIGHT[NQP], XI[NQP][3], GNI[NQP][3][NPE];
  int64_t e;
  ref_tables(WEIGHT, XI, GNI);
  for (e = 0; e < nel; e++) {
    double elc[3 * NPE], ux[NPE], uy[NPE], uz[NPE], NIp[NQP][4], Ye[4] = {0, 0, 0, 0};
    double detJ[NQP], dNdx[NQP][NPE], dNdy[NQP][NPE], dNdz[NQP][NPE];
    int64_t nid[NPE];
    int k, p;
    element_nodes(mx, my, e, nid);
    gather_coords(coords, nid, elc);
    for (k = 0; k < NPE; k++) {
      ux[k] = u[3 * nid[k]];
      uy[k] = u[3 * nid[k] + 1];
      uz[k] = u[3 * nid[k] + 2];
    }
    for (p = 0; p < NQP; p++) p1grel_ni(XI[p], elc, NIp[p]);
    ref_geometry(elc, GNI, detJ, dNdx, dNdy, dNdz);
    for (p = 0; p < NQP; p++) {
      const double fac = WEIGHT[p] * detJ[p];
      double s0 = 0, s1 = 0, s2 = 0, div;
      for (k = 0; k < NPE; k++) {
        s0 += ux[k] * dNdx[p][k];
        s1 += uy[k] * dNdy[p][k];
        s2 += uz[k] * dNdz[p][k];
      }
      div = s0 + s1 + s2;
      for (k = 0; k < 4; k++) Ye[k] += -fac * NIp[p][k] * div;
    }
    for (k = 0; k < 4; k++) yp[4 * e + k] += Ye[k];
  }
}

/* A12 = B^T p, ref path (stokes_operators_mf.c:792-860, def.c:423-516). */
void ora_a12_ref(int mx, int my, int mz, const double *coords, const double *p, double *yu)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double WEIGHT[NQP], XI[NQP][3], GNI[NQP][3][NPE];
  int64_t e;
  ref_tables(WEIGHT, XI, GNI);
  for (e = 0; e < nel; e++) {
    double elc[3 * NPE], NIp[NQP][4], Ye[3 * NPE];
    double detJ[NQP], dNdx[NQP][NPE], dNdy[NQP][NPE], dNdz[NQP][NPE];
    const double *elp = &p[4 * e];
    int64_t nid[NPE];
    int k, q;
    element_nodes(mx, my, e, nid);
    gather_coords(coords, nid, elc);
    for (q = 0; q < NQP; q++) p1grel_ni(XI[q], elc, NIp[q]);
    ref_geometry(elc, GNI, detJ, dNdx, dNdy, dNdz);
    memset(Ye, 0, sizeof Ye);
    for (q = 0; q < NQP; q++) {
      const double fac = WEIGHT[q] * detJ[q];
      const double pg = NIp[q][0] * elp[0] + NIp[q][1] * elp[1] + NIp[q][2] * elp[2] + NIp[q][3] * elp[3];
      for (k = 0; k < NPE; k++) {
        Ye[3 * k] += -fac * dNdx[q][k] * pg;
        Ye[3 * k + 1] += -fac * dNdy[q][k] * pg;
        Ye[3 * k + 2] += -fac * dNdz[q][k] * pg;
      }
    }
    for (k = 0; k < NPE; k++) {
      yu[3 * nid[k]] += Ye[3 * k];
      yu[3 * nid[k] + 1] += Ye[3 * k + 1];
      yu[3 * nid[k] + 2] += Ye[3 * k + 2];
    }
  }
}

/* A12 with the AVX path's algorithm, scalar (stokes_operators_avx.c:640-829). */
void ora_a12_tensor(int mx, int my, int mz, const double *coords, const double *p, double *yu)
{
  const int64_t nel = (int64_t)mx * my * mz;
  double B[3][3], D[3][3], w[NQP], x1[3], xi[NQP][3];
  int64_t e;
  int i, j, k, q = 0;
  tensor_tables(B, D, w, x1);
  for (k = 0; k < 3; k++)
    for (j = 0; j < 3; j++)
      for (i = 0; i < 3; i++) {
        xi[q][0] = x1[i]; xi[q][1] = x1[j]; xi[q][2] = x1[k];
        q++;
      }
  for (e = 0; e < nel; e++) {
    double elx[3][NQP], elc[3 * NPE], elv[3][NQP], NIp[NQP][4];
    double dx[3][3][NQP], dxdet[NQP], dp[NQP], dv[3][3][NQP];
    const double *elp = &p[4 * e];
    int64_t nid[NPE];
    int l, n;
    element_nodes(mx, my, e, nid);
    for (n = 0; n < NPE; n++)
      for (l = 0; l < 3; l++) {
        elx[l][n] = coords[3 * nid[n] + l];
        elc[3 * n + l] = coords[3 * nid[n] + l];
      }
    for (q = 0; q < NQP; q++) p1grel_ni(xi[q], elc, NIp[q]);
    memset(dx, 0, sizeof dx);
    tensor_contract(D, B, B, GRAD, elx, dx[0]);
    tensor_contract(B, D, B, GRAD, elx, dx[1]);
    tensor_contract(B, B, D, GRAD, elx, dx[2]);
    jacobian_invert(dx, dxdet);
    for (q = 0; q < NQP; q++) {
      dp[q] = 0;
      for (i = 0; i < 4; i++) dp[q] += NIp[q][i] * elp[i];
    }
    /* QuadratureAction_A12_AVX: stress = -p I */
    for (q = 0; q < NQP; q++) {
      const double wt = w[q] * dxdet[q], Dp = -dp[q];
      for (l = 0; l < 3; l++)
        for (k = 0; k < 3; k++) {
          double s = 0.0;
          for (j = 0; j < 3; j++) s += (j == l ? Dp : 0.0) * dx[j][k][q];
          dv[k][l][q] = wt * s;
        }
    }
    memset(elv, 0, sizeof elv);
    tensor_contract(D, B, B, GRAD_TRANSPOSE, dv[0], elv);
    tensor_contract(B, D, B, GRAD_TRANSPOSE, dv[1], elv);
    tensor_contract(B, B, D, GRAD_TRANSPOSE, dv[2], elv);
    for (n = 0; n < NPE; n++)
      for (l = 0; l < 3; l++) yu[3 * nid[n] + l] += elv[l][n];
  }
}

/* ------------------------------------------------------------------------ */
/* BCList semantics (dmda_bcs.c) and the MatShell wrappers                    */
/* ------------------------------------------------------------------------ */

/* BCListInsertLocalZero (dmda_bcs.c:581-608). */
void ora_bc_zero(int64_t n, const uint8_t *mask, double *x)
{
  int64_t k;
  for (k = 0; k < n; k++)
    if (mask[k]) x[k] = 0.0;
}

/* BCListInsertDirichlet_MatMult with scale 1 (dmda_bcs.c:655-689). */
void ora_bc_copy(int64_t n, const uint8_t *mask, const double *x, double *y)
{
  int64_t k;
  for (k = 0; k < n; k++)
    if (mask[k]) y[k] = x[k];
}

/* BCListInsertValueIntoDirichletSlot / BCListInsertZero (dmda_bcs.c:490-541). */
void ora_bc_value(int64_t n, const uint8_t *mask, double value, double *y)
{
  int64_t k;
  for (k = 0; k < n; k++)
    if (mask[k]) y[k] = value;
}

static int64_t nvel(int mx, int my, int mz)
{
  return 3 * (int64_t)(2 * mx + 1) * (2 * my + 1) * (2 * mz + 1);
}

/* MatMult_MFStokes_A11 (stokes_operators.c:1156-1222) on one rank. */
void ora_matmult_a11(int mx, int my, int mz, const double *coords, const double *eta,
                     const uint8_t *mask, const double *x, double *y, int variant)
{
  const int64_t n = nvel(mx, my, mz);
  double *xl = (double *)malloc(sizeof(double) * n);
  memcpy(xl, x, sizeof(double) * n);
  ora_bc_zero(n, mask, xl);
  memset(y, 0, sizeof(double) * n);
  if (variant == 1) ora_a11_ref(mx, my, mz, coords, eta, xl, y);
  else ora_a11_tensor(mx, my, mz, coords, eta, xl, y);
  ora_bc_copy(n, mask, x, y);
  free(xl);
}

/* MatGetDiagonal_MFStokes_A11 (stokes_operators.c:1072-1113). */
void ora_getdiag_a11(int mx, int my, int mz, const double *coords, const double *eta,
                     const uint8_t *mask, double *y)
{
  const int64_t n = nvel(mx, my, mz);
  memset(y, 0, sizeof(double) * n);
  ora_a11_diag(mx, my, mz, coords, eta, y);
  ora_bc_value(n, mask, 1.0, y);
}

/* MatMult_MFStokes_A12 (stokes_operators.c:1301-1370): no pressure BC, velocity
 * Dirichlet rows zeroed. variant 0 = AVX algorithm, 1 = ref. */
void ora_matmult_a12(int mx, int my, int mz, const double *coords, const uint8_t *mask,
                     const double *p, double *yu, int variant)
{
  const int64_t n = nvel(mx, my, mz);
  memset(yu, 0, sizeof(double) * n);
  if (variant == 1) ora_a12_ref(mx, my, mz, coords, p, yu);
  else ora_a12_tensor(mx, my, mz, coords, p, yu);
  ora_bc_value(n, mask, 0.0, yu);
}

/* MatMult_MFStokes_A21 (stokes_operators.c:1444-1509): Dirichlet columns of u
 * zeroed, no pressure BC. */
void ora_matmult_a21(int mx, int my, int mz, const double *coords, const uint8_t *mask,
                     const double *u, double *yp)
{
  const int64_t n = nvel(mx, my, mz);
  const int64_t nel = (int64_t)mx * my * mz;
  double *ul = (double *)malloc(sizeof(double) * n);
  memcpy(ul, u, sizeof(double) * n);
  ora_bc_zero(n, mask, ul);
  memset(yp, 0, sizeof(double) * 4 * nel);
  ora_a21_ref(mx, my, mz, coords, ul, yp);
  free(ul);
}

/* ---- marker -> Gauss-point coefficients (Q1 projection) ------------------
 * Restates src/material_point_utils.c:1090-1190 (_SwarmUpdateGauss
 * PropertiesLocalL2ProjectionQ1_MPntPStokes_FineGrid) and :957-1088
 * (..._InterpolateToQuadratePoints) on one rank:
 *   node sums over the markers p of element wil[p], in marker order:
 *     A1 += N_i eta_p, A2 += N_i rho_p, B += N_i, where N_i is the Q1 basis
 *     (pTatinConstructNI_Q1_3D, :503-520) at xi_p on the 8 element vertices
 *     (Q2 nodes 0,2,6,8,18,20,24,26) and 1 on the other 19 nodes;
 *   A1 /= B, A2 /= B;
 *   per element and Gauss point q: sum of the Q1 basis at xi_q times the
 *   vertex values, clamped to [min, max] of the element's 27 node values.
 * The Gauss abscissae are those of QuadratureCreateGauss_3pnt_3D
 * (src/quadrature.c:136-167): +-0.774596669241483, 0. */
static void q1_basis(const double xi[3], double N[8])
{
  const double x = xi[0], y = xi[1], z = xi[2];
  N[0] = 0.125 * (1.0 - x) * (1.0 - y) * (1.0 - z);
  N[1] = 0.125 * (1.0 + x) * (1.0 - y) * (1.0 - z);
  N[2] = 0.125 * (1.0 - x) * (1.0 + y) * (1.0 - z);
  N[3] = 0.125 * (1.0 + x) * (1.0 + y) * (1.0 - z);
  N[4] = 0.125 * (1.0 - x) * (1.0 - y) * (1.0 + z);
  N[5] = 0.125 * (1.0 + x) * (1.0 - y) * (1.0 + z);
  N[6] = 0.125 * (1.0 - x) * (1.0 + y) * (1.0 + z);
  N[7] = 0.125 * (1.0 + x) * (1.0 + y) * (1.0 + z);
}

static const int q1_vertex_node[8] = {0, 2, 6, 8, 18, 20, 24, 26};

void ora_marker_project(int mx, int my, int mz, int64_t npoints, const int32_t *wil, const double *xi,
                        const double *eta_p, const double *rho_p, double *eta_qp, double *rho_qp)
{
  const int64_t nel = (int64_t)mx * my * mz;
  const int64_t nn = (int64_t)(2 * mx + 1) * (2 * my + 1) * (2 * mz + 1);
  int32_t *el = (int32_t *)malloc(sizeof(int32_t) * 27 * (size_t)(nel > 0 ? nel : 1));
  double *A1 = (double *)calloc((size_t)nn, sizeof(double));
  double *A2 = (double *)calloc((size_t)nn, sizeof(double));
  double *B = (double *)calloc((size_t)nn, sizeof(double));
  const double g[3] = {-0.774596669241483, 0.0, 0.774596669241483};
  if (!el || !A1 || !A2 || !B) goto done;
  ora_elements_q2(mx, my, mz, el);
  for (int64_t p = 0; p < npoints; p++) {
    double N1[8], Ni[27];
    q1_basis(&xi[3 * p], N1);
    for (int i = 0; i < 27; i++) Ni[i] = 1.0;
    for (int v = 0; v < 8; v++) Ni[q1_vertex_node[v]] = N1[v];
    const int32_t *en = &el[27 * (int64_t)wil[p]];
    for (int i = 0; i < 27; i++) {
      A1[en[i]] += Ni[i] * eta_p[p];
      A2[en[i]] += Ni[i] * rho_p[p];
      B[en[i]] += Ni[i];
    }
  }
  for (int64_t k = 0; k < nn; k++) {
    A1[k] = A1[k] / B[k];
    A2[k] = A2[k] / B[k];
  }
  for (int64_t e = 0; e < nel; e++) {
    const int32_t *en = &el[27 * e];
    double lo1 = 1.0e32, hi1 = -1.0e32, lo2 = 1.0e32, hi2 = -1.0e32;
    for (int i = 0; i < 27; i++) {
      if (A1[en[i]] < lo1) lo1 = A1[en[i]];
      if (A1[en[i]] > hi1) hi1 = A1[en[i]];
      if (A2[en[i]] < lo2) lo2 = A2[en[i]];
      if (A2[en[i]] > hi2) hi2 = A2[en[i]];
    }
    for (int q = 0; q < 27; q++) {
      const double xq[3] = {g[q % 3], g[(q / 3) % 3], g[q / 9]};
      double N1[8], a = 0.0, b = 0.0;
      q1_basis(xq, N1);
      for (int v = 0; v < 8; v++) {
        a += N1[v] * A1[en[q1_vertex_node[v]]];
        b += N1[v] * A2[en[q1_vertex_node[v]]];
      }
      if (a < lo1) a = lo1;
      if (a > hi1) a = hi1;
      if (b < lo2) b = lo2;
      if (b > hi2) b = hi2;
      eta_qp[27 * e + q] = a;
      rho_qp[27 * e + q] = b;
    }
  }
done:
  free(el); free(A1); free(A2); free(B);
}

double ora_a11_flops(int64_t nel)
{
  return (double)nel * (9.0 * 3 * NQP * (6 + 6 + 6) + NQP * (14 + 1 + 27) + NQP * (5 * 9 + 6 + 6 + 6 * 9));
}
