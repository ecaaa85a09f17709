/*
 * CPU oracle for the pTatin3D matrix-free Q2-P1disc Stokes operator.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the GPU kernels are
 * compared against (tests, the smoke check and the CPU-baseline leg of the
 * benchmark).  Nothing in the product path links or calls it.
 *
 * It restates, in plain C without PETSc, the reference's CPU arithmetic for
 * one MPI rank (ghosted local numbering == global numbering):
 *   - element -> node table        src/dmda_element_q2p1.c:368-469
 *   - Q2 basis / 3x3 Gauss tables  src/element_utils_q2.c:276-333
 *   - geometry (J, detJ, dN/dx)    src/element_utils_q2.c:399-476
 *   - P1 "global relative" basis   src/element_utils_q2.c:183-224
 *   - tensor A11                   src/stokes_operators_tensor.c:40-286
 *   - "ref" A11                    src/stokes_operators_mf.c:237-351
 *                                  + src/stokes_q2p1_mf_operators_def.c:151-257
 *   - diag(A11)                    src/stokes_operators_mf.c:71-135
 *                                  + src/stokes_q2p1_mf_operators_diag_def.c:120-205
 *   - A21 (B u, divergence)        src/stokes_operators_mf.c:862-937
 *                                  + src/stokes_q2p1_mf_operators_def.c:517-538
 *   - A12 (B^T p, gradient), ref   src/stokes_operators_mf.c:792-860
 *                                  + src/stokes_q2p1_mf_operators_def.c:423-516
 *   - A12, AVX algorithm (scalar)  src/stokes_operators_avx.c:640-829
 *   - BC masking semantics         src/dmda_bcs.c:490-541,581-608,655-689
 *   - MatShell wrappers            src/stokes_operators.c:1072-1113,1156-1222,
 *                                  1301-1370,1444-1509
 *
 * Layouts (identical to the reference's single-rank local vectors):
 *   coords[3*N], u[3*N], y[3*N]  interleaved (x,y,z) per node, node id
 *                                i + j*X + k*X*Y with X=2mx+1, Y=2my+1
 *   eta[27*nel]                  element-major, quadrature point minor,
 *                                qp index = a*9 + b*3 + c (c along xi)
 *   p[4*nel]                     element-major, 4 P1 dofs per element
 *   mask[3*N]                    nonzero = Dirichlet dof
 */
#ifndef PT_ORACLE_H
#define PT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void ora_gauss3(double x[3], double w[3]);
void ora_elements_q2(int mx, int my, int mz, int32_t *elnidx);

/* Element-loop kernels: accumulate (+=) unassembled contributions into y. */
void ora_a11_tensor(int mx, int my, int mz, const double *coords, const double *eta,
                    const double *u, double *y);
void ora_a11_ref(int mx, int my, int mz, const double *coords, const double *eta,
                 const double *u, double *y);
void ora_a11_diag(int mx, int my, int mz, const double *coords, const double *eta,
                  double *y);
void ora_a21_ref(int mx, int my, int mz, const double *coords, const double *u, double *yp);
void ora_a12_ref(int mx, int my, int mz, const double *coords, const double *p, double *yu);
void ora_a12_tensor(int mx, int my, int mz, const double *coords, const double *p, double *yu);

/* BCList semantics on a dof mask (scale == 1). */
void ora_bc_zero(int64_t n, const uint8_t *mask, double *x);
void ora_bc_copy(int64_t n, const uint8_t *mask, const double *x, double *y);
void ora_bc_value(int64_t n, const uint8_t *mask, double value, double *y);

/* MatShell-level operators (variant 0 = tensor, 1 = ref). y is overwritten. */
void ora_matmult_a11(int mx, int my, int mz, const double *coords, const double *eta,
                     const uint8_t *mask, const double *x, double *y, int variant);
void ora_getdiag_a11(int mx, int my, int mz, const double *coords, const double *eta,
                     const uint8_t *mask, double *y);
void ora_matmult_a12(int mx, int my, int mz, const double *coords, const uint8_t *mask,
                     const double *p, double *yu, int variant);
void ora_matmult_a21(int mx, int my, int mz, const double *coords, const uint8_t *mask,
                     const double *u, double *yp);

/* Reference flop count of one tensor A11 apply (stokes_operators_tensor.c:279-281). */
/* Marker -> Gauss-point (eta, rho), the reference's Q1 projection on one rank
 * (src/material_point_utils.c:957-1190). */
void ora_marker_project(int mx, int my, int mz, int64_t npoints, const int32_t *wil, const double *xi,
                        const double *eta_p, const double *rho_p, double *eta_qp, double *rho_qp);
double ora_a11_flops(int64_t nel);

/* Momentum residual FormFunctionLocal_U (src/stokes_form_function.c:99-243):
 * ru += A11 u + A12 p - sum_q w detJ N fu_q; fu holds 3 values per Gauss point. */
void ora_residual_u(int mx, int my, int mz, const double *coords, const double *eta, const double *fu,
                    const double *u, const double *pr, double *ru);

/* Number of OpenMP threads the element loops use (1 when built without OpenMP). */
int ora_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
