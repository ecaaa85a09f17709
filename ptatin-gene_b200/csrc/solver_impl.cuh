// Krylov solves of A11 u = f on the device (the precision and serving forms).
//
// This is the consumer side of the operator: pTatin3D solves the viscous block
// with FGMRES preconditioned by multigrid whose smoothers are Chebyshev–Jacobi
// sweeps on the A11 shell (src/ptatin_driver_linear_ts.c:559-883, the PETSc
// KSPFGMRES / KSPCHEBYSHEV + PCJACOBI configuration with the eigenvalue window
// "esteig 0,0.2,0,1.1").  Here the fine level alone is solved:
//
//   outer  FGMRES(m) (right, flexible) or flexible CG, FP64 residuals,
//          FP64 MatMult_MFStokes_A11 (BC rows identity), FP64 dot products;
//   inner  Chebyshev of degree k on D^-1 A with D = MatGetDiagonal (BC slots 1),
//          window [emin, emax] * lambda_max(D^-1 A), lambda_max from a few
//          Jacobi-PCG (Lanczos) steps; optionally FP32 vectors, FP32 A11 apply
//          and FP32 D^-1, the inner solve rounded back to FP64 for the outer.
//
// Dot products are deterministic: a fixed grid, a fixed per-thread stride
// order and fixed tree reductions, so a solve is bitwise repeatable.
// Included from pt_b200.cu after struct pt_op.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

namespace {

constexpr int RED_BLOCKS = 148 * 4;
constexpr int RED_THREADS = 256;
constexpr int MDOT_CHUNK = 8;

template <typename T>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// partial[j*RED_BLOCKS + b] = sum over this block's strided indices of v_j[i]*w[i], j < nv (<= MDOT_CHUNK)
__global__ void __launch_bounds__(RED_THREADS) mdot_partial_kernel(const double *const *__restrict__ V, int nv,
                                                                  const double *__restrict__ w, int64_t n,
                                                                  double *__restrict__ partial)
{
  __shared__ double sh[RED_THREADS];
  double acc[MDOT_CHUNK];
#pragma unroll
  for (int j = 0; j < MDOT_CHUNK; j++) acc[j] = 0.0;
  const int64_t stride = (int64_t)RED_BLOCKS * RED_THREADS;
  for (int64_t i = (int64_t)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += stride) {
    const double wi = w[i];
#pragma unroll
    for (int j = 0; j < MDOT_CHUNK; j++)
      if (j < nv) acc[j] = fma(V[j][i], wi, acc[j]);
  }
  for (int j = 0; j < nv; j++) {
    const double s = block_sum<double>(acc[j], sh);
    if (threadIdx.x == 0) partial[j * RED_BLOCKS + blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(RED_THREADS) mdot_final_kernel(const double *__restrict__ partial, int nv,
                                                                double *__restrict__ out)
{
  __shared__ double sh[RED_THREADS];
  for (int j = 0; j < nv; j++) {
    double a = 0.0;
    for (int b = threadIdx.x; b < RED_BLOCKS; b += RED_THREADS) a += partial[j * RED_BLOCKS + b];
    const double s = block_sum<double>(a, sh);
    if (threadIdx.x == 0) out[j] = s;
  }
}

// w -= sum_j h[j] v_j  (j < nv <= 64), fixed order
__global__ void maxpy_kernel(const double *const *__restrict__ V, const double *__restrict__ h, int nv,
                             double *__restrict__ w, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = w[i];
    for (int j = 0; j < nv; j++) v = fma(-h[j], V[j][i], v);
    w[i] = v;
  }
}

// x += sum_j h[j] z_j
__global__ void maxpy_add_kernel(const double *const *__restrict__ Z, const double *__restrict__ h, int nv,
                                 double *__restrict__ x, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = x[i];
    for (int j = 0; j < nv; j++) v = fma(h[j], Z[j][i], v);
    x[i] = v;
  }
}

// y = a x + b y
template <typename T>
__global__ void axpby_kernel(T a, const T *__restrict__ x, T b, T *__restrict__ y, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// r = b - r  (r holds A x on entry)
__global__ void resid_kernel(const double *__restrict__ b, double *__restrict__ r, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - r[i];
}

template <typename TO, typename TI>
__global__ void convert_kernel(const TI *__restrict__ a, TO *__restrict__ b, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (TO)a[i];
}

__global__ void reciprocal_kernel(const double *__restrict__ d, double *__restrict__ dinv, float *__restrict__ dinv32,
                                  int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = 1.0 / d[i];
    dinv[i] = v;
    dinv32[i] = (float)v;
  }
}

// z = s * dinv .* r ; d = z
template <typename T>
__global__ void cheb_first_kernel(T s, const T *__restrict__ dinv, const T *__restrict__ r, T *__restrict__ d,
                                  T *__restrict__ z, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T v = s * dinv[i] * r[i];
    d[i] = v;
    z[i] = v;
  }
}

// az holds A z on entry: d = alpha d + beta dinv .* (r - A z); z += d
template <typename T>
__global__ void cheb_step_kernel(T alpha, T beta, const T *__restrict__ dinv, const T *__restrict__ r,
                                 const T *__restrict__ az, T *__restrict__ d, T *__restrict__ z, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T v = alpha * d[i] + beta * dinv[i] * (r[i] - az[i]);
    d[i] = v;
    z[i] += v;
  }
}

// deterministic pseudo-random vector in [-1, 1] (splitmix64 of the index)
__global__ void hash_vec_kernel(double *__restrict__ x, int64_t n, uint64_t seed)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = (uint64_t)i + seed * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

unsigned vgrid(int64_t n)
{
  const int64_t b = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

// Largest eigenvalue of a symmetric tridiagonal matrix (diagonal a[0..n),
// off-diagonal b[0..n-1)) by bisection on Sturm counts.  Host and device.
__host__ __device__ inline double tridiag_lmax(const double *a, const double *b, int n)
{
  if (n == 0) return 0.0;
  double lo = a[0], hi = a[0];
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < n ? fabs(b[i]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    int c = 0;
    double q = a[0] - mid;
    if (q < 0) c++;
    for (int i = 1; i < n; i++) {
      const double qq = (q == 0.0) ? 1e-300 : q;
      q = a[i] - mid - b[i - 1] * b[i - 1] / qq;
      if (q < 0) c++;
    }
    if (c >= n) hi = mid;
    else lo = mid;
  }
  return hi;
}

double tridiag_lambda_max(const std::vector<double> &a, const std::vector<double> &b)
{
  return tridiag_lmax(a.data(), b.data(), (int)a.size());
}

}  // namespace

#include "mg_impl.cuh"

struct pt_solver {
  pt_op *op;
  pt_solve_opts o;
  int64_t n;
  // FP64 work vectors
  double *r, *w, *x0, *dinv, *t1, *t2, *t3;
  double *V, *Z;  // FGMRES bases ((m+1) and m vectors) or FCG p/q/z/rold
  double *partial, *dres;  // reduction scratch
  double *hbuf;            // coefficient staging (device)
  double *hhost;           // pinned host copy
  const double **dptr;     // device array of vector pointers
  // FP32 smoother vectors
  float *dinv32, *r32, *z32, *d32, *az32;
  double lambda_max;
  bool have_diag;
  int64_t n64, n32;
  pt_mg *mg;
  bool setup_done;
  uint64_t op_state;  // op->state the set-up was made for
};

namespace {

pt_status sv_dots(pt_solver *s, const double *const *vecs_host, int nv, const double *w, double *out, int64_t n = -1)
{
  if (n < 0) n = s->n;
  // vector-pointer table goes through a small device array
  for (int base = 0; base < nv; base += MDOT_CHUNK) {
    const int k = std::min(MDOT_CHUNK, nv - base);
    PT_CUDA(cudaMemcpyAsync(s->dptr, vecs_host + base, sizeof(double *) * k, cudaMemcpyHostToDevice, s->op->stream));
    mdot_partial_kernel<<<RED_BLOCKS, RED_THREADS, 0, s->op->stream>>>(s->dptr, k, w, n, s->partial);
    PT_LAUNCHED(s->op);
    mdot_final_kernel<<<1, RED_THREADS, 0, s->op->stream>>>(s->partial, k, s->dres + base);
    PT_LAUNCHED(s->op);
  }
  PT_CUDA(cudaMemcpyAsync(s->hhost, s->dres, sizeof(double) * nv, cudaMemcpyDeviceToHost, s->op->stream));
  PT_CUDA(cudaStreamSynchronize(s->op->stream));
  for (int j = 0; j < nv; j++) out[j] = s->hhost[j];
  return PT_OK;
}

pt_status sv_dot(pt_solver *s, const double *a, const double *b, double *out, int64_t n = -1)
{
  const double *v[1] = {a};
  return sv_dots(s, v, 1, b, out, n);
}

// w -= sum h_j v_j  (sign = -1) or x += sum h_j z_j (sign = +1)
pt_status sv_maxpy(pt_solver *s, const double *const *vecs_host, const double *h, int nv, double *w, int sign)
{
  for (int base = 0; base < nv; base += 64) {
    const int k = std::min(64, nv - base);
    PT_CUDA(cudaMemcpyAsync(s->dptr + 64, vecs_host + base, sizeof(double *) * k, cudaMemcpyHostToDevice, s->op->stream));
    PT_CUDA(cudaMemcpyAsync(s->hbuf, h + base, sizeof(double) * k, cudaMemcpyHostToDevice, s->op->stream));
    if (sign < 0) maxpy_kernel<<<vgrid(s->n), 256, 0, s->op->stream>>>(s->dptr + 64, s->hbuf, k, w, s->n);
    else maxpy_add_kernel<<<vgrid(s->n), 256, 0, s->op->stream>>>(s->dptr + 64, s->hbuf, k, w, s->n);
    PT_LAUNCHED(s->op);
    // the host arrays are reused right away: keep the copies ordered
    PT_CUDA(cudaStreamSynchronize(s->op->stream));
  }
  return PT_OK;
}

template <typename T>
pt_status sv_axpby(pt_solver *s, T a, const T *x, T b, T *y, int64_t n = -1)
{
  if (n < 0) n = s->n;
  axpby_kernel<T><<<vgrid(n), 256, 0, s->op->stream>>>(a, x, b, y, n);
  PT_LAUNCHED(s->op);
  return PT_OK;
}

pt_status sv_matmult64(pt_solver *s, const double *x, double *y)
{
  s->n64++;
  return pt_matmult_a11_d(s->op, x, y);
}

pt_status sv_matmult32(pt_solver *s, const float *x, float *y)
{
  s->n32++;
  return pt_matmult_a11_f32_d(s->op, x, y);
}

pt_status sv_setup_diag(pt_solver *s)
{
  if (s->have_diag) return PT_OK;
  pt_status st = pt_getdiag_a11_d(s->op, s->t1);
  if (st != PT_OK) return st;
  reciprocal_kernel<<<vgrid(s->n), 256, 0, s->op->stream>>>(s->t1, s->dinv, s->dinv32, s->n);
  PT_LAUNCHED(s->op);
  s->have_diag = true;
  return PT_OK;
}

// lambda_max(D^-1 A) of operator `op` (n dofs, inverse diagonal dinv) from
// eig_its steps of Jacobi-PCG on a pseudo-random rhs (Lanczos tridiagonal).
// Uses the solver's FP64 work vectors (fine-level size >= n).
template <typename ApplyFn>
pt_status sv_lanczos_fn(pt_solver *s, int64_t n, const double *dinv, double *lmax, ApplyFn apply)
{
  double *b = s->t2, *p = s->t3, *q = s->w, *r = s->r, *z = s->t1;
  cudaStream_t st = s->op->stream;
  hash_vec_kernel<<<vgrid(n), 256, 0, st>>>(b, n, 12345u);
  PT_LAUNCHED(s->op);
  PT_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  cheb_first_kernel<double><<<vgrid(n), 256, 0, st>>>(1.0, dinv, r, z, p, n);  // z = p = D^-1 r
  PT_LAUNCHED(s->op);
  double rz;
  pt_status stt = sv_dot(s, r, z, &rz, n);
  if (stt != PT_OK) return stt;
  std::vector<double> alphas, betas, diag, off;
  for (int k = 0; k < s->o.eig_its && rz > 0.0; k++) {
    if ((stt = apply(p, q)) != PT_OK) return stt;
    double pq;
    if ((stt = sv_dot(s, p, q, &pq, n)) != PT_OK) return stt;
    if (!(pq > 0.0)) break;
    const double alpha = rz / pq;
    if ((stt = sv_axpby<double>(s, -alpha, q, 1.0, r, n)) != PT_OK) return stt;
    cheb_first_kernel<double><<<vgrid(n), 256, 0, st>>>(1.0, dinv, r, z, z, n);
    PT_LAUNCHED(s->op);
    double rz_new;
    if ((stt = sv_dot(s, r, z, &rz_new, n)) != PT_OK) return stt;
    const double beta = rz_new / rz;
    if ((stt = sv_axpby<double>(s, 1.0, z, beta, p, n)) != PT_OK) return stt;
    alphas.push_back(alpha);
    betas.push_back(beta);
    rz = rz_new;
  }
  const int m = (int)alphas.size();
  if (m == 0) return fail(PT_ERR_STATE, "eigenvalue estimate failed (A11 not positive definite?)");
  for (int k = 0; k < m; k++) {
    double t = 1.0 / alphas[k];
    if (k > 0) t += betas[k - 1] / alphas[k - 1];
    diag.push_back(t);
    if (k + 1 < m) off.push_back(std::sqrt(betas[k]) / alphas[k]);
  }
  *lmax = tridiag_lambda_max(diag, off);
  return PT_OK;
}

pt_status sv_lanczos(pt_solver *s, pt_op *op, int64_t n, const double *dinv, double *lmax)
{
  return sv_lanczos_fn(s, n, dinv, lmax, [&](const double *x, double *y) {
    if (op == s->op) s->n64++;
    return pt_matmult_a11_d(op, x, y);
  });
}

pt_status sv_estimate_lambda(pt_solver *s) { return sv_lanczos(s, s->op, s->n, s->dinv, &s->lambda_max); }

// ---- multigrid set-up -------------------------------------------------------

void mg_free(pt_mg *mg)
{
  if (!mg) return;
  if (mg->gexec) cudaGraphExecDestroy(mg->gexec);
  for (pt_mg_level &L : mg->lv) {
    void *p[] = {L.dinv64, L.dinv32, L.x, L.b, L.r, L.d, L.az, L.dl, L.t1, L.Ae, L.ye, L.Ainv, L.Ah, L.Ascale};
    for (void *q : p) cudaFree(q);
    if (L.Ae64 && (void *)L.Ae64 != L.Ae) cudaFree(L.Ae64);
    if (L.own && L.op) pt_op_destroy(L.op);
  }
  delete mg;
}

// Coarse level of level f: half the elements per axis, coordinates and
// Dirichlet mask injected; vf_c (the coarse vertex viscosity) restricted from
// vf_f and interpolated to the coarse Gauss points.
pt_status mg_coarsen(const pt_op *f, const double *vf_f, double *vf_c, pt_op **out)
{
  pt_mesh_desc d{};
  d.mx = f->mx / 2; d.my = f->my / 2; d.mz = f->mz / 2;
  pt_op *c = nullptr;
  pt_status st = pt_op_create(&d, &c);
  if (st != PT_OK) return st;
  *out = c;  // the caller owns it from here on
  if ((st = pt_op_set_stream(c, (void *)f->stream)) != PT_OK) return st;
  // small levels keep their own element matrices (mg_level_setup)
  c->a11_kernel = (f->a11_kernel == A11_EBE) ? A11_STREAM : f->a11_kernel;
  const MgBox fb = mgbox(f), cb = mgbox(c);
  inject_coords_kernel<<<vgrid(c->nnodes), 256, 0, c->stream>>>(fb, cb, f->d_coords, c->d_coords);
  PT_LAUNCHED(c);
  if ((st = finish_coords(c)) != PT_OK) return st;
  restrict_vertex_kernel<<<vgrid((int64_t)(cb.mx + 1) * (cb.my + 1) * (cb.mz + 1)), 256, 0, c->stream>>>(fb, cb, vf_f,
                                                                                                        vf_c);
  PT_LAUNCHED(c);
  eta_from_vertex_kernel<<<vgrid(27 * c->nel), 256, 0, c->stream>>>(cb, vf_c, c->d_eta);
  PT_LAUNCHED(c);
  if ((st = finish_eta(c)) != PT_OK) return st;
  inject_mask_kernel<<<vgrid(c->nnodes), 256, 0, c->stream>>>(fb, cb, f->d_mask, c->d_mask);
  PT_LAUNCHED(c);
  if (f->has_mask) return finish_mask(c);  // the packed bits the streaming kernel reads
  return PT_OK;
}

constexpr int64_t MG_EBE_MAX_ELEMENTS = 32768;  // levels up to 32^3 elements store element matrices
constexpr int64_t MG_DENSE_MAX_DOFS = 1200;     // coarsest level solved by a dense inverse up to this size

// Dense inverse of the coarsest level's masked operator (Dirichlet rows and
// columns replaced by the identity), from its FP64 element matrices:
// assembled on the host, Cholesky-factored, inverted, uploaded as T.
pt_status mg_dense_inverse(pt_mg_level &L, bool fp32)
{
  const pt_op *op = L.op;
  const int64_t n = L.n, nel = op->nel;
  double *dAe = L.Ae64;  // Galerkin level: its own matrices; else re-discretised ones
  if (!dAe) {
    PT_CUDA(cudaMalloc(&dAe, sizeof(double) * ptk::EBE_LD * nel));
    ptk::element_matrix_kernel<double><<<(unsigned)nel, 96, 0, op->stream>>>(op->box, op->d_coords, op->d_eta, dAe);
  }
  std::vector<double> Ae(ptk::EBE_LD * nel), A(n * n, 0.0);
  std::vector<uint8_t> mask(n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(Ae.data(), dAe, sizeof(double) * Ae.size(), cudaMemcpyDeviceToHost, op->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mask.data(), op->d_mask, n, cudaMemcpyDeviceToHost, op->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
  if (dAe != L.Ae64) cudaFree(dAe);
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "coarse element matrices: %s", cudaGetErrorString(e));
  const int64_t X = op->box.X, XY = op->box.XY;
  for (int64_t el = 0; el < nel; el++) {
    const int64_t ei = el % op->mx, ej = (el / op->mx) % op->my, ek = el / ((int64_t)op->mx * op->my);
    int64_t g[81];
    for (int nn = 0; nn < 27; nn++) {
      const int64_t node = (2 * ei + nn % 3) + (2 * ej + (nn / 3) % 3) * X + (2 * ek + nn / 9) * XY;
      for (int l = 0; l < 3; l++) g[3 * nn + l] = 3 * node + l;
    }
    const double *m = &Ae[el * ptk::EBE_LD];
    for (int jj = 0; jj < 81; jj++) {
      if (mask[g[jj]]) continue;
      for (int ii = 0; ii < 81; ii++)
        if (!mask[g[ii]]) A[g[ii] * n + g[jj]] += m[ptk::ebe_sym(ii, jj)];
    }
  }
  for (int64_t i = 0; i < n; i++)
    if (mask[i]) A[i * n + i] = 1.0;
  // A = L L^T (lower triangle in place), W = L^-1, A^-1 = W^T W
  for (int64_t j = 0; j < n; j++) {
    double d = A[j * n + j];
    for (int64_t k = 0; k < j; k++) d -= A[j * n + k] * A[j * n + k];
    if (!(d > 0.0)) return fail(PT_ERR_STATE, "coarse operator is not positive definite");
    d = std::sqrt(d);
    A[j * n + j] = d;
    for (int64_t i = j + 1; i < n; i++) {
      double v = A[i * n + j];
      for (int64_t k = 0; k < j; k++) v -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = v / d;
    }
  }
  std::vector<double> W(n * n, 0.0);
  for (int64_t c = 0; c < n; c++) {  // column c of L^-1 by forward substitution
    W[c * n + c] = 1.0 / A[c * n + c];
    for (int64_t i = c + 1; i < n; i++) {
      double v = 0.0;
      for (int64_t k = c; k < i; k++) v -= A[i * n + k] * W[k * n + c];
      W[i * n + c] = v / A[i * n + i];
    }
  }
  std::vector<double> inv(n * n, 0.0);
  for (int64_t i = 0; i < n; i++)
    for (int64_t j = 0; j <= i; j++) {
      double v = 0.0;
      for (int64_t k = i; k < n; k++) v += W[k * n + i] * W[k * n + j];
      inv[i * n + j] = inv[j * n + i] = v;
    }
  const size_t ts = fp32 ? sizeof(float) : sizeof(double);
  PT_CUDA(cudaMalloc(&L.Ainv, ts * n * n));
  if (fp32) {
    std::vector<float> f(inv.begin(), inv.end());
    PT_CUDA(cudaMemcpy(L.Ainv, f.data(), ts * n * n, cudaMemcpyHostToDevice));
  } else {
    PT_CUDA(cudaMemcpy(L.Ainv, inv.data(), ts * n * n, cudaMemcpyHostToDevice));
  }
  return PT_OK;
}

// Work vectors, inverse diagonal and lambda_max(D^-1 A) of level L; element
// matrices when the level is small; the dense inverse on a small coarsest level.
pt_status mg_level_setup(pt_solver *s, pt_mg &mg, pt_mg_level &L, const pt_op *next)
{
  const size_t ts = mg.fp32 ? sizeof(float) : sizeof(double);
  L.n = L.op->nvel;
  L.nel = L.op->nel;
  PT_CUDA(cudaMalloc(&L.dinv64, sizeof(double) * L.n));
  PT_CUDA(cudaMalloc(&L.dinv32, sizeof(float) * L.n));
  void **vecs[] = {&L.x, &L.b, &L.r, &L.d, &L.az, &L.dl};
  for (void **v : vecs) PT_CUDA(cudaMalloc(v, ts * L.n));
  if (next) {  // transfer temporaries: 3 (2mcx+1)(2my+1)(2mz+1) values each
    const int64_t nt = 3LL * (2 * next->mx + 1) * (2 * L.op->my + 1) * (2 * L.op->mz + 1);
    PT_CUDA(cudaMalloc(&L.t1, 2 * ts * nt));
    L.t2 = (char *)L.t1 + ts * nt;
  }
  pt_status st = PT_OK;
  if (L.Ae64) {
    // Galerkin level: diagonal, lambda_max and applies from its element matrices
    PT_CUDA(cudaMalloc(&L.ye, sizeof(double) * 81 * L.nel));
    ptk::ebe_diag_kernel<<<vgrid(L.n), 256, 0, L.op->stream>>>(L.op->box, L.Ae64, s->t1);
    PT_LAUNCHED(L.op);
    if ((st = bc_value(L.op, 1.0, s->t1)) != PT_OK) return st;
  } else if ((st = pt_getdiag_a11_d(L.op, s->t1)) != PT_OK) {
    return st;
  }
  reciprocal_kernel<<<vgrid(L.n), 256, 0, s->op->stream>>>(s->t1, L.dinv64, L.dinv32, L.n);
  PT_LAUNCHED(s->op);
  if (L.Ae64) {
    st = sv_lanczos_fn(s, L.n, L.dinv64, &L.lmax, [&](const double *x, double *y) {
      ptk::ebe_apply_kernel<double, true><<<(unsigned)L.nel, 96, 0, L.op->stream>>>(L.op->box, L.Ae64, x,
                                                                                     L.op->d_mask, (double *)L.ye);
      PT_LAUNCHED(L.op);
      ptk::ebe_gather_kernel<double, true><<<vgrid(L.n), 256, 0, L.op->stream>>>(L.op->box, (const double *)L.ye, x,
                                                                                L.op->d_mask, y);
      PT_LAUNCHED(L.op);
      return PT_OK;
    });
    if (st != PT_OK) return st;
    if (!next && L.n <= MG_DENSE_MAX_DOFS) return mg_dense_inverse(L, mg.fp32);
    if (mg.fp32 && mg.coarse_half) {
      PT_CUDA(cudaMalloc(&L.Ah, sizeof(__half) * ptk::EBE_LD * L.nel));
      PT_CUDA(cudaMalloc(&L.Ascale, sizeof(float) * L.nel));
      ptk::ebe_to_half_kernel<<<(unsigned)L.nel, 128, 0, L.op->stream>>>(L.Ae64, L.Ah, L.Ascale);
      PT_LAUNCHED(L.op);
    } else if (mg.fp32) {
      PT_CUDA(cudaMalloc(&L.Ae, sizeof(float) * ptk::EBE_LD * L.nel));
      ptk::convert_kernel<float><<<vgrid(ptk::EBE_LD * L.nel), 256, 0, L.op->stream>>>(L.Ae64, (float *)L.Ae,
                                                                                     ptk::EBE_LD * L.nel);
      PT_LAUNCHED(L.op);
    } else {
      L.Ae = L.Ae64;
    }
    return PT_OK;
  }
  if ((st = sv_lanczos(s, L.op, L.n, L.dinv64, &L.lmax)) != PT_OK) return st;
  if (!mg.assembled) return PT_OK;
  if (!next && L.n <= MG_DENSE_MAX_DOFS && (st = mg_dense_inverse(L, mg.fp32)) != PT_OK) return st;
  if (L.nel <= MG_EBE_MAX_ELEMENTS && !L.Ainv) {
    PT_CUDA(cudaMalloc(&L.Ae, ts * ptk::EBE_LD * L.nel));
    PT_CUDA(cudaMalloc(&L.ye, ts * 81 * L.nel));
    if (mg.fp32)
      ptk::element_matrix_kernel<float><<<(unsigned)L.nel, 96, 0, L.op->stream>>>(L.op->box, L.op->d_coords, L.op->d_eta,
                                                                             (float *)L.Ae);
    else
      ptk::element_matrix_kernel<double><<<(unsigned)L.nel, 96, 0, L.op->stream>>>(L.op->box, L.op->d_coords,
                                                                              L.op->d_eta, (double *)L.Ae);
    PT_LAUNCHED(L.op);
  }
  return PT_OK;
}

constexpr int64_t MG_GALERKIN_MAX_ELEMENTS = 262144;  // Galerkin levels up to 64^3 elements (7.0 GB FP64, packed)

// Galerkin coarse operators (mg_assembled = 2): every level from the first
// one of <= MG_GALERKIN_MAX_ELEMENTS elements down gets element matrices
// P^T A P from the level above -- from that level's quadrature when it runs
// matrix-free (the reference's OP_TYPE_MFGALERKIN), from its Galerkin
// matrices below that (OP_TYPE_GALERKIN).  Levels above stay re-discretised.
pt_status mg_galerkin(pt_mg &mg)
{
  constexpr size_t smem = ptk::galerkin_smem_bytes();
  pt_status as = kernel_attrs((const void *)ptk::galerkin_kernel<true>, smem, false);
  if (as == PT_OK) as = kernel_attrs((const void *)ptk::galerkin_kernel<false>, smem, false);
  if (as != PT_OK) return as;
  for (size_t l = 1; l < mg.lv.size(); l++) {
    pt_mg_level &F = mg.lv[l - 1], &C = mg.lv[l];
    if (!F.Ae64 && C.op->nel > MG_GALERKIN_MAX_ELEMENTS) continue;
    PT_CUDA(cudaMalloc(&C.Ae64, sizeof(double) * ptk::EBE_LD * C.op->nel));
    ptk::GalerkinArgs a;
    a.fb = F.op->box;
    a.cmx = C.op->mx; a.cmy = C.op->my; a.cmz = C.op->mz;
    a.coords = F.op->d_coords;
    a.eta = F.op->d_eta;
    a.Af = F.Ae64;
    a.mask = F.op->has_mask ? F.op->d_mask : nullptr;
    a.Ac = C.Ae64;
    if (F.Ae64) ptk::galerkin_kernel<false><<<(unsigned)C.op->nel, ptk::GAL_THREADS, smem, C.op->stream>>>(a);
    else ptk::galerkin_kernel<true><<<(unsigned)C.op->nel, ptk::GAL_THREADS, smem, C.op->stream>>>(a);
    PT_LAUNCHED(C.op);
  }
  return PT_OK;
}

pt_status mg_build(pt_solver *s)
{
  if (!s->op->full_box) return fail(PT_ERR_UNSUPPORTED, "multigrid needs a one-rank box (node box = element box)");
  pt_mg *mg = new (std::nothrow) pt_mg();
  if (!mg) return fail(PT_ERR_OOM, "host allocation failed");
  s->mg = mg;  // freed by pt_solver_destroy, also after a failure here
  mg->fp32 = s->o.cheby_fp32 != 0;
  mg->degree = s->o.cheby_degree;
  mg->fine_degree = s->o.mg_fine_degree > 0 ? s->o.mg_fine_degree : s->o.cheby_degree;
  mg->coarse_degree = s->o.mg_coarse_degree > 0 ? s->o.mg_coarse_degree : 24;
  mg->emin = s->o.cheby_emin;
  mg->emax = s->o.cheby_emax;
  mg->coarse_half = s->o.mg_coarse_half != 0;
  mg->use_graph = s->o.pc_graph != 0;
  mg->assembled = s->o.mg_assembled != 0;
  const int maxl = s->o.mg_levels > 0 ? s->o.mg_levels : 32;
  pt_mg_level L0{};
  L0.op = s->op;
  mg->lv.push_back(L0);
  pt_status st = upload_q1_table();
  if (st != PT_OK) return st;
  // two vertex-field buffers (fine level's size), swapped level by level
  const pt_op *op = s->op;
  const int64_t nv0 = (int64_t)(op->mx + 1) * (op->my + 1) * (op->mz + 1);
  double *vf[2] = {nullptr, nullptr};
  PT_CUDA(cudaMalloc(&vf[0], sizeof(double) * 2 * nv0));
  vf[1] = vf[0] + nv0;
  vertex_field_kernel<<<vgrid(nv0), 256, 0, op->stream>>>(mgbox(op), op->d_eta, vf[0]);
  st = cudaGetLastError() == cudaSuccess ? PT_OK : fail(PT_ERR_CUDA, "vertex field kernel launch failed");
  while (st == PT_OK && (int)mg->lv.size() < maxl) {
    const pt_op *f = mg->lv.back().op;
    if ((f->mx & 1) || (f->my & 1) || (f->mz & 1) || f->mx < 4 || f->my < 4 || f->mz < 4) break;
    pt_mg_level L{};
    L.own = true;
    mg->lv.push_back(L);
    const int cur = ((int)mg->lv.size() - 2) & 1;
    st = mg_coarsen(f, vf[cur], vf[cur ^ 1], &mg->lv.back().op);
  }
  if (st == PT_OK && cudaStreamSynchronize(op->stream) != cudaSuccess) st = fail(PT_ERR_CUDA, "multigrid set-up failed");
  cudaFree(vf[0]);
  if (st != PT_OK) return st;
  if (s->o.mg_assembled == 2 && (st = mg_galerkin(*mg)) != PT_OK) return st;
  for (size_t l = 0; l < mg->lv.size(); l++) {
    const pt_op *next = l + 1 < mg->lv.size() ? mg->lv[l + 1].op : nullptr;
    if ((st = mg_level_setup(s, *mg, mg->lv[l], next)) != PT_OK) return st;
  }
  // FP32 smoothing keeps the FP32 copies only
  if (mg->fp32)
    for (pt_mg_level &L : mg->lv)
      if (L.Ae64 && (void *)L.Ae64 != L.Ae) {
        cudaFree(L.Ae64);
        L.Ae64 = nullptr;
      }
  s->lambda_max = mg->lv[0].lmax;
  return PT_OK;
}

// Capture one V-cycle (level-0 b -> level-0 x) as a CUDA graph.  A first
// eager cycle sets every kernel attribute; the capture runs on a private
// stream (the levels' stream is swapped for the capture and put back).
template <typename T>
pt_status mg_capture(pt_solver *s)
{
  pt_mg &mg = *s->mg;
  pt_status st = mg_vcycle<T>(mg, 0);
  if (st != PT_OK) return st;
  PT_CUDA(cudaStreamSynchronize(s->op->stream));
  cudaStream_t cap;
  PT_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  std::vector<cudaStream_t> saved;
  for (pt_mg_level &L : mg.lv) {
    saved.push_back(L.op->stream);
    L.op->stream = cap;
  }
  const int64_t f0 = mg.fine_applies;
  const double c0 = mg.coarse_work;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = mg_vcycle<T>(mg, 0);
    e = cudaStreamEndCapture(cap, &g);
  }
  for (size_t i = 0; i < mg.lv.size(); i++) mg.lv[i].op->stream = saved[i];
  mg.graph_fine = mg.fine_applies - f0;
  mg.graph_coarse = mg.coarse_work - c0;
  mg.fine_applies = f0;
  mg.coarse_work = c0;
  if (e == cudaSuccess && st == PT_OK) e = cudaGraphInstantiate(&mg.gexec, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cap);
  if (st != PT_OK) return st;
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "V-cycle graph capture: %s", cudaGetErrorString(e));
  return PT_OK;
}

template <typename T>
pt_status mg_run(pt_solver *s)
{
  pt_mg &mg = *s->mg;
  if (!mg.use_graph) return mg_vcycle<T>(mg, 0);
  if (!mg.gexec) {
    pt_status st = mg_capture<T>(s);
    if (st != PT_OK) return st;
  }
  PT_CUDA(cudaGraphLaunch(mg.gexec, s->op->stream));
  mg.fine_applies += mg.graph_fine;
  mg.coarse_work += mg.graph_coarse;
  return PT_OK;
}

// Preconditioner set-up (PCSetUp): inverse diagonal, lambda_max or the level
// hierarchy; redone when the op's coordinates, viscosity or mask changed.
pt_status sv_setup(pt_solver *s)
{
  if (s->setup_done && s->op_state == s->op->state) return PT_OK;
  s->have_diag = false;
  s->lambda_max = 0.0;
  mg_free(s->mg);
  s->mg = nullptr;
  s->setup_done = false;
  pt_status st = PT_OK;
  if (s->o.pc != PT_PC_NONE && (st = sv_setup_diag(s)) != PT_OK) return st;
  if (s->o.pc == PT_PC_CHEBY_JACOBI && (st = sv_estimate_lambda(s)) != PT_OK) return st;
  if (s->o.pc == PT_PC_MG && (st = mg_build(s)) != PT_OK) {
    mg_free(s->mg);
    s->mg = nullptr;
    return st;
  }
  s->setup_done = true;
  s->op_state = s->op->state;
  return PT_OK;
}

pt_status sv_precond_mg(pt_solver *s, const double *r, double *z)
{
  pt_mg &mg = *s->mg;
  pt_mg_level &L0 = mg.lv[0];
  cudaStream_t st = s->op->stream;
  if (mg.fp32) {
    convert_kernel<float, double><<<vgrid(s->n), 256, 0, st>>>(r, (float *)L0.b, s->n);
    PT_LAUNCHED(s->op);
    pt_status stt = mg_run<float>(s);
    if (stt != PT_OK) return stt;
    convert_kernel<double, float><<<vgrid(s->n), 256, 0, st>>>((float *)L0.x, z, s->n);
    PT_LAUNCHED(s->op);
  } else {
    PT_CUDA(cudaMemcpyAsync(L0.b, r, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, st));
    pt_status stt = mg_run<double>(s);
    if (stt != PT_OK) return stt;
    PT_CUDA(cudaMemcpyAsync(z, L0.x, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, st));
  }
  return PT_OK;
}

// z = P r (P = the configured preconditioner), FP64 in/out.
pt_status sv_precond(pt_solver *s, const double *r, double *z)
{
  const pt_solve_opts &o = s->o;
  if (o.pc == PT_PC_NONE) {
    PT_CUDA(cudaMemcpyAsync(z, r, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, s->op->stream));
    return PT_OK;
  }
  if (o.pc == PT_PC_MG) return sv_precond_mg(s, r, z);
  if (o.pc == PT_PC_JACOBI) {
    cheb_first_kernel<double><<<vgrid(s->n), 256, 0, s->op->stream>>>(1.0, s->dinv, r, z, z, s->n);
    PT_LAUNCHED(s->op);
    return PT_OK;
  }
  // Chebyshev on D^-1 A over [emin, emax] (Saad, Iterative Methods, Alg. 12.1 with a diagonal preconditioner)
  const double emax = o.cheby_emax * s->lambda_max, emin = o.cheby_emin * s->lambda_max;
  const double theta = 0.5 * (emax + emin), delta = 0.5 * (emax - emin), sigma = theta / delta;
  double rho = 1.0 / sigma;
  pt_status st;
  if (o.cheby_fp32) {
    convert_kernel<float, double><<<vgrid(s->n), 256, 0, s->op->stream>>>(r, s->r32, s->n);
    PT_LAUNCHED(s->op);
    cheb_first_kernel<float><<<vgrid(s->n), 256, 0, s->op->stream>>>((float)(1.0 / theta), s->dinv32, s->r32, s->d32,
                                                                       s->z32, s->n);
    PT_LAUNCHED(s->op);
    for (int k = 1; k < o.cheby_degree; k++) {
      if ((st = sv_matmult32(s, s->z32, s->az32)) != PT_OK) return st;
      const double rho_new = 1.0 / (2.0 * sigma - rho);
      cheb_step_kernel<float><<<vgrid(s->n), 256, 0, s->op->stream>>>((float)(rho_new * rho), (float)(2.0 * rho_new / delta),
                                                                        s->dinv32, s->r32, s->az32, s->d32, s->z32, s->n);
      PT_LAUNCHED(s->op);
      rho = rho_new;
    }
    convert_kernel<double, float><<<vgrid(s->n), 256, 0, s->op->stream>>>(s->z32, z, s->n);
    PT_LAUNCHED(s->op);
    return PT_OK;
  }
  double *d = s->t3, *az = s->t2;
  cheb_first_kernel<double><<<vgrid(s->n), 256, 0, s->op->stream>>>(1.0 / theta, s->dinv, r, d, z, s->n);
  PT_LAUNCHED(s->op);
  for (int k = 1; k < o.cheby_degree; k++) {
    if ((st = sv_matmult64(s, z, az)) != PT_OK) return st;
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    cheb_step_kernel<double><<<vgrid(s->n), 256, 0, s->op->stream>>>(rho_new * rho, 2.0 * rho_new / delta, s->dinv, r,
                                                                       az, d, z, s->n);
    PT_LAUNCHED(s->op);
    rho = rho_new;
  }
  return PT_OK;
}

pt_status sv_fgmres(pt_solver *s, const double *b, double *x, pt_solve_stats *stats)
{
  const int m = s->o.restart;
  const int64_t n = s->n;
  std::vector<double> H((m + 1) * m), cs(m), sn(m), g(m + 1), h(m + 1), h2(m + 1), y(m);
  std::vector<const double *> Vp(m + 1), Zp(m);
  for (int j = 0; j <= m; j++) Vp[j] = s->V + (int64_t)j * n;
  for (int j = 0; j < m; j++) Zp[j] = s->Z + (int64_t)j * n;
  pt_status st;
  double beta;
  // r = b - A x
  if ((st = sv_matmult64(s, x, s->r)) != PT_OK) return st;
  resid_kernel<<<vgrid(n), 256, 0, s->op->stream>>>(b, s->r, n);
  PT_LAUNCHED(s->op);
  if ((st = sv_dot(s, s->r, s->r, &beta)) != PT_OK) return st;
  beta = std::sqrt(beta);
  stats->rnorm0 = beta;
  const double tol = std::max(s->o.rtol * beta, s->o.atol);
  int its = 0;
  while (beta > tol && its < s->o.max_it) {
    // v0 = r / beta
    axpby_kernel<double><<<vgrid(n), 256, 0, s->op->stream>>>(1.0 / beta, s->r, 0.0, s->V, n);
    PT_LAUNCHED(s->op);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && its < s->o.max_it; j++) {
      double *vj = s->V + (int64_t)j * n, *zj = s->Z + (int64_t)j * n, *vn = s->V + (int64_t)(j + 1) * n;
      if ((st = sv_precond(s, vj, zj)) != PT_OK) return st;
      if ((st = sv_matmult64(s, zj, vn)) != PT_OK) return st;
      // classical Gram-Schmidt, twice
      if ((st = sv_dots(s, Vp.data(), j + 1, vn, h.data())) != PT_OK) return st;
      if ((st = sv_maxpy(s, Vp.data(), h.data(), j + 1, vn, -1)) != PT_OK) return st;
      if ((st = sv_dots(s, Vp.data(), j + 1, vn, h2.data())) != PT_OK) return st;
      if ((st = sv_maxpy(s, Vp.data(), h2.data(), j + 1, vn, -1)) != PT_OK) return st;
      for (int i = 0; i <= j; i++) h[i] += h2[i];
      double hn;
      if ((st = sv_dot(s, vn, vn, &hn)) != PT_OK) return st;
      hn = std::sqrt(hn);
      if (hn > 0.0) {
        axpby_kernel<double><<<vgrid(n), 256, 0, s->op->stream>>>(1.0 / hn, vn, 0.0, vn, n);
        PT_LAUNCHED(s->op);
      }
      // Givens rotations on column j
      for (int i = 0; i < j; i++) {
        const double t = cs[i] * h[i] + sn[i] * h[i + 1];
        h[i + 1] = -sn[i] * h[i] + cs[i] * h[i + 1];
        h[i] = t;
      }
      const double den = std::hypot(h[j], hn);
      cs[j] = den > 0 ? h[j] / den : 1.0;
      sn[j] = den > 0 ? hn / den : 0.0;
      h[j] = den;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      for (int i = 0; i <= j; i++) H[i * m + j] = h[i];
      its++;
      if (std::fabs(g[j + 1]) <= tol || hn == 0.0) {
        j++;
        break;
      }
    }
    // y = H^-1 g, x += Z y
    for (int i = j - 1; i >= 0; i--) {
      double t = g[i];
      for (int k = i + 1; k < j; k++) t -= H[i * m + k] * y[k];
      y[i] = t / H[i * m + i];
    }
    if ((st = sv_maxpy(s, Zp.data(), y.data(), j, x, +1)) != PT_OK) return st;
    // true residual
    if ((st = sv_matmult64(s, x, s->r)) != PT_OK) return st;
    resid_kernel<<<vgrid(n), 256, 0, s->op->stream>>>(b, s->r, n);
    PT_LAUNCHED(s->op);
    if ((st = sv_dot(s, s->r, s->r, &beta)) != PT_OK) return st;
    beta = std::sqrt(beta);
  }
  stats->its = its;
  stats->rnorm = beta;
  stats->converged = beta <= tol;
  return PT_OK;
}

// Flexible CG (Polak-Ribiere beta), tolerant of the inexact FP32 inner solve.
pt_status sv_fcg(pt_solver *s, const double *b, double *x, pt_solve_stats *stats)
{
  const int64_t n = s->n;
  double *p = s->V, *q = s->V + n, *z = s->V + 2 * n, *rold = s->V + 3 * n;
  pt_status st;
  if ((st = sv_matmult64(s, x, s->r)) != PT_OK) return st;
  resid_kernel<<<vgrid(n), 256, 0, s->op->stream>>>(b, s->r, n);
  PT_LAUNCHED(s->op);
  double rr;
  if ((st = sv_dot(s, s->r, s->r, &rr)) != PT_OK) return st;
  double rnorm = std::sqrt(rr);
  stats->rnorm0 = rnorm;
  const double tol = std::max(s->o.rtol * rnorm, s->o.atol);
  if ((st = sv_precond(s, s->r, z)) != PT_OK) return st;
  PT_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->op->stream));
  double rz;
  if ((st = sv_dot(s, s->r, z, &rz)) != PT_OK) return st;
  int its = 0;
  while (rnorm > tol && its < s->o.max_it) {
    if ((st = sv_matmult64(s, p, q)) != PT_OK) return st;
    double pq;
    if ((st = sv_dot(s, p, q, &pq)) != PT_OK) return st;
    if (!(pq > 0.0)) break;
    const double alpha = rz / pq;
    if ((st = sv_axpby<double>(s, alpha, p, 1.0, x)) != PT_OK) return st;
    PT_CUDA(cudaMemcpyAsync(rold, s->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->op->stream));
    if ((st = sv_axpby<double>(s, -alpha, q, 1.0, s->r)) != PT_OK) return st;
    if ((st = sv_dot(s, s->r, s->r, &rr)) != PT_OK) return st;
    rnorm = std::sqrt(rr);
    its++;
    if (rnorm <= tol) break;
    if ((st = sv_precond(s, s->r, z)) != PT_OK) return st;
    // beta = z.(r - rold) / rz
    const double *zz[2] = {s->r, rold};
    double d2[2];
    if ((st = sv_dots(s, zz, 2, z, d2)) != PT_OK) return st;
    const double beta = (d2[0] - d2[1]) / rz;
    rz = d2[0];
    if ((st = sv_axpby<double>(s, 1.0, z, beta, p)) != PT_OK) return st;
  }
  // report the true residual
  if ((st = sv_matmult64(s, x, s->r)) != PT_OK) return st;
  resid_kernel<<<vgrid(n), 256, 0, s->op->stream>>>(b, s->r, n);
  PT_LAUNCHED(s->op);
  if ((st = sv_dot(s, s->r, s->r, &rr)) != PT_OK) return st;
  stats->its = its;
  stats->rnorm = std::sqrt(rr);
  stats->converged = stats->rnorm <= tol * (1.0 + 1e-6);
  return PT_OK;
}

}  // namespace

extern "C" {

void pt_solve_opts_default(pt_solve_opts *o)
{
  if (!o) return;
  o->ksp = PT_KSP_FGMRES;
  o->restart = 30;
  o->max_it = 10000;
  o->rtol = 1e-8;
  o->atol = 0.0;
  o->pc = PT_PC_CHEBY_JACOBI;
  o->cheby_degree = 3;
  o->cheby_fp32 = 1;
  o->cheby_emin = 0.2;
  o->cheby_emax = 1.1;
  o->eig_its = 20;
  o->mg_levels = 0;
  o->mg_coarse_degree = 24;
  o->pc_graph = 1;
  o->mg_assembled = 2;
  o->mg_fine_degree = 0;
  o->mg_coarse_half = 1;
}

pt_status pt_solver_create(pt_op *op, const pt_solve_opts *opts, pt_solver **out)
{
  if (!op || !opts || !out) return fail(PT_ERR_BAD_ARG, "NULL argument");
  *out = nullptr;
  if (opts->ksp != PT_KSP_FGMRES && opts->ksp != PT_KSP_FCG) return fail(PT_ERR_BAD_ARG, "unknown ksp %d", opts->ksp);
  if (opts->pc < PT_PC_NONE || opts->pc > PT_PC_MG) return fail(PT_ERR_BAD_ARG, "unknown pc %d", opts->pc);
  if (opts->restart < 1 || opts->restart > 256) return fail(PT_ERR_BAD_ARG, "restart must be in [1, 256]");
  if (opts->cheby_degree < 1 || opts->cheby_degree > 64) return fail(PT_ERR_BAD_ARG, "cheby_degree must be in [1, 64]");
  if (opts->mg_fine_degree < 0 || opts->mg_fine_degree > 64)
    return fail(PT_ERR_BAD_ARG, "mg_fine_degree must be in [0, 64]");
  if (opts->mg_coarse_half != 0 && opts->mg_coarse_half != 1)
    return fail(PT_ERR_BAD_ARG, "mg_coarse_half must be 0 or 1");
  if (!(opts->cheby_emin > 0.0) || !(opts->cheby_emax > opts->cheby_emin))
    return fail(PT_ERR_BAD_ARG, "need 0 < cheby_emin < cheby_emax");
  pt_status st = check_ready(op, true);
  if (st != PT_OK) return st;
  pt_solver *s = new (std::nothrow) pt_solver();
  if (!s) return fail(PT_ERR_OOM, "host allocation failed");
  s->op = op;
  s->o = *opts;
  s->n = op->nvel;
  const int64_t n = s->n;
  const int nb = opts->ksp == PT_KSP_FGMRES ? 2 * opts->restart + 1 : 4;
  cudaError_t e = cudaSuccess;
  double **f64[] = {&s->r, &s->w, &s->x0, &s->dinv, &s->t1, &s->t2, &s->t3};
  for (double **p : f64)
    if (e == cudaSuccess) e = cudaMalloc(p, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->V, sizeof(double) * n * nb);
  if (e == cudaSuccess) s->Z = s->V + (int64_t)(opts->restart + 1) * n;
  float **f32[] = {&s->dinv32, &s->r32, &s->z32, &s->d32, &s->az32};
  for (float **p : f32)
    if (e == cudaSuccess) e = cudaMalloc(p, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->partial, sizeof(double) * RED_BLOCKS * MDOT_CHUNK);
  if (e == cudaSuccess) e = cudaMalloc(&s->dres, sizeof(double) * 512);
  if (e == cudaSuccess) e = cudaMalloc(&s->hbuf, sizeof(double) * 512);
  if (e == cudaSuccess) e = cudaMalloc((void **)&s->dptr, sizeof(double *) * 128);
  if (e == cudaSuccess) e = cudaMallocHost(&s->hhost, sizeof(double) * 512);
  if (e != cudaSuccess) {
    pt_status r = fail(e == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_CUDA, "pt_solver_create: %s",
                       cudaGetErrorString(e));
    pt_solver_destroy(s);
    return r;
  }
  *out = s;
  return PT_OK;
}

pt_status pt_solver_apply_pc_d(pt_solver *s, const double *r, double *z)
{
  if (!s || !r || !z) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (r == z) return fail(PT_ERR_BAD_ARG, "r and z must not alias");
  pt_status st = sv_setup(s);
  if (st != PT_OK) return st;
  return sv_precond(s, r, z);
}

pt_status pt_solver_destroy(pt_solver *s)
{
  if (!s) return PT_OK;
  if (s->op && s->op->stream) cudaStreamSynchronize(s->op->stream);
  void *ptrs[] = {s->r, s->w, s->x0, s->dinv, s->t1, s->t2, s->t3, s->V, s->dinv32, s->r32, s->z32, s->d32,
                  s->az32, s->partial, s->dres, s->hbuf, (void *)s->dptr};
  for (void *p : ptrs) cudaFree(p);
  if (s->hhost) cudaFreeHost(s->hhost);
  mg_free(s->mg);
  delete s;
  return PT_OK;
}

pt_status pt_solver_solve_d(pt_solver *s, const double *b, double *x, pt_solve_stats *stats)
{
  if (!s || !b || !x || !stats) return fail(PT_ERR_BAD_ARG, "NULL argument");
  memset(stats, 0, sizeof *stats);
  const auto t0 = std::chrono::steady_clock::now();
  s->n64 = s->n32 = 0;
  if (s->mg) {
    s->mg->fine_applies = 0;
    s->mg->coarse_work = 0.0;
  }
  pt_status st = sv_setup(s);
  if (st != PT_OK) return st;
  stats->lambda_max = s->lambda_max;
  if (s->o.ksp == PT_KSP_FGMRES) st = sv_fgmres(s, b, x, stats);
  else st = sv_fcg(s, b, x, stats);
  if (st != PT_OK) return st;
  PT_CUDA(cudaStreamSynchronize(s->op->stream));
  stats->a11_f64 = s->n64;
  stats->a11_f32 = s->n32;
  if (s->mg) {
    (s->mg->fp32 ? stats->a11_f32 : stats->a11_f64) += s->mg->fine_applies;
    stats->a11_coarse = s->mg->coarse_work;
    stats->mg_levels = (int32_t)s->mg->lv.size();
  }
  stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return PT_OK;
}

}  // extern "C"
