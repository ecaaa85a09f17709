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

// Largest eigenvalue of a symmetric tridiagonal matrix (bisection on Sturm counts).
double tridiag_lambda_max(const std::vector<double> &a, const std::vector<double> &b)
{
  const int n = (int)a.size();
  if (n == 0) return 0.0;
  double lo = a[0], hi = a[0];
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto count_below = [&](double x) {
    int c = 0;
    double q = a[0] - x;
    if (q < 0) c++;
    for (int i = 1; i < n; i++) {
      const double qq = (q == 0.0) ? 1e-300 : q;
      q = a[i] - x - b[i - 1] * b[i - 1] / qq;
      if (q < 0) c++;
    }
    return c;
  };
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= n) hi = mid;
    else lo = mid;
  }
  return hi;
}

}  // namespace

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
};

namespace {

pt_status sv_dots(pt_solver *s, const double *const *vecs_host, int nv, const double *w, double *out)
{
  // vector-pointer table goes through a small device array
  for (int base = 0; base < nv; base += MDOT_CHUNK) {
    const int k = std::min(MDOT_CHUNK, nv - base);
    PT_CUDA(cudaMemcpyAsync(s->dptr, vecs_host + base, sizeof(double *) * k, cudaMemcpyHostToDevice, s->op->stream));
    mdot_partial_kernel<<<RED_BLOCKS, RED_THREADS, 0, s->op->stream>>>(s->dptr, k, w, s->n, s->partial);
    PT_LAUNCHED(s->op);
    mdot_final_kernel<<<1, RED_THREADS, 0, s->op->stream>>>(s->partial, k, s->dres + base);
    PT_LAUNCHED(s->op);
  }
  PT_CUDA(cudaMemcpyAsync(s->hhost, s->dres, sizeof(double) * nv, cudaMemcpyDeviceToHost, s->op->stream));
  PT_CUDA(cudaStreamSynchronize(s->op->stream));
  for (int j = 0; j < nv; j++) out[j] = s->hhost[j];
  return PT_OK;
}

pt_status sv_dot(pt_solver *s, const double *a, const double *b, double *out)
{
  const double *v[1] = {a};
  return sv_dots(s, v, 1, b, out);
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
pt_status sv_axpby(pt_solver *s, T a, const T *x, T b, T *y)
{
  axpby_kernel<T><<<vgrid(s->n), 256, 0, s->op->stream>>>(a, x, b, y, s->n);
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

// lambda_max(D^-1 A) from eig_its steps of Jacobi-PCG on a pseudo-random rhs (Lanczos tridiagonal).
pt_status sv_estimate_lambda(pt_solver *s)
{
  double *b = s->t2, *x = s->x0, *p = s->t3, *q = s->w, *r = s->r, *z = s->t1;
  hash_vec_kernel<<<vgrid(s->n), 256, 0, s->op->stream>>>(b, s->n, 12345u);
  PT_LAUNCHED(s->op);
  PT_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, s->op->stream));
  PT_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * s->n, s->op->stream));
  cheb_first_kernel<double><<<vgrid(s->n), 256, 0, s->op->stream>>>(1.0, s->dinv, r, z, p, s->n);  // z = p = D^-1 r
  PT_LAUNCHED(s->op);
  double rz;
  pt_status st = sv_dot(s, r, z, &rz);
  if (st != PT_OK) return st;
  std::vector<double> alphas, betas, diag, off;
  for (int k = 0; k < s->o.eig_its && rz > 0.0; k++) {
    if ((st = sv_matmult64(s, p, q)) != PT_OK) return st;
    double pq;
    if ((st = sv_dot(s, p, q, &pq)) != PT_OK) return st;
    if (!(pq > 0.0)) break;
    const double alpha = rz / pq;
    if ((st = sv_axpby<double>(s, -alpha, q, 1.0, r)) != PT_OK) return st;
    cheb_first_kernel<double><<<vgrid(s->n), 256, 0, s->op->stream>>>(1.0, s->dinv, r, z, z, s->n);
    PT_LAUNCHED(s->op);
    double rz_new;
    if ((st = sv_dot(s, r, z, &rz_new)) != PT_OK) return st;
    const double beta = rz_new / rz;
    if ((st = sv_axpby<double>(s, 1.0, z, beta, p)) != PT_OK) return st;
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
  s->lambda_max = tridiag_lambda_max(diag, off);
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
}

pt_status pt_solver_create(pt_op *op, const pt_solve_opts *opts, pt_solver **out)
{
  if (!op || !opts || !out) return fail(PT_ERR_BAD_ARG, "NULL argument");
  *out = nullptr;
  if (opts->ksp != PT_KSP_FGMRES && opts->ksp != PT_KSP_FCG) return fail(PT_ERR_BAD_ARG, "unknown ksp %d", opts->ksp);
  if (opts->pc < PT_PC_NONE || opts->pc > PT_PC_CHEBY_JACOBI) return fail(PT_ERR_BAD_ARG, "unknown pc %d", opts->pc);
  if (opts->restart < 1 || opts->restart > 256) return fail(PT_ERR_BAD_ARG, "restart must be in [1, 256]");
  if (opts->cheby_degree < 1 || opts->cheby_degree > 64) return fail(PT_ERR_BAD_ARG, "cheby_degree must be in [1, 64]");
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

pt_status pt_solver_destroy(pt_solver *s)
{
  if (!s) return PT_OK;
  if (s->op && s->op->stream) cudaStreamSynchronize(s->op->stream);
  void *ptrs[] = {s->r, s->w, s->x0, s->dinv, s->t1, s->t2, s->t3, s->V, s->dinv32, s->r32, s->z32, s->d32,
                  s->az32, s->partial, s->dres, s->hbuf, (void *)s->dptr};
  for (void *p : ptrs) cudaFree(p);
  if (s->hhost) cudaFreeHost(s->hhost);
  delete s;
  return PT_OK;
}

pt_status pt_solver_solve_d(pt_solver *s, const double *b, double *x, pt_solve_stats *stats)
{
  if (!s || !b || !x || !stats) return fail(PT_ERR_BAD_ARG, "NULL argument");
  memset(stats, 0, sizeof *stats);
  const auto t0 = std::chrono::steady_clock::now();
  s->n64 = s->n32 = 0;
  pt_status st;
  if (s->o.pc != PT_PC_NONE) {
    if ((st = sv_setup_diag(s)) != PT_OK) return st;
  }
  if (s->o.pc == PT_PC_CHEBY_JACOBI && !(s->lambda_max > 0.0)) {
    if ((st = sv_estimate_lambda(s)) != PT_OK) return st;
  }
  stats->lambda_max = s->lambda_max;
  if (s->o.ksp == PT_KSP_FGMRES) st = sv_fgmres(s, b, x, stats);
  else st = sv_fcg(s, b, x, stats);
  if (st != PT_OK) return st;
  PT_CUDA(cudaStreamSynchronize(s->op->stream));
  stats->a11_f64 = s->n64;
  stats->a11_f32 = s->n32;
  stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return PT_OK;
}

}  // extern "C"
