// Serving form: a request loop of viscous solves A11 u = f on independent
// one-rank boxes, continuously batched.
//
// Each admitted request keeps its coordinates, Gauss-point viscosity, K
// factors, Dirichlet mask and Krylov state resident on the device, in
// stream-ordered allocations from the server's memory pool.  Admission only
// enqueues work: uploads, geometry, diagonal, a device-side Lanczos estimate
// of lambda_max(D^-1 A) and the first preconditioned residual run on a
// set-up stream while the batch iterates on the main stream; a request joins
// the batch once its set-up event has completed.  All
// active requests advance together, one preconditioned flexible-CG iteration
// at a time: the A11 applies of every request go through one batched
// work-list (one launch per colour / tile-width class, batch_impl.cuh) and
// the vector updates and dot products through chunk-list kernels over all
// requests, so an iteration costs the same ~20 launches whatever the number
// of requests.  Requests join between iterations as slots and memory free up
// (admission against a byte budget; their set-up runs on a second stream
// while the batch iterates) and leave when converged.
//
// Per request the arithmetic is independent of the batch: the batched apply
// sums every node in the request's own colour order (bitwise its single-op
// result), dot products reduce the request's own fixed chunks in a fixed
// order, and scalars live per request.  A result is therefore bitwise the
// same alone and in any mix.
//
// Iteration (Polak-Ribiere flexible CG, M = Chebyshev(deg)-Jacobi on D^-1 A
// over [emin, emax] * lambda_max, in FP32 or FP64):
//   q = A p;  alpha = rz / (p.q);  x += alpha p;  r -= alpha q;  stop if
//   r.r <= max(rtol^2 r0.r0, atol^2);  z = M r;
//   beta = -alpha (z.q) / rz;  rz = z.r;  p = z + beta p.
// (z.(r_new - r_old) = -alpha z.q, so r_old is not stored.)
// Included from pt_b200.cu after the solver and the batched apply.
#pragma once

#include <chrono>
#include <deque>
#include <vector>

namespace {

constexpr int SRV_CH = 2048;        // dofs per chunk
constexpr int SRV_THREADS = 256;
constexpr int SRV_MAX_DEG = 16;

struct SrvSlot {
  int64_t n;
  double *x, *r, *p, *q;
  void *z, *d, *az;          // smoother precision
  const void *dinv;          // smoother precision
  int64_t nch;
  double *part;              // 2 * nch partial sums
};

struct SrvScal {
  double rz, alpha, beta, rr, rr0, tol2;
  double rtol2, atol2;
  double theta_inv, lmax;
  double ca[SRV_MAX_DEG], cb[SRV_MAX_DEG];
  int32_t its, status, max_it, deg;
};

enum { SRV_ACTIVE = 0, SRV_CONVERGED = 1, SRV_MAXIT = 2, SRV_BREAKDOWN = 3 };

template <typename T>
__device__ __forceinline__ double srv_block_sum(double v, double *sh)
{
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = SRV_THREADS / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// chunk c of slot s: [c*CH, min(n, (c+1)*CH))
__device__ __forceinline__ void srv_chunk(const SrvSlot &S, int c, int64_t &i0, int64_t &i1)
{
  i0 = (int64_t)c * SRV_CH;
  i1 = i0 + SRV_CH < S.n ? i0 + SRV_CH : S.n;
}

// partial[c][0] = p.q over the chunk
__global__ void __launch_bounds__(SRV_THREADS) srv_pq_kernel(const int2 *__restrict__ items, const SrvSlot *slots,
                                                             const SrvScal *scal)
{
  __shared__ double sh[SRV_THREADS];
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  if (scal[it.x].status != SRV_ACTIVE) return;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  double a = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) a = fma(S.p[i], S.q[i], a);
  a = srv_block_sum<double>(a, sh);
  if (threadIdx.x == 0) S.part[2 * it.y] = a;
}

// x += alpha p; r -= alpha q; partial[c][0] = r.r
__global__ void __launch_bounds__(SRV_THREADS) srv_update_kernel(const int2 *__restrict__ items, const SrvSlot *slots,
                                                                 const SrvScal *scal)
{
  __shared__ double sh[SRV_THREADS];
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  if (scal[it.x].status != SRV_ACTIVE) return;
  const double alpha = scal[it.x].alpha;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  double a = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    S.x[i] = fma(alpha, S.p[i], S.x[i]);
    const double r = fma(-alpha, S.q[i], S.r[i]);
    S.r[i] = r;
    a = fma(r, r, a);
  }
  a = srv_block_sum<double>(a, sh);
  if (threadIdx.x == 0) S.part[2 * it.y] = a;
}

// z = d = theta^-1 D^-1 r  (smoother precision)
template <typename T>
__global__ void __launch_bounds__(SRV_THREADS) srv_cheb_first_kernel(const int2 *__restrict__ items,
                                                                     const SrvSlot *slots, const SrvScal *scal)
{
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  if (scal[it.x].status != SRV_ACTIVE) return;
  const T s = (T)scal[it.x].theta_inv;
  const T *dinv = (const T *)S.dinv;
  T *z = (T *)S.z, *d = (T *)S.d;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    const T v = s * dinv[i] * (T)S.r[i];
    d[i] = v;
    z[i] = v;
  }
}

// step k: d = ca[k] d + cb[k] D^-1 (r - A z); z += d
template <typename T>
__global__ void __launch_bounds__(SRV_THREADS) srv_cheb_step_kernel(const int2 *__restrict__ items,
                                                                    const SrvSlot *slots, const SrvScal *scal, int k)
{
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  const SrvScal &P = scal[it.x];
  if (P.status != SRV_ACTIVE || k >= P.deg) return;
  const T ca = (T)P.ca[k], cb = (T)P.cb[k];
  const T *dinv = (const T *)S.dinv, *az = (const T *)S.az;
  T *z = (T *)S.z, *d = (T *)S.d;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    const T v = ca * d[i] + cb * dinv[i] * ((T)S.r[i] - az[i]);
    d[i] = v;
    z[i] += v;
  }
}

// partial[c] = (z.r, z.q)
template <typename T>
__global__ void __launch_bounds__(SRV_THREADS) srv_zdots_kernel(const int2 *__restrict__ items, const SrvSlot *slots,
                                                                const SrvScal *scal)
{
  __shared__ double sh[SRV_THREADS];
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  if (scal[it.x].status != SRV_ACTIVE) return;
  const T *z = (const T *)S.z;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  double a = 0.0, b = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    const double zi = (double)z[i];
    a = fma(zi, S.r[i], a);
    b = fma(zi, S.q[i], b);
  }
  a = srv_block_sum<double>(a, sh);
  b = srv_block_sum<double>(b, sh);
  if (threadIdx.x == 0) {
    S.part[2 * it.y] = a;
    S.part[2 * it.y + 1] = b;
  }
}

// p = z + beta p
template <typename T>
__global__ void __launch_bounds__(SRV_THREADS) srv_p_kernel(const int2 *__restrict__ items, const SrvSlot *slots,
                                                            const SrvScal *scal)
{
  const int2 it = items[blockIdx.x];
  const SrvSlot S = slots[it.x];
  if (scal[it.x].status != SRV_ACTIVE) return;
  const double beta = scal[it.x].beta;
  const T *z = (const T *)S.z;
  int64_t i0, i1;
  srv_chunk(S, it.y, i0, i1);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) S.p[i] = fma(beta, S.p[i], (double)z[i]);
}

enum { SRV_F_ALPHA = 0, SRV_F_RR = 1, SRV_F_BETA = 2, SRV_F_INIT_RR = 3, SRV_F_INIT_RZ = 4 };

// Per slot (block): reduce the slot's chunk partials in a fixed order, then
// the scalar recurrences.
template <int PHASE>
__global__ void __launch_bounds__(SRV_THREADS) srv_final_kernel(const int *__restrict__ act, const SrvSlot *slots,
                                                                SrvScal *scal)
{
  __shared__ double sh[SRV_THREADS];
  const int s = act[blockIdx.x];
  const SrvSlot S = slots[s];
  SrvScal &P = scal[s];
  if (PHASE != SRV_F_INIT_RR && P.status != SRV_ACTIVE) return;
  double a = 0.0, b = 0.0;
  for (int64_t c = threadIdx.x; c < S.nch; c += SRV_THREADS) {
    a += S.part[2 * c];
    if (PHASE == SRV_F_BETA) b += S.part[2 * c + 1];
  }
  a = srv_block_sum<double>(a, sh);
  if (PHASE == SRV_F_BETA) b = srv_block_sum<double>(b, sh);
  if (threadIdx.x != 0) return;
  if (PHASE == SRV_F_ALPHA) {
    if (a > 0.0 && isfinite(a)) P.alpha = P.rz / a;
    else { P.alpha = 0.0; P.status = SRV_BREAKDOWN; }
  } else if (PHASE == SRV_F_RR) {
    P.rr = a;
    P.its++;
    if (a <= P.tol2) P.status = SRV_CONVERGED;
    else if (!isfinite(a)) P.status = SRV_BREAKDOWN;
    else if (P.its >= P.max_it) P.status = SRV_MAXIT;
  } else if (PHASE == SRV_F_BETA) {
    P.beta = -P.alpha * b / P.rz;
    P.rz = a;
    if (!(a > 0.0) || !isfinite(P.beta)) P.status = SRV_BREAKDOWN;
  } else if (PHASE == SRV_F_INIT_RR) {
    P.rr0 = P.rr = a;
    P.tol2 = fmax(P.rtol2 * a, P.atol2);
    P.its = 0;
    P.beta = 0.0;
    P.status = (a <= P.tol2) ? SRV_CONVERGED : SRV_ACTIVE;
  } else {  // SRV_F_INIT_RZ
    P.rz = a;
    if (!(a > 0.0)) P.status = SRV_BREAKDOWN;
  }
}

// dinv = 1 / diag in the smoother's precision
template <typename T>
__global__ void convert_inv_kernel(const double *__restrict__ d, T *__restrict__ dinv, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dinv[i] = (T)(1.0 / d[i]);
}

// ---- device-side Lanczos estimate of lambda_max(D^-1 A) at admission --------
// Jacobi-preconditioned CG from a pseudo-random vector, eig_its steps, its
// coefficients kept on the device; the tridiagonal's largest eigenvalue and
// the Chebyshev coefficients are formed by one thread.  The same recurrence
// as the single-op solver's estimate (sv_lanczos), without host reads.
constexpr int SRV_MAX_LZ = 64;

struct LzState {
  double rz;
  double alpha[SRV_MAX_LZ], beta[SRV_MAX_LZ];
  int m, stop;
};

// r = hash(i); z = r / diag; p = z; part[c] = r.z
__global__ void __launch_bounds__(SRV_THREADS) lz_start_kernel(int64_t n, const double *__restrict__ diag,
                                                               double *__restrict__ r, double *__restrict__ z,
                                                               double *__restrict__ p, double *__restrict__ part)
{
  __shared__ double sh[SRV_THREADS];
  const int64_t i0 = (int64_t)blockIdx.x * SRV_CH, i1 = min(n, i0 + SRV_CH);
  double a = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    uint64_t h = (uint64_t)i + 12345ull * 0x9E3779B97F4A7C15ull;
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
    h ^= h >> 31;
    const double v = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    const double w = v / diag[i];
    r[i] = v;
    z[i] = w;
    p[i] = w;
    a = fma(v, w, a);
  }
  a = srv_block_sum<double>(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// part[c] = a.b
__global__ void __launch_bounds__(SRV_THREADS) lz_dot_kernel(int64_t n, const double *__restrict__ a,
                                                             const double *__restrict__ b, double *__restrict__ part)
{
  __shared__ double sh[SRV_THREADS];
  const int64_t i0 = (int64_t)blockIdx.x * SRV_CH, i1 = min(n, i0 + SRV_CH);
  double acc = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) acc = fma(a[i], b[i], acc);
  acc = srv_block_sum<double>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// r -= alpha_k q; z = r / diag; part[c] = r.z
__global__ void __launch_bounds__(SRV_THREADS) lz_update_kernel(int64_t n, const LzState *L, int k,
                                                                const double *__restrict__ q,
                                                                const double *__restrict__ diag,
                                                                double *__restrict__ r, double *__restrict__ z,
                                                                double *__restrict__ part)
{
  __shared__ double sh[SRV_THREADS];
  if (L->stop) return;
  const double alpha = L->alpha[k];
  const int64_t i0 = (int64_t)blockIdx.x * SRV_CH, i1 = min(n, i0 + SRV_CH);
  double a = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) {
    const double rv = fma(-alpha, q[i], r[i]);
    const double zv = rv / diag[i];
    r[i] = rv;
    z[i] = zv;
    a = fma(rv, zv, a);
  }
  a = srv_block_sum<double>(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// p = z + beta_k p
__global__ void __launch_bounds__(SRV_THREADS) lz_p_kernel(int64_t n, const LzState *L, int k,
                                                           const double *__restrict__ z, double *__restrict__ p)
{
  if (L->stop) return;
  const double beta = L->beta[k];
  const int64_t i0 = (int64_t)blockIdx.x * SRV_CH, i1 = min(n, i0 + SRV_CH);
  for (int64_t i = i0 + threadIdx.x; i < i1; i += SRV_THREADS) p[i] = fma(beta, p[i], z[i]);
}

// Sum the chunk partials (fixed order); MODE 0: rz0, 1: p.q -> alpha_k,
// 2: r.z -> beta_k, rz.
template <int MODE>
__global__ void __launch_bounds__(SRV_THREADS) lz_sum_kernel(int64_t nch, const double *__restrict__ part, LzState *L,
                                                             int k)
{
  __shared__ double sh[SRV_THREADS];
  double a = 0.0;
  for (int64_t c = threadIdx.x; c < nch; c += SRV_THREADS) a += part[c];
  a = srv_block_sum<double>(a, sh);
  if (threadIdx.x != 0) return;
  if (MODE == 0) {
    L->rz = a;
    L->m = 0;
    L->stop = !(a > 0.0);
    return;
  }
  if (L->stop) return;
  if (MODE == 1) {
    if (!(a > 0.0)) L->stop = 1;
    else L->alpha[k] = L->rz / a;
  } else {
    L->beta[k] = a / L->rz;
    L->rz = a;
    L->m = k + 1;
    if (!(a > 0.0)) L->stop = 1;
  }
}

// lambda_max from the Lanczos tridiagonal, then the Chebyshev coefficients
// (Saad, Alg. 12.1) of degree deg on [emin, emax] * lambda_max.
__global__ void lz_finish_kernel(const LzState *L, double emin, double emax, int deg, SrvScal *P)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int m = L->m;
  double a[SRV_MAX_LZ], b[SRV_MAX_LZ];
  for (int k = 0; k < m; k++) {
    a[k] = 1.0 / L->alpha[k] + (k > 0 ? L->beta[k - 1] / L->alpha[k - 1] : 0.0);
    if (k + 1 < m) b[k] = sqrt(L->beta[k]) / L->alpha[k];
  }
  const double lmax = tridiag_lmax(a, b, m);
  P->lmax = lmax;
  if (!(lmax > 0.0)) {
    P->status = SRV_BREAKDOWN;
    return;
  }
  const double hi = emax * lmax, lo = emin * lmax;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  P->theta_inv = 1.0 / theta;
  double rho = 1.0 / sigma;
  for (int k = 1; k < deg; k++) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    P->ca[k] = rn * rho;
    P->cb[k] = 2.0 * rn / delta;
    rho = rn;
  }
  P->deg = deg;
}

}  // namespace

struct SrvReq {
  int64_t id;
  pt_mesh_desc desc;
  const double *h_coords, *h_eta, *h_f;
  const uint8_t *h_mask;
  double *h_x;
  pt_op *op = nullptr;
  int slot = -1;
  int64_t n = 0, nch = 0;
  size_t bytes = 0;
  double *vec = nullptr;     // x, r, p, q (FP64), partials
  void *svec = nullptr;      // z, d, az, dinv (smoother precision)
  double *tmp = nullptr;     // set-up scratch: diagonal (FP64), Lanczos state, partials
  cudaEvent_t ready = nullptr;
  bool joined = false;
  SrvSlot S{};               // host copies of the slot's descriptor and initial scalars
  SrvScal P{};
  double t_submit = 0.0, t_admit = 0.0, t_done = 0.0;
  SrvScal fin{};             // scalars at retirement
};

struct pt_server {
  pt_server_opts o;
  bool fp32;
  cudaStream_t main = nullptr, setup = nullptr;
  cudaMemPool_t pool = nullptr;
  std::deque<SrvReq *> queue;
  std::vector<SrvReq *> slots;
  std::deque<SrvReq *> done;
  SrvSlot *d_slots = nullptr;
  SrvScal *d_scal = nullptr, *h_scal = nullptr;
  unsigned int *h_bad = nullptr;  // pinned, per slot: geometry check of the set-up
  int64_t bytes_in_use = 0;
  bool dirty = true;
  // current batch
  pt_batch *batch = nullptr;
  std::vector<int> act;
  int *d_act = nullptr;
  int2 *d_items = nullptr;
  int64_t nitems = 0;
  void *d_ptrs = nullptr;     // p[], q[], z[], az[] tables of the batch
  std::vector<int> h_act;     // host copies of the uploaded tables (kept until the next rebuild)
  std::vector<int2> h_items;
  std::vector<void *> h_ptrs;
  int64_t iterations = 0, launches = 0;
  double t_enqueue = 0.0, t_admit = 0.0, t_wait = 0.0, t_retire = 0.0;  // host seconds per phase
  std::chrono::steady_clock::time_point t0;
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

size_t srv_bytes(const pt_mesh_desc &d, bool fp32)
{
  // op: coords (f64+f32), eta (f64+f32), mask, K (f64+f32, rows padded to 32);
  // request: x r p q, z d az dinv, partials; set-up scratch (diagonal + Lanczos)
  const int64_t nx = 2 * (int64_t)d.mx + 1, ny = 2 * (int64_t)d.my + 1, nz = 2 * (int64_t)d.mz + 1;
  const int64_t nvel = 3 * nx * ny * nz, nel = (int64_t)d.mx * d.my * d.mz;
  const int64_t tx = d.mx <= 32 ? 32 : (d.mx <= 64 ? 64 : 128);
  const int64_t mxp = (d.mx + tx - 1) / tx * tx;
  const size_t ts = fp32 ? 4 : 8;
  const int64_t nch = (nvel + SRV_CH - 1) / SRV_CH;
  const size_t op = nvel * 12 + 27 * nel * 12 + nvel + (size_t)d.my * d.mz * 243 * mxp * 12;
  const size_t req = nvel * 32 + nvel * 4 * ts + 2 * 8 * nch;
  const size_t setup = nvel * 8 + sizeof(LzState) + 8 * nch;
  return op + req + setup;
}

void srv_release(pt_server *s, SrvReq *r)
{
  // stream-ordered frees on the main stream: after the last batched use
  if (r->op) {
    r->op->stream = s->main;
    pt_op_destroy(r->op);
  }
  if (r->vec) cudaFreeAsync(r->vec, s->main);
  if (r->svec) cudaFreeAsync(r->svec, s->main);
  if (r->tmp) cudaFreeAsync(r->tmp, s->main);
  if (r->ready) cudaEventDestroy(r->ready);
  r->op = nullptr;
  r->vec = nullptr;
  r->svec = nullptr;
  r->tmp = nullptr;
  r->ready = nullptr;
  s->bytes_in_use -= (int64_t)r->bytes;
}

std::vector<int2> srv_items(const std::vector<int> &slots_in, const std::vector<SrvReq *> &slots)
{
  std::vector<int2> it;
  for (int s : slots_in)
    for (int64_t c = 0; c < slots[s]->nch; c++) it.push_back(make_int2(s, (int)c));
  return it;
}

template <typename T>
pt_status srv_apply_single(pt_op *op, const T *u, T *y);
template <>
pt_status srv_apply_single<float>(pt_op *op, const float *u, float *y) { return pt_matmult_a11_f32_d(op, u, y); }
template <>
pt_status srv_apply_single<double>(pt_op *op, const double *u, double *y) { return pt_matmult_a11_d(op, u, y); }

// z = M r for the slots in `items` (one request at admission, or the batch):
// the smoother's applies go through `apply()`.
template <typename T, typename F>
pt_status srv_precond(pt_server *s, const int2 *items, int64_t nitems, cudaStream_t st, F apply)
{
  srv_cheb_first_kernel<T><<<(unsigned)nitems, SRV_THREADS, 0, st>>>(items, s->d_slots, s->d_scal);
  s->launches++;
  for (int k = 1; k < s->o.cheby_degree; k++) {
    pt_status e = apply();
    if (e != PT_OK) return e;
    srv_cheb_step_kernel<T><<<(unsigned)nitems, SRV_THREADS, 0, st>>>(items, s->d_slots, s->d_scal, k);
    s->launches++;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "server smoother launch: %s", cudaGetErrorString(e));
  return PT_OK;
}

// Geometry (K in FP64 and FP32) without a host read: the count of points with
// w*eta/detJ <= 0 goes to pinned memory, read when the set-up has completed.
pt_status srv_geometry(pt_op *op, unsigned int *h_bad)
{
  const int64_t nk = (int64_t)op->my * op->mz * 243 * op->MXP;
  PT_CUDA(op_alloc(op, (void **)&op->d_K, sizeof(double) * nk));
  PT_CUDA(op_alloc(op, (void **)&op->d_K32, sizeof(float) * nk));
  PT_CUDA(op_alloc(op, (void **)&op->d_bad, sizeof(unsigned int)));
  PT_CUDA(cudaMemsetAsync(op->d_bad, 0, sizeof(unsigned int), op->stream));
  ptk::geom_kernel<double><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->MXP, op->d_coords, op->d_eta,
                                                                       op->d_K, op->d_bad);
  PT_LAUNCHED(op);
  ptk::geom_kernel<float><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->MXP, op->d_coords, op->d_eta,
                                                                      op->d_K32, op->d_bad);
  PT_LAUNCHED(op);
  PT_CUDA(cudaMemcpyAsync(h_bad, op->d_bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, op->stream));
  op->geom_dirty = false;
  op->geom_ok = true;  // provisional: the request fails at join if h_bad > 0
  return PT_OK;
}

// Admission: everything enqueued on the set-up stream, no host wait.  Device
// state from the pool, uploads, geometry, diagonal, Lanczos lambda_max and
// Chebyshev coefficients, r0 = f, z0 = M r0, p0 = z0; then the ready event.
template <typename T>
pt_status srv_admit(pt_server *s, SrvReq *r, int slot)
{
  const cudaStream_t st = s->setup;
  pt_status e = op_create_impl(&r->desc, s->pool, st, &r->op);
  if (e != PT_OK) return e;
  pt_op *op = r->op;
  if (!op->full_box) return fail(PT_ERR_UNSUPPORTED, "request %lld: one-rank boxes only", (long long)r->id);
  op->a11_kernel = A11_STREAM;  // the batch runs the streaming kernel; set-up applies use the same
  if (s->o.lz > 0) {
    op->LZ = std::min(s->o.lz, op->mz);
    op->nzc = (op->mz + op->LZ - 1) / op->LZ;
  }
  const int64_t n = op->nvel;
  PT_CUDA(cudaMemcpyAsync(op->d_coords, r->h_coords, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  if ((e = finish_coords(op)) != PT_OK) return e;
  PT_CUDA(cudaMemcpyAsync(op->d_eta, r->h_eta, sizeof(double) * 27 * op->nel, cudaMemcpyHostToDevice, st));
  if ((e = finish_eta(op)) != PT_OK) return e;
  if (r->h_mask) {
    PT_CUDA(cudaMemcpyAsync(op->d_mask, r->h_mask, n, cudaMemcpyHostToDevice, st));
    if ((e = finish_mask(op)) != PT_OK) return e;
  }
  s->h_bad[slot] = 0;
  if ((e = srv_geometry(op, &s->h_bad[slot])) != PT_OK) return e;
  r->n = n;
  r->nch = (n + SRV_CH - 1) / SRV_CH;
  PT_CUDA(cudaMallocFromPoolAsync((void **)&r->vec, sizeof(double) * (4 * n + 2 * r->nch), s->pool, st));
  PT_CUDA(cudaMallocFromPoolAsync(&r->svec, sizeof(T) * 4 * n, s->pool, st));
  PT_CUDA(cudaMallocFromPoolAsync((void **)&r->tmp, sizeof(double) * (n + r->nch) + sizeof(LzState), s->pool, st));
  double *x = r->vec, *rr = x + n, *p = rr + n, *q = p + n, *part = q + n;
  T *z = (T *)r->svec, *d = z + n, *az = d + n, *dinv = az + n;
  double *diag = r->tmp, *lpart = diag + n;
  LzState *L = reinterpret_cast<LzState *>(lpart + r->nch);
  const unsigned nb = (unsigned)r->nch;
  // diagonal (Dirichlet slots 1) and its inverse in the smoother's precision
  if ((e = pt_getdiag_a11_d(op, diag)) != PT_OK) return e;
  convert_inv_kernel<T><<<vgrid(n), 256, 0, st>>>(diag, dinv, n);
  // slot descriptor and scalars (coefficients filled by the Lanczos finish)
  SrvSlot &S = r->S;
  S = SrvSlot{};
  S.n = n; S.x = x; S.r = rr; S.p = p; S.q = q; S.z = z; S.d = d; S.az = az; S.dinv = dinv;
  S.nch = r->nch; S.part = part;
  SrvScal &P = r->P;
  P = SrvScal{};
  P.rtol2 = s->o.rtol * s->o.rtol;
  P.atol2 = s->o.atol * s->o.atol;
  P.max_it = s->o.max_it;
  P.deg = s->o.cheby_degree;
  PT_CUDA(cudaMemcpyAsync(s->d_slots + slot, &S, sizeof S, cudaMemcpyHostToDevice, st));
  PT_CUDA(cudaMemcpyAsync(s->d_scal + slot, &P, sizeof P, cudaMemcpyHostToDevice, st));
  // Lanczos on scratch vectors x (r), r (z), p, q
  lz_start_kernel<<<nb, SRV_THREADS, 0, st>>>(n, diag, x, rr, p, lpart);
  lz_sum_kernel<0><<<1, SRV_THREADS, 0, st>>>(r->nch, lpart, L, 0);
  const int its = std::min(s->o.eig_its, SRV_MAX_LZ);
  for (int k = 0; k < its; k++) {
    if ((e = pt_matmult_a11_d(op, p, q)) != PT_OK) return e;
    lz_dot_kernel<<<nb, SRV_THREADS, 0, st>>>(n, p, q, lpart);
    lz_sum_kernel<1><<<1, SRV_THREADS, 0, st>>>(r->nch, lpart, L, k);
    lz_update_kernel<<<nb, SRV_THREADS, 0, st>>>(n, L, k, q, diag, x, rr, lpart);
    lz_sum_kernel<2><<<1, SRV_THREADS, 0, st>>>(r->nch, lpart, L, k);
    lz_p_kernel<<<nb, SRV_THREADS, 0, st>>>(n, L, k, rr, p);
  }
  lz_finish_kernel<<<1, 1, 0, st>>>(L, s->o.cheby_emin, s->o.cheby_emax, s->o.cheby_degree, s->d_scal + slot);
  s->launches += 3 + 5 * its;
  // Krylov start: x = 0, p = 0, q = 0, r = f
  PT_CUDA(cudaMemsetAsync(r->vec, 0, sizeof(double) * (4 * n + 2 * r->nch), st));
  PT_CUDA(cudaMemsetAsync(r->svec, 0, sizeof(T) * 3 * n, st));
  PT_CUDA(cudaMemcpyAsync(rr, r->h_f, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  // one-request chunk list and slot list (host copies live in the request until join)
  std::vector<int> one{slot};
  std::vector<int2> it = srv_items(one, s->slots);
  int2 *d_it = nullptr;
  int *d_one = nullptr;
  PT_CUDA(cudaMallocFromPoolAsync((void **)&d_it, sizeof(int2) * it.size(), s->pool, st));
  PT_CUDA(cudaMallocFromPoolAsync((void **)&d_one, sizeof(int), s->pool, st));
  PT_CUDA(cudaMemcpyAsync(d_it, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice, st));
  PT_CUDA(cudaMemcpyAsync(d_one, &r->slot, sizeof(int), cudaMemcpyHostToDevice, st));
  const unsigned ni = (unsigned)it.size();
  // r.r (alpha = 0 leaves x and r as they are)
  srv_update_kernel<<<ni, SRV_THREADS, 0, st>>>(d_it, s->d_slots, s->d_scal);
  srv_final_kernel<SRV_F_INIT_RR><<<1, SRV_THREADS, 0, st>>>(d_one, s->d_slots, s->d_scal);
  e = srv_precond<T>(s, d_it, ni, st, [&]() { return srv_apply_single<T>(op, z, az); });
  if (e != PT_OK) return e;
  srv_zdots_kernel<T><<<ni, SRV_THREADS, 0, st>>>(d_it, s->d_slots, s->d_scal);
  srv_final_kernel<SRV_F_INIT_RZ><<<1, SRV_THREADS, 0, st>>>(d_one, s->d_slots, s->d_scal);
  srv_p_kernel<T><<<ni, SRV_THREADS, 0, st>>>(d_it, s->d_slots, s->d_scal);
  s->launches += 5;
  PT_CUDA(cudaFreeAsync(d_it, st));
  PT_CUDA(cudaFreeAsync(d_one, st));
  PT_CUDA(cudaEventCreateWithFlags(&r->ready, cudaEventDisableTiming));
  PT_CUDA(cudaEventRecord(r->ready, st));
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return fail(PT_ERR_CUDA, "request set-up: %s", cudaGetErrorString(ce));
  return PT_OK;
}

// Requests whose set-up has completed join the batch (or fail, if their
// geometry check found w*eta/detJ <= 0).
pt_status srv_join(pt_server *s)
{
  for (int i = 0; i < (int)s->slots.size(); i++) {
    SrvReq *r = s->slots[i];
    if (!r || r->joined) continue;
    const cudaError_t q = cudaEventQuery(r->ready);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return fail(PT_ERR_CUDA, "request set-up: %s", cudaGetErrorString(q));
    if (s->h_bad[i] != 0) {
      r->t_done = s->now();
      r->fin = SrvScal{};
      r->fin.status = SRV_BREAKDOWN;
      srv_release(s, r);
      s->slots[i] = nullptr;
      s->done.push_back(r);
      continue;
    }
    r->op->stream = s->main;  // its applies now run in the batch
    r->joined = true;
    s->dirty = true;
  }
  return PT_OK;
}

// Rebuild the batch of joined requests: work-list, chunk list, pointer tables
// (stream-ordered on the main stream).
pt_status srv_rebuild(pt_server *s)
{
  const cudaStream_t st = s->main;
  if (s->batch) pt_batch_destroy(s->batch);
  s->batch = nullptr;
  if (s->d_act) cudaFreeAsync(s->d_act, st);
  if (s->d_items) cudaFreeAsync(s->d_items, st);
  if (s->d_ptrs) cudaFreeAsync(s->d_ptrs, st);
  s->d_act = nullptr;
  s->d_items = nullptr;
  s->d_ptrs = nullptr;
  s->act.clear();
  for (int i = 0; i < (int)s->slots.size(); i++)
    if (s->slots[i] && s->slots[i]->joined) s->act.push_back(i);
  s->nitems = 0;
  s->dirty = false;
  if (s->act.empty()) return PT_OK;
  std::vector<pt_op *> ops;
  const int na = (int)s->act.size();
  for (int i : s->act) ops.push_back(s->slots[i]->op);
  pt_status e = batch_create_impl(na, ops.data(), nullptr, s->o.tile_x, s->pool, st, &s->batch);
  if (e != PT_OK) return e;
  const size_t ts = s->fp32 ? sizeof(float) : sizeof(double);
  s->h_ptrs.assign(4 * na, nullptr);
  for (int k = 0; k < na; k++) {
    SrvReq *r = s->slots[s->act[k]];
    const int64_t n = r->n;
    s->h_ptrs[k] = r->vec + 2 * n;                         // p
    s->h_ptrs[na + k] = r->vec + 3 * n;                    // q
    s->h_ptrs[2 * na + k] = r->svec;                       // z
    s->h_ptrs[3 * na + k] = (char *)r->svec + 2 * ts * n;  // az
  }
  s->h_items = srv_items(s->act, s->slots);
  s->h_act = s->act;
  s->nitems = (int64_t)s->h_items.size();
  PT_CUDA(cudaMallocFromPoolAsync(&s->d_ptrs, sizeof(void *) * s->h_ptrs.size(), s->pool, st));
  PT_CUDA(cudaMallocFromPoolAsync((void **)&s->d_items, sizeof(int2) * s->h_items.size(), s->pool, st));
  PT_CUDA(cudaMallocFromPoolAsync((void **)&s->d_act, sizeof(int) * na, s->pool, st));
  PT_CUDA(cudaMemcpyAsync(s->d_ptrs, s->h_ptrs.data(), sizeof(void *) * s->h_ptrs.size(), cudaMemcpyHostToDevice, st));
  PT_CUDA(cudaMemcpyAsync(s->d_items, s->h_items.data(), sizeof(int2) * s->h_items.size(), cudaMemcpyHostToDevice, st));
  PT_CUDA(cudaMemcpyAsync(s->d_act, s->h_act.data(), sizeof(int) * na, cudaMemcpyHostToDevice, st));
  return PT_OK;
}

// One flexible-CG iteration of every joined request, enqueued on the main stream.
template <typename T>
pt_status srv_iterate(pt_server *s)
{
  const cudaStream_t st = s->main;
  const unsigned ni = (unsigned)s->nitems, na = (unsigned)s->act.size();
  const int n = (int)na;
  void **tab = (void **)s->d_ptrs;
  pt_status e = batch_apply<double, true>(s->batch, (const double *const *)tab, (double *const *)(tab + n), st);
  if (e != PT_OK) return e;
  s->launches += s->batch->classes.size() + 1;
  srv_pq_kernel<<<ni, SRV_THREADS, 0, st>>>(s->d_items, s->d_slots, s->d_scal);
  srv_final_kernel<SRV_F_ALPHA><<<na, SRV_THREADS, 0, st>>>(s->d_act, s->d_slots, s->d_scal);
  srv_update_kernel<<<ni, SRV_THREADS, 0, st>>>(s->d_items, s->d_slots, s->d_scal);
  srv_final_kernel<SRV_F_RR><<<na, SRV_THREADS, 0, st>>>(s->d_act, s->d_slots, s->d_scal);
  s->launches += 4;
  e = srv_precond<T>(s, s->d_items, ni, st, [&]() {
    s->launches += s->batch->classes.size() + 1;
    return batch_apply<T, true>(s->batch, (const T *const *)(tab + 2 * n), (T *const *)(tab + 3 * n), st);
  });
  if (e != PT_OK) return e;
  srv_zdots_kernel<T><<<ni, SRV_THREADS, 0, st>>>(s->d_items, s->d_slots, s->d_scal);
  srv_final_kernel<SRV_F_BETA><<<na, SRV_THREADS, 0, st>>>(s->d_act, s->d_slots, s->d_scal);
  srv_p_kernel<T><<<ni, SRV_THREADS, 0, st>>>(s->d_items, s->d_slots, s->d_scal);
  s->launches += 3;
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return fail(PT_ERR_CUDA, "server iteration launch: %s", cudaGetErrorString(ce));
  s->iterations++;
  return PT_OK;
}

// Retire finished requests (main stream idle): solution to the host,
// resources freed in stream order.
pt_status srv_retire(pt_server *s)
{
  const int ns = (int)s->slots.size();
  PT_CUDA(cudaMemcpyAsync(s->h_scal, s->d_scal, sizeof(SrvScal) * ns, cudaMemcpyDeviceToHost, s->main));
  PT_CUDA(cudaStreamSynchronize(s->main));
  for (int i = 0; i < ns; i++) {
    SrvReq *r = s->slots[i];
    if (!r || !r->joined || s->h_scal[i].status == SRV_ACTIVE) continue;
    PT_CUDA(cudaMemcpyAsync(r->h_x, r->vec, sizeof(double) * r->n, cudaMemcpyDeviceToHost, s->main));
    PT_CUDA(cudaStreamSynchronize(s->main));
    r->t_done = s->now();
    r->fin = s->h_scal[i];
    srv_release(s, r);
    s->slots[i] = nullptr;
    s->done.push_back(r);
    s->dirty = true;
  }
  return PT_OK;
}

}  // namespace

extern "C" {

void pt_server_opts_default(pt_server_opts *o)
{
  memset(o, 0, sizeof *o);
  o->memory_budget_bytes = (int64_t)120 << 30;
  o->max_active = 256;
  o->lz = 0;
  o->tile_x = 64;
  o->cheby_fp32 = 1;
  o->cheby_degree = 3;
  o->cheby_emin = 0.2;
  o->cheby_emax = 1.1;
  o->eig_its = 20;
  o->rtol = 1e-8;
  o->atol = 0.0;
  o->max_it = 20000;
}

pt_status pt_server_create(const pt_server_opts *opts, pt_server **out)
{
  if (!opts || !out) return fail(PT_ERR_BAD_ARG, "NULL argument");
  *out = nullptr;
  if (opts->max_active < 1 || opts->max_active > 4096) return fail(PT_ERR_BAD_ARG, "max_active must be in [1, 4096]");
  if (opts->cheby_degree < 1 || opts->cheby_degree > SRV_MAX_DEG)
    return fail(PT_ERR_BAD_ARG, "cheby_degree must be in [1, %d]", SRV_MAX_DEG);
  if (!(opts->cheby_emin > 0.0) || !(opts->cheby_emax > opts->cheby_emin))
    return fail(PT_ERR_BAD_ARG, "need 0 < cheby_emin < cheby_emax");
  if (opts->memory_budget_bytes <= 0) return fail(PT_ERR_BAD_ARG, "memory budget must be positive");
  if (opts->tile_x != 0 && opts->tile_x != 32 && opts->tile_x != 64 && opts->tile_x != 128)
    return fail(PT_ERR_BAD_ARG, "tile_x must be 0, 32, 64 or 128");
  pt_server *s = new (std::nothrow) pt_server();
  if (!s) return fail(PT_ERR_OOM, "host allocation failed");
  s->o = *opts;
  s->fp32 = opts->cheby_fp32 != 0;
  s->t0 = std::chrono::steady_clock::now();
  s->slots.assign(opts->max_active, nullptr);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->main, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->setup, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    // request state lives in a pool that keeps freed memory for reuse
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = dev;
    e = cudaMemPoolCreate(&s->pool, &pp);
    if (e == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->d_slots, sizeof(SrvSlot) * opts->max_active);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_scal, sizeof(SrvScal) * opts->max_active);
  if (e == cudaSuccess) e = cudaMemset(s->d_scal, 0, sizeof(SrvScal) * opts->max_active);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_scal, sizeof(SrvScal) * opts->max_active);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_bad, sizeof(unsigned int) * opts->max_active);
  if (e != cudaSuccess) {
    pt_status r = fail(PT_ERR_CUDA, "pt_server_create: %s", cudaGetErrorString(e));
    pt_server_destroy(s);
    return r;
  }
  *out = s;
  return PT_OK;
}

pt_status pt_server_destroy(pt_server *s)
{
  if (!s) return PT_OK;
  if (s->main) cudaStreamSynchronize(s->main);
  if (s->setup) cudaStreamSynchronize(s->setup);
  for (SrvReq *r : s->slots)
    if (r) {
      srv_release(s, r);
      delete r;
    }
  for (SrvReq *r : s->queue) delete r;
  for (SrvReq *r : s->done) delete r;
  if (s->batch) pt_batch_destroy(s->batch);
  if (s->d_act) cudaFreeAsync(s->d_act, s->main);
  if (s->d_items) cudaFreeAsync(s->d_items, s->main);
  if (s->d_ptrs) cudaFreeAsync(s->d_ptrs, s->main);
  if (s->main) cudaStreamSynchronize(s->main);
  cudaFree(s->d_slots);
  cudaFree(s->d_scal);
  if (s->h_scal) cudaFreeHost(s->h_scal);
  if (s->h_bad) cudaFreeHost(s->h_bad);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  if (s->main) cudaStreamDestroy(s->main);
  if (s->setup) cudaStreamDestroy(s->setup);
  delete s;
  return PT_OK;
}

double pt_server_time(const pt_server *s) { return s ? s->now() : 0.0; }

pt_status pt_server_submit(pt_server *s, int64_t id, const pt_mesh_desc *desc, const double *coords,
                           const double *eta, const uint8_t *mask, const double *f, double *x)
{
  if (!s || !desc || !coords || !eta || !f || !x) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (desc->mx < 1 || desc->my < 1 || desc->mz < 1) return fail(PT_ERR_BAD_ARG, "element counts must be >= 1");
  if (desc->nx || desc->ny || desc->nz || desc->ox || desc->oy || desc->oz)
    return fail(PT_ERR_UNSUPPORTED, "requests are one-rank boxes (node box = element box)");
  const size_t bytes = srv_bytes(*desc, s->fp32);
  if ((int64_t)bytes > s->o.memory_budget_bytes)
    return fail(PT_ERR_BAD_ARG, "request needs %zu bytes, more than the whole budget", bytes);
  SrvReq *r = new (std::nothrow) SrvReq();
  if (!r) return fail(PT_ERR_OOM, "host allocation failed");
  r->id = id;
  r->desc = *desc;
  r->h_coords = coords;
  r->h_eta = eta;
  r->h_mask = mask;
  r->h_f = f;
  r->h_x = x;
  r->bytes = bytes;
  r->t_submit = s->now();
  s->queue.push_back(r);
  return PT_OK;
}

pt_status pt_server_step(pt_server *s, int32_t iterations, int32_t *n_active, int32_t *n_queued)
{
  if (!s || iterations < 0) return fail(PT_ERR_BAD_ARG, "bad argument");
  pt_status e;
  double tp = s->now();
  if ((e = srv_join(s)) != PT_OK) return e;
  if (s->dirty && (e = srv_rebuild(s)) != PT_OK) return e;
  // 1. iterations of the current batch, enqueued (no host wait)
  if (!s->act.empty())
    for (int k = 0; k < iterations; k++) {
      e = s->fp32 ? srv_iterate<float>(s) : srv_iterate<double>(s);
      if (e != PT_OK) return e;
    }
  double tq = s->now();
  s->t_enqueue += tq - tp;
  tp = tq;
  // 2. admissions (set-up enqueued on the second stream): FIFO, as slots and
  //    the budget allow
  while (!s->queue.empty()) {
    SrvReq *r = s->queue.front();
    int slot = -1;
    for (int i = 0; i < (int)s->slots.size(); i++)
      if (!s->slots[i]) { slot = i; break; }
    if (slot < 0 || s->bytes_in_use + (int64_t)r->bytes > s->o.memory_budget_bytes) break;
    s->queue.pop_front();
    s->slots[slot] = r;
    r->slot = slot;
    s->bytes_in_use += (int64_t)r->bytes;
    r->t_admit = s->now();
    e = s->fp32 ? srv_admit<float>(s, r, slot) : srv_admit<double>(s, r, slot);
    if (e != PT_OK) {
      cudaStreamSynchronize(s->setup);
      srv_release(s, r);
      s->slots[slot] = nullptr;
      delete r;
      return e;
    }
  }
  tq = s->now();
  s->t_admit += tq - tp;
  tp = tq;
  // 3. wait for the batch, retire finished requests
  PT_CUDA(cudaStreamSynchronize(s->main));
  tq = s->now();
  s->t_wait += tq - tp;
  tp = tq;
  if ((e = srv_retire(s)) != PT_OK) return e;
  // nothing to iterate: wait for pending set-ups instead of spinning
  bool any_joined = false, any_pending = false;
  for (SrvReq *r : s->slots)
    if (r) (r->joined ? any_joined : any_pending) = true;
  if (!any_joined && any_pending) PT_CUDA(cudaStreamSynchronize(s->setup));
  s->t_retire += s->now() - tp;
  if (n_active) {
    int na = 0;
    for (SrvReq *r : s->slots) na += r != nullptr;
    *n_active = na;
  }
  if (n_queued) *n_queued = (int32_t)s->queue.size();
  return PT_OK;
}

pt_status pt_server_next_done(pt_server *s, pt_server_result *res)
{
  if (!s || !res) return fail(PT_ERR_BAD_ARG, "NULL argument");
  memset(res, 0, sizeof *res);
  res->id = -1;
  if (s->done.empty()) return PT_OK;
  SrvReq *r = s->done.front();
  s->done.pop_front();
  const SrvScal &P = r->fin;
  res->id = r->id;
  res->its = P.its;
  res->status = P.status;
  res->converged = P.status == SRV_CONVERGED;
  res->rnorm0 = std::sqrt(P.rr0);
  res->rnorm = std::sqrt(P.rr);
  res->lambda_max = P.lmax;
  res->t_submit = r->t_submit;
  res->t_admit = r->t_admit;
  res->t_done = r->t_done;
  delete r;
  return PT_OK;
}

pt_status pt_server_timers(const pt_server *s, double *enqueue, double *admit, double *wait, double *retire)
{
  if (!s) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (enqueue) *enqueue = s->t_enqueue;
  if (admit) *admit = s->t_admit;
  if (wait) *wait = s->t_wait;
  if (retire) *retire = s->t_retire;
  return PT_OK;
}

pt_status pt_server_stats(const pt_server *s, int64_t *iterations, int64_t *launches, int64_t *bytes_in_use)
{
  if (!s) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (iterations) *iterations = s->iterations;
  if (launches) *launches = s->launches;
  if (bytes_in_use) *bytes_in_use = s->bytes_in_use;
  return PT_OK;
}

}  // extern "C"
