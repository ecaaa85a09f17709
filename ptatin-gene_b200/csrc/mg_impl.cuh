// Geometric multigrid V-cycle on re-discretised Q2 levels, used as the
// preconditioner PT_PC_MG of the device Krylov solve.
//
// This is the structure of the reference's viscous-block preconditioner
// (src/ptatin_driver_linear_ts.c:482-514, 674-712): a hierarchy of nested
// structured Q2 meshes whose coordinates are restricted by injection
// (DMDARestrictCoordinatesHierarchy, :511), the matrix-free A11 re-discretised
// on every level ("-A11_operator_type ...,1"), Chebyshev-Jacobi smoothing
// (KSPCHEBYSHEV + PCJACOBI, window 0.2..1.1 of the estimated lambda_max).
// Here the levels run the same B200 kernels; the smoother is FP32 or FP64.
//
// Level l+1 has half the elements of level l per axis; coarse node i is fine
// node 2i.  Gauss-point viscosity of the coarse levels follows the reference's
// default coefficient projection (coefficient_projection_type 1, "Q1", with
// -mp_hierarchy_projection_type 0; material_point_utils.c:1325-1500): the fine
// Gauss-point viscosity is projected (lumped L2) onto a Q1 vertex field, the
// vertex field is carried down the hierarchy by normalised restriction, and
// each level's Gauss points interpolate their level's vertex field.
// Prolongation is Q2 interpolation in reference coordinates: along one axis a
// fine node 4e+m (m = 0..4) of coarse element e takes the coarse element's
// basis values at xi = -1 + m/2; restriction is its transpose.  Both are
// applied one axis at a time.  Dirichlet dofs (the injected mask) are zeroed
// after both transfers.
// Included from solver_impl.cuh after its vector kernels.
#pragma once

#include <vector>

namespace {

struct MgBox {
  int mx, my, mz;          // elements per axis of the level
  int64_t X, XY;           // node strides
};

__global__ void inject_coords_kernel(MgBox f, MgBox c, const double *__restrict__ xf, double *__restrict__ xc)
{
  const int64_t nc = c.X * (2 * (int64_t)c.my + 1) * (2 * (int64_t)c.mz + 1);
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nc; n += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = n % c.X, j = (n / c.X) % (2 * c.my + 1), k = n / c.XY;
    const int64_t nf = 2 * i + 2 * j * f.X + 2 * k * f.XY;
#pragma unroll
    for (int d = 0; d < 3; d++) xc[3 * n + d] = xf[3 * nf + d];
  }
}

__global__ void inject_mask_kernel(MgBox f, MgBox c, const uint8_t *__restrict__ mf, uint8_t *__restrict__ mc)
{
  const int64_t nc = c.X * (2 * (int64_t)c.my + 1) * (2 * (int64_t)c.mz + 1);
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nc; n += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = n % c.X, j = (n / c.X) % (2 * c.my + 1), k = n / c.XY;
    const int64_t nf = 2 * i + 2 * j * f.X + 2 * k * f.XY;
#pragma unroll
    for (int d = 0; d < 3; d++) mc[3 * n + d] = mf[3 * nf + d];
  }
}

// Q1 vertex basis at the 27 Gauss points: c_N1[q][v], q = a*9+b*3+c (c along
// xi), vertex v = k*4+j*2+i (i along xi).
__constant__ double c_N1[27][8];

// Lumped Q1 projection of the Gauss-point viscosity onto the element vertices
// (material_point_utils.c:1196-1323): vertex value = sum over the adjacent
// elements and their Gauss points of N1_v(xi_q) eta_q, divided by the sum of
// N1_v(xi_q).  One thread per vertex, a fixed order over the <= 8 elements.
__global__ void vertex_field_kernel(MgBox b, const double *__restrict__ eta, double *__restrict__ vf)
{
  const int VX = b.mx + 1, VY = b.my + 1;
  const int64_t nv = (int64_t)VX * VY * (b.mz + 1);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nv; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % VX), j = (int)((t / VX) % VY), k = (int)(t / ((int64_t)VX * VY));
    double num = 0.0, den = 0.0;
    for (int dk = 0; dk < 2; dk++)
      for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
          const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= b.mx || ej >= b.my || ek >= b.mz) continue;
          const int v = (1 - dk) * 4 + (1 - dj) * 2 + (1 - di);  // this vertex within element (ei,ej,ek)
          const double *e = eta + 27 * (ei + (int64_t)b.mx * (ej + (int64_t)b.my * ek));
          for (int q = 0; q < 27; q++) {
            num = fma(c_N1[q][v], e[q], num);
            den += c_N1[q][v];
          }
        }
    vf[t] = num / den;
  }
}

// Coarse vertex field from the fine one: weights (1/4, 1/2, 1/4) per axis on
// fine vertices 2I-1, 2I, 2I+1, renormalised at the box faces (a weighted
// average, so positive fields stay positive).
__global__ void restrict_vertex_kernel(MgBox f, MgBox c, const double *__restrict__ vf, double *__restrict__ vc)
{
  const int VX = c.mx + 1, VY = c.my + 1;
  const int FX = f.mx + 1, FY = f.my + 1, FZ = f.mz + 1;
  const int64_t nv = (int64_t)VX * VY * (c.mz + 1);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nv; t += (int64_t)gridDim.x * blockDim.x) {
    const int I = (int)(t % VX), J = (int)((t / VX) % VY), K = (int)(t / ((int64_t)VX * VY));
    double acc = 0.0, wsum = 0.0;
    for (int oz = -1; oz <= 1; oz++) {
      const int z = 2 * K + oz;
      if (z < 0 || z >= FZ) continue;
      const double wz = oz == 0 ? 0.5 : 0.25;
      for (int oy = -1; oy <= 1; oy++) {
        const int y = 2 * J + oy;
        if (y < 0 || y >= FY) continue;
        const double wy = oy == 0 ? 0.5 : 0.25;
        for (int ox = -1; ox <= 1; ox++) {
          const int x = 2 * I + ox;
          if (x < 0 || x >= FX) continue;
          const double w = wz * wy * (ox == 0 ? 0.5 : 0.25);
          acc = fma(w, vf[x + (int64_t)FX * (y + (int64_t)FY * z)], acc);
          wsum += w;
        }
      }
    }
    vc[t] = acc / wsum;
  }
}

// Gauss-point viscosity of a level from its vertex field (Q1 interpolation).
__global__ void eta_from_vertex_kernel(MgBox b, const double *__restrict__ vf, double *__restrict__ eta)
{
  const int VX = b.mx + 1, VY = b.my + 1;
  const int64_t nel = (int64_t)b.mx * b.my * b.mz;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nel * 27; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / 27;
    const int q = (int)(t % 27);
    const int ei = (int)(e % b.mx), ej = (int)((e / b.mx) % b.my), ek = (int)(e / ((int64_t)b.mx * b.my));
    double v = 0.0;
#pragma unroll
    for (int n = 0; n < 8; n++) {
      const int i = ei + (n & 1), j = ej + ((n >> 1) & 1), k = ek + (n >> 2);
      v = fma(c_N1[q][n], vf[i + (int64_t)VX * (j + (int64_t)VY * k)], v);
    }
    eta[t] = v;
  }
}

// c_N1 from the Gauss abscissae (host side, once per process and device).
pt_status upload_q1_table()
{
  static bool done[64] = {false};
  static std::mutex mu;
  int dev = 0;
  PT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 64 && done[dev]) return PT_OK;
  const double g[3] = {-q2::GS, 0.0, q2::GS};
  double t[27][8];
  for (int a = 0; a < 3; a++)
    for (int bq = 0; bq < 3; bq++)
      for (int cq = 0; cq < 3; cq++)
        for (int v = 0; v < 8; v++) {
          const double nx = (v & 1) ? 0.5 * (1.0 + g[cq]) : 0.5 * (1.0 - g[cq]);
          const double ny = ((v >> 1) & 1) ? 0.5 * (1.0 + g[bq]) : 0.5 * (1.0 - g[bq]);
          const double nz = ((v >> 2) & 1) ? 0.5 * (1.0 + g[a]) : 0.5 * (1.0 - g[a]);
          t[a * 9 + bq * 3 + cq][v] = nx * ny * nz;
        }
  PT_CUDA(cudaMemcpyToSymbol(c_N1, t, sizeof t));
  if (dev < 64) done[dev] = true;
  return PT_OK;
}

// ---- transfers, one axis at a time ------------------------------------------
// P = Pz (x) Py (x) Px.  Along one axis with mc coarse elements (2mc+1 coarse,
// 4mc+1 fine nodes), fine node 4e+m takes the coarse element's Q2 basis at
// xi = -1 + m/2:
//   m even: coarse node (4e+m)/2 (injection)
//   m = 1 : 3/8 c[2e] + 3/4 c[2e+1] - 1/8 c[2e+2]
//   m = 3 : -1/8 c[2e] + 3/4 c[2e+1] + 3/8 c[2e+2]
// and the transpose, for coarse node I:
//   I even: r[2I] + 3/8 (r[2I-1] + r[2I+1]) - 1/8 (r[2I-3] + r[2I+3])
//   I odd : r[2I] + 3/4 (r[2I-1] + r[2I+1])
// (terms outside the box dropped).  Arrays are [n2][n1][n0][3]; a pass maps
// one axis and keeps the other two; one thread per output value.
struct Dims3 {
  int n[3];
};

template <typename T, int AXIS, bool PROLONG, int FINAL>
__global__ void transfer_axis_kernel(Dims3 din, Dims3 dout, const T *__restrict__ in, T *__restrict__ out,
                                     const uint8_t *__restrict__ mask)
{
  // FINAL: 0 = write, 1 = out = mask ? 0 : out + v (prolongation into x), 2 = out = mask ? 0 : v
  const int64_t nout = 3 * (int64_t)dout.n[0] * dout.n[1] * dout.n[2];
  const int64_t s_in = AXIS == 0 ? 3 : (AXIS == 1 ? 3 * (int64_t)din.n[0] : 3 * (int64_t)din.n[0] * din.n[1]);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nout; t += (int64_t)gridDim.x * blockDim.x) {
    const int d = (int)(t % 3);
    const int64_t node = t / 3;
    int o[3];
    o[0] = (int)(node % dout.n[0]);
    o[1] = (int)((node / dout.n[0]) % dout.n[1]);
    o[2] = (int)(node / ((int64_t)dout.n[0] * dout.n[1]));
    const int a = o[AXIS];
    int q[3] = {o[0], o[1], o[2]};
    q[AXIS] = 0;
    const T *base = in + 3 * (q[0] + (int64_t)din.n[0] * (q[1] + (int64_t)din.n[1] * q[2])) + d;
    T v;
    if (PROLONG) {
      const int mc = (din.n[AXIS] - 1) / 2;
      int e = a >> 2;
      if (e > mc - 1) e = mc - 1;
      const int m = a - 4 * e;
      const T *c = base + (int64_t)(2 * e) * s_in;
      if (m == 0) v = c[0];
      else if (m == 2) v = c[s_in];
      else if (m == 4) v = c[2 * s_in];
      else if (m == 1) v = T(0.375) * c[0] + T(0.75) * c[s_in] - T(0.125) * c[2 * s_in];
      else v = T(-0.125) * c[0] + T(0.75) * c[s_in] + T(0.375) * c[2 * s_in];
    } else {
      const int nf = din.n[AXIS];
      const int i = 2 * a;
      auto at = [&](int k) { return (k >= 0 && k < nf) ? base[(int64_t)k * s_in] : T(0); };
      if ((a & 1) == 0)
        v = at(i) + T(0.375) * (at(i - 1) + at(i + 1)) - T(0.125) * (at(i - 3) + at(i + 3));
      else
        v = at(i) + T(0.75) * (at(i - 1) + at(i + 1));
    }
    if (FINAL == 0) out[t] = v;
    else if (FINAL == 1) out[t] = mask[t] ? T(0) : out[t] + v;
    else out[t] = mask[t] ? T(0) : v;
  }
}

// Small levels store their element matrices (kernels_ebe.cuh): the
// streaming kernel on a handful of CTAs costs about as much per apply as on
// a large level, because each CTA's z-march is a latency chain; the reference
// assembles its coarse levels (OP_TYPE_REDISC_ASM, ptatin_driver_linear_ts.c:
// 636-712).

// x = Ainv b on the coarsest level (dense symmetric inverse, one warp per row).
template <typename T>
__global__ void dense_apply_kernel(int n, const T *__restrict__ Ainv, const T *__restrict__ b, T *__restrict__ x)
{
  const int lane = threadIdx.x & 31;
  const int row = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (row >= n) return;
  const T *a = Ainv + (int64_t)row * n;
  T acc = T(0);
  for (int j = lane; j < n; j += 32) acc = fma(a[j], b[j], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) x[row] = acc;
}

template <typename T>
__global__ void sub_kernel(const T *__restrict__ b, const T *__restrict__ ax, T *__restrict__ r, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - ax[i];
}

template <typename T>
__global__ void add_kernel(const T *__restrict__ a, T *__restrict__ x, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += a[i];
}

MgBox mgbox(const pt_op *op)
{
  MgBox b;
  b.mx = op->mx; b.my = op->my; b.mz = op->mz;
  b.X = 2 * (int64_t)op->mx + 1;
  b.XY = b.X * (2 * (int64_t)op->my + 1);
  return b;
}

}  // namespace

struct pt_mg_level {
  pt_op *op;
  bool own;
  int64_t n;
  double lmax;
  double *dinv64;
  float *dinv32;
  void *x, *b, *r, *d, *az, *dl;  // T-sized work vectors
  void *t1, *t2;                   // transfer temporaries (to / from the next coarser level)
  void *Ae, *ye;                   // element matrices and per-element outputs (small levels), else null
  double *Ae64;                    // Galerkin levels: FP64 element matrices P^T A P (Ae aliases or converts them)
  __half *Ah;                      // Galerkin levels under FP32 smoothing: the matrices in FP16, scaled per
  float *Ascale;                   // element by Ascale (mg_coarse_half), replacing an FP32 copy in Ae
  void *Ainv;                      // dense inverse (coarsest level, when small), else null
  int64_t nel;
};

struct pt_mg {
  std::vector<pt_mg_level> lv;
  bool fp32;
  int degree, coarse_degree, fine_degree;
  double emin, emax;
  bool coarse_half;      // FP32 smoothing: Galerkin levels' matrices stored in FP16 (scaled per element)
  int64_t fine_applies;  // A11 applies on level 0 inside V-cycles
  double coarse_work;    // coarse-level applies weighted by elements / fine elements
  bool assembled;  // element matrices on small levels, dense inverse on a small coarsest level
  // the V-cycle captured once as a CUDA graph (its launches are fixed)
  bool use_graph;
  cudaGraphExec_t gexec;
  int64_t graph_fine;  // level-0 applies per replay
  double graph_coarse;
};

namespace {

template <typename T>
pt_status mg_matmult(pt_mg &mg, pt_mg_level &L, const T *x, T *y)
{
  if (L.op == mg.lv[0].op) mg.fine_applies++;
  else mg.coarse_work += (double)L.op->nel / (double)mg.lv[0].op->nel;
  if constexpr (std::is_same<T, float>::value) {
    if (L.Ah) {
      ebe_h_carveout<true>();
      ptk::ebe_apply_h_kernel<true><<<(unsigned)L.nel, 96, 0, L.op->stream>>>(L.op->box, L.Ah, L.Ascale, x,
                                                                               L.op->d_mask, (float *)L.ye);
      PT_LAUNCHED(L.op);
      ptk::ebe_gather_kernel<float, true><<<vgrid(L.n), 256, 0, L.op->stream>>>(L.op->box, (const float *)L.ye, x,
                                                                                L.op->d_mask, y);
      PT_LAUNCHED(L.op);
      return PT_OK;
    }
  }
  if (L.Ae) {
    ebe_carveout<T, true>();
    ptk::ebe_apply_kernel<T, true><<<(unsigned)L.nel, 96, 0, L.op->stream>>>(L.op->box, (const T *)L.Ae, x,
                                                                              L.op->d_mask, (T *)L.ye);
    PT_LAUNCHED(L.op);
    ptk::ebe_gather_kernel<T, true><<<vgrid(L.n), 256, 0, L.op->stream>>>(L.op->box, (const T *)L.ye, x,
                                                                          L.op->d_mask, y);
    PT_LAUNCHED(L.op);
    return PT_OK;
  }
  if (std::is_same<T, double>::value) return pt_matmult_a11_d(L.op, (const double *)x, (double *)y);
  return pt_matmult_a11_f32_d(L.op, (const float *)x, (float *)y);
}

template <typename T>
const T *mg_dinv(const pt_mg_level &L);
template <>
const double *mg_dinv<double>(const pt_mg_level &L) { return L.dinv64; }
template <>
const float *mg_dinv<float>(const pt_mg_level &L) { return L.dinv32; }

// x <- x + Cheb_k(D^-1 A)(b - A x): k Chebyshev steps on level L
template <typename T>
pt_status mg_cheby(pt_mg &mg, pt_mg_level &L, const T *b, T *x, bool x_zero, int k)
{
  cudaStream_t st = L.op->stream;
  const int64_t n = L.n;
  T *r = (T *)L.r, *d = (T *)L.d, *az = (T *)L.az, *dl = (T *)L.dl;
  const double emax = mg.emax * L.lmax, emin = mg.emin * L.lmax;
  const double theta = 0.5 * (emax + emin), delta = 0.5 * (emax - emin), sigma = theta / delta;
  double rho = 1.0 / sigma;
  pt_status s;
  const T *rr = b;
  if (!x_zero) {
    if ((s = mg_matmult<T>(mg, L, x, az)) != PT_OK) return s;
    sub_kernel<T><<<vgrid(n), 256, 0, st>>>(b, az, r, n);
    PT_LAUNCHED(L.op);
    rr = r;
  }
  // correction dl (= z of the recurrence) from residual rr
  cheb_first_kernel<T><<<vgrid(n), 256, 0, st>>>((T)(1.0 / theta), mg_dinv<T>(L), rr, d, dl, n);
  PT_LAUNCHED(L.op);
  for (int i = 1; i < k; i++) {
    if ((s = mg_matmult<T>(mg, L, dl, az)) != PT_OK) return s;
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    cheb_step_kernel<T><<<vgrid(n), 256, 0, st>>>((T)(rho_new * rho), (T)(2.0 * rho_new / delta), mg_dinv<T>(L), rr,
                                                   az, d, dl, n);
    PT_LAUNCHED(L.op);
    rho = rho_new;
  }
  if (x_zero) {
    PT_CUDA(cudaMemcpyAsync(x, dl, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
  } else {
    add_kernel<T><<<vgrid(n), 256, 0, st>>>(dl, x, n);
    PT_LAUNCHED(L.op);
  }
  return PT_OK;
}

template <typename T>
pt_status mg_vcycle(pt_mg &mg, int l)
{
  pt_mg_level &L = mg.lv[l];
  T *x = (T *)L.x, *b = (T *)L.b;
  pt_status s;
  if (l + 1 == (int)mg.lv.size()) {
    if (L.Ainv) {
      dense_apply_kernel<T><<<(unsigned)((L.n * 32 + 255) / 256), 256, 0, L.op->stream>>>((int)L.n, (const T *)L.Ainv,
                                                                                          b, x);
      PT_LAUNCHED(L.op);
      return PT_OK;
    }
    return mg_cheby<T>(mg, L, b, x, true, mg.coarse_degree);
  }
  const int degree = l == 0 ? mg.fine_degree : mg.degree;
  if ((s = mg_cheby<T>(mg, L, b, x, true, degree)) != PT_OK) return s;
  // residual -> coarse rhs
  pt_mg_level &C = mg.lv[l + 1];
  if ((s = mg_matmult<T>(mg, L, x, (T *)L.az)) != PT_OK) return s;
  sub_kernel<T><<<vgrid(L.n), 256, 0, L.op->stream>>>(b, (T *)L.az, (T *)L.r, L.n);
  PT_LAUNCHED(L.op);
  const cudaStream_t st = L.op->stream;
  const int fx = 2 * L.op->mx + 1, fy = 2 * L.op->my + 1, fz = 2 * L.op->mz + 1;
  const int cx = 2 * C.op->mx + 1, cy = 2 * C.op->my + 1, cz = 2 * C.op->mz + 1;
  const Dims3 dF{{fx, fy, fz}}, dXf{{cx, fy, fz}}, dXYf{{cx, cy, fz}}, dC{{cx, cy, cz}};
  T *t1 = (T *)L.t1, *t2 = (T *)L.t2;
  // b_c = R r_f: x, then y, then z (masked)
  transfer_axis_kernel<T, 0, false, 0><<<vgrid(3LL * cx * fy * fz), 256, 0, st>>>(dF, dXf, (T *)L.r, t1, nullptr);
  PT_LAUNCHED(L.op);
  transfer_axis_kernel<T, 1, false, 0><<<vgrid(3LL * cx * cy * fz), 256, 0, st>>>(dXf, dXYf, t1, t2, nullptr);
  PT_LAUNCHED(L.op);
  transfer_axis_kernel<T, 2, false, 2><<<vgrid(C.n), 256, 0, st>>>(dXYf, dC, t2, (T *)C.b, C.op->d_mask);
  PT_LAUNCHED(L.op);
  if ((s = mg_vcycle<T>(mg, l + 1)) != PT_OK) return s;
  // x_f += P x_c: z, then y, then x (masked add)
  transfer_axis_kernel<T, 2, true, 0><<<vgrid(3LL * cx * cy * fz), 256, 0, st>>>(dC, dXYf, (T *)C.x, t2, nullptr);
  PT_LAUNCHED(L.op);
  transfer_axis_kernel<T, 1, true, 0><<<vgrid(3LL * cx * fy * fz), 256, 0, st>>>(dXYf, dXf, t2, t1, nullptr);
  PT_LAUNCHED(L.op);
  transfer_axis_kernel<T, 0, true, 1><<<vgrid(L.n), 256, 0, st>>>(dXf, dF, t1, x, L.op->d_mask);
  PT_LAUNCHED(L.op);
  return mg_cheby<T>(mg, L, b, x, false, degree);
}

}  // namespace
