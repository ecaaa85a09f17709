// Stored element matrices ("b200_ebe" and the small multigrid levels).
//
// An element's 81x81 matrix is the colour kernel's element operator applied
// to the unit vectors (exact FP64 arithmetic of the reference's element
// kernel, adjugate form), in FP64 or FP32.  The matrix is symmetric, so only
// its upper triangle is stored, packed by columns: entry (i, j), i <= j, dof
// index 3n+l, at j(j+1)/2 + i; 3321 values per element, padded to EBE_LD so
// that each element's block starts on a 16-byte boundary.  An apply is two
// launches: a GEMV per element into per-element outputs (the packed block
// staged in shared memory by cp.async), and a gather per dof that sums the
// (at most 8) element contributions of its node in a fixed order -- a node-
// centred scatter, deterministic without atomics.  It reads 26.6 KB per
// element (FP64), so it pays only where the streaming kernel is latency-bound
// (small boxes: a few CTAs, each marching its layers one after another) and
// on multigrid levels whose operator only exists as element matrices.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "kernels_colour.cuh"
#include "q2_core.cuh"

namespace ptk {

constexpr int EBE_LD = 3328;  // packed upper triangle (3321) padded to a multiple of 16 bytes

// Packed position of entry (i, j) of a symmetric element matrix.
__host__ __device__ __forceinline__ int ebe_sym(int i, int j)
{
  return i <= j ? j * (j + 1) / 2 + i : i * (i + 1) / 2 + j;
}


// Column j of element e's matrix: the element operator of the colour kernel
// applied to the unit vector e_j.  Block = element, 81 threads.
template <typename T>
__global__ void __launch_bounds__(96) element_matrix_kernel(Box b, const double *__restrict__ coords,
                                                            const double *__restrict__ eta, T *__restrict__ Ae)
{
  const int j = threadIdx.x;
  if (j >= 81) return;
  const int64_t e = blockIdx.x;
  const int ei = (int)(e % b.mx), ej = (int)((e / b.mx) % b.my), ek = (int)(e / ((int64_t)b.mx * b.my));
  int64_t nid[27];
  element_nodes(b, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  const int nj = j / 3, lj = j % 3;
  double Ug[3][3][27];
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++)
      for (int q = 0; q < 27; q++) Ug[k][l][q] = 0.0;
  {
    double f[27], I[27];
    for (int n = 0; n < 27; n++) f[n] = n == nj ? 1.0 : 0.0;
    q2::interp(f, I);
    q2::grad_colloc(I, Ug[0][lj], Ug[1][lj], Ug[2][lj]);
  }
  for (int q = 0; q < 27; q++) {
    double J[3][3], adj[3][3], G[3][3], d[3][3];
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) {
        J[k][l] = Jg[k][l][q];
        G[k][l] = Ug[k][l][q];
      }
    const double det = q2::adjugate(J, adj);
    const double c = q2::weight(q) * eta[27 * e + q] / det;
    q2::qp_viscous(adj, c, G, d);
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) Ug[k][l][q] = d[k][l];
  }
  T *blk = Ae + e * EBE_LD;
  for (int l = 0; l < 3; l++) {
    double r[27], f[27];
    q2::grad_colloc_t(Ug[0][l], Ug[1][l], Ug[2][l], r);
    q2::interp_t(r, f);
    for (int n = 0; n < 27; n++)
      if (3 * n + l <= j) blk[ebe_sym(3 * n + l, j)] = (T)f[n];
  }
  if (j < EBE_LD - 3321) blk[3321 + j] = T(0);
}

template <typename S>
__device__ __forceinline__ S ld_shared(uint32_t a);
template <>
__device__ __forceinline__ double ld_shared<double>(uint32_t a)
{
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}
template <>
__device__ __forceinline__ float ld_shared<float>(uint32_t a)
{
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
template <>
__device__ __forceinline__ __half ld_shared<__half>(uint32_t a)
{
  unsigned short v;
  asm volatile("ld.shared.b16 %0, [%1];" : "=h"(v) : "r"(a));
  return __ushort_as_half(v);
}
__device__ __forceinline__ double ebe_val(double a) { return a; }
__device__ __forceinline__ float ebe_val(float a) { return a; }
__device__ __forceinline__ float ebe_val(__half a) { return __half2float(a); }

// Row t of an element's packed symmetric matrix (storage S, shared address
// sbase) times ue (T, 84 entries, 16-byte aligned, 81..83 zero), summed in the
// order j = 0..80.  Entry (t, j) sits in column t of the upper triangle
// (offset b1 + j) for j < t and in column j (offset b2 + j(j+1)/2) for j >= t;
// fully unrolled, both offsets are immediates and each entry costs one shared
// load (a warp's row-part loads are consecutive, conflict-free), and u is read
// 16 bytes at a time.  Warp W holds rows 32W..32W+31, so columns j < 32W are
// column-part entries for every lane and j >= 32W+32 row-part entries: only
// the 32 columns in between choose per lane.  Measured on 262,144 elements
// against a loop with computed indices: FP16 storage 0.84 -> 0.57 ms, FP32
// 0.98 -> 0.80 ms, FP64 1.71 -> 1.45 ms, bitwise the same sums.
template <typename S, typename T, int W>
__device__ __forceinline__ T ebe_row_w(uint32_t b1, uint32_t b2, int t, const T *ue)
{
  constexpr int VW = 16 / (int)sizeof(T);
  T acc = T(0);
#pragma unroll
  for (int j0 = 0; j0 < 84; j0 += VW) {
    T xv[VW];
    if constexpr (VW == 4) {
      const float4 q = reinterpret_cast<const float4 *>(ue)[j0 / 4];
      xv[0] = q.x; xv[1] = q.y; xv[2] = q.z; xv[3] = q.w;
    } else {
      const double2 q = reinterpret_cast<const double2 *>(ue)[j0 / 2];
      xv[0] = q.x; xv[1] = q.y;
    }
#pragma unroll
    for (int c = 0; c < VW; c++) {
      const int j = j0 + c;
      if (j < 81) {
        const uint32_t col = b1 + (uint32_t)sizeof(S) * j;
        const uint32_t row = b2 + (uint32_t)sizeof(S) * (j * (j + 1) / 2);
        const uint32_t a = j < 32 * W ? col : (j >= 32 * W + 32 ? row : (j < t ? col : row));
        acc = fma((T)ebe_val(ld_shared<S>(a)), xv[c], acc);
      }
    }
  }
  return acc;
}

template <typename S, typename T>
__device__ __forceinline__ T ebe_row(uint32_t sbase, int t, const T *ue)
{
  const uint32_t b1 = sbase + (uint32_t)sizeof(S) * (uint32_t)(t * (t + 1) / 2);
  const uint32_t b2 = sbase + (uint32_t)sizeof(S) * (uint32_t)t;
  const int w = t >> 5;  // warp-uniform
  if (w == 0) return ebe_row_w<S, T, 0>(b1, b2, t, ue);
  if (w == 1) return ebe_row_w<S, T, 1>(b1, b2, t, ue);
  return ebe_row_w<S, T, 2>(b1, b2, t, ue);
}

// ye[e][i] = sum_j A_e(i, j) u_j in the order j = 0..80 (MASKED: Dirichlet
// entries of u taken as 0).  The element's packed block is copied to shared
// memory with 16-byte cp.async while u is gathered.
template <typename T, bool MASKED>
__global__ void __launch_bounds__(96) ebe_apply_kernel(Box b, const T *__restrict__ Ae, const T *__restrict__ u,
                                                       const uint8_t *__restrict__ mask, T *__restrict__ ye)
{
  __shared__ __align__(16) T S[EBE_LD];
  __shared__ __align__(16) T ue[84];
  const int t = threadIdx.x;
  const int64_t e = blockIdx.x;
  {
    constexpr int NCH = EBE_LD * (int)sizeof(T) / 16;
    const char *src = reinterpret_cast<const char *>(Ae + e * EBE_LD);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(S);
    for (int c = t; c < NCH; c += blockDim.x)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16u * c), "l"(src + 16 * (int64_t)c)
                   : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  const int ei = (int)(e % b.mx), ej = (int)((e / b.mx) % b.my), ek = (int)(e / ((int64_t)b.mx * b.my));
  if (t < 84) {
    T v = T(0);
    if (t < 81) {
      const int n = t / 3, l = t % 3;
      const int64_t node = b.off + (2 * ei + n % 3) + (2 * (int64_t)ej + (n / 3) % 3) * b.X + (2 * (int64_t)ek + n / 9) * b.XY;
      const int64_t k = 3 * node + l;
      v = (MASKED && mask[k]) ? T(0) : u[k];
    }
    ue[t] = v;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  if (t < 81) ye[e * 81 + t] = ebe_row<T, T>((uint32_t)__cvta_generic_to_shared(S), t, ue);
}

// FP16 copy of packed FP64 element matrices for an FP32 apply (multigrid
// coarse levels under FP32 smoothing): each element's block divided by its
// largest magnitude, scale[e] = that magnitude, so every entry is stored to
// within 2^-12 of the element's largest entry (subnormal FP16 below 6.1e-5 of
// it) and the FP16 range never matters.  Block = element, 128 threads.
__global__ void __launch_bounds__(128) ebe_to_half_kernel(const double *__restrict__ A, __half *__restrict__ Ah,
                                                          float *__restrict__ scale)
{
  __shared__ double wmax[4];
  const int t = threadIdx.x;
  const int64_t e = blockIdx.x;
  const double *a = A + e * EBE_LD;
  double m = 0.0;
  for (int i = t; i < 3321; i += 128) m = fmax(m, fabs(a[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) wmax[t >> 5] = m;
  __syncthreads();
  m = fmax(fmax(wmax[0], wmax[1]), fmax(wmax[2], wmax[3]));
  const double sc = m > 0.0 ? m : 1.0;
  for (int i = t; i < EBE_LD; i += 128) Ah[e * EBE_LD + i] = __double2half(i < 3321 ? a[i] / sc : 0.0);
  if (t == 0) scale[e] = (float)sc;
}

// ebe_apply_kernel<float> on the FP16 copy: ye[e][i] = scale[e] * sum_j
// A_e(i, j) u_j, FP32 arithmetic, j = 0..80 in order.  Reads 6.6 KB per
// element instead of 13.3 KB.
template <bool MASKED>
__global__ void __launch_bounds__(96) ebe_apply_h_kernel(Box b, const __half *__restrict__ Ah,
                                                         const float *__restrict__ scale, const float *__restrict__ u,
                                                         const uint8_t *__restrict__ mask, float *__restrict__ ye)
{
  __shared__ __align__(16) __half S[EBE_LD];
  __shared__ __align__(16) float ue[84];
  const int t = threadIdx.x;
  const int64_t e = blockIdx.x;
  {
    constexpr int NCH = EBE_LD * (int)sizeof(__half) / 16;
    const char *src = reinterpret_cast<const char *>(Ah + e * EBE_LD);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(S);
    for (int c = t; c < NCH; c += blockDim.x)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16u * c), "l"(src + 16 * (int64_t)c)
                   : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  const int ei = (int)(e % b.mx), ej = (int)((e / b.mx) % b.my), ek = (int)(e / ((int64_t)b.mx * b.my));
  if (t < 84) {
    float v = 0.0f;
    if (t < 81) {
      const int n = t / 3, l = t % 3;
      const int64_t node = b.off + (2 * ei + n % 3) + (2 * (int64_t)ej + (n / 3) % 3) * b.X + (2 * (int64_t)ek + n / 9) * b.XY;
      const int64_t k = 3 * node + l;
      v = (MASKED && mask[k]) ? 0.0f : u[k];
    }
    ue[t] = v;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  if (t < 81) ye[e * 81 + t] = ebe_row<__half, float>((uint32_t)__cvta_generic_to_shared(S), t, ue) * scale[e];
}

// y_k = sum over the (<= 8) elements of node k of their ye entry, in a fixed
// order (MASKED: y_k = x_k on Dirichlet dofs; ACC: added to y).  One-rank
// boxes (node box = element box).
template <typename T, bool MASKED, bool ACC = false>
__global__ void ebe_gather_kernel(Box b, const T *__restrict__ ye, const T *__restrict__ x,
                                  const uint8_t *__restrict__ mask, T *__restrict__ y)
{
  const int64_t n = 3 * b.XY * (2 * (int64_t)b.mz + 1);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    if (MASKED && mask[t]) {
      y[t] = x[t];
      continue;
    }
    const int l = (int)(t % 3);
    const int64_t node = t / 3;
    const int i = (int)(node % b.X), j = (int)((node / b.X) % (2 * b.my + 1)), k = (int)(node / b.XY);
    // per axis: (element, local index) pairs, lower element first
    int ex[2], lx[2], nx = 0, ey[2], ly[2], ny = 0, ez[2], lz[2], nz = 0;
    if (i & 1) { ex[0] = i >> 1; lx[0] = 1; nx = 1; }
    else {
      if (i > 0) { ex[nx] = (i >> 1) - 1; lx[nx++] = 2; }
      if ((i >> 1) < b.mx) { ex[nx] = i >> 1; lx[nx++] = 0; }
    }
    if (j & 1) { ey[0] = j >> 1; ly[0] = 1; ny = 1; }
    else {
      if (j > 0) { ey[ny] = (j >> 1) - 1; ly[ny++] = 2; }
      if ((j >> 1) < b.my) { ey[ny] = j >> 1; ly[ny++] = 0; }
    }
    if (k & 1) { ez[0] = k >> 1; lz[0] = 1; nz = 1; }
    else {
      if (k > 0) { ez[nz] = (k >> 1) - 1; lz[nz++] = 2; }
      if ((k >> 1) < b.mz) { ez[nz] = k >> 1; lz[nz++] = 0; }
    }
    T acc = T(0);
    for (int c = 0; c < nz; c++)
      for (int bb = 0; bb < ny; bb++)
        for (int a = 0; a < nx; a++) {
          const int64_t e = ex[a] + (int64_t)b.mx * (ey[bb] + (int64_t)b.my * ez[c]);
          acc += ye[e * 81 + 3 * (lx[a] + 3 * ly[bb] + 9 * lz[c]) + l];
        }
    y[t] = ACC ? y[t] + acc : acc;
  }
}

// diag(A11)_k = sum over the elements of node k of their matrix diagonal
// entry (fixed order, as ebe_gather_kernel).
__global__ void ebe_diag_kernel(Box b, const double *__restrict__ Ae, double *__restrict__ d)
{
  const int64_t n = 3 * b.XY * (2 * (int64_t)b.mz + 1);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % 3);
    const int64_t node = t / 3;
    const int i = (int)(node % b.X), j = (int)((node / b.X) % (2 * b.my + 1)), k = (int)(node / b.XY);
    int ex[2], lx[2], nx = 0, ey[2], ly[2], ny = 0, ez[2], lz[2], nz = 0;
    if (i & 1) { ex[0] = i >> 1; lx[0] = 1; nx = 1; }
    else {
      if (i > 0) { ex[nx] = (i >> 1) - 1; lx[nx++] = 2; }
      if ((i >> 1) < b.mx) { ex[nx] = i >> 1; lx[nx++] = 0; }
    }
    if (j & 1) { ey[0] = j >> 1; ly[0] = 1; ny = 1; }
    else {
      if (j > 0) { ey[ny] = (j >> 1) - 1; ly[ny++] = 2; }
      if ((j >> 1) < b.my) { ey[ny] = j >> 1; ly[ny++] = 0; }
    }
    if (k & 1) { ez[0] = k >> 1; lz[0] = 1; nz = 1; }
    else {
      if (k > 0) { ez[nz] = (k >> 1) - 1; lz[nz++] = 2; }
      if ((k >> 1) < b.mz) { ez[nz] = k >> 1; lz[nz++] = 0; }
    }
    double acc = 0.0;
    for (int c = 0; c < nz; c++)
      for (int bb = 0; bb < ny; bb++)
        for (int a = 0; a < nx; a++) {
          const int64_t e = ex[a] + (int64_t)b.mx * (ey[bb] + (int64_t)b.my * ez[c]);
          const int jj = 3 * (lx[a] + 3 * ly[bb] + 9 * lz[c]) + l;
          acc += Ae[e * EBE_LD + ebe_sym(jj, jj)];
        }
    d[t] = acc;
  }
}

}  // namespace ptk
