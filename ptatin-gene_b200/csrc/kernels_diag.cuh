// Streaming diag(A11) kernel: the diagonal from the stored Gauss-point factor
// K, on the streaming A11 kernel's tiles.
//
// Same decomposition as the A11 apply (kernels_stream.cuh): a CTA owns TX
// consecutive elements of one element row (one thread each) and marches over
// a z-chunk of layers; the three node planes of the output live in shared
// memory and are flushed once, by colour-ordered launches (first toucher
// stores, later colours red.add), so each node's sum is formed in a fixed
// order and the result is bitwise repeatable.  There is no input vector, so
// there are no u planes and no mask: per quadrature plane and velocity
// component m the thread reads row m of K at the plane's 9 points and forms
// Q_m of q2::diag_form_plane; component m of its 27 nodes gets Q_m and every
// component gets S = sum_m Q_m (diag(n, l) = Q_l(n) + S(n)).
//
// The reference's diagonal (src/stokes_operators.c:1072-1113 ->
// src/stokes_q2p1_mf_operators_diag_def.c:120-205) recomputes the Jacobian and
// sums w det eta (|grad N_n|^2 + (dN_n/dx_l)^2) point by node.
#pragma once

#include "kernels_stream.cuh"

namespace ptk {

// zeta factors of Gauss plane A: [A][BB, EB, EE][node plane k]
__constant__ double c_zdiag[3][3][3] = {
    {{q2::dg::bb(0, 0), q2::dg::bb(0, 1), q2::dg::bb(0, 2)},
     {q2::dg::eb(0, 0), q2::dg::eb(0, 1), q2::dg::eb(0, 2)},
     {q2::dg::ee(0, 0), q2::dg::ee(0, 1), q2::dg::ee(0, 2)}},
    {{q2::dg::bb(1, 0), q2::dg::bb(1, 1), q2::dg::bb(1, 2)},
     {q2::dg::eb(1, 0), q2::dg::eb(1, 1), q2::dg::eb(1, 2)},
     {q2::dg::ee(1, 0), q2::dg::ee(1, 1), q2::dg::ee(1, 2)}},
    {{q2::dg::bb(2, 0), q2::dg::bb(2, 1), q2::dg::bb(2, 2)},
     {q2::dg::eb(2, 0), q2::dg::eb(2, 1), q2::dg::eb(2, 2)},
     {q2::dg::ee(2, 0), q2::dg::ee(2, 1), q2::dg::ee(2, 2)}}};

template <int TX>
constexpr size_t diag_smem_bytes()
{
  using L = TileLayout<TX>;
  return sizeof(double) * ((size_t)L::TILE + L::SIDE);
}

// One element (thread t), quadrature plane A: Q_m for m = 0..2 into the
// tile, then S.  Ke points at K(row, q = 0, r = 0, ex).
template <int TX, bool KTX>
__device__ __forceinline__ void diag_element_plane(int A, double *yt, double *side, const int sl[3], int t, int warp,
                                                   bool to_side, unsigned amask, const double *__restrict__ Ke,
                                                   int64_t MXP_)
{
  const int64_t MXP = KTX ? (int64_t)TX : MXP_;
  double z[3][3];
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int k = 0; k < 3; k++) z[s][k] = c_zdiag[A][s][k];
  const double *kp = Ke + (int64_t)(9 * A) * 9 * MXP;
  double S[27];
#pragma unroll 1
  for (int m = 0; m < 3; m++) {
    const double *km = kp + (int64_t)(3 * m) * MXP;
    double Q[27];
    q2::diag_form_plane<double>([&](int p, int d) { return ldk(km + (int64_t)(9 * p + d) * MXP); }, z, Q);
    if (m == 0) {
#pragma unroll
      for (int n = 0; n < 27; n++) S[n] = Q[n];
    } else {
#pragma unroll
      for (int n = 0; n < 27; n++) S[n] += Q[n];
    }
    tile_add_nodes<double, TX>(yt, side, sl, t, warp, to_side, amask, m, Q);
  }
#pragma unroll 1
  for (int l = 0; l < 3; l++) tile_add_nodes<double, TX>(yt, side, sl, t, warp, to_side, amask, l, S);
}

// One tile (x-tile tx, row ej, z-chunk zc); the whole CTA.
template <int TX, bool KTX>
__device__ __forceinline__ void diag_tile(const StreamGrid &g, int tx, int ej, int zc, const double *__restrict__ K,
                                          double *__restrict__ y)
{
  const int64_t MXP = KTX ? (int64_t)TX : g.MXP;
  using L = TileLayout<TX>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *yt = reinterpret_cast<double *>(smem_raw);
  double *side = yt + L::TILE;
  const int ex0 = tx * TX;
  // programmatic dependent launch, as in the A11 kernel: a later colour may
  // start on the SMs this grid frees and waits before its first flush
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int ex = ex0 + t;
  const bool active = ex < g.b.mx;
  const int ek0 = zc * g.LZ, ek1 = min(ek0 + g.LZ, g.b.mz);
  const bool zlo_shared = zc > 0, zhi_shared = ek1 < g.b.mz;

  for (int k = 0; k < 3; k++) zero_slot<double, TX>(yt, side, (int)((2 * (int64_t)ek0 + k) % 3));
  __syncthreads();

  const bool to_side = (lane == 31) && (warp < L::NW - 1);
  const unsigned amask = __ballot_sync(0xffffffffu, active);
  if (t == 0) prefetch_k_plane(K + kidx(ej + (int64_t)g.b.my * ek0, 0, 0, MXP, 0), (uint32_t)(sizeof(double) * 81 * MXP));

#pragma unroll 1
  for (int ek = ek0; ek < ek1; ek++) {
    const int64_t row = ej + (int64_t)g.b.my * ek;
    const int s0 = (int)((2 * (int64_t)ek) % 3), s1 = (s0 + 1) % 3, s2 = (s0 + 2) % 3;
    const int sl[3] = {s0, s1, s2};
    const bool more = ek + 1 < ek1;
    if (active) {
      const int64_t krow = kidx(row, 0, 0, MXP, ex);
      const uint32_t kb = (uint32_t)(sizeof(double) * 81 * MXP);
#pragma unroll 1
      for (int A = 0; A < 3; A++) {
        if (t == 0 && (A < 2 || more))
          prefetch_k_plane(A < 2 ? K + kidx(row, 9 * (A + 1), 0, MXP, 0) : K + kidx(row + g.b.my, 0, 0, MXP, 0), kb);
        diag_element_plane<TX, KTX>(A, yt, side, sl, t, warp, to_side, amask, K + krow, MXP);
      }
    }
    __syncthreads();
    if (ek == ek0) asm volatile("griddepcontrol.wait;" ::: "memory");
    flush_plane<double, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek, s0, ek == ek0 && zlo_shared, y);
    flush_plane<double, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek + 1, s1, false, y);
    if (!more) flush_plane<double, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek + 2, s2, zhi_shared, y);
    // the flushed slots (zeroed as read) take the next layer's sums
    if (more) __syncthreads();
  }
}

// Resident CTAs per SM the register budget is sized for: 256 threads per SM
// (230 registers, no spill).  Measured at 128^3 with the batched tile adds:
// 1.44 ms against 1.63 ms at 384 threads per SM (168 registers, a small
// spill); before the adds were batched, 1.93 ms against 2.39 ms, and 2.53 ms
// for a form without S in registers (Q_m added to all three components, 128
// registers, 384 threads per SM, three times the shared-memory adds).
template <int TX>
constexpr int diag_min_blocks()
{
  return 256 / TX;
}

template <int TX, bool KTX>
__global__ void __launch_bounds__(TX, diag_min_blocks<TX>()) diag_stream_kernel(StreamGrid g, const double *__restrict__ K,
                                                                               double *__restrict__ y)
{
  const int bid = blockIdx.x;
  const int ixc = bid % g.nxc, iyc = (bid / g.nxc) % g.nyc, izc = bid / (g.nxc * g.nyc);
  diag_tile<TX, KTX>(g, g.px + 2 * ixc, g.py + 2 * iyc, g.zc0 + 2 * izc, K, y);
}

}  // namespace ptk
