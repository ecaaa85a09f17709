// Streaming A11 kernel, TMEM revision ("b200" for rows of 65..128 elements).
//
// Same algorithm and tiling as a11_stream_kernel (kernels_stream.cuh) with two
// changes aimed at its measured bottleneck (one Gauss point of K lookahead,
// two warps per scheduler, long-scoreboard stalls):
//
//  * the element's 81 output values per node plane triple live in tensor memory
//    (TMEM), private to the thread: 3 node-plane slots x 27 values, 162 32-bit
//    columns of the thread's TMEM lane.  Accumulation is tcgen05.ld / add /
//    tcgen05.st, the shared y tile is gone, and at the end of a layer each
//    thread hands its i=2 node column to its right neighbour (warp shuffle;
//    shared memory across warps) before writing its own columns to global y;
//  * the freed shared memory holds a 4-deep per-thread ring of the Gauss-point
//    factor K filled with cp.async (the asynchronous global->shared copy), so
//    the K of a point is requested three points before it is needed.
//
// TMEM: each CTA (4 warps, warp w on lane quarter w) allocates 256 columns;
// the shared-memory footprint allows at most two CTAs per SM, so 512 columns
// always suffice and tcgen05.alloc never waits on a third CTA.  The waits used
// are the hardware ones (tcgen05.wait::ld/st, cp.async.wait_group); there is no
// software spin.
#pragma once

#include <cstdint>

#include "kernels_stream.cuh"

namespace ptk {

constexpr int TM_TX = 128;   // elements (threads) per CTA
constexpr int TM_KD = 4;     // K ring depth (Gauss points in flight)
constexpr int TM_COLS = 256; // TMEM columns allocated per CTA

// TMEM column of y-accumulator value (slot s, comp l, row j, col i): one
// double = 2 columns.
__device__ __forceinline__ uint32_t ycol(int s, int l, int j, int i) { return (uint32_t)((s * 27 + l * 9 + j * 3 + i) * 2); }

__device__ __forceinline__ void tm_st2(uint32_t a, double v)
{
  const unsigned long long b = __double_as_longlong(v);
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a), "r"((uint32_t)b),
               "r"((uint32_t)(b >> 32)));
}

__device__ __forceinline__ double tm_ld2(uint32_t a)
{
  uint32_t lo, hi;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "r"(a));
  return __longlong_as_double(((unsigned long long)hi << 32) | lo);
}

// nine consecutive doubles (18 columns) as x16 + x2
__device__ __forceinline__ void tm_ld9(uint32_t a, double v[9])
{
  uint32_t r[18];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(a));
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[16]), "=r"(r[17]) : "r"(a + 16));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 9; k++) v[k] = __longlong_as_double(((unsigned long long)r[2 * k + 1] << 32) | r[2 * k]);
}

__device__ __forceinline__ void tm_st9(uint32_t a, const double v[9])
{
  uint32_t r[18];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const unsigned long long b = __double_as_longlong(v[k]);
    r[2 * k] = (uint32_t)b;
    r[2 * k + 1] = (uint32_t)(b >> 32);
  }
  asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
               ::"r"(a), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
                 "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]),
                 "r"(r[16])
               : "memory");
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a + 16), "r"(r[16]), "r"(r[17]) : "memory");
}

__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 8-byte asynchronous global -> shared copy
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

struct TmLayout {
  using L = TileLayout<TM_TX>;
  static constexpr int UT = L::TILE;                 // u tile doubles
  static constexpr int KR = TM_KD * 9 * TM_TX;       // K ring doubles: [stage][r][t]
  static constexpr int SIDE = (TM_TX / 32) * 27;     // i=2 column of lane 31 per warp: [w][slot][comp][row]
};

constexpr size_t tmem_smem_bytes() { return sizeof(double) * (TmLayout::UT + TmLayout::KR + TmLayout::SIDE) + 16; }

// Issue the 9 K values of this thread's Gauss point g (g = layer offset * 27 + q)
// into ring stage g % TM_KD and commit one cp.async group (empty when idle).
__device__ __forceinline__ void tm_issue_k(double *kring, const double *__restrict__ K, const StreamGrid &g, int ej,
                                           int ek0, int ex, int t, int gq, int gq_end, bool active)
{
  if (active && gq < gq_end) {
    const int ek = ek0 + gq / 27, q = gq % 27;
    const double *src = K + kidx(ej + (int64_t)g.b.my * ek, q, 0, g.MXP, ex);
    double *dst = kring + (gq % TM_KD) * 9 * TM_TX + t;
#pragma unroll
    for (int r = 0; r < 9; r++) cp_async8(dst + r * TM_TX, src + (int64_t)r * g.MXP);
  }
  cp_async_commit();
}

// One element, quadrature plane A of the layer whose first Gauss point has
// chunk index gl (= (ek - ek0) * 27).
// Inactive threads (past the row's last element) run the same instruction
// stream -- tcgen05.ld/st are warp-collective -- but add zero.
template <int A>
__device__ __forceinline__ void tm_element_plane(const double *ut, double *kring, const int sl[3], int t,
                                                 uint32_t tlane, const double *__restrict__ K, const StreamGrid &g,
                                                 int ej, int ek0, int ex, int gl, int gq_end, bool active)
{
  using L = TileLayout<TM_TX>;
  double G[3][3][9];
#pragma unroll
  for (int l = 0; l < 3; l++) {
    double Q[9], R[9];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int n = 2 * t + i;
        q2::zeta_fwd<double, A>(ut[L::at(l, sl[0], j, n)], ut[L::at(l, sl[1], j, n)], ut[L::at(l, sl[2], j, n)],
                                Q[3 * j + i], R[3 * j + i]);
      }
    q2::plane_fwd(Q, R, G[0][l], G[1][l], G[2][l]);
  }
#pragma unroll
  for (int p = 0; p < 9; p++) {
    const int gq = gl + 9 * A + p;
    tm_issue_k(kring, K, g, ej, ek0, ex, t, gq + TM_KD - 1, gq_end, active);
    cp_async_wait<TM_KD - 1>();
    double Kq[9];
#pragma unroll
    for (int r = 0; r < 9; r++) Kq[r] = kring[((gq % TM_KD) * 9 + r) * TM_TX + t];
    q2::qp_action_K(Kq, G, p);
  }
#pragma unroll
  for (int l = 0; l < 3; l++) {
    double Qt[9], Rt[9];
    q2::plane_bwd(G[0][l], G[1][l], G[2][l], Qt, Rt);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      double acc[9];
      tm_ld9(tlane + ycol(sl[k], l, 0, 0), acc);
#pragma unroll
      for (int ji = 0; ji < 9; ji++) {
        double c0, c1, c2;
        q2::zeta_bwd<double, A>(Qt[ji], Rt[ji], c0, c1, c2);
        const double c = (k == 0 ? c0 : (k == 1 ? c1 : c2));
        acc[ji] += active ? c : 0.0;
      }
      tm_st9(tlane + ycol(sl[k], l, 0, 0), acc);
    }
  }
  tm_wait_st();
}

// Write node plane slot s of this thread's columns to global y: node 2t
// (own i=0 plus the left neighbour's i=2) and 2t+1, and for the tile's last
// thread the right edge 2*TM_TX.  v[l][j][i] are the thread's 27 values, inl
// the left neighbour's i=2 column [l][j].
template <bool MASKED>
__device__ __forceinline__ void tm_write_plane(const StreamGrid &g, int tx, int ex0, int ej, int64_t P, bool zshared,
                                               int t, int nact, const double v[3][3][3], const double inl[3][3],
                                               double *__restrict__ y, const double *__restrict__ x,
                                               const uint8_t *__restrict__ mask)
{
  const bool xlo = tx > 0, xhi = ex0 + TM_TX < g.b.mx;
  const bool ylo = ej > 0, yhi = ej < g.b.my - 1;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int64_t node0 = g.b.off + 2 * (int64_t)ex0 + (2 * (int64_t)ej + j) * g.b.X + P * g.b.XY;
    const bool yb = (j == 0 && ylo) || (j == 2 && yhi);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      // (local node, value) pairs this thread writes
      const int nn[3] = {2 * t, 2 * t + 1, 2 * TM_TX};
      const double vv[3] = {v[c][j][0] + inl[c][j], v[c][j][1], v[c][j][2]};
      const bool doit[3] = {t <= nact, t < nact, t == TM_TX - 1 && nact == TM_TX};
#pragma unroll
      for (int w = 0; w < 3; w++) {
        if (!doit[w]) continue;
        const int n = nn[w];
        const int64_t k = 3 * (node0 + n) + c;
        if (MASKED && mask[k]) {
          y[k] = x[k];
          continue;
        }
        const bool xb = (n == 0 && xlo) || (n == 2 * TM_TX && xhi);
        const bool first = !((xb && g.px) || (yb && g.py) || (zshared && g.pz));
        if (first) y[k] = vv[w];
        else y[k] = y[k] + vv[w];
      }
    }
  }
}

template <bool MASKED>
__global__ void __launch_bounds__(TM_TX, 2) a11_tmem_kernel(StreamGrid g, const double *__restrict__ K,
                                                           const double *__restrict__ u,
                                                           const uint8_t *__restrict__ mask, double *__restrict__ y)
{
  using L = TileLayout<TM_TX>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *ut = reinterpret_cast<double *>(smem_raw);
  double *kring = ut + TmLayout::UT;
  double *side = kring + TmLayout::KR;
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(side + TmLayout::SIDE);

  const int bid = blockIdx.x;
  const int ixc = bid % g.nxc, iyc = (bid / g.nxc) % g.nyc, izc = bid / (g.nxc * g.nyc);
  const int tx = g.px + 2 * ixc, ej = g.py + 2 * iyc, zc = g.zc0 + 2 * izc;
  const int ex0 = tx * TM_TX;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int ex = ex0 + t;
  const int nact = min(TM_TX, g.b.mx - ex0);
  const bool active = t < nact;
  const int ek0 = zc * g.LZ, ek1 = min(ek0 + g.LZ, g.b.mz);
  const bool zlo_shared = zc > 0, zhi_shared = ek1 < g.b.mz;
  const int gq_end = (ek1 - ek0) * 27;

  // TMEM: 256 columns for the CTA; warp w owns lanes 32w..32w+31
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(taddr_s)), "r"(TM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // u planes of the first layer; K points 0 .. KD-2 in flight
  for (int k = 0; k < 3; k++) {
    const int64_t P = 2 * (int64_t)ek0 + k;
    load_plane<double, TM_TX, MASKED>(ut, g, ex0, ej, P, (int)(P % 3), u, mask);
  }
  for (int gq = 0; gq < TM_KD - 1; gq++) tm_issue_k(kring, K, g, ej, ek0, ex, t, gq, gq_end, active);
  if (t == 0) prefetch_k_plane(K + kidx(ej + (int64_t)g.b.my * ek0, 0, 0, g.MXP, 0), (uint32_t)(sizeof(double) * 81 * g.MXP));
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tlane = *taddr_s + ((uint32_t)(32 * warp) << 16);
  // zero the three accumulator slots
  {
    const double z9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
      for (int l = 0; l < 3; l++) tm_st9(tlane + ycol(s, l, 0, 0), z9);
    tm_wait_st();
  }

#pragma unroll 1
  for (int ek = ek0; ek < ek1; ek++) {
    const int64_t row = ej + (int64_t)g.b.my * ek;
    const int s0 = (int)((2 * (int64_t)ek) % 3), s1 = (s0 + 1) % 3, s2 = (s0 + 2) % 3;
    const int sl[3] = {s0, s1, s2};
    const int gl = (ek - ek0) * 27;

    // inactive threads run the same sequence (their K copies are empty and
    // their accumulators stay zero) so that tcgen05 collectives stay warp-uniform
    tm_element_plane<0>(ut, kring, sl, t, tlane, K, g, ej, ek0, ex, gl, gq_end, active);
    if (t == 0) prefetch_k_plane(K + kidx(row, 18, 0, g.MXP, 0), (uint32_t)(sizeof(double) * 81 * g.MXP));
    tm_element_plane<1>(ut, kring, sl, t, tlane, K, g, ej, ek0, ex, gl, gq_end, active);
    if (t == 0 && ek + 1 < ek1)
      prefetch_k_plane(K + kidx(row + g.b.my, 0, 0, g.MXP, 0), (uint32_t)(sizeof(double) * 81 * g.MXP));
    tm_element_plane<2>(ut, kring, sl, t, tlane, K, g, ej, ek0, ex, gl, gq_end, active);

    // ---- flush node planes 2ek, 2ek+1 (and 2ek+2 at the chunk's end)
    const bool last = ek + 1 == ek1;
    const int nfl = last ? 3 : 2;
    // i=2 node columns first: they go to the right neighbour
    double i2[3][3][3];  // [slot k][comp][row]
#pragma unroll
    for (int k = 0; k < 3; k++)
      if (k < nfl)
#pragma unroll
        for (int l = 0; l < 3; l++)
#pragma unroll
          for (int j = 0; j < 3; j++) i2[k][l][j] = tm_ld2(tlane + ycol(sl[k], l, j, 2));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (lane == 31) {
#pragma unroll
      for (int k = 0; k < 3; k++)
        if (k < nfl)
#pragma unroll
          for (int l = 0; l < 3; l++)
#pragma unroll
            for (int j = 0; j < 3; j++) side[warp * 27 + k * 9 + l * 3 + j] = i2[k][l][j];
    }
    __syncthreads();  // side buffer written; every thread is done with the u tile
    if (!last) {
      load_plane<double, TM_TX, MASKED>(ut, g, ex0, ej, 2 * (int64_t)ek + 3, s0, u, mask);
      load_plane<double, TM_TX, MASKED>(ut, g, ex0, ej, 2 * (int64_t)ek + 4, s1, u, mask);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (k < nfl) {
        double vk[3][3][3];  // [comp][row][col]
#pragma unroll
        for (int l = 0; l < 3; l++) {
          double a9[9];
          tm_ld9(tlane + ycol(sl[k], l, 0, 0), a9);
#pragma unroll
          for (int ji = 0; ji < 9; ji++) vk[l][ji / 3][ji % 3] = a9[ji];
        }
        double inl[3][3];
#pragma unroll
        for (int l = 0; l < 3; l++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            const double up = __shfl_up_sync(0xffffffffu, i2[k][l][j], 1);
            inl[l][j] = lane > 0 ? up : (warp > 0 ? side[(warp - 1) * 27 + k * 9 + l * 3 + j] : 0.0);
          }
        const int64_t P = 2 * (int64_t)ek + k;
        const bool zsh = (k == 0 && ek == ek0 && zlo_shared) || (k == 2 && zhi_shared);
        tm_write_plane<MASKED>(g, tx, ex0, ej, P, zsh, t, nact, vk, inl, y, u, mask);
      }
    }
    if (!last) {
      const double z9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int l = 0; l < 3; l++) {
        tm_st9(tlane + ycol(s0, l, 0, 0), z9);
        tm_st9(tlane + ycol(s1, l, 0, 0), z9);
      }
      tm_wait_st();
    }
    __syncthreads();  // next layer's u planes are in place; side buffer free
  }

  cp_async_wait<0>();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*taddr_s), "r"(TM_COLS));
}

}  // namespace ptk
