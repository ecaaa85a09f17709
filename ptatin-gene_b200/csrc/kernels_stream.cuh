// Streaming A11 kernel ("b200"): precomputed quadrature-point geometry,
// z-marching tiles staged in shared memory, deterministic colour-ordered
// flushes.
//
// Geometry.  At set-up (coordinates or viscosity change) one kernel stores,
// per element and Gauss point,
//     K = h * sqrt(c) * adj(J),   c = w * eta / det(J),   h = 1/(2 sqrt(3/5)),
// nine values.  With A = K Gu' (Gu' = h^-1 d u/d xi, the scaled reference
// gradient computed below) the viscous action is dv' = (A + A^T) K, which
// equals h^-1 * w*det*(2 eta sym(grad u)) J^-T of the reference
// (src/stokes_operators_tensor.c:127-179) -- the scales cancel against the
// scaled transpose contractions.  The apply therefore reads K instead of
// coordinates + eta and does no Jacobian work.  c must be > 0 (valid,
// positively oriented elements and positive viscosity); the op falls back to
// the 8-colour kernel otherwise.
//
// Work decomposition.  A CTA owns TX consecutive elements along x (one
// thread each) of one element row (ej) and marches over a chunk of LZ element
// layers in z.  Per layer it holds three node planes of u and of y in shared
// memory (component-planar, even/odd node split so a warp's 32 elements read
// consecutive words), computes each element quadrature plane by quadrature
// plane (the live state is one plane's 3x3 velocity gradient, 81 values), and
// accumulates the transposed contractions into the y planes.  Within a warp
// the shared node column of neighbouring elements is updated in program
// order with a __syncwarp between the i=0 and i=2 passes; the column shared
// between two warps goes to a per-warp side buffer.  Completed node planes
// are flushed to global y once.
//
// Data movement.  A layer's two new node planes of u are fetched with
// cp.async (no registers) into the u slots the finished layer frees, while
// that layer's completed y planes are flushed; their rows are prefetched to
// L2 one layer ahead, and each quadrature plane of K one plane ahead.  The
// MatShell apply's Dirichlet columns come from a packed bit mask whose words
// are fetched with the plane and applied in shared memory; its Dirichlet rows
// are set by a separate pass after the colour launches.
//
// Determinism across CTAs.  Tiles are coloured by the parity of their x-tile,
// row and z-chunk index; colours run as separate launches in a fixed order.
// A node on a tile boundary is stored by the first colour that touches it and
// added to by the later ones (red.global.add: no read-back).  Each launch
// touches a node from one CTA only and the launches are ordered, so every
// node's sum is formed in a fixed order: the result is bitwise the same run
// after run, and the same as a read-modify-write.
#pragma once

#include <cstdint>

#include "kernels_colour.cuh"
#include "q2_core.cuh"
#include "q2_plane.cuh"

namespace ptk {

struct StreamGrid {
  Box b;
  int TX, ntx;        // elements per tile along x, tiles along x
  int LZ, nzc;        // layers per z-chunk, z-chunks
  int px, py, pz;     // colour of this launch
  int nxc, nyc, nzcc; // tiles of this colour per axis
  int zc0;            // first z-chunk of this launch (parity pz; pz for a whole-box launch)
  int64_t MXP;        // padded row length of the K array (elements)
};

// K index: ((row*27 + q)*9 + r)*MXP + ex,  row = ej + my*ek.
__host__ __device__ __forceinline__ int64_t kidx(int64_t row, int q, int r, int64_t MXP, int ex)
{
  return ((row * 27 + q) * 9 + r) * MXP + ex;
}

// ---------------------------------------------------------------------------
// Set-up kernel: K for every element and Gauss point.  Returns through
// *bad the number of points with c <= 0 or non-finite c.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) geom_kernel(Box bx, int64_t MXP, const double *__restrict__ coords,
                                                   const double *__restrict__ eta, T *__restrict__ K,
                                                   unsigned int *__restrict__ bad)
{
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)bx.mx * bx.my * bx.mz) return;
  const int ei = (int)(e % bx.mx);
  const int64_t row = e / bx.mx;
  const int ej = (int)(row % bx.my), ek = (int)(row / bx.my);
  int64_t nid[27];
  element_nodes(bx, ei, ej, ek, nid);
  double Jg[3][3][27], Xq[3][27];
  element_jacobian(coords, nid, Jg, Xq);
  unsigned nbad = 0;
#pragma unroll 1
  for (int q = 0; q < 27; q++) {
    double J[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int l = 0; l < 3; l++) J[k][l] = Jg[k][l][q];
    T Kq[9];
    if (!q2::geom_K(J, q2::weight(q) * eta[27 * e + q], Kq)) nbad++;
#pragma unroll
    for (int r = 0; r < 9; r++) K[kidx(row, q, r, MXP, ei)] = Kq[r];
  }
  if (nbad) atomicAdd(bad, nbad);
}

// Bulk L2 prefetch (TMA unit) of a contiguous K block, in pieces of at most
// 32 KiB; addresses and sizes are multiples of 16 bytes (MXP is a multiple
// of 32 elements).
__device__ __forceinline__ void prefetch_k_plane(const void *p, uint32_t bytes)
{
  const char *c = reinterpret_cast<const char *>(p);
  for (uint32_t off = 0; off < bytes; off += 32768u) {
    const uint32_t n = min(32768u, bytes - off);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + off), "r"(n) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Shared-memory tile
// ---------------------------------------------------------------------------
// Node planes are indexed by slot s = p % 3 (p = absolute node-plane index in
// the chunk, 2*layer + k).  One plane-row of one component holds the tile's
// 2TX+1 nodes split even/odd: node 2m -> m, node 2m+1 -> TX+1+m.
template <int TX>
struct TileLayout {
  static constexpr int NXN = 2 * TX + 1;
  static constexpr int ROW = NXN;              // one (comp, slot, row)
  static constexpr int PLANE = 3 * ROW;        // 3 rows
  // 3 slots, plus 2 values of padding: the plane fetch and flush walk the
  // global (node, component) order, and without it the three components of
  // neighbouring nodes fall in the same shared-memory banks (FP64: 3.9 -> 2.6
  // wavefronts per warp access by the bank model; 128^3 MatMult 1.581 ->
  // 1.560 ms).  The compute phase reads consecutive positions either way.
  static constexpr int COMP = 3 * PLANE + 2;
  static constexpr int TILE = 3 * COMP;        // 3 components
  static constexpr int NW = TX / 32;
  // side buffer: the i=2 column of lane 31 of warps 0..NW-2: [w][slot][row][comp]
  static constexpr int SIDE = (NW > 1 ? NW - 1 : 1) * 27;
  __host__ __device__ static constexpr int pos(int n) { return (n & 1) ? (TX + 1 + (n >> 1)) : (n >> 1); }
  __host__ __device__ static constexpr int at(int comp, int slot, int row, int n)
  {
    return comp * COMP + slot * PLANE + row * ROW + pos(n);
  }
};

// Dirichlet bits of the tile's node planes: per slot and plane row, the
// 32-bit words of the packed mask (bit k = dof k of the local vector) that
// cover the row's <= 3*(2TX+1) dofs, which start anywhere in a word.
template <int TX>
__host__ __device__ constexpr int mask_row_words() { return (3 * (2 * TX + 1) + 31) / 32 + 1; }

template <typename T, int TX>
constexpr size_t stream_smem_bytes()
{
  using L = TileLayout<TX>;
  return sizeof(T) * (2 * (size_t)L::TILE + L::SIDE) + sizeof(uint32_t) * 9 * mask_row_words<TX>();
}

// First node of plane-row r of node plane P in the tile starting at element
// ex0 of row ej.
__device__ __forceinline__ int64_t row_node0(const StreamGrid &g, int ex0, int ej, int r, int64_t P)
{
  return g.b.off + 2 * (int64_t)ex0 + (2 * (int64_t)ej + r) * g.b.X + P * g.b.XY;
}

// Copies the words of the packed Dirichlet mask that cover the three rows of
// node plane P into the slot's mask words (asynchronous 4-byte copies).
template <int TX>
__device__ __forceinline__ void stage_mask(uint32_t *mw, const StreamGrid &g, int ex0, int ej, int64_t P, int s,
                                           const uint32_t *__restrict__ mbits)
{
  using L = TileLayout<TX>;
  const int nd = 3 * min(L::NXN, 2 * (g.b.mx - ex0) + 1);
#pragma unroll 1
  for (int r = 0; r < 3; r++) {
    const int64_t k0 = 3 * row_node0(g, ex0, ej, r, P);
    const int64_t w0 = k0 >> 5;
    const int nw = (int)(((k0 + nd - 1) >> 5) - w0 + 1);
    if ((int)threadIdx.x < nw) {
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&mw[(s * 3 + r) * mask_row_words<TX>() + threadIdx.x]);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(mbits + w0 + threadIdx.x) : "memory");
    }
  }
}

// Fetches node plane P (rows 0..2) of u into slot s with asynchronous 4- or
// 8-byte copies straight into the component-planar tile (cp.async: no
// registers, the copies run while the thread flushes y).  MASKED: the
// Dirichlet entries, whose bits the slot's staged mask words hold (visible to
// every thread), are written as zeros instead -- the MatShell apply's column
// rule.  The caller commits and waits.
template <typename T, int TX, bool MASKED>
__device__ __forceinline__ void fetch_plane(T *ut, const uint32_t *mw, const StreamGrid &g, int ex0, int ej, int64_t P,
                                            int s, const T *__restrict__ u, bool mk)
{
  using L = TileLayout<TX>;
  const int nd = 3 * min(L::NXN, 2 * (g.b.mx - ex0) + 1);
#pragma unroll 1
  for (int r = 0; r < 3; r++) {
    const int64_t k0 = 3 * row_node0(g, ex0, ej, r, P);
    const T *src = u + k0;
    const uint32_t *w = mw + (s * 3 + r) * mask_row_words<TX>();
    const int b0 = (int)(k0 & 31);
    for (int d = threadIdx.x; d < nd; d += TX) {
      const int n = d / 3, c = d - 3 * n;
      T *dst = &ut[L::at(c, s, r, n)];
      if (MASKED && mk) {
        const int pos = b0 + d;
        if ((w[pos >> 5] >> (pos & 31)) & 1u) {
          *dst = T(0);
          continue;
        }
      }
      const uint32_t sd = (uint32_t)__cvta_generic_to_shared(dst);
      if (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sd), "l"(src + d) : "memory");
      else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sd), "l"(src + d) : "memory");
    }
  }
}

__device__ __forceinline__ void fetch_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void fetch_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// L2 prefetch (TMA unit, no registers) of the u rows of node plane P, each
// row segment rounded out to 16-byte boundaries inside the array of nu values.
template <typename T, int TX>
__device__ __forceinline__ void prefetch_u_plane(const StreamGrid &g, int ex0, int ej, int64_t P, const T *u,
                                                 int64_t nu)
{
  using L = TileLayout<TX>;
  const int nd = 3 * min(L::NXN, 2 * (g.b.mx - ex0) + 1);
  for (int r = 0; r < 3; r++) {
    const int64_t k0 = 3 * row_node0(g, ex0, ej, r, P);
    const uintptr_t a = (uintptr_t)(u + k0) & ~(uintptr_t)15;
    const uintptr_t e = (uintptr_t)(u + min(k0 + nd, nu)) & ~(uintptr_t)15;
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
  }
}

template <typename T, int TX>
__device__ __forceinline__ void zero_slot(T *yt, T *side, int s)
{
  using L = TileLayout<TX>;
  for (int i = threadIdx.x; i < 3 * L::PLANE; i += TX) {
    const int c = i / L::PLANE, rest = i - c * L::PLANE;
    yt[c * L::COMP + s * L::PLANE + rest] = T(0);
  }
  for (int i = threadIdx.x; i < (L::NW > 1 ? L::NW - 1 : 0) * 9; i += TX) {
    const int w = i / 9, rc = i - 9 * w;
    side[w * 27 + s * 9 + rc] = T(0);
  }
}

// Flush node plane P (in slot s) to global y, zeroing each y-tile (and side
// buffer) entry as it is read, so the slot is ready for its next plane with
// no further pass or barrier.  zshared: the plane is the chunk's first/last
// plane and shared with a neighbouring chunk.  A node on a
// tile boundary is stored by the first colour that touches it and added to
// by the later ones; the colours are separate launches in a fixed order and
// a launch touches each node from one CTA only, so the adds (red.global.add,
// no read-back) happen in a fixed order: the sums are deterministic and equal
// to a read-modify-write.  Dirichlet rows are set after the colour passes.
template <typename T, int TX>
__device__ __forceinline__ void flush_plane(T *yt, T *side, const StreamGrid &g, int tx, int ex0, int ej, int64_t P,
                                            int s, bool zshared, T *__restrict__ y)
{
  using L = TileLayout<TX>;
  const int nvalid = min(L::NXN, 2 * (g.b.mx - ex0) + 1);
  const bool xlo = tx > 0, xhi = ex0 + TX < g.b.mx;
  const bool ylo = ej > 0, yhi = ej < g.b.my - 1;
  const int nd = 3 * nvalid;
#pragma unroll 1
  for (int r = 0; r < 3; r++) {
    const int64_t node0 = row_node0(g, ex0, ej, r, P);
    const bool yb = (r == 0 && ylo) || (r == 2 && yhi);
    for (int d = threadIdx.x; d < nd; d += TX) {
      const int n = d / 3, c = d - 3 * n;
      T v = yt[L::at(c, s, r, n)];
      yt[L::at(c, s, r, n)] = T(0);
      if (L::NW > 1 && (n & 63) == 0 && n > 0 && n < 2 * TX) {
        T *sb = &side[((n >> 6) - 1) * 27 + s * 9 + r * 3 + c];
        v += *sb;
        *sb = T(0);
      }
      const int64_t k = 3 * node0 + d;
      const bool xb = (n == 0 && xlo) || (n == 2 * TX && xhi);
      const bool first = !((xb && g.px) || (yb && g.py) || (zshared && g.pz));
      if (first) y[k] = v;
      else atomicAdd(&y[k], v);
    }
  }
}

// zeta contraction and its transpose for Gauss plane A given at run time:
// rows A of B and D/h (q2_plane.cuh) from constant memory, so one copy of the
// plane code serves all three planes (three unrolled copies measured 6-11%
// slower: instruction fetch stalls).
__constant__ double c_zB[3][3] = {{q2::B0, q2::B1, q2::B2}, {0.0, 1.0, 0.0}, {q2::B2, q2::B1, q2::B0}};
__constant__ double c_zD[3][3] = {{q2::DZ00, q2::DZ01, q2::DZ02}, {-q2::GS, 0.0, q2::GS},
                                  {q2::DZ20, q2::DZ21, q2::DZ22}};

template <typename T>
__device__ __forceinline__ void zeta_fwd_rt(int A, T n0, T n1, T n2, T &q, T &r)
{
  q = T(c_zB[A][0]) * n0 + (T(c_zB[A][1]) * n1 + T(c_zB[A][2]) * n2);
  r = T(c_zD[A][0]) * n0 + (T(c_zD[A][1]) * n1 + T(c_zD[A][2]) * n2);
}

template <typename T>
__device__ __forceinline__ void zeta_bwd_rt(int A, T q, T r, T &c0, T &c1, T &c2)
{
  c0 = T(c_zB[A][0]) * q + T(c_zD[A][0]) * r;
  c1 = T(c_zB[A][1]) * q + T(c_zD[A][1]) * r;
  c2 = T(c_zB[A][2]) * q + T(c_zD[A][2]) * r;
}

// Adds V (27 node values [k*9 + j*3 + i]) to component l of thread t's nodes
// in the tile: node columns i = 0, 1, then (after the warp's other lanes)
// i = 2, whose column lane 31 of every warp but the last keeps in the side
// buffer, so a column shared by two elements is summed in a fixed order.
// Each group's entries are all read before any is written: the slots are
// runtime indices, so the compiler cannot tell the 18 (9) addresses apart and
// would otherwise wait out a shared-memory round trip per entry.
template <typename T, int TX>
__device__ __forceinline__ void tile_add_nodes(T *yt, T *side, const int sl[3], int t, int warp, bool to_side,
                                               unsigned amask, int l, const T V[27])
{
  using L = TileLayout<TX>;
  {
    T *b0 = yt + L::at(l, 0, 0, 2 * t), *b1 = yt + L::at(l, 0, 0, 2 * t + 1);
    T c[18];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        c[6 * k + 2 * j] = b0[sl[k] * L::PLANE + j * L::ROW];
        c[6 * k + 2 * j + 1] = b1[sl[k] * L::PLANE + j * L::ROW];
      }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        b0[sl[k] * L::PLANE + j * L::ROW] = c[6 * k + 2 * j] + V[9 * k + 3 * j];
        b1[sl[k] * L::PLANE + j * L::ROW] = c[6 * k + 2 * j + 1] + V[9 * k + 3 * j + 1];
      }
  }
  __syncwarp(amask);
  {
    // column i = 2: the next lane's i = 0 column, or the side buffer
    T *b2 = to_side ? side + warp * 27 + l : yt + L::at(l, 0, 0, 2 * t + 2);
    const int ss = to_side ? 9 : L::PLANE, rs = to_side ? 3 : L::ROW;
    T c[9];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int j = 0; j < 3; j++) c[3 * k + j] = b2[sl[k] * ss + j * rs];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int j = 0; j < 3; j++) b2[sl[k] * ss + j * rs] = c[3 * k + j] + V[9 * k + 3 * j + 2];
  }
  __syncwarp(amask);
}

// K is read once per apply.  FP64: loaded without allocating in L1 (beside
// 225 KB of tiles the L1 left is small and K lines evicted the rest; measured
// at 128^3: MatMult 1.566 -> 1.495 ms, diagonal 1.419 -> 1.387 ms).  FP32
// keeps the default load (0.955 vs 0.962 ms with the hint).
__device__ __forceinline__ double ldk(const double *p)
{
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ldk(const float *p) { return *p; }

// One element (thread t of the tile), quadrature plane A: forward from the u
// tile, viscous action with K, transpose accumulated into the y tile.  KTX:
// the K rows are one tile wide (MXP == TX), a compile-time stride whose
// offsets fold into the loads (measured 2% faster in FP64 at 128^3, bitwise
// the same result; no gain in FP32).
template <typename T, int TX, bool KTX>
__device__ __forceinline__ void element_plane(int A, const T *ut, T *yt, T *side, const int sl[3], int t, int warp,
                                              bool to_side, unsigned amask, const T *__restrict__ Ke, int64_t MXP_)
{
  const int64_t MXP = KTX ? (int64_t)TX : MXP_;
  using L = TileLayout<TX>;
  T G[3][3][9];  // [d][l][b*3+c]
#pragma unroll
  for (int l = 0; l < 3; l++) {
    T Q[9], R[9];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int n = 2 * t + i;
        zeta_fwd_rt<T>(A, ut[L::at(l, sl[0], j, n)], ut[L::at(l, sl[1], j, n)], ut[L::at(l, sl[2], j, n)],
                           Q[3 * j + i], R[3 * j + i]);
      }
    q2::plane_fwd(Q, R, G[0][l], G[1][l], G[2][l]);
  }

  // viscous action: K of the next two points is in flight while one computes
  // (measured at 128^3: FP64 2.18 -> 2.02 ms, FP32 1.20 -> 1.12 ms)
  constexpr bool DEEP = true;
  const T *kp = Ke + (int64_t)(9 * A) * 9 * MXP;
  T Kn[9], Kn2[9];
#pragma unroll
  for (int r = 0; r < 9; r++) Kn[r] = ldk(kp + (int64_t)r * MXP);
  if (DEEP) {
#pragma unroll
    for (int r = 0; r < 9; r++) Kn2[r] = ldk(kp + (int64_t)(9 + r) * MXP);
  }
#pragma unroll
  for (int p = 0; p < 9; p++) {
    T Kq[9];
#pragma unroll
    for (int r = 0; r < 9; r++) Kq[r] = Kn[r];
    if (DEEP) {
#pragma unroll
      for (int r = 0; r < 9; r++) Kn[r] = Kn2[r];
      if (p < 7) {
#pragma unroll
        for (int r = 0; r < 9; r++) Kn2[r] = ldk(kp + (int64_t)(9 * (p + 2) + r) * MXP);
      }
    } else if (p < 8) {
#pragma unroll
      for (int r = 0; r < 9; r++) Kn[r] = ldk(kp + (int64_t)(9 * (p + 1) + r) * MXP);
    }
    q2::qp_action_K(Kq, G, p);
  }

  // transpose, one component at a time; node columns i = 0, 1, 2 in order
#pragma unroll
  for (int l = 0; l < 3; l++) {
    T Qt[9], Rt[9];
    q2::plane_bwd(G[0][l], G[1][l], G[2][l], Qt, Rt);
    T C[27];  // [k*9 + j*3 + i]
#pragma unroll
    for (int ji = 0; ji < 9; ji++) zeta_bwd_rt<T>(A, Qt[ji], Rt[ji], C[ji], C[9 + ji], C[18 + ji]);
    tile_add_nodes<T, TX>(yt, side, sl, t, warp, to_side, amask, l, C);
  }
}

// ---------------------------------------------------------------------------
// The apply kernel
// ---------------------------------------------------------------------------
// One tile (x-tile tx, row ej, z-chunk zc) of one problem; the whole CTA.
// MASKED (and mbits non-null): Dirichlet columns of u zeroed from the packed
// mask mbits.  KTX: g.MXP == TX (one x-tile per row).
template <typename T, int TX, bool MASKED, bool KTX = false, bool NULLABLE = false>
__device__ __forceinline__ void stream_tile(const StreamGrid &g, int tx, int ej, int zc, const T *__restrict__ K,
                                            const T *__restrict__ u, const uint32_t *__restrict__ mbits,
                                            T *__restrict__ y)
{
  const int64_t MXP = KTX ? (int64_t)TX : g.MXP;
  using L = TileLayout<TX>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ut = reinterpret_cast<T *>(smem_raw);
  T *yt = ut + L::TILE;
  T *side = yt + L::TILE;
  uint32_t *mw = reinterpret_cast<uint32_t *>(side + L::SIDE);
  const int ex0 = tx * TX;
  // Programmatic dependent launch: once every CTA of this grid has started,
  // a grid launched after it with programmatic stream serialization may
  // begin on the SMs this grid frees (its prologue and first layer overlap
  // this grid's last wave); that grid waits below before writing y.  Both
  // instructions do nothing for an ordinary launch.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int ex = ex0 + t;
  const bool active = ex < g.b.mx;
  const int ek0 = zc * g.LZ, ek1 = min(ek0 + g.LZ, g.b.mz);
  const bool zlo_shared = zc > 0, zhi_shared = ek1 < g.b.mz;
  // u holds at least the node planes up to the element box's last one
  const int64_t nu = 3 * g.b.XY * (int64_t)(g.b.off / g.b.XY + 2 * (int64_t)g.b.mz + 1);

  // masked apply of a problem that has a mask (a batched apply mixes boxes
  // with and without one, NULLABLE: those get the plain apply and read no
  // mask; a single-op masked launch always has the packed bits)
  const bool mk = MASKED && (!NULLABLE || mbits != nullptr);

  // prologue: the Dirichlet words and then planes 2ek0 .. 2ek0+2 of u; zero y
  if (mk) {
    for (int k = 0; k < 3; k++) {
      const int64_t P = 2 * (int64_t)ek0 + k;
      stage_mask<TX>(mw, g, ex0, ej, P, (int)(P % 3), mbits);
    }
    fetch_commit();
    fetch_wait();
  }
  for (int k = 0; k < 3; k++) zero_slot<T, TX>(yt, side, (int)((2 * (int64_t)ek0 + k) % 3));
  __syncthreads();
  for (int k = 0; k < 3; k++) {
    const int64_t P = 2 * (int64_t)ek0 + k;
    fetch_plane<T, TX, MASKED>(ut, mw, g, ex0, ej, P, (int)(P % 3), u, mk);
  }
  fetch_commit();
  fetch_wait();
  __syncthreads();

  // the node column of a thread's i=2 nodes lives in the side buffer for
  // lane 31 of every warp but the last
  const bool to_side = (lane == 31) && (warp < L::NW - 1);
  const unsigned amask = __ballot_sync(0xffffffffu, active);
  if (t == 0) prefetch_k_plane(K + kidx(ej + (int64_t)g.b.my * ek0, 0, 0, MXP, 0), (uint32_t)(sizeof(T) * 81 * MXP));

#pragma unroll 1
  for (int ek = ek0; ek < ek1; ek++) {
    const int64_t row = ej + (int64_t)g.b.my * ek;
    const int s0 = (int)((2 * (int64_t)ek) % 3), s1 = (s0 + 1) % 3, s2 = (s0 + 2) % 3;
    const int sl[3] = {s0, s1, s2};
    const bool more = ek + 1 < ek1;
    if (more) {
      // the next layer's Dirichlet words land in the mask slots this layer no
      // longer needs, and its two new node planes go to L2, while it computes
      if (mk) {
        stage_mask<TX>(mw, g, ex0, ej, 2 * (int64_t)ek + 3, s0, mbits);
        stage_mask<TX>(mw, g, ex0, ej, 2 * (int64_t)ek + 4, s1, mbits);
        fetch_commit();
      }
      if (t == 32) {
        prefetch_u_plane<T, TX>(g, ex0, ej, 2 * (int64_t)ek + 3, u, nu);
        prefetch_u_plane<T, TX>(g, ex0, ej, 2 * (int64_t)ek + 4, u, nu);
      }
    }

    if (active) {
      // each quadrature plane's K is prefetched to L2 while the one before it computes
      const int64_t krow = kidx(row, 0, 0, MXP, ex);
      const uint32_t kb = (uint32_t)(sizeof(T) * 81 * MXP);
#pragma unroll 1
      for (int A = 0; A < 3; A++) {
        if (t == 0 && (A < 2 || more))
          prefetch_k_plane(A < 2 ? K + kidx(row, 9 * (A + 1), 0, MXP, 0) : K + kidx(row + g.b.my, 0, 0, MXP, 0), kb);
        element_plane<T, TX, KTX>(A, ut, yt, side, sl, t, warp, to_side, amask, K + krow, MXP);
      }
    }
    if (mk) fetch_wait();  // this thread's staged words
    __syncthreads();

    // u slots s0, s1 are free: node planes 2ek+3, 2ek+4 land there while
    // planes 2ek and 2ek+1 (complete for this CTA) are flushed and their y
    // slots zeroed for the next layer
    if (more) {
      fetch_plane<T, TX, MASKED>(ut, mw, g, ex0, ej, 2 * (int64_t)ek + 3, s0, u, mk);
      fetch_plane<T, TX, MASKED>(ut, mw, g, ex0, ej, 2 * (int64_t)ek + 4, s1, u, mk);
      fetch_commit();
    }
    // y is written from here on: the previous grid in the stream (an earlier
    // colour of this apply, when launched programmatically) must be complete
    // and its stores visible.  u, K and the mask bits are read before this
    // point, so a programmatic launch is only made where the previous grid
    // does not write them (the colours after the first of one apply).
    if (ek == ek0) asm volatile("griddepcontrol.wait;" ::: "memory");
    flush_plane<T, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek, s0, ek == ek0 && zlo_shared, y);
    flush_plane<T, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek + 1, s1, false, y);
    if (!more) flush_plane<T, TX>(yt, side, g, tx, ex0, ej, 2 * (int64_t)ek + 2, s2, zhi_shared, y);
    if (more) {
      fetch_wait();
      __syncthreads();
    }
  }
}

// Resident CTAs per SM the register budget is sized for.  FP64 keeps one
// quadrature plane's gradient (81 doubles) live: 256 threads per SM.  FP32
// rows of 128 elements fit 4 CTAs (512 threads, 128 registers, 4 x 55.8 KB
// of tiles) -- measured 1.34x faster than 2 CTAs at 128^3; narrower FP32
// tiles measured best at 256 threads per SM.
template <typename T, int TX>
constexpr int stream_min_blocks()
{
  return (sizeof(T) == 4 && TX == 128) ? 4 : 256 / TX;
}

template <typename T, int TX, bool MASKED, bool KTX = false>
__global__ void __launch_bounds__(TX, stream_min_blocks<T, TX>()) a11_stream_kernel(StreamGrid g, const T *__restrict__ K,
                                                                  const T *__restrict__ u,
                                                                  const uint32_t *__restrict__ mbits,
                                                                  T *__restrict__ y)
{
  // tile of this CTA within the colour class
  const int bid = blockIdx.x;
  const int ixc = bid % g.nxc, iyc = (bid / g.nxc) % g.nyc, izc = bid / (g.nxc * g.nyc);
  stream_tile<T, TX, MASKED, KTX>(g, g.px + 2 * ixc, g.py + 2 * iyc, g.zc0 + 2 * izc, K, u, mbits, y);
}

// ---------------------------------------------------------------------------
// Batched form: one launch per (colour, tile width) over the concatenated
// work-list of many independent problems.  A work item is (problem, x-tile,
// row, z-chunk) of that colour; the problem descriptor carries its box, its
// tiling and its K; the vector pointers come from per-problem tables.
// ---------------------------------------------------------------------------
struct BatchProb {
  Box b;
  int ntx, LZ, nzc;
  int64_t MXP;
  const void *K;          // T* of the problem's Gauss-point factor
  const uint8_t *mask;    // Dirichlet mask (MatShell level) or null
  const uint32_t *mbits;  // the same mask packed one bit per dof
  int64_t nvel;           // length of the problem's vectors
};

template <typename T, int TX, bool MASKED>
__global__ void __launch_bounds__(TX, stream_min_blocks<T, TX>()) a11_stream_batch_kernel(const BatchProb *__restrict__ probs,
                                                                        const int4 *__restrict__ items, int px, int py,
                                                                        int pz, const T *const *__restrict__ uptr,
                                                                        T *const *__restrict__ yptr)
{
  const int4 it = items[blockIdx.x];  // (problem, tx, ej, zc)
  const BatchProb p = probs[it.x];
  StreamGrid g;
  g.b = p.b;
  g.TX = TX; g.ntx = p.ntx; g.LZ = p.LZ; g.nzc = p.nzc; g.MXP = p.MXP;
  g.px = px; g.py = py; g.pz = pz;
  g.nxc = g.nyc = g.nzcc = 0;
  g.zc0 = pz;
  stream_tile<T, TX, MASKED, false, true>(g, it.y, it.z, it.w, reinterpret_cast<const T *>(p.K), uptr[it.x],
                             MASKED ? p.mbits : nullptr, yptr[it.x]);
}

}  // namespace ptk
