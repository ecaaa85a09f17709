// C ABI of libpt_b200.so (declared in include/pt_b200.h).
//
// The op owns device copies of the mesh data (coordinates, quadrature-point
// viscosity, Dirichlet mask), FP32 shadows of coordinates/viscosity for the
// single-precision apply, and staging vectors for the host-pointer calls.
// Kernels live in kernels_*.cuh; this file does argument checking, memory,
// streams and the BC fix-ups of the MatShell-level calls.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "pt_b200.h"
#include "kernels_colour.cuh"
#include "kernels_stream.cuh"
#include "kernels_diag.cuh"
#include "kernels_ebe.cuh"
#include "kernels_markers.cuh"
#include "kernels_bmat.cuh"
#include "kernels_galerkin.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace {

thread_local std::string g_err;

pt_status fail(pt_status s, const char *fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return s;
}

#define PT_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t _e = (call);                                                                       \
    if (_e != cudaSuccess)                                                                         \
      return fail(_e == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_CUDA, "%s: %s (%s:%d)",    \
                  #call, cudaGetErrorString(_e), __FILE__, __LINE__);                              \
  } while (0)

#define PT_LAUNCHED(op)                                                                            \
  do {                                                                                             \
    (op)->launches++;                                                                              \
    cudaError_t _e = cudaGetLastError();                                                           \
    if (_e != cudaSuccess)                                                                         \
      return fail(PT_ERR_CUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(_e), __FILE__,     \
                  __LINE__);                                                                       \
  } while (0)

enum A11Kernel { A11_STREAM = 0, A11_COLOUR = 1, A11_EBE = 3 };

// "b200" picks stored element matrices for one-rank boxes up to this many
// elements (packed FP64 + FP32 matrices: 40 KB per element, 1.3 GB at 32^3)
// and the streaming kernel above.  Measured FP64 / FP32 apply, stored
// matrices vs streaming: 16^3 0.037 / 0.023 vs 0.26 / 0.22 ms, 32^3 0.24 /
// 0.14 vs 0.35 / 0.30 ms, 40^3 0.45 / 0.27 vs 0.36 / 0.27 ms.
constexpr int64_t EBE_AUTO_MAX_ELEMENTS = 32768;
// pipelined host-pointer applies: groups of about PIPE_LAYERS element layers,
// at most PIPE_GROUPS of them
constexpr int PIPE_LAYERS = 6;
constexpr int PIPE_GROUPS = 32;

}  // namespace

struct pt_op {
  ptk::Box box;
  int mx, my, mz;
  int64_t nnodes, nvel, nel, npres;
  cudaStream_t stream;
  bool own_stream;
  double *d_coords, *d_eta;
  float *d_coords32, *d_eta32;
  uint8_t *d_mask;
  uint32_t *d_mbits;  // the mask packed one bit per dof (the streaming kernel's column rule)
  bool has_coords, has_eta, has_mask;
  double *d_u, *d_y, *d_p, *d_yp; // staging for _h calls
  // streaming kernel: per-Gauss-point geometry K (FP64 and FP32 copies)
  double *d_K;
  float *d_K32;
  unsigned int *d_bad;
  int64_t MXP;
  int TX, ntx, LZ, nzc;
  bool geom_dirty, geom_ok, full_box, ebe_valid;
  bool be_valid;  // d_Be matches the coordinates
  double *d_Be;   // divergence blocks [nel][4][81] (one-rank boxes, built on first B / B^T use)
  int a11_kernel;
  int64_t launches;
  uint64_t state;  // bumped whenever coordinates, viscosity or the mask change
  int device;
  cudaMemPool_t pool;  // non-null: buffers are stream-ordered allocations from this pool on `stream`
  // stored element matrices (A11_EBE): FP64 and FP32, per-element outputs
  double *d_Ae;
  float *d_Ae32;
  double *d_ye;
  // marker projection scratch (grown on demand)
  void *mk_scratch;
  size_t mk_bytes;
  // pipelined host applies: copy streams and per-group events (created on first use)
  cudaStream_t h2d, d2h;
  cudaEvent_t ev_in[PIPE_GROUPS], ev_done[PIPE_GROUPS];
  bool pipe_ready;
  // strided viscosity uploads: two pinned chunks and their copy events (first use)
  double *h_stage[2];
  cudaEvent_t ev_stage[2];
  // momentum residual: Gauss-point body force [27 nel][3] and its load vector
  double *d_fu, *d_F;
  bool has_fu, F_valid;
};

namespace {

// Device buffers of an op: cudaMalloc, or stream-ordered from the op's pool
// (no device-wide synchronisation on free; used by the request server).
cudaError_t op_alloc(pt_op *op, void **p, size_t bytes)
{
  if (op->pool) return cudaMallocFromPoolAsync(p, bytes, op->pool, op->stream);
  return cudaMalloc(p, bytes);
}

void op_free(pt_op *op, void *p)
{
  if (!p) return;
  if (op->pool) cudaFreeAsync(p, op->stream);
  else cudaFree(p);
}

constexpr int TPB = 128;

inline unsigned nblocks(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

__global__ void to_f32_kernel(const double *__restrict__ a, float *__restrict__ b, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

template <typename T>
__global__ void bc_copy_kernel(const uint8_t *__restrict__ mask, const T *__restrict__ x, T *__restrict__ y, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (mask[i]) y[i] = x[i];
}

__global__ void bc_value_kernel(const uint8_t *__restrict__ mask, double v, double *__restrict__ y, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (mask[i]) y[i] = v;
}

__global__ void sub_kernel(const double *__restrict__ a, double *__restrict__ y, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] -= a[i];
}

// y_k = x_k on the Dirichlet dofs, from the packed mask (one thread per word,
// set bits only): the MatShell rows of the streaming apply.
template <typename T>
__global__ void bc_bits_kernel(const uint32_t *__restrict__ bits, const T *__restrict__ x, T *__restrict__ y, int64_t n)
{
  const int64_t nw = (n + 31) / 32;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t b = bits[w];
    while (b) {
      const int j = __ffs(b) - 1;
      b &= b - 1;
      const int64_t k = 32 * w + j;
      y[k] = x[k];
    }
  }
}

// bits[w] bit j = mask[32w + j] != 0 (one warp per word)
__global__ void pack_mask_kernel(const uint8_t *__restrict__ mask, uint32_t *__restrict__ bits, int64_t n)
{
  const int64_t nw = (n + 31) / 32;
  const int64_t wpb = blockDim.x / 32;
  for (int64_t w = (int64_t)blockIdx.x * wpb + threadIdx.x / 32; w < nw; w += (int64_t)gridDim.x * wpb) {
    const int64_t i = 32 * w + (threadIdx.x & 31);
    const unsigned b = __ballot_sync(0xffffffffu, i < n && mask[i]);
    if ((threadIdx.x & 31) == 0) bits[w] = b;
  }
}

unsigned grid_stride_blocks(int64_t n)
{
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

// One-time, per-device set-up of a kernel's launch attributes: the dynamic
// shared-memory limit (smem > 0) and, for the tiled kernels, the largest shared-memory
// carve-out (so every entry point launches a kernel at the same occupancy).
// Guarded by a mutex: host threads may launch on several devices at once.
std::mutex g_attr_mu;
std::vector<std::pair<const void *, int>> g_attr_done;

pt_status kernel_attrs(const void *fn, size_t smem, bool max_carveout = true)
{
  int dev = 0;
  PT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_attr_mu);
  for (const auto &d : g_attr_done)
    if (d.first == fn && d.second == dev) return PT_OK;
  if (smem) PT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (max_carveout)
    PT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
  g_attr_done.push_back({fn, dev});
  return PT_OK;
}

pt_status check_ready(const pt_op *op, bool need_eta)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (!op->has_coords) return fail(PT_ERR_STATE, "coordinates not set (pt_op_set_coords_*)");
  if (need_eta && !op->has_eta) return fail(PT_ERR_STATE, "viscosity not set (pt_op_set_eta_*)");
  return PT_OK;
}

pt_status upload_diag_tables()
{
  static bool done[64] = {false};
  static std::mutex mu;
  int dev = 0;
  PT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 64 && done[dev]) return PT_OK;
  // dN_n/dxi_d at Gauss point q (tensor-product Q2 basis).
  double b[3][3], db[3][3];
  const double x[3] = {-q2::GS, 0.0, q2::GS};
  for (int q = 0; q < 3; q++) {
    const double t = x[q];
    b[q][0] = 0.5 * t * (t - 1.0); b[q][1] = (1.0 + t) * (1.0 - t); b[q][2] = 0.5 * (1.0 + t) * t;
    db[q][0] = t - 0.5; db[q][1] = -2.0 * t; db[q][2] = t + 0.5;
  }
  static double tab[27][27][3];
  for (int a = 0; a < 3; a++)
    for (int bq = 0; bq < 3; bq++)
      for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++)
          for (int j = 0; j < 3; j++)
            for (int i = 0; i < 3; i++) {
              const int q = 9 * a + 3 * bq + c, n = 9 * k + 3 * j + i;
              tab[q][n][0] = db[c][i] * b[bq][j] * b[a][k];
              tab[q][n][1] = b[c][i] * db[bq][j] * b[a][k];
              tab[q][n][2] = b[c][i] * b[bq][j] * db[a][k];
            }
  PT_CUDA(cudaMemcpyToSymbol(ptk::c_dN, tab, sizeof tab));
  if (dev < 64) done[dev] = true;
  return PT_OK;
}


// ---- streaming kernel: geometry set-up and launch -----------------------------

// Enumerates the colour classes of the streaming tiles over z-chunks [zb, ze)
// in their fixed order and calls launch(cfg, g) for each non-empty class with
// the grid and launch configuration filled in.  The first launch is ordinary
// (the grid before it may write the kernel's inputs); the later ones are
// programmatic: each may start on the SMs the previous colour frees and waits
// inside before writing its output (measured at 128^3: 1.74 -> 1.63 ms with
// every A11 colour programmatic, bitwise the same result).
template <int TX, typename F>
pt_status stream_colours(pt_op *op, size_t smem, int zb, int ze, F &&launch)
{
  if (ze < 0) ze = op->nzc;
  ptk::StreamGrid g;
  g.b = op->box;
  g.TX = TX; g.ntx = op->ntx; g.LZ = op->LZ; g.nzc = op->nzc; g.MXP = op->MXP;
  cudaLaunchAttribute pdl[1] = {};
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  bool first = true;
  for (int pz = 0; pz < 2; pz++)
    for (int py = 0; py < 2; py++)
      for (int px = 0; px < 2; px++) {
        g.px = px; g.py = py; g.pz = pz;
        g.nxc = (op->ntx - px + 1) / 2;
        g.nyc = (op->my - py + 1) / 2;
        g.zc0 = zb + ((zb & 1) != pz);  // first chunk >= zb of parity pz
        g.nzcc = g.zc0 < ze ? (ze - g.zc0 + 1) / 2 : 0;
        const int64_t n = (int64_t)g.nxc * g.nyc * g.nzcc;
        if (n == 0) continue;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)n);
        cfg.blockDim = dim3(TX);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = op->stream;
        cfg.attrs = first ? nullptr : pdl;
        cfg.numAttrs = first ? 0 : 1;
        pt_status s = launch(cfg, g);
        if (s != PT_OK) return s;
        PT_LAUNCHED(op);
        first = false;
      }
  return PT_OK;
}

// Launches the streaming kernel's colour passes over z-chunks [zb, ze)
// (ze < 0: all).  A sub-range must start at chunk 0 or at an odd chunk and end
// after an even one, or at the last chunk, so the node sums keep the order of
// the whole-box launch (the even chunk of a boundary plane stores, the odd one
// adds).
// KTX: one x-tile per row (MXP == TX), the K stride a compile-time constant
// (FP64 only: it measured no faster in FP32).
template <typename T, int TX, bool MASKED, bool KTX>
pt_status launch_stream_tx_k(pt_op *op, const T *K, const T *u, T *y, int zb, int ze)
{
  if (MASKED && !op->d_mbits) return fail(PT_ERR_STATE, "masked apply without the packed Dirichlet bits");
  if (KTX && op->MXP != TX) return fail(PT_ERR_STATE, "K row stride differs from the tile width");
  constexpr size_t smem = ptk::stream_smem_bytes<T, TX>();
  pt_status as = kernel_attrs((const void *)ptk::a11_stream_kernel<T, TX, MASKED, KTX>, smem);
  if (as != PT_OK) return as;
  const uint32_t *mb = MASKED ? op->d_mbits : nullptr;
  return stream_colours<TX>(op, smem, zb, ze, [&](const cudaLaunchConfig_t &cfg, const ptk::StreamGrid &g) {
    const cudaError_t e = cudaLaunchKernelEx(&cfg, ptk::a11_stream_kernel<T, TX, MASKED, KTX>, g, K, u, mb, y);
    if (e != cudaSuccess) return fail(PT_ERR_CUDA, "streaming A11 launch: %s", cudaGetErrorString(e));
    return PT_OK;
  });
}

template <typename T, int TX, bool MASKED>
pt_status launch_stream_tx(pt_op *op, const T *K, const T *u, T *y, int zb = 0, int ze = -1)
{
  if constexpr (sizeof(T) == 8) {
    if (op->MXP == TX) return launch_stream_tx_k<T, TX, MASKED, true>(op, K, u, y, zb, ze);
  }
  return launch_stream_tx_k<T, TX, MASKED, false>(op, K, u, y, zb, ze);
}

// diag(A11) on the streaming tiles from the stored K (whole box, one launch
// per colour class, programmatic like the apply).
template <int TX, bool KTX>
pt_status launch_diag_stream_tx(pt_op *op, double *d)
{
  constexpr size_t smem = ptk::diag_smem_bytes<TX>();
  pt_status as = kernel_attrs((const void *)ptk::diag_stream_kernel<TX, KTX>, smem);
  if (as != PT_OK) return as;
  const double *K = op->d_K;
  return stream_colours<TX>(op, smem, 0, -1, [&](const cudaLaunchConfig_t &cfg, const ptk::StreamGrid &g) {
    const cudaError_t e = cudaLaunchKernelEx(&cfg, ptk::diag_stream_kernel<TX, KTX>, g, K, d);
    if (e != cudaSuccess) return fail(PT_ERR_CUDA, "streaming diag launch: %s", cudaGetErrorString(e));
    return PT_OK;
  });
}

pt_status launch_diag_stream(pt_op *op, double *d)
{
  if (op->TX == 32) return op->MXP == 32 ? launch_diag_stream_tx<32, true>(op, d) : launch_diag_stream_tx<32, false>(op, d);
  if (op->TX == 64) return op->MXP == 64 ? launch_diag_stream_tx<64, true>(op, d) : launch_diag_stream_tx<64, false>(op, d);
  return op->MXP == 128 ? launch_diag_stream_tx<128, true>(op, d) : launch_diag_stream_tx<128, false>(op, d);
}

template <typename T, bool MASKED>
pt_status launch_stream(pt_op *op, const T *K, const T *u, T *y)
{
  if (op->TX == 32) return launch_stream_tx<T, 32, MASKED>(op, K, u, y);
  if (op->TX == 64) return launch_stream_tx<T, 64, MASKED>(op, K, u, y);
  return launch_stream_tx<T, 128, MASKED>(op, K, u, y);
}

// Recompute K when coordinates or viscosity changed.  Sets geom_ok = false
// (and the op falls back to the colour kernel) if any c = w eta / det <= 0.
pt_status ensure_geometry(pt_op *op)
{
  if (!op->geom_dirty) return PT_OK;
  const int64_t nk = (int64_t)op->my * op->mz * 243 * op->MXP;
  if (!op->d_K) {
    PT_CUDA(op_alloc(op, (void **)&op->d_K, sizeof(double) * nk));
    PT_CUDA(op_alloc(op, (void **)&op->d_K32, sizeof(float) * nk));
    PT_CUDA(op_alloc(op, (void **)&op->d_bad, sizeof(unsigned int)));
  }
  PT_CUDA(cudaMemsetAsync(op->d_bad, 0, sizeof(unsigned int), op->stream));
  ptk::geom_kernel<double><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->MXP, op->d_coords, op->d_eta,
                                                                       op->d_K, op->d_bad);
  PT_LAUNCHED(op);
  ptk::geom_kernel<float><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->MXP, op->d_coords, op->d_eta,
                                                                      op->d_K32, op->d_bad);
  PT_LAUNCHED(op);
  unsigned int bad = 0;
  PT_CUDA(cudaMemcpyAsync(&bad, op->d_bad, sizeof bad, cudaMemcpyDeviceToHost, op->stream));
  PT_CUDA(cudaStreamSynchronize(op->stream));
  op->geom_ok = (bad == 0);
  op->geom_dirty = false;
  op->ebe_valid = false;
  return PT_OK;
}

// Element matrices of the current geometry (A11_EBE), built on first use.
pt_status ensure_ebe(pt_op *op)
{
  if (op->ebe_valid) return PT_OK;
  if (!op->d_Ae) PT_CUDA(op_alloc(op, (void **)&op->d_Ae, sizeof(double) * ptk::EBE_LD * op->nel));
  if (!op->d_Ae32) PT_CUDA(op_alloc(op, (void **)&op->d_Ae32, sizeof(float) * ptk::EBE_LD * op->nel));
  if (!op->d_ye) PT_CUDA(op_alloc(op, (void **)&op->d_ye, sizeof(double) * 81 * op->nel));
  ptk::element_matrix_kernel<double><<<(unsigned)op->nel, 96, 0, op->stream>>>(op->box, op->d_coords, op->d_eta,
                                                                               op->d_Ae);
  PT_LAUNCHED(op);
  ptk::element_matrix_kernel<float><<<(unsigned)op->nel, 96, 0, op->stream>>>(op->box, op->d_coords, op->d_eta,
                                                                              op->d_Ae32);
  PT_LAUNCHED(op);
  op->ebe_valid = true;
  return PT_OK;
}

template <typename T>
const T *op_Ae(const pt_op *op);
template <>
const double *op_Ae<double>(const pt_op *op) { return op->d_Ae; }
template <>
const float *op_Ae<float>(const pt_op *op) { return op->d_Ae32; }

// The element GEMV stages 13-27 KB per CTA: ask for the largest shared-memory
// carve-out so that 8 (FP64) to 16 (FP32) elements run per SM.
template <typename T, bool MASKED>
pt_status ebe_carveout()
{
  return kernel_attrs((const void *)ptk::ebe_apply_kernel<T, MASKED>, 0, true);
}

template <bool MASKED>
pt_status ebe_h_carveout()
{
  return kernel_attrs((const void *)ptk::ebe_apply_h_kernel<MASKED>, 0, true);
}

template <typename T>
pt_status launch_ebe(pt_op *op, const T *u, T *y, bool masked)
{
  pt_status s = ensure_ebe(op);
  if (s != PT_OK) return s;
  if ((s = ebe_carveout<T, true>()) != PT_OK || (s = ebe_carveout<T, false>()) != PT_OK) return s;
  T *ye = reinterpret_cast<T *>(op->d_ye);
  if (masked) {
    ptk::ebe_apply_kernel<T, true><<<(unsigned)op->nel, 96, 0, op->stream>>>(op->box, op_Ae<T>(op), u, op->d_mask, ye);
    PT_LAUNCHED(op);
    ptk::ebe_gather_kernel<T, true><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->box, ye, u, op->d_mask,
                                                                                         y);
  } else {
    ptk::ebe_apply_kernel<T, false><<<(unsigned)op->nel, 96, 0, op->stream>>>(op->box, op_Ae<T>(op), u, nullptr, ye);
    PT_LAUNCHED(op);
    ptk::ebe_gather_kernel<T, false><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->box, ye, u, nullptr, y);
  }
  PT_LAUNCHED(op);
  return PT_OK;
}

// ---- A11 dispatch -----------------------------------------------------------

// The streaming and stored-matrix applies set y_k = x_k on Dirichlet dofs
// inside launch_a11, so MatMult needs no separate pass after them.
bool a11_sets_bc_rows(const pt_op *op)
{
  const bool stream = op->a11_kernel == A11_STREAM;
  const bool ebe = op->a11_kernel == A11_EBE && op->full_box;
  return (stream || ebe) && op->geom_ok && !op->geom_dirty;
}

template <typename T>
const T *op_K(const pt_op *op);
template <>
const double *op_K<double>(const pt_op *op) { return op->d_K; }
template <>
const float *op_K<float>(const pt_op *op) { return op->d_K32; }

template <typename T>
pt_status launch_a11(pt_op *op, const T *coords, const T *eta, const T *u, T *y, bool masked)
{
  if (op->a11_kernel == A11_EBE && op->full_box) {
    pt_status s = ensure_geometry(op);
    if (s != PT_OK) return s;
    if (op->geom_ok) return launch_ebe<T>(op, u, y, masked);
  }
  if (op->a11_kernel == A11_STREAM) {
    pt_status s = ensure_geometry(op);
    if (s != PT_OK) return s;
    if (op->geom_ok) {
      if (!op->full_box) PT_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * op->nvel, op->stream));
      if (masked) {
        // Dirichlet columns inside the kernel; rows y_k = x_k after its colour passes
        if ((s = launch_stream<T, true>(op, op_K<T>(op), u, y)) != PT_OK) return s;
        bc_bits_kernel<T><<<grid_stride_blocks((op->nvel + 31) / 32), 256, 0, op->stream>>>(op->d_mbits, u, y, op->nvel);
        PT_LAUNCHED(op);
        return PT_OK;
      }
      return launch_stream<T, false>(op, op_K<T>(op), u, y);
    }
  }
  PT_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * op->nvel, op->stream));
  for (int c = 0; c < 8; c++) {
    ptk::ColourGrid g = ptk::colour_grid(op->box, c);
    const int64_t n = (int64_t)g.ncx * g.ncy * g.ncz;
    if (n == 0) continue;
    if (masked)
      ptk::a11_colour_kernel<T, true><<<nblocks(n), TPB, 0, op->stream>>>(g, coords, eta, u, op->d_mask, y);
    else
      ptk::a11_colour_kernel<T, false><<<nblocks(n), TPB, 0, op->stream>>>(g, coords, eta, u, nullptr, y);
    PT_LAUNCHED(op);
  }
  return PT_OK;
}

pt_status diag_d(pt_op *op, double *d)
{
  pt_status s;
  if (op->a11_kernel == A11_EBE && op->full_box) {
    // the stored element matrices carry the diagonal: one gather
    if ((s = ensure_geometry(op)) != PT_OK) return s;
    if (op->geom_ok) {
      if ((s = ensure_ebe(op)) != PT_OK) return s;
      ptk::ebe_diag_kernel<<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->box, op->d_Ae, d);
      PT_LAUNCHED(op);
      return PT_OK;
    }
  }
  if (op->a11_kernel == A11_STREAM) {
    // the streaming tiles from the stored K, as the apply
    if ((s = ensure_geometry(op)) != PT_OK) return s;
    if (op->geom_ok) {
      if (!op->full_box) PT_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * op->nvel, op->stream));
      return launch_diag_stream(op, d);
    }
  }
  s = upload_diag_tables();
  if (s != PT_OK) return s;
  PT_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * op->nvel, op->stream));
  for (int c = 0; c < 8; c++) {
    ptk::ColourGrid g = ptk::colour_grid(op->box, c);
    const int64_t n = (int64_t)g.ncx * g.ncy * g.ncz;
    if (n == 0) continue;
    ptk::diag_colour_kernel<<<nblocks(n), TPB, 0, op->stream>>>(g, op->d_coords, op->d_eta, d);
    PT_LAUNCHED(op);
  }
  return PT_OK;
}

// Divergence blocks of the current coordinates (one-rank boxes), built on first use.
pt_status ensure_be(pt_op *op)
{
  if (op->be_valid) return PT_OK;
  if (!op->d_Be) PT_CUDA(op_alloc(op, (void **)&op->d_Be, sizeof(double) * ptk::BMAT_LD * op->nel));
  ptk::bmat_kernel<<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->d_coords, op->d_Be);
  PT_LAUNCHED(op);
  op->be_valid = true;
  return PT_OK;
}

pt_status a21_d(pt_op *op, const double *u, double *yp, bool masked)
{
  if (op->full_box) {
    pt_status s = ensure_be(op);
    if (s != PT_OK) return s;
    if (masked)
      ptk::bmat_a21_kernel<true><<<nblocks(32 * op->nel), TPB, 0, op->stream>>>(op->box, op->d_Be, u, op->d_mask, yp);
    else
      ptk::bmat_a21_kernel<false><<<nblocks(32 * op->nel), TPB, 0, op->stream>>>(op->box, op->d_Be, u, nullptr, yp);
    PT_LAUNCHED(op);
    return PT_OK;
  }
  if (masked)
    ptk::a21_kernel<true><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->d_coords, u, op->d_mask, yp);
  else
    ptk::a21_kernel<false><<<nblocks(op->nel), TPB, 0, op->stream>>>(op->box, op->d_coords, u, nullptr, yp);
  PT_LAUNCHED(op);
  return PT_OK;
}

// yu = B^T p, or yu += B^T p (accumulate)
pt_status a12_d(pt_op *op, const double *p, double *yu, bool accumulate = false)
{
  if (op->full_box) {
    // one-rank box: node by node from the stored blocks
    pt_status s = ensure_be(op);
    if (s != PT_OK) return s;
    if (accumulate)
      ptk::bmat_a12_gather_kernel<true><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->box, op->d_Be, p, yu);
    else
      ptk::bmat_a12_gather_kernel<false><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->box, op->d_Be, p, yu);
    PT_LAUNCHED(op);
    return PT_OK;
  }
  if (!accumulate) PT_CUDA(cudaMemsetAsync(yu, 0, sizeof(double) * op->nvel, op->stream));
  for (int c = 0; c < 8; c++) {
    ptk::ColourGrid g = ptk::colour_grid(op->box, c);
    const int64_t n = (int64_t)g.ncx * g.ncy * g.ncz;
    if (n == 0) continue;
    ptk::a12_colour_kernel<<<nblocks(n), TPB, 0, op->stream>>>(g, op->d_coords, p, yu);
    PT_LAUNCHED(op);
  }
  return PT_OK;
}

pt_status bc_copy(pt_op *op, const double *x, double *y)
{
  if (!op->has_mask) return PT_OK;
  bc_copy_kernel<double><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->d_mask, x, y, op->nvel);
  PT_LAUNCHED(op);
  return PT_OK;
}

pt_status bc_copy32(pt_op *op, const float *x, float *y)
{
  if (!op->has_mask) return PT_OK;
  bc_copy_kernel<float><<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->d_mask, x, y, op->nvel);
  PT_LAUNCHED(op);
  return PT_OK;
}

pt_status bc_value(pt_op *op, double v, double *y)
{
  if (!op->has_mask) return PT_OK;
  bc_value_kernel<<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->d_mask, v, y, op->nvel);
  PT_LAUNCHED(op);
  return PT_OK;
}

// Host-pointer wrapper: copy nin doubles in, run f, copy nout doubles out, sync.
template <typename F>
pt_status host_call(pt_op *op, const double *in, int64_t nin, double *din, double *out, int64_t nout, double *dout, F f)
{
  if (!out) return fail(PT_ERR_BAD_ARG, "output pointer is NULL");
  if (nin > 0) {
    if (!in) return fail(PT_ERR_BAD_ARG, "input pointer is NULL");
    PT_CUDA(cudaMemcpyAsync(din, in, sizeof(double) * nin, cudaMemcpyHostToDevice, op->stream));
  }
  pt_status s = f();
  if (s != PT_OK) return s;
  PT_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, op->stream));
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

bool is_pinned(const void *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host-array A11 apply with the copies overlapped with the compute: the box
// is cut into groups of z-chunks; group g's input node planes go up on one
// copy stream, its colour passes run when they have arrived, and every node
// plane that no later group touches comes down on a second copy stream.  The
// passes are those of the whole-box launch cut by z-range (see
// launch_stream_tx), so the result is bitwise the one-shot apply's.  Used for
// pinned host arrays on a one-rank box with the streaming kernel; returns
// false when that does not apply.
template <bool MASKED>
pt_status a11_host_pipelined(pt_op *op, const double *hu, double *hy, bool *done)
{
  *done = false;
  if (!op->full_box || op->a11_kernel != A11_STREAM || !is_pinned(hu) || !is_pinned(hy)) return PT_OK;
  pt_status s = ensure_geometry(op);
  if (s != PT_OK) return s;
  if (!op->geom_ok || op->nzc < 2) return PT_OK;
  if (!op->pipe_ready) {
    PT_CUDA(cudaStreamCreateWithFlags(&op->h2d, cudaStreamNonBlocking));
    PT_CUDA(cudaStreamCreateWithFlags(&op->d2h, cudaStreamNonBlocking));
    for (int g = 0; g < PIPE_GROUPS; g++) {
      PT_CUDA(cudaEventCreateWithFlags(&op->ev_in[g], cudaEventDisableTiming));
      PT_CUDA(cudaEventCreateWithFlags(&op->ev_done[g], cudaEventDisableTiming));
    }
    op->pipe_ready = true;
  }
  if (!op->d_u || !op->d_y) return PT_OK;  // callers stage first
  // groups of chunks [c0, c1] of about PIPE_LAYERS element layers: each ends
  // at an even chunk or at the last one, so each later group starts at an odd
  // chunk.  Finer groups shorten the head (compute waits for the first group's
  // planes) and the tail (the last group's planes come down after its
  // compute); at 128^3 groups of 6 layers measured 10.3-10.6 ms against 11.0
  // for 8 groups, with pure copies in 8 pieces each way at 9.3 ms.
  std::vector<std::pair<int, int>> groups;
  for (int per = std::max(1, (PIPE_LAYERS + op->LZ - 1) / op->LZ);; per++) {
    groups.clear();
    for (int c0 = 0; c0 < op->nzc;) {
      int c1 = std::min(op->nzc - 1, c0 + per - 1);
      if (c1 < op->nzc - 1 && (c1 & 1)) c1++;
      groups.push_back({c0, c1});
      c0 = c1 + 1;
    }
    if ((int)groups.size() <= PIPE_GROUPS) break;
  }
  const int64_t plane = 3 * op->box.XY;  // doubles per node plane
  const int64_t nplanes = 2 * (int64_t)op->mz + 1;
  int64_t up = 0, down = 0;  // next plane to upload / download
  PT_CUDA(cudaEventRecord(op->ev_done[0], op->stream));  // earlier work on the op's stream precedes the copies
  PT_CUDA(cudaStreamWaitEvent(op->h2d, op->ev_done[0], 0));
  for (size_t gi = 0; gi < groups.size(); gi++) {
    const int c0 = groups[gi].first, c1 = groups[gi].second;
    const bool last = gi + 1 == groups.size();
    const int64_t top = 2 * (int64_t)std::min((c1 + 1) * op->LZ, op->mz);  // top node plane of the group
    if (top + 1 > up) {
      PT_CUDA(cudaMemcpyAsync(op->d_u + up * plane, hu + up * plane, sizeof(double) * (top + 1 - up) * plane,
                              cudaMemcpyHostToDevice, op->h2d));
      up = top + 1;
    }
    PT_CUDA(cudaEventRecord(op->ev_in[gi], op->h2d));
    PT_CUDA(cudaStreamWaitEvent(op->stream, op->ev_in[gi], 0));
    if (op->TX == 32) s = launch_stream_tx<double, 32, MASKED>(op, op->d_K, op->d_u, op->d_y, c0, c1 + 1);
    else if (op->TX == 64) s = launch_stream_tx<double, 64, MASKED>(op, op->d_K, op->d_u, op->d_y, c0, c1 + 1);
    else s = launch_stream_tx<double, 128, MASKED>(op, op->d_K, op->d_u, op->d_y, c0, c1 + 1);
    if (s != PT_OK) return s;
    PT_CUDA(cudaEventRecord(op->ev_done[gi], op->stream));
    const int64_t fin = last ? nplanes : top;  // planes below `fin` are final
    if (MASKED && fin > down) {  // their Dirichlet rows, y_k = x_k
      const int64_t o = down * plane, m = (fin - down) * plane;
      bc_copy_kernel<double><<<grid_stride_blocks(m), 256, 0, op->stream>>>(op->d_mask + o, op->d_u + o, op->d_y + o, m);
      PT_LAUNCHED(op);
      PT_CUDA(cudaEventRecord(op->ev_done[gi], op->stream));
    }
    if (fin > down) {
      PT_CUDA(cudaStreamWaitEvent(op->d2h, op->ev_done[gi], 0));
      PT_CUDA(cudaMemcpyAsync(hy + down * plane, op->d_y + down * plane, sizeof(double) * (fin - down) * plane,
                              cudaMemcpyDeviceToHost, op->d2h));
      down = fin;
    }
  }
  PT_CUDA(cudaStreamSynchronize(op->d2h));
  *done = true;
  return PT_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char *pt_last_error(void) { return g_err.c_str(); }
const char *pt_version(void) { return "pt_b200 0.1 (sm_100a)"; }

// pool == null: pt_op_create (own stream, cudaMalloc).  Otherwise every
// buffer comes from `pool`, ordered on `stream`, which the op then uses.
static pt_status op_create_impl(const pt_mesh_desc *desc, cudaMemPool_t pool, cudaStream_t stream, pt_op **out)
{
  if (!desc || !out) return fail(PT_ERR_BAD_ARG, "NULL argument");
  *out = nullptr;
  if (desc->mx < 1 || desc->my < 1 || desc->mz < 1)
    return fail(PT_ERR_BAD_ARG, "element counts must be >= 1 (got %d x %d x %d)", desc->mx, desc->my, desc->mz);
  const int64_t nx = desc->nx ? desc->nx : 2 * (int64_t)desc->mx + 1;
  const int64_t ny = desc->ny ? desc->ny : 2 * (int64_t)desc->my + 1;
  const int64_t nz = desc->nz ? desc->nz : 2 * (int64_t)desc->mz + 1;
  if (desc->ox < 0 || desc->oy < 0 || desc->oz < 0 || desc->ox + 2 * (int64_t)desc->mx + 1 > nx ||
      desc->oy + 2 * (int64_t)desc->my + 1 > ny || desc->oz + 2 * (int64_t)desc->mz + 1 > nz)
    return fail(PT_ERR_BAD_ARG, "element box (%d,%d,%d)+(%d,%d,%d) does not fit the node box %lld x %lld x %lld",
                desc->ox, desc->oy, desc->oz, desc->mx, desc->my, desc->mz, (long long)nx, (long long)ny, (long long)nz);
  const int64_t nnodes = nx * ny * nz;
  if (nnodes > ((int64_t)1 << 40)) return fail(PT_ERR_BAD_ARG, "mesh too large");
  pt_op *op = (pt_op *)calloc(1, sizeof(pt_op));
  if (!op) return fail(PT_ERR_OOM, "host allocation failed");
  op->mx = desc->mx; op->my = desc->my; op->mz = desc->mz;
  op->box.mx = desc->mx; op->box.my = desc->my; op->box.mz = desc->mz;
  op->box.X = nx; op->box.XY = nx * ny;
  op->box.off = desc->ox + desc->oy * nx + desc->oz * nx * ny;
  op->nnodes = nnodes;
  op->nvel = 3 * nnodes;
  op->nel = (int64_t)desc->mx * desc->my * desc->mz;
  op->npres = 4 * op->nel;
  op->full_box = (nx == 2 * (int64_t)desc->mx + 1) && (ny == 2 * (int64_t)desc->my + 1) &&
                 (nz == 2 * (int64_t)desc->mz + 1);
  op->a11_kernel = (op->full_box && op->nel <= EBE_AUTO_MAX_ELEMENTS) ? A11_EBE : A11_STREAM;
  op->TX = desc->mx <= 32 ? 32 : (desc->mx <= 64 ? 64 : 128);
  op->ntx = (desc->mx + op->TX - 1) / op->TX;
  op->MXP = (int64_t)op->ntx * op->TX;
  pt_op_set_tiling(op, 0);
  op->geom_dirty = true;
  cudaError_t e = cudaGetDevice(&op->device);
  if (pool) {
    op->pool = pool;
    op->stream = stream;
  } else {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) op->own_stream = true;
  }
  if (e == cudaSuccess) e = op_alloc(op, (void **)&op->d_coords, sizeof(double) * op->nvel);
  if (e == cudaSuccess) e = op_alloc(op, (void **)&op->d_eta, sizeof(double) * 27 * op->nel);
  if (e == cudaSuccess) e = op_alloc(op, (void **)&op->d_coords32, sizeof(float) * op->nvel);
  if (e == cudaSuccess) e = op_alloc(op, (void **)&op->d_eta32, sizeof(float) * 27 * op->nel);
  if (e == cudaSuccess) e = op_alloc(op, (void **)&op->d_mask, op->nvel);
  if (e == cudaSuccess) e = cudaMemsetAsync(op->d_mask, 0, op->nvel, op->stream);
  if (e == cudaSuccess && !pool) e = cudaStreamSynchronize(op->stream);
  if (e != cudaSuccess) {
    pt_status s = fail(e == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_CUDA, "pt_op_create: %s",
                       cudaGetErrorString(e));
    pt_op_destroy(op);
    return s;
  }
  *out = op;
  return PT_OK;
}

pt_status pt_op_create(const pt_mesh_desc *desc, pt_op **out) { return op_create_impl(desc, nullptr, nullptr, out); }

pt_status pt_op_destroy(pt_op *op)
{
  if (!op) return PT_OK;
  // pooled ops free in stream order (after the op's queued work); others wait
  if (op->stream && !op->pool) cudaStreamSynchronize(op->stream);
  void *bufs[] = {op->d_coords, op->d_eta, op->d_coords32, op->d_eta32, op->d_mask, op->d_u,
                  op->d_y, op->d_p, op->d_K, op->d_K32, op->d_bad, op->d_Ae, op->d_Ae32, op->d_ye,
                  op->mk_scratch, op->d_Be, op->d_yp, op->d_mbits, op->d_fu, op->d_F};
  for (void *b : bufs) op_free(op, b);
  for (int b = 0; b < 2; b++)
    if (op->h_stage[b]) {
      cudaEventSynchronize(op->ev_stage[b]);
      cudaEventDestroy(op->ev_stage[b]);
      cudaFreeHost(op->h_stage[b]);
    }
  if (op->own_stream && op->stream) cudaStreamDestroy(op->stream);
  if (op->pipe_ready) {
    cudaStreamSynchronize(op->h2d);
    cudaStreamSynchronize(op->d2h);
    cudaStreamDestroy(op->h2d);
    cudaStreamDestroy(op->d2h);
    for (int g = 0; g < PIPE_GROUPS; g++) {
      cudaEventDestroy(op->ev_in[g]);
      cudaEventDestroy(op->ev_done[g]);
    }
  }
  free(op);
  return PT_OK;
}

pt_status pt_op_set_stream(pt_op *op, void *stream)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  PT_CUDA(cudaStreamSynchronize(op->stream));
  if (op->own_stream) PT_CUDA(cudaStreamDestroy(op->stream));
  op->own_stream = false;
  op->stream = (cudaStream_t)stream;  // NULL: the legacy default stream
  return PT_OK;
}

pt_status pt_op_get_sizes(const pt_op *op, int64_t *nvel, int64_t *npres, int64_t *nel)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (nvel) *nvel = op->nvel;
  if (npres) *npres = op->npres;
  if (nel) *nel = op->nel;
  return PT_OK;
}

static pt_status finish_coords(pt_op *op)
{
  to_f32_kernel<<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->d_coords, op->d_coords32, op->nvel);
  PT_LAUNCHED(op);
  op->has_coords = true;
  op->geom_dirty = true;
  op->be_valid = false;
  op->F_valid = false;
  op->state++;
  return PT_OK;
}

static pt_status finish_eta(pt_op *op)
{
  to_f32_kernel<<<grid_stride_blocks(27 * op->nel), 256, 0, op->stream>>>(op->d_eta, op->d_eta32, 27 * op->nel);
  PT_LAUNCHED(op);
  op->has_eta = true;
  op->geom_dirty = true;
  op->state++;
  return PT_OK;
}

pt_status pt_op_set_coords_h(pt_op *op, const double *coords)
{
  if (!op || !coords) return fail(PT_ERR_BAD_ARG, "NULL argument");
  PT_CUDA(cudaMemcpyAsync(op->d_coords, coords, sizeof(double) * op->nvel, cudaMemcpyHostToDevice, op->stream));
  pt_status s = finish_coords(op);
  if (s != PT_OK) return s;
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

pt_status pt_op_set_coords_d(pt_op *op, const double *coords)
{
  if (!op || !coords) return fail(PT_ERR_BAD_ARG, "NULL argument");
  PT_CUDA(cudaMemcpyAsync(op->d_coords, coords, sizeof(double) * op->nvel, cudaMemcpyDeviceToDevice, op->stream));
  return finish_coords(op);
}

pt_status pt_op_set_eta_h(pt_op *op, const double *eta)
{
  if (!op || !eta) return fail(PT_ERR_BAD_ARG, "NULL argument");
  PT_CUDA(cudaMemcpyAsync(op->d_eta, eta, sizeof(double) * 27 * op->nel, cudaMemcpyHostToDevice, op->stream));
  pt_status s = finish_eta(op);
  if (s != PT_OK) return s;
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

pt_status pt_op_set_eta_d(pt_op *op, const double *eta)
{
  if (!op || !eta) return fail(PT_ERR_BAD_ARG, "NULL argument");
  PT_CUDA(cudaMemcpyAsync(op->d_eta, eta, sizeof(double) * 27 * op->nel, cudaMemcpyDeviceToDevice, op->stream));
  return finish_eta(op);
}

// Gathers eta0[i*stride] (the eta member of an array of QPntVolCoefStokes
// records) through two op-owned pinned chunks: while one chunk's copy runs on
// the op's stream the host fills the other.  The chunks are allocated once.
constexpr int64_t ETA_STAGE_DOUBLES = (int64_t)1 << 19;  // 4 MiB per chunk

pt_status pt_op_set_eta_strided_h(pt_op *op, const double *eta0, int64_t stride)
{
  if (!op || !eta0) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (stride < 1) return fail(PT_ERR_BAD_ARG, "stride must be >= 1 (got %lld)", (long long)stride);
  if (stride == 1) return pt_op_set_eta_h(op, eta0);
  if (!op->h_stage[0]) {
    for (int b = 0; b < 2; b++) {
      PT_CUDA(cudaMallocHost(&op->h_stage[b], sizeof(double) * ETA_STAGE_DOUBLES));
      PT_CUDA(cudaEventCreateWithFlags(&op->ev_stage[b], cudaEventDisableTiming));
    }
  }
  const int64_t n = 27 * op->nel;
  for (int64_t c0 = 0, k = 0; c0 < n; c0 += ETA_STAGE_DOUBLES, k++) {
    const int b = (int)(k & 1);
    const int64_t m = std::min(ETA_STAGE_DOUBLES, n - c0);
    PT_CUDA(cudaEventSynchronize(op->ev_stage[b]));  // the copy that last read this chunk is done
    double *dst = op->h_stage[b];
    const double *src = eta0 + c0 * stride;
    for (int64_t i = 0; i < m; i++) dst[i] = src[i * stride];
    PT_CUDA(cudaMemcpyAsync(op->d_eta + c0, dst, sizeof(double) * m, cudaMemcpyHostToDevice, op->stream));
    PT_CUDA(cudaEventRecord(op->ev_stage[b], op->stream));
  }
  pt_status s = finish_eta(op);
  if (s != PT_OK) return s;
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

// After d_mask changed: its packed bits (allocated on first use), on the op's stream.
static pt_status finish_mask(pt_op *op)
{
  const int64_t nw = (op->nvel + 31) / 32;
  if (!op->d_mbits) PT_CUDA(op_alloc(op, (void **)&op->d_mbits, sizeof(uint32_t) * nw));
  pack_mask_kernel<<<grid_stride_blocks(32 * nw), 256, 0, op->stream>>>(op->d_mask, op->d_mbits, op->nvel);
  PT_LAUNCHED(op);
  op->has_mask = true;
  op->state++;
  return PT_OK;
}

pt_status pt_op_set_bc_mask_h(pt_op *op, const uint8_t *mask)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (!mask) {
    PT_CUDA(cudaMemsetAsync(op->d_mask, 0, op->nvel, op->stream));
    op->has_mask = false;
    op->state++;
  } else {
    PT_CUDA(cudaMemcpyAsync(op->d_mask, mask, op->nvel, cudaMemcpyHostToDevice, op->stream));
    pt_status s = finish_mask(op);
    if (s != PT_OK) return s;
  }
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

static pt_status ensure_staging(pt_op *op)
{
  if (!op->d_u) PT_CUDA(op_alloc(op, (void **)&op->d_u, sizeof(double) * op->nvel));
  if (!op->d_y) PT_CUDA(op_alloc(op, (void **)&op->d_y, sizeof(double) * op->nvel));
  if (!op->d_p) PT_CUDA(op_alloc(op, (void **)&op->d_p, sizeof(double) * op->npres));
  if (!op->d_yp) PT_CUDA(op_alloc(op, (void **)&op->d_yp, sizeof(double) * op->npres));
  return PT_OK;
}

// ---- SpMVOp level -----------------------------------------------------------

pt_status pt_a11_apply_d(pt_op *op, const double *u, double *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!u || !y) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return launch_a11<double>(op, op->d_coords, op->d_eta, u, y, false);
}

pt_status pt_a11_apply_h(pt_op *op, const double *u, double *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  bool done = false;
  if (u && y && (s = a11_host_pipelined<false>(op, u, y, &done)) != PT_OK) return s;
  if (done) return PT_OK;
  return host_call(op, u, op->nvel, op->d_u, y, op->nvel, op->d_y,
                   [&]() { return launch_a11<double>(op, op->d_coords, op->d_eta, op->d_u, op->d_y, false); });
}

pt_status pt_a11_apply_f32_d(pt_op *op, const float *u, float *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!u || !y) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return launch_a11<float>(op, op->d_coords32, op->d_eta32, u, y, false);
}

pt_status pt_a11_diag_d(pt_op *op, double *d)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!d) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return diag_d(op, d);
}

pt_status pt_a11_diag_h(pt_op *op, double *d)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, nullptr, 0, nullptr, d, op->nvel, op->d_y, [&]() { return diag_d(op, op->d_y); });
}

pt_status pt_a21_apply_d(pt_op *op, const double *u, double *yp)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if (!u || !yp) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return a21_d(op, u, yp, false);
}

pt_status pt_a21_apply_h(pt_op *op, const double *u, double *yp)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, u, op->nvel, op->d_u, yp, op->npres, op->d_p, [&]() { return a21_d(op, op->d_u, op->d_p, false); });
}

pt_status pt_a12_apply_d(pt_op *op, const double *p, double *yu)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if (!p || !yu) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return a12_d(op, p, yu);
}

pt_status pt_a12_apply_h(pt_op *op, const double *p, double *yu)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, p, op->npres, op->d_p, yu, op->nvel, op->d_y, [&]() { return a12_d(op, op->d_p, op->d_y); });
}

// ---- MatShell level -----------------------------------------------------------

pt_status pt_matmult_a11_d(pt_op *op, const double *x, double *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!x || !y) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if (x == y) return fail(PT_ERR_BAD_ARG, "x and y must not alias");
  if ((s = launch_a11<double>(op, op->d_coords, op->d_eta, x, y, op->has_mask)) != PT_OK) return s;
  if (a11_sets_bc_rows(op)) return PT_OK;
  return bc_copy(op, x, y);
}

pt_status pt_matmult_a11_h(pt_op *op, const double *x, double *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  bool done = false;
  if (x && y && op->has_mask && (s = a11_host_pipelined<true>(op, x, y, &done)) != PT_OK) return s;
  if (done) return PT_OK;
  return host_call(op, x, op->nvel, op->d_u, y, op->nvel, op->d_y,
                   [&]() { return pt_matmult_a11_d(op, op->d_u, op->d_y); });
}

pt_status pt_matmult_a11_f32_d(pt_op *op, const float *x, float *y)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!x || !y) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if (x == y) return fail(PT_ERR_BAD_ARG, "x and y must not alias");
  if ((s = launch_a11<float>(op, op->d_coords32, op->d_eta32, x, y, op->has_mask)) != PT_OK) return s;
  if (a11_sets_bc_rows(op)) return PT_OK;
  return bc_copy32(op, x, y);
}

pt_status pt_getdiag_a11_d(pt_op *op, double *d)
{
  pt_status s = pt_a11_diag_d(op, d);
  if (s != PT_OK) return s;
  return bc_value(op, 1.0, d);
}

pt_status pt_getdiag_a11_h(pt_op *op, double *d)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, nullptr, 0, nullptr, d, op->nvel, op->d_y, [&]() { return pt_getdiag_a11_d(op, op->d_y); });
}

pt_status pt_matmult_a12_d(pt_op *op, const double *p, double *yu)
{
  pt_status s = pt_a12_apply_d(op, p, yu);
  if (s != PT_OK) return s;
  return bc_value(op, 0.0, yu);
}

pt_status pt_matmult_a12_h(pt_op *op, const double *p, double *yu)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, p, op->npres, op->d_p, yu, op->nvel, op->d_y, [&]() { return pt_matmult_a12_d(op, op->d_p, op->d_y); });
}

pt_status pt_matmult_a21_d(pt_op *op, const double *u, double *yp)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if (!u || !yp) return fail(PT_ERR_BAD_ARG, "NULL vector");
  return a21_d(op, u, yp, op->has_mask);
}

pt_status pt_matmult_a21_h(pt_op *op, const double *u, double *yp)
{
  pt_status s = check_ready(op, false);
  if (s != PT_OK) return s;
  if ((s = ensure_staging(op)) != PT_OK) return s;
  return host_call(op, u, op->nvel, op->d_u, yp, op->npres, op->d_p, [&]() { return pt_matmult_a21_d(op, op->d_u, op->d_p); });
}

// ---- the whole Stokes operator ---------------------------------------------

pt_status pt_stokes_a_apply_d(pt_op *op, const double *u, const double *p, double *yu, double *yp)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!u || !p || !yu || !yp) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if (u == yu) return fail(PT_ERR_BAD_ARG, "u and yu must not alias");
  if ((s = launch_a11<double>(op, op->d_coords, op->d_eta, u, yu, false)) != PT_OK) return s;
  if ((s = a12_d(op, p, yu, true)) != PT_OK) return s;
  return a21_d(op, u, yp, false);
}

pt_status pt_matmult_a_d(pt_op *op, const double *xu, const double *xp, double *yu, double *yp)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!xu || !xp || !yu || !yp) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if (xu == yu) return fail(PT_ERR_BAD_ARG, "xu and yu must not alias");
  // Dirichlet columns zeroed inside the masked kernels; rows set back to x after B^T p
  if ((s = launch_a11<double>(op, op->d_coords, op->d_eta, xu, yu, op->has_mask)) != PT_OK) return s;
  if ((s = a12_d(op, xp, yu, true)) != PT_OK) return s;
  if ((s = bc_copy(op, xu, yu)) != PT_OK) return s;
  return a21_d(op, xu, yp, op->has_mask);
}

static pt_status stokes_host(pt_op *op, const double *u, const double *p, double *yu, double *yp, bool matshell)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!u || !p || !yu || !yp) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if ((s = ensure_staging(op)) != PT_OK) return s;
  double *dyp = op->d_yp;
  cudaError_t e = cudaMemcpyAsync(op->d_u, u, sizeof(double) * op->nvel, cudaMemcpyHostToDevice, op->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(op->d_p, p, sizeof(double) * op->npres, cudaMemcpyHostToDevice, op->stream);
  if (e == cudaSuccess) {
    s = matshell ? pt_matmult_a_d(op, op->d_u, op->d_p, op->d_y, dyp) : pt_stokes_a_apply_d(op, op->d_u, op->d_p, op->d_y, dyp);
    if (s == PT_OK) e = cudaMemcpyAsync(yu, op->d_y, sizeof(double) * op->nvel, cudaMemcpyDeviceToHost, op->stream);
    if (s == PT_OK && e == cudaSuccess)
      e = cudaMemcpyAsync(yp, dyp, sizeof(double) * op->npres, cudaMemcpyDeviceToHost, op->stream);
    if (s == PT_OK && e == cudaSuccess) e = cudaStreamSynchronize(op->stream);
  }
  if (s != PT_OK) return s;
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "Stokes operator host call: %s", cudaGetErrorString(e));
  return PT_OK;
}

pt_status pt_stokes_a_apply_h(pt_op *op, const double *u, const double *p, double *yu, double *yp)
{
  return stokes_host(op, u, p, yu, yp, false);
}

pt_status pt_matmult_a_h(pt_op *op, const double *xu, const double *xp, double *yu, double *yp)
{
  return stokes_host(op, xu, xp, yu, yp, true);
}

// ---- momentum residual (FormFunctionLocal_U) ---------------------------------

static pt_status fu_alloc(pt_op *op)
{
  if (!op->d_fu) PT_CUDA(op_alloc(op, (void **)&op->d_fu, sizeof(double) * 3 * 27 * op->nel));
  return PT_OK;
}

pt_status pt_op_set_body_force_h(pt_op *op, const double *fu)
{
  if (!op || !fu) return fail(PT_ERR_BAD_ARG, "NULL argument");
  pt_status s = fu_alloc(op);
  if (s != PT_OK) return s;
  PT_CUDA(cudaMemcpyAsync(op->d_fu, fu, sizeof(double) * 3 * 27 * op->nel, cudaMemcpyHostToDevice, op->stream));
  PT_CUDA(cudaStreamSynchronize(op->stream));
  op->has_fu = true;
  op->F_valid = false;
  return PT_OK;
}

pt_status pt_op_set_body_force_d(pt_op *op, const double *fu)
{
  if (!op || !fu) return fail(PT_ERR_BAD_ARG, "NULL argument");
  pt_status s = fu_alloc(op);
  if (s != PT_OK) return s;
  PT_CUDA(cudaMemcpyAsync(op->d_fu, fu, sizeof(double) * 3 * 27 * op->nel, cudaMemcpyDeviceToDevice, op->stream));
  op->has_fu = true;
  op->F_valid = false;
  return PT_OK;
}

pt_status pt_op_set_body_force_strided_h(pt_op *op, const double *fu0, int64_t stride)
{
  if (!op || !fu0) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (stride < 3) return fail(PT_ERR_BAD_ARG, "stride must be >= 3 (got %lld)", (long long)stride);
  const int64_t nq = 27 * op->nel;
  std::vector<double> tmp((size_t)(3 * nq));
  for (int64_t i = 0; i < nq; i++)
    for (int c = 0; c < 3; c++) tmp[(size_t)(3 * i + c)] = fu0[i * stride + c];
  return pt_op_set_body_force_h(op, tmp.data());
}

// F = the body-force load vector of the current coordinates and body force.
static pt_status ensure_body_force(pt_op *op)
{
  if (op->F_valid) return PT_OK;
  if (!op->d_F) PT_CUDA(op_alloc(op, (void **)&op->d_F, sizeof(double) * op->nvel));
  PT_CUDA(cudaMemsetAsync(op->d_F, 0, sizeof(double) * op->nvel, op->stream));
  for (int c = 0; c < 8; c++) {
    ptk::ColourGrid g = ptk::colour_grid(op->box, c);
    const int64_t n = (int64_t)g.ncx * g.ncy * g.ncz;
    if (n == 0) continue;
    ptk::body_force_colour_kernel<<<nblocks(n), TPB, 0, op->stream>>>(g, op->d_coords, op->d_fu, op->d_F);
    PT_LAUNCHED(op);
  }
  op->F_valid = true;
  return PT_OK;
}

pt_status pt_residual_u_d(pt_op *op, const double *u, const double *p, double *ru)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!op->has_fu) return fail(PT_ERR_STATE, "body force not set (pt_op_set_body_force_*)");
  if (!u || !p || !ru) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if (u == ru) return fail(PT_ERR_BAD_ARG, "u and ru must not alias");
  // u as given (the caller inserted the Dirichlet values): no column rule
  if ((s = launch_a11<double>(op, op->d_coords, op->d_eta, u, ru, false)) != PT_OK) return s;
  if ((s = a12_d(op, p, ru, true)) != PT_OK) return s;
  if ((s = ensure_body_force(op)) != PT_OK) return s;
  sub_kernel<<<grid_stride_blocks(op->nvel), 256, 0, op->stream>>>(op->d_F, ru, op->nvel);
  PT_LAUNCHED(op);
  return PT_OK;
}

pt_status pt_residual_u_h(pt_op *op, const double *u, const double *p, double *ru)
{
  pt_status s = check_ready(op, true);
  if (s != PT_OK) return s;
  if (!u || !p || !ru) return fail(PT_ERR_BAD_ARG, "NULL vector");
  if ((s = ensure_staging(op)) != PT_OK) return s;
  PT_CUDA(cudaMemcpyAsync(op->d_u, u, sizeof(double) * op->nvel, cudaMemcpyHostToDevice, op->stream));
  PT_CUDA(cudaMemcpyAsync(op->d_p, p, sizeof(double) * op->npres, cudaMemcpyHostToDevice, op->stream));
  if ((s = pt_residual_u_d(op, op->d_u, op->d_p, op->d_y)) != PT_OK) return s;
  PT_CUDA(cudaMemcpyAsync(ru, op->d_y, sizeof(double) * op->nvel, cudaMemcpyDeviceToHost, op->stream));
  PT_CUDA(cudaStreamSynchronize(op->stream));
  return PT_OK;
}

// ---- marker -> Gauss-point coefficients --------------------------------------

pt_status pt_project_markers_d(pt_op *op, int64_t n, const int32_t *wil, const double *xi, const double *eta,
                               const double *rho, double *eta_qp, double *rho_qp, int install)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (n < 0 || n > INT32_MAX) return fail(PT_ERR_BAD_ARG, "marker count must be in [0, 2^31)");
  if (n > 0 && (!wil || !xi || !eta || !rho)) return fail(PT_ERR_BAD_ARG, "NULL marker array");
  const cudaStream_t st = op->stream;
  const int64_t nel = op->nel;
  const int64_t nn = (int64_t)(2 * op->mx + 1) * (2 * op->my + 1) * (2 * op->mz + 1);
  if (nn > INT32_MAX) return fail(PT_ERR_BAD_ARG, "marker projection: element box has 2^31 nodes or more");
  // keys in [0, nel], nel standing for "outside the box": sort over nel's bits
  int bits = 1;
  while (bits < 31 && (int64_t(1) << bits) <= nel) bits++;
  // scratch (op-owned, grown on demand and reused): keys in and sorted, marker
  // indices in and sorted, starts, element partials, node values, qp outputs
  // when the caller passes none, sort workspace
  const int64_t nm = n > 0 ? n : 1;
  size_t tmp_bytes = 0;
  cudaError_t e = cudaSuccess;
  if (n > 0)
    e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (const int32_t *)nullptr, (int32_t *)nullptr,
                                        (const int32_t *)nullptr, (int32_t *)nullptr, (int)n, 0, bits, st);
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "marker projection: %s", cudaGetErrorString(e));
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t sz[9] = {up(4 * nm),         up(4 * nm),     up(4 * nm),
                        up(8 * (nel + 1)),   up(8 * 81 * nel), up(8 * 2 * nn),
                        eta_qp ? 0 : up(8 * 27 * nel), up(tmp_bytes), up(4 * nm)};
  size_t total = 0;
  for (size_t b : sz) total += b;
  if (total > op->mk_bytes) {
    op_free(op, op->mk_scratch);
    op->mk_scratch = nullptr;
    op->mk_bytes = 0;
    PT_CUDA(op_alloc(op, &op->mk_scratch, total));
    op->mk_bytes = total;
  }
  char *cur = (char *)op->mk_scratch;
  void *ptrs[9];
  for (int i = 0; i < 9; i++) {
    ptrs[i] = sz[i] ? cur : nullptr;
    cur += sz[i];
  }
  int32_t *keys = (int32_t *)ptrs[0], *iota = (int32_t *)ptrs[1], *order = (int32_t *)ptrs[2];
  int64_t *start = (int64_t *)ptrs[3];
  double *part = (double *)ptrs[4], *v1 = (double *)ptrs[5];
  double *eq = eta_qp ? eta_qp : (double *)ptrs[6], *rq = rho_qp;
  void *tmp = ptrs[7];
  int32_t *kin = (int32_t *)ptrs[8];
  pt_status s = PT_OK;
  if (e == cudaSuccess) {
    if (n > 0) {
      ptk::mk_keys_kernel<<<grid_stride_blocks(n), 256, 0, st>>>(wil, n, (int32_t)nel, kin, iota);
      e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kin, keys, iota, order, (int)n, 0, bits, st);
    }
    if (e == cudaSuccess) {
      ptk::mk_starts_kernel<<<grid_stride_blocks(nel + 1), 256, 0, st>>>(keys, n, nel, start);
      ptk::mk_element_kernel<<<nblocks(32 * nel), TPB, 0, st>>>(nel, start, order, xi, eta, rho, part);
      ptk::mk_node_kernel<<<grid_stride_blocks(nn), 256, 0, st>>>(op->mx, op->my, op->mz, part, v1, v1 + nn);
      ptk::mk_qp_kernel<<<nblocks(32 * nel), TPB, 0, st>>>(op->mx, op->my, op->mz, v1, v1 + nn, eq, rq);
      e = cudaGetLastError();
      op->launches += 4 + (n > 0 ? 2 : 0);
    }
    // markers outside the element box (key nel, sorted last) are not
    // projected: report them
    int64_t inside = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&inside, start + nel, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && install) s = pt_op_set_eta_d(op, eq);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && s == PT_OK && inside != n)
      s = fail(PT_ERR_BAD_ARG, "%lld markers have an element index outside [0, %lld)", (long long)(n - inside),
               (long long)nel);
  }
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "marker projection: %s", cudaGetErrorString(e));
  return s;
}

pt_status pt_project_markers_h(pt_op *op, int64_t n, const int32_t *wil, const double *xi, const double *eta,
                               const double *rho, double *eta_qp, double *rho_qp, int install)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (n < 0 || n > INT32_MAX) return fail(PT_ERR_BAD_ARG, "marker count must be in [0, 2^31)");
  if (n > 0 && (!wil || !xi || !eta || !rho)) return fail(PT_ERR_BAD_ARG, "NULL marker array");
  const cudaStream_t st = op->stream;
  const int64_t nm = n > 0 ? n : 1, nq = 27 * op->nel;
  int32_t *dw = nullptr;
  double *dx = nullptr, *de = nullptr, *dr = nullptr, *deq = nullptr, *drq = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&dw, sizeof(int32_t) * nm, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&dx, sizeof(double) * 3 * nm, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&de, sizeof(double) * nm, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&dr, sizeof(double) * nm, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&deq, sizeof(double) * nq, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&drq, sizeof(double) * nq, st);
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(dw, wil, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(dx, xi, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(de, eta, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(dr, rho, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  pt_status s = PT_OK;
  if (e == cudaSuccess) s = pt_project_markers_d(op, n, dw, dx, de, dr, deq, drq, install);
  if (e == cudaSuccess && s == PT_OK && eta_qp)
    e = cudaMemcpyAsync(eta_qp, deq, sizeof(double) * nq, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && s == PT_OK && rho_qp)
    e = cudaMemcpyAsync(rho_qp, drq, sizeof(double) * nq, cudaMemcpyDeviceToHost, st);
  void *bufs[] = {dw, dx, de, dr, deq, drq};
  for (void *b : bufs)
    if (b) cudaFreeAsync(b, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "marker projection: %s", cudaGetErrorString(e));
  return s;
}

pt_status pt_op_set_a11_kernel(pt_op *op, const char *name)
{
  if (!op || !name) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (!strcmp(name, "b200")) op->a11_kernel = (op->full_box && op->nel <= EBE_AUTO_MAX_ELEMENTS) ? A11_EBE : A11_STREAM;
  else if (!strcmp(name, "b200_stream")) op->a11_kernel = A11_STREAM;
  else if (!strcmp(name, "b200_ebe")) op->a11_kernel = A11_EBE;
  else if (!strcmp(name, "b200_colour")) op->a11_kernel = A11_COLOUR;
  else return fail(PT_ERR_BAD_ARG, "No -a11_op %s", name);
  return PT_OK;
}

pt_status pt_op_set_tiling(pt_op *op, int32_t lz)
{
  if (!op) return fail(PT_ERR_BAD_ARG, "op is NULL");
  if (lz < 0) return fail(PT_ERR_BAD_ARG, "lz must be >= 0");
  if (lz == 0) {  // the default: about 2048 CTAs, at least 2 layers per z-chunk where possible
    const int64_t txy = (int64_t)op->ntx * op->my;
    int nzc = (int)((2048 + txy - 1) / txy);
    nzc = nzc < 1 ? 1 : (nzc > (op->mz + 1) / 2 ? (op->mz + 1) / 2 : nzc);
    if (nzc < 1) nzc = 1;
    lz = (op->mz + nzc - 1) / nzc;
  }
  op->LZ = lz < op->mz ? lz : op->mz;
  op->nzc = (op->mz + op->LZ - 1) / op->LZ;
  return PT_OK;
}

int32_t pt_op_get_tiling(const pt_op *op) { return op ? op->LZ : 0; }

const char *pt_op_get_a11_kernel(const pt_op *op)
{
  if (!op) return "";
  switch (op->a11_kernel) {
    case A11_STREAM: return "b200_stream";
    case A11_EBE: return "b200_ebe";
    default: return "b200_colour";
  }
}

int64_t pt_op_launch_count(const pt_op *op) { return op ? op->launches : 0; }
void pt_op_reset_launch_count(pt_op *op)
{
  if (op) op->launches = 0;
}

}  // extern "C"

// ============================================================================
// A11 apply that allocates nothing (pt_a11_apply_noalloc_d).
//
// Some callers cannot ask the CUDA allocator for memory at the moment they
// need the operator: applications that hand the whole device to their own
// fixed-size memory pool up front (an extra cudaMalloc then simply fails),
// processes running under a hard device-memory limit that is already used up,
// and latency-critical paths that must not take cudaMalloc/cudaFree's
// device-wide synchronisation.  For them this entry point
// runs the streaming kernel on caller-owned coordinates, viscosity, input and
// output, and keeps the kernel's scratch -- the Gauss-point geometry factor K
// and the set-up check counter -- in file-scope device arrays of fixed size
// that every GPU loading this library holds until the process exits.
// ============================================================================

namespace {

// Capacity of the scratch K array, in doubles: 2^21 (16 MiB).  A mesh fits
// when my*mz*243*MXP <= this, MXP = mx rounded up to the tile width (32, 64 or
// a multiple of 128); a 16^3 box needs 1,990,656.
constexpr int64_t NOALLOC_K_CAP = (int64_t)1 << 21;

__device__ __align__(256) double g_noalloc_K[NOALLOC_K_CAP];
__device__ __align__(256) unsigned int g_noalloc_bad[64];

struct NoallocDev {
  double *K;
  unsigned int *bad;
  bool ready;
};
NoallocDev g_noalloc[64];
std::mutex g_noalloc_mu;

// Device addresses of the scratch arrays for the current device, looked up
// once per device with that device current.  The host-side names of the
// arrays are not device addresses; kernels only ever get these pointers.
pt_status noalloc_scratch(int dev, double **K, unsigned int **bad)
{
  if (dev < 0 || dev >= 64) return fail(PT_ERR_UNSUPPORTED, "device index %d beyond 63", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocDev &d = g_noalloc[dev];
  if (!d.ready) {
    cudaError_t e = cudaGetSymbolAddress((void **)&d.K, g_noalloc_K);
    if (e != cudaSuccess) return fail(PT_ERR_CUDA, "cudaGetSymbolAddress(K scratch): %s", cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void **)&d.bad, g_noalloc_bad);
    if (e != cudaSuccess) return fail(PT_ERR_CUDA, "cudaGetSymbolAddress(check counter): %s", cudaGetErrorString(e));
    d.ready = true;
  }
  *K = d.K;
  *bad = d.bad;
  return PT_OK;
}

template <int TX>
pt_status noalloc_launch(const ptk::StreamGrid &g0, int my, const double *K, const double *u, double *y,
                         cudaStream_t stream)
{
  constexpr size_t smem = ptk::stream_smem_bytes<double, TX>();
  pt_status as = kernel_attrs((const void *)ptk::a11_stream_kernel<double, TX, false>, smem);
  if (as != PT_OK) return as;
  ptk::StreamGrid g = g0;
  for (int pz = 0; pz < 2; pz++)
    for (int py = 0; py < 2; py++)
      for (int px = 0; px < 2; px++) {
        g.px = px; g.py = py; g.pz = pz;
        g.nxc = (g.ntx - px + 1) / 2;
        g.nyc = (my - py + 1) / 2;
        g.nzcc = (g.nzc - pz + 1) / 2;
        g.zc0 = pz;
        const int64_t n = (int64_t)g.nxc * g.nyc * g.nzcc;
        if (n == 0) continue;
        ptk::a11_stream_kernel<double, TX, false><<<(unsigned)n, TX, smem, stream>>>(g, K, u, nullptr, y);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(PT_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
      }
  return PT_OK;
}

}  // namespace

extern "C" pt_status pt_a11_apply_noalloc_d(const pt_mesh_desc *desc, const double *coords, const double *eta,
                                            const double *u, double *y, void *stream)
{
  if (!desc || !coords || !eta || !u || !y) return fail(PT_ERR_BAD_ARG, "NULL argument");
  if (desc->mx < 1 || desc->my < 1 || desc->mz < 1)
    return fail(PT_ERR_BAD_ARG, "element counts must be >= 1 (got %d x %d x %d)", desc->mx, desc->my, desc->mz);
  const int64_t nx = 2 * (int64_t)desc->mx + 1, ny = 2 * (int64_t)desc->my + 1, nz = 2 * (int64_t)desc->mz + 1;
  if ((desc->nx && desc->nx != nx) || (desc->ny && desc->ny != ny) || (desc->nz && desc->nz != nz) || desc->ox ||
      desc->oy || desc->oz)
    return fail(PT_ERR_UNSUPPORTED, "pt_a11_apply_noalloc_d takes one-rank boxes only (node box 2m+1, no offset)");
  const int TX = desc->mx <= 32 ? 32 : (desc->mx <= 64 ? 64 : 128);
  const int ntx = (desc->mx + TX - 1) / TX;
  const int64_t MXP = (int64_t)ntx * TX;
  const int64_t nk = (int64_t)desc->my * desc->mz * 243 * MXP;
  if (nk > NOALLOC_K_CAP)
    return fail(PT_ERR_BAD_ARG,
                "mesh %d x %d x %d needs %lld doubles of geometry scratch; pt_a11_apply_noalloc_d holds %lld "
                "(e.g. 16 x 16 x 16); use an op (pt_op_create) for larger meshes",
                desc->mx, desc->my, desc->mz, (long long)nk, (long long)NOALLOC_K_CAP);
  int dev = 0;
  PT_CUDA(cudaGetDevice(&dev));
  double *K = nullptr;
  unsigned int *bad = nullptr;
  pt_status s = noalloc_scratch(dev, &K, &bad);
  if (s != PT_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;

  ptk::Box bx;
  bx.mx = desc->mx; bx.my = desc->my; bx.mz = desc->mz;
  bx.X = nx; bx.XY = nx * ny; bx.off = 0;
  const int64_t nel = (int64_t)desc->mx * desc->my * desc->mz;
  // the counter keeps the previous call's value: clear it first
  PT_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), st));
  ptk::geom_kernel<double><<<nblocks(nel), TPB, 0, st>>>(bx, MXP, coords, eta, K, bad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));

  ptk::StreamGrid g;
  g.b = bx;
  g.TX = TX; g.ntx = ntx; g.MXP = MXP;
  {
    const int64_t txy = (int64_t)ntx * desc->my;
    int nzc = (int)((2048 + txy - 1) / txy);
    nzc = nzc < 1 ? 1 : (nzc > (desc->mz + 1) / 2 ? (desc->mz + 1) / 2 : nzc);
    if (nzc < 1) nzc = 1;
    g.LZ = (desc->mz + nzc - 1) / nzc;
    g.nzc = (desc->mz + g.LZ - 1) / g.LZ;
  }
  if (TX == 32) s = noalloc_launch<32>(g, desc->my, K, u, y, st);
  else if (TX == 64) s = noalloc_launch<64>(g, desc->my, K, u, y, st);
  else s = noalloc_launch<128>(g, desc->my, K, u, y, st);
  if (s != PT_OK) return s;

  // the geometry check: every w*eta/detJ must be positive
  unsigned int nbad = 0;
  PT_CUDA(cudaMemcpyAsync(&nbad, bad, sizeof nbad, cudaMemcpyDeviceToHost, st));
  PT_CUDA(cudaStreamSynchronize(st));
  if (nbad)
    return fail(PT_ERR_BAD_ARG, "%u Gauss points with w*eta/detJ <= 0 (inverted element or non-positive eta); "
                "y is not valid -- use an op, which falls back to the colour kernel", nbad);
  return PT_OK;
}

#include "solver_impl.cuh"
#include "batch_impl.cuh"
#include "server_impl.cuh"
