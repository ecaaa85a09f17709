// Batched A11 over many independent one-rank boxes (the batched and served
// forms).  A pt_batch is a work-list built once from a set of ops: every
// (problem, x-tile, row, z-chunk) tile of every problem, grouped by colour
// (parity of x-tile, row and z-chunk) and tile width.  An apply is one launch
// per non-empty (colour, width) class over the concatenated list -- colours
// run in a fixed order, so the per-node summation order is the same as a
// problem's own apply and each result is bitwise the one it gets alone.
// Included from pt_b200.cu after struct pt_op.
#pragma once

#include <map>
#include <vector>

struct pt_batch {
  int n;
  std::vector<pt_op *> ops;
  ptk::BatchProb *d_probs64, *d_probs32;
  int4 *d_items;
  struct Cls {
    int px, py, pz, TX;
    int64_t off, count;
  };
  std::vector<Cls> classes;
  int64_t tiles;
  // pooled (server) batches: stream-ordered buffers; host copies kept until destroy
  cudaMemPool_t pool;
  cudaStream_t stream;
  std::vector<ptk::BatchProb> h64, h32;
  std::vector<int4> hitems;
};

namespace {

// programmatic: a class after the first of one apply may start on the SMs
// the previous class frees; the tile waits in-kernel before writing y (the
// classes of one apply read the same u, K and mask bits)
template <typename T, int TX, bool MASKED>
pt_status batch_launch_cls(const pt_batch *b, const pt_batch::Cls &c, const T *const *u, T *const *y, cudaStream_t st,
                           bool programmatic)
{
  constexpr size_t smem = ptk::stream_smem_bytes<T, TX>();
  pt_status as = kernel_attrs((const void *)ptk::a11_stream_batch_kernel<T, TX, MASKED>, smem);
  if (as != PT_OK) return as;
  const ptk::BatchProb *probs = std::is_same<T, double>::value ? b->d_probs64 : b->d_probs32;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)c.count);
  cfg.blockDim = dim3(TX);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = programmatic ? pdl : nullptr;
  cfg.numAttrs = programmatic ? 1 : 0;
  const int4 *items = b->d_items + c.off;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, ptk::a11_stream_batch_kernel<T, TX, MASKED>, probs, items, c.px, c.py,
                                           c.pz, u, y);
  if (e != cudaSuccess) return fail(PT_ERR_CUDA, "batched kernel launch: %s", cudaGetErrorString(e));
  return PT_OK;
}

// Dirichlet rows of every masked problem after the colour passes: y_k = x_k
// (blockIdx.y = problem).
template <typename T>
__global__ void batch_bc_kernel(const ptk::BatchProb *__restrict__ probs, const T *const *__restrict__ uptr,
                                T *const *__restrict__ yptr)
{
  const ptk::BatchProb &p = probs[blockIdx.y];
  if (!p.mask) return;
  const T *x = uptr[blockIdx.y];
  T *y = yptr[blockIdx.y];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.nvel; i += (int64_t)gridDim.x * blockDim.x)
    if (p.mask[i]) y[i] = x[i];
}

// MASKED: the MatShell apply of every problem with a mask (columns inside the
// kernel, rows by one more launch).
template <typename T, bool MASKED>
pt_status batch_apply(pt_batch *b, const T *const *u, T *const *y, void *stream)
{
  if (!b || !u || !y) return fail(PT_ERR_BAD_ARG, "NULL argument");
  const cudaStream_t st = (cudaStream_t)stream;
  bool first = true;
  for (const pt_batch::Cls &c : b->classes) {
    pt_status s;
    if (c.TX == 32) s = batch_launch_cls<T, 32, MASKED>(b, c, u, y, st, !first);
    else if (c.TX == 64) s = batch_launch_cls<T, 64, MASKED>(b, c, u, y, st, !first);
    else s = batch_launch_cls<T, 128, MASKED>(b, c, u, y, st, !first);
    if (s != PT_OK) return s;
    first = false;
  }
  if (MASKED) {
    const ptk::BatchProb *probs = std::is_same<T, double>::value ? b->d_probs64 : b->d_probs32;
    batch_bc_kernel<T><<<dim3(32, (unsigned)b->n), 256, 0, st>>>(probs, u, y);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PT_ERR_CUDA, "batched Dirichlet rows: %s", cudaGetErrorString(e));
  }
  return PT_OK;
}

}  // namespace

extern "C" {

// pool == null: cudaMalloc + synchronous upload; else buffers from `pool`
// with asynchronous uploads, both ordered on `stream`.
static pt_status batch_create_impl(int n, pt_op *const *ops, const int32_t *lz, int32_t tile_x, cudaMemPool_t pool,
                                   cudaStream_t stream, pt_batch **out)
{
  if (!out || n < 1 || !ops) return fail(PT_ERR_BAD_ARG, "need n >= 1 ops");
  if (tile_x != 0 && tile_x != 32 && tile_x != 64 && tile_x != 128)
    return fail(PT_ERR_BAD_ARG, "tile_x must be 0, 32, 64 or 128");
  *out = nullptr;
  std::vector<ptk::BatchProb> p64(n), p32(n);
  // class key: (pass, TX) -> items
  std::map<std::pair<int, int>, std::vector<int4>> cls;
  int64_t tiles = 0;
  for (int i = 0; i < n; i++) {
    pt_op *op = ops[i];
    pt_status s = check_ready(op, true);
    if (s != PT_OK) return s;
    if (!op->full_box) return fail(PT_ERR_UNSUPPORTED, "batch problem %d: one-rank boxes only", i);
    if ((s = ensure_geometry(op)) != PT_OK) return s;
    if (!op->geom_ok) return fail(PT_ERR_BAD_ARG, "batch problem %d has w*eta/detJ <= 0 somewhere", i);
    // any tile width covers the box: tiles read K columns ex < mx <= MXP
    const int TX = tile_x ? tile_x : op->TX;
    ptk::BatchProb d;
    d.b = op->box;
    d.ntx = (op->mx + TX - 1) / TX;
    d.MXP = op->MXP;
    int L = (lz && lz[i] > 0) ? lz[i] : op->LZ;
    if (L > op->mz) L = op->mz;
    d.LZ = L;
    d.nzc = (op->mz + L - 1) / L;
    if (op->has_mask && !op->d_mbits) return fail(PT_ERR_STATE, "batch problem %d: mask without its packed bits", i);
    d.mask = op->has_mask ? op->d_mask : nullptr;
    d.mbits = op->has_mask ? op->d_mbits : nullptr;
    d.nvel = op->nvel;
    d.K = op->d_K;
    p64[i] = d;
    d.K = op->d_K32;
    p32[i] = d;
    for (int zc = 0; zc < d.nzc; zc++)
      for (int ej = 0; ej < op->my; ej++)
        for (int tx = 0; tx < d.ntx; tx++) {
          const int pass = (tx & 1) + 2 * (ej & 1) + 4 * (zc & 1);
          cls[{pass, TX}].push_back(make_int4(i, tx, ej, zc));
          tiles++;
        }
  }
  pt_batch *b = new (std::nothrow) pt_batch();
  if (!b) return fail(PT_ERR_OOM, "host allocation failed");
  b->n = n;
  b->ops.assign(ops, ops + n);
  b->tiles = tiles;
  b->pool = pool;
  b->stream = stream;
  std::vector<int4> &all = b->hitems;
  for (auto &kv : cls) {
    pt_batch::Cls c;
    c.px = kv.first.first & 1; c.py = (kv.first.first >> 1) & 1; c.pz = (kv.first.first >> 2) & 1;
    c.TX = kv.first.second;
    c.off = (int64_t)all.size();
    c.count = (int64_t)kv.second.size();
    all.insert(all.end(), kv.second.begin(), kv.second.end());
    b->classes.push_back(c);
  }
  b->h64 = p64;
  b->h32 = p32;
  cudaError_t e;
  const size_t bp = sizeof(ptk::BatchProb) * n, bi = sizeof(int4) * all.size();
  if (pool) {
    e = cudaMallocFromPoolAsync((void **)&b->d_probs64, bp, pool, stream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&b->d_probs32, bp, pool, stream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&b->d_items, bi, pool, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_probs64, b->h64.data(), bp, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_probs32, b->h32.data(), bp, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_items, all.data(), bi, cudaMemcpyHostToDevice, stream);
  } else {
    e = cudaMalloc(&b->d_probs64, bp);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_probs32, bp);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_items, bi);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_probs64, p64.data(), bp, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_probs32, p32.data(), bp, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, all.data(), bi, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    pt_status s = fail(e == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_CUDA, "pt_batch_create: %s",
                       cudaGetErrorString(e));
    pt_batch_destroy(b);
    return s;
  }
  *out = b;
  return PT_OK;
}

pt_status pt_batch_create_tiled(int n, pt_op *const *ops, const int32_t *lz, int32_t tile_x, pt_batch **out)
{
  return batch_create_impl(n, ops, lz, tile_x, nullptr, nullptr, out);
}

pt_status pt_batch_create(int n, pt_op *const *ops, const int32_t *lz, pt_batch **out)
{
  return batch_create_impl(n, ops, lz, 0, nullptr, nullptr, out);
}

pt_status pt_batch_destroy(pt_batch *b)
{
  if (!b) return PT_OK;
  void *bufs[] = {b->d_probs64, b->d_probs32, b->d_items};
  for (void *p : bufs) {
    if (!p) continue;
    if (b->pool) cudaFreeAsync(p, b->stream);
    else cudaFree(p);
  }
  delete b;
  return PT_OK;
}

int64_t pt_batch_launches_per_apply(const pt_batch *b) { return b ? (int64_t)b->classes.size() : 0; }
int64_t pt_batch_tiles(const pt_batch *b) { return b ? b->tiles : 0; }

pt_status pt_batch_a11_apply_d(pt_batch *b, const double *const *u, double *const *y, int masked, void *stream)
{
  return masked ? batch_apply<double, true>(b, u, y, stream) : batch_apply<double, false>(b, u, y, stream);
}

pt_status pt_batch_a11_apply_f32_d(pt_batch *b, const float *const *u, float *const *y, int masked, void *stream)
{
  return masked ? batch_apply<float, true>(b, u, y, stream) : batch_apply<float, false>(b, u, y, stream);
}

}  // extern "C"
