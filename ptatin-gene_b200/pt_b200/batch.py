"""Batched A11 over many independent boxes (pt_batch_* in the C ABI), and the
work-list autotuner.

A ``BatchA11`` is built once from a list of set-up ``MatStokesMF`` ops; an apply
is one launch per (colour, tile width) class over the concatenated tile
work-list, and each problem's result is bitwise what its own apply gives.
"""
from __future__ import annotations

import ctypes

from . import _capi


def _ptr_table(tensors, device):
    import torch
    return torch.tensor([t.data_ptr() for t in tensors], dtype=torch.int64, device=device)


class BatchA11:
    def __init__(self, ops, lz=None, tile_x=0):
        self.ops = list(ops)
        n = len(self.ops)
        arr = (ctypes.c_void_p * n)(*[op.handle.value for op in self.ops])
        lzs = None
        if lz is not None:
            vals = [int(lz)] * n if isinstance(lz, int) else [int(v) for v in lz]
            lzs = (ctypes.c_int32 * n)(*vals)
        h = ctypes.c_void_p()
        _capi.call("pt_batch_create_tiled", n, arr, lzs, int(tile_x), ctypes.byref(h))
        self._h = h
        self._tables = {}
        lib = _capi.load()
        self.launches_per_apply = int(lib.pt_batch_launches_per_apply(h))
        self.tiles = int(lib.pt_batch_tiles(h))

    def tables(self, us, ys):
        """Device pointer tables for the given per-problem vectors (cached)."""
        key = (tuple(t.data_ptr() for t in us), tuple(t.data_ptr() for t in ys))
        tab = self._tables.get(key)
        if tab is None:
            tab = (_ptr_table(us, us[0].device), _ptr_table(ys, ys[0].device))
            self._tables[key] = tab
        return tab

    def apply(self, us, ys, masked=True, stream=None):
        """ys[i] = A11_i us[i] (FP64 or FP32 by the tensors' dtype)."""
        import torch
        ut, yt = self.tables(us, ys)
        st = (stream or torch.cuda.current_stream()).cuda_stream
        name = "pt_batch_a11_apply_f32_d" if us[0].dtype == torch.float32 else "pt_batch_a11_apply_d"
        _capi.call(name, self._h, ctypes.c_void_p(ut.data_ptr()), ctypes.c_void_p(yt.data_ptr()), int(masked),
                   ctypes.c_void_p(st))
        return ys

    def destroy(self):
        if getattr(self, "_h", None):
            _capi.call("pt_batch_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass


def autotune_lz(ops, us, ys, candidates=(1, 2, 4, 8, 0), reps=3, masked=True):
    """Pick the z-chunk depth (element layers per tile; 0 = each op's default)
    that makes one batched apply fastest on these problems.  Returns
    (best_lz, {lz: ms})."""
    best, times = autotune(ops, us, ys, lz_candidates=candidates, tile_candidates=(0,), reps=reps, masked=masked)
    return best[0], {lz: t for (lz, _), t in times.items()}


def autotune(ops, us, ys, lz_candidates=(1, 2, 4, 0), tile_candidates=(0, 64), reps=3, masked=True):
    """Pick the tile schedule -- z-chunk depth (element layers per tile; 0 =
    each op's default) and tile width (0 = each op's own) -- that makes one
    batched apply fastest on these problems.  Returns ((lz, tile_x),
    {(lz, tile_x): ms})."""
    import torch
    times = {}
    for lz in lz_candidates:
        for tx in tile_candidates:
            times[(lz, tx)] = _time_batch(ops, us, ys, lz, tx, reps, masked, torch)
    best = min(times, key=times.get)
    return best, times


def _time_batch(ops, us, ys, lz, tile_x, reps, masked, torch):
    """Mean ms of one batched apply under a schedule (CUDA events)."""
    with BatchA11(ops, lz=lz if lz else None, tile_x=tile_x) as b:
        b.apply(us, ys, masked)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(reps):
            b.apply(us, ys, masked)
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / reps
