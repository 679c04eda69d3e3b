"""LBVH broad phase through the C ABI (mirrors engine-gpu's GpuMorton, GpuRadixSort,
GpuKarras, GpuBvhAabb and GpuBvhTraverse, engine-gpu/src/{morton,radix,karras,bvh_aabb,
bvh_traverse}.rs, as one object)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr


class Lbvh:
    def __init__(self, ctx):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        check(self.lib.mguso_lbvh_create(ctx.h, C.byref(h)))
        self.h = h
        ctx.own(self)
        self.nt = 0

    def build(self, pos_dev: int, nv: int, tris_dev: int, nt: int, key_bits: int = 30, stream: int = 0):
        check(self.lib.mguso_lbvh_build(self.h, pos_dev, nv, tris_dev, nt, key_bits, stream))
        self.nt = nt

    def query_points(self, pts_dev: int, npts: int, dhat: float, pairs_dev: int, cap: int, count_dev: int,
                     stream: int = 0):
        check(self.lib.mguso_lbvh_query_points(self.h, pts_dev, npts, C.c_float(dhat), pairs_dev, cap, count_dev,
                                               stream))

    def status(self) -> int:
        return self.lib.mguso_lbvh_status(self.h)

    def download(self):
        nt = self.nt
        keys = np.empty(nt, np.uint64)
        perm = np.empty(nt, np.uint32)
        m = max(nt - 1, 0)
        left = np.empty(max(m, 1), np.uint32)
        right = np.empty(max(m, 1), np.uint32)
        node = np.empty((max(m, 1), 6), np.float32)
        check(self.lib.mguso_lbvh_download(self.h, ptr(keys) if nt else None, ptr(perm) if nt else None,
                                           ptr(left), ptr(right), ptr(node)))
        return keys, perm, left[:m], right[:m], node[:m]

    def stage_times(self, enable: bool = True):
        ms = np.zeros(6, np.float32)
        check(self.lib.mguso_lbvh_stage_times(self.h, 1 if enable else 0, ptr(ms)))
        return dict(zip(["morton", "sort", "karras", "refit", "query_prep", "traverse"], ms.tolist()))

    def close(self):
        if self.h:
            self.lib.mguso_lbvh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_query(ctx, positions: np.ndarray, tris: np.ndarray, key_bits: int, dhat: float, cap: int | None = None):
    """Host-buffer LBVH build + point query. Returns (keys, perm, pairs[count, 2], count)."""
    lib = ctx.lib
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    nv, nt = p.shape[0], t.shape[0]
    if cap is None:
        cap = 8 * nv + 1024
    keys = np.empty(max(nt, 1), np.uint64)
    perm = np.empty(max(nt, 1), np.uint32)
    pairs = np.empty((cap, 2), np.uint32)
    cnt = C.c_uint64()
    rc = lib.mguso_lbvh_build_query(ctx.h, ptr(p), nv, ptr(t), nt, key_bits, C.c_float(dhat), ptr(keys), ptr(perm),
                                    ptr(pairs), cap, C.byref(cnt))
    if rc == 6 and cnt.value > cap:  # PAIR_OVERFLOW: retry with the reported count
        return build_query(ctx, positions, tris, key_bits, dhat, int(cnt.value))
    check(rc)
    return keys[:nt], perm[:nt], pairs[:cnt.value], int(cnt.value)


def radix_sort_pairs(ctx, keys_dev: int, vals_dev: int, n: int, key_bits: int, stream: int = 0):
    check(ctx.lib.mguso_radix_sort_pairs(ctx.h, keys_dev, vals_dev, n, key_bits, stream))


def radix_sort_status(ctx):
    """Waits for the device; raises if the last radix_sort_pairs gave up its look-back wait."""
    check(ctx.lib.mguso_radix_sort_status(ctx.h))


# The allocation-free sort keeps its temporaries in a fixed device array of the library.
NOALLOC_MAX_PAIRS = 1 << 18


def radix_sort_pairs_noalloc(keys_dev: int, vals_dev: int, n: int, key_bits: int, stream: int = 0):
    """Sorts (key, payload) pairs in place on the current device without allocating device
    memory, for hosts that may not allocate once running (all memory handed to their own
    pool, or no room for cudaMalloc's device-wide synchronisation in a per-frame path).
    n <= NOALLOC_MAX_PAIRS; overlapping calls share the scratch array and race."""
    check(_lib.load().mguso_radix_sort_pairs_noalloc(keys_dev, vals_dev, n, key_bits, stream))
