"""Lending and return of the host blocks of the exported fields (no GPU:
the page-locked allocation is replaced by plain memory)."""

import gc

import numpy as np

from nfgs_b200.hostmem import PinnedPool


class _Blk:
    def __init__(self, nbytes):
        self.buf = np.zeros(nbytes, dtype=np.uint8)

    def data_ptr(self):
        return self.buf.ctypes.data

    def numel(self):
        return self.buf.size


class _Pool(PinnedPool):
    allocs = 0

    def _alloc(self, nbytes):
        type(self).allocs += 1
        return _Blk(nbytes)


def test_block_reused_after_release():
    pool = _Pool(limit=2)
    a = pool.empty(1000, np.float32)
    assert a.dtype == np.float32 and a.shape == (1000,) and a.flags.writeable
    a[:] = 3.0
    ptr = a.ctypes.data
    view = a.reshape(10, 100)[2]
    del a
    gc.collect()
    assert pool.lent == 1          # the view still holds the block
    del view
    gc.collect()
    assert pool.lent == 0
    b = pool.empty(1000, np.float32)
    assert b.ctypes.data == ptr and _Pool.allocs == 1


def test_limit_falls_back():
    pool = _Pool(limit=2)
    a = pool.empty(10, np.float64)
    b = pool.empty(10, np.float64)
    assert a is not None and b is not None
    assert pool.empty(10, np.float64) is None   # the caller takes pageable memory
    del a
    gc.collect()
    assert pool.empty(10, np.float64) is not None


def test_allocation_failure_returns_none():
    class Failing(PinnedPool):
        def _alloc(self, nbytes):
            raise RuntimeError("no pinned memory")

    pool = Failing()
    assert pool.empty(10, np.float32) is None and pool.lent == 0
