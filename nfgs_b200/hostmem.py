"""Page-locked host blocks for the exported fields.

`fields_to_numpy` returns the six field volumes in one host block (201 MB
at the benchmark size).  A fresh pageable block is faulted in while the copy
runs, which costs more than the copy itself; a page-locked block that the
device copy can write directly, reused by the next call once the caller has
dropped the arrays of the previous one, costs neither.  The pool lends at
most `LIMIT` blocks at a time and keeps at most `LIMIT` free ones; beyond
that the caller gets pageable memory, so callers that keep many results do
not pin their memory.
"""

from __future__ import annotations

import threading
import weakref

import numpy as np

LIMIT = 2


class _Lease:
    """Owner of one lent block: numpy arrays made from it keep it alive, and
    when the last of them is gone the block returns to the pool."""

    def __init__(self, blk):
        self.blk = blk
        self.__array_interface__ = {"data": (blk.data_ptr(), False), "shape": (blk.numel(),), "typestr": "|u1",
                                    "version": 3}


class PinnedPool:
    def __init__(self, limit: int = LIMIT):
        self.limit = limit
        self.free: dict[int, list] = {}
        self.lent = 0
        self.lock = threading.Lock()

    @staticmethod
    def _alloc(nbytes: int):
        import torch

        return torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)

    def _give_back(self, blk, nbytes: int):
        with self.lock:
            self.lent -= 1
            lst = self.free.setdefault(nbytes, [])
            if len(lst) < self.limit:
                lst.append(blk)

    def empty(self, n: int, dtype) -> np.ndarray | None:
        """A flat array of n elements in a page-locked block, or None when
        the pool has lent its limit or pinned memory is unavailable."""
        dtype = np.dtype(dtype)
        nbytes = int(n) * dtype.itemsize
        with self.lock:
            if self.lent >= self.limit:
                return None
            lst = self.free.get(nbytes)
            blk = lst.pop() if lst else None
            self.lent += 1
        if blk is None:
            try:
                blk = self._alloc(nbytes)
            except Exception:
                with self.lock:
                    self.lent -= 1
                return None
        lease = _Lease(blk)
        weakref.finalize(lease, self._give_back, blk, nbytes)
        return np.asarray(lease).view(dtype)


POOL = PinnedPool()
