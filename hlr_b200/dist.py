"""Row-sharded product of one H-matrix over several GPUs, one process per GPU.

The rows (internal ordering) are cut into contiguous ranges of about equal
stored bytes, at positions that no leaf block straddles: boundaries of row
clusters.  Rank r owns the leaves of its rows, a rectangular
(r1 - r0) x n H-matrix, and the matching slice of every vector.  This is the
per-cluster ownership of y in HLR's cluster-wise product (``mul_vec_cl``,
tbb/detail/arith.hh:406-448), spread over processes instead of threads.
Each product has one exchange step:

* op N: y_r += alpha A_r x needs all of x, so the ranks' slices of x are
  all-gathered first;
* op T / C: y += alpha A^T x is the sum over ranks of A_r^T x_r, a vector of
  full length per rank, so the partial results are summed across ranks and
  each rank keeps its slice (reduce-scatter on NCCL, all-reduce elsewhere).

The collectives go through ``torch.distributed``.  The local product is the
caller's: ``hlr_b200.mul_vec`` on the rank's uploaded shard (see
``upload_shard``), or any function with the same meaning.  Square matrices
only: x and y share one partition.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence

from . import _capi

LocalMul = Callable[[float, int, object, object], None]   # (alpha, op, x, y): y += alpha op(A_r) x


def _blocks(desc) -> List[_capi.hlrc_block]:
    return [desc.blocks[i] for i in range(int(desc.nblocks))]


def _block_bytes(b: _capi.hlrc_block) -> int:
    if b.kind == 0:   # dense
        return 8 * int(b.nrows) * int(b.ncols)
    return 8 * int(b.rank) * (int(b.nrows) + int(b.ncols))


def row_cuts(src, parts: int) -> List[int]:
    """Cut positions 0 = c_0 <= c_1 <= ... <= c_parts = nrows of an H-matrix
    (HostMatrix, LeafList or ``hlrc_h_desc``): no leaf block straddles a
    cut, and the stored bytes of the leaves between consecutive cuts are
    about equal (``hlrc_row_cuts``).  Shards may be empty when there are
    fewer cut positions than parts."""
    from . import check, lib
    if parts < 1:
        raise ValueError("parts must be >= 1")
    desc = src.h_desc() if hasattr(src, "h_desc") else src
    out = (C.c_int64 * (parts + 1))()
    check(lib().hlrc_row_cuts(C.byref(desc), parts, out), "hlrc_row_cuts")
    return [int(c) for c in out]


def shard_desc(src, r0: int, r1: int) -> _capi.hlrc_h_desc:
    """The leaves of rows [r0, r1) as an (r1 - r0) x ncols H-matrix
    descriptor (rows shifted by -r0; the leaf data is shared with ``src``,
    which must outlive the descriptor).  Raises if a leaf straddles r0 or
    r1."""
    desc = src.h_desc() if hasattr(src, "h_desc") else src
    if not 0 <= r0 <= r1 <= int(desc.nrows):
        raise ValueError("bad row range")
    mine = []
    for b in _blocks(desc):
        b0, b1 = int(b.row0), int(b.row0) + int(b.nrows)
        if b1 <= r0 or b0 >= r1:
            continue
        if b0 < r0 or b1 > r1:
            raise ValueError(f"leaf rows [{b0}, {b1}) straddle the shard [{r0}, {r1})")
        c = _capi.hlrc_block.from_buffer_copy(b)
        c.row0 = b0 - r0
        mine.append(c)
    arr = (_capi.hlrc_block * max(1, len(mine)))(*mine)
    d = _capi.hlrc_h_desc()
    d.nrows, d.ncols, d.nblocks = r1 - r0, int(desc.ncols), len(mine)
    d.blocks = C.cast(arr, C.POINTER(_capi.hlrc_block))
    d._owner = (src, desc, arr)
    return d


def upload_shard(src, cuts: Sequence[int], rank: int, **upload_kw):
    """Uploads rank ``rank``'s shard (rows [cuts[rank], cuts[rank+1])) with
    ``hlr_b200.upload`` and returns the device matrix."""
    from . import upload
    return upload(shard_desc(src, int(cuts[rank]), int(cuts[rank + 1])), **upload_kw)


class RowShards:
    """One rank's view of a row partition ``cuts`` and the collectives of
    the sharded product.  ``group`` is a torch.distributed process group
    (None: the default group; with world size 1 no collective runs)."""

    def __init__(self, cuts: Sequence[int], rank: int, world: int, group=None):
        if len(cuts) != world + 1 or list(cuts) != sorted(cuts) or cuts[0] != 0:
            raise ValueError("cuts must be world + 1 non-decreasing positions starting at 0")
        if not 0 <= rank < world:
            raise ValueError("rank out of range")
        self.cuts = [int(c) for c in cuts]
        self.rank, self.world, self.group = rank, world, group
        self.n = self.cuts[-1]
        self.r0, self.r1 = self.cuts[rank], self.cuts[rank + 1]
        self.width = max(self.cuts[i + 1] - self.cuts[i] for i in range(world))

    def _nccl(self) -> bool:
        import torch.distributed as dist
        return dist.get_backend(self.group) == "nccl"

    def gather(self, x_local):
        """All of x from the ranks' slices (one all-gather of padded slices)."""
        import torch
        import torch.distributed as dist
        if x_local.shape[0] != self.r1 - self.r0:
            raise ValueError("x_local does not match this rank's rows")
        if self.world == 1:
            return x_local
        pad = torch.zeros(self.width, dtype=x_local.dtype, device=x_local.device)
        pad[: x_local.shape[0]] = x_local
        if self._nccl():   # one contiguous buffer: no gather list, and no copy when the shards are equal
            buf = torch.empty(self.world * self.width, dtype=x_local.dtype, device=x_local.device)
            dist.all_gather_into_tensor(buf, pad, group=self.group)
            if self.world * self.width == self.n:
                return buf
            parts = [buf[i * self.width:(i + 1) * self.width] for i in range(self.world)]
        else:
            parts = [torch.empty_like(pad) for _ in range(self.world)]
            dist.all_gather(parts, pad, group=self.group)
        return torch.cat([parts[i][: self.cuts[i + 1] - self.cuts[i]] for i in range(self.world)])

    def reduce(self, part):
        """This rank's slice of the sum over ranks of full-length vectors."""
        import torch
        import torch.distributed as dist
        if part.shape[0] != self.n:
            raise ValueError("partial result must have full length")
        if self.world == 1:
            return part
        if self._nccl():
            buf = torch.zeros(self.world * self.width, dtype=part.dtype, device=part.device)
            for i in range(self.world):
                a, b = self.cuts[i], self.cuts[i + 1]
                buf[i * self.width: i * self.width + (b - a)] = part[a:b]
            out = torch.empty(self.width, dtype=part.dtype, device=part.device)
            dist.reduce_scatter_tensor(out, buf, group=self.group)
            return out[: self.r1 - self.r0]
        dist.all_reduce(part, group=self.group)
        return part[self.r0:self.r1]

    def mul_vec(self, alpha: float, op: int, local_mul: LocalMul, x_local, y_local,
                scratch: Optional[object] = None) -> None:
        """y_local += alpha op(M) x over the whole matrix, this rank's part:
        ``local_mul(alpha, op, x, y)`` applies the rank's shard A_r (rows
        [r0, r1)); x_local / y_local are this rank's slices of x and y.  For
        op T / C a full-length scratch vector can be passed (zeroed here)."""
        import torch
        if alpha == 0.0:
            return
        if op == 0:
            local_mul(alpha, 0, self.gather(x_local), y_local)
            return
        part = scratch if scratch is not None else torch.zeros(self.n, dtype=y_local.dtype, device=y_local.device)
        part.zero_()
        local_mul(alpha, op, x_local, part)
        y_local += self.reduce(part)
