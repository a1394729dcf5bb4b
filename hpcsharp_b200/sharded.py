"""Sort of one array spread over ranks, one process per GPU (torch.distributed, NCCL).

HPCsharp sorts one array per process: SortRadixPar splits it across host threads
(RadixSortLsdParallel.cs:49-232), never across machines.  `sort_sharded` keeps that result for
an array whose shards live on several GPUs: the concatenation of the ranks' outputs, in rank
order, is the stable LSD sort of the concatenation of their inputs (same order transforms as
the plain sort).  With balance=True rank r ends with as many keys as it started with, so the
array keeps its layout over the ranks, as an in-place sort would.

Steps; every rank takes the same collective steps in the same order:
  1. sizes      all_gather of the shard sizes; element i of rank r's shard has global
                position offset_r + i.
  2. splitters  each rank draws up to `samples` keys at stratified random positions; the
                (key, global position) samples are all-gathered in rank order, every rank
                sorts them with the stable GPU pairs sort and takes world-1 evenly spaced
                ones, so all ranks hold the same splitters.
  3. partition  hpcs_shard_partition_dev: part b = the elements with b splitters at or below
                them in (key order, global position) order; stable.  Equal keys may be split
                between parts, so duplicates cannot overload a rank.
  4. exchange   all_gather of the part sizes, then all_to_all of the keys (and items).
  5. sort       the plain GPU sort of what arrived.  Arrivals are in rank order and each in
                shard order, and the sort is stable, so equal keys stay in global order.
  6. rebalance  (balance=True) one more all_to_all moves contiguous pieces of the sorted runs
                to the ranks whose target slices hold them.

The per-rank kernels sit behind `ops` (DeviceOps: the library's partition and sorts on
torch's current stream).  Collectives go through the default process group, or `group`;
with a backend other than NCCL, device tensors are staged through host memory for each
collective.
"""
from __future__ import annotations

import numpy as np

SIGNED_VIEW = {4: "int32", 8: "int64"}
MAX_PARTS = 64  # HPCS_MAX_PARTS of the C ABI: one part per rank


def _torch():
    import torch

    return torch


class DeviceOps:
    """The per-rank kernels of the sharded sort: hpcs_shard_partition_dev and the plain
    sorts of the library, enqueued on torch's current stream of the tensors' device.  Keys
    arrive as int32 / int64 tensors holding the bytes of `dtype` keys."""

    def __init__(self, ctx, dtype: str):
        self.ctx = ctx
        self.dtype = dtype

    def _stream(self, t) -> int:
        from . import native

        return native.torch_stream(t.device)

    def sort(self, keys) -> None:
        if keys.numel():
            self.ctx.sort_dev(keys, dtype=self.dtype, stream=self._stream(keys))

    def sort_pairs(self, keys, items) -> None:
        if keys.numel():
            self.ctx.sort_pairs_dev(keys, items, dtype=self.dtype, stream=self._stream(keys))

    def partition(self, keys, items, gpos0: int, split_keys, split_gpos, parts: int):
        torch = _torch()
        keys_out = torch.empty_like(keys)
        items_out = torch.empty_like(items) if items is not None else None
        counts = torch.zeros(parts, dtype=torch.int64, device=keys.device)
        if keys.numel():
            self.ctx.shard_partition_dev(keys, items, gpos0, split_keys if parts > 1 else None,
                                         split_gpos if parts > 1 else None, parts, keys_out, items_out, counts,
                                         dtype=self.dtype, stream=self._stream(keys))
        return keys_out, items_out, counts


class _Comm:
    """The collectives of the sharded sort on one process group."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.staged = dist.get_backend(group) != "nccl"

    def _out(self, t):
        return t.cpu() if self.staged and t.is_cuda else t

    def all_gather(self, t) -> list:
        """The world's copies of the equal-sized tensor t, in rank order, on t's device."""
        torch = _torch()
        src = self._out(t.contiguous())
        bufs = [torch.empty_like(src) for _ in range(self.world)]
        self.dist.all_gather(bufs, src, group=self.group)
        return [b.to(t.device) for b in bufs]

    def all_to_all(self, send, send_sizes: list[int], recv_sizes: list[int]):
        torch = _torch()
        src = self._out(send.contiguous())
        out = torch.empty(sum(recv_sizes), dtype=send.dtype, device=src.device)
        self.dist.all_to_all_single(out, src, output_split_sizes=list(recv_sizes),
                                    input_split_sizes=list(send_sizes), group=self.group)
        return out.to(send.device)


def _bits(t):
    """The same bytes as a signed integer tensor (what the collectives move)."""
    torch = _torch()
    return t.view(getattr(torch, SIGNED_VIEW[t.element_size()]))


def sample_positions(n: int, count: int, seed: int, rank: int) -> np.ndarray:
    """`count` stratified random positions in [0, n), ascending: one per stratum of n/count."""
    if count <= 0:
        return np.zeros(0, dtype=np.int64)
    rng = np.random.default_rng([seed, rank])
    u = rng.random(count)
    pos = np.floor((np.arange(count) + u) * (n / count)).astype(np.int64)
    return np.clip(pos, 0, n - 1)


def splitter_indices(total: int, parts: int) -> list[int]:
    """Indices into the sorted sample of the parts-1 splitters (evenly spaced)."""
    return [(j * total) // parts for j in range(1, parts)]


def rebalance_sizes(held: list[int], target: list[int], rank: int) -> tuple[list[int], list[int]]:
    """Sizes of the pieces rank `rank` sends to / receives from each rank when the sorted runs
    of `held` keys per rank (in global order) move to slices of `target` keys per rank."""
    world = len(held)
    hold_at = np.concatenate([[0], np.cumsum(held)]).tolist()
    want_at = np.concatenate([[0], np.cumsum(target)]).tolist()

    def overlap(a0, a1, b0, b1):
        return max(0, min(a1, b1) - max(a0, b0))

    send = [overlap(hold_at[rank], hold_at[rank + 1], want_at[d], want_at[d + 1]) for d in range(world)]
    recv = [overlap(hold_at[s], hold_at[s + 1], want_at[rank], want_at[rank + 1]) for s in range(world)]
    return send, recv


def sort_sharded(keys, items=None, *, ops, group=None, samples: int = 1024, seed: int = 0,
                 balance: bool = True):
    """Stable sort of the array whose rank-order concatenation of shards is `keys`.

    keys: this rank's shard (a 1-D tensor of 4- or 8-byte keys, read as `ops.dtype`);
    items: optional uint32 payload (an int32 tensor of the same length) that moves with its
    key, as in SortRadix(keys, items).  Returns (keys_out, items_out): this rank's slice of the
    sorted array -- with balance=True the slice of global positions this rank's input held,
    otherwise the part chosen by the splitters.  The inputs are not modified."""
    torch = _torch()
    comm = _Comm(group)
    world, rank = comm.world, comm.rank
    if world > MAX_PARTS:
        raise ValueError(f"sort_sharded takes at most {MAX_PARTS} ranks (one partition part per rank)")
    kb = _bits(keys)  # collectives, gathers and the ops see the keys' bytes as int32 / int64
    dev = kb.device
    n = kb.numel()

    # 1. shard sizes and global offsets
    sizes = [int(x) for x in torch.cat(comm.all_gather(torch.tensor([n], dtype=torch.int64, device=dev))).tolist()]
    gpos0 = int(sum(sizes[:rank]))

    # 2. splitters from a stratified sample, identical on every rank
    counts = [min(samples, s) for s in sizes]
    pos_t = torch.from_numpy(sample_positions(n, counts[rank], seed, rank)).to(dev)
    mine_k = torch.zeros(samples, dtype=kb.dtype, device=dev)
    mine_g = torch.zeros(samples, dtype=torch.int64, device=dev)
    if counts[rank]:
        mine_k[:counts[rank]] = kb[pos_t]
        mine_g[:counts[rank]] = pos_t + gpos0
    all_k = comm.all_gather(mine_k)
    all_g = comm.all_gather(mine_g)
    sk = torch.cat([all_k[r][:counts[r]] for r in range(world)]).contiguous()
    sg = torch.cat([all_g[r][:counts[r]] for r in range(world)])
    total = sk.numel()
    if total == 0:  # every shard is empty
        return keys.clone(), (items.clone() if items is not None else None)
    order = torch.arange(total, dtype=torch.int32, device=dev)
    ops.sort_pairs(sk, order)  # stable: equal keys keep ascending global position
    pick = torch.tensor(splitter_indices(total, world), dtype=torch.int64, device=dev)
    split_keys = sk[pick].contiguous()
    split_gpos = sg[order.to(torch.int64)][pick].contiguous()

    # 3. partition this shard
    part_k, part_i, part_n = ops.partition(kb, items, gpos0, split_keys, split_gpos, world)

    # 4. exchange the parts
    matrix = [[int(x) for x in row.tolist()] for row in comm.all_gather(part_n)]  # matrix[src][dst]
    send = matrix[rank]
    recv = [matrix[s][rank] for s in range(world)]
    got_k = comm.all_to_all(part_k, send, recv)
    got_i = comm.all_to_all(part_i, send, recv) if items is not None else None

    # 5. local stable sort of this rank's part
    if got_i is not None:
        ops.sort_pairs(got_k, got_i)
    else:
        ops.sort(got_k)
    if not balance:
        return got_k.view(keys.dtype), got_i

    # 6. move the sorted runs to the input layout
    held = [sum(matrix[s][d] for s in range(world)) for d in range(world)]
    send, recv = rebalance_sizes(held, sizes, rank)
    out_k = comm.all_to_all(got_k, send, recv)
    out_i = comm.all_to_all(got_i, send, recv) if got_i is not None else None
    return out_k.view(keys.dtype), out_i
