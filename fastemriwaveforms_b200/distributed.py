"""One waveform split across the GPUs of a torch.distributed group.

The output samples of a waveform are independent given the (small) spline
and folded coefficients, so rank r of W sums the samples
[r*C, min((r+1)*C, out_len)) with C = ceil(out_len / W): every rank builds the
splines redundantly (~0.3 ms at one year, 3843 modes), launches only the work
units inside its range, and the forward needs no communication.  With
``gather=True`` the slices are assembled on every rank by one
``all_gather_into_tensor`` (NCCL over NVLink).  In the backward each rank's
adjoint kernels see only its samples, and one ``all_reduce`` (sum) completes
the gradients.  No collective is fused into a kernel: the only exchange steps
are the optional gather and the gradient reduction.

Host-side pieces (``shard_range``, ``restrict_units``, ``clip_seg_start``,
``gather_waveform``, ``reduce_gradients``) are plain functions so that they run
on any backend (gloo on CPU included).
"""
from __future__ import annotations

import numpy as np
import torch

from .summation import InterpolatedModeSum, _upload


def shard_range(out_len: int, rank: int, world: int) -> tuple[int, int]:
    """Samples [lo, hi) owned by `rank`: equal contiguous chunks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    chunk = -(-out_len // world)
    lo = min(rank * chunk, out_len)
    return lo, min(lo + chunk, out_len)


def restrict_units(units: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """Work units {segment, first, end} (flat, 3 per unit) clipped to [lo, hi)."""
    u = np.asarray(units, dtype=np.int32).reshape(-1, 3).copy()
    u[:, 1] = np.maximum(u[:, 1], lo)
    u[:, 2] = np.minimum(u[:, 2], hi)
    return np.ascontiguousarray(u[u[:, 2] > u[:, 1]].reshape(-1))


def clip_seg_start(seg_start: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """Segment sample boundaries clipped to [lo, hi): segments outside become empty."""
    return np.clip(np.asarray(seg_start, dtype=np.int32), lo, hi).astype(np.int32)


def gather_waveform(local: torch.Tensor, out_len: int, rank: int, world: int, group=None) -> torch.Tensor:
    """Assembles the full waveform from every rank's slice (`local` holds this
    rank's samples at their absolute positions)."""
    import torch.distributed as dist

    chunk = -(-out_len // world)
    lo, hi = shard_range(out_len, rank, world)
    mine = torch.zeros(chunk, dtype=local.dtype, device=local.device)
    mine[: hi - lo] = local[lo:hi]
    full = torch.empty(world * chunk, dtype=local.dtype, device=local.device)
    dist.all_gather_into_tensor(torch.view_as_real(full).reshape(-1), torch.view_as_real(mine).reshape(-1),
                                group=group)
    out = local.clone()
    out[:out_len] = full[:out_len]
    return out


def reduce_gradients(tensors, group=None):
    """Sums gradient tensors over the group in place (complex as float pairs)."""
    import torch.distributed as dist

    for t in tensors:
        if t is None:
            continue
        dist.all_reduce(torch.view_as_real(t) if t.is_complex() else t, op=dist.ReduceOp.SUM, group=group)
    return tensors


class ShardedInterpolatedModeSum(InterpolatedModeSum):
    """``InterpolatedModeSum`` whose samples are split across ranks.

    args:
        group: torch.distributed process group (default: the world).
        rank, world: explicit shard (then no process group is needed when
            gather=False and no gradients are reduced).
        gather: assemble the full waveform on every rank (all_gather).
        reduce_grads: sum gradients over the group in the backward.
    """

    def __init__(self, group=None, rank: int | None = None, world: int | None = None, gather: bool = True,
                 reduce_grads: bool = True, **kwargs):
        super().__init__(**kwargs)
        self.group = group
        if rank is None or world is None:
            import torch.distributed as dist

            rank, world = dist.get_rank(group), dist.get_world_size(group)
        self.rank, self.world = int(rank), int(world)
        self.gather = gather
        self.reduce_grads = reduce_grads

    def _prepare(self, *args, **kwargs):
        p = super()._prepare(*args, **kwargs)
        lo, hi = shard_range(p.out_len, self.rank, self.world)
        seg = p.seg
        local = restrict_units(seg.units_host, lo, hi)
        seg.units_host = local
        seg.nunits = len(local) // 3
        seg.d_units = _upload(local if seg.nunits else np.zeros(3, np.int32), p.dev)
        seg.seg_start = clip_seg_start(seg.seg_start, lo, hi)
        if hasattr(seg, "_bwd"):
            del seg._bwd
        p.shard = (lo, hi)
        return p

    def _launch(self, p, out, host_out=None):
        if host_out is not None:
            raise ValueError("host_out is not supported when the waveform is split across ranks.")
        super()._launch(p, out)
        if self.gather and self.world > 1:
            out.copy_(gather_waveform(out, p.out_len, self.rank, self.world, self.group))
        return out

    def _backward_hook(self, p, grad, need_teuk, need_pc):
        g_teuk, g_pc = InterpolatedModeSum._backward(p, grad, need_teuk, need_pc)
        if self.reduce_grads and self.world > 1:
            reduce_gradients([g_teuk, g_pc], self.group)
        return g_teuk, g_pc
