"""calc_all_response_fields of one model sharded over the ranks of a
torch.distributed process group (one process per GPU).

GALIC partitions particles over MPI tasks and sums the per-type response
grids with MPI_Allreduce (main.c:201-231, 259-285).  Here every rank
integrates the orbits order[rank::world] and the instantaneous energy of
particles rank::world into its context's fixed-point accumulators
(galic_calc_all_shard), the accumulators are summed as int64 words
(all_reduce SUM: exact, so every rank holds bit for bit what a one-GPU pass
gives), and each rank converts them and evaluates the merit function
(galic_calc_all_finish).  NCCL moves the words over NVLink; no floating-point
reduction is involved.
"""
import ctypes as C

from . import _ffi
from .context import _check


class _DeviceWords:
    """A device int64 array seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, words):
        self.__cuda_array_interface__ = {"shape": (int(words),), "typestr": "<i8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def accumulator_tensor(ctx):
    """The context's fixed-point accumulators as a torch int64 CUDA tensor (a view)."""
    import torch

    ptr = C.c_void_p()
    words = C.c_size_t()
    _check(ctx.lib.galic_accumulators(ctx.h, C.byref(ptr), C.byref(words)), "galic_accumulators")
    return torch.as_tensor(_DeviceWords(ptr.value, words.value), device=f"cuda:{torch.cuda.current_device()}")


def sharded_pass(run_shard, accumulators, finish, group=None):
    """The exchange of one sharded pass: run_shard(rank, world) fills this
    rank's accumulators, accumulators() returns them as an int64 tensor,
    which is summed over the group in place, then finish() runs on every rank.
    Returns (rank, world)."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    run_shard(rank, world)
    acc = accumulators()
    dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    if acc.is_cuda:
        torch.cuda.synchronize(acc.device)
    finish()
    return rank, world


def calc_all_sharded(ctx, form=_ffi.GALIC_FORM_FP64, group=None):
    """One calc_all_response_fields pass of ctx's model over the group; returns
    the orbit-steps of all ranks."""
    import torch
    import torch.distributed as dist

    sharded_pass(lambda r, w: _check(ctx.lib.galic_calc_all_shard(ctx.h, int(form), r, w), "galic_calc_all_shard"),
                 lambda: accumulator_tensor(ctx),
                 lambda: _check(ctx.lib.galic_calc_all_finish(ctx.h), "galic_calc_all_finish"), group)
    steps = torch.tensor([ctx.last_orbit_steps()], dtype=torch.int64, device=f"cuda:{torch.cuda.current_device()}")
    dist.all_reduce(steps, op=dist.ReduceOp.SUM, group=group)
    return int(steps.item())
