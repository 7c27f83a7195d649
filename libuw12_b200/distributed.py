"""One UW12 evaluation split over the ranks of a torch.distributed group.

Each rank evaluates its shard (``uw12c_set_shard``): contiguous, balanced
ranges of the aux functions (fitted densities, MO transforms of the
three-index tensors, 2-el Fock, t~ dX Fock) and of the occupied orbitals
(X_AB and t, direct Fock, same-spin three-electron terms).  The partial
intermediates the later terms need whole -- the fitted densities, B1 and
the stacked RI rows of each potential, the M x M X_AB and t -- are summed
over the ranks inside the evaluation through the all-reduce hook
(``uw12c_set_allreduce``), here ``torch.distributed.all_reduce`` (NCCL over
NVLink for device buffers) on the library's stream.  The partial Fock
matrices and energies are summed by one more all-reduce at the end.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import form_fock, set_allreduce, set_shard


class _DeviceSpan:
    """``__cuda_array_interface__`` of ``count`` float64 values at a device
    address, so that torch can wrap library memory without a copy."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3}


def device_view(ptr: int, count: int, device):
    """A torch float64 tensor aliasing ``count`` values at device address ``ptr``."""
    import torch
    return torch.as_tensor(_DeviceSpan(ptr, count), device=device)


def nccl_allreduce(group=None, device=None):
    """The all-reduce hook for sharded evaluations: sums the library's buffer
    over ``group`` with torch.distributed, ordered on the library's stream."""
    import torch
    import torch.distributed as dist

    def fn(ptr: int, count: int, stream: int):
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        t = device_view(ptr, count, dev)
        s = torch.cuda.ExternalStream(stream, device=dev) if stream else \
            torch.cuda.default_stream(dev)
        with torch.cuda.stream(s):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return fn


def allreduce_partials(fock, energies, group=None):
    """Sums a partial Fock tensor (in place) and a partial energy tensor over
    the group; both are torch tensors on the group's device."""
    import torch.distributed as dist
    dist.all_reduce(fock, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(energies, op=dist.ReduceOp.SUM, group=group)
    return fock, energies


def form_fock_sharded(W, V, WV, abs_p, orbitals: Sequence[np.ndarray],
                      occupations: Sequence[np.ndarray], n_active: Sequence[int],
                      indirect_term: bool, calculate_fock: bool, scale_opp_spin: float,
                      scale_same_spin: float, fock_out, group=None):
    """Evaluates this rank's shard into ``fock_out`` (a CUDA float64 tensor of
    n_ao * n_ao * n_spin elements) and all-reduces it.  Returns the total energy
    and the (E2, E3, E4) terms; ``fock_out`` holds the full Fock matrix."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    set_shard(rank, world)
    set_allreduce(nccl_allreduce(group, fock_out.device))
    try:
        e, _, terms = form_fock(W, V, WV, abs_p, orbitals, occupations, n_active, indirect_term,
                                calculate_fock, scale_opp_spin, scale_same_spin,
                                fock_out=fock_out.data_ptr())
    finally:
        set_allreduce(None)
        set_shard(0, 1)
    en = torch.tensor([e, *terms], dtype=torch.float64, device=fock_out.device)
    allreduce_partials(fock_out, en, group)
    vals = en.tolist()
    return vals[0], tuple(vals[1:4])
