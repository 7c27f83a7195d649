"""One UW12 evaluation split over the ranks of a torch.distributed group.

Each rank evaluates its shard (``uw12c_set_shard``: a contiguous part of the
aux functions of the t~ dX Fock term and of the occupied orbitals k of the
same-spin three-electron energy and Fock; every other contribution on rank
0), then the partial Fock matrices and energies are summed with one
all-reduce (NCCL over NVLink for device tensors).  Every rank holds the full
integrals; only the results travel.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import form_fock, set_shard


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
    try:
        e, _, terms = form_fock(W, V, WV, abs_p, orbitals, occupations, n_active, indirect_term,
                                calculate_fock, scale_opp_spin, scale_same_spin,
                                fock_out=fock_out.data_ptr())
    finally:
        set_shard(0, 1)
    en = torch.tensor([e, *terms], dtype=torch.float64, device=fock_out.device)
    allreduce_partials(fock_out, en, group)
    vals = en.tolist()
    return vals[0], tuple(vals[1:4])
