"""Replica sharding of independent forward solves over ranks (one process per GPU).

The reference splits frequencies round-robin over MPI ranks (SETFREQIP,
src/solver_mpi/n_ebfem_bxyz_mpi.f90:332-355) and broadcasts every rank's
site responses so that rank 0 can write all files (SENDRECVRESULT, :360-392).
Here a rank owns the systems ``ip, ip+np, ...``, solves them on its own GPU
(batched inside the GPU), and the site results are exchanged with one
all-gather -- the only collective; a single solve never spans GPUs.
"""
from __future__ import annotations

import numpy as np


def setfreqip(nfreq: int, ip: int, np_: int) -> list[int]:
    """0-based indices of the frequencies rank ``ip`` of ``np_`` solves (SETFREQIP)."""
    if np_ < 1 or not (0 <= ip < np_):
        raise ValueError("rank out of range")
    nfreq_ip = nfreq // np_ + (1 if nfreq - (nfreq // np_) * np_ > 0 else 0)
    out = []
    for i in range(1, nfreq_ip + 1):
        ii = ip + 1 + (i - 1) * np_
        if ii <= nfreq:
            out.append(ii - 1)
    return out


def gather_site_results(local: dict[int, np.ndarray], nfreq: int, shape, group=None) -> np.ndarray:
    """All-gather per-frequency site responses (complex arrays of ``shape``) into (nfreq, *shape) on every rank.

    Replaces the broadcast loop of SENDRECVRESULT.  Uses torch.distributed
    (NCCL between GPUs, gloo on CPU) when a process group is initialised,
    else returns the local table.
    """
    import torch
    import torch.distributed as dist

    full = np.zeros((nfreq,) + tuple(shape), dtype=np.complex128)
    for k, v in local.items():
        full[k] = v
    if not (dist.is_available() and dist.is_initialized()):
        return full
    ws = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    mine = torch.from_numpy(np.ascontiguousarray(full.view(np.float64))).to(dev)
    mask = torch.zeros(nfreq, dtype=torch.float64, device=dev)
    for k in local:
        mask[k] = 1.0
    bufs = [torch.empty_like(mine) for _ in range(ws)]
    masks = [torch.empty_like(mask) for _ in range(ws)]
    dist.all_gather(bufs, mine, group=group)
    dist.all_gather(masks, mask, group=group)
    out = np.zeros_like(full)
    seen = np.zeros(nfreq, dtype=np.int64)
    for b, mk in zip(bufs, masks):
        arr = b.cpu().numpy().view(np.complex128).reshape(full.shape)
        sel = mk.cpu().numpy() > 0
        out[sel] = arr[sel]
        seen += sel
    if np.any(seen != 1):
        raise RuntimeError("every frequency must be solved by exactly one rank")
    return out
