"""Replica parallelism across GPUs: one process per GPU, no data-path
collective.

The reconstruction does not shard within one recon (one recon fits one GPU);
the reference's multi-GPU mode (`-mgpu`, main_mri.cu:770-834) hands whole
slices to one host thread per GPU and gathers the images on the host.  Here
each rank (one process per GPU, launched by torchrun) takes a contiguous range
of the slices, reconstructs it on its own GPU, and the images are gathered on
rank 0; timing is the maximum over ranks.  The process group exists only for
these host-side steps: NCCL when CUDA is available, gloo otherwise (the CPU
tests run the same code with world size 2 over gloo).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(timeout_s: float = 300.0, backend: str | None = None) -> tuple[int, int, int]:
    """Joins the process group when WORLD_SIZE > 1 (MASTER_ADDR / MASTER_PORT
    from the environment) and selects this rank's GPU.  Returns env()."""
    ws, rank, local = env()
    if ws > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, ws: int) -> float:
    """Maximum of a per-rank scalar (elapsed seconds) over all ranks."""
    if ws == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def slice_range(n_slices: int, ws: int, rank: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of n_slices for `rank`; the first
    n_slices % ws ranks take one slice more.  Every slice belongs to exactly
    one rank; a rank may get none when ws > n_slices."""
    if n_slices < 0 or ws < 1 or not 0 <= rank < ws:
        raise ValueError("need n_slices >= 0, ws >= 1, 0 <= rank < ws")
    base, extra = divmod(n_slices, ws)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_images(local: np.ndarray, n_slices: int, ws: int, rank: int) -> np.ndarray | None:
    """Rank 0 receives the [n_slices][N] complex images of all ranks in slice
    order (each rank passes its slice_range share); other ranks get None."""
    local = np.asarray(local)
    if ws == 1:
        return local
    import torch.distributed as dist
    parts = [None] * ws if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    out = np.concatenate([p.reshape(-1, local.shape[-1]) if p.size else
                          np.zeros((0, local.shape[-1]), local.dtype) for p in parts])
    if out.shape[0] != n_slices:
        raise RuntimeError(f"gathered {out.shape[0]} slices, expected {n_slices}")
    return out


def finalize(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
