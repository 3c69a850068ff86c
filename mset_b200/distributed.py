"""Tilt sharding of the batched iteration over GPUs: one process per GPU,
torch.distributed (NCCL) for the single exchange of an iteration.

Each rank holds a disjoint set of tilts (measured patterns, probes, scan
positions) and the same lab-frame volume.  Per iteration:

  phase 1 (device, per rank): inverse-rotate the volume into each local
          tilt's beam frame, run the batched forward + adjoint pass, rotate
          the slab gradients back and sum them (FP64, nv^3);
  all-reduce (sum) of that gradient over ranks: the only collective, 8 nv^3
          bytes (16 MB at 128^3), issued on the session stream;
  phase 2 (device, every rank identically): update, positivity, TV-FISTA,
          probe and position updates of the local tilts.

The reference runs its tilts sequentially on one GPU (Run_MSET_recon.m:119-187);
with the batched method the tilts are independent inside a pass, so the split
needs no other communication.
"""
from __future__ import annotations

import ctypes as C
from typing import Protocol

import numpy as np

from ._lib import check


def tilt_shard(ntilts: int, world: int, rank: int) -> list[int]:
    """Contiguous, balanced block of tilt indices for `rank` (sizes differ by
    at most one; the first ntilts % world ranks take one extra)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(ntilts, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


class IterationBackend(Protocol):
    def phase1(self) -> None: ...
    def gradient(self): ...          # tensor aliasing the phase-1 gradient sum
    def phase2(self) -> None: ...
    def stream(self): ...            # context manager ordering the collective


class _DevArray:
    """__cuda_array_interface__ view of a device buffer owned by the library."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class GpuBackend:
    """IterationBackend over a BatchSession after iteration_setup()."""

    def __init__(self, bs, use_graph: bool = True):
        import torch

        self.bs = bs
        self.use_graph = use_graph
        g, cnt, st, err = C.c_void_p(), C.c_size_t(), C.c_void_p(), C.c_void_p()
        check("mset_batch_device_info", bs._lib.mset_batch_device_info(bs._h, C.byref(g), C.byref(cnt),
                                                                        C.byref(st), C.byref(err)))
        dev = torch.cuda.current_device()
        self._g = torch.as_tensor(_DevArray(g.value, cnt.value, "<f8"), device=f"cuda:{dev}")
        self._err = torch.as_tensor(_DevArray(err.value, bs.ntilts, "<f8"), device=f"cuda:{dev}")
        self._stream = torch.cuda.ExternalStream(st.value, device=f"cuda:{dev}")

    def phase1(self):
        check("mset_batch_iterate_phase", self.bs._lib.mset_batch_iterate_phase(self.bs._h, 1, int(self.use_graph)))

    def phase2(self):
        check("mset_batch_iterate_phase", self.bs._lib.mset_batch_iterate_phase(self.bs._h, 2, int(self.use_graph)))

    def gradient(self):
        return self._g

    def errors(self):
        return self._err

    def stream(self):
        import torch
        return torch.cuda.stream(self._stream)


def sharded_iterate(backend: IterationBackend, niter: int, group=None, world: int | None = None) -> None:
    """niter iterations; the phase-1 gradients of all ranks are summed with
    one all-reduce per iteration (every rank takes the same collective steps
    in the same order)."""
    import torch.distributed as dist

    if world is None:
        world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    for _ in range(niter):
        backend.phase1()
        if world > 1:
            with backend.stream():
                dist.all_reduce(backend.gradient(), op=dist.ReduceOp.SUM, group=group)
        backend.phase2()
