"""Direction sharding of one solve: block partition and exchange functions.

A solve is split over handles by directions, as the reference splits it
over MPI ranks (``StaticBTESynthetic.cpp:247-300``): each handle sweeps a
contiguous block of directions, and every outer iteration the moments and
boundary values are summed over the handles
(``gbte_set_direction_shard`` in ``include/giftbte.h``). The exchange is a
sum of doubles in place; this module provides two of them:

- :func:`torch_exchange`: ``torch.distributed.all_reduce`` over a process
  group, one process per GPU (NCCL on device memory; gloo on host memory
  for the CPU tests of the plumbing);
- :class:`ThreadExchange`: several handles in one process, one host thread
  each. The threads meet at a barrier, handle 0 adds the buffers in handle
  order on the host, and each thread copies the sum back. No kernel waits
  on another handle's kernels, so the handles may share one GPU.
"""
from __future__ import annotations

import ctypes
import threading
from typing import Callable, List, Optional, Tuple

import numpy as np


def direction_blocks(num_directions: int, parts: int) -> List[Tuple[int, int]]:
    """(begin, count) of each part: num_directions // parts directions each,
    one more for the first num_directions % parts parts, as the reference
    counts its ranks' local directions (``StaticBTESynthetic.cpp:247-254``),
    laid out as contiguous blocks."""
    if parts < 1 or parts > num_directions:
        raise ValueError(f"cannot split {num_directions} directions into {parts} non-empty blocks")
    base, extra = divmod(num_directions, parts)
    out, b = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((b, n))
        b += n
    return out


class _DeviceDoubles:
    """``__cuda_array_interface__`` view of ``n`` doubles at a device address
    (version 2: no stream synchronisation by the consumer)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2,
                                         "strides": None}


def host_doubles(ptr: int, n: int) -> np.ndarray:
    """numpy view of ``n`` doubles at a host address."""
    if n == 0:
        return np.zeros(0)
    return np.ctypeslib.as_array((ctypes.c_double * n).from_address(ptr))


def device_tensor(ptr: int, n: int):
    """torch tensor aliasing ``n`` doubles of device memory at ``ptr``."""
    import torch

    return torch.as_tensor(_DeviceDoubles(ptr, n), device="cuda")


def torch_exchange(group=None, device: str = "cuda") -> Callable[[int, int, int], None]:
    """An exchange that all-reduces (sum) the buffer over ``group`` with
    torch.distributed. device="cuda": the buffer is device memory and the
    all-reduce is ordered on the solver's stream (the current stream while
    it is issued); device="cpu": host memory (gloo)."""
    import torch
    import torch.distributed as dist

    def fn(buf: int, n: int, stream: int) -> None:
        if device == "cpu":
            dist.all_reduce(torch.from_numpy(host_doubles(buf, n)), group=group)
            return
        ext = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
        with torch.cuda.stream(ext):
            dist.all_reduce(device_tensor(buf, n), group=group)

    return fn


class ThreadExchange:
    """Exchange among ``parts`` handles driven by ``parts`` threads of one
    process. ``member(k)`` is handle k's exchange function. Every call
    copies the buffer to the host (after the handle's stream), waits at a
    barrier for the other handles (at most ``timeout`` seconds; a timeout
    or a failed member breaks the barrier and every member's call raises),
    and takes the sum in handle order, so the result is the same on every
    handle and from run to run."""

    def __init__(self, parts: int, timeout: float = 300.0):
        self.parts = parts
        self.timeout = timeout
        self._barrier = threading.Barrier(parts)
        self._bufs: List[Optional[np.ndarray]] = [None] * parts
        self._sum: Optional[np.ndarray] = None
        self.calls = 0

    def member(self, k: int, device: str = "cuda") -> Callable[[int, int, int], None]:
        def fn(buf: int, n: int, stream: int) -> None:
            if device == "cpu":
                self._bufs[k] = host_doubles(buf, n).copy()
            else:
                import torch

                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    self._bufs[k] = device_tensor(buf, n).cpu().numpy()
            self._barrier.wait(self.timeout)
            if k == 0:
                if any(b is None or b.shape != (n,) for b in self._bufs):
                    self._barrier.abort()
                    raise RuntimeError("shard members exchanged buffers of different sizes")
                acc = self._bufs[0].copy()
                for b in self._bufs[1:]:
                    acc += b
                self._sum = acc
                self.calls += 1
            self._barrier.wait(self.timeout)
            out = self._sum
            self._barrier.wait(self.timeout)  # every member has the sum before the next call replaces it
            self._bufs[k] = None
            if device == "cpu":
                host_doubles(buf, n)[:] = out
            else:
                import torch

                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    device_tensor(buf, n).copy_(torch.from_numpy(out))

        return fn

    def abort(self) -> None:
        """Break the barrier: every member waiting on it raises."""
        self._barrier.abort()


def solve_sharded(handles, exchange: ThreadExchange, **solve_kw) -> list:
    """Run ``solve(**solve_kw)`` on every handle of a thread-exchange shard
    set, one thread each; returns their stats (raises the first failure,
    after breaking the barrier so that the other members return)."""
    out: list = [None] * len(handles)
    errs: list = [None] * len(handles)

    def run(k):
        try:
            out[k] = handles[k].solve(**solve_kw)
        except BaseException as e:
            errs[k] = e
            exchange.abort()

    ts = [threading.Thread(target=run, args=(k,)) for k in range(len(handles))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for e in errs:
        if e is not None:
            raise e
    return out
