"""Serving several independent voltage streams on one GPU.

The reference serves its streams through per-stream block pipelines
(``BlockPipeliner``, services/corr_fast_integration.py:2593) feeding
``process_block`` (:2229).  Here every stream owns a ``SearchPipeline``: its
correlator ring, stage-2 ring (the per-DM FIFOs), static-sky state and
detector buffers stay resident on the device for the life of the stream.

* Continuous batching, not a queue: each stream has a worker thread that
  runs its blocks on its own CUDA stream.  Blocks of different streams that
  arrive while others are on the GPU start at once, and their kernels overlap
  on the device.  The Python thread releases the interpreter lock while a
  stream waits on the device or in a kernel launch.
* Admission by device memory: a block's device copy is admitted only when
  it fits a byte budget shared by all streams (``DeviceBudget``).  The
  resident state is allocated when the stream is created; the budget governs
  the in-flight block copies.
* Blocks may hold any whole number of chunks (uneven lengths).
* Each result records the block's arrival and completion times, for
  arrival-to-candidate latency.
* An optional ``prepare(stream, block_index, device_block)`` runs on the
  block's device copy, on the stream's CUDA stream, before the search (the
  served benchmark draws its injected bursts in there).

A stream's candidates do not depend on what runs beside it: pipelines share
no state, only the GPU.
"""

from __future__ import annotations

import contextlib
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import torch


class DeviceBudget:
    """Bytes of device memory that in-flight block copies may hold at once."""

    def __init__(self, nbytes: int):
        if nbytes <= 0:
            raise ValueError("budget must be positive")
        self.capacity = int(nbytes)
        self.used = 0
        self.peak = 0
        self._cv = threading.Condition()

    def acquire(self, n: int, timeout: Optional[float] = None) -> None:
        """Wait until ``n`` bytes fit, then hold them.  A request larger than
        the whole budget can never be admitted and raises ValueError."""
        if n > self.capacity:
            raise ValueError(f"block of {n} bytes exceeds the device budget of {self.capacity}")
        with self._cv:
            if not self._cv.wait_for(lambda: self.used + n <= self.capacity, timeout):
                raise TimeoutError(f"no room for {n} bytes within {timeout} s")
            self.used += n
            self.peak = max(self.peak, self.used)

    def release(self, n: int) -> None:
        with self._cv:
            self.used -= n
            if self.used < 0:
                raise RuntimeError("device budget released more than it held")
            self._cv.notify_all()


@dataclass
class BlockResult:
    index: int                  # block number within its stream
    packets: int                # packets per chgroup page of the block
    t_arrival: float            # host time the block was handed in (perf_counter s)
    t_admit: float              # its device copy was admitted under the budget
    t_done: float               # its candidates were on the host
    candidates: list = field(default_factory=list)

    @property
    def latency_s(self) -> float:
        return self.t_done - self.t_arrival


class StreamServer:
    """Run several ``SearchPipeline``s (one per voltage stream) side by side.

    ``submit(i, raw)`` hands a host block ``(G, npkt, nant, nchan, 2, 2)``
    uint8 to stream i (pinned memory lets its copy overlap other work);
    ``close()`` ends every stream after its queued blocks; ``join()`` waits
    and re-raises the first error of any worker."""

    def __init__(self, pipelines: Sequence, budget_bytes: int,
                 prepare: Optional[Callable[[int, int, torch.Tensor], None]] = None):
        self.pipes = list(pipelines)
        self.budget = DeviceBudget(budget_bytes)
        self.prepare = prepare
        self._queues: List[queue.Queue] = [queue.Queue() for _ in self.pipes]
        self.results: List[List[BlockResult]] = [[] for _ in self.pipes]
        self._errors: List[BaseException] = []
        self._threads: List[threading.Thread] = []

    def start(self) -> "StreamServer":
        for i in range(len(self.pipes)):
            th = threading.Thread(target=self._worker, args=(i,), daemon=True,
                                  name=f"dsb200-stream-{i}")
            th.start()
            self._threads.append(th)
        return self

    def submit(self, stream: int, raw: torch.Tensor, t_arrival: Optional[float] = None) -> None:
        self.pipes[stream].block_packets(raw)  # reject a malformed block at the door
        self._queues[stream].put((raw, time.perf_counter() if t_arrival is None else t_arrival))

    def close(self) -> None:
        for q in self._queues:
            q.put(None)

    def join(self, timeout: Optional[float] = None) -> None:
        for th in self._threads:
            th.join(timeout)
            if th.is_alive():
                raise TimeoutError(f"{th.name} did not finish within {timeout} s")
        if self._errors:
            raise self._errors[0]

    def latencies_s(self) -> List[float]:
        return [r.latency_s for rs in self.results for r in rs]

    # ------------------------------------------------------------------
    def _stream_ctx(self, dev):
        if getattr(dev, "type", None) == "cuda":
            return torch.cuda.stream(torch.cuda.Stream(dev))
        return contextlib.nullcontext()

    def _worker(self, i: int) -> None:
        pipe = self.pipes[i]
        q = self._queues[i]
        try:
            with self._stream_ctx(pipe.dev):
                k = 0
                while True:
                    item = q.get()
                    if item is None:
                        return
                    raw, t_arr = item
                    n = raw.numel()
                    self.budget.acquire(n)
                    t_admit = time.perf_counter()
                    try:
                        dev_raw = raw.to(pipe.dev, non_blocking=True)
                        if self.prepare is not None:
                            if dev_raw.data_ptr() == raw.data_ptr():
                                dev_raw = raw.clone()   # never change the caller's block
                            self.prepare(i, k, dev_raw)
                        cands = pipe.process_block(dev_raw)
                        if getattr(pipe.dev, "type", None) == "cuda":
                            # the block's copy is released only once nothing reads it
                            torch.cuda.current_stream(pipe.dev).synchronize()
                        del dev_raw
                    finally:
                        self.budget.release(n)
                    self.results[i].append(BlockResult(k, pipe.block_packets(raw), t_arr,
                                                       t_admit, time.perf_counter(), cands))
                    k += 1
        except BaseException as exc:  # noqa: BLE001  (reported by join)
            self._errors.append(exc)
            # drain this stream so that close() and join() still end
            while q.get() is not None:
                pass
