"""Overlapped host-to-device staging of forcing intervals.

The reference's run scripts keep forcing I/O off the routing path with a
DataLoader over pinned memory and a side CUDA stream
(scripts/run_daily_bin.py:104-119).  `InputPrefetcher` does the same for the
device model: `submit(host_runoff)` copies a later interval's runoff from
pinned host memory into one of `depth` device buffers on a copy stream, while
earlier intervals route on the model's stream; `set_inputs()` makes the
model's stream wait for that copy and stages it with a device-to-device copy.
Events keep a buffer from being refilled before the model has consumed it.
"""
from __future__ import annotations

import torch


class InputPrefetcher:
    def __init__(self, model, depth: int = 2):
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.model = model
        self.device = model.device
        runoff = model.base.runoff
        self.shape = tuple(runoff.shape)
        self.depth = int(depth)
        self.bufs = [torch.empty(self.shape, dtype=runoff.dtype, device=self.device)
                     for _ in range(self.depth)]
        self.ready = [torch.cuda.Event() for _ in range(self.depth)]
        self.free = [torch.cuda.Event() for _ in range(self.depth)]
        self.hold = [None] * self.depth          # host tensors kept alive until copied
        self.copy_stream = torch.cuda.Stream(self.device)
        self.head = 0
        self.tail = 0
        self.pending = 0

    def submit(self, host_runoff: torch.Tensor) -> None:
        """Start the copy of one interval's runoff (model order, pinned host
        memory for a truly asynchronous copy)."""
        if self.pending == self.depth:
            raise RuntimeError("every staging buffer is in flight: call set_inputs() first")
        i = self.head
        src = torch.as_tensor(host_runoff).reshape(self.shape)
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(self.free[i])   # the model has consumed buffer i
            self.bufs[i].copy_(src, non_blocking=True)
            self.ready[i].record(self.copy_stream)
        self.hold[i] = src
        self.head = (i + 1) % self.depth
        self.pending += 1

    def set_inputs(self) -> None:
        """Stage the oldest submitted interval into the model (on the model's
        current stream, after its copy has landed)."""
        if self.pending == 0:
            raise RuntimeError("no interval submitted")
        i = self.tail
        stream = torch.cuda.current_stream(self.device)
        stream.wait_event(self.ready[i])
        self.model.set_inputs(self.bufs[i])
        self.free[i].record(stream)
        self.hold[i] = None
        self.tail = (i + 1) % self.depth
        self.pending -= 1
