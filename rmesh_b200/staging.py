"""Double-buffered host-to-device upload of training targets.

A training loop that keeps its target images in pinned host memory pays one
host-to-device copy per step (12 bytes per pixel).  ``TargetStager`` issues
that copy on its own CUDA stream into one of ``depth`` device buffers, so the
copy of step i+1's targets runs while step i's kernels run:

    stager = TargetStager(renderer, n_floats)
    nxt = stager.put(gt_host[0])
    for i in range(steps):
        cur = nxt
        if i + 1 < steps:
            nxt = stager.put(gt_host[i + 1])
        renderer.train_step_views(cams, cur, ...)

The handle ``put`` returns is accepted wherever ``train_step_views`` and
``accumulate_views`` take targets; the renderer's stream waits for exactly
that copy before the step.  A buffer is refilled only after all work enqueued
on the renderer's stream before the refill (which includes the buffer's last
step) has finished.
"""
from __future__ import annotations


class StagedTargets:
    """One step's targets on the device plus the event that marks their copy done."""

    __slots__ = ("tensor", "ready", "_stager", "used")

    def __init__(self, tensor, ready, stager):
        self.tensor = tensor
        self.ready = ready
        self._stager = stager
        self.used = False

    def numel(self) -> int:
        return int(self.tensor.numel())

    def _before_step(self) -> int:
        """Makes the renderer's stream wait for the copy; returns the device pointer."""
        if self.used:
            raise ValueError("staged targets were already used by a step")
        self.used = True
        self._stager._lib_stream.wait_event(self.ready)
        return self.tensor.data_ptr()


class TargetStager:
    """``depth`` device buffers of ``n_floats`` floats filled on a copy stream."""

    def __init__(self, renderer, n_floats: int, depth: int = 2):
        import torch

        if depth < 2:
            raise ValueError("depth must be at least 2")
        dev = torch.device("cuda", renderer.device_index)
        self._lib_stream = renderer.torch_stream()
        self._copy = torch.cuda.Stream(device=dev)
        self._bufs = [torch.empty(int(n_floats), dtype=torch.float32, device=dev) for _ in range(depth)]
        self._held = [None] * depth  # the handle last filled into each buffer
        self._next = 0

    def put(self, host) -> StagedTargets:
        """Starts copying ``host`` (a float32 CPU tensor of ``n_floats`` values,
        pinned for an asynchronous copy) into the next buffer."""
        import torch

        k = self._next
        if self._held[k] is not None and not self._held[k].used:
            raise ValueError(f"all {len(self._bufs)} buffers hold targets that no step has used yet")
        buf = self._bufs[k]
        if host.numel() != buf.numel() or host.dtype != torch.float32:
            raise ValueError(f"targets must be {buf.numel()} float32 values")
        self._next = (k + 1) % len(self._bufs)
        free = torch.cuda.Event()
        free.record(self._lib_stream)
        self._copy.wait_event(free)
        with torch.cuda.stream(self._copy):
            buf.copy_(host.reshape(-1), non_blocking=True)
        ready = torch.cuda.Event()
        ready.record(self._copy)
        self._held[k] = StagedTargets(buf, ready, self)
        return self._held[k]
