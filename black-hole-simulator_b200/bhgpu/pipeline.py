"""Host-resident states stepped through the GPU with their copies overlapped.

A caller whose states live in host memory -- an ensemble of independent
boxes, or one box paged in and out between other work -- hands each state
to ``HostPipeline.submit`` as pinned host tensors in the pool layout of
``AmrTree`` (U, W [npatch, 8, 8000], Bf [npatch, 3, 8400]).  The state is
copied into one of the pipeline's device trees on a host-to-device copy
stream, advanced by ``steps`` calls of rk2integrator::step on a compute
stream, and copied back on a device-to-host copy stream.  Consecutive
submissions go to different trees, so the upload of one state, the step of
the previous one and the download of the one before that run at the same
time: the two copy directions use separate copy engines, and the step uses
the SMs.  Each state's result is bit-identical to stepping it alone on one
tree.

Only the GPU-side order is managed here; the host must not reuse an input
tensor before its upload has finished, nor read an output tensor before
its download has finished.  The ``Event`` returned by ``submit`` marks the
end of that submission's download, and ``synchronize`` waits for all of
them.
"""
from __future__ import annotations

import torch

from .solver import AmrTree, RK2Integrator


class HostPipeline:
    def __init__(self, trees: list[AmrTree], integrator: RK2Integrator, steps: int = 1):
        if not trees:
            raise ValueError("HostPipeline needs at least one device tree")
        shape = (trees[0].U.shape, trees[0].Bf.shape)
        if any((t.U.shape, t.Bf.shape) != shape for t in trees):
            raise ValueError("the trees of a HostPipeline must share one pool shape")
        self.trees, self.rk, self.steps = list(trees), integrator, int(steps)
        dev = trees[0].device
        self.s_in = torch.cuda.Stream(dev)
        self.s_run = torch.cuda.Stream(dev)
        self.s_out = torch.cuda.Stream(dev)
        self._freed: list[torch.cuda.Event | None] = [None] * len(self.trees)
        self._k = 0

    def submit(self, U, W, Bf, out_U, out_W, out_Bf) -> torch.cuda.Event:
        """Upload (U, W, Bf), step, download into (out_U, out_W, out_Bf);
        returns the event recorded after the download."""
        slot = self._k % len(self.trees)
        self._k += 1
        t = self.trees[slot]
        with torch.cuda.stream(self.s_in):
            if self._freed[slot] is not None:          # this tree's previous download
                self.s_in.wait_event(self._freed[slot])
            t.U.copy_(U, non_blocking=True)
            t.W.copy_(W, non_blocking=True)
            t.Bf.copy_(Bf, non_blocking=True)
            loaded = torch.cuda.Event()
            loaded.record(self.s_in)
        with torch.cuda.stream(self.s_run):
            self.s_run.wait_event(loaded)
            for _ in range(self.steps):
                self.rk.step(t, sync=False, check_domain=False)
            done = torch.cuda.Event()
            done.record(self.s_run)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(done)
            out_U.copy_(t.U, non_blocking=True)
            out_W.copy_(t.W, non_blocking=True)
            out_Bf.copy_(t.Bf, non_blocking=True)
            freed = torch.cuda.Event()
            freed.record(self.s_out)
        self._freed[slot] = freed
        return freed

    def synchronize(self):
        for e in self._freed:
            if e is not None:
                e.synchronize()

    def check(self):
        """Raise DomainError if any tree's device error word is set (after
        synchronize); clears the word of the trees it reads."""
        self.synchronize()
        for t in self.trees:
            t.check()
