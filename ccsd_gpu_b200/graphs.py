"""CUDA-graph replay of the fixed-shape iteration bodies (T and Lambda updates).

One CCSD or Lambda iteration launches hundreds of small kernels (packs,
tensor-core GEMMs, cuBLAS, elementwise); for small molecules the host spends
several times longer issuing them than the GPU spends running them.  The
update function is pure device work on fixed shapes, so it is captured once
and replayed: the inputs are copied into the captured tensors, the graph is
launched, and the outputs are copied out.  The convergence norm, DIIS and the
energy stay outside the graph (they read values on the host).
"""
import torch


class StepGraph:
    """``fn(*tensors) -> tuple of tensors`` captured after one eager call."""

    def __init__(self, fn, enabled=True):
        self.fn = fn
        self.enabled = bool(enabled) and torch.cuda.is_available()
        self.graph = None
        self.failed = None

    def __call__(self, *inputs):
        if not self.enabled:
            return self.fn(*inputs)
        if self.graph is None:
            out = self.fn(*inputs)      # eager: fills the offset and packed-operand caches
            self._capture(inputs)
            return out
        for d, x in zip(self.static_in, inputs):
            d.copy_(x)
        self.graph.replay()
        return tuple(o.clone() for o in self.static_out)

    def _capture(self, inputs):
        self.static_in = [x.detach().clone() for x in inputs]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.fn(*self.static_in)    # warm-up on the capture stream's side, as torch requires
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        try:
            with torch.cuda.graph(g):
                self.static_out = tuple(self.fn(*self.static_in))
        except RuntimeError as e:       # not capturable here: stay eager
            self.failed = repr(e)
            self.enabled = False
            return
        self.graph = g
