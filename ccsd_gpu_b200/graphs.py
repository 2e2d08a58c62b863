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


class _SolveGraph:
    def __init__(self, fn, consts, inputs):
        from .contract import mark_constant, pack_cache_disabled
        self.fn = fn
        self.consts = {k: v.detach().clone() for k, v in consts.items()}
        # constants as in the eager solve, so contractions take the same routes
        mark_constant(*self.consts.values())
        self.static_in = [x.detach().clone() for x in inputs]
        with pack_cache_disabled():         # packs of the constants become graph nodes
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                fn(self.consts, *self.static_in)
            torch.cuda.current_stream().wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.static_out = tuple(fn(self.consts, *self.static_in))
        self.graph = g

    def load(self, consts):
        for k, v in consts.items():
            self.consts[k].copy_(v)

    def __call__(self, *inputs):
        for d, x in zip(self.static_in, inputs):
            d.copy_(x)
        self.graph.replay()
        return tuple(o.clone() for o in self.static_out)


_SOLVE_GRAPHS = {}
_SOLVE_GRAPHS_MAX = 32
# split-precision bodies are cached only while their ladder (2 o^2 v^4 flops)
# is below this: beyond it the per-replay re-pack of the integrals costs more
# than the host overhead a graph saves
GRAPH_MAX_LADDER_FLOPS = 1e12


# FP64 bodies are captured only while their vvvv block is below this size: a
# captured graph keeps its memory pool (the body's temporaries) for as long
# as the cache holds it, and at large nvir that pool is tens of GB
GRAPH_MAX_FP64_VVVV_BYTES = 4e9


def graph_cache_ok(mode, nocc, nvir):
    if mode == "fp64":
        return 8.0 * float(nvir) ** 4 < GRAPH_MAX_FP64_VVVV_BYTES
    return 2.0 * nocc * nocc * float(nvir) ** 4 < GRAPH_MAX_LADDER_FLOPS


def solve_step(key, fn, consts, enabled=True):
    """A replayable iteration body shared by every solve of the same shape.

    ``fn(consts, *inputs)`` is pure device work on the tensors of the dict
    ``consts`` (integrals, intermediates: fixed within one solve) and on the
    per-iteration ``inputs``.  The graph for ``key`` is captured once (the
    first call runs eagerly); later solves copy their own ``consts`` into the
    captured tensors and replay.  The packed-operand cache is off during the
    capture, so a split-precision body re-packs its constant operands inside
    the graph on every replay (from the captured tensors, i.e. the current
    solve's values).
    """
    if not (enabled and torch.cuda.is_available()):
        return lambda *inputs: fn(consts, *inputs)
    key = (torch.cuda.current_device(),) + tuple(key)
    entry = _SOLVE_GRAPHS.get(key)
    state = {"entry": entry, "first": entry is None}
    if entry is not None:
        entry.load(consts)

    def step(*inputs):
        if state["entry"] is None:
            out = fn(consts, *inputs)
            try:
                e = _SolveGraph(fn, consts, inputs)
            except RuntimeError:                 # not capturable here: stay eager
                state["entry"] = False
                return out
            if len(_SOLVE_GRAPHS) >= _SOLVE_GRAPHS_MAX:
                _SOLVE_GRAPHS.pop(next(iter(_SOLVE_GRAPHS)))
            _SOLVE_GRAPHS[key] = e
            state["entry"] = e
            return out
        if state["entry"] is False:
            return fn(consts, *inputs)
        return state["entry"](*inputs)
    return step


def clear_solve_graphs():
    _SOLVE_GRAPHS.clear()
