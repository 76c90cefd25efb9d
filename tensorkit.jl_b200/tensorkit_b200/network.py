"""Whole-network `@tensor` plans replayed as CUDA graphs.

A `NetworkPlan` fixes one `@tensor` expression on fixed input buffers: the first call
builds every tree-transformer table and grouped-GEMM plan of the pairwise contractions
(cached per structure), then the transform→GEMM→transform launches of the whole network
are captured once into a CUDA graph on the library stream, with every intermediate buffer
owned by the plan. `replay()` relaunches the graph; new input values are written into
`plan.inputs[name].data` in place. This is the counterpart of evaluating
`TO.tensorcontract!` step by step (src/tensors/tensoroperations.jl:130-161, 392-462)
with temporaries from a fixed allocator, minus the host work per replay.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from . import tensor as _tensor_mod
from .backend import get_context, using_precision
from .tensoroperations import tensor

__all__ = ["NetworkPlan"]


class NetworkPlan:
    def __init__(self, expr: str, precision: str = "plain", slices: int = 0, **inputs):
        self.expr = expr
        self.precision = precision
        self.slices = slices
        self.inputs = inputs
        dev = next(iter(inputs.values())).data.device
        self.ctx = get_context(dev.index)
        self.graph = None
        self.output = None
        self._buffers = []
        self.kernels_per_replay = 0

    def run_eager(self):
        """Evaluate the network once without capture (builds every table and plan)."""
        import torch
        with torch.cuda.stream(self.ctx.stream), using_precision(self.precision, self.slices):
            out = tensor(self.expr, **self.inputs)
        return out

    def capture(self):
        import torch
        self.run_eager()
        self.ctx.stream.synchronize()
        lib = self.ctx.lib
        n0 = self.ctx.launch_count()
        _tensor_mod._ALLOC_LOG = []
        try:
            with torch.cuda.stream(self.ctx.stream), using_precision(self.precision, self.slices):
                L.check(lib.tkb_graph_begin(self.ctx.handle), self.ctx.handle)
                try:
                    out = tensor(self.expr, **self.inputs)
                except Exception:
                    g = C.c_void_p()
                    lib.tkb_graph_end(self.ctx.handle, C.byref(g))
                    if g:
                        lib.tkb_graph_destroy(g)
                    raise
                g = C.c_void_p()
                L.check(lib.tkb_graph_end(self.ctx.handle, C.byref(g)), self.ctx.handle)
        finally:
            self._buffers = _tensor_mod._ALLOC_LOG or []
            _tensor_mod._ALLOC_LOG = None
        self.graph = g
        self.output = out
        self.kernels_per_replay = self.ctx.launch_count() - n0
        return self

    def replay(self):
        if self.graph is None:
            self.capture()
        L.check(self.ctx.lib.tkb_graph_launch(self.ctx.handle, self.graph), self.ctx.handle)
        return self.output

    def free(self):
        if self.graph is not None:
            self.ctx.synchronize()
            self.ctx.lib.tkb_graph_destroy(self.graph)
            self.graph = None
        self._buffers = []

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
