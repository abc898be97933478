"""One T3 iteration captured as a CUDA graph (torch.cuda.CUDAGraph).

The step is compute_r3_tri (dcc.t3_residual.T3Residual.compute) followed by
the P3_full symmetrize, divide, update and norms (update_t3_): about thirty
kernel launches plus the cuBLAS calls of the FP64 pieces.  Captured once on
static buffers, each iteration is one graph launch; new inputs are copied
into the same buffers (`inputs`, `t3`) before `replay()`.  Capture needs a
step without host reads: the residual is built with the W_oooo pair symmetry
assumed (woooo_pair_symmetric=True), and device status words are read only
after replays (`status_ok`)."""
from __future__ import annotations

import torch

from . import t3_residual


class T3IterationGraph:
    def __init__(self, res, inputs, t3, r3=None, norms=None, workspace=None):
        if not res.woooo_pair_symmetric:
            raise ValueError("capture needs T3Residual(..., woooo_pair_symmetric=True)")
        self.res, self.inputs, self.t3 = res, inputs, t3
        self.r3 = torch.empty_like(t3) if r3 is None else r3
        self.norms = torch.empty(2, dtype=torch.float64, device=t3.device) if norms is None else norms
        self.ws = torch.empty(1 << 16, dtype=torch.float64, device=t3.device) if workspace is None else workspace
        # warm up on a side stream (library handles, tensor-map encoder, allocator pools)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._step()
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()

    def _step(self):
        self.res.compute(self.inputs, self.t3, self.r3)
        t3_residual.update_t3_(self.t3, self.r3, self.inputs, norms=self.norms, workspace=self.ws, write_r3=False)

    def replay(self):
        """One iteration: t3 += the symmetrized, divided residual; norms = [|r3|^2, |r3_active|^2]."""
        self.graph.replay()
        return self.norms

    def status_ok(self):
        return self.res.status_ok()
