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


class T4Iteration:
    """One T4 update of update_amps_rccsdtq_tri_ (distr_cc/rccsdtq.py:1431-1463):
    r4 = compute_r4_tri (OO batch included), r4 <- (1 - P[4] - P[3,1]) r4, r4 /= D_ijklabcd,
    norms = [|r4|^2, |r4|^2] (every virtual index is active), t4 += r4.

    `d` holds the inputs (dcc.synthetic.make_t4_inputs names them); the step reads
    d.t4 and updates it in place.  It makes no host read and no host-to-device copy, so
    T4IterationGraph can capture it."""

    def __init__(self, d, precision="bf16x3"):
        self.d, self.precision = d, precision
        self.nocc, self.nv = d.t2.shape[0], d.t2.shape[2]
        self.r4 = torch.empty_like(d.t4)
        self.norms = torch.zeros(2, dtype=torch.float64, device=d.t4.device)

    def step(self):
        from . import _c_rccsdtq, t4_residual
        d, r4, n4 = self.d, self.r4, self.d.t4.shape[0]
        t4_residual.compute_r4_tri_(r4, d.eris, d.F_vv, d.W_vvvo, d.W_vooo, d.W_vvvv, d.W_oooo, d.W_ovov, d.t2,
                                    d.t3, d.t4, self.nocc, self.precision, F_oo=d.F_oo, W_ovvo=d.W_ovvo)
        _c_rccsdtq.t4_project_1_minus_p4_p31_inplace_(r4, n4, self.nv)
        _c_rccsdtq.r4_local_tri_divide(r4, d.eia, d.ijkl)
        flat = r4.view(-1)
        self.norms.copy_(torch.dot(flat, flat).expand(2))
        _c_rccsdtq.t4_add_(d.t4, r4, n4, self.nv)
        return self.norms


class T4IterationGraph:
    """T4Iteration captured as one CUDA graph: the ~300 small launches of the T4
    residual at nvir ~ 11 (einsums, block forms, scatters) replay without per-launch host
    overhead.  New inputs are copied into the same tensors before `replay()`."""

    def __init__(self, it):
        self.it = it
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        saved = it.d.t4.clone()
        with torch.cuda.stream(side):
            it.step()  # warm-up: library handles, split buffers, cached index tensors
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        it.d.t4.copy_(saved)
        del saved
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            it.step()

    def replay(self):
        self.graph.replay()
        return self.it.norms
