"""torch.autograd wrapper of batched SSSP (a thin ctypes shim used by tests).

forward : per-graph float32 weight tensors (CSR edge order, on the GPU)
          -> one flat float32 tensor with every query's distances; query q
             occupies [offsets[q], offsets[q] + n_q) (Batch.layout()), the
             padding between queries is 0 and unreached vertices hold FLT_MAX
backward: dL/d(flat distances) -> per-graph dL/dw, computed by the engine's
          adjoint kernels (adds_batch_backward): lambda summed up the
          tie-broken shortest-path tree, queries summed in order.
The gradient is the one taken along the shortest-path tree (a distance is
piecewise linear in the weights; ties take the smallest-index tight edge).
Unreached vertices carry no gradient.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Batch


class _SSSP(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch: Batch, graphs: list, *weights):
        for g, w in zip(graphs, weights):
            g.set_weights(w.detach().contiguous().data_ptr())
        batch.run()
        off, tot = batch.layout()
        flat = torch.zeros(int(tot), dtype=torch.float32, device=weights[0].device)
        batch.dist_all(flat.data_ptr())
        ctx.batch = batch
        ctx.off = off
        ctx.shapes = [w.shape for w in weights]
        return flat

    @staticmethod
    def backward(ctx, grad_flat):
        g = grad_flat.contiguous()
        base = g.data_ptr()
        ptrs = [base + 4 * int(o) for o in ctx.off]
        gw = [torch.zeros(s, dtype=torch.float32, device=g.device) for s in ctx.shapes]
        torch.cuda.synchronize(g.device)
        ctx.batch.backward(ptrs, [t.data_ptr() for t in gw])
        return (None, None, *gw)


def batched_sssp(batch: Batch, graphs: list, weights: list):
    """Flat distances of every query of `batch`; graphs[i] receives
    weights[i] (the distinct graphs, in the order the batch first uses them)."""
    return _SSSP.apply(batch, graphs, *weights)


def query_offsets(batch: Batch) -> np.ndarray:
    return batch.layout()[0]
