"""Batched execution of several plans under one CUDA graph (dfft_graph_*)."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _gpu_util import out_extents, random_input

pytestmark = pytest.mark.gpu


def test_graph_batch_of_uneven_fields_matches_eager():
    import torch
    specs = [((64, 64, 64), True, "float32", (2, 1, 1), (1, 2, 1)),
             ((96, 64, 48), False, "float64", (2, 2, 1), (1, 2, 2)),
             ((128, 128, 128), False, "float32", (4, 4, 1), (1, 4, 4))]
    items, eager, refs, bufs = [], [], [], []
    for i, (g, real, prec, tin, tout) in enumerate(specs):
        go = out_extents(g, (0, 1, 2), real)
        p = dfft.Plan(g, go, (0, 1, 2), tin, tout, real_input=real, precision=prec)
        x = random_input(g, real, 10 + i, prec)
        xin = torch.from_numpy(dfft.scatter_blocks(p, x, "in")).cuda()
        cdt = torch.complex64 if prec == "float32" else torch.complex128
        y = torch.empty(p.buffer_elements("out"), dtype=cdt, device="cuda")
        z = torch.empty_like(xin)
        ye = torch.empty_like(y)
        dfft.execute(p, xin, ye, dfft.Direction.forward)
        items += [(p, xin, y, dfft.Direction.forward, i), (p, y, z, dfft.Direction.backward, i)]
        eager.append(ye)
        refs.append((p, x, real, prec))
        bufs.append((y, z))
    graph = dfft.Graph(items)
    for _ in range(2):
        for y, z in bufs:
            y.zero_()
            z.zero_()
        graph.launch()
        torch.cuda.synchronize()
        for (y, z), ye, (p, x, real, prec) in zip(bufs, eager, refs):
            assert torch.equal(y, ye)  # same kernels, same data: identical
            xb = dfft.gather_blocks(p, z.cpu().numpy(), "in")
            tol = 1e-12 if prec == "float64" else 1e-6
            assert O.rel_l2(xb, x) <= tol
