"""Helpers of the GPU parity tests: move concatenated per-rank buffers to and
from the device with torch (plumbing only) and run dfft.execute."""
import numpy as np
import torch

import dfft

_TORCH = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
          np.dtype(np.complex128): torch.complex128, np.dtype(np.complex64): torch.complex64}


def dtypes(plan):
    f = np.float64 if plan.precision == "float64" else np.float32
    c = np.complex128 if plan.precision == "float64" else np.complex64
    return (f if plan.real_input else c), c


def run(plan, x_global, forward=True):
    """Global numpy array in -> global numpy array out through the GPU plan."""
    din, dout = dtypes(plan)
    src_side, dst_side = ("in", "out") if forward else ("out", "in")
    src_dt, dst_dt = (din, dout) if forward else (dout, din)
    flat = dfft.scatter_blocks(plan, np.asarray(x_global).astype(src_dt), src_side)
    t_in = torch.from_numpy(np.ascontiguousarray(flat)).cuda()
    t_out = torch.empty(plan.buffer_elements(dst_side), dtype=_TORCH[np.dtype(dst_dt)], device="cuda")
    dfft.execute(plan, t_in, t_out, dfft.Direction.forward if forward else dfft.Direction.backward)
    torch.cuda.synchronize()
    return dfft.gather_blocks(plan, t_out.cpu().numpy(), dst_side)


def random_input(shape, real, seed, precision="float64"):
    rng = np.random.default_rng(seed)
    if real:
        x = rng.uniform(-1.0, 1.0, shape)
    else:
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if precision == "float32":
        x = x.astype(np.float32 if real else np.complex64)
    return x


def out_extents(gin, axes, real):
    g = list(gin)
    if real:
        g[axes[-1]] = gin[axes[-1]] // 2 + 1
    return tuple(g)
