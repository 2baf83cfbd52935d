"""Worker processes of the multi-process tests of dfft.DistributedPlan.

Each process joins a torch.distributed group (127.0.0.1 rendezvous), builds
the plan of its own rank, runs every case forward and backward and saves its
local outputs and the exchange buffers it sent and received to `outdir`.

mode "oracle": gloo on CPU; the plan is host-only and its segments are the
    oracle's (OracleRankEngine), so the process-group logic, the exchange
    schedule and the byte layout of the exchanged buffers are exercised
    without a GPU.
mode "gpu":    gloo between processes that share one GPU (buffers staged
    through host memory by DistributedPlan); the segments are the library's
    CUDA kernels.  No kernel waits on another process.
"""
import os
from datetime import timedelta

import numpy as np


def case_input(case, seed):
    rng = np.random.default_rng(seed)
    shape = tuple(case["in_extents"])
    if case["real_input"]:
        return rng.uniform(-1.0, 1.0, shape)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def plan_kwargs(case):
    keys = ("in_extents", "out_extents", "axes", "in_topology", "out_topology", "real_input", "precision", "norm",
            "layout")
    return {k: case[k] for k in keys if k in case}


def _make_plan_class(mode):
    import torch

    from dfft import DistributedPlan
    from _rank_oracle import OracleRankEngine

    class Recording(DistributedPlan):
        """DistributedPlan whose segments are recorded (and, in oracle mode,
        computed on the host)."""

        def setup(self, case):
            self.case = case
            self.record = {}
            self.engine = OracleRankEngine(self.plan, self.rank, case) if mode == "oracle" else None

        def _segment(self, direction, s, inp, out, send, recv, stream):
            fwd = int(direction) == 0
            if recv is not None:
                self.record[(fwd, s - 1, "recv")] = recv.detach().cpu().numpy().copy()
            if mode == "oracle":
                order = "C" if self.case.get("layout", "right") == "right" else "F"
                xs = self.exchanges[direction]
                raw = None
                if s > 0:
                    x = xs[s - 1]
                    dt = np.complex128 if x.element_bytes == 16 else np.float64
                    raw = recv.numpy().view(dt)
                src = None
                if s == 0:
                    shape = self.local_shape("in" if fwd else "out")
                    src = inp.numpy().reshape(shape, order=order)
                kind, arr = self.engine.segment(fwd, s, src, raw)
                if kind == "send":
                    send.numpy()[:] = self.engine.buffer_bytes(arr)
                else:
                    out.numpy()[:] = np.asarray(arr).astype(out.numpy().dtype).ravel(order=order)
            else:
                super()._segment(direction, s, inp, out, send, recv, stream)
                torch.cuda.synchronize()
            if send is not None:
                self.record[(fwd, s, "send")] = send.detach().cpu().numpy().copy()

    return Recording


def worker(rank, world, port, cases, outdir, mode):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        Recording = _make_plan_class(mode)
        for ci, case in enumerate(cases):
            dev = "cpu"
            if mode == "gpu":
                torch.cuda.set_device(0)
                dev = "cuda"
            plan = Recording(**plan_kwargs(case), analyze_only=(mode == "oracle"))
            plan.setup(case)
            order = "C" if case.get("layout", "right") == "right" else "F"
            x = case_input(case, case.get("seed", 0))
            box = tuple(slice(s, s + e) for s, e in zip(plan.local_starts("in"), plan.local_shape("in")))
            xl = np.ascontiguousarray(x[box].ravel(order=order))
            if case.get("precision", "float64") == "float32":
                xl = xl.astype(np.float32 if case["real_input"] else np.complex64)
            cdt = torch.complex128 if case.get("precision", "float64") == "float64" else torch.complex64
            t_in = torch.from_numpy(xl).to(dev)
            n_out = int(np.prod(plan.local_shape("out")))
            y = torch.zeros(n_out, dtype=cdt, device=dev)
            plan.execute(t_in, y, 0)
            xb = torch.zeros_like(t_in)
            plan.execute(y, xb, 1)
            res = {"y": y.cpu().numpy(), "xb": xb.cpu().numpy()}
            if mode == "gpu":
                # the same transform through the C driver with the exchange callback
                y2 = torch.zeros_like(y)
                plan.execute_exchanged(t_in, y2, 0)
                xb2 = torch.zeros_like(t_in)
                plan.execute_exchanged(y2, xb2, 1)
                torch.cuda.synchronize()
                res["y2"] = y2.cpu().numpy()
                res["xb2"] = xb2.cpu().numpy()
            for (fwd, k, which), v in plan.record.items():
                res[f"{'f' if fwd else 'b'}_{k}_{which}"] = v
            np.savez(os.path.join(outdir, f"case{ci}_rank{rank}.npz"), **res)
            dist.barrier()
            del plan
    finally:
        dist.destroy_process_group()
