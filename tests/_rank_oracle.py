"""Per-rank test engines for the one-process-per-GPU path (dfft.DistributedPlan).

* ``OracleRankEngine``: one rank's block walk on the host (numpy pocketfft
  FFTs, ``dfft_oracle.pack`` / ``unpack``), segment by segment like a per-rank
  plan: used by the CPU (gloo) tests in place of the GPU segments, so that the
  process-group logic of DistributedPlan runs against the oracle.
* ``emulate_ranks``: every rank's GPU program in ONE process on one GPU, with
  the all-to-all of each exchange done by device copies between the ranks'
  buffers (no kernel waits on another rank).
"""
import numpy as np

import dfft_oracle as O


def logical(ext, m):
    """Extents in logical axis order of a block whose dim i holds axis m[i]."""
    out = [0] * len(m)
    for i, a in enumerate(m):
        out[a] = ext[i]
    return tuple(out)


def local_box(plan, rank, which):
    ext, st = plan.local_extents(rank, which)
    return tuple(slice(s, s + e) for s, e in zip(st, ext))


def scale_of(plan_args, forward):
    gin, gout, axes, norm = plan_args["in_extents"], plan_args["out_extents"], plan_args["axes"], plan_args["norm"]
    N = float(np.prod([max(gin[a], gout[a]) for a in axes]))
    if forward:
        return {"backward": 1.0, "forward": 1.0 / N, "ortho": 1.0 / np.sqrt(N), "none": 1.0}[norm]
    return {"backward": 1.0 / N, "forward": 1.0, "ortho": 1.0 / np.sqrt(N), "none": 1.0}[norm]


class OracleRankEngine:
    """Segments of rank `rank`'s program computed on the host.

    ``plan`` is any dfft.Plan over the same problem (its block lists are
    queried); ``args`` the plan arguments (in_extents, out_extents, axes,
    real_input, norm, layout)."""

    def __init__(self, plan, rank, args):
        self.rank = rank
        self.args = args
        self.blocks = plan.block_infos(rank)
        self.right = args.get("layout", "right") == "right"
        self.D = len(args["in_extents"])

    def _segments(self, forward):
        """Lists of FFT blocks between exchanges, and the transpose blocks."""
        nb = len(self.blocks)
        order = range(nb) if forward else range(nb - 1, -1, -1)
        segs, cur, xs = [], [], []
        for i in order:
            b = self.blocks[i]
            if b["block_type"] == "FFT":
                cur.append(b)
            else:
                segs.append(cur)
                cur = []
                xs.append(b)
        segs.append(cur)
        return segs, xs

    def _fft_axes(self, b):
        D, m = self.D, b["in_map"]
        return [m[D - 1 - j] if self.right else m[j] for j in range(b["fft_dim"])]

    def segment(self, forward, s, inp, recv_bytes):
        """Returns ("send", buffer array) or ("out", local array)."""
        a = self.args
        real = a["real_input"]
        segs, xs = self._segments(forward)
        cdt = np.complex128
        if s == 0:
            loc = np.asarray(inp)
        else:
            b = xs[s - 1]
            bext = tuple(b["buffer_extents"])
            if forward:
                axis, shape = b["out_axis"], logical(b["out_extents"], b["out_map"])
            else:
                axis, shape = b["in_axis"], logical(b["in_extents"], b["in_map"])
            dt = recv_bytes.dtype
            recv = recv_bytes.reshape(bext, order="C" if self.right else "F")
            loc = O.unpack(recv, tuple(range(self.D)), axis, shape, dtype=dt, layout_right=self.right)
        blocks = segs[s]
        if forward:
            for b in blocks:
                for j, ax in enumerate(self._fft_axes(b)):
                    if not np.iscomplexobj(loc) and real:
                        loc = np.fft.rfft(loc, axis=ax)
                    else:
                        loc = np.fft.fft(loc.astype(cdt), axis=ax)
        else:
            for b in blocks:
                axes = self._fft_axes(b)
                for jj in range(len(axes) - 1, -1, -1):
                    ax = axes[jj]
                    if real and b["block_idx"] == 0 and jj == 0:
                        n = a["in_extents"][ax]
                        loc = np.fft.irfft(loc, n=n, axis=ax) * n
                    else:
                        loc = np.fft.ifft(loc, axis=ax) * loc.shape[ax]
        if s < len(xs):
            b = xs[s]
            axis = b["in_axis"] if forward else b["out_axis"]
            buf = O.pack(loc, tuple(range(self.D)), axis, tuple(b["buffer_extents"]), self.right)
            return "send", buf
        return "out", loc * scale_of(a, forward)

    def buffer_bytes(self, buf):
        return np.ascontiguousarray(buf.ravel(order="C" if self.right else "F")).view(np.uint8)

    def bytes_to_buffer(self, raw, dtype):
        return np.frombuffer(raw.tobytes(), dtype=dtype)


def emulate_ranks(plans, ins, outs, direction):
    """Run every rank's per-rank plan on the current GPU in one process.

    plans[r] = dfft.Plan(..., process_rank=r); ins / outs: per-rank device
    tensors.  Returns the per-exchange lists of every rank's send and recv
    buffers (uint8 device tensors) for inspection."""
    import torch
    from dfft.distributed import exchange_group, exchange_schedule, execute_segment
    P = len(plans)
    sched = [exchange_schedule(p, direction) for p in plans]
    nx = len(sched[0])
    assert all(len(s) == nx for s in sched)
    dev = ins[0].device
    record = []
    recvs = [None] * P
    for s in range(nx + 1):
        sends = [None] * P
        for r in range(P):
            send = None
            if s < nx:
                send = torch.zeros(sched[r][s].nbytes, dtype=torch.uint8, device=dev)
                sends[r] = send
            execute_segment(plans[r], direction, s, ins[r], outs[r], send, recvs[r])
        if s == nx:
            break
        new_recvs = []
        for r in range(P):
            x = sched[r][s]
            sub, members = exchange_group(plans[r], direction, s, r, x.group_size)
            chunk = x.nbytes // x.group_size
            recv = torch.empty(x.nbytes, dtype=torch.uint8, device=dev)
            for j, m in enumerate(members):
                assert sched[m][s].nbytes == x.nbytes
                assert exchange_group(plans[m], direction, s, m, x.group_size) == (j, members), (m, members)
                # MPI_Alltoall: chunk j of r's recv is chunk sub(r) of member j's send
                recv[j * chunk:(j + 1) * chunk] = sends[m][sub * chunk:(sub + 1) * chunk]
            new_recvs.append(recv)
        record.append((sends, new_recvs))
        recvs = new_recvs
    torch.cuda.synchronize()
    return record
