"""Python mirror of the reference's distributed plan interface.

Reference API (paths relative to the reference's ``distributed/src/``)::

    KokkosFFT::Distributed::Plan plan(exec, in, out, axes, in_topology,
                                      out_topology, comm, norm);   // _Plan.hpp:154-181
    KokkosFFT::Distributed::execute(plan, in, out, direction);     // _Plan.hpp:212-238
    plan.name();                                                   // _Plan.hpp:200

Here one process drives one GPU and the ranks of the topologies are virtual.
Instead of per-rank views the plan takes the global extents, and ``execute``
takes buffers that hold the local blocks of all ranks concatenated in rank
order (see ``Plan.local_extents`` / ``Plan.local_offset`` and the
``scatter_blocks`` / ``gather_blocks`` helpers).  Errors raise
``DistributedFFTError`` with the library's message, like the reference's
``std::runtime_error``.
"""
import ctypes
import enum

import numpy as np

from ._lib import BlockInfo, PlanDesc, lib, MAX_RANK


class Direction(enum.IntEnum):
    forward = 0
    backward = 1


class Normalization(enum.IntEnum):
    backward = 0
    forward = 1
    ortho = 2
    none = 3


class ExecMode(enum.IntEnum):
    fused = 0
    literal = 1
    literal_capture = 2


class Status(enum.IntEnum):
    SUCCESS = 0
    INVALID_ARGUMENT = 1
    INVALID_TOPOLOGY = 2
    INVALID_EXTENTS = 3
    UNSUPPORTED = 4
    CUDA = 5
    ALLOC = 6
    INTERNAL = 7
    TIMEOUT = 8


class DistributedFFTError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{Status(status).name}: {message}")
        self.status = Status(status)


def _check(status):
    if status != 0:
        msg = lib.dfft_last_error_string().decode()
        raise DistributedFFTError(status, msg)


def _as_norm(norm):
    if isinstance(norm, str):
        return Normalization[norm]
    return Normalization(norm)


def _ptr(x):
    """Device pointer of a torch tensor, or an int / ctypes pointer as is."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(int(x))


class Plan:
    """Distributed FFT plan over virtual ranks on the current CUDA device.

    Parameters mirror the reference constructor:
      in_extents / out_extents : global extents of the input / output view
          (for R2C the input is real and out_extents[last FFT axis] = n // 2 + 1)
      axes : FFT axes (1 to 3; negative values count from the end)
      in_topology / out_topology : ranks along each axis
      real_input : R2C forward / C2R backward plan (else C2C)
      precision : "float64", "float32" or "float32_compensated" (complex64 with
                  the last radix pass of the two-line C2C stages compensated)
      norm : Normalization (default backward)
      layout : memory order of the local blocks, "right" (C) or "left" (Fortran)
      in_topology_layout / out_topology_layout : rank order of the topologies
      exec_mode : "fused" (default) or "literal" (reference block sequence)
      stream : CUDA stream handle (int) the plan launches on
      analyze_only : plan on the host only (no device memory; cannot execute)
      process_rank : build only this world rank's program (one process per
                     GPU; executed by dfft.DistributedPlan segment by segment)
    """

    def __init__(self, in_extents, out_extents, axes, in_topology, out_topology, real_input=False,
                 precision="float64", norm=Normalization.backward, layout="right", in_topology_layout="right",
                 out_topology_layout="right", exec_mode="fused", stream=None, analyze_only=False,
                 process_rank=None):
        rank = len(in_extents)
        if not (len(out_extents) == len(in_topology) == len(out_topology) == rank):
            raise DistributedFFTError(Status.INVALID_ARGUMENT, "extents and topologies must have the view rank")
        if rank > MAX_RANK:
            raise DistributedFFTError(Status.UNSUPPORTED, f"view rank {rank} > {MAX_RANK}")
        d = PlanDesc()
        lib.dfft_plan_desc_init(ctypes.byref(d))
        d.rank = rank
        axes = list(axes)
        if not 1 <= len(axes) <= 3:
            raise DistributedFFTError(Status.INVALID_ARGUMENT, "the Rank of FFT axes must be between 1 and 3")
        d.fft_rank = len(axes)
        for i, a in enumerate(axes):
            d.axes[i] = int(a)
        for k in range(rank):
            d.in_extents[k] = int(in_extents[k])
            d.out_extents[k] = int(out_extents[k])
            d.in_topology[k] = int(in_topology[k])
            d.out_topology[k] = int(out_topology[k])
        d.in_topology_layout_right = 1 if in_topology_layout == "right" else 0
        d.out_topology_layout_right = 1 if out_topology_layout == "right" else 0
        d.view_layout_right = 1 if layout == "right" else 0
        d.kind = 1 if real_input else 0
        if precision not in ("float64", "float32", "float32_compensated"):
            raise DistributedFFTError(Status.INVALID_ARGUMENT, f"unknown precision {precision}")
        d.precision = {"float64": 0, "float32": 1, "float32_compensated": 2}[precision]
        d.normalization = int(_as_norm(norm))
        d.exec_mode = int(ExecMode[exec_mode] if isinstance(exec_mode, str) else exec_mode)
        d.stream = ctypes.c_void_p(int(stream)) if stream else None
        self._desc = d
        self.rank = rank
        self.real_input = bool(real_input)
        self.precision = precision
        self.in_extents = tuple(int(x) for x in in_extents)
        self.out_extents = tuple(int(x) for x in out_extents)
        self.axes = tuple(int(a) % rank for a in axes)
        self.in_topology = tuple(int(x) for x in in_topology)
        self.out_topology = tuple(int(x) for x in out_topology)
        self.layout = layout
        self._h = ctypes.c_void_p()
        self.process_rank = None if process_rank is None else int(process_rank)
        if process_rank is None:
            fn = lib.dfft_plan_analyze if analyze_only else lib.dfft_plan_create
            _check(fn(ctypes.byref(self._h), ctypes.byref(d)))
        else:
            fn = lib.dfft_plan_analyze_rank if analyze_only else lib.dfft_plan_create_rank
            _check(fn(ctypes.byref(self._h), ctypes.byref(d), int(process_rank)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.dfft_plan_destroy(h)
            self._h = None

    # -- reference-facing queries ------------------------------------------
    def name(self):
        return lib.dfft_plan_name(self._h).decode()

    @property
    def nprocs(self):
        n = ctypes.c_int64()
        _check(lib.dfft_get_nprocs(self._h, ctypes.byref(n)))
        return n.value

    def local_extents(self, rank, which="in"):
        """(extents, starts) of a rank's block (compute_local_extents_and_starts)."""
        e = (ctypes.c_uint64 * MAX_RANK)()
        s = (ctypes.c_uint64 * MAX_RANK)()
        _check(lib.dfft_get_local_extents(self._h, rank, 0 if which == "in" else 1, e, s))
        return tuple(e[:self.rank]), tuple(s[:self.rank])

    def local_offset(self, rank, which="in"):
        o = ctypes.c_uint64()
        _check(lib.dfft_get_local_offset(self._h, rank, 0 if which == "in" else 1, ctypes.byref(o)))
        return o.value

    def buffer_elements(self, which="in"):
        c = ctypes.c_uint64()
        _check(lib.dfft_get_buffer_elements(self._h, 0 if which == "in" else 1, ctypes.byref(c)))
        return c.value

    @property
    def max_buffer_size(self):
        c = ctypes.c_uint64()
        _check(lib.dfft_get_max_buffer_size(self._h, ctypes.byref(c)))
        return c.value

    def block_infos(self, rank=0):
        n = ctypes.c_int64()
        _check(lib.dfft_get_num_blocks(self._h, ctypes.byref(n)))
        out = []
        D = self.rank
        for b in range(n.value):
            bi = BlockInfo()
            _check(lib.dfft_get_block_info(self._h, rank, b, ctypes.byref(bi)))
            out.append(dict(
                block_type="FFT" if bi.block_type == 1 else "Transpose", block_idx=bi.block_idx,
                fft_dim=bi.fft_dim, in_axis=bi.in_axis, out_axis=bi.out_axis, comm_axis=bi.comm_axis,
                in_topology=tuple(bi.in_topology[:D]), out_topology=tuple(bi.out_topology[:D]),
                in_extents=tuple(bi.in_extents[:D]), out_extents=tuple(bi.out_extents[:D]),
                buffer_extents=tuple(bi.buffer_extents[:D + 1]), in_map=tuple(bi.in_map[:D]),
                out_map=tuple(bi.out_map[:D])))
        return out

    def topology_chain(self):
        n = ctypes.c_int64(0)
        _check(lib.dfft_get_topology_chain(self._h, ctypes.byref(n), None, None, None))
        cnt = n.value
        topos = (ctypes.c_uint64 * (cnt * self.rank))()
        tr = (ctypes.c_int64 * max(cnt, 1))()
        lay = (ctypes.c_int64 * max(cnt, 1))()
        _check(lib.dfft_get_topology_chain(self._h, ctypes.byref(n), topos, tr, lay))
        t = [tuple(topos[i * self.rank:(i + 1) * self.rank]) for i in range(cnt)]
        return t, list(tr[:max(cnt - 1, 0)]), list(lay[:cnt])

    def launch_count(self, direction=Direction.forward):
        n = ctypes.c_int64()
        _check(lib.dfft_get_launch_count(self._h, int(direction), ctypes.byref(n)))
        return n.value

    def device_error(self, reset=False):
        """0, or the code a kernel's bounded wait left (1: a TMA tile load timed out)."""
        c = ctypes.c_int32()
        _check(lib.dfft_get_device_error(self._h, 1 if reset else 0, ctypes.byref(c)))
        return c.value

    def workspace_bytes(self):
        n = ctypes.c_uint64()
        _check(lib.dfft_get_workspace_bytes(self._h, ctypes.byref(n)))
        return n.value

    def export_buffers(self, direction, block, which):
        """Data recorded by the last ``exec_mode="literal_capture"`` execute for
        transpose block ``block``:

        * ``"send"`` / ``"recv"``: all ranks' buffers, shape (nprocs, *buffer_extents)
          in the reference's buffer order;
        * ``"pack_in"`` / ``"unpack_out"``: list of every rank's local array (dims
          in the order of the block's map) that was packed / unpacked."""
        infos = [self.block_infos(r) for r in range(self.nprocs)]
        bi = infos[0][block]
        if bi["block_type"] != "Transpose":
            raise DistributedFFTError(Status.INVALID_ARGUMENT, "not a transpose block")
        real = self.real_input and all(b["block_type"] == "Transpose" for b in infos[0][:block])
        dt = (np.float64 if real else np.complex128) if self.precision == "float64" else \
            (np.float32 if real else np.complex64)
        order = "C" if self.layout == "right" else "F"
        code = dict(send=0, recv=1, pack_in=2, unpack_out=3)[which]
        fwd = Direction(direction) == Direction.forward
        if code < 2:
            bext = tuple(bi["buffer_extents"])
            per_rank = int(np.prod(bext))
            flat = np.zeros(self.nprocs * per_rank, dtype=dt)
        else:
            side = "in_extents" if (code == 2) == fwd else "out_extents"
            shapes = [tuple(infos[r][block][side]) for r in range(self.nprocs)]
            flat = np.zeros(sum(int(np.prod(s)) for s in shapes), dtype=dt)
        _check(lib.dfft_debug_export_buffers(self._h, int(direction), block, code,
                                             flat.ctypes.data_as(ctypes.c_void_p), flat.nbytes))
        if code < 2:
            return np.stack([flat[r * per_rank:(r + 1) * per_rank].reshape(bext, order=order)
                             for r in range(self.nprocs)])
        out, off = [], 0
        for s in shapes:
            n = int(np.prod(s))
            out.append(flat[off:off + n].reshape(s, order=order))
            off += n
        return out


class Graph:
    """A CUDA graph holding a batch of transforms: ``items`` is a list of
    (plan, in_buf, out_buf, direction[, branch]); items with the same branch
    run in order, different branches run concurrently (default: one branch per
    item).  Every ``launch()`` replays them on the same buffers."""

    def __init__(self, items):
        n = len(items)
        br = (ctypes.c_int32 * n)(*[int(it[4]) if len(it) > 4 else i for i, it in enumerate(items)])
        plans = (ctypes.c_void_p * n)(*[it[0]._h.value for it in items])
        ins = (ctypes.c_void_p * n)(*[_ptr(it[1]).value for it in items])
        outs = (ctypes.c_void_p * n)(*[_ptr(it[2]).value for it in items])
        dirs = (ctypes.c_int32 * n)(*[int(Direction(it[3])) for it in items])
        self._keep = [it[0] for it in items]  # plans must outlive the graph
        self._h = ctypes.c_void_p()
        _check(lib.dfft_graph_create(ctypes.byref(self._h), plans, ins, outs, dirs, br, n))

    @classmethod
    def _from_handle(cls, h, keep):
        g = cls.__new__(cls)
        g._h, g._keep = h, keep
        return g

    def launch(self, stream=None):
        _check(lib.dfft_graph_launch(self._h, ctypes.c_void_p(int(stream)) if stream else None))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.dfft_graph_destroy(h)
            self._h = None


class Batch:
    """Batched execution of distinct plans (fields of uneven sizes): one
    persistent launch per stage of all fields.  ``execute(ins, outs,
    direction)`` transforms ins[i] -> outs[i] with plans[i]."""

    def __init__(self, plans):
        n = len(plans)
        arr = (ctypes.c_void_p * n)(*[p._h.value for p in plans])
        self._keep = list(plans)  # plans must outlive the batch
        self._h = ctypes.c_void_p()
        _check(lib.dfft_batch_create(ctypes.byref(self._h), arr, n))

    def execute(self, ins, outs, direction, stream=None):
        n = len(self._keep)
        if len(ins) != n or len(outs) != n:
            raise DistributedFFTError(Status.INVALID_ARGUMENT, "one input and one output per plan")
        a = (ctypes.c_void_p * n)(*[_ptr(x).value for x in ins])
        b = (ctypes.c_void_p * n)(*[_ptr(x).value for x in outs])
        _check(lib.dfft_batch_execute(self._h, a, b, int(Direction(direction)),
                                      ctypes.c_void_p(int(stream)) if stream else None))

    def launch_count(self, direction=Direction.forward):
        n = ctypes.c_int64()
        _check(lib.dfft_batch_get_launch_count(self._h, int(Direction(direction)), ctypes.byref(n)))
        return n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.dfft_batch_destroy(h)
            self._h = None


def all_topologies(kind, in_topology, out_topology, axes, in_layout="right", out_layout="right"):
    """get_all_slab_topologies / get_all_pencil_topologies on their own.

    Returns the chain for slabs, and (chain, trans_axes, layouts) for pencils."""
    rank = len(in_topology)
    pencil = 1 if kind == "pencil" else 0
    it = (ctypes.c_uint64 * rank)(*in_topology)
    ot = (ctypes.c_uint64 * rank)(*out_topology)
    ax = (ctypes.c_int32 * len(axes))(*axes)
    n = ctypes.c_int64(0)
    _check(lib.dfft_get_all_topologies(pencil, rank, it, 1 if in_layout == "right" else 0, ot,
                                       1 if out_layout == "right" else 0, len(axes), ax, ctypes.byref(n),
                                       None, None, None))
    cnt = n.value
    topos = (ctypes.c_uint64 * (cnt * rank))()
    tr = (ctypes.c_int64 * max(cnt, 1))()
    lay = (ctypes.c_int64 * max(cnt, 1))()
    _check(lib.dfft_get_all_topologies(pencil, rank, it, 1 if in_layout == "right" else 0, ot,
                                       1 if out_layout == "right" else 0, len(axes), ax, ctypes.byref(n),
                                       topos, tr, lay))
    chain = [tuple(topos[i * rank:(i + 1) * rank]) for i in range(cnt)]
    if not pencil:
        return chain
    return chain, list(tr[:max(cnt - 1, 0)]), list(lay[:cnt])


def execute(plan, in_buf, out_buf, direction, stream=None):
    """execute(plan, in, out, direction) on concatenated per-rank buffers.

    Forward: ``in_buf`` holds the input layout, ``out_buf`` receives the output
    layout.  Backward: ``in_buf`` holds the (complex) output layout and
    ``out_buf`` receives the input layout.  Asynchronous on the plan's stream
    (or ``stream``)."""
    direction = Direction(direction)
    if stream is None:
        _check(lib.dfft_execute(plan._h, _ptr(in_buf), _ptr(out_buf), int(direction)))
    else:
        _check(lib.dfft_execute_on_stream(plan._h, _ptr(in_buf), _ptr(out_buf), int(direction),
                                          ctypes.c_void_p(int(stream))))


def execute_adjoint(plan, in_buf, out_buf, direction, stream=None):
    """Adjoint (conjugate transpose, normalisation included) of the plan's
    forward (``direction=forward``: output layout -> input layout) or backward
    transform (input layout -> output layout)."""
    direction = Direction(direction)
    _check(lib.dfft_execute_adjoint(plan._h, _ptr(in_buf), _ptr(out_buf), int(direction),
                                    ctypes.c_void_p(int(stream)) if stream else None))


def scatter_blocks(plan, global_array, which="in"):
    """Concatenate the per-rank blocks of a global (numpy) array in rank order,
    each block in the plan's memory order."""
    a = np.asarray(global_array)
    parts = []
    for r in range(plan.nprocs):
        ext, st = plan.local_extents(r, which)
        sl = tuple(slice(s, s + e) for s, e in zip(st, ext))
        blk = a[sl]
        parts.append(np.ravel(blk, order="C" if plan.layout == "right" else "F"))
    return np.concatenate(parts) if parts else np.zeros(0, a.dtype)


def gather_blocks(plan, flat, which="in", dtype=None):
    """Inverse of scatter_blocks: rebuild the global (numpy) array."""
    flat = np.asarray(flat)
    shape = plan.in_extents if which == "in" else plan.out_extents
    out = np.zeros(shape, dtype=dtype or flat.dtype)
    for r in range(plan.nprocs):
        ext, st = plan.local_extents(r, which)
        off = plan.local_offset(r, which)
        n = int(np.prod(ext))
        blk = flat[off:off + n].reshape(ext, order="C" if plan.layout == "right" else "F")
        out[tuple(slice(s, s + e) for s, e in zip(st, ext))] = blk
    return out
