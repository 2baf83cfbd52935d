"""One process per GPU: the reference's distributed plan over a real communicator.

Python mirror of ``KokkosFFT::Distributed::Plan(exec, in, out, axes,
in_topology, out_topology, comm)`` (KokkosFFT_Distributed_Plan.hpp:154-238)
on one rank of a ``torch.distributed`` process group of
``prod(in_topology)`` processes.  Each process holds its own local input and
output blocks (``local_shape``: the rank's block of the input / output
topology, logical axis order, C order for LayoutRight views) on its own GPU.

The rank's program (``dfft_plan_create_rank``) runs as segments of fused FFT
stage kernels; between two segments the send buffer, written by the last
stage in the reference's pack order, goes through ``all_to_all_single`` over
the exchange's group -- the whole group for slab plans, the row / column
sub-communicator of the Cartesian grid over the split entries of in_topology
for pencil plans (KokkosFFT_Distributed_PencilPlan.hpp:32-71, created with
``new_group`` once per plan) -- the reference's MPI_Alltoall /
ncclSend-ncclRecv exchange (KokkosFFT_Distributed_MPI_All2All.hpp:23-58,
KokkosFFT_Distributed_NCCL_All2All.hpp:21-89).  With the NCCL backend the
device buffers go to NCCL directly (NVLink / NVSwitch); a gloo group stages
them through host memory.
"""
import ctypes

from ._lib import EXCHANGE_FN, ExchangeInfo, lib
from .plan import Direction, DistributedFFTError, Normalization, Plan, Status, _check, _ptr


class Exchange:
    """One all-to-all of a direction: transpose block, group, buffer size."""

    def __init__(self, info, sub_rank, members):
        self.block = int(info.block)
        self.comm_axis = int(info.comm_axis)
        self.padded = bool(info.padded)
        self.elements = int(info.elements)
        self.element_bytes = int(info.element_bytes)
        self.group_size = int(info.group_size)
        self.nbytes = self.elements * self.element_bytes
        self.sub_rank = sub_rank
        self.members = tuple(members)  # group ranks by sub-rank
        self.process_group = None


def exchange_schedule(plan, direction):
    """The exchanges of a per-rank plan (``Plan(..., process_rank=r)``) in
    execution order, as seen by its own rank."""
    h = plan._h
    n = ctypes.c_int64()
    _check(lib.dfft_get_num_exchanges(h, int(direction), ctypes.byref(n)))
    out = []
    for k in range(n.value):
        info = ExchangeInfo()
        _check(lib.dfft_get_exchange_info(h, int(direction), k, ctypes.byref(info)))
        out.append(Exchange(info, *exchange_group(plan, direction, k, plan.process_rank, info.group_size)))
    return out


def exchange_group(plan, direction, k, rank, group_size=None):
    """(sub-rank, members) of exchange k of a direction seen by world rank `rank`."""
    h = plan._h
    if group_size is None:
        info = ExchangeInfo()
        _check(lib.dfft_get_exchange_info(h, int(direction), k, ctypes.byref(info)))
        group_size = info.group_size
    sub = ctypes.c_int64()
    mem = (ctypes.c_int64 * group_size)()
    _check(lib.dfft_get_exchange_group(h, int(direction), k, int(rank), ctypes.byref(sub), mem))
    return sub.value, tuple(mem)


def execute_segment(plan, direction, segment, inp, out, send, recv, stream=None):
    """Run segment `segment` of a per-rank plan (dfft_execute_segment)."""
    _check(lib.dfft_execute_segment(plan._h, int(direction), int(segment), _ptr(inp), _ptr(out), _ptr(send),
                                    _ptr(recv), None if stream is None else ctypes.c_void_p(int(stream))))


class DistributedPlan:
    """A distributed FFT plan of which this process executes one rank.

    Arguments as for ``dfft.Plan`` (global extents and topologies), plus
      group : the torch.distributed process group whose ranks are the
              topology's ranks (default: the world group); its size must be
              prod(in_topology)
      analyze_only : host-side planning only (exchange schedule and groups;
              no device memory, no execution)
    """

    def __init__(self, in_extents, out_extents, axes, in_topology, out_topology, real_input=False,
                 precision="float64", norm=Normalization.backward, layout="right", in_topology_layout="right",
                 out_topology_layout="right", group=None, stream=None, analyze_only=False):
        import torch
        import torch.distributed as dist
        if not dist.is_available() or not dist.is_initialized():
            raise DistributedFFTError(Status.INVALID_ARGUMENT, "torch.distributed is not initialized")
        self.group = group if group is not None else dist.group.WORLD
        self.rank = dist.get_rank(self.group)
        self.world_size = dist.get_world_size(self.group)
        self.plan = Plan(in_extents, out_extents, axes, in_topology, out_topology, real_input=real_input,
                         precision=precision, norm=norm, layout=layout, in_topology_layout=in_topology_layout,
                         out_topology_layout=out_topology_layout, stream=stream, analyze_only=analyze_only,
                         process_rank=self.rank)
        if self.plan.nprocs != self.world_size:
            raise DistributedFFTError(
                Status.INVALID_TOPOLOGY,
                f"the topology has {self.plan.nprocs} ranks but the communicator has {self.world_size}")
        self.analyze_only = analyze_only
        self.device = torch.device("cpu") if analyze_only else torch.device("cuda", torch.cuda.current_device())
        self.exchanges = {d: exchange_schedule(self.plan, d) for d in (Direction.forward, Direction.backward)}
        self._make_groups(dist)
        nbytes = max([x.nbytes for xs in self.exchanges.values() for x in xs] + [16])
        # send / recv buffers shared by every exchange (bytes; zeroed once, the
        # padded exchanges clear the send buffer again before their segment)
        self._send = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        self._recv = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)

    # -- schedule -----------------------------------------------------------
    def exchange_groups(self, direction, k):
        """(sub-rank, members) of exchange k of a direction for every rank."""
        size = self.exchanges[Direction(direction)][k].group_size
        return [exchange_group(self.plan, direction, k, r, size) for r in range(self.world_size)]

    def _make_groups(self, dist):
        """One process group per distinct member set, created by every process
        of the communicator in the same order (dist.new_group is collective)."""
        order = []
        for d in (Direction.forward, Direction.backward):
            for k in range(len(self.exchanges[d])):
                for _, members in self.exchange_groups(d, k):
                    if list(members) != sorted(members):
                        raise DistributedFFTError(Status.INTERNAL, "exchange group members out of rank order")
                    if members not in order:
                        order.append(members)
        world = tuple(range(self.world_size))
        local = self.group is not dist.group.WORLD
        groups = {}
        for members in order:
            if members == world:
                groups[members] = self.group
                continue
            if local:
                # a sub-group of a sub-communicator: only its members take part
                if self.rank in members:
                    ranks = [dist.get_global_rank(self.group, m) for m in members]
                    groups[members] = dist.new_group(ranks=ranks, use_local_synchronization=True)
            else:
                groups[members] = dist.new_group(ranks=list(members))
        for xs in self.exchanges.values():
            for x in xs:
                x.process_group = groups[x.members]  # this rank's own groups always exist

    # -- local blocks --------------------------------------------------------
    def local_shape(self, which="in"):
        """Extents (logical axis order) of this rank's block of the input /
        output topology."""
        return self.plan.local_extents(self.rank, which)[0]

    def local_starts(self, which="in"):
        return self.plan.local_extents(self.rank, which)[1]

    # -- execution -----------------------------------------------------------
    def _segment(self, direction, s, inp, out, send, recv, stream):
        execute_segment(self.plan, direction, s, inp, out, send, recv, stream)

    def _all_to_all(self, x, send, recv):
        import torch
        import torch.distributed as dist
        pg = x.process_group
        if send.device.type == "cuda" and dist.get_backend(pg) != "nccl":
            hs = send.cpu()
            hr = torch.empty_like(hs)
            dist.all_to_all_single(hr, hs, group=pg)
            recv.copy_(hr)
        else:
            dist.all_to_all_single(recv, send, group=pg)

    def execute(self, inp, out, direction=Direction.forward):
        """Forward: this rank's input block -> its output block; backward: the
        reverse.  Tensors on this process's device, contiguous."""
        import torch
        direction = Direction(direction)
        for t in (inp, out):
            if not t.is_contiguous():
                raise DistributedFFTError(Status.INVALID_ARGUMENT, "local blocks must be contiguous")
        stream = torch.cuda.current_stream(self.device).cuda_stream if self.device.type == "cuda" else None
        xs = self.exchanges[direction]
        for s in range(len(xs) + 1):
            send = recv = None
            if s < len(xs):
                send = self._send[:xs[s].nbytes]
                if xs[s].padded:
                    send.zero_()
            if s > 0:
                recv = self._recv[:xs[s - 1].nbytes]
            self._segment(direction, s, inp, out, send, recv, stream)
            if s < len(xs):
                self._all_to_all(xs[s], send, self._recv[:xs[s].nbytes])
        return out

    def execute_exchanged(self, inp, out, direction=Direction.forward):
        """The same transform through the C driver dfft_execute_exchanged: the
        library runs the segments and calls back into Python for every
        all-to-all (what a C / MPI host binds to its own communicator)."""
        import torch
        direction = Direction(direction)
        xs = self.exchanges[direction]
        stream = torch.cuda.current_stream(self.device).cuda_stream
        errors = []

        def exchange(user, k, send_p, recv_p, bytes_per_peer, st):
            try:
                x = xs[k]
                send = self._send[:x.nbytes]
                recv = self._recv[:x.nbytes]
                if send.data_ptr() != send_p or recv.data_ptr() != recv_p or bytes_per_peer * x.group_size != x.nbytes:
                    raise RuntimeError("exchange callback got unexpected buffers")
                self._all_to_all(x, send, recv)
                if k + 1 < len(xs) and xs[k + 1].padded:
                    self._send[:xs[k + 1].nbytes].zero_()
                return 0
            except Exception as e:  # reported through the status below
                errors.append(e)
                return 1

        cb = EXCHANGE_FN(exchange)
        if xs and xs[0].padded:
            self._send[:xs[0].nbytes].zero_()
        status = lib.dfft_execute_exchanged(self.plan._h, _ptr(inp), _ptr(out), int(direction), _ptr(self._send),
                                            _ptr(self._recv), cb, None, ctypes.c_void_p(stream))
        if errors:
            raise errors[0]
        _check(status)
        return out

    def forward(self, inp, out):
        return self.execute(inp, out, Direction.forward)

    def backward(self, inp, out):
        return self.execute(inp, out, Direction.backward)
