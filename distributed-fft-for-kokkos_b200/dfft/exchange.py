"""The reference's data-movement layer and layout math through the C ABI.

Python mirrors of (paths relative to the reference's ``distributed/src/``)::

    Impl::pack(exec, src, dst, src_map, axis)          // _PackUnpack.hpp:439-460
    Impl::unpack(exec, src, dst, dst_map, axis)        // _PackUnpack.hpp:478-499
    Impl::all2all(send, recv, comm)                    // _MPI_All2All.hpp:23-58
    Impl::TransBlock(exec, buffer_extents, src_map, src_axis, dst_map, dst_axis)
        (comm, in, out, send, recv, direction)         // _TransBlock.hpp:38-107
    rank_to_coord, compute_local_extents_and_starts    // _MPI_Extents.hpp:492-577
    Impl::compute_buffer_extents<Layout>               // _Extents.hpp:35-90
    Impl::permute_map_by_axes<Layout>                  // _Mapping.hpp:39-110
    Impl::propose_transpose_block                      // _BlockAnalyses.hpp:93-136

Views and buffers are torch tensors on the GPU (any element type of 4, 8 or
16 bytes).  ``pack`` / ``unpack`` act on one rank's view like the reference;
``all2all`` and ``TransBlock`` act on every virtual rank at once, with the
ranks' buffers / blocks concatenated in rank order.
"""
import ctypes

from ._lib import BlockInfo, TransBlockDesc, lib
from .plan import Direction, _check, _ptr


def _u64(v):
    return (ctypes.c_uint64 * max(1, len(v)))(*[int(x) for x in v])


def _i32(v):
    return (ctypes.c_int32 * max(1, len(v)))(*[int(x) for x in v])


def _stream(stream):
    return None if stream is None else ctypes.c_void_p(int(stream))


def _layout_right(layout):
    if layout not in ("right", "left"):
        raise ValueError("layout must be 'right' or 'left'")
    return 1 if layout == "right" else 0


def pack(src, dst, src_map, axis, src_extents, buffer_extents, layout="right", stream=None):
    """dst (buffer, rank D+1) <- src (view of rank D with extents src_extents,
    dimension i holding logical axis src_map[i]) split along logical `axis`."""
    D = len(src_extents)
    _check(lib.dfft_pack(D, _u64(src_extents), _i32(src_map), int(axis), _u64(buffer_extents), _layout_right(layout),
                         src.element_size(), _ptr(src), _ptr(dst), _stream(stream)))


def unpack(src, dst, dst_map, axis, buffer_extents, dst_extents, layout="right", stream=None):
    """dst (view with extents dst_extents, permuted by dst_map) <- src (buffer)
    merged along logical `axis`."""
    D = len(dst_extents)
    _check(lib.dfft_unpack(D, _u64(buffer_extents), _i32(dst_map), int(axis), _u64(dst_extents),
                           _layout_right(layout), src.element_size(), _ptr(src), _ptr(dst), _stream(stream)))


def all2all(send, recv, nprocs, buffer_extents, comm_axis=-1, cart_topology=None, layout="right", stream=None):
    """MPI_Alltoall of every virtual rank over the world (comm_axis -1) or the
    row / column communicators (0 / 1) of the Cartesian grid of cart_topology."""
    cart = list(cart_topology) if cart_topology is not None else []
    _check(lib.dfft_all2all(int(nprocs), len(buffer_extents), _u64(buffer_extents), _layout_right(layout),
                            int(comm_axis), len(cart), _u64(cart), send.element_size(), _ptr(send), _ptr(recv),
                            _stream(stream)))


class TransBlock:
    """pack -> all2all -> unpack over every rank of a topology pair."""

    def __init__(self, global_extents, in_topology, out_topology, src_map, src_axis, dst_map, dst_axis,
                 element_bytes, layout="right", in_topology_layout="right", out_topology_layout="right",
                 comm_axis=-1, cart_topology=None):
        D = len(global_extents)
        d = TransBlockDesc()
        d.rank = D
        for k in range(D):
            d.global_extents[k] = int(global_extents[k])
            d.in_topology[k] = int(in_topology[k])
            d.out_topology[k] = int(out_topology[k])
            d.src_map[k] = int(src_map[k])
            d.dst_map[k] = int(dst_map[k])
            if cart_topology is not None:
                d.cart_topology[k] = int(cart_topology[k])
        d.in_topology_layout_right = _layout_right(in_topology_layout)
        d.out_topology_layout_right = _layout_right(out_topology_layout)
        d.src_axis = int(src_axis)
        d.dst_axis = int(dst_axis)
        d.view_layout_right = _layout_right(layout)
        d.element_bytes = int(element_bytes)
        d.comm_axis = int(comm_axis)
        h = ctypes.c_void_p()
        _check(lib.dfft_trans_block_create(ctypes.byref(h), ctypes.byref(d)))
        self._h = h
        self.rank = D

    def buffer_extents(self):
        out = (ctypes.c_uint64 * (self.rank + 1))()
        _check(lib.dfft_trans_block_buffer_extents(self._h, out))
        return tuple(int(x) for x in out)

    def __call__(self, inp, out, send, recv, direction=Direction.forward, stream=None):
        _check(lib.dfft_trans_block_execute(self._h, _ptr(inp), _ptr(out), _ptr(send), _ptr(recv),
                                            int(Direction(direction)), _stream(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.dfft_trans_block_destroy(h)
            self._h = None


def rank_to_coord(topology, rank, layout="right"):
    out = (ctypes.c_uint64 * len(topology))()
    _check(lib.dfft_rank_to_coord(len(topology), _u64(topology), _layout_right(layout), int(rank), out))
    return tuple(int(x) for x in out)


def compute_local_extents_and_starts(global_extents, topology, rank, layout="right"):
    D = len(global_extents)
    e, s = (ctypes.c_uint64 * D)(), (ctypes.c_uint64 * D)()
    _check(lib.dfft_compute_local_extents_and_starts(D, _u64(global_extents), _u64(topology), _layout_right(layout),
                                                     int(rank), e, s))
    return tuple(int(x) for x in e), tuple(int(x) for x in s)


def compute_buffer_extents(global_extents, in_topology, out_topology, layout="right"):
    D = len(global_extents)
    out = (ctypes.c_uint64 * (D + 1))()
    _check(lib.dfft_compute_buffer_extents(D, _u64(global_extents), _u64(in_topology), _u64(out_topology),
                                           _layout_right(layout), out))
    return tuple(int(x) for x in out)


def permute_map_by_axes(src_map, axes, layout="right"):
    if isinstance(axes, int):
        axes = [axes]
    D = len(src_map)
    out = (ctypes.c_int32 * D)()
    _check(lib.dfft_permute_map_by_axes(D, _i32(src_map), len(axes), _i32(axes), _layout_right(layout), out))
    return tuple(int(x) for x in out)


def propose_transpose_block(map, in_topology, out_topology, in_extents, global_extents, axes, rank,
                            is_layout_right, is_last, in_axis, out_axis, comm_axis, block_idx, size_factor,
                            layout="right"):
    """Returns (block info dict, max buffer size)."""
    D = len(map)
    info = BlockInfo()
    mb = ctypes.c_uint64()
    _check(lib.dfft_propose_transpose_block(
        D, _i32(map), _u64(in_topology), _u64(out_topology), _u64(in_extents), _u64(global_extents), len(axes),
        _i32(axes), int(rank), int(bool(is_layout_right)), int(bool(is_last)), int(in_axis), int(out_axis),
        int(comm_axis), int(block_idx), int(size_factor), _layout_right(layout), ctypes.byref(info),
        ctypes.byref(mb)))
    blk = dict(block_type="FFT" if info.block_type == 1 else "Transpose", block_idx=info.block_idx,
               in_axis=info.in_axis, out_axis=info.out_axis, comm_axis=info.comm_axis,
               in_topology=tuple(info.in_topology[:D]), out_topology=tuple(info.out_topology[:D]),
               in_extents=tuple(info.in_extents[:D]), out_extents=tuple(info.out_extents[:D]),
               buffer_extents=tuple(info.buffer_extents[:D + 1]), in_map=tuple(info.in_map[:D]),
               out_map=tuple(info.out_map[:D]))
    return blk, int(mb.value)
