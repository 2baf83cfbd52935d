"""ctypes binding of include/dfft.h (the C ABI of libdfft.so).

The shared library is built in tree (``make -C csrc``) and loaded from this
directory; there is no fallback implementation, so a missing or unloadable
library raises at import time.
"""
import ctypes
import os

MAX_RANK = 4

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdfft.so")


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("rank", ctypes.c_int32),
        ("fft_rank", ctypes.c_int32),
        ("axes", ctypes.c_int32 * 3),
        ("in_extents", ctypes.c_uint64 * MAX_RANK),
        ("out_extents", ctypes.c_uint64 * MAX_RANK),
        ("in_topology", ctypes.c_uint64 * MAX_RANK),
        ("out_topology", ctypes.c_uint64 * MAX_RANK),
        ("in_topology_layout_right", ctypes.c_int32),
        ("out_topology_layout_right", ctypes.c_int32),
        ("view_layout_right", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("normalization", ctypes.c_int32),
        ("exec_mode", ctypes.c_int32),
        ("stream", ctypes.c_void_p),
    ]


class BlockInfo(ctypes.Structure):
    _fields_ = [
        ("block_type", ctypes.c_int32),
        ("block_idx", ctypes.c_int32),
        ("fft_dim", ctypes.c_int32),
        ("in_axis", ctypes.c_int32),
        ("out_axis", ctypes.c_int32),
        ("comm_axis", ctypes.c_int32),
        ("in_topology", ctypes.c_uint64 * MAX_RANK),
        ("out_topology", ctypes.c_uint64 * MAX_RANK),
        ("in_extents", ctypes.c_uint64 * MAX_RANK),
        ("out_extents", ctypes.c_uint64 * MAX_RANK),
        ("buffer_extents", ctypes.c_uint64 * (MAX_RANK + 1)),
        ("in_map", ctypes.c_uint64 * MAX_RANK),
        ("out_map", ctypes.c_uint64 * MAX_RANK),
    ]


class TransBlockDesc(ctypes.Structure):
    _fields_ = [
        ("rank", ctypes.c_int32),
        ("global_extents", ctypes.c_uint64 * MAX_RANK),
        ("in_topology", ctypes.c_uint64 * MAX_RANK),
        ("out_topology", ctypes.c_uint64 * MAX_RANK),
        ("in_topology_layout_right", ctypes.c_int32),
        ("out_topology_layout_right", ctypes.c_int32),
        ("src_map", ctypes.c_int32 * MAX_RANK),
        ("dst_map", ctypes.c_int32 * MAX_RANK),
        ("src_axis", ctypes.c_int32),
        ("dst_axis", ctypes.c_int32),
        ("view_layout_right", ctypes.c_int32),
        ("element_bytes", ctypes.c_int32),
        ("comm_axis", ctypes.c_int32),
        ("cart_topology", ctypes.c_uint64 * MAX_RANK),
    ]


class ExchangeInfo(ctypes.Structure):
    _fields_ = [
        ("block", ctypes.c_int64),
        ("comm_axis", ctypes.c_int32),
        ("padded", ctypes.c_int32),
        ("elements", ctypes.c_uint64),
        ("element_bytes", ctypes.c_uint64),
        ("group_size", ctypes.c_int64),
    ]


# int32_t (*)(void* user, int64_t k, const void* send, void* recv, uint64_t bytes_per_peer, void* stream)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_uint64, ctypes.c_void_p)


class NsDiag(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("enstrophy", ctypes.c_double), ("divergence_l2", ctypes.c_double)]


NS_MAX_BINS = 2048

_U64P = ctypes.POINTER(ctypes.c_uint64)
_I32P = ctypes.POINTER(ctypes.c_int32)

# name -> (restype, argtypes); the complete list of entry points of dfft.h
SIGNATURES = {
    "dfft_plan_desc_init": (None, [ctypes.POINTER(PlanDesc)]),
    "dfft_plan_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PlanDesc)]),
    "dfft_plan_analyze": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PlanDesc)]),
    "dfft_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dfft_plan_create_rank": (
        ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PlanDesc), ctypes.c_int64]),
    "dfft_plan_analyze_rank": (
        ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PlanDesc), ctypes.c_int64]),
    "dfft_get_num_exchanges": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "dfft_get_exchange_info": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ExchangeInfo)]),
    "dfft_get_exchange_group": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                       ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "dfft_execute_segment": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_execute_exchanged": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                       ctypes.c_void_p, EXCHANGE_FN, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_execute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    "dfft_execute_on_stream": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "dfft_execute_adjoint": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "dfft_plan_name": (ctypes.c_char_p, [ctypes.c_void_p]),
    "dfft_get_nprocs": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "dfft_get_local_extents": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                       ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "dfft_get_local_offset": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "dfft_get_buffer_elements": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "dfft_get_num_blocks": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "dfft_get_block_info": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(BlockInfo)]),
    "dfft_get_max_buffer_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "dfft_get_topology_chain": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_uint64),
                       ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "dfft_debug_export_buffers": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                       ctypes.c_uint64]),
    "dfft_get_device_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "dfft_get_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "dfft_get_workspace_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "dfft_get_all_topologies": (
        ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32,
                       ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32, ctypes.c_int32,
                       ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                       ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int64),
                       ctypes.POINTER(ctypes.c_int64)]),
    "dfft_execute_local_c2c_noalloc": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                       ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    "dfft_graph_create": (
        ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                       ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                       ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), ctypes.c_int64]),
    "dfft_graph_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), ctypes.c_int64]),
    "dfft_batch_execute": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32,
                       ctypes.c_void_p]),
    "dfft_batch_get_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "dfft_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dfft_ns_graph_create": (
        ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                       ctypes.c_int64, ctypes.c_int32]),
    "dfft_graph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dfft_ns_create": (
        ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                       ctypes.c_double]),
    "dfft_ns_init_taylor_green": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "dfft_ns_rhs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_energy": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "dfft_ns_velocity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_vorticity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_diagnostics": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(NsDiag), ctypes.c_void_p]),
    "dfft_ns_write_diagnostics": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                       ctypes.POINTER(NsDiag), ctypes.c_void_p]),
    "dfft_ns_rhs_adjoint": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_step_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_ns_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dfft_pack": (
        ctypes.c_int, [ctypes.c_int32, _U64P, _I32P, ctypes.c_int32, _U64P, ctypes.c_int32, ctypes.c_int32,
                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_unpack": (
        ctypes.c_int, [ctypes.c_int32, _U64P, _I32P, ctypes.c_int32, _U64P, ctypes.c_int32, ctypes.c_int32,
                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_all2all": (
        ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, _U64P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _U64P,
                       ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "dfft_trans_block_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(TransBlockDesc)]),
    "dfft_trans_block_buffer_extents": (ctypes.c_int, [ctypes.c_void_p, _U64P]),
    "dfft_trans_block_execute": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_int32, ctypes.c_void_p]),
    "dfft_trans_block_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dfft_rank_to_coord": (ctypes.c_int, [ctypes.c_int32, _U64P, ctypes.c_int32, ctypes.c_int64, _U64P]),
    "dfft_compute_local_extents_and_starts": (
        ctypes.c_int, [ctypes.c_int32, _U64P, _U64P, ctypes.c_int32, ctypes.c_int64, _U64P, _U64P]),
    "dfft_compute_buffer_extents": (ctypes.c_int, [ctypes.c_int32, _U64P, _U64P, _U64P, ctypes.c_int32, _U64P]),
    "dfft_permute_map_by_axes": (
        ctypes.c_int, [ctypes.c_int32, _I32P, ctypes.c_int32, _I32P, ctypes.c_int32, _I32P]),
    "dfft_propose_transpose_block": (
        ctypes.c_int, [ctypes.c_int32, _I32P, _U64P, _U64P, _U64P, _U64P, ctypes.c_int32, _I32P, ctypes.c_int64,
                       ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64,
                       ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(BlockInfo), _U64P]),
    "dfft_last_error_string": (ctypes.c_char_p, []),
    "dfft_version": (ctypes.c_char_p, []),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libdfft.so not found at {LIB_PATH}; build it with `make -C distributed-fft-for-kokkos_b200/csrc` "
            "(or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()
