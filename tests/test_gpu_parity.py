"""GPU parity of the CUDA execute path against the CPU oracle.

Tolerances: FP64 rel-L2 <= 1e-12 against the FP64 oracle (numpy pocketfft on
the same inputs); FP32 rel-L2 <= 1e-6 against the FP64 oracle applied to the
FP32-rounded inputs.  Pack / all-to-all / unpack buffers are compared bit for
bit with the oracle's restatement of the reference kernels applied to the same
(captured) data."""
import itertools

import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _gpu_util import out_extents, random_input, run
from _plan_info import plan_info

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 1e-6}


def check_roundtrip(gin, axes, tin, tout, real, precision="float64", exec_mode="fused", norm="backward",
                    layout="right", seed=0, tol=None):
    gout = out_extents(gin, axes, real)
    plan = dfft.Plan(gin, gout, axes, tin, tout, real_input=real, precision=precision, norm=norm, layout=layout,
                     exec_mode=exec_mode)
    x = random_input(gin, real, seed, precision)
    X = run(plan, x, True)
    ref = O.global_fft(x, axes, real, norm=norm)
    tol = tol or TOL[precision]
    e_fwd = O.rel_l2(X, ref)
    assert e_fwd <= tol, (plan.name(), gin, axes, tin, tout, e_fwd)
    xb = run(plan, ref, False)
    ref_b = O.global_ifft(ref, axes, real, gin, norm=norm)
    e_bwd = O.rel_l2(xb, ref_b)
    assert e_bwd <= tol, (plan.name(), gin, axes, tin, tout, e_bwd)
    return plan, e_fwd, e_bwd


def test_cfg1_slab_r2c_64cubed_fp64():
    # 64^3 real U[-1,1) seed 0, slab (2,1,1) -> (1,2,1), R2C forward + C2R backward
    plan, ef, eb = check_roundtrip((64, 64, 64), (0, 1, 2), (2, 1, 1), (1, 2, 1), True, seed=0)
    assert plan.name() == "SlabPlan"
    # normalised roundtrip is the identity
    x = random_input((64, 64, 64), True, 0)
    y = run(plan, run(plan, x, True), False)
    assert O.rel_l2(y, x) <= 1e-12


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
@pytest.mark.parametrize("axes", list(itertools.permutations(range(3))))
def test_slab_odd_shape_all_axes(axes, exec_mode):
    # Test_SlabPlan.cpp uses (8,7,6) to exercise uneven bins and zero padding
    for tin, tout in [((1, 1, 2), (1, 2, 1)), ((2, 1, 1), (1, 1, 2)), ((1, 2, 1), (2, 1, 1)),
                      ((1, 1, 3), (3, 1, 1)), ((2, 1, 1), (2, 1, 1))]:
        for real in (True, False):
            check_roundtrip((8, 7, 6), axes, tin, tout, real, exec_mode=exec_mode)


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
@pytest.mark.parametrize("axes", list(itertools.permutations(range(3))))
def test_pencil_odd_shape_all_axes(axes, exec_mode):
    # Test_PencilPlan.cpp uses (8,7,5)
    for tin, tout in [((1, 2, 2), (2, 2, 1)), ((2, 2, 1), (1, 2, 2)), ((1, 2, 3), (2, 3, 1)),
                      ((2, 1, 2), (2, 2, 1)), ((2, 3, 1), (2, 3, 1))]:
        for real in (True, False):
            check_roundtrip((8, 7, 5), axes, tin, tout, real, exec_mode=exec_mode)


@pytest.mark.parametrize("norm", ["backward", "forward", "ortho", "none"])
def test_normalizations(norm):
    check_roundtrip((16, 12, 10), (0, 1, 2), (2, 1, 1), (1, 2, 1), True, norm=norm)
    check_roundtrip((16, 12, 10), (0, 1, 2), (2, 2, 1), (1, 2, 2), False, norm=norm, exec_mode="literal")


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
def test_batched_4d_views(exec_mode):
    # navier-stokes-MPI-batched: (3, nx, ny, nz) with FFT axes {1, 2, 3}
    check_roundtrip((3, 16, 12, 10), (1, 2, 3), (1, 2, 1, 1), (1, 1, 2, 1), True, exec_mode=exec_mode)
    check_roundtrip((3, 16, 12, 10), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2), False, exec_mode=exec_mode)


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
def test_layout_left(exec_mode):
    check_roundtrip((8, 7, 6), (0, 1, 2), (1, 1, 2), (2, 1, 1), True, layout="left", exec_mode=exec_mode)
    check_roundtrip((8, 7, 5), (2, 1, 0), (1, 2, 2), (2, 2, 1), False, layout="left", exec_mode=exec_mode)


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
def test_lower_rank_fft_plans(exec_mode):
    # 1D and 2D FFT plans on 3D views, 2D FFT on 2D views (SlabInternalPlan<1/2>)
    check_roundtrip((8, 7, 6), (2,), (2, 1, 1), (1, 2, 1), True, exec_mode=exec_mode)
    check_roundtrip((8, 7, 6), (1, 2), (1, 1, 2), (2, 1, 1), False, exec_mode=exec_mode)
    check_roundtrip((12, 10), (0, 1), (2, 1), (1, 2), True, exec_mode=exec_mode)
    check_roundtrip((8, 7, 5), (0, 2), (1, 2, 2), (2, 2, 1), True, exec_mode=exec_mode)


def test_fused_equals_literal_c2c():
    # The fused path and the reference block sequence agree to FP64 rounding.
    # They are not bit-identical: a stage may run on the register-resident
    # kernel in one path and on the generic Stockham kernel in the other (the
    # choice depends on the layouts), and those derive their twiddles
    # differently.  The exchanges themselves are checked bit for bit below.
    gin = (32, 24, 20)
    x = random_input(gin, False, 5)
    pf = dfft.Plan(gin, gin, (0, 1, 2), (4, 2, 1), (1, 4, 2), exec_mode="fused")
    pl = dfft.Plan(gin, gin, (0, 1, 2), (4, 2, 1), (1, 4, 2), exec_mode="literal")
    a, b = run(pf, x, True), run(pl, x, True)
    assert O.rel_l2(a, b) <= 1e-14


def _bitwise_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def check_exchanges_bit_exact(plan, x, forward=True):
    """Every transpose block: GPU send == oracle pack(GPU pack input),
    GPU recv == oracle all2all(GPU send), GPU unpack output == oracle unpack(GPU recv)."""
    run(plan, x, forward)
    info = plan_info(plan)
    right = plan.layout == "right"
    P = plan.nprocs
    direction = dfft.Direction.forward if forward else dfft.Direction.backward
    blocks = [plan.block_infos(r) for r in range(P)]
    n_checked = 0
    for i, b in enumerate(blocks[0]):
        if b["block_type"] != "Transpose":
            continue
        pin = plan.export_buffers(direction, i, "pack_in")
        send = plan.export_buffers(direction, i, "send")
        recv = plan.export_buffers(direction, i, "recv")
        uout = plan.export_buffers(direction, i, "unpack_out")
        src_map, src_axis, dst_map, dst_axis = (b["in_map"], b["in_axis"], b["out_map"], b["out_axis"]) if forward \
            else (b["out_map"], b["out_axis"], b["in_map"], b["in_axis"])
        for r in range(P):
            ref = O.pack(pin[r], src_map, src_axis, b["buffer_extents"], right)
            assert _bitwise_equal(send[r], ref), ("pack", i, r)
        groups = O.exchange_groups(plan.in_topology, P, b["comm_axis"], info["pencil"])
        ref_recv = O.all2all(list(send), groups, right)
        for r in range(P):
            assert _bitwise_equal(recv[r], ref_recv[r]), ("all2all", i, r)
            shape = uout[r].shape
            ref_u = O.unpack(recv[r], dst_map, dst_axis, shape, dtype=recv.dtype, layout_right=right)
            assert _bitwise_equal(uout[r], ref_u), ("unpack", i, r)
        n_checked += 1
    return n_checked


def test_cfg1_pack_buffers_bit_exact():
    # per-rank pack buffers (2,32,32,33) complex128 of the 64^3 R2C slab plan
    gin = (64, 64, 64)
    plan = dfft.Plan(gin, out_extents(gin, (0, 1, 2), True), (0, 1, 2), (2, 1, 1), (1, 2, 1), real_input=True,
                     exec_mode="literal_capture")
    x = random_input(gin, True, 0)
    assert check_exchanges_bit_exact(plan, x, True) == 1
    send = plan.export_buffers(dfft.Direction.forward, 1, "send")
    assert send.shape == (2, 2, 32, 32, 33) and send.dtype == np.complex128
    X = O.global_fft(x, (0, 1, 2), True)
    assert check_exchanges_bit_exact(plan, X, False) == 1


@pytest.mark.parametrize("gin,tin,tout,real,layout", [
    ((8, 7, 6), (1, 1, 2), (1, 2, 1), True, "right"),
    ((8, 7, 5), (1, 2, 3), (2, 3, 1), False, "right"),
    ((8, 7, 5), (2, 2, 1), (1, 2, 2), True, "right"),
    ((8, 7, 6), (1, 1, 2), (2, 1, 1), True, "left"),
    ((8, 7, 5), (1, 2, 2), (2, 2, 1), False, "left"),
    ((3, 8, 7, 5), (1, 2, 2, 1), (1, 1, 2, 2), True, "right"),
])
def test_exchange_buffers_bit_exact_ragged(gin, tin, tout, real, layout):
    axes = tuple(range(len(gin) - 3, len(gin)))
    plan = dfft.Plan(gin, out_extents(gin, axes, real), axes, tin, tout, real_input=real, layout=layout,
                     exec_mode="literal_capture")
    x = random_input(gin, real, 3)
    assert check_exchanges_bit_exact(plan, x, True) >= 1
    X = O.global_fft(x, axes, real)
    assert check_exchanges_bit_exact(plan, X, False) >= 1


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_cfg2_pencil_c2c_256cubed(precision):
    # 256^3 complex N(0,1) seed 1, pencil (4,4,1) -> (1,4,4)
    gin = (256, 256, 256)
    plan = dfft.Plan(gin, gin, (0, 1, 2), (4, 4, 1), (1, 4, 4), precision=precision)
    assert plan.name() == "PencilPlan"
    x = random_input(gin, False, 1, precision)
    X = run(plan, x, True)
    ref = O.global_fft(x, (0, 1, 2), False)
    assert O.rel_l2(X, ref) <= TOL[precision]
    xb = run(plan, X, False)
    assert O.rel_l2(xb, x) <= TOL[precision] * 2


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_headline_512cubed_pencil_c2c(precision):
    """The bench workload itself: 512^3 C2C, pencil (4,4,1) -> (1,4,4), N(0,1)
    complex from seed 1 (FP32 runs use the FP64 draws rounded).  Forward and
    backward against the FP64 oracle on the same (rounded) inputs: rel-L2 <=
    1e-12 in FP64, <= 1e-6 in FP32."""
    gin = (512, 512, 512)
    plan = dfft.Plan(gin, gin, (0, 1, 2), (4, 4, 1), (1, 4, 4), precision=precision)
    x = random_input(gin, False, 1, precision)
    X = run(plan, x, True)
    ref = O.global_fft(x, (0, 1, 2), False, workers=-1)
    e_fwd = O.rel_l2(X, ref)
    del X
    assert e_fwd <= TOL[precision], e_fwd
    xb = run(plan, ref, False)  # backward of the exact spectrum
    ref_b = x.astype(np.complex128)
    e_bwd = O.rel_l2(xb, ref_b)
    assert e_bwd <= TOL[precision], e_bwd


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_r2c_256cubed_pencil(precision):
    """256^3 real U[-1,1) seed 1, R2C forward and C2R backward on the pencil
    (4,4,1) -> (1,4,4), against the FP64 oracle."""
    gin = (256, 256, 256)
    plan, ef, eb = check_roundtrip(gin, (0, 1, 2), (4, 4, 1), (1, 4, 4), True, precision=precision, seed=1)
    assert plan.name() == "PencilPlan"


def test_cfg2_transposes_bit_exact_256cubed():
    gin = (256, 256, 256)
    plan = dfft.Plan(gin, gin, (0, 1, 2), (4, 4, 1), (1, 4, 4), exec_mode="literal_capture")
    x = random_input(gin, False, 1)
    assert check_exchanges_bit_exact(plan, x, True) == 2


def test_input_not_modified_and_errors():
    import torch
    gin = (16, 12, 10)
    plan = dfft.Plan(gin, out_extents(gin, (0, 1, 2), True), (0, 1, 2), (2, 1, 1), (1, 2, 1), real_input=True)
    x = random_input(gin, True, 9)
    t_in = torch.from_numpy(dfft.scatter_blocks(plan, x, "in")).cuda()
    keep = t_in.clone()
    t_out = torch.empty(plan.buffer_elements("out"), dtype=torch.complex128, device="cuda")
    dfft.execute(plan, t_in, t_out, dfft.Direction.forward)
    torch.cuda.synchronize()
    assert torch.equal(t_in, keep)
    with pytest.raises(dfft.DistributedFFTError):
        dfft.execute(plan, t_in, t_in, dfft.Direction.forward)
    with pytest.raises(ValueError):
        dfft.execute(plan, t_in, t_out, 7)


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 24, 48, 96, 192, 384, 768])
def test_register_kernel_line_lengths(n, precision):
    # lines along the unit-stride axis (a-fast rows) and across it (b-fast rows),
    # on a slab exchange so the rows also cross virtual-rank blocks
    for gin, axes, tin, tout in [((4, 6, n), (2,), (2, 1, 1), (1, 2, 1)), ((n, 3, 32), (0,), (1, 1, 2), (1, 1, 2)),
                                 ((n, 3, 32), (0,), (1, 2, 1), (1, 1, 2))]:
        check_roundtrip(gin, axes, tin, tout, False, precision=precision)
    # R2C / C2R on contiguous lines (two real lines per register line); 15
    # lines per block leave the last line of a pair empty
    for gin, axes, tin, tout in [((4, 6, n), (2,), (2, 1, 1), (1, 2, 1)), ((3, 5, n), (2,), (1, 1, 1), (1, 1, 1)),
                                 ((6, 4, n), (1, 2), (2, 1, 1), (1, 2, 1))]:
        check_roundtrip(gin, axes, tin, tout, True, precision=precision)


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("gin,axes,tin,tout,real", [
    ((96, 64, 48), (0, 1, 2), (3, 2, 1), (1, 3, 2), True),     # out z = 25 over 2 ranks: 13 / 12
    ((64, 96, 48), (0, 1, 2), (2, 2, 1), (1, 2, 2), True),
    ((48, 40, 64), (0, 1, 2), (3, 1, 1), (1, 3, 1), False),    # y = 40 over 3 ranks: 14 / 13 / 13
    ((3, 32, 24, 64), (1, 2, 3), (1, 3, 2, 1), (1, 1, 3, 2), True),
])
def test_register_kernels_on_ragged_blocks(gin, axes, tin, tout, real, precision):
    # rank blocks of unequal size make the layout tables general (per-rank
    # strides); the register kernels then address each line as base + p * stride
    check_roundtrip(gin, axes, tin, tout, real, precision=precision)


def test_fp32_pair_kernel_misaligned_buffers_fall_back():
    """Two-lines-per-thread stages move line pairs with 16-byte accesses; a
    caller buffer that is only complex64-aligned (8 bytes) runs the one-line
    kernel instead, with bit-identical results."""
    import torch
    gin = (64, 64, 64)
    plan = dfft.Plan(gin, gin, (0, 1, 2), (2, 2, 1), (1, 2, 2), precision="float32")
    x = random_input(gin, False, 4, "float32")
    flat = dfft.scatter_blocks(plan, x, "in")
    n = flat.size
    t_in = torch.from_numpy(np.ascontiguousarray(flat)).cuda()
    store = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
    aligned = store[:n]
    shifted = store[1:]  # 8 bytes past a 16-byte boundary
    ref = torch.empty(n, dtype=torch.complex64, device="cuda")
    dfft.execute(plan, t_in, ref, dfft.Direction.forward)
    dfft.execute(plan, t_in, shifted, dfft.Direction.forward)
    torch.cuda.synchronize()
    assert torch.equal(shifted.view(torch.float32), ref.view(torch.float32))
    X = dfft.gather_blocks(plan, ref.cpu().numpy(), "out")
    assert O.rel_l2(X, O.global_fft(x, (0, 1, 2), False)) <= TOL["float32"]
    back_store = torch.zeros(n + 1, dtype=torch.complex64, device="cuda")
    dfft.execute(plan, shifted.clone(), back_store[1:], dfft.Direction.backward)
    dfft.execute(plan, ref, aligned, dfft.Direction.backward)
    torch.cuda.synchronize()
    assert torch.equal(back_store[1:].view(torch.float32), aligned.view(torch.float32))
