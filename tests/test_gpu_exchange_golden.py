"""The GPU data-movement kernels against the reference's own unit-test
vectors, bit for bit.

dfft_pack / dfft_unpack / dfft_all2all / dfft_trans_block_* run the same
kernels (csrc/transpose.cu) as the plans' literal programs.  Every case of
tests/golden/exchange_fixtures.* (restated from Test_Pack.cpp, Test_Unpack.cpp,
Test_All2All.cpp and Test_TransBlock.cpp of the reference's
distributed/unit_test/) runs through the C ABI with 4-, 8- and 16-byte
elements (float32, float64, complex128 holding (v, -v)) and must reproduce
the expected buffers exactly, zero padding included."""
import numpy as np
import pytest

import dfft
from _golden import Fixtures
from dfft import exchange as X

pytestmark = pytest.mark.gpu

FX = Fixtures()
ELEMS = {"float32": np.float32, "float64": np.float64, "complex128": np.complex128}


def dev(a, kind):
    import torch
    a = np.asarray(a)
    if kind == "complex128":
        a = a.astype(np.float64) - 1j * a.astype(np.float64)
    return torch.from_numpy(np.ascontiguousarray(a.astype(ELEMS[kind]))).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def same(got, exp, kind):
    e = np.asarray(exp)
    if kind == "complex128":
        e = e.astype(np.float64) - 1j * e.astype(np.float64)
    e = e.astype(ELEMS[kind])
    return got.shape == e.shape and np.array_equal(got.view(np.uint8), e.view(np.uint8))


@pytest.mark.parametrize("kind", list(ELEMS))
def test_pack_and_unpack_reference_vectors(kind):
    import torch
    n = 0
    for c in FX.of_kind("pack_unpack"):
        view = dev(FX.flat(c["view"]), kind)
        buf_exp = FX.flat(c["buffer"])
        buf = torch.full_like(dev(buf_exp, kind), 77)  # padding must come out as zeros
        X.pack(view, buf, c["map"], c["axis"], c["view_extents"], c["buffer_extents"], c["layout"])
        assert same(host(buf), buf_exp, kind), ("pack", c["pack_source"], c["layout"], c["nprocs"], c["rank"],
                                                c["map"], c["tag"])
        out = torch.zeros_like(view)
        X.unpack(dev(buf_exp, kind), out, c["map"], c["axis"], c["buffer_extents"], c["view_extents"], c["layout"])
        assert same(host(out), FX.flat(c["view"]), kind), ("unpack", c["unpack_source"], c["layout"], c["nprocs"],
                                                            c["rank"], c["map"], c["tag"])
        n += 1
    assert n == 800


@pytest.mark.parametrize("kind", list(ELEMS))
def test_all2all_reference_vectors(kind):
    import torch
    for c in FX.of_kind("all2all"):
        send = dev(FX.flat(c["send"]), kind)
        recv = torch.zeros_like(send)
        X.all2all(send, recv, c["nprocs"], c["buffer_extents"], c["comm_axis"], c["cart_topology"], c["layout"])
        assert same(host(recv), FX.flat(c["expected"]), kind), (c["source"], c["layout"], c["nprocs"])


@pytest.mark.parametrize("kind", list(ELEMS))
def test_trans_block_reference_vectors(kind):
    import torch
    esize = {"float32": 4, "float64": 8, "complex128": 16}[kind]
    for c in FX.of_kind("trans_block"):
        tb = X.TransBlock(c["global_extents"], c["in_topology"], c["out_topology"], c["src_map"], c["src_axis"],
                          c["dst_map"], c["dst_axis"], esize, layout=c["layout"],
                          in_topology_layout=c["in_topology_layout"], out_topology_layout=c["out_topology_layout"],
                          comm_axis=c["comm_axis"], cart_topology=c["cart_topology"])
        assert list(tb.buffer_extents()) == c["buffer_extents"]
        P = int(np.prod(c["in_topology"]))
        nbuf = P * int(np.prod(c["buffer_extents"]))
        inp = dev(FX.flat(c["input"]), kind)
        out = dev(np.zeros(FX.flat(c["expected"]).size), kind)
        send = dev(np.zeros(nbuf), kind)
        recv = dev(np.zeros(nbuf), kind)
        tb(inp, out, send, recv, dfft.Direction.forward)
        assert same(host(out), FX.flat(c["expected"]), kind), (c["source"], c["layout"], c["in_topology"],
                                                               c["dst_map"])
        back = torch.zeros_like(inp)
        tb(out, back, send, recv, dfft.Direction.backward)
        assert same(host(back), FX.flat(c["input"]), kind), ("backward", c["source"], c["layout"], c["dst_map"])


def test_exchange_errors_before_launch():
    import torch
    x = torch.zeros(64, dtype=torch.float64, device="cuda")
    y = torch.zeros(64, dtype=torch.float64, device="cuda")
    # buffer process extent 3 on a world of 2 ranks: the reference's all2all throws
    with pytest.raises(dfft.DistributedFFTError, match="does not match MPI size"):
        X.all2all(x, y, 2, (3, 2, 2), -1)
    # aliasing input and send buffer (TransBlock::good)
    tb = X.TransBlock((4, 4), (1, 2), (2, 1), (0, 1), 0, (0, 1), 1, 8)
    with pytest.raises(dfft.DistributedFFTError, match="aliasing"):
        tb(x, y, x, torch.zeros_like(x))
