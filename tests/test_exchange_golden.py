"""The oracle's exchange restatement and the library's host layout math
against the reference's own unit-test known answers (no GPU).

Golden vectors: tests/golden/make_exchange_fixtures.py restates the
expected-buffer constructions of Test_Pack.cpp, Test_Unpack.cpp,
Test_All2All.cpp and Test_TransBlock.cpp, and extracts the explicit tables of
Test_Mapping.cpp and Test_MPI_Extents.cpp (paths relative to the reference's
distributed/unit_test/)."""
import numpy as np
import pytest

import dfft_oracle as O
from _golden import Fixtures, distribute_extents
from dfft import exchange as X

FX = Fixtures()


def _equal(a, b):
    return np.asarray(a).shape == np.asarray(b).shape and np.array_equal(a, b)


def test_fixture_inventory():
    kinds = {}
    for c in FX.cases:
        kinds[c["kind"]] = kinds.get(c["kind"], 0) + 1
    # 2 layouts x (nprocs 1..4: 10 rank cases) x (2 x 2 orders/buffers in 2D + 6 x 6 in 3D)
    assert kinds == {"pack_unpack": 800, "all2all": 16, "trans_block": 132}


def test_oracle_pack_unpack_match_reference_tests():
    for c in FX.of_kind("pack_unpack"):
        right = c["layout"] == "right"
        view = FX.array(c["view"], c["view_extents"], c["layout"])
        buf = FX.array(c["buffer"], c["buffer_extents"], c["layout"])
        got = O.pack(view, c["map"], c["axis"], c["buffer_extents"], right)
        assert _equal(got, buf), (c["pack_source"], c["layout"], c["nprocs"], c["rank"], c["map"], c["tag"])
        back = O.unpack(buf, c["map"], c["axis"], c["view_extents"], layout_right=right)
        assert _equal(back, view), (c["unpack_source"], c["layout"], c["nprocs"], c["rank"], c["map"], c["tag"])


def _groups(c):
    if c["comm_axis"] < 0:
        return O.exchange_groups(None, c["nprocs"], -1, False)
    return O.exchange_groups(c["cart_topology"], c["nprocs"], c["comm_axis"], True)


def test_oracle_all2all_matches_reference_tests():
    for c in FX.of_kind("all2all"):
        sends = FX.per_rank(c["send"], c["nprocs"], c["buffer_extents"], c["layout"])
        refs = FX.per_rank(c["expected"], c["nprocs"], c["buffer_extents"], c["layout"])
        got = O.all2all(sends, _groups(c), c["layout"] == "right")
        for r in range(c["nprocs"]):
            assert _equal(got[r], refs[r]), (c["source"], c["layout"], c["nprocs"], r)


def _blocks_shapes(gext, topo, topo_layout, vmap):
    shapes = []
    for r in range(int(np.prod(topo))):
        ext = X.compute_local_extents_and_starts(gext, topo, r, topo_layout)[0]
        shapes.append(tuple(ext[m] for m in vmap))
    return shapes


def split_blocks(flat, shapes, layout):
    out, at = [], 0
    for s in shapes:
        n = int(np.prod(s))
        out.append(flat[at:at + n].reshape(s, order="C" if layout == "right" else "F"))
        at += n
    return out


def test_oracle_trans_block_matches_reference_tests():
    """pack -> all2all -> unpack of the oracle, rank by rank, reproduces the
    TransBlock tests' expected blocks (the global array's block in the
    destination topology, permuted by the destination map)."""
    for c in FX.of_kind("trans_block"):
        right = c["layout"] == "right"
        P = int(np.prod(c["in_topology"]))
        ins = split_blocks(FX.flat(c["input"]), _blocks_shapes(c["global_extents"], c["in_topology"],
                                                               c["in_topology_layout"], c["src_map"]), c["layout"])
        oshape = _blocks_shapes(c["global_extents"], c["out_topology"], c["out_topology_layout"], c["dst_map"])
        exp = split_blocks(FX.flat(c["expected"]), oshape, c["layout"])
        sends = [O.pack(ins[r], c["src_map"], c["src_axis"], c["buffer_extents"], right) for r in range(P)]
        cart = c["cart_topology"]
        groups = O.exchange_groups(cart, P, c["comm_axis"], cart is not None)
        recvs = O.all2all(sends, groups, right)
        for r in range(P):
            out = O.unpack(recvs[r], c["dst_map"], c["dst_axis"], oshape[r], layout_right=right)
            assert _equal(out, exp[r]), (c["source"], c["layout"], c["in_topology"], c["dst_map"], r)


# ---- host layout math through the C ABI ----------------------------------
def test_permute_map_by_axes_tables():
    t = FX.tables["permute_map_by_axes"]
    assert len(t["rows"]) == 44
    for row in t["rows"]:
        got = X.permute_map_by_axes(row["src_map"], row["axis"], row["layout"])
        assert list(got) == row["expected"], (t["source"], row)


def test_rank_to_coord_tables():
    t = FX.tables["rank_to_coord"]
    assert len(t["rows"]) == 68
    for row in t["rows"]:
        got = X.rank_to_coord(row["topology"], row["rank"], row["layout"])
        assert list(got) == row["expected"], (t["source"], row)


@pytest.mark.parametrize("layout", ["right", "left"])
def test_buffer_extents_known_answers(layout):
    # Test_Extents.cpp:20-60: (13, 8, 17, 5), X / Y / Z pencils over p0 = 2, p1 = 3
    n0, n1, n2, n3, p0, p1 = 13, 8, 17, 5, 2, 3
    ext = (n0, n1, n2, n3)
    t0, t1, t2 = (1, p0, p1, 1), (p0, 1, p1, 1), (p0, p1, 1, 1)
    if layout == "left":
        ref01 = ((n0 - 1) // p0 + 1, (n1 - 1) // p0 + 1, (n2 - 1) // p1 + 1, n3, p0)
        ref12 = ((n0 - 1) // p0 + 1, (n1 - 1) // p1 + 1, (n2 - 1) // p1 + 1, n3, p1)
    else:
        ref01 = (p0, (n0 - 1) // p0 + 1, (n1 - 1) // p0 + 1, (n2 - 1) // p1 + 1, n3)
        ref12 = (p1, (n0 - 1) // p0 + 1, (n1 - 1) // p1 + 1, (n2 - 1) // p1 + 1, n3)
    assert X.compute_buffer_extents(ext, t0, t1, layout) == ref01
    assert X.compute_buffer_extents(ext, t1, t2, layout) == ref12


@pytest.mark.parametrize("n,nprocs,starts,lengths", [
    (10, 3, [0, 4, 7], [4, 3, 3]), (12, 3, [0, 4, 8], [4, 4, 4]),
    (128, 6, [0, 22, 44, 65, 86, 107], [22, 22, 21, 21, 21, 21])])
def test_bin_mapping_known_answers(n, nprocs, starts, lengths):
    # Test_Pack.cpp:583-592 (bin_mapping), through the local extents / starts
    # of a (n, 1) view split over (nprocs, 1), and the oracle's bin_mapping
    got = [X.compute_local_extents_and_starts((n, 1), (nprocs, 1), r) for r in range(nprocs)]
    assert [g[1][0] for g in got] == starts and [g[0][0] for g in got] == lengths
    assert [O.bin_mapping(n, nprocs, r) for r in range(nprocs)] == list(zip(starts, lengths))


@pytest.mark.parametrize("nprocs", [1, 2, 3, 4, 5, 6])
def test_local_starts_and_extents_equal_pattern(nprocs):
    # Test_MPI_Extents.cpp:338-395 / :494-...: (19, 32) on {1, P} and {P, 1};
    # starts accumulate the extents of the lower ranks
    gn0, gn1 = 19, 32
    acc0 = acc1 = 0
    for r in range(nprocs):
        e0, s0 = X.compute_local_extents_and_starts((gn0, gn1), (1, nprocs), r)
        e1, s1 = X.compute_local_extents_and_starts((gn0, gn1), (nprocs, 1), r)
        assert e0 == (gn0, distribute_extents(gn1, r, nprocs)[1]) and s0 == (0, acc0)
        assert e1 == (distribute_extents(gn0, r, nprocs)[1], gn1) and s1 == (acc1, 0)
        acc0 += e0[1]
        acc1 += e1[0]


@pytest.mark.parametrize("layout", ["right", "left"])
@pytest.mark.parametrize("axes", [[2], []])
@pytest.mark.parametrize("is_last", [True, False])
def test_propose_transpose_block(layout, axes, is_last):
    """Test_BlockAnalyses.cpp:93-176: map {2, 0, 1}, in (16, 16, 16) of
    global (64, 64, 16), {4, 4, 1} -> {4, 1, 4}, in_axis 1, out_axis 2,
    comm_axis 1, block 3, size factor 2, for every rank of the topology."""
    right = layout == "right"
    for rank in range(16):
        blk, mb = X.propose_transpose_block((2, 0, 1), (4, 4, 1), (4, 1, 4), (16, 16, 16), (64, 64, 16), axes, rank,
                                            right, is_last, 1, 2, 1, 3, 2, layout)
        assert blk["block_type"] == "Transpose" and blk["in_map"] == (2, 0, 1)
        assert (blk["in_axis"], blk["out_axis"], blk["comm_axis"], blk["block_idx"]) == (1, 2, 1, 3)
        assert blk["in_topology"] == (4, 4, 1) and blk["out_topology"] == (4, 1, 4)
        assert blk["in_extents"] == (16, 16, 16)
        if is_last:
            ref_map = (0, 1, 2)
        else:
            ref_map = X.permute_map_by_axes((2, 0, 1), axes if axes else [2], layout)
        assert blk["out_map"] == ref_map
        ext, _ = X.compute_local_extents_and_starts((64, 64, 16), (4, 1, 4), rank, layout)
        assert blk["out_extents"] == tuple(ext[m] for m in ref_map)
        ref_buf = X.compute_buffer_extents((64, 64, 16), (4, 4, 1), (4, 1, 4), layout)
        assert blk["buffer_extents"] == ref_buf
        sizes = [int(np.prod(blk["in_extents"])), int(np.prod(ref_buf)), int(np.prod(blk["out_extents"]))]
        assert mb == max(sizes) * 2
