"""The host planner against the reference's own known-answer tables.

tests/golden/topology_tables.json holds every row of the
get_all_slab_topologies / get_all_pencil_topologies tests of the reference
(distributed/unit_test/Test_Topologies.cpp, extracted by
tests/golden/extract_topology_tables.py); they are replayed for
nprocs = 1..6 like the reference's parameterised suites."""
import itertools
import json
import os

import pytest

import dfft

TABLES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "topology_tables.json")))["tables"]


def _topos(t, nprocs):
    env = dict(nprocs=nprocs, np0=t["np0"] or 0)
    return {k: (tuple(int(eval(v, {}, env)) for v in d["values"]), d["layout"]) for k, d in t["topologies"].items()}


@pytest.mark.parametrize("table", TABLES, ids=[t["function"] for t in TABLES])
@pytest.mark.parametrize("nprocs", [2, 3, 4, 5, 6])
def test_topology_chain_tables(table, nprocs):
    topos = _topos(table, nprocs)
    assert table["rows"]
    for r in table["rows"]:
        ti, lt = topos[r["inp"]]
        to, lo = topos[r["out"]]
        axes = [int(a) for a in table["axes"][r["axes"]]]
        expected = [topos[c][0] for c in r["chain"]]
        got = dfft.all_topologies(table["kind"], ti, to, axes, lt, lo)
        if table["kind"] == "pencil":
            assert got == (expected, r["trans_axes"], r["layouts"]), (r, got)
        else:
            assert got == expected, (r, got)


@pytest.mark.parametrize("table", TABLES, ids=[t["function"] for t in TABLES])
def test_topology_chain_throws_for_one_proc(table):
    # nprocs == 1: shared topologies are rejected (EXPECT_THROW in the reference)
    topos = _topos(table, 1)
    for (ti, lt), (to, lo) in itertools.product(topos.values(), repeat=2):
        for ax in table["axes"].values():
            with pytest.raises(dfft.DistributedFFTError) as e:
                dfft.all_topologies(table["kind"], ti, to, [int(a) for a in ax], lt, lo)
            assert e.value.status == dfft.Status.INVALID_TOPOLOGY


def test_worked_examples_block_lists():
    # 64^3 R2C slab (2,1,1) -> (1,2,1): FFT2(R2C) -> T -> FFT1, buffer (2,32,32,33)
    p = dfft.Plan((64, 64, 64), (64, 64, 33), (0, 1, 2), (2, 1, 1), (1, 2, 1), real_input=True, analyze_only=True)
    assert p.name() == "SlabPlan"
    b = p.block_infos(0)
    assert [x["block_type"] for x in b] == ["FFT", "Transpose", "FFT"]
    assert b[0]["fft_dim"] == 2 and b[2]["fft_dim"] == 1
    assert b[1]["buffer_extents"] == (2, 32, 32, 33)
    assert b[1]["out_map"] == (1, 2, 0) and b[1]["out_extents"] == (32, 33, 64)
    assert p.local_extents(1, "out") == ((64, 32, 33), (0, 32, 0))
    # 256^3 C2C pencil (4,4,1) -> (1,4,4): chain, trans axes, layouts
    q = dfft.Plan((256,) * 3, (256,) * 3, (0, 1, 2), (4, 4, 1), (1, 4, 4), analyze_only=True)
    assert q.name() == "PencilPlan"
    assert q.topology_chain() == ([(4, 4, 1), (4, 1, 4), (1, 4, 4)], [1, 0], [1, 1, 1])
    assert [x["buffer_extents"] for x in q.block_infos(0) if x["block_type"] == "Transpose"] == [(4, 64, 64, 64)] * 2


def test_factory_errors():
    # internal_plan_factory / are_valid_extents error paths
    with pytest.raises(dfft.DistributedFFTError) as e:
        dfft.Plan((8, 8, 8), (8, 8, 8), (0, 1, 2), (2, 1, 1), (1, 1, 4), analyze_only=True)
    assert e.value.status == dfft.Status.INVALID_TOPOLOGY
    with pytest.raises(dfft.DistributedFFTError) as e:
        dfft.Plan((8, 8, 8), (8, 8, 8), (0, 1, 2), (2, 2, 2), (2, 2, 2), analyze_only=True)
    assert "Brick" in str(e.value)
    with pytest.raises(dfft.DistributedFFTError) as e:
        dfft.Plan((8, 8, 8), (8, 8, 4), (0, 1, 2), (2, 1, 1), (1, 2, 1), real_input=True, analyze_only=True)
    assert e.value.status == dfft.Status.INVALID_EXTENTS
    with pytest.raises(dfft.DistributedFFTError):
        dfft.Plan((8, 8, 8), (8, 8, 7), (0, 1, 2), (2, 1, 1), (1, 2, 1), analyze_only=True)
    with pytest.raises(dfft.DistributedFFTError):
        dfft.Plan((8, 8), (8, 8), (0, 1), (2, 2), (2, 2), analyze_only=True)  # pencil needs rank >= 3
    with pytest.raises(dfft.DistributedFFTError):
        dfft.Plan((8, 8, 8), (8, 8, 8), (0, 0, 2), (2, 1, 1), (1, 2, 1), analyze_only=True)
    p = dfft.Plan((8, 8, 8), (8, 8, 8), (0, 1, 2), (1, 1, 1), (1, 1, 1), analyze_only=True)
    assert p.name() == "SharedPlan"
