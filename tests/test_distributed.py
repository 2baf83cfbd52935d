"""Host-side tests of the one-process-per-GPU path (dfft.DistributedPlan,
per-rank plans of the C ABI), run on CPU.

* The exchange schedule of every per-rank plan (transpose blocks in execution
  order, buffer sizes, groups) against the oracle's walk and its world / row /
  column communicators (dfft_oracle.exchange_groups, the restatement of
  KokkosFFT_Distributed_PencilPlan.hpp:32-71).
* The host engine of the multi-process tests (OracleRankEngine, one rank's
  segments) against the oracle's literal walk over all ranks.
* DistributedPlan itself over real gloo process groups of 2 and 4 processes
  (127.0.0.1), with the oracle's segments standing in for the GPU: outputs vs
  the FP64 global transform (rel-L2 <= 1e-12), and every received buffer bit
  for bit equal to the MPI_Alltoall permutation of the senders' buffers."""
import os
import socket

import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _dist_worker import case_input
from _plan_info import plan_info
from _rank_oracle import OracleRankEngine, local_box
from dfft.distributed import exchange_group, exchange_schedule


def _case(gin, axes, tin, tout, real, layout="right", norm="backward", seed=0):
    gout = list(gin)
    if real:
        gout[axes[-1]] = gin[axes[-1]] // 2 + 1
    return dict(in_extents=tuple(gin), out_extents=tuple(gout), axes=tuple(axes), in_topology=tuple(tin),
                out_topology=tuple(tout), real_input=real, layout=layout, norm=norm, seed=seed,
                precision="float64")


CASES2 = [
    _case((8, 7, 6), (0, 1, 2), (1, 1, 2), (1, 2, 1), False),
    _case((8, 7, 6), (0, 1, 2), (2, 1, 1), (1, 1, 2), True, norm="ortho"),
    _case((8, 7, 6), (2, 1, 0), (1, 2, 1), (2, 1, 1), True, layout="left"),
    _case((8, 7, 6), (1, 2), (1, 1, 2), (2, 1, 1), False),
    _case((12, 10), (0, 1), (2, 1), (1, 2), True, norm="forward"),
    _case((3, 16, 12, 10), (1, 2, 3), (1, 2, 1, 1), (1, 1, 2, 1), True),
]
CASES4 = [
    _case((8, 7, 5), (0, 1, 2), (1, 2, 2), (2, 2, 1), False),
    _case((8, 7, 5), (0, 1, 2), (2, 2, 1), (1, 2, 2), True),
    _case((8, 7, 5), (2, 1, 0), (1, 2, 2), (2, 2, 1), False, layout="left"),
    _case((3, 8, 7, 5), (1, 2, 3), (1, 1, 2, 2), (1, 2, 2, 1), True),
]
CASES3 = [
    _case((8, 7, 6), (0, 1, 2), (1, 1, 3), (3, 1, 1), True),
]


def _plan(case, **kw):
    keys = ("in_extents", "out_extents", "axes", "in_topology", "out_topology", "real_input", "norm", "layout")
    return dfft.Plan(**{k: case[k] for k in keys}, analyze_only=True, **kw)


@pytest.mark.parametrize("case", CASES2 + CASES3 + CASES4)
def test_rank_exchange_schedule(case):
    full = _plan(case)
    P = full.nprocs
    info = plan_info(full, case["norm"])
    blocks = info["blocks"][0]
    trans = [i for i, b in enumerate(blocks) if b["block_type"] == "Transpose"]
    for d, order in ((dfft.Direction.forward, trans), (dfft.Direction.backward, trans[::-1])):
        for r in range(P):
            rp = _plan(case, process_rank=r)
            xs = exchange_schedule(rp, d)
            assert [x.block for x in xs] == order
            for k, x in enumerate(xs):
                b = rp.block_infos(r)[x.block]
                assert x.elements == int(np.prod(b["buffer_extents"]))
                pc = b["buffer_extents"][0] if case["layout"] == "right" else b["buffer_extents"][-1]
                assert x.group_size == pc
                groups = O.exchange_groups(case["in_topology"], P, b["comm_axis"], info["pencil"])
                assert (x.sub_rank, list(x.members)) == (groups[r][0], groups[r][1])
                for q in range(P):
                    assert exchange_group(rp, d, k, q) == (groups[q][0], tuple(groups[q][1]))


def test_rank_plan_errors():
    case = CASES4[0]
    with pytest.raises(dfft.DistributedFFTError):
        _plan(case, process_rank=4)  # rank >= topology size
    rp = _plan(case, process_rank=1)
    with pytest.raises(dfft.DistributedFFTError):
        dfft.execute(rp, 0, 0, dfft.Direction.forward)  # per-rank plans run segment by segment
    from dfft.distributed import execute_segment
    with pytest.raises(dfft.DistributedFFTError):
        execute_segment(rp, dfft.Direction.forward, 0, 16, 32, 64, None)  # host-only plan
    full = _plan(case)
    with pytest.raises(dfft.DistributedFFTError):
        exchange_schedule(full, dfft.Direction.forward)  # not a per-rank plan


def _engine_run(case, forward, x):
    """All ranks of OracleRankEngine on the host with oracle.all2all."""
    full = _plan(case)
    P = full.nprocs
    info = plan_info(full, case["norm"])
    engines = [OracleRankEngine(full, r, case) for r in range(P)]
    src, dst = ("in", "out") if forward else ("out", "in")
    loc = [x[local_box(full, r, src)] for r in range(P)]
    sends_all = []
    recvs = [None] * P
    s = 0
    while True:
        res = [engines[r].segment(forward, s, loc[r] if s == 0 else None, recvs[r]) for r in range(P)]
        if res[0][0] == "out":
            out = np.zeros(case["out_extents"] if forward else case["in_extents"], dtype=res[0][1].dtype)
            for r in range(P):
                out[local_box(full, r, dst)] = res[r][1]
            return out, sends_all
        sends = [a for _, a in res]
        sends_all.append(sends)
        blocks = info["blocks"][0]
        trans = [i for i, b in enumerate(blocks) if b["block_type"] == "Transpose"]
        b = blocks[trans[s] if forward else trans[::-1][s]]
        groups = O.exchange_groups(case["in_topology"], P, b["comm_axis"], info["pencil"])
        recvs = O.all2all(sends, groups, case["layout"] == "right")
        s += 1


@pytest.mark.parametrize("case", CASES2 + CASES3 + CASES4)
def test_oracle_rank_engine_matches_literal_walk(case):
    full = _plan(case)
    x = case_input(case, 0)
    rec = {}
    ref = O.execute_literal(x, plan_info(full, case["norm"]), True, record=rec)
    y, sends = _engine_run(case, True, x)
    assert O.rel_l2(y, ref) <= 1e-12
    assert O.rel_l2(y, O.global_fft(x, case["axes"], case["real_input"], norm=case["norm"])) <= 1e-12
    # the send buffers of every exchange: the literal walk's, padding included
    for k, i in enumerate(sorted(rec)):
        for r, buf in enumerate(sends[k]):
            lit = rec[i]["send"][r]
            assert buf.shape == lit.shape
            assert np.abs(buf - lit).max() <= 1e-12 * max(1.0, np.abs(lit).max())
            assert np.all(buf[lit == 0] == 0)  # zero padding (random data is never exactly 0)
    xb, _ = _engine_run(case, False, y)
    assert O.rel_l2(xb, O.global_ifft(y, case["axes"], case["real_input"], case["in_extents"],
                                      norm=case["norm"])) <= 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_processes(world, cases, outdir, mode):
    import torch.multiprocessing as mp
    from _dist_worker import worker
    mp.start_processes(worker, args=(world, _free_port(), cases, str(outdir), mode), nprocs=world, join=True,
                       start_method="spawn")


def check_process_results(cases, outdir, world, tol, check_exchanged=False):
    for ci, case in enumerate(cases):
        full = _plan(case)
        res = [dict(np.load(os.path.join(outdir, f"case{ci}_rank{r}.npz"))) for r in range(world)]
        order = "C" if case["layout"] == "right" else "F"
        x = case_input(case, case["seed"])
        ref = O.global_fft(x, case["axes"], case["real_input"], norm=case["norm"])
        keys = ["y"] + (["y2"] if check_exchanged else [])
        for key in keys:
            y = np.zeros(case["out_extents"], dtype=np.complex128)
            for r in range(world):
                ext, _ = full.local_extents(r, "out")
                y[local_box(full, r, "out")] = res[r][key].reshape(ext, order=order)
            assert O.rel_l2(y, ref) <= tol, (ci, key, O.rel_l2(y, ref))
        for key in ["xb"] + (["xb2"] if check_exchanged else []):
            xb = np.zeros(case["in_extents"], dtype=res[0][key].dtype)
            for r in range(world):
                ext, _ = full.local_extents(r, "in")
                xb[local_box(full, r, "in")] = res[r][key].reshape(ext, order=order)
            assert O.rel_l2(xb, x) <= tol, (ci, key)
        # every recv buffer is the all-to-all permutation of the send buffers
        for fwd, d in (("f", dfft.Direction.forward), ("b", dfft.Direction.backward)):
            rps = [_plan(case, process_rank=r) for r in range(world)]
            xs = exchange_schedule(rps[0], d)
            for k, x0 in enumerate(xs):
                chunk = x0.nbytes // x0.group_size
                for r in range(world):
                    sub, members = exchange_group(rps[r], d, k, r)
                    recv = res[r][f"{fwd}_{k}_recv"]
                    for j, m in enumerate(members):
                        send = res[m][f"{fwd}_{k}_send"]
                        assert np.array_equal(recv[j * chunk:(j + 1) * chunk], send[sub * chunk:(sub + 1) * chunk])


@pytest.mark.parametrize("world,cases", [(2, CASES2), (4, CASES4)])
def test_distributed_plan_gloo(world, cases, tmp_path):
    run_processes(world, cases, tmp_path, "oracle")
    check_process_results(cases, tmp_path, world, 1e-12)
    # the send buffers the processes exchanged are the oracle walk's
    for ci, case in enumerate(cases):
        full = _plan(case)
        rec = {}
        O.execute_literal(case_input(case, case["seed"]), plan_info(full, case["norm"]), True, record=rec)
        for k, i in enumerate(sorted(rec)):
            for r in range(world):
                got = np.load(os.path.join(tmp_path, f"case{ci}_rank{r}.npz"))[f"f_{k}_send"]
                lit = rec[i]["send"][r]
                lit_bytes = np.ascontiguousarray(lit.ravel(order="C" if case["layout"] == "right" else "F"))
                g = got.view(lit_bytes.dtype)
                assert np.abs(g - lit_bytes).max() <= 1e-12 * max(1.0, np.abs(lit_bytes).max())
                assert np.all(g[lit_bytes == 0] == 0)
