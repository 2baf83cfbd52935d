"""GPU tests of the one-process-per-GPU path: per-rank plans
(dfft_plan_create_rank, dfft_execute_segment) and dfft.DistributedPlan.

* Every rank's program of a topology runs in ONE process on the GPU with the
  all-to-all of each exchange done by device copies between the ranks' send
  and recv buffers (emulate_ranks; no kernel waits on another rank): the
  gathered outputs against the FP64 oracle (rel-L2 <= 1e-12 FP64, <= 1e-6
  FP32 on the FP32-rounded inputs), the send buffers each rank's last stage
  wrote against the oracle's pack of the same rank (same tolerance, padding
  exactly zero), and the backward transform back to the input.
* Two processes (slab plans) and four processes (pencil plans: the row /
  column sub-communicators) sharing the GPU run DistributedPlan over gloo
  groups (buffers staged through host memory; no kernel waits on another
  process),
  through both the Python segment loop and the C driver with the exchange
  callback (dfft_execute_exchanged): outputs against the oracle, received
  buffers bit for bit the all-to-all permutation of the sent ones."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _dist_worker import case_input
from _rank_oracle import OracleRankEngine, emulate_ranks, local_box
from test_distributed import CASES2, CASES3, CASES4, _case, check_process_results, run_processes

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 1e-6}


def _rank_plans(case, precision):
    keys = ("in_extents", "out_extents", "axes", "in_topology", "out_topology", "real_input", "norm", "layout")
    kw = {k: case[k] for k in keys}
    full = dfft.Plan(**kw, precision=precision, analyze_only=True)
    return full, [dfft.Plan(**kw, precision=precision, process_rank=r) for r in range(full.nprocs)]


def _run(case, precision="float64", stages=None):
    """stages: expected launches per direction of every rank's program (the
    FFT stages alone: pack and unpack folded into their stores and loads)."""
    import torch
    full, plans = _rank_plans(case, precision)
    P = full.nprocs
    if stages is not None:
        for p in plans:
            assert p.launch_count(dfft.Direction.forward) == stages
            assert p.launch_count(dfft.Direction.backward) == stages
    order = "C" if case["layout"] == "right" else "F"
    x = case_input(case, case["seed"])
    rdt = np.float64 if precision == "float64" else np.float32
    cdt = np.complex128 if precision == "float64" else np.complex64
    tc = torch.complex128 if precision == "float64" else torch.complex64
    x = x.astype(rdt if case["real_input"] else cdt)
    ins = [torch.from_numpy(np.ascontiguousarray(x[local_box(full, r, "in")].ravel(order=order))).cuda()
           for r in range(P)]
    outs = [torch.zeros(int(np.prod(full.local_extents(r, "out")[0])), dtype=tc, device="cuda") for r in range(P)]
    rec = emulate_ranks(plans, ins, outs, dfft.Direction.forward)
    y = np.zeros(case["out_extents"], dtype=cdt)
    for r in range(P):
        y[local_box(full, r, "out")] = outs[r].cpu().numpy().reshape(full.local_extents(r, "out")[0], order=order)
    ref = O.global_fft(x, case["axes"], case["real_input"], norm=case["norm"])
    e = O.rel_l2(y, ref)
    assert e <= TOL[precision], (case, precision, e)
    # send buffers of the forward exchanges against the oracle's per-rank walk
    engines = [OracleRankEngine(full, r, case) for r in range(P)]
    loc = [x[local_box(full, r, "in")] for r in range(P)]
    recvs = [None] * P
    for k, (sends, recv_dev) in enumerate(rec):
        for r in range(P):
            kind, buf = engines[r].segment(True, k, loc[r] if k == 0 else None, recvs[r])
            assert kind == "send"
            want = np.ascontiguousarray(buf.ravel(order=order))
            cplx = np.iscomplexobj(want)
            got = sends[r].cpu().numpy().view(cdt if cplx else rdt)
            assert got.shape == want.shape
            assert np.abs(got - want).max() <= 10 * TOL[precision] * max(1.0, np.abs(want).max()), (k, r)
            assert np.all(got[want == 0] == 0), (k, r)  # padding stays zero
        # the oracle walk continues from the data the GPU ranks received
        recvs = [recv_dev[r].cpu().numpy().view(cdt if cplx else rdt).astype(np.complex128 if cplx else np.float64)
                 for r in range(P)]
    # backward from the oracle spectrum
    ins_b = [torch.from_numpy(np.ascontiguousarray(ref[local_box(full, r, "out")].astype(cdt).ravel(order=order)))
             .cuda() for r in range(P)]
    outs_b = [torch.zeros_like(ins[r]) for r in range(P)]
    emulate_ranks(plans, ins_b, outs_b, dfft.Direction.backward)
    xb = np.zeros(case["in_extents"], dtype=x.dtype)
    for r in range(P):
        xb[local_box(full, r, "in")] = outs_b[r].cpu().numpy().reshape(full.local_extents(r, "in")[0], order=order)
    want_b = O.global_ifft(ref.astype(cdt), case["axes"], case["real_input"], case["in_extents"], norm=case["norm"])
    eb = O.rel_l2(xb, want_b)
    assert eb <= TOL[precision], (case, precision, eb)
    for p in plans:
        assert p.device_error() == 0


@pytest.mark.parametrize("case", CASES2 + CASES3 + CASES4)
def test_rank_programs_small(case):
    _run(case, "float64")


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("case", [
    _case((64, 64, 64), (0, 1, 2), (2, 2, 1), (1, 2, 2), False),
    _case((64, 48, 40), (0, 1, 2), (1, 2, 2), (2, 2, 1), True),
    _case((96, 64, 128), (0, 1, 2), (1, 1, 4), (4, 1, 1), False),
    _case((3, 32, 24, 20), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2), True),
])
def test_rank_programs_medium(case, precision):
    _run(case, precision, stages=len(case["axes"]) if case["in_extents"] == (64, 64, 64) else None)


def test_rank_programs_256cubed_pencil_fp32():
    # the headline pencil at 256^3 on 16 per-rank programs: register / TMA
    # stages on the exchange buffers
    _run(_case((256, 256, 256), (0, 1, 2), (4, 4, 1), (1, 4, 4), False, seed=1), "float32", stages=3)


def test_distributed_plan_two_processes_on_one_gpu(tmp_path):
    cases = CASES2[:3] + [_case((32, 24, 20), (0, 1, 2), (2, 1, 1), (1, 2, 1), True)]
    run_processes(2, cases, tmp_path, "gpu")
    check_process_results(cases, tmp_path, 2, 1e-12, check_exchanged=True)


def test_distributed_plan_four_processes_pencil_on_one_gpu(tmp_path):
    # pencil topologies: row / column sub-communicators created by the plan,
    # the library's CUDA segments between the exchanges
    cases = [CASES4[0], CASES4[3], _case((32, 24, 20), (0, 1, 2), (2, 2, 1), (1, 2, 2), True)]
    run_processes(4, cases, tmp_path, "gpu")
    check_process_results(cases, tmp_path, 4, 1e-12, check_exchanged=True)
