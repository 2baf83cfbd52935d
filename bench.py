#!/usr/bin/env python
"""Benchmark of the distributed 3D FFT execute path on B200.

Workload (one step): forward + backward 512^3 C2C transform in complex64 on a
pencil topology (4,4,1) -> (1,4,4) of 16 virtual ranks, fused execution.
Every GPU (rank) runs its own field ("weak" scaling, no data-path collective:
the virtual ranks of a topology live on one GPU).

Reported:
  value      whole-job algorithmic HBM throughput in GB/s: per direction one
             read + one write of the field per axis stage (3 stages), i.e.
             12 * N * 8 bytes per step, over the device time of the step
  gflops     5 N log2 N flops per complex transform direction
  fp64_*     the plain FP64 path (same plan, complex128) and the time ratio
  e2e        the same metric through the C ABI with host buffers: pinned
             host -> device copy of the input, forward, backward, device ->
             host copy of the result, every step
  roofline   the FFT stage kernel (every launch of the step) against the
             measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (numpy restatement of the reference block walk)
             on a bounded 256^3 sample of the same pencil, all host threads,
             rank 0 only

``--impl reference`` times the CPU restatement of the reference's execute
path (the reference itself cannot be built here: Kokkos, kokkos-fft, FFTW and
MPI are absent) on the host with all available threads.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "distributed-fft-for-kokkos_b200"))

N_EDGE = 512
TOPO_IN, TOPO_OUT = (4, 4, 1), (1, 4, 4)
CPU_SAMPLE_EDGE = 256
REF_BUDGET_S = 150.0
WORKLOAD = (f"{N_EDGE}^3 C2C complex64 forward+backward, pencil {TOPO_IN}->{TOPO_OUT} "
            f"(16 virtual ranks on one GPU), fused")
METRIC = "3D FFT fwd+bwd algorithmic HBM throughput"


def algo_bytes(n, elem):
    # per direction: 3 axis stages x (read + write) of n^3 elements
    return 2 * 3 * 2 * n ** 3 * elem


def flops(n):
    N = n ** 3
    return 2 * 5 * N * math.log2(N)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def start_clock_sampler(device):
    fd, path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
    os.close(fd)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "100"], stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        p = None
    return p, path


def stop_clock_sampler(p, path):
    if p is not None:
        p.terminate()
        try:
            p.wait(timeout=5)
        except Exception:
            p.kill()
    sm, mx, reasons = [], None, set()
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
    finally:
        try:
            os.remove(path)
        except OSError:
            pass
    sm.sort()
    return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(steps=2, workers=None, n=CPU_SAMPLE_EDGE):
    """CPU oracle (numpy restatement of the reference's block walk: pocketfft
    local FFTs on `workers` threads, pack / all-to-all / unpack) on a bounded
    sample of the workload: the same pencil at n^3 (256^3 by default).  The
    block list comes from oracle/plans/ (precomputed planner output), so this
    leg loads no product code."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import dfft_oracle as O

    with open(os.path.join(ROOT, "oracle", "plans", f"c2c_{n}_pencil_441_144.json")) as f:
        info = json.load(f)["plan"]
    workers = workers or os.cpu_count() or 1
    rng = np.random.default_rng(1)
    x = (rng.standard_normal((n,) * 3) + 1j * rng.standard_normal((n,) * 3)).astype(np.complex64)
    t0 = time.perf_counter()
    for _ in range(steps):
        y = O.execute_literal(x, info, True, workers=workers)
        O.execute_literal(y, info, False, workers=workers)
    dt = (time.perf_counter() - t0) / steps
    return {
        "value": round(algo_bytes(n, 8) / dt / 1e9, 3), "unit": "GB/s", "cores": workers, "kind": "port",
        "cpu_model": cpu_model(), "ms_per_step": round(dt * 1e3, 1),
        "sample": f"{n}^3 C2C complex64 fwd+bwd on the same pencil {TOPO_IN}->{TOPO_OUT} (a bounded sample of the "
                  f"{N_EDGE}^3 workload, same GB/s metric), numpy restatement of the reference block walk (pocketfft "
                  f"local FFTs on {workers} threads, pack/all2all/unpack), {steps} steps"}


def workload_config(world):
    return {"workload": WORKLOAD, "n": N_EDGE, "topology_in": list(TOPO_IN), "topology_out": list(TOPO_OUT),
            "precision": "complex64", "exec_mode": "fused", "graph": True,
            "l2": "inputs (1 GiB per field) larger than the 126 MB L2",
            "parallelism": f"weak, one {N_EDGE}^3 field per GPU x {world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workers = os.cpu_count() or 1
    # the sample edge: 256^3, halved while the timed steps would take more
    # than REF_BUDGET_S of CPU time (the whole run stays within a few minutes)
    edge = CPU_SAMPLE_EDGE
    warm = cpu_baseline(steps=1, workers=workers, n=edge)  # warm-up (imports, allocator)
    while edge > 64 and warm["ms_per_step"] / 1e3 * max(1, args.steps) > REF_BUDGET_S:
        edge //= 2
        warm = cpu_baseline(steps=1, workers=workers, n=edge)
    res = []
    for _ in range(max(1, args.steps)):
        res.append(cpu_baseline(steps=1, workers=workers, n=edge))
    v = sorted(r["value"] for r in res)[len(res) // 2]
    cb = dict(res[0])
    cb["value"] = v
    cb["sample"] += f" (median of {len(res)} timed steps after 1 warm-up)"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.gpus),
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def large_single_field(args, stream, barrier, max_over_ranks, gen):
    """1024^3 FP32 C2C fwd+bwd, plain and with the compensated last radix pass,
    their rel-L2 against the FP64 path on the same inputs; 1024^3 FP64
    R2C / C2R fwd+bwd; Taylor-Green RK4 steps at 512^3 (FP32 and FP64), all
    on pencils of 8 x 8 virtual ranks (the reference's perf sweep reaches
    n = 1024)."""
    import torch

    import dfft

    n = 1024
    g = (n, n, n)
    steps = max(3, args.steps // 10)
    tin, tout = (8, 8, 1), (1, 8, 8)

    def time_pair(plan, a, b, c, k):
        for _ in range(args.warmup):
            dfft.execute(plan, a, b, dfft.Direction.forward)
            dfft.execute(plan, b, c, dfft.Direction.backward)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            dfft.execute(plan, a, b, dfft.Direction.forward)
            dfft.execute(plan, b, c, dfft.Direction.backward)
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / k)

    res = {"n": n, "topology_in": list(tin), "topology_out": list(tout), "timed_steps": steps}
    x = torch.randn(n ** 3, dtype=torch.complex64, device="cuda", generator=gen)
    outs = {}
    for prec in ("float32", "float32_compensated"):
        p = dfft.Plan(g, g, (0, 1, 2), tin, tout, precision=prec, stream=stream.cuda_stream)
        y = torch.empty_like(x)
        z = torch.empty_like(x)
        ms = time_pair(p, x, y, z, steps)
        dfft.execute(p, x, y, dfft.Direction.forward)
        key = "fp32" if prec == "float32" else "fp32_compensated"
        res[key + "_ms_per_fwd_bwd"] = round(ms, 4)
        res[key + "_GBps"] = round(algo_bytes(n, 8) / (ms * 1e-3) / 1e9, 1)
        outs[key] = y
        del p, z
        torch.cuda.empty_cache()
    peak, _ = measured_peak()
    res["fp32_frac_of_measured_hbm"] = round(res["fp32_GBps"] / peak, 4)
    p64 = dfft.Plan(g, g, (0, 1, 2), tin, tout, precision="float64", stream=stream.cuda_stream)
    y64 = torch.empty(n ** 3, dtype=torch.complex128, device="cuda")
    dfft.execute(p64, x.to(torch.complex128), y64, dfft.Direction.forward)
    torch.cuda.synchronize()
    nrm = torch.linalg.vector_norm(y64)
    for key, y in outs.items():
        res["rel_l2_" + key + "_vs_fp64"] = float(torch.linalg.vector_norm(y.to(torch.complex128) - y64) / nrm)
    del p64, y64, outs, x
    torch.cuda.empty_cache()
    # FP64 R2C / C2R
    pr = dfft.Plan(g, (n, n, n // 2 + 1), (0, 1, 2), tin, tout, real_input=True, precision="float64",
                   stream=stream.cuda_stream)
    xr = torch.randn(n ** 3, dtype=torch.float64, device="cuda", generator=gen)
    yr = torch.empty(pr.buffer_elements("out"), dtype=torch.complex128, device="cuda")
    zr = torch.empty_like(xr)
    ms = time_pair(pr, xr, yr, zr, max(3, steps // 2))
    res["fp64_r2c_c2r_ms_per_fwd_bwd"] = round(ms, 4)
    # per direction: the real field once, the half spectrum (n^2 (n/2+1)) five
    # times (R2C write, then read + write of the two C2C stages)
    res["fp64_r2c_c2r_GBps"] = round(2 * (n ** 3 * 8 + 5 * n * n * (n // 2 + 1) * 16) / (ms * 1e-3) / 1e9, 1)
    res["fp64_r2c_c2r_roundtrip_rel_l2"] = float(torch.linalg.vector_norm(zr - xr) / torch.linalg.vector_norm(xr))
    del pr, xr, yr, zr
    torch.cuda.empty_cache()
    # Taylor-Green at 512^3, Re 1600, dt 1e-3
    m = 512
    tg = {"n": m, "re": 1600, "dt": 1e-3, "topology_in": [1, 8, 8, 1], "topology_out": [1, 1, 8, 8]}
    energies = {}
    for prec in ("float32", "float64"):
        pl = dfft.Plan((3, m, m, m), (3, m, m, m // 2 + 1), (1, 2, 3), (1, 8, 8, 1), (1, 1, 8, 8), real_input=True,
                       precision=prec, stream=stream.cuda_stream)
        st = dfft.NavierStokes(pl, nu=1.0 / 1600.0, dt=1e-3, lx=2.0)
        uk = torch.empty(pl.buffer_elements("out"), dtype=torch.complex64 if prec == "float32" else torch.complex128,
                         device="cuda")
        st.init_taylor_green(uk, stream=stream.cuda_stream)
        e0 = st.energy(uk, stream=stream.cuda_stream)
        st.step(uk, stream=stream.cuda_stream)
        barrier()
        k = 4
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(k):
            st.step(uk, stream=stream.cuda_stream)
        t1.record(stream)
        barrier()
        tg[prec + "_ms_per_rk4_step"] = round(max_over_ranks(t0.elapsed_time(t1) / k), 3)
        energies[prec] = st.energy(uk, stream=stream.cuda_stream) / e0
        del st, pl, uk
        torch.cuda.empty_cache()
    tg["energy_ratio_after_5_steps_fp64"] = energies["float64"]
    tg["rel_diff_energy_fp32_vs_fp64"] = abs(energies["float32"] / energies["float64"] - 1.0)
    tg["fp32_over_fp64_speedup"] = round(tg["float64_ms_per_rk4_step"] / tg["float32_ms_per_rk4_step"], 3)
    res["taylor_green_512"] = tg
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="run only the FP32 warm-up and timed steps (for ncu captures); prints no bench line")
    ap.add_argument("--profile-ns", type=int, default=0, metavar="EDGE",
                    help="run only one FP32 Navier-Stokes RK4 step of a Taylor-Green field on EDGE^3 (for ncu "
                         "captures); prints no bench line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import numpy as np
    import torch

    import dfft

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = N_EDGE
    g = (n, n, n)
    stream = torch.cuda.current_stream()
    if args.profile_ns:
        e = args.profile_ns
        pl = dfft.Plan((3, e, e, e), (3, e, e, e // 2 + 1), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2), real_input=True,
                       precision="float32", stream=stream.cuda_stream)
        st = dfft.NavierStokes(pl, nu=1.0 / 1600.0, dt=1e-3, lx=2.0)
        uk = torch.empty(pl.buffer_elements("out"), dtype=torch.complex64, device="cuda")
        st.init_taylor_green(uk, stream=stream.cuda_stream)
        st.step(uk, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        print(f"profile run: Navier-Stokes {e}^3 energy {st.energy(uk, stream=stream.cuda_stream):.6f} "
              "(not a bench value)", flush=True)
        return

    def make(precision):
        return dfft.Plan(g, g, (0, 1, 2), TOPO_IN, TOPO_OUT, precision=precision, stream=stream.cuda_stream)

    def timed(plan, a, b, c, steps):
        for _ in range(args.warmup):
            dfft.execute(plan, a, b, dfft.Direction.forward)
            dfft.execute(plan, b, c, dfft.Direction.backward)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            dfft.execute(plan, a, b, dfft.Direction.forward)
            dfft.execute(plan, b, c, dfft.Direction.backward)
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    # ---- FP32 fused path (headline): fwd + bwd captured in one CUDA graph ----
    p32 = make("float32")
    a32 = torch.randn(n ** 3, dtype=torch.complex64, device="cuda", generator=gen)
    b32 = torch.empty_like(a32)
    c32 = torch.empty_like(a32)
    ms32_eager = max_over_ranks(timed(p32, a32, b32, c32, max(3, args.steps // 4)))
    graph = dfft.Graph([(p32, a32, b32, dfft.Direction.forward, 0), (p32, b32, c32, dfft.Direction.backward, 0)])

    def timed_graph(steps):
        for _ in range(args.warmup):
            graph.launch(stream.cuda_stream)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            graph.launch(stream.cuda_stream)
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    sampler = start_clock_sampler(local)
    ms32 = max_over_ranks(timed_graph(args.steps))
    clocks = stop_clock_sampler(*sampler)
    launches = p32.launch_count(dfft.Direction.forward) + p32.launch_count(dfft.Direction.backward)
    if args.profile:
        print(f"profile run: {ms32:.4f} ms per step (not a bench value)", flush=True)
        return

    # ---- plain FP64 path and the error of the FP32 result ----
    p64 = make("float64")
    a64 = a32.to(torch.complex128)
    b64 = torch.empty_like(a64)
    c64 = torch.empty_like(a64)
    ms64 = max_over_ranks(timed(p64, a64, b64, c64, max(3, args.steps // 2)))
    dfft.execute(p32, a32, b32, dfft.Direction.forward)
    dfft.execute(p64, a64, b64, dfft.Direction.forward)
    torch.cuda.synchronize()
    err_fwd = float(torch.linalg.vector_norm(b32.to(torch.complex128) - b64) / torch.linalg.vector_norm(b64))
    err_rt = float(torch.linalg.vector_norm(c32.to(torch.complex128) - a64) / torch.linalg.vector_norm(a64))
    del a64, b64, c64, p64
    torch.cuda.empty_cache()

    # ---- 16 uneven fields (edges from {64,96,128,192}, rng seed 2): FP32 graph
    # of all fields (concurrent branches) vs the plain FP64 per-field loop ----
    import numpy as np
    edges = np.random.default_rng(2).choice([64, 96, 128, 192], size=16)
    batch = {}
    for prec in ("float32", "float64"):
        dt = torch.complex64 if prec == "float32" else torch.complex128
        fields = []
        for e in edges:
            e = int(e)
            pl = dfft.Plan((e,) * 3, (e,) * 3, (0, 1, 2), (2, 2, 1), (1, 2, 2), precision=prec,
                           stream=stream.cuda_stream)
            x = torch.randn(e ** 3, dtype=dt, device="cuda", generator=gen)
            fields.append((pl, x, torch.empty_like(x), torch.empty_like(x)))
        batch[prec] = fields
    items = []
    for i, (pl, x, y, z) in enumerate(batch["float32"]):
        items += [(pl, x, y, dfft.Direction.forward, i), (pl, y, z, dfft.Direction.backward, i)]
    bsteps = max(3, args.steps // 10)

    def timed_launch(fn):
        for _ in range(args.warmup):
            fn()
        barrier()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(bsteps):
            fn()
        t1.record(stream)
        barrier()
        return max_over_ranks(t0.elapsed_time(t1) / bsteps)

    # per-field transforms on concurrent graph branches (dfft_graph_create)
    bgraph = dfft.Graph(items)
    ms_branch32 = timed_launch(lambda: bgraph.launch(stream.cuda_stream))
    # one persistent launch per stage of all 16 fields (dfft_batch_execute),
    # forward + backward captured in one CUDA graph
    fb = dfft.Batch([f[0] for f in batch["float32"]])
    xs, ys, zs = ([f[k] for f in batch["float32"]] for k in (1, 2, 3))
    fb.execute(xs, ys, dfft.Direction.forward, stream=stream.cuda_stream)
    fb.execute(ys, zs, dfft.Direction.backward, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    batch_graph = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream()
    cap.wait_stream(stream)
    with torch.cuda.graph(batch_graph, stream=cap):
        fb.execute(xs, ys, dfft.Direction.forward, stream=cap.cuda_stream)
        fb.execute(ys, zs, dfft.Direction.backward, stream=cap.cuda_stream)
    torch.cuda.synchronize()
    ms_batch32 = timed_launch(batch_graph.replay)
    batch_launches = fb.launch_count(dfft.Direction.forward) + fb.launch_count(dfft.Direction.backward)

    def loop64():
        for pl, x, y, z in batch["float64"]:
            dfft.execute(pl, x, y, dfft.Direction.forward)
            dfft.execute(pl, y, z, dfft.Direction.backward)
    ms_batch64 = timed_launch(loop64)
    batch_bytes = sum(algo_bytes(int(e), 8) for e in edges)
    del batch, bgraph, items, batch_graph, fb, xs, ys, zs
    torch.cuda.empty_cache()

    # ---- batched Navier-Stokes RK4 step (Taylor-Green, Re 1600, dt 1e-3) on
    # the same 16 uneven grids: FP32, all fields in one CUDA graph on 4
    # concurrent streams, vs the plain FP64 per-field loop ----
    ns_res = {}
    ns_fields = {}
    for prec in ("float32", "float64"):
        dt = torch.complex64 if prec == "float32" else torch.complex128
        fl = []
        for e in edges:
            e = int(e)
            pl = dfft.Plan((3, e, e, e), (3, e, e, e // 2 + 1), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2),
                           real_input=True, precision=prec, stream=stream.cuda_stream)
            st = dfft.NavierStokes(pl, nu=1.0 / 1600.0, dt=1e-3, lx=2.0)
            uk = torch.empty(pl.buffer_elements("out"), dtype=dt, device="cuda")
            st.init_taylor_green(uk, stream=stream.cuda_stream)
            fl.append((pl, st, uk))
        ns_fields[prec] = fl
    torch.cuda.synchronize()
    # one RK4 step of all 16 fields in a library-owned CUDA graph: every
    # transform of all fields batched into one launch per stage
    # (dfft_ns_graph_create)
    ns_steps = max(3, args.steps // 20)
    ms_ns = {}
    for batched in (True, False):
        ns_graph = dfft.step_graph([f[1] for f in ns_fields["float32"]], [f[2] for f in ns_fields["float32"]],
                                   batched=batched)
        for _ in range(args.warmup):
            ns_graph.launch(stream.cuda_stream)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ns_steps):
            ns_graph.launch(stream.cuda_stream)
        e1.record(stream)
        barrier()
        ms_ns[batched] = max_over_ranks(e0.elapsed_time(e1) / ns_steps)
    ms_ns32 = min(ms_ns.values())
    n32 = 2 * (args.warmup + ns_steps)  # RK4 steps the FP32 fields took

    def ns_loop64():
        for pl, st, uk in ns_fields["float64"]:
            st.step(uk, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        ns_loop64()
    barrier()
    e0.record(stream)
    for _ in range(ns_steps):
        ns_loop64()
    e1.record(stream)
    barrier()
    ms_ns64 = max_over_ranks(e0.elapsed_time(e1) / ns_steps)
    n64 = args.warmup + ns_steps
    for _ in range(n32 - n64):  # bring the FP64 fields to the same time as the FP32 fields
        ns_loop64()
    e_rel = max(abs(f32[1].energy(f32[2], stream=stream.cuda_stream) / f64[1].energy(f64[2], stream=stream.cuda_stream)
                    - 1.0) for f32, f64 in zip(ns_fields["float32"], ns_fields["float64"]))
    ns_res = {"edges": [int(e) for e in edges], "topology_in": [1, 2, 2, 1], "topology_out": [1, 1, 2, 2],
              "re": 1600, "dt": 1e-3, "rk4_steps_timed": ns_steps,
              "fp32_step_graph_ms_per_step": round(ms_ns32, 4),
              "fp32_batched_transforms_graph_ms": round(ms_ns[True], 4),
              "fp32_per_field_branches_graph_ms": round(ms_ns[False], 4),
              "fp64_loop_ms_per_step": round(ms_ns64, 4), "speedup": round(ms_ns64 / ms_ns32, 3),
              "transforms_per_step": 20 * len(edges),
              "max_rel_energy_diff_fp32_vs_fp64": e_rel, "sim_time": round(n32 * 1e-3, 4)}
    del ns_fields, ns_graph
    torch.cuda.empty_cache()

    # ---- end to end through the C ABI with host buffers ----
    # Every step copies its input from pinned host memory, runs forward +
    # backward (dfft_execute) and copies the result back.  Steps are
    # software-pipelined over two device buffer sets and three streams: the
    # host-to-device copy of step i+1 and the device-to-host copy of step i-1
    # run while step i transforms (the link carries both directions at once).
    h_in = a32.cpu().pin_memory()
    h_outs = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    dev_in = [a32, torch.empty_like(a32)]
    dev_out = [c32, torch.empty_like(c32)]
    s_h2d, s_d2h = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]       # input landed
    ev_fwd = [torch.cuda.Event() for _ in range(2)]      # input consumed by the forward transform
    ev_out = [torch.cuda.Event() for _ in range(2)]      # output written
    ev_read = [torch.cuda.Event() for _ in range(2)]     # output copied to the host
    for k in range(2):
        ev_fwd[k].record(stream)
        ev_read[k].record(stream)

    def e2e_step(i):
        k = i % 2
        s_h2d.wait_event(ev_fwd[k])
        with torch.cuda.stream(s_h2d):
            dev_in[k].copy_(h_in, non_blocking=True)
        ev_in[k].record(s_h2d)
        stream.wait_event(ev_in[k])
        dfft.execute(p32, dev_in[k], b32, dfft.Direction.forward)
        ev_fwd[k].record(stream)
        stream.wait_event(ev_read[k])
        dfft.execute(p32, b32, dev_out[k], dfft.Direction.backward)
        ev_out[k].record(stream)
        s_d2h.wait_event(ev_out[k])
        with torch.cuda.stream(s_d2h):
            h_outs[k].copy_(dev_out[k], non_blocking=True)
        ev_read[k].record(s_d2h)

    e2e_steps = max(3, args.steps // 2)
    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_h2d.wait_event(e0)
    s_d2h.wait_event(e0)
    for i in range(e2e_steps):
        e2e_step(i)
    stream.wait_event(ev_read[(e2e_steps - 1) % 2])
    stream.wait_event(ev_read[(e2e_steps - 2) % 2])
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / e2e_steps)

    # ---- large single field: 1024^3 FP32 C2C (plain and compensated last
    # pass) and 1024^3 FP64 R2C / C2R on a pencil of 8 x 8 virtual ranks, and
    # the Taylor-Green vortex at 512^3 (FP32 and FP64 RK4 steps) ----
    del a32, b32, c32, graph, p32, dev_in, dev_out
    torch.cuda.empty_cache()
    large = large_single_field(args, stream, barrier, max_over_ranks, gen)

    step_bytes = algo_bytes(n, 8)
    value = world * step_bytes / (ms32 * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    per_launch_bytes = step_bytes / launches
    launch_ms = ms32 / launches
    achieved = per_launch_bytes / (launch_ms * 1e-3) / 1e9
    traffic = None  # dram bytes per launch from the committed ncu capture of this workload
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            traffic = int(json.load(f)["fft_stage_kernels_512cubed_c64"]["traffic_per_launch_bytes"])
    except (OSError, KeyError, ValueError):
        pass

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms32, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (complex N(0,1), torch generator seed 1234+rank)",
            "config": workload_config(world),
            "gflops": round(world * flops(n) / (ms32 * 1e-3) / 1e9, 1),
            "execution": "CUDA graph of forward + backward (plan-time autotuned kernels)",
            "eager_ms_per_step": round(ms32_eager, 4),
            "batch16_uneven": {"edges": [int(e) for e in edges],
                               "fp32_batched_graph_ms": round(ms_batch32, 4),
                               "fp32_batched_launches_per_fwd_bwd": int(batch_launches),
                               "fp32_per_field_branch_graph_ms": round(ms_branch32, 4),
                               "fp64_loop_ms": round(ms_batch64, 4),
                               "speedup": round(ms_batch64 / ms_batch32, 3),
                               "fp32_batched_graph_GBps": round(batch_bytes / (ms_batch32 * 1e-3) / 1e9, 1),
                               "fp32_batched_frac_of_measured_hbm": round(
                                   batch_bytes / (ms_batch32 * 1e-3) / 1e9 / measured_peak()[0], 4)},
            "navier_stokes_batch16": ns_res,
            "large_single_field": large,
            "fp64_ms_per_step": round(ms64, 4),
            "fp32_over_fp64_speedup": round(ms64 / ms32, 3),
            "rel_l2_fp32_vs_fp64_forward": err_fwd,
            "rel_l2_fp32_roundtrip": err_rt,
            "e2e": {"value": round(world * step_bytes / (ms_e2e * 1e-3) / 1e9, 2), "unit": "GB/s",
                    "ms_per_step": round(ms_e2e, 3), "h2d_bytes_per_step": int(h_in.numel() * 8),
                    "d2h_bytes_per_step": int(h_outs[0].numel() * 8),
                    "pipelining": "two device buffer sets; H2D of step i+1 and D2H of step i-1 overlap the "
                                  "transforms of step i (separate copy streams)"},
            "roofline": {"bound": "hbm", "kernel": "fft_pair_stream_kernel (a-fast z stages) + fft_pair_tma_kernel (TMA-fed b-fast y / x stages): every launch of the step, 3 axis stages per direction",
                         "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "algorithmic_bytes_per_launch": int(per_launch_bytes)},
            "clocks": clocks,
            "gpu_launches": int(launches * args.steps),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(steps=2, workers=os.cpu_count())
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
