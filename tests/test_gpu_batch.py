"""Batched execution (one persistent launch per stage of many fields) and the
library-owned CUDA graph of one Navier-Stokes RK4 step of many fields.

The 16 fields of the uneven-batch configuration (edges drawn from {64, 96,
128, 192} with numpy's default_rng(2)) on pencils (2,2,1) -> (1,2,2): the
batch's outputs against each plan's own dfft_execute (rel-L2 <= 1e-12 FP64,
<= 1e-6 FP32) and against the FP64 oracle on the smallest field; one launch
per axis stage and value class per direction.  R2C plans of the
Navier-Stokes example, (3, n, n, n) -> (3, n, n, n/2+1), batch the same way.
The Navier-Stokes graph advances every field by one step as the per-field
dfft_ns_step does."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O

pytestmark = pytest.mark.gpu

EDGES = [int(e) for e in np.random.default_rng(2).choice([64, 96, 128, 192], size=16)]


def _rel(a, b):
    import torch
    return float(torch.linalg.vector_norm((a - b).to(torch.complex128)) /
                 torch.linalg.vector_norm(b.to(torch.complex128)))


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_batch_c2c_uneven_fields(precision):
    import torch
    cdt = torch.complex128 if precision == "float64" else torch.complex64
    tol = 1e-12 if precision == "float64" else 1e-6
    gen = torch.Generator(device="cuda").manual_seed(7)
    plans = [dfft.Plan((e,) * 3, (e,) * 3, (0, 1, 2), (2, 2, 1), (1, 2, 2), precision=precision) for e in EDGES]
    xs = [torch.randn(e ** 3, dtype=cdt, device="cuda", generator=gen) for e in EDGES]
    ys = [torch.empty_like(x) for x in xs]
    zs = [torch.empty_like(x) for x in xs]
    batch = dfft.Batch(plans)
    # one launch per axis stage and value class (powers of two; 3 * 2^k)
    classes = len(set(EDGES))  # one launch per line length and stage
    assert batch.launch_count(dfft.Direction.forward) == 3 * classes
    assert batch.launch_count(dfft.Direction.backward) == 3 * classes
    batch.execute(xs, ys, dfft.Direction.forward)
    batch.execute(ys, zs, dfft.Direction.backward)
    torch.cuda.synchronize()
    for p, x, y, z in zip(plans, xs, ys, zs):
        ref = torch.empty_like(x)
        dfft.execute(p, x, ref, dfft.Direction.forward)
        back = torch.empty_like(x)
        dfft.execute(p, ref, back, dfft.Direction.backward)
        torch.cuda.synchronize()
        assert _rel(y, ref) <= tol
        assert _rel(z, x) <= tol
        assert p.device_error() == 0
    # the smallest field against the FP64 oracle
    i = int(np.argmin(EDGES))
    p = plans[i]
    X = dfft.gather_blocks(p, ys[i].cpu().numpy(), "out")
    xg = dfft.gather_blocks(p, xs[i].cpu().numpy(), "in")
    assert O.rel_l2(X, O.global_fft(xg, (0, 1, 2), False)) <= tol


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_batch_r2c_navier_stokes_plans(precision):
    import torch
    rdt = torch.float64 if precision == "float64" else torch.float32
    cdt = torch.complex128 if precision == "float64" else torch.complex64
    tol = 1e-12 if precision == "float64" else 1e-6
    edges = [24, 32, 48, 64]
    plans = [dfft.Plan((3, e, e, e), (3, e, e, e // 2 + 1), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2),
                       real_input=True, precision=precision) for e in edges]
    gen = torch.Generator(device="cuda").manual_seed(8)
    xs = [torch.randn(p.buffer_elements("in"), dtype=rdt, device="cuda", generator=gen) for p in plans]
    ys = [torch.empty(p.buffer_elements("out"), dtype=cdt, device="cuda") for p in plans]
    zs = [torch.empty_like(x) for x in xs]
    batch = dfft.Batch(plans)
    batch.execute(xs, ys, dfft.Direction.forward)
    batch.execute(ys, zs, dfft.Direction.backward)
    torch.cuda.synchronize()
    for p, x, y, z in zip(plans, xs, ys, zs):
        ref = torch.empty_like(y)
        dfft.execute(p, x, ref, dfft.Direction.forward)
        torch.cuda.synchronize()
        assert _rel(y, ref) <= tol
        assert _rel(z.to(torch.complex128), x.to(torch.complex128)) <= tol


def test_batch_rejects_bad_sets():
    a = dfft.Plan((16, 16, 16), (16, 16, 16), (0, 1, 2), (2, 1, 1), (1, 2, 1))
    b = dfft.Plan((16, 16, 16), (16, 16, 16), (0, 1, 2), (2, 1, 1), (1, 2, 1), precision="float32")
    c = dfft.Plan((16, 16, 16), (16, 16, 16), (0, 1, 2), (2, 1, 1), (1, 2, 1), exec_mode="literal")
    for plans in ([a, a], [a, b], [c]):
        with pytest.raises(dfft.DistributedFFTError):
            dfft.Batch(plans)


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_navier_stokes_step_graph(precision, batched):
    import torch
    cdt = torch.complex128 if precision == "float64" else torch.complex64
    tol = 1e-12 if precision == "float64" else 1e-5
    edges = [24, 32, 48, 32]
    states, uks, refs = [], [], []
    for e in edges:
        p = dfft.Plan((3, e, e, e), (3, e, e, e // 2 + 1), (1, 2, 3), (1, 2, 2, 1), (1, 1, 2, 2), real_input=True,
                      precision=precision)
        s = dfft.NavierStokes(p, nu=0.01, dt=0.01, lx=2.0)
        uk = torch.empty(p.buffer_elements("out"), dtype=cdt, device="cuda")
        s.init_taylor_green(uk)
        states.append(s)
        uks.append(uk)
        # per-field reference: its own state object on a copy
        s2 = dfft.NavierStokes(p, nu=0.01, dt=0.01, lx=2.0)
        refs.append((s2, uk.clone()))
    g = dfft.step_graph(states, uks, batched=batched)
    for _ in range(3):
        g.launch()
        for s2, r in refs:
            s2.step(r)
    torch.cuda.synchronize()
    for uk, (s2, r) in zip(uks, refs):
        assert _rel(uk, r) <= tol
    del g
