"""Line lengths outside the register and single-stage kernels: a prime
factor above 13 (the chirp-z stage) and lines too long for one stage's
shared memory (the four-step stage: FP64 8192, FP32 16384, and a chirp-z
line whose own FFTs need the four-step stage).  C2C and R2C / C2R, slab and
pencil, fused and literal programs, all four normalisations, and the adjoint
identity, against the FP64 oracle (pocketfft handles any length).
Tolerances as everywhere: FP64 rel-L2 <= 1e-12, FP32 <= 1e-6."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _gpu_util import out_extents, random_input, run

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 1e-6}


def _roundtrip(gin, axes, tin, tout, real, precision, exec_mode="fused", norm="backward", seed=0):
    gout = out_extents(gin, axes, real)
    plan = dfft.Plan(gin, gout, axes, tin, tout, real_input=real, precision=precision, exec_mode=exec_mode,
                     norm=norm)
    x = random_input(gin, real, seed, precision)
    X = run(plan, x, True)
    ref = O.global_fft(x, axes, real, norm=norm)
    assert O.rel_l2(X, ref) <= TOL[precision], (gin, axes, tin, tout, real, precision)
    xb = run(plan, ref, False)
    assert O.rel_l2(xb, O.global_ifft(ref, axes, real, gin, norm=norm)) <= TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("real", [False, True])
@pytest.mark.parametrize("gin,tin,tout", [
    ((17, 19, 23), (2, 1, 1), (1, 2, 1)),
    ((17, 19, 23), (2, 2, 1), (1, 2, 2)),
    ((34, 119, 16), (1, 2, 1), (2, 1, 1)),     # 119 = 7 * 17, 34 = 2 * 17
    ((1009, 6, 8), (1, 2, 1), (1, 1, 2)),      # a long prime line
])
def test_prime_lengths(gin, tin, tout, real, precision):
    _roundtrip(gin, (0, 1, 2), tin, tout, real, precision)


@pytest.mark.parametrize("exec_mode", ["fused", "literal"])
@pytest.mark.parametrize("norm", ["backward", "forward", "ortho", "none"])
def test_prime_lengths_modes(exec_mode, norm):
    _roundtrip((17, 19, 10), (0, 2, 1), (1, 1, 2), (1, 2, 1), True, "float64", exec_mode=exec_mode, norm=norm)


def test_prime_length_adjoint_identity():
    import torch
    gin, axes = (17, 12, 19), (0, 1, 2)
    gout = out_extents(gin, axes, True)
    plan = dfft.Plan(gin, gout, axes, (2, 1, 1), (1, 2, 1), real_input=True)
    x = torch.from_numpy(dfft.scatter_blocks(plan, random_input(gin, True, 1), "in")).cuda()
    y = torch.from_numpy(dfft.scatter_blocks(plan, random_input(gout, False, 2), "out")).cuda()
    fx = torch.empty(plan.buffer_elements("out"), dtype=torch.complex128, device="cuda")
    fhy = torch.empty_like(x)
    dfft.execute(plan, x, fx, dfft.Direction.forward)
    dfft.execute_adjoint(plan, y, fhy, dfft.Direction.forward)
    torch.cuda.synchronize()
    lhs = float((fx.conj() * y).real.sum())
    rhs = float((x * fhy).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("gin,tin,tout,real,precision", [
    ((8192, 4, 4), (1, 2, 1), (1, 1, 2), False, "float64"),
    ((8192, 4, 4), (1, 2, 2), (2, 2, 1), True, "float64"),
    ((4, 4, 8192), (2, 1, 1), (1, 2, 1), True, "float64"),     # the R2C axis itself
    ((16384, 2, 4), (1, 2, 1), (1, 1, 2), False, "float32"),
    ((4099, 3, 4), (1, 3, 1), (1, 1, 3), False, "float64"),   # prime: chirp-z with 8192-point four-step FFTs
])
def test_long_lines(gin, tin, tout, real, precision):
    _roundtrip(gin, (0, 1, 2), tin, tout, real, precision)
