"""TMA-fed b-fast stages (fft_tma.cu) against the FP64 oracle.

With DFFT_AUTOTUNE=0 every complex64 b-fast stage whose source layout a
tensor map can describe runs the TMA-fed kernel (the default variant), so
these cases exercise it on every supported line length, on plain
intermediate arrays (3D tensor maps) and on rank-blocked caller buffers
(5D tensor maps: block axes plus rank coordinates), including ragged last
tiles along b.  Tolerance: FP32 rel-L2 <= 1e-6 against the FP64 oracle on the
FP32-rounded inputs; the plan's device error word must stay 0."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _gpu_util import random_input, run

pytestmark = pytest.mark.gpu


def _check(gin, tin, tout, seed=0):
    plan = dfft.Plan(gin, gin, (0, 1, 2), tin, tout, precision="float32")
    x = random_input(gin, False, seed, "float32")
    X = run(plan, x, True)
    ref = O.global_fft(x, (0, 1, 2), False)
    assert O.rel_l2(X, ref) <= 1e-6, (gin, tin, tout)
    xb = run(plan, ref.astype(np.complex64), False)
    assert O.rel_l2(xb, O.global_ifft(ref.astype(np.complex64), (0, 1, 2), False, gin)) <= 1e-6, (gin, tin, tout)
    assert plan.device_error() == 0


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024])
def test_tma_stage_line_lengths(n, monkeypatch):
    monkeypatch.setenv("DFFT_AUTOTUNE", "0")
    # y and x stages are b-fast (z is the unit-stride axis); the backward x
    # stage reads the (1, 4, 4) output blocks through a 5D tensor map
    _check((n, 32, 64), (4, 4, 1), (1, 4, 4))
    _check((32, n, 128), (2, 2, 1), (1, 2, 2))
    # z extent not a multiple of the tile width: the last tile's box runs past
    # the array and is zero filled
    _check((n, 24, 40), (2, 1, 1), (1, 2, 1))


def test_tma_stage_autotuned_headline_shape():
    # the bench's pencil at 256^3 with the tuner free to choose
    _check((256, 256, 256), (4, 4, 1), (1, 4, 4), seed=1)


def test_tma_stage_layout_left(monkeypatch):
    monkeypatch.setenv("DFFT_AUTOTUNE", "0")
    gin = (64, 48, 128)
    plan = dfft.Plan(gin, gin, (0, 1, 2), (1, 2, 2), (2, 2, 1), precision="float32", layout="left")
    x = random_input(gin, False, 3, "float32")
    X = run(plan, x, True)
    assert O.rel_l2(X, O.global_fft(x, (0, 1, 2), False)) <= 1e-6
    assert plan.device_error() == 0


@pytest.mark.parametrize("gin,tin,tout", [
    ((256, 256, 256), (4, 4, 1), (1, 4, 4)),   # a-fast z stage + TMA-fed y / x stages
    ((64, 128, 512), (2, 2, 1), (1, 2, 2)),
    ((512, 16, 32), (2, 1, 1), (1, 2, 1)),
])
def test_compensated_fp32_last_pass(gin, tin, tout):
    """float32_compensated (last radix pass in hi + lo float pairs with exact
    twiddle products and two-sum additions) stays within the FP32 bound and is
    at least as accurate as the plain FP32 form on the same inputs."""
    x = random_input(gin, False, 5, "float32")
    ref = O.global_fft(x, (0, 1, 2), False)
    errs = {}
    for prec in ("float32", "float32_compensated"):
        plan = dfft.Plan(gin, gin, (0, 1, 2), tin, tout, precision=prec)
        X = run(plan, x, True)
        errs[prec] = O.rel_l2(X, ref)
        xb = run(plan, ref.astype(np.complex64), False)
        assert O.rel_l2(xb, O.global_ifft(ref.astype(np.complex64), (0, 1, 2), False, gin)) <= 1e-6
        assert plan.device_error() == 0
    assert errs["float32_compensated"] <= 1e-6
    assert errs["float32_compensated"] <= errs["float32"] * 1.02, errs
