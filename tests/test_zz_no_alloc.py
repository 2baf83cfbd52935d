"""The no-allocation local 3D FFT entry point against the regular one.

dfft_execute_local_c2c_noalloc exists for callers that cannot call cudaMalloc
(their device memory is owned by another allocator, or they run in a
latency-critical loop where cudaMalloc / cudaFree may synchronise the device).
It keeps its intermediate array in a library-owned device array instead of
plan scratch.  This test calls it through the C ABI twice in a row with
different data and checks each result against dfft_execute on an equivalent
single-rank (SharedPlan) plan, with the tolerances of the other parity tests.
The file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

import dfft
from dfft._lib import lib

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 1e-6}


def _rel(a, b):
    import torch
    a = a.to(torch.complex128)
    b = b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_noalloc_matches_plan_two_calls(precision):
    import torch
    shape = (64, 32, 128)
    dt = torch.complex128 if precision == "float64" else torch.complex64
    prec = 0 if precision == "float64" else 1
    plan = dfft.Plan(shape, shape, (0, 1, 2), (1, 1, 1), (1, 1, 1), precision=precision)
    gen = torch.Generator(device="cuda").manual_seed(7)
    for call in range(2):
        x = torch.randn(shape, dtype=dt, device="cuda", generator=gen)
        for direction in (dfft.Direction.forward, dfft.Direction.backward):
            ref = torch.empty_like(x)
            got = torch.empty_like(x)
            dfft.execute(plan, x, ref, direction)
            st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(got.data_ptr()),
                                                    shape[0], shape[1], shape[2], prec, int(direction), 0, None)
            assert st == 0, lib.dfft_last_error_string().decode()
            torch.cuda.synchronize()
            assert _rel(got, ref) <= TOL[precision], (call, direction)
            # and against numpy directly
            xn = x.cpu().numpy().astype(np.complex128)
            exp = np.fft.fftn(xn) if direction == dfft.Direction.forward else np.fft.ifftn(xn)
            assert _rel(got, torch.from_numpy(exp).cuda()) <= TOL[precision]


_NORM = {0: "backward", 1: "forward", 2: "ortho", 3: None}


@pytest.mark.parametrize("precision", ["float64", "float32"])
@pytest.mark.parametrize("shape", [(16, 16, 16), (16, 16, 4096), (4096, 16, 16)])
@pytest.mark.parametrize("norm", [0, 1, 2, 3])
def test_noalloc_norms_extreme_lengths_side_stream(precision, shape, norm):
    """Every normalisation, the shortest and longest line lengths (4096 points
    take the two-line tile and, in FP64, more than 48 KB of shared memory),
    issued on a non-default stream; two calls in a row, each against numpy."""
    import torch
    dt = torch.complex128 if precision == "float64" else torch.complex64
    prec = 0 if precision == "float64" else 1
    side = torch.cuda.Stream()
    gen = torch.Generator(device="cuda").manual_seed(11 + norm)
    for call in range(2):
        x = torch.randn(shape, dtype=dt, device="cuda", generator=gen)
        got = torch.empty_like(x)
        side.wait_stream(torch.cuda.current_stream())
        for direction in (dfft.Direction.forward, dfft.Direction.backward):
            st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(got.data_ptr()),
                                                    shape[0], shape[1], shape[2], prec, int(direction), norm,
                                                    ctypes.c_void_p(side.cuda_stream))
            assert st == 0, lib.dfft_last_error_string().decode()
            side.synchronize()
            xn = x.cpu().numpy().astype(np.complex128)
            if norm == 3:  # no scaling in either direction
                exp = np.fft.fftn(xn) if direction == dfft.Direction.forward else np.fft.ifftn(xn) * xn.size
            else:
                f = np.fft.fftn if direction == dfft.Direction.forward else np.fft.ifftn
                exp = f(xn, norm=_NORM[norm])
            assert _rel(got, torch.from_numpy(exp).cuda()) <= TOL[precision], (call, direction, norm)


def test_noalloc_rejects_misaligned_pointers():
    import torch
    x = torch.zeros(16 ** 3 + 1, dtype=torch.complex128, device="cuda")
    y = torch.zeros(16 ** 3 + 1, dtype=torch.complex128, device="cuda")
    # 8 bytes into a complex128 array: fine for complex64, not for complex128
    st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr() + 8), ctypes.c_void_p(y.data_ptr()),
                                            16, 16, 16, 0, 0, 0, None)
    assert st == dfft.Status.INVALID_ARGUMENT
    assert "aligned" in lib.dfft_last_error_string().decode()
    st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr() + 4),
                                            16, 16, 16, 1, 0, 0, None)
    assert st == dfft.Status.INVALID_ARGUMENT
    torch.cuda.synchronize()


def test_noalloc_rejects_sizes_beyond_limit():
    import torch
    x = torch.zeros(16, dtype=torch.complex64, device="cuda")
    y = torch.zeros(16, dtype=torch.complex64, device="cuda")
    # 1024^2 x 16 complex128 = 256 MiB > 64 MiB scratch
    st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                            1024, 1024, 16, 0, 0, 0, None)
    assert st == dfft.Status.UNSUPPORTED
    assert "64 MiB" in lib.dfft_last_error_string().decode()
    st = lib.dfft_execute_local_c2c_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                            24, 32, 32, 0, 0, 0, None)
    assert st == dfft.Status.UNSUPPORTED
    assert "power of two" in lib.dfft_last_error_string().decode()
