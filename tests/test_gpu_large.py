"""Large single-field configuration on the GPU: 1024^3 FP32 C2C and 1024^3
FP64 R2C / C2R on a pencil of 8 x 8 virtual ranks, (8,8,1) -> (1,8,8) (the
reference's perf sweep reaches n = 1024, distributed/perf_test/PerfTest_FFT3D.cpp:71-74),
and the Taylor-Green vortex at 512^3 for 10 RK4 steps.

The 1024^3 FP64 oracle over the whole array does not fit a test's time, so
the FP64 results are checked exactly on whole output planes: plane k0 of the
transform is the 2D transform of sum_n0 exp(-2 pi i k0 n0 / 1024) x[n0]
(numpy, FP64).  The FP32 results are then compared with the GPU FP64 result
over the whole array.  Tolerances: FP64 rel-L2 <= 1e-12, FP32 <= 1e-6; the
compensated FP32 form must not be less accurate than the plain one.  Inputs:
complex N(0,1) / real N(0,1) from torch's CUDA generator with seed 4."""
import numpy as np
import pytest

import dfft

pytestmark = pytest.mark.gpu

N1K = 1024
TIN, TOUT = (8, 8, 1), (1, 8, 8)


def _rel(a, b):
    import torch
    num = torch.linalg.vector_norm((a - b).to(torch.complex128) if a.is_complex() else (a - b).double())
    return float(num / torch.linalg.vector_norm(b.to(torch.complex128) if b.is_complex() else b.double()))


def _plane(plan, flat, k0, n):
    """Global output plane [k0, :, :] of a (1,8,8) output buffer, as numpy."""
    import torch
    nz = plan.out_extents[2]
    out = torch.empty((n, nz), dtype=flat.dtype, device=flat.device)
    for r in range(plan.nprocs):
        ext, st = plan.local_extents(r, "out")
        off = plan.local_offset(r, "out")
        blk = flat[off:off + int(np.prod(ext))].view(*ext)
        out[st[1]:st[1] + ext[1], st[2]:st[2] + ext[2]] = blk[k0]
    return out.cpu().numpy()


def _oracle_plane(xh, k0, real):
    """FP64 plane k0 of fftn (or rfftn, last axis halved) of host array xh."""
    n = xh.shape[0]
    w = np.exp(-2j * np.pi * k0 * np.arange(n) / n)
    s = np.zeros(xh.shape[1:], dtype=np.complex128)
    for c in range(0, n, 64):
        s += np.tensordot(w[c:c + 64], xh[c:c + 64].astype(np.complex128), axes=(0, 0))
    f = np.fft.fft2(s)
    return f[:, : xh.shape[2] // 2 + 1] if real else f


def test_cfg5_1024cubed_c2c_fp32_and_compensated():
    import torch
    n = N1K
    g = (n, n, n)
    gen = torch.Generator(device="cuda").manual_seed(4)
    p64 = dfft.Plan(g, g, (0, 1, 2), TIN, TOUT, precision="float64")
    x32 = torch.randn(n ** 3, dtype=torch.complex64, device="cuda", generator=gen)  # in the (8,8,1) layout
    y64 = torch.empty(n ** 3, dtype=torch.complex128, device="cuda")
    dfft.execute(p64, x32.to(torch.complex128), y64, dfft.Direction.forward)
    torch.cuda.synchronize()
    # the FP64 result on two whole planes against the host oracle
    xg = np.empty(g, dtype=np.complex64)
    xf = x32.cpu().numpy()
    for r in range(p64.nprocs):
        ext, st = p64.local_extents(r, "in")
        off = p64.local_offset(r, "in")
        xg[st[0]:st[0] + ext[0], st[1]:st[1] + ext[1], st[2]:st[2] + ext[2]] = \
            xf[off:off + int(np.prod(ext))].reshape(ext)
    del xf
    for k0 in (0, 357):
        ref = _oracle_plane(xg, k0, False)
        got = _plane(p64, y64, k0, n)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12, k0
    del xg, p64
    torch.cuda.empty_cache()
    errs = {}
    for prec in ("float32", "float32_compensated"):
        p = dfft.Plan(g, g, (0, 1, 2), TIN, TOUT, precision=prec)
        y32 = torch.empty_like(x32)
        dfft.execute(p, x32, y32, dfft.Direction.forward)
        xb = torch.empty_like(x32)
        dfft.execute(p, y32, xb, dfft.Direction.backward)
        torch.cuda.synchronize()
        errs[prec] = (_rel(y32, y64), _rel(xb, x32))
        assert p.device_error() == 0
        del p, y32, xb
        torch.cuda.empty_cache()
    for prec, (ef, er) in errs.items():
        assert ef <= 1e-6 and er <= 1e-6, (prec, ef, er)
    assert errs["float32_compensated"][0] <= errs["float32"][0] * 1.02, errs


def test_cfg5_1024cubed_r2c_fp64():
    import torch
    n = N1K
    gin, gout = (n, n, n), (n, n, n // 2 + 1)
    gen = torch.Generator(device="cuda").manual_seed(4)
    p = dfft.Plan(gin, gout, (0, 1, 2), TIN, TOUT, real_input=True, precision="float64")
    x = torch.randn(n ** 3, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.empty(p.buffer_elements("out"), dtype=torch.complex128, device="cuda")
    dfft.execute(p, x, y, dfft.Direction.forward)
    xb = torch.empty_like(x)
    dfft.execute(p, y, xb, dfft.Direction.backward)
    torch.cuda.synchronize()
    assert _rel(xb, x) <= 1e-12
    xg = np.empty(gin, dtype=np.float64)
    xf = x.cpu().numpy()
    for r in range(p.nprocs):
        ext, st = p.local_extents(r, "in")
        off = p.local_offset(r, "in")
        xg[st[0]:st[0] + ext[0], st[1]:st[1] + ext[1], st[2]:st[2] + ext[2]] = \
            xf[off:off + int(np.prod(ext))].reshape(ext)
    del xf
    for k0 in (0, 511, 700):
        ref = _oracle_plane(xg, k0, True)
        got = _plane(p, y, k0, n)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12, k0


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_taylor_green_512cubed_10_steps(precision):
    """Energy budget of the vortex at Re 1600: E(t_{n+1}) - E(t_n) =
    -nu dt (Omega_n + Omega_{n+1}) (trapezoid rule of dE/dt = -2 nu Omega,
    Omega the enstrophy, both reduced in FP64); the field stays divergence
    free; E(t) / E(0) = exp(-6 nu t) to first order for t << 1."""
    import torch
    n, nu, dt = 512, 1.0 / 1600.0, 1e-3
    plan = dfft.Plan((3, n, n, n), (3, n, n, n // 2 + 1), (1, 2, 3), (1, 8, 8, 1), (1, 1, 8, 8), real_input=True,
                     precision=precision)
    ns = dfft.NavierStokes(plan, nu=nu, dt=dt, lx=2.0)
    cdt = torch.complex128 if precision == "float64" else torch.complex64
    uk = torch.empty(plan.buffer_elements("out"), dtype=cdt, device="cuda")
    ns.init_taylor_green(uk)
    d0 = ns.diagnostics(uk, num_bins=0)
    assert abs(d0["energy"] / np.pi ** 3 - 1.0) < (1e-12 if precision == "float64" else 1e-6)
    assert abs(d0["enstrophy"] / (3.0 * d0["energy"]) - 1.0) < (1e-12 if precision == "float64" else 1e-6)
    prev = d0
    resid = []
    for _ in range(10):
        ns.step(uk)
        d = ns.diagnostics(uk, num_bins=0)
        de = d["energy"] - prev["energy"]
        budget = -nu * dt * (prev["enstrophy"] + d["enstrophy"])
        resid.append(abs(de - budget) / abs(budget))
        assert d["divergence_l2"] <= (1e-12 if precision == "float64" else 1e-5) * np.sqrt(d["enstrophy"])
        prev = d
    # FP32: the fields' rounding (~3e-7 of E) is a tenth of one step's decay
    assert max(resid) <= (1e-4 if precision == "float64" else 0.25), resid
    ratio = prev["energy"] / d0["energy"]
    assert abs(ratio / np.exp(-6.0 * nu * 10 * dt) - 1.0) <= (1e-6 if precision == "float64" else 1e-5)
