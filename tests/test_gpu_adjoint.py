"""Adjoint kernels of the distributed transforms.

* <F x, y> = <x, F^H y> (real inner product) for forward and backward
  transforms, C2C and R2C, slab / pencil, ragged shapes;
* the torch.autograd.Function harness against torch.fft's own autograd;
* loss L(u) = sum |i k . u_hat|^2 (u_hat = R2C of u) on 128^3: adjoint
  gradient vs central finite differences (eps 1e-6 FP64, 1e-3 FP32) on 64
  random directions and vs an FP64 CPU reference gradient."""
import numpy as np
import pytest

import dfft
import dfft_oracle as O
from _gpu_util import out_extents, random_input

pytestmark = pytest.mark.gpu


def _inner(a, b):
    return float(np.real(np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())))


@pytest.mark.parametrize("gin,axes,tin,tout,real", [
    ((16, 12, 10), (0, 1, 2), (2, 1, 1), (1, 2, 1), True),
    ((16, 12, 10), (0, 1, 2), (2, 2, 1), (1, 2, 2), False),
    ((8, 7, 6), (0, 2, 1), (1, 1, 2), (1, 2, 1), True),
    ((8, 7, 5), (0, 1, 2), (1, 2, 3), (2, 3, 1), True),
    ((3, 16, 12, 10), (1, 2, 3), (1, 2, 1, 1), (1, 1, 2, 1), True),
    ((8, 7, 6), (2,), (2, 1, 1), (1, 2, 1), True),
])
@pytest.mark.parametrize("norm", ["backward", "ortho"])
def test_adjoint_inner_product_identity(gin, axes, tin, tout, real, norm):
    import torch
    gout = out_extents(gin, axes, real)
    plan = dfft.Plan(gin, gout, axes, tin, tout, real_input=real, norm=norm)
    x = random_input(gin, real, 1)
    y = random_input(gout, False, 2)
    xin = torch.from_numpy(dfft.scatter_blocks(plan, x, "in")).cuda()
    yin = torch.from_numpy(dfft.scatter_blocks(plan, y, "out")).cuda()
    Fx = torch.empty(plan.buffer_elements("out"), dtype=torch.complex128, device="cuda")
    FHy = torch.empty_like(xin)
    dfft.execute(plan, xin, Fx, dfft.Direction.forward)
    dfft.execute_adjoint(plan, yin, FHy, dfft.Direction.forward)
    torch.cuda.synchronize()
    lhs = _inner(Fx.cpu().numpy(), yin.cpu().numpy())
    rhs = _inner(xin.cpu().numpy(), FHy.cpu().numpy())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)
    # backward transform B: input layout <- output layout
    Bz = torch.empty_like(xin)
    BHx = torch.empty_like(Fx)
    dfft.execute(plan, yin, Bz, dfft.Direction.backward)
    dfft.execute_adjoint(plan, xin, BHx, dfft.Direction.backward)
    torch.cuda.synchronize()
    if real:
        # the C2R input space: imaginary parts of DC / Nyquist are ignored by
        # C2R, so compare on the Hermitian-consistent part produced by R2C
        ycons = torch.empty_like(Fx)
        dfft.execute(plan, Bz, ycons, dfft.Direction.forward)
        torch.cuda.synchronize()
        yv = ycons
        Bz2 = torch.empty_like(xin)
        dfft.execute(plan, yv, Bz2, dfft.Direction.backward)
        torch.cuda.synchronize()
        lhs = _inner(Bz2.cpu().numpy(), xin.cpu().numpy())
        rhs = _inner(yv.cpu().numpy(), BHx.cpu().numpy())
    else:
        lhs = _inner(Bz.cpu().numpy(), xin.cpu().numpy())
        rhs = _inner(yin.cpu().numpy(), BHx.cpu().numpy())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_autograd_matches_torch_fft():
    import torch
    from dfft.autograd import fft
    gin, axes = (16, 12, 10), (0, 1, 2)
    plan = dfft.Plan(gin, out_extents(gin, axes, True), axes, (2, 1, 1), (1, 2, 1), real_input=True)
    x = random_input(gin, True, 4)
    w = random_input(out_extents(gin, axes, True), False, 5)
    xin = torch.from_numpy(dfft.scatter_blocks(plan, x, "in")).cuda().requires_grad_(True)
    win = torch.from_numpy(dfft.scatter_blocks(plan, w, "out")).cuda()
    y = fft(xin, plan)
    loss = (y.abs() ** 2 * win.real).sum() + (y * win.conj()).real.sum()
    loss.backward()
    g_ours = dfft.gather_blocks(plan, xin.grad.cpu().numpy(), "in")
    xt = torch.from_numpy(x).requires_grad_(True)
    yt = torch.fft.rfftn(xt, dim=axes)
    wt = torch.from_numpy(w)
    lt = (yt.abs() ** 2 * wt.real).sum() + (yt * wt.conj()).real.sum()
    lt.backward()
    assert O.rel_l2(g_ours, xt.grad.numpy()) <= 1e-12


@pytest.mark.parametrize("precision,eps,tol", [("float64", 1e-6, 1e-7), ("float32", 1e-3, 1e-2)])
def test_cfg4_gradient_vs_finite_differences(precision, eps, tol):
    # L(u) = sum |i k . u_hat|^2, u_hat = R2C of u, 128^3, u ~ U[-1,1) seed 3
    import torch
    from dfft.autograd import fft
    n = 128
    gin, axes = (n, n, n), (0, 1, 2)
    gout = out_extents(gin, axes, True)
    plan = dfft.Plan(gin, gout, axes, (2, 2, 1), (1, 2, 2), real_input=True, precision=precision)
    rdt = torch.float64 if precision == "float64" else torch.float32
    u = random_input(gin, True, 3)
    k = np.fft.fftfreq(n) * n
    kz = np.fft.rfftfreq(n) * n
    ksum = k[:, None, None] + k[None, :, None] + kz[None, None, :]   # k . (1,1,1)
    kin = torch.from_numpy(dfft.scatter_blocks(plan, ksum.astype(np.complex128), "out")).cuda().real.to(rdt)

    def loss_of(ubuf):
        uh = fft(ubuf, plan)
        return ((kin * uh.abs()) ** 2).sum(dtype=torch.float64)

    ub = torch.from_numpy(dfft.scatter_blocks(plan, u, "in")).cuda().to(rdt).requires_grad_(True)
    L = loss_of(ub)
    L.backward()
    g = ub.grad.detach()
    # FP64 CPU reference gradient: dL/du = 2 * Re(R2C^H (k^2 uhat)) computed with torch.fft
    ut = torch.from_numpy(u).requires_grad_(True)
    Lt = ((torch.from_numpy(ksum) * torch.fft.rfftn(ut).abs()) ** 2).sum()
    Lt.backward()
    g_ref = dfft.gather_blocks(plan, g.double().cpu().numpy(), "in")
    assert O.rel_l2(g_ref, ut.grad.numpy()) <= (1e-12 if precision == "float64" else 1e-5)
    rng = np.random.default_rng(64)
    gnorm = float(g.double().norm())
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            d = rng.standard_normal(gin)
            d /= np.linalg.norm(d)
            db = torch.from_numpy(dfft.scatter_blocks(plan, d, "in")).cuda().to(rdt)
            lp = float(loss_of(ub.detach() + eps * db))
            lm = float(loss_of(ub.detach() - eps * db))
            fd = (lp - lm) / (2 * eps)
            an = float((g.double() * db.double()).sum())
            worst = max(worst, abs(fd - an) / gnorm)  # d has unit norm
    assert worst <= tol, worst
