"""Adjoints of the Navier-Stokes right-hand side and RK4 step, and the
gradient of L(u0) = 1/2 sum_x u(T)^2 after 10 steps (the second loss of the
differentiation configuration).

* <J d, c> = <d, J^T c> for the right-hand side and the step, J d from a
  central difference of the forward solver (FP64, eps 1e-6);
* the loss gradient against an FP64 CPU reference gradient: the oracle's
  right-hand side and RK4 (ns_oracle) restated with torch.fft on the CPU and
  differentiated by torch.autograd (32^3);
* the loss gradient on 128^3, u0 ~ U[-1, 1) seed 3, against central finite
  differences on 64 random unit directions (eps 1e-6 FP64, 1e-3 FP32).
Real inner product of the half spectrum: Re sum conj(a) b."""
import numpy as np
import pytest

import dfft
import ns_oracle as N
from _gpu_util import random_input

pytestmark = pytest.mark.gpu

NU, DT, LX = 1.0 / 1600.0, 1e-3, 2.0


def _setup(n, precision="float64", tin=(1, 2, 2, 1), tout=(1, 1, 2, 2)):
    plan = dfft.Plan((3, n, n, n), (3, n, n, n // 2 + 1), (1, 2, 3), tin, tout, real_input=True,
                     precision=precision)
    return plan, dfft.NavierStokes(plan, nu=NU, dt=DT, lx=LX)


def _inner(a, b):
    import torch
    if a.is_complex():
        return float((a.real.double() * b.real.double() + a.imag.double() * b.imag.double()).sum())
    return float((a.double() * b.double()).sum())


def _spectrum(plan, seed):
    import torch
    n = plan.in_extents[1]
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3, n, n, n))
    k, _, inv_ksq = N.wavenumbers(n, n, n, LX)
    y = N.projection(np.fft.rfftn(u, axes=(1, 2, 3)), k, inv_ksq) / n ** 1.5
    return torch.from_numpy(dfft.scatter_blocks(plan, y, "out")).cuda()


@pytest.mark.parametrize("shape_tin_tout", [
    (16, (1, 2, 2, 1), (1, 1, 2, 2)),
    (24, (1, 3, 2, 1), (1, 1, 3, 2)),
])
def test_rhs_and_step_adjoint_identity(shape_tin_tout):
    import torch
    n, tin, tout = shape_tin_tout
    plan, ns = _setup(n, "float64", tin, tout)
    y = _spectrum(plan, 1)
    c = _spectrum(plan, 2)
    d = _spectrum(plan, 3)
    eps = 1e-6

    def rhs(v):
        v = v.clone()
        out = torch.empty_like(v)
        ns.rhs(v, out)
        return out

    jd = (rhs(y + eps * d) - rhs(y - eps * d)) / (2 * eps)
    jtc = torch.empty_like(y)
    ns.rhs_adjoint(y, c, jtc)
    lhs, r = _inner(jd, c), _inner(d, jtc)
    assert abs(lhs - r) <= 1e-7 * max(abs(lhs), 1e-30), (lhs, r)

    def step(v):
        v = v.clone()
        ns.step(v)
        return v

    jd = (step(y + eps * d) - step(y - eps * d)) / (2 * eps)
    lam = c.clone()
    ns.step_adjoint(y, lam)
    lhs, r = _inner(jd, c), _inner(d, lam)
    assert abs(lhs - r) <= 1e-7 * max(abs(lhs), 1e-30), (lhs, r)


def _torch_cpu_loss_grad(u0, steps):
    """FP64 CPU reference: the oracle's solver in torch.fft, differentiated by
    torch.autograd; returns dL/du0 for L = 1/2 sum u(T)^2."""
    import torch
    n = u0.shape[1]
    shape = (n, n, n)
    k, ksq, inv_ksq = N.wavenumbers(n, n, n, LX)
    kt = [torch.from_numpy(np.broadcast_to(kk, (n, n, n // 2 + 1)).copy()) for kk in k]
    ksq_t, inv_t = torch.from_numpy(ksq), torch.from_numpy(inv_ksq)
    mask = torch.from_numpy(N.alias_mask(n, n, n))

    def proj(r):
        div = (kt[0] * r[0] + kt[1] * r[1] + kt[2] * r[2]) * inv_t
        return torch.stack([r[a] - kt[a] * div for a in range(3)])

    def rhs(y):
        yd = y * mask
        u = torch.fft.irfftn(yd, s=shape, dim=(1, 2, 3))
        du = [torch.fft.irfftn(1j * kt[a] * yd, s=shape, dim=(1, 2, 3)) for a in range(3)]
        adv = torch.stack([u[0] * du[0][j] + u[1] * du[1][j] + u[2] * du[2][j] for j in range(3)])
        advk = torch.fft.rfftn(adv, dim=(1, 2, 3)) * mask
        return yd, proj(-advk - NU * ksq_t * yd)

    ut = torch.from_numpy(u0).requires_grad_(True)
    y = torch.fft.rfftn(ut, dim=(1, 2, 3))
    for _ in range(steps):
        y0, f = rhs(y)
        k1 = f * DT
        _, f = rhs(y0 + k1 / 2)
        k2 = f * DT
        _, f = rhs(y0 + k2 / 2)
        k3 = f * DT
        _, f = rhs(y0 + k3)
        y = y0 + (k1 + 2 * k2 + 2 * k3 + f * DT) / 6
    uT = torch.fft.irfftn(y, s=shape, dim=(1, 2, 3))
    (0.5 * (uT ** 2).sum()).backward()
    return ut.grad.numpy()


def test_loss_gradient_vs_cpu_reference():
    import torch
    from dfft.autograd import navier_stokes
    n, steps = 32, 10
    plan, ns = _setup(n)
    u0 = random_input((3, n, n, n), True, 3)
    ub = torch.from_numpy(dfft.scatter_blocks(plan, u0, "in")).cuda().requires_grad_(True)
    uT = navier_stokes(ub, ns, steps)
    (0.5 * (uT ** 2).sum()).backward()
    g = dfft.gather_blocks(plan, ub.grad.cpu().numpy(), "in")
    g_ref = _torch_cpu_loss_grad(u0, steps)
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) <= 1e-10


@pytest.mark.parametrize("precision,eps,tol", [("float64", 1e-6, 1e-7), ("float32", 1e-3, 1e-2)])
def test_cfg4_loss2_gradient_vs_finite_differences(precision, eps, tol):
    import torch
    from dfft.autograd import navier_stokes
    n, steps = 128, 10
    plan, ns = _setup(n, precision)
    rdt = torch.float64 if precision == "float64" else torch.float32
    u0 = random_input((3, n, n, n), True, 3)
    ub = torch.from_numpy(dfft.scatter_blocks(plan, u0, "in")).cuda().to(rdt).requires_grad_(True)

    def loss_of(v):
        uT = navier_stokes(v, ns, steps)
        return 0.5 * (uT.double() ** 2).sum()

    L = loss_of(ub)
    L.backward()
    g = ub.grad.detach().double()
    gnorm = float(g.norm())
    rng = np.random.default_rng(64)
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            d = rng.standard_normal((3, n, n, n))
            d /= np.linalg.norm(d)
            db = torch.from_numpy(dfft.scatter_blocks(plan, d, "in")).cuda()
            lp = float(loss_of(ub.detach() + (eps * db).to(rdt)))
            lm = float(loss_of(ub.detach() - (eps * db).to(rdt)))
            fd = (lp - lm) / (2 * eps)
            an = float((g * db).sum())
            worst = max(worst, abs(fd - an) / gnorm)
    assert worst <= tol, worst
