"""torch.autograd binding of the distributed transforms (test harness of the
adjoint kernels).

``fft(x, plan, direction)`` applies ``execute`` in the forward pass and the
plan's adjoint (``dfft_execute_adjoint``) in the backward pass, on the
concatenated per-rank buffers.  With PyTorch's convention for complex
gradients the gradient of a real loss with respect to a real R2C input is
Re(F^H g), which is exactly what the Hermitian-weighted adjoint computes.

``navier_stokes(u0, ns, steps)`` runs the pseudo-spectral solver from a
physical field u0 (forward transform, ``steps`` RK4 steps, backward
transform) and back-propagates with the step adjoint
(``dfft_ns_step_adjoint``), which recomputes each step's stage states from the
step's input state; only those states are kept (one spectral buffer per
step).
"""
import torch

from .plan import Direction, execute, execute_adjoint

_COMPLEX = {"float64": torch.complex128, "float32": torch.complex64, "float32_compensated": torch.complex64}
_REAL = {"float64": torch.float64, "float32": torch.float32, "float32_compensated": torch.float32}


def _dtypes(plan):
    c = _COMPLEX[plan.precision]
    return (_REAL[plan.precision] if plan.real_input else c), c


class DistributedFFTFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan, direction):
        direction = Direction(direction)
        din, dout = _dtypes(plan)
        fwd = direction == Direction.forward
        out = torch.empty(plan.buffer_elements("out" if fwd else "in"), dtype=dout if fwd else din, device=x.device)
        execute(plan, x.contiguous(), out, direction, stream=torch.cuda.current_stream().cuda_stream)
        ctx.plan = plan
        ctx.direction = direction
        return out

    @staticmethod
    def backward(ctx, g):
        plan, direction = ctx.plan, ctx.direction
        din, dout = _dtypes(plan)
        fwd = direction == Direction.forward
        grad = torch.empty(plan.buffer_elements("in" if fwd else "out"), dtype=din if fwd else dout, device=g.device)
        execute_adjoint(plan, g.contiguous(), grad, direction, stream=torch.cuda.current_stream().cuda_stream)
        return grad, None, None


def fft(x, plan, direction=Direction.forward):
    return DistributedFFTFunction.apply(x, plan, direction)


class NavierStokesFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, ns, steps):
        plan = ns._plan
        din, dout = _dtypes(plan)
        stream = torch.cuda.current_stream().cuda_stream
        uk = torch.empty(plan.buffer_elements("out"), dtype=dout, device=u0.device)
        execute(plan, u0.contiguous(), uk, Direction.forward, stream=stream)
        states = []
        for _ in range(int(steps)):
            states.append(uk.clone())
            ns.step(uk, stream=stream)
        uT = torch.empty(plan.buffer_elements("in"), dtype=din, device=u0.device)
        execute(plan, uk, uT, Direction.backward, stream=stream)
        ctx.ns, ctx.states = ns, states
        return uT

    @staticmethod
    def backward(ctx, g):
        ns = ctx.ns
        plan = ns._plan
        din, dout = _dtypes(plan)
        stream = torch.cuda.current_stream().cuda_stream
        lam = torch.empty(plan.buffer_elements("out"), dtype=dout, device=g.device)
        execute_adjoint(plan, g.contiguous(), lam, Direction.backward, stream=stream)
        for uk in reversed(ctx.states):
            ns.step_adjoint(uk, lam, stream=stream)
        grad = torch.empty(plan.buffer_elements("in"), dtype=din, device=g.device)
        execute_adjoint(plan, lam, grad, Direction.forward, stream=stream)
        ctx.states = None
        return grad, None, None


def navier_stokes(u0, ns, steps):
    """u(T) after `steps` RK4 steps of the solver `ns` from the physical field u0."""
    return NavierStokesFunction.apply(u0, ns, steps)
