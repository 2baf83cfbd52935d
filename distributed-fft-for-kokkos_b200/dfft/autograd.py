"""torch.autograd binding of the distributed transforms (test harness of the
adjoint kernels).

``fft(x, plan, direction)`` applies ``execute`` in the forward pass and the
plan's adjoint (``dfft_execute_adjoint``) in the backward pass, on the
concatenated per-rank buffers.  With PyTorch's convention for complex
gradients the gradient of a real loss with respect to a real R2C input is
Re(F^H g), which is exactly what the Hermitian-weighted adjoint computes.
"""
import torch

from .plan import Direction, execute, execute_adjoint

_COMPLEX = {"float64": torch.complex128, "float32": torch.complex64}
_REAL = {"float64": torch.float64, "float32": torch.float32}


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
