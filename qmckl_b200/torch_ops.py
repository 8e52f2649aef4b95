"""PyTorch autograd face of MO VGL.

PyTorch is used here only as the autograd wrapper around the C ABI: the
forward pass is qmckl_b200_mo_vgl_device and the backward pass is the
hand-written adjoint qmckl_b200_mo_vgl_adjoint_device, which recomputes the
AOs and their derivatives instead of keeping anything of the forward pass.

    mo = mo_vgl(ctx, coord, nucl_coord, coefficient)      # [P][5][mo]
    loss = (W * mo).sum(); loss.backward()

coord        [3][P] float64 CUDA tensor (the device layout of the points)
nucl_coord   [nucl][3] float64 tensor (any device)
coefficient  [mo][ao] float64 tensor (any device; the qmckl_set_mo_basis_coefficient layout)

The context keeps its own copy of the nuclear coordinates and MO
coefficients (qmckl_set_nucleus_coord / qmckl_set_mo_basis_coefficient);
they are pushed into it whenever the tensors given differ from the last ones
pushed, forward and backward alike, so interleaved evaluations at other
geometries (finite differences, line searches) stay correct.
"""
import numpy as np
import torch

from . import qmckl as pq

# context -> (nucl tensor, its version, coefficient tensor, its version); the
# tensors are held so that their storage cannot be reused by another tensor
_pushed = {}


def _push(context, nucl_coord, coefficient):
    last = _pushed.get(context)
    if last is not None and last[0] is nucl_coord and last[1] == nucl_coord._version:
        same_nucl = True
    else:
        same_nucl = False
    if last is not None and last[2] is coefficient and last[3] == coefficient._version:
        same_coef = True
    else:
        same_coef = False
    if not same_nucl:
        pq.set_nucleus_coord(context, "N", nucl_coord.detach().to("cpu", torch.float64).contiguous().numpy().reshape(-1))
    if not same_coef:
        pq.set_mo_basis_coefficient(context, coefficient.detach().to("cpu", torch.float64).contiguous().numpy()
                                    .reshape(-1))
    _pushed[context] = (nucl_coord, nucl_coord._version, coefficient, coefficient._version)


def forget(context):
    """Drop the cached references of a context (call before qmckl_context_destroy)."""
    _pushed.pop(context, None)


class MoVgl(torch.autograd.Function):
    """mo_vgl[P][5][mo] of the points `coord` ([3][P], CUDA, float64)."""

    @staticmethod
    def forward(fctx, context, coord, nucl_coord, coefficient):
        if not coord.is_cuda or coord.dtype != torch.float64 or coord.dim() != 2 or coord.shape[0] != 3:
            raise ValueError("coord must be a [3][P] float64 CUDA tensor")
        _push(context, nucl_coord, coefficient)
        c = coord.detach().contiguous()
        P = c.shape[1]
        M = coefficient.shape[0]
        out = torch.empty((P, 5, M), dtype=torch.float64, device=c.device)
        pq.b200_set_stream(context, torch.cuda.current_stream(c.device).cuda_stream)
        pq.b200_mo_vgl_device(context, P, c.data_ptr(), out.data_ptr())
        fctx.context = context
        fctx.save_for_backward(c, nucl_coord, coefficient)
        return out

    @staticmethod
    def backward(fctx, grad):
        c, nucl_coord, coefficient = fctx.saved_tensors
        context = fctx.context
        _push(context, nucl_coord, coefficient)
        dev = c.device
        P = c.shape[1]
        w = grad.detach().to(dev, torch.float64).contiguous()
        need_r, need_n, need_c = fctx.needs_input_grad[1], fctx.needs_input_grad[2], fctx.needs_input_grad[3]
        g_coef = torch.empty(tuple(coefficient.shape), dtype=torch.float64, device=dev) if need_c else None
        g_nucl = torch.empty(tuple(nucl_coord.shape), dtype=torch.float64, device=dev) if need_n else None
        g_coord = torch.empty((3, P), dtype=torch.float64, device=dev) if need_r else None
        if need_r or need_n or need_c:
            pq.b200_set_stream(context, torch.cuda.current_stream(dev).cuda_stream)
            pq.b200_mo_vgl_adjoint_device(context, P, c.data_ptr(), w.data_ptr(),
                                          g_coef.data_ptr() if need_c else 0,
                                          g_nucl.data_ptr() if need_n else 0,
                                          g_coord.data_ptr() if need_r else 0)
        if g_nucl is not None:
            g_nucl = g_nucl.to(nucl_coord.device, nucl_coord.dtype)
        if g_coef is not None:
            g_coef = g_coef.to(coefficient.device, coefficient.dtype)
        return None, g_coord, g_nucl, g_coef


def mo_vgl(context, coord, nucl_coord, coefficient):
    """Differentiable MO VGL: [P][5][mo] (see the module docstring)."""
    return MoVgl.apply(context, coord, nucl_coord, coefficient)


def nucl_coord_tensor(sysd, device="cpu"):
    """[nucl][3] tensor of a system dict (whose nucl_coord is [3][nucl])."""
    return torch.tensor(np.ascontiguousarray(np.asarray(sysd["nucl_coord"]).T), dtype=torch.float64, device=device)
