"""Differentiable orientation-averaged extinction of a batch of spheroids.

``extinction(params, wavelength, thetas, coefficients)`` is a
torch.autograd.Function: params is an (n, 4) float64 tensor of
(Re m, Im m, r_ev, axis ratio) per grain; the result is an (n, ntheta, 3)
tensor of (Qext, Qextpol, Qextcpol) (equal to the reference's
(Qabs, Qabspol) when the scattering subtraction is off). The forward pass
runs the convergence loop on the GPU; the backward pass evaluates the
hand-written tangent kernels (dT = -(dRgQ + T dQ) Q^-1 with the forward LU
factors) at the converged orders and contracts them with the incoming
gradient. The converged order is piecewise constant in the parameters, so
the derivative is the one at fixed order.

PyTorch is used here only for the autograd plumbing; the arithmetic runs in
libtmx.so.
"""
import numpy as np
import torch

from .tmatrix import Context

_ctx = None


def _context():
    global _ctx
    if _ctx is None:
        _ctx = Context(0)
    return _ctx


class Extinction(torch.autograd.Function):

    @staticmethod
    def forward(ctx, params, wavelength, thetas, coefficients, schedule):
        p = params.detach().cpu().numpy().astype(np.float64)
        th = np.atleast_1d(np.asarray(thetas, np.float64))
        c = None if coefficients is None else np.asarray(coefficients, np.float64)
        tm = _context()
        res = tm.tmatrix_batch(p[:, 2], wavelength, p[:, 0] + 1j * p[:, 1], p[:, 3],
                               **schedule)
        q = tm.observables(th, c)
        ctx.state = (p, wavelength, th, c, res.nmax.copy(), res.ngauss.copy(),
                     tm.batch_id)
        return torch.as_tensor(q, dtype=params.dtype, device=params.device)

    @staticmethod
    def backward(ctx, grad):
        p, wavelength, th, c, nmax, ngauss, batch = ctx.state
        tm = _context()
        if tm.batch_id != batch:
            # another batch ran since the forward: its T-matrices and LU
            # factors are gone, so recompute the blocks at the forward's orders
            tm.tmatrix_batch_fixed(p[:, 2], wavelength, p[:, 0] + 1j * p[:, 1],
                                   p[:, 3], nmax, ngauss)
        # else the context still holds the forward's batch, whose block
        # rounds kept their LU factors: only the tangent kernels run
        _, dq = tm.gradients(th, c)
        g = grad.detach().cpu().numpy().astype(np.float64)
        # sum over angles and coefficients of grad * dq, per grain and
        # parameter (one batched matrix-vector product)
        n = g.shape[0]
        gp = np.matmul(g.reshape(n, 1, -1), dq.reshape(n, -1, dq.shape[-1]))[:, 0, :]
        return (torch.as_tensor(gp, dtype=grad.dtype, device=grad.device),
                None, None, None, None)


def extinction(params, wavelength, thetas, coefficients=None, min_order=10,
               max_order=100, gauss_legendre_factor=2, tolerance=1e-4):
    """Differentiable (Qext, Qextpol, Qextcpol) of grains given as rows
    (Re m, Im m, r_ev, axis ratio) of params."""
    schedule = dict(min_order=min_order, max_order=max_order,
                    gauss_legendre_factor=gauss_legendre_factor,
                    tolerance=tolerance)
    return Extinction.apply(params, wavelength, thetas, coefficients, schedule)
