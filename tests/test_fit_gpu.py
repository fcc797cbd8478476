"""Gradient-based fit through the differentiable extinction
(costuum_b200.autograd): 100 Adam steps recover (Re m, Im m, axis ratio) of
a spheroid from synthetic Q_ext(lambda) curves at 16 wavelengths seen from
two directions of a particle aligned with the z axis (the radius is known).
The target comes from the same forward model at the true parameters. (A
random-orientation curve alone does not tell an axis ratio d from roughly
1/d, so it would not pin d.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_adam_fit_recovers_parameters():
    import torch

    from costuum_b200.autograd import extinction

    lam = np.logspace(np.log10(0.6e-6), np.log10(3e-6), 16)
    r_ev = 0.3e-6
    th = [0.3, 1.2]
    truth = torch.tensor([1.6, 0.05, 1.4], dtype=torch.float64)

    def q_ext(x):
        rows = torch.stack([x[0].expand(16), x[1].expand(16),
                            torch.full((16,), r_ev, dtype=torch.float64),
                            x[2].expand(16)], dim=1)
        return extinction(rows, lam, th)[:, :, 0].reshape(-1)

    with torch.no_grad():
        target = q_ext(truth)
    x = torch.tensor([1.45, 0.02, 1.15], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([x], lr=0.01)
    losses = []
    for _ in range(100):
        opt.zero_grad()
        loss = torch.sum(((q_ext(x) - target) / target) ** 2)
        loss.backward()
        opt.step()
        with torch.no_grad():
            x[1].clamp_(min=1e-4)
        losses.append(float(loss.detach()))
    assert losses[-1] < 1e-3 * losses[0], (losses[0], losses[-1])
    assert np.allclose(x.detach().numpy(), truth.numpy(), rtol=0.05), x
