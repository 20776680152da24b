"""Host-side pieces of the adjoint harness (milkywayathome_client_b200/adjoint.py), no GPU.

The reverse orbit (nbReverseOrbit, nbody/src/nbody_orbit_integrator.c:44-86) runs
nsteps = floor(tstop / dt) + 1 leapfrog steps of length tstop / nsteps.  The step count is a
whole number and is not differentiated, so the gradient of the start point with respect to the
forward time tstop flows only through the step length.  This isolates that one gradient
component: autograd's derivative must equal a central finite difference taken at the same
step count, and the harness must not touch the tensor's autograd graph to read the count.
"""
import warnings

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_reverse_orbit_forward_time_gradient_through_step_length():
    from milkywayathome_client_b200 import adjoint, nbody
    pot = nbody.milky_way_potential()
    pos = torch.tensor([-21.6, -10.4, 23.2], dtype=torch.float64)
    vel = torch.tensor([-156.0, 79.0, 107.0], dtype=torch.float64)
    dt = 1e-3
    t0 = 0.2505                               # floor(t / dt) + 1 = 251 steps for t near t0
    tstop = torch.tensor(t0, dtype=torch.float64, requires_grad=True)
    with warnings.catch_warnings():
        warnings.simplefilter("error")        # no scalar conversion of a tensor that needs grad
        x, v = adjoint.reverse_orbit(pot, pos, vel, tstop, dt)
    w = torch.tensor([0.3, -1.1, 0.7], dtype=torch.float64)
    loss = (x * w).sum() + (v * w).sum()
    (g,) = torch.autograd.grad(loss, tstop)

    def f(t):
        xx, vv = adjoint.reverse_orbit(pot, pos, vel, torch.tensor(t, dtype=torch.float64), dt)
        return float((xx * w).sum() + (vv * w).sum())

    h = 1e-7                                  # keeps the step count at 251 on both sides
    assert int(np.floor((t0 - h) / dt)) == int(np.floor((t0 + h) / dt)) == 250
    fd = (f(t0 + h) - f(t0 - h)) / (2.0 * h)
    assert abs(g.item() - fd) <= 1e-6 * max(1.0, abs(fd))
    assert g.item() != 0.0
