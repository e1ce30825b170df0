"""The calibration harness (blaze.calibrate.EnsembleRun, a
torch.autograd.Function over the GPU forward and reverse sweep): gradients of
the calibration loss -- bed height and side-wall normal-force profile against
targets from hidden parameters -- with respect to kn, restitution, mu,
mu_wall and the initial velocities, against the same loss differentiated
through the FP32 restatement's reverse sweep (same FP32 trajectory, so the
same force-profile bins), within 1e-3 relative.  The restatement's reverse
sweep itself is pinned to central finite differences in FP64
(tests/test_adjoint_oracle.py)."""
import numpy as np
import pytest
import torch

from bindings import EnsRestated
from blaze import calibrate as CAL
from blaze import ensemble as E

pytestmark = pytest.mark.gpu

T = 300
SEG = 100


@pytest.fixture(scope="module")
def setup():
    S, W, p, r = CAL.calibration_ensemble(nsys=2, n=300, base=2.5, seed=4)
    hidden = np.array([[8e4, 0.55, 0.45, 0.45]] * 2)
    guess = np.array([[1e5, 0.5, 0.4, 0.4], [1.2e5, 0.6, 0.3, 0.5]])
    run = CAL.Runner(S, W, p, r, T, SEG)
    v0 = torch.tensor(CAL.initial_velocity(run.ens.n).astype(np.float32).astype(np.float64))
    with torch.no_grad():
        hp = torch.tensor(hidden)
        pos, vel = CAL.EnsembleRun.apply(hp, v0, run)
        target = CAL.observables(pos, vel, hp, S, r)
    return S, W, p, r, guess, run, target, v0


def test_autograd_matches_restatement(setup):
    S, W, p, r, guess, run, target, vinit = setup
    params = torch.tensor(guess, requires_grad=True)
    v0 = vinit.clone().requires_grad_(True)
    pos, vel = CAL.EnsembleRun.apply(params, v0, run)
    loss = CAL.loss_fn(pos, vel, params, S, r, target)
    loss.backward()
    g_params = params.grad.numpy().copy()
    g_v0 = v0.grad.numpy().copy()
    assert np.all(np.isfinite(g_params)) and np.any(g_params != 0)

    # the same loss through the FP32 restatement
    Sg = CAL.with_params(S, guess)
    o = EnsRestated(Sg, W, E.LAW_LINEAR, 1e-5, 0.02, 32, precision="f32")
    o.set_state(p, r, vinit.numpy())
    assert o.adj_record(T) == 0
    st = o.state()
    order = np.argsort(st["pid"])
    np.testing.assert_array_equal(st["pos"][order], pos.detach().numpy())
    pos_o = torch.tensor(st["pos"][order], requires_grad=True)
    vel_o = torch.tensor(st["vel"][order], requires_grad=True)
    params_o = torch.tensor(guess, requires_grad=True)
    lo = CAL.loss_fn(pos_o, vel_o, params_o, Sg, r, target)
    lo.backward()
    gx = pos_o.grad.numpy()[st["pid"]]
    gv = vel_o.grad.numpy()[st["pid"]]
    _, gv0_o, _, gc = o.adj_reverse(gx, gv, np.zeros(gx.shape))
    gu = E.user_param_grads(gc, Sg)[:, [0, 2, 3, 4]] + params_o.grad.numpy()
    rel = np.abs(g_params - gu) / np.maximum(np.abs(gu), 1e-30)
    print("parameter gradients (kn, e, mu, mu_wall):\n", g_params, "\nrelative error:\n", rel)
    assert np.all(rel < 1e-3), rel
    scale = np.abs(gv0_o).max()
    assert np.abs(g_v0 - gv0_o).max() < 1e-3 * scale
