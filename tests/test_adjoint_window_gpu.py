"""Windowed reverse mode (blaze_ens_adj_backward_window) on the reduced
calibration workload over its full 3,000-step horizon: 4 systems x 2,000
spheres settling in 5 cm boxes (the calibration configuration at a tenth of
its particles per system), checkpoints every 100 steps, the last 50 steps
reversed, loss = mean height per system.

The GPU's forward equals the FP32 restatement's bit for bit over the 3,000
steps, and its windowed law-constant gradients equal the FP32 restatement's
windowed reverse sweep within 1e-4 (the reverse summation order differs);
tests/test_adjoint_oracle.py pins the windowed sweep to FP64 central finite
differences at the same horizon.  Every gradient is finite, where the full
3,000-step sweep overflows FP32 (the pathwise derivative of this chaotic
flow grows about 5 % per step)."""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import calibrate
from blaze import ensemble as E

pytestmark = pytest.mark.gpu

NSYS, N, T, SEG, WIN = 4, 2000, 3000, 100, 50


def test_windowed_gradients_at_full_horizon():
    S, W, p, r = calibrate.calibration_ensemble(nsys=NSYS, n=N, seed=4)
    v0 = calibrate.initial_velocity(len(p))
    gx_pid = np.zeros(p.shape)
    gx_pid[:, 2] = 1.0 / N        # d(sum over systems of the mean height) / dz

    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    ens.set_state(p, r, v0)
    adj = E.Adjoint(ens, T, SEG, tape_bytes=-1)
    assert adj.forward() == 0
    st = ens.state()
    _, _, _, gc = adj.backward(gx_pid[st["pid"]], None, None, window=WIN)
    adj.close()
    ens.close()
    assert np.isfinite(gc).all()

    o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision="f32")
    o.set_state(p, r, v0)
    assert o.step(T - WIN) == 0
    assert o.adj_record(WIN) == 0
    so = o.state()
    np.testing.assert_array_equal(st["pos"].astype(np.float64), so["pos"])
    np.testing.assert_array_equal(st["pid"], so["pid"])
    _, _, _, th = o.adj_reverse(gx_pid[so["pid"]], np.zeros(p.shape), np.zeros(p.shape))
    for k in (0, 1, 2, 3, 4):   # kn, kt, 2 beta, mu, mu_wall
        rel = np.abs(gc[:, k] - th[:, k]) / np.maximum(np.abs(th[:, k]), 1e-30)
        print("constant %d: windowed gradients %s, relative to the FP32 sweep %s"
              % (k, gc[:, k], rel))
        assert np.all(rel < 1e-4), (k, rel)
