"""GPU reverse mode (blaze_ens_adj_*) against the FP64 reverse sweep of the
restatement, which tests/test_adjoint_oracle.py pins to central finite
differences.

Case: two box systems (40 and 60 spheres) thrown at random velocities,
200 steps of dt = 1e-5 s, checkpoints every 64 steps (the backward
recomputes four segments).  The GPU's forward equals the FP32 restatement's
bit for bit, and its reverse sweep equals the FP32 restatement's reverse
sweep within 1e-4 (the summation order of the reverse differs).  Against the
FP64 reverse sweep the FP32 gradients differ by ~1e-3 to 3e-3 of the largest
component (1e-4 to 3e-3 relative for the law constants): the FP32 and FP64
trajectories separate over 200 steps of contacts; the FP32 restatement shows
the same differences, so they are precision, stated and bounded at 1e-2.
"""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import ensemble as E
from blaze import synth

pytestmark = pytest.mark.gpu

T = 200
SEG = 64


@pytest.fixture(scope="module")
def case():
    S, W, p, r = synth.box_ensemble([40, 60], seed=4, mus=[0.3, 0.6], restitutions=[0.5, 0.8],
                                    height_factor=4.0)
    rng = np.random.default_rng(0)
    v0 = rng.normal(scale=30.0, size=p.shape).astype(np.float32)
    wx = rng.normal(size=p.shape)
    wv = rng.normal(size=p.shape) * 1e-2
    return S, W, p, r, v0, wx, wv


@pytest.fixture(scope="module")
def gpu_grads(case):
    S, W, p, r, v0, wx, wv = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    ens.set_state(p, r, v0)
    adj = E.Adjoint(ens, T, SEG)
    assert adj.forward() == 0
    st = ens.state()
    gx, gv0, gw0, gc = adj.backward(wx[st["pid"]], wv[st["pid"]], None)
    adj.close()
    ens.close()
    return st, gx, gv0, gw0, gc


@pytest.fixture(scope="module", params=["f32", "f64"])
def oracle_grads(case, request):
    S, W, p, r, v0, wx, wv = case
    o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision=request.param)
    o.set_state(p, r, v0)
    assert o.adj_record(T) == 0
    st = o.state()
    dx0, dv0, dw0, th = o.adj_reverse(wx[st["pid"]], wv[st["pid"]], np.zeros(p.shape))
    return dx0, dv0, dw0, th, request.param


TOL = {"f32": 1e-4, "f64": 1e-2}


def test_forward_equals_fp32_restatement(case, gpu_grads):
    S, W, p, r, v0, wx, wv = case
    o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision="f32")
    o.set_state(p, r, v0)
    o.step(T)
    b = o.state()
    a = gpu_grads[0]
    np.testing.assert_array_equal(a["pos"].astype(np.float64), b["pos"])
    np.testing.assert_array_equal(a["pid"], b["pid"])


@pytest.mark.parametrize("k,name", [(0, "position"), (1, "velocity"), (2, "angular velocity")])
def test_initial_state_gradient(gpu_grads, oracle_grads, k, name):
    g = gpu_grads[1 + k].astype(np.float64)
    o = oracle_grads[k]
    scale = np.abs(o).max()
    assert scale > 0
    err = np.abs(g - o).max() / scale
    prec = oracle_grads[4]
    print("%s gradient vs %s reverse sweep: max error %.2e of the largest component"
          % (name, prec, err))
    assert err < TOL[prec]


def test_law_constant_gradient(gpu_grads, oracle_grads):
    g = gpu_grads[4]
    o = oracle_grads[3]
    rel = np.abs(g - o) / np.maximum(np.abs(o), 1e-30)
    prec = oracle_grads[4]
    print("law-constant gradients vs %s, relative error per (system, constant):\n" % prec, rel)
    assert np.all(rel < TOL[prec]), rel
